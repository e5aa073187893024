// Split-precision tensor-core form of the 256-point y-line transforms.
//
// The plain form runs every transform as shared-memory Stockham stages of
// FP32 radix-16 butterflies (fft.cuh).  Here the two radix-16 stages of a
// 256-point C2C transform become dense contractions on the 5th-generation
// tensor cores: a 16-point DFT of 16 complex inputs is a 32 x 32 real matrix
// acting on the inputs' (re, im) pairs, and one tile of 8 lines x 16
// butterflies is a 128 x 32 x 32 product -- exactly one tcgen05.mma of shape
// M = 128, N = 32 per 8-deep K slice, one row per thread of the 128-thread
// block, the accumulator rows in the 128 TMEM lanes.
//
// Precision: TF32 keeps 10 explicit mantissa bits, so each operand x is split
// into x_hi = tf32(x) and x_lo = x - x_hi (read by the MMA as TF32), and the
// product is
// A_lo B_hi + A_hi B_lo + A_hi B_hi (three products, FP32 accumulation in
// TMEM; the dropped A_lo B_lo term is ~2^-22 relative), the 3xTF32 scheme of
// Ootomo & Yokota (2022).  The DFT matrices are built in FP64 and split the
// same way (k_dft16_tables).
//
// Operands live in shared memory in the K-major, 128-byte-swizzled layout
// the MMA reads directly: a row of 32 TF32 values is one 128-byte line, the
// 16-byte chunk c of row m sits at chunk c ^ (m & 7), 8-row groups 1024 bytes
// apart; the K slice s of an MMA starts 32 s bytes into the line.  Stage 0's
// pretwiddled outputs are scattered straight into stage 1's operand rows (the
// Stockham exchange), which this swizzle makes free of bank conflicts.
//
// Replaces the transform work of the reference's cufftExecC2C calls
// (cuviscoelas_3D.cu:1272-1562) on the y axis; the multipliers, layout and
// results are those of k_cy in step_kernels.cu.
#include <cstdint>
#include <cstdio>

#include "engine.cuh"
#include "../../include/qvti.h"

namespace qvti {
namespace {

constexpr int kTcThreads = 128;  // 8 lines x 16 butterflies, one MMA row each
constexpr int kTcLines = 8;
constexpr int kTcN = 256;        // transform length of this form
constexpr uint32_t kTmemCols = 32;

// G index of each of the 21 fields of the x and y passes (all but the
// one-axis fields, is_gz / is_gy), the order k_cy's inverse pass uses.
struct GxyTable {
    int v[kNumGxy];
};
constexpr GxyTable make_gxy()
{
    GxyTable t{};
    int n = 0;
    for (int o = 0; o < kNumG; ++o)
        if (!is_gz(o) && !is_gy(o)) t.v[n++] = o;
    return t;
}
__constant__ GxyTable c_gxy_tc = make_gxy();

// ------------------------------------------------------------ PTX wrappers --
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ float tf32_round(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// K-major, 128-byte swizzle shared-memory matrix descriptor (tcgen05): start
// address >> 4 in bits 0-13, leading byte offset (unused by swizzled K-major
// layouts; 1) in 16-29, stride byte offset (1024 >> 4: next 8-row group) in
// 32-45, descriptor version 1 in 46-47, swizzle mode 2 (128B) in 61-63.
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr)
{
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Instruction descriptor, kind::tf32: D F32 (bits 4-5 = 1), A and B TF32
// (bits 7-9, 10-12 = 2), both K-major, N >> 3 in bits 17-22, M >> 4 in 24-28.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accum)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accum));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Test an mbarrier phase; a thread whose phase is not complete is suspended
// (issuing nothing) until it completes or ~0.1 ms pass.
__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2, %3;\n\t"
        "selp.b32 %0, 1, 0, P;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity), "r"(100000u)
        : "memory");
    return ok != 0;
}

// Wait for an mbarrier phase, at most `limit` SM clock cycles (default ~2 s
// at the B200's 1.97 GHz, for an MMA round); false on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, long long limit = 4000000000ll)
{
    const long long t0 = clock64();
    while (!mbar_try(mbar, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}

// 32 consecutive TMEM columns of this thread's lane (warp w reads lanes
// 32 (w % 4) .. + 31).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v)
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Float offset of (row m, 16-byte chunk c) in a swizzled 128-row operand.
__device__ __forceinline__ int sw_at(int m, int c) { return m * 32 + ((c ^ (m & 7)) << 2); }

// Write 16 complex values as row m of the hi and lo operands.
__device__ __forceinline__ void put_row(float* Ahi, float* Alo, int m, const float2* v)
{
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const float4 x = make_float4(v[2 * c].x, v[2 * c].y, v[2 * c + 1].x, v[2 * c + 1].y);
        const float4 h = make_float4(tf32_round(x.x), tf32_round(x.y), tf32_round(x.z), tf32_round(x.w));
        // the MMA reads the low part as TF32 (its last 13 bits ignored):
        // ~2^-21 of x, below the FP32 rounding of the sums
        const float4 l = make_float4(x.x - h.x, x.y - h.y, x.z - h.z, x.w - h.w);
        *reinterpret_cast<float4*>(Ahi + sw_at(m, c)) = h;
        *reinterpret_cast<float4*>(Alo + sw_at(m, c)) = l;
    }
}

// Stage 0 -> stage 1 exchange: the pretwiddled output q of butterfly j of
// line p is element r = j of stage 1's butterfly q of that line.
__device__ __forceinline__ void scatter_rows(float* Ahi, float* Alo, int p, int j, const float2* y)
{
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int m = p * 16 + q;
        const int off = sw_at(m, j >> 1) + 2 * (j & 1);
        const float2 h = make_float2(tf32_round(y[q].x), tf32_round(y[q].y));
        const float2 l = make_float2(y[q].x - h.x, y[q].y - h.y);
        *reinterpret_cast<float2*>(Ahi + off) = h;
        *reinterpret_cast<float2*>(Alo + off) = l;
    }
}

// One MMA round: D = A_lo B_hi + A_hi B_lo + A_hi B_hi over K = 32 (4 slices
// of 8), issued by one thread, completion signalled on the mbarrier.
__device__ __forceinline__ void mma_round(uint32_t tmem, const float* Ahi, const float* Alo, const float* Bhi,
                                          const float* Blo, uint32_t mbar)
{
    const uint32_t ah = smem_u32(Ahi), al = smem_u32(Alo), bh = smem_u32(Bhi), bl = smem_u32(Blo);
    uint32_t acc = 0;
#pragma unroll
    for (int s = 0; s < 4; ++s) { mma_tf32(tmem, desc_sw128(al + 32 * s), desc_sw128(bh + 32 * s), acc); acc = 1; }
#pragma unroll
    for (int s = 0; s < 4; ++s) mma_tf32(tmem, desc_sw128(ah + 32 * s), desc_sw128(bl + 32 * s), 1);
#pragma unroll
    for (int s = 0; s < 4; ++s) mma_tf32(tmem, desc_sw128(ah + 32 * s), desc_sw128(bh + 32 * s), 1);
    mma_commit(mbar);
}

// Everything a round needs between writing its operands and reading its
// results.  Returns false if the MMA did not complete in time.
__device__ __forceinline__ bool run_round(uint32_t tmem, const float* Ahi, const float* Alo, const float* Bhi,
                                          const float* Blo, uint32_t mbar, uint32_t& phase, float* out32)
{
    fence_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (threadIdx.x == 0) mma_round(tmem, Ahi, Alo, Bhi, Blo, mbar);
    const bool ok = mbar_wait(mbar, phase);
    phase ^= 1u;
    tc_after_sync();
    if (__syncthreads_or(!ok)) return false;  // the same decision in every warp
    tmem_ld32(tmem + ((uint32_t)((threadIdx.x >> 5) & 3) << 21), out32);  // lane 32 (w % 4) in bits 16+
    return true;
}

// ---------------------------------------------------------------- kernels --
// C2C along y of 256-point lines, tiles of 8 lines, persistent over
// (field, tile) pairs.  Forward: H[c] -> Hy[c] (and, when Yv[c] is set, the
// y derivative with the identity dispersion operator, scaled by 1/(ny nz),
// into Yv[c], as k_cy does); inverse: G in place over the 21 fields of the
// x and y passes.  The next tile's inputs are loaded into registers before
// the current tile's MMA rounds, so their HBM latency overlaps the tensor-core
// work.
//
// Shared memory (from a 1024-byte aligned base): A hi, A lo (16 KB each);
// the DFT matrices (inverse hi/lo; forward hi/lo first when !INV); twiddles;
// the shift table (!INV); mbarrier and TMEM address slot.
template <bool INV>
constexpr size_t tc_smem()
{
    return 1024 + 2 * 16384 + (INV ? 2 : 4) * 4096 + (INV ? 1 : 2) * kTcN * 8 + 64;
}

template <bool INV>
__global__ void __launch_bounds__(kTcThreads, INV ? 5 : 4) k_cy_tc(KP k, int nfield, long long line0, long long line_end)
{
    extern __shared__ unsigned char tc_raw[];
    const uint32_t s0 = smem_u32(tc_raw);
    unsigned char* base = tc_raw + ((1024u - (s0 & 1023u)) & 1023u);  // 1024-byte aligned (swizzle atom)
    float* Ahi = reinterpret_cast<float*>(base);
    float* Alo = Ahi + 4096;
    float* Bf_hi = Alo + 4096;                  // forward matrices (not present when INV)
    float* Bi_hi = INV ? Bf_hi : Bf_hi + 2048;  // inverse hi, then lo
    float* Bi_lo = Bi_hi + 1024;
    float* Bf_lo = Bf_hi + 1024;
    float2* tw = reinterpret_cast<float2*>(Bi_lo + 1024);
    float2* tsh = tw + kTcN;  // only when !INV
    uint64_t* mbar_p = reinterpret_cast<uint64_t*>(tw + (INV ? 1 : 2) * kTcN);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar_p + 1);
    const uint32_t mbar = smem_u32(mbar_p);

    const int t = threadIdx.x, p = t >> 4, j = t & 15;
    if (t < 32) {  // warp 0 owns the TMEM allocation
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // dft16: [fwd hi | fwd lo | inv hi | inv lo]
    for (int i = t; i < (INV ? 2 : 4) * 1024; i += kTcThreads) Bf_hi[i] = k.dft16[(INV ? 2048 : 0) + i];
    for (int i = t; i < kTcN; i += kTcThreads) tw[i] = k.tw_y[i];
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *tslot;
    uint32_t phase = 0;
    bool ok = true;

    // tile counts fit 32 bits (at most 21 fields x (nz/2+1) nx / 8 tiles);
    // only the element offsets need 64
    const int nlines = (int)(line_end - line0);
    const int ntile = (nlines + kTcLines - 1) / kTcLines;
    const int total = ntile * nfield;
    const float inv_n = 1.0f / ((float)kTcN * (float)k.nz);
    const float* Bhi = INV ? Bi_hi : Bf_hi;
    const float* Blo = INV ? Bi_lo : Bf_lo;
    // tile w: field c, lines [first, first + lv)
    auto tile = [&](int w, int& c, long long& first, int& lv) {
        c = w / ntile;
        const int t = (w - c * ntile) * kTcLines;
        first = line0 + t;
        lv = min(kTcLines, nlines - t);
    };
    // stage 0 inputs of butterfly j of line p: x[j + 16 r]
    auto load = [&](int c, long long first, int lv, float2* v) {
        const float2* src = (INV ? k.G[c_gxy_tc.v[c]] : k.H[c]) + first * kTcN;
#pragma unroll
        for (int r = 0; r < 16; ++r) v[r] = p < lv ? src[(long long)p * kTcN + j + 16 * r] : make_float2(0.f, 0.f);
    };
    int c, lv, shift_c = -1;  // shift_c: field whose shift table is in tsh
    long long first;
    float2 v[16];
    int w = blockIdx.x;
    if (w < total) {
        tile(w, c, first, lv);
        load(c, first, lv, v);
    }
    for (; ok && w < total; w += gridDim.x) {
        const long long off = first * kTcN;
        float2* dst = (INV ? k.G[c_gxy_tc.v[c]] : k.Hy[c]) + off;
        float2* ydst = (!INV && k.Yv[c]) ? k.Yv[c] + off : nullptr;
        if (ydst && shift_c != c) {
            // all threads are past the previous tile's reads of tsh (the
            // barrier in its last round)
            const float2* T = c == 1 ? k.Fy : k.By;  // dy vy forward shift, dy vx / dy vz backward
            for (int i = t; i < kTcN; i += kTcThreads) tsh[i] = T[i];
            shift_c = c;  // made visible by the next round's barrier
        }
        put_row(Ahi, Alo, t, v);
        // the next tile's inputs, in flight during this tile's rounds
        const int c_cur = c, lv_cur = lv;
        const int wn = w + gridDim.x;
        if (wn < total) {
            tile(wn, c, first, lv);
            load(c, first, lv, v);
        }
        float d[32];
        if (!(ok = run_round(tmem, Ahi, Alo, Bhi, Blo, mbar, phase, d))) break;
        // twiddles w^(q j) of stage 1, then the exchange into stage 1's rows;
        // the round's completion means the MMA no longer reads A
        float2 y[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const float2 a = make_float2(d[2 * q], d[2 * q + 1]);
            const float2 wq = tw[q * j];
            y[q] = INV ? cmulc(a, wq) : cmul(a, wq);
        }
        scatter_rows(Ahi, Alo, p, j, y);
        if (!(ok = run_round(tmem, Ahi, Alo, Bhi, Blo, mbar, phase, d))) break;
        // thread (p, j) holds X[j + 16 q]
        if (p < lv_cur) {
#pragma unroll
            for (int q = 0; q < 16; ++q) dst[(long long)p * kTcN + j + 16 * q] = make_float2(d[2 * q], d[2 * q + 1]);
        }
        if (!INV && ydst) {
            // inverse transform of X T / (ny nz): stage 0 of butterfly j takes
            // exactly the X[j + 16 r] this thread holds
            float2 u[16];
#pragma unroll
            for (int q = 0; q < 16; ++q)
                u[q] = cmul(make_float2(d[2 * q], d[2 * q + 1]), cscale(tsh[j + 16 * q], inv_n));
            put_row(Ahi, Alo, t, u);
            if (!(ok = run_round(tmem, Ahi, Alo, Bi_hi, Bi_lo, mbar, phase, d))) break;
#pragma unroll
            for (int q = 0; q < 16; ++q) y[q] = cmulc(make_float2(d[2 * q], d[2 * q + 1]), tw[q * j]);
            scatter_rows(Ahi, Alo, p, j, y);
            if (!(ok = run_round(tmem, Ahi, Alo, Bi_hi, Bi_lo, mbar, phase, d))) break;
            if (p < lv_cur) {
#pragma unroll
                for (int q = 0; q < 16; ++q)
                    ydst[(long long)p * kTcN + j + 16 * q] = make_float2(d[2 * q], d[2 * q + 1]);
            }
        }
        (void)c_cur;
    }
    if (!ok && t == 0 && k.err) atomicExch(k.err, QVTI_ERR_TIMEOUT);
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (t < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// The timeout path of the bounded waits, exercised without a fault: one
// thread waits, at most `limit` cycles, on an mbarrier phase that nothing
// completes, then records QVTI_ERR_TIMEOUT in the engine's device error flag
// exactly as a stalled MMA round would.
__global__ void k_wait_probe(int* err, long long limit)
{
    __shared__ uint64_t bar;
    const uint32_t mbar = smem_u32(&bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (!mbar_wait(mbar, 0, limit) && err) atomicExch(err, QVTI_ERR_TIMEOUT);
}

// 16-point DFT matrices for the MMA's B operand (N = 32 outputs x K = 32
// inputs, both as interleaved re/im), FP64-built and split into TF32 hi and
// lo parts, stored in the swizzled K-major layout the kernel copies as is:
// [forward hi | forward lo | inverse hi | inverse lo], 1024 floats each.
// Output n = 2q + f (f = 0 real, 1 imaginary), input k = 2r + e:
//   forward  Re: a cos + b sin    Im: -a sin + b cos     (theta = 2 pi q r / 16)
//   inverse  Re: a cos - b sin    Im:  a sin + b cos
__global__ void k_dft16_tables(float* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * 1024) return;
    const int inv = i >> 10, e = i & 1023, n = e >> 5, kk = e & 31;
    const int q = n >> 1, f = n & 1, r = kk >> 1, ee = kk & 1;
    double s, c;
    sincospi(2.0 * ((q * r) & 15) / 16.0, &s, &c);
    double v;
    if (f == 0) v = ee == 0 ? c : (inv ? -s : s);
    else v = ee == 0 ? (inv ? s : -s) : c;
    const float hi = tf32_round((float)v);
    const float lo = tf32_round((float)(v - (double)hi));
    const int at = n * 32 + ((((kk >> 2) ^ (n & 7))) << 2) + (kk & 3);
    out[inv * 2048 + at] = hi;
    out[inv * 2048 + 1024 + at] = lo;
}

}  // namespace

bool tc_cy_available(const KP& k) { return k.ny == kTcN && k.dft16 != nullptr; }

size_t tc_cy_smem() { return tc_smem<false>(); }

int configure_tc_kernels()
{
    cudaError_t e = cudaFuncSetAttribute((const void*)k_cy_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)tc_smem<false>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute((const void*)k_cy_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tc_smem<true>());
    return (int)e;
}

void launch_dft16_tables(float* out, cudaStream_t st) { k_dft16_tables<<<16, 128, 0, st>>>(out); }

void launch_wait_probe(int* err, long long limit_cycles, cudaStream_t st)
{
    k_wait_probe<<<1, 1, 0, st>>>(err, limit_cycles);
}

void launch_cy_tc(const KP& k, bool inv, int nfield, long long line0, long long line_end, cudaStream_t st)
{
    const long long tiles = (line_end - line0 + kTcLines - 1) / kTcLines * nfield;
    long long grid = 148ll * (inv ? 5 : 4);  // resident blocks per SM (shared memory, registers)
    if (grid > tiles) grid = tiles;
    if (inv) k_cy_tc<true><<<(unsigned)grid, kTcThreads, tc_smem<true>(), st>>>(k, nfield, line0, line_end);
    else k_cy_tc<false><<<(unsigned)grid, kTcThreads, tc_smem<false>(), st>>>(k, nfield, line0, line_end);
}

}  // namespace qvti
