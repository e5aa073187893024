// Time-step kernels of the B200 viscoelastic pseudospectral engine.
//
// One time step of the reference (cuviscoelas_3D.cu:1255-1630: 29 launches,
// 63 cuFFT C2C transforms) becomes 11 launches here:
//
//   k_vy   y-pencils of the stresses: dy sxy, dy syy, dy syz (1D spectral
//          derivatives, C-PML memory terms in the y slab) added to R
//   k_vx   x-pencils: dx sxx, dx sxy, dx sxz, C-PML x terms, velocity update
//          (cuda_kernel_calculate_v, cu:1018-1101)
//   k_fz   z-pencils: R2C of vx, vy, vz (two real pencils per complex FFT)
//   k_cy   y-lines: C2C forward of the 3 half spectra
//   k_mx   x-pencils in k-space: forward x, then the 27 constant-Q derivative
//          spectra Ap_j(|k|) * ik e^{+-ik d/2} * V (cu:475-744 fused), each
//          inverse-transformed along x on chip
//   k_cy   y-lines: C2C inverse of the 27 spectra
//   k_iz   z-pencils: C2R of the 27 fields, stress update with constant-Q
//          dispersion + loss and C-PML (cuda_kernel_calculate_p,
//          cu:800-1015), source injection (cu:747-777), and the z
//          derivatives of the new stresses for the next velocity update
//   k_rec  receiver sampling (cu:782-791)
//
// The stress-divergence derivatives need no 3D transform at all: their
// multiplier depends on one wavenumber component, so IFFT3(M(kx) FFT3(f)) is
// the 1D spectral derivative along x of every x line (likewise y, z).
#include <algorithm>
#include <cstdio>
#include <type_traits>

#include "engine.cuh"

namespace qvti {

namespace {

constexpr int kThreads = 256;
constexpr int kEpi = 4;  // cells per thread and trip in the velocity-kernel epilogues

// Element offsets fit in 32 bits: the engine accepts at most 1024^3 cells
// (qvti_create), and 32-bit offsets take one multiply-add per address.
__device__ __forceinline__ int cell(const KP& k, int x, int y, int z) { return (x * k.ny + y) * k.nz + z; }
__device__ __forceinline__ int spec(const KP& k, int kz, int x, int y) { return (kz * k.nx + x) * k.ny + y; }
__device__ __forceinline__ bool in_slab(int i, int n, int pml) { return i < pml || i >= n - pml; }

// Bulk prefetch of `bytes` (multiple of 16, 16-byte aligned) into L2.  The
// address operand is warp-uniform in hardware: issue it from one thread (a
// per-lane address makes the compiler serialise the lanes).
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}
__device__ __forceinline__ void load_table(float2* s, const float2* g, int n)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) s[i] = g[i];
}

// A transform of the tile through the compile-time path (N > 0: length N, PC
// pencils, NT threads) or the runtime one (N == 0: plan pl, prt pencils,
// layout ps_rt/is_rt).  LY is the shared-memory layout (kLine, kPencil,
// kLinePad); the padded layouts carry one padding row every 16 indices in
// both paths.
template <int N, int PC, int NT, int LY, bool INV, bool ROLL = false, class Load, class Store>
__device__ __forceinline__ void fft_any(const FftPlan& pl, const float2* tw, float2* A, float2* B, int prt, int ps_rt,
                                        int is_rt, Load load, Store store)
{
    if constexpr (N > 0) FftCT<N, PC, NT, LY, false, ROLL>::template run<INV>(tw, A, B, load, store);
    else fft_run<LY == kPencil>(pl, tw, A, B, prt, ps_rt, is_rt, INV, load, store, LY == kLine ? 0 : 4);
}
template <int N, int PC, int NT, int LY>
__device__ __forceinline__ float2* out_any(const FftPlan& pl, float2* A, float2* B)
{
    if constexpr (N > 0) return FftCT<N, PC, NT, LY>::out_buf(A, B);
    else return fft_out_buf(pl, A, B);
}

// Derivative bookkeeping for the 9 stress-side derivatives d (G index
// o = 3 d + j): component, axis, forward(1)/backward(0) staggered shift.
// d: 0 dx vx, 1 dy vy, 2 dz vz (forward shift, kvx_x kvy_y kvz_z),
//    3 dz vx, 4 dx vz, 5 dy vx, 6 dx vy, 7 dz vy, 8 dy vz (backward shift)
// -- the table assignment of cuviscoelas_3D.cu:1342-1562.
__constant__ int c_comp[9] = {0, 1, 2, 0, 2, 0, 1, 1, 2};
__constant__ int c_axis[9] = {0, 1, 2, 2, 0, 1, 0, 2, 1};
__constant__ int c_fwd[9] = {1, 1, 1, 0, 0, 0, 0, 0, 0};
// G indices that go through the x and y passes (all but kGz)
__constant__ int c_gxy[kNumGxy] = {0, 1, 2, 3, 5, 6, 8, 9, 11, 12, 13, 14, 15, 17, 18, 19, 20, 21, 23, 24, 26};

// ------------------------------------------------------------------ k_fz --
// R2C along z of vx, vy, vz.  Tile: one x, P consecutive y rows (P even);
// rows (2q, 2q+1) share one complex transform.  Output H[f][kz][x][y].
template <int N>
__global__ void __launch_bounds__(kThreads) k_fz(KP k, int P_rt)
{
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    const int P = N > 0 ? 16 : P_rt;
    const int n = N > 0 ? N : k.nz, Qp = P / 2, ps = n + n / 16;
    float2* tw = sm;
    float2* A = tw + n;
    float2* B = A + Qp * ps;
    load_table(tw, k.tw_z, n);
    __syncthreads();
    const int f = blockIdx.z, x = blockIdx.y, y0 = blockIdx.x * P;
    const int yv = min(P, k.ny - y0);  // rows of the tile inside the grid (even)
    const float* src = k.v[f];
    float2* Z = out_any<N, 8, kThreads, kLinePad>(k.pz, A, B);
    auto load = [&](int q, int i) -> float2 {
        if (2 * q >= yv) return make_float2(0.f, 0.f);
        const int b = cell(k, x, y0 + 2 * q, i);
        return make_float2(src[b], src[b + n]);
    };
    auto store = [&](int q, int i, float2 v) { Z[q * ps + i] = v; };
    fft_any<N, 8, kThreads, kLinePad, false>(k.pz, tw, A, B, Qp, ps, 1, load, store);
    float2* H = k.H[f];
    for (int t = threadIdx.x; t < k.nkz * P; t += blockDim.x) {
        const int p = t % P, kz = t / P, q = p >> 1;
        if (p >= yv) continue;
        const float2 z = Z[q * ps + kz];
        const float2 zm = cconj(Z[q * ps + (kz ? n - kz : 0)]);
        H[spec(k, kz, x, y0 + p)] = (p & 1) ? unpack_b(z, zm) : unpack_a(z, zm);
    }
}

// ------------------------------------------------------------------ k_cy --
// C2C along y, in place, on L contiguous y lines per block (lines (kz, x)
// starting at line0).  Line-major mapping on a padded tile: each half warp
// reads or writes 16 consecutive points (128 bytes) of one line, so a warp
// access touches two lines, and the radix-16 shared-memory stages are
// conflict-free.  The field is H[0..2] (forward) or G[0..26] (inverse), by
// blockIdx.y.
constexpr int kCyThreads = 128;  // L = 8 lines x 256 points = one radix-16 butterfly per thread

template <int N, bool INV>
__global__ void __launch_bounds__(kCyThreads) k_cy(KP k, int L_rt, long long line0, long long line_end)
{
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    const int L = N > 0 ? 8 : L_rt;
    const int n = N > 0 ? N : k.ny;
    float2* tw = sm;
    float2* A = tw + n;
    float2* B = A + L * (n + n / 16);
    float2* C = B + L * (n + n / 16);  // forward with Yv: the lines' y spectra, [L][n]
    load_table(tw, k.tw_y, n);
    __syncthreads();
    // forward: H -> Hy (H stays for k_sigma's kz-only fields); inverse: G in
    // place, blockIdx.y over the fields that went through k_mx
    const int c = blockIdx.y;
    const long long first = line0 + (long long)blockIdx.x * L;
    const int lv = (int)min((long long)L, line_end - first);  // lines of the tile inside the batch
    const long long off = first * n;
    const float2* src = (INV ? k.G[c_gxy[c]] : k.H[c]) + off;
    float2* dst = (INV ? k.G[c_gxy[c]] : k.Hy[c]) + off;
    const bool ydv = !INV && k.Yv[c] != nullptr;
    auto load = [&](int p, int i) -> float2 { return p < lv ? src[(long long)p * n + i] : make_float2(0.f, 0.f); };
    auto store = [&](int p, int i, float2 v) {
        if (p < lv) dst[(long long)p * n + i] = v;
        if (ydv) C[p * n + i] = v;
    };
    fft_any<N, 8, kCyThreads, kLinePad, INV>(k.py, tw, A, B, L, n + n / 16, 1, load, store);
    if constexpr (!INV) {
        if (ydv) {
            // the y derivative with the identity dispersion operator, scaled
            // by 1/(ny nz) like a field of the x and y passes (1/ntp times
            // the x round trip's nx): dy vy (c = 1, forward shift), dy vx and
            // dy vz (backward)
            const float2* T = c == 1 ? k.Fy : k.By;
            const float inv_n = 1.0f / ((float)n * (float)k.nz);
            float2* yd = k.Yv[c] + off;
            auto load_d = [&](int p, int i) -> float2 { return cmul(C[p * n + i], cscale(T[i], inv_n)); };
            auto store_d = [&](int p, int i, float2 v) {
                if (p < lv) yd[(long long)p * n + i] = v;
            };
            fft_any<N, 8, kCyThreads, kLinePad, true>(k.py, tw, A, B, L, n + n / 16, 1, load_d, store_d);
        }
    }
}

// ------------------------------------------------------------------ k_mx --
// x-pencils of a (kz, y-chunk) tile in k-space for one velocity component c
// (blockIdx.z): forward x-FFT of V_c, then the 9 fields that use V_c --
// 3 derivatives x 3 dispersion operators Ap_j D_d V_c -- each inverse
// x-transformed on chip.  blockIdx.y + kz0 is the kz plane.
template <int N>
__global__ void __launch_bounds__(kThreads) k_mx(KP k, int P_rt, int kz0)
{
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    const int P = N > 0 ? 16 : P_rt;
    const int n = N > 0 ? N : k.nx;
    // the second transform buffer exists only for transforms of more than
    // two stages (a two-stage transform reads its input through `load` and
    // writes its output through `store`)
    const int nbuf = (N > 0 ? ct_nst(N) : k.px.nst) > 2 ? 2 : 1;
    float2* tw = sm;
    float2* tFx = tw + n;
    float2* tBx = tFx + n;
    float2* V = tBx + n;            // [n][P]
    float2* A = V + n * P;
    float2* B = A + (n + n / 16) * P;
    float2* tFBy = A + nbuf * (n + n / 16) * P;  // [2][P]: Fy, By of the tile's rows
    float* tkx = reinterpret_cast<float*>(tFBy + 2 * P);
    float* tky = tkx + n;                         // [P]
    const int kz = kz0 + blockIdx.y, y0 = blockIdx.x * P, c = blockIdx.z;
    const int yv = min(P, k.ny - y0);  // rows of the tile inside the grid
    load_table(tw, k.tw_x, n);
    load_table(tFx, k.Fx, n);
    load_table(tBx, k.Bx, n);
    for (int i = threadIdx.x; i < n; i += blockDim.x) tkx[i] = k.kx[i];
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        const bool in = i < yv;
        tky[i] = in ? k.ky[y0 + i] : 0.f;
        tFBy[i] = in ? k.Fy[y0 + i] : make_float2(0.f, 0.f);
        tFBy[P + i] = in ? k.By[y0 + i] : make_float2(0.f, 0.f);
    }
    __syncthreads();

    {
        const float2* H = k.Hy[c];
        auto load = [&](int p, int i) -> float2 { return p < yv ? H[spec(k, kz, i, y0 + p)] : make_float2(0.f, 0.f); };
        auto store = [&](int p, int i, float2 v) { V[i * P + p] = v; };
        fft_any<N, 16, kThreads, kPencil, false>(k.px, tw, A, B, P, 1, P, load, store);
    }

    const float kzv = k.kz[kz];
    const float kz2 = kzv * kzv;
    const float2 tFz = k.Fz[kz], tBz = k.Bz[kz];
    for (int d = 0; d < 9; ++d) {
        if (c_comp[d] != c) continue;
        const int ax = c_axis[d], fw = c_fwd[d];
        for (int j = 0; j < 3; ++j) {
            if (is_gz(3 * d + j) || is_gy(3 * d + j)) continue;  // one-axis fields: formed elsewhere
            float2* G = k.G[3 * d + j];
            auto load = [&](int p, int i) -> float2 {
                const float kyv = tky[p];
                const float kxv = tkx[i];
                float k2 = kxv * kxv + kyv * kyv + kz2;
                k2 = fmaxf(k2, 1e-10f);  // the reference sets |k|^2 = 1e-10 at DC (cu:74)
                // |k|^-1 and |k| from the hardware reciprocal square root
                // (~2 ulp): far below the FP32 transforms' own rounding
                const float rk = rsqrtf(k2);
                const float ap = j == 1 ? 1.0f : (j == 0 ? rk : k2 * rk);
                float2 T;
                if (ax == 0) T = fw ? tFx[i] : tBx[i];
                else if (ax == 1) T = fw ? tFBy[p] : tFBy[P + p];
                else T = fw ? tFz : tBz;
                return cmul(V[i * P + p], cscale(T, ap * k.inv_ntp));
            };
            auto store = [&](int p, int i, float2 v) {
                if (p < yv) G[spec(k, kz, i, y0 + p)] = v;
            };
            fft_any<N, 16, kThreads, kPencil, true>(k.px, tw, A, B, P, 1, P, load, store);
        }
    }
}

// --------------------------------------------------------------- k_sigma --
// Constant-Q set of one modulus from its effective velocity c = v cos(pi g/2)
// (cuviscoelas_3D.cu:195-205): eta1 = -rho c g w0, eta2 = rho c^2,
// eta3 = rho c^3 g / w0, tau1 = rho c g pi, tau2 = rho c^2 g^2 pi / w0.
// c is built in FP64 at setup; the products are rebuilt here in FP32.
__device__ __forceinline__ void qset_f(float rho, float c, float g, float w0, float inv_w0, float o[5])
{
    const float pi = 3.1415926f;
    const float rc = rho * c, rc2 = rc * c;
    o[0] = -rc * g * w0;
    o[1] = rc2;
    o[2] = rc2 * c * g * inv_w0;
    o[3] = rc * g * pi;
    o[4] = rc2 * g * g * pi * inv_w0;
}

constexpr int kSigmaRows = 4;  // y rows per k_sigma tile (compile-time path)
// A compile-time length keeps the C2R's real fields in the buffer its last
// stage reads (that stage writes each result into the slot it read, see
// k_sigma) on 288 threads: 9 fields x 2 pencils x 16 radix-16 butterflies,
// one task per thread in a radix-16 stage.  That drops a separate real tile
// (37 KB at 256 points, so three blocks fit an SM instead of two).
constexpr bool sigma_inplace(int n) { return n > 0; }
constexpr int sigma_threads(int n) { return sigma_inplace(n) ? 9 * kSigmaRows / 2 * 16 : kThreads; }
// Compile-time lengths can run the 27 fields as three groups of nine
// (normal; xz and the A half of xy; the B half of xy and yz), every transform
// stage a full round of 288 butterflies; the xy update's A half is folded into
// the stored sxy and Qxy in the first shear group and completed in the next.
constexpr bool sigma_regroup(int n) { return n > 0; }
// Two-stage compile-time lengths can keep the z-derivative pass's stresses
// out of a buffer of their own: the pass re-reads the stresses the update
// has just stored (L2) and parks its results in the transform buffer, which
// is free by then.  The smaller tile leaves the SM more L1.
constexpr bool sigma_nod_ok(int n) { return n > 0 && ct_nst(n) == 2; }
constexpr size_t sigma_smem_ct(int n, bool nod = false)  // smem_sigma for a compile-time length
{
    const size_t bufA = (size_t)9 * (kSigmaRows / 2) * (n + n / 16);  // float2
    const size_t nb = ct_nst(n) > 2 ? 2 : 1;
    const size_t sreal = sigma_inplace(n) ? 0 : (size_t)9 * kSigmaRows * (n + 1);
    const size_t dbuf = nod ? 0 : (size_t)3 * kSigmaRows * (n + 1);
    return 8 * ((size_t)n + nb * bufA + 2 * (size_t)n) + 4 * (sreal + dbuf + 4 * (size_t)n + 4 * kSigmaRows);
}
// Resident blocks per SM the register budget is sized for: as many as the
// tile's shared memory admits (at most 3), so a length whose tiles already
// limit residency gets the registers to keep more loads in flight.
constexpr int sigma_min_blocks(int n, bool nod = false)
{
    if (n == 0) return 3;
    const size_t b = (228 * 1024) / (sigma_smem_ct(n, nod) + 1024);
    return b < 1 ? 1 : b > 3 ? 3 : (int)b;
}
constexpr int sigma_cells(int n) { return (n == 256 && !sigma_inplace(n)) ? 2 : 1; }

// z-pencils of one x and P y rows (P/2 pencil pairs): C2R of the 27
// derivative fields group by group, each group batched into one transform
// and followed by its stress update; then the z derivatives of the new szz,
// sxz, syz for the next velocity update (cu:1279-1306: partz2, partz1,
// partz3) with their C-PML z terms, and the source injection.  Groups on the
// compile-time path: normal (G 0..8), xz with the A half of xy (9..17), the
// B half of xy with yz (18..26) -- nine fields, 288 butterflies per stage,
// one per thread; on the runtime path: normal, xz, xy, yz (9, 6, 6, 6).  At
// two-stage lengths the z pass re-reads the stresses it differentiates
// (just stored, in L2) instead of buffering them: the 12 KB saved lets the
// SM keep ~92 KB of L1 beside three resident tiles (measured at 256^3:
// 2.14 ms with four groups and the buffer, 2.08 with either change, 1.95
// with both).
//
// RAG: the grid's last y tile is partial (ny not a multiple of the tile); a
// separate instantiation, so the masks cost the full tiles no registers.
template <int N, bool RAG>
__global__ void __launch_bounds__(sigma_threads(N), sigma_min_blocks(N, sigma_nod_ok(N))) k_sigma(KP k, int P_rt)
{
    constexpr bool REGRP = sigma_regroup(N), NOD = sigma_nod_ok(N);
    constexpr bool INPLACE = sigma_inplace(N);
    constexpr int NT = sigma_threads(N);
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    const int P = N > 0 ? kSigmaRows : P_rt;
    const int n = N > 0 ? N : k.nz, Qp = P / 2, np1 = n + 1, nx = k.nx, ny = k.ny, pml = k.pml;
    const int two_buf = N > 0 ? (ct_nst(N) > 2) : (k.pz.nst > 2);
    const int bufA = 9 * Qp * (n + n / 16);
    float2* tw = sm;
    float2* A = tw + n;
    // S [9][P][np1]: the group's real fields.  In place: S overlays A and
    // there is no B (the z-derivative pass uses D as its second buffer);
    // otherwise B aliases S when the transform has two stages.
    float2* B = A + bufA;
    // the buffer the C2R's last stage reads: with the results written back in
    // place, the group's real fields live there
    float2* Lb = (N > 0 && ((ct_nst(N) - 2) & 1)) ? B : A;
    float* S = reinterpret_cast<float*>(B + (two_buf ? bufA : 0));  // not used in place
    // [3][P][np1]: szz sxz syz for the z pass (NOD: in the transform buffer
    // past the z pass's own stage buffer of 6 line-padded pencils, used only
    // once the groups are done)
    float* D = NOD ? reinterpret_cast<float*>(A + 3 * (kSigmaRows / 2) * (n + n / 16)) : INPLACE ? S : S + 9 * P * np1;
    float* tz = NOD ? reinterpret_cast<float*>(A + bufA) : D + 3 * P * np1;  // [4][n]: az bz azh bzh
    float* ty = tz + 4 * n;                                               // [4][P]: ay by ayh byh of the rows
    float2* tzs = reinterpret_cast<float2*>(ty + 4 * P);                  // [2][n]: Fz Bz
    constexpr int NGRP = REGRP ? 3 : 4;
    const int x = blockIdx.y, y0 = blockIdx.x * P;
    const int yv = RAG ? min(P, ny - y0) : P;  // rows of the tile inside the grid (even)
    load_table(tw, k.tw_z, n);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        tz[i] = k.az[i];
        tz[n + i] = k.bz[i];
        tz[2 * n + i] = k.azh[i];
        tz[3 * n + i] = k.bzh[i];
        tzs[i] = k.Fz[i];
        tzs[n + i] = k.Bz[i];
    }
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        const bool in = !RAG || i < yv;
        ty[i] = in ? k.ay[y0 + i] : 0.f;
        ty[P + i] = in ? k.by[y0 + i] : 0.f;
        ty[2 * P + i] = in ? k.ayh[y0 + i] : 0.f;
        ty[3 * P + i] = in ? k.byh[y0 + i] : 0.f;
    }
    const float axv = k.ax[x], bxv = k.bx[x], axhv = k.axh[x], bxhv = k.bxh[x];
    // where each of the 27 fields comes from: G (x/y passes), Yv (forward y
    // pass, already scaled) or H times the z shift multiplier (kind 1:
    // forward, 2: backward)
    __shared__ const float2* s_src[kNumG];
    __shared__ int s_kind[kNumG];
    for (int o = threadIdx.x; o < kNumG; o += blockDim.x) {
        s_src[o] = is_gz(o) ? k.H[o == 7 ? 2 : o == 10 ? 0 : 1] : is_gy(o) ? k.Yv[o == 4 ? 1 : o == 16 ? 0 : 2] : k.G[o];
        s_kind[o] = is_gz(o) ? (o == 7 ? 1 : 2) : 0;
    }
    __syncthreads();
    const int it = *k.d_it;
    const float inv_nz = 1.0f / n;
    // inv_dt enters only the loss terms (the spectral time derivative of the
    // constant-Q loss operator): their sign and presence follow the medium
    // (k.loss_scale: 1 viscoelastic, 0 dispersion only, -1 Q-compensated)
    const float dt = k.dt, ls = k.loss_scale, inv_dt = ls / k.dt;
    const float w0 = k.w0, inv_w0 = 1.0f / k.w0;
    const int src_ip = (k.s_ix >= 0) ? cell(k, k.s_ix, k.s_iy, k.s_iz) : -1;

    // L2 prefetch of the contiguous P*nz runs of the stresses, loss
    // potentials and coefficients a group's update reads, issued one group
    // ahead by one thread.  (The half spectra are read by the transform's
    // first stage, which keeps 16 loads per thread in flight; prefetching
    // them 32 bytes at a time cost more instructions than it saved.)
    auto prefetch_group = [&](int g) {
        if (g >= NGRP) return;
        const int c0 = cell(k, x, y0, 0);
        const unsigned run = 4u * yv * n;
        if (threadIdx.x == 0) {
            if (g == 0) {
                const float* arr[13] = {k.s[0], k.s[1], k.s[2], k.Q[0], k.Q[1], k.Q[2], k.mrho, k.mgp, k.mgs,
                                        k.mc11, k.mc33, k.mc13, k.mcs};
                for (int a = 0; a < 13; ++a) prefetch_l2(arr[a] + c0, run);
            } else {
                // stresses and loss potentials the group updates (REGRP: xz;
                // xy and yz), then the shear set
                const int s1 = REGRP ? (g == 1 ? 4 : 3) : (g == 1 ? 4 : g == 2 ? 3 : 5);
                prefetch_l2(k.s[s1] + c0, run);
                prefetch_l2(k.Q[s1] + c0, run);
                if (REGRP && g == 2) {
                    prefetch_l2(k.s[5] + c0, run);
                    prefetch_l2(k.Q[5] + c0, run);
                }
                for (int j = 0; j < 5; ++j) prefetch_l2(k.MU[j] + c0, run);
            }
        }
    };
    prefetch_group(0);

    // C-PML state of one shear term: g the shear component (1 xz, 2 xy, 3
    // yz), hb its B half (xz vz_x, xy vy_x, yz vz_y) or A half (xz vx_z,
    // xy vx_y, yz vy_z); the slab it lives in, its memory variables (loaded
    // here) and profile.
    struct ShearTerm {
        bool on;
        int is, m;
        float qo, po, a, b;
    };
    auto shear_term = [&](int g, bool hb, int p, int y, int z) -> ShearTerm {
        ShearTerm t;
        t.m = (g - 1) * 2 + (hb ? 1 : 0);
        const bool ysl = hb ? g == 3 : g == 2;  // y slab; otherwise A: z slab, B: x slab
        t.on = ysl ? in_slab(y, ny, pml) : hb ? in_slab(x, nx, pml) : in_slab(z, n, pml);
        t.is = !t.on ? 0 : ysl ? slab_y(k, x, y, z) : hb ? slab_x(k, x, y, z) : slab_z(k, x, y, z);
        t.qo = t.on ? k.qs[t.m][t.is] : 0.f;
        t.po = t.on ? k.phs[t.m][t.is] : 0.f;
        t.a = ysl ? ty[2 * P + p] : hb ? axhv : tz[2 * n + z];
        t.b = ysl ? ty[3 * P + p] : hb ? bxhv : tz[3 * n + z];
        return t;
    };
    auto shear_ph = [&](const ShearTerm& t, float d, float q) {
        const float T = d + (q - t.qo) * inv_dt;
        return t.on ? t.po + dt * (-t.a * t.po - t.b * T) : 0.f;
    };
    auto shear_store = [&](const ShearTerm& t, float q, float ph) {
        if (t.on) { k.qs[t.m][t.is] = q; k.phs[t.m][t.is] = ph; }
    };

    for (int grp = 0; grp < NGRP; ++grp) {
        const int NF = (REGRP || grp == 0) ? 9 : 6;
        const int o0 = REGRP ? 9 * grp : grp == 0 ? 0 : 9 + (grp - 1) * 6;
        const int npen = NF * Qp;
        prefetch_group(grp + 1);
        // 1. batched C2R along z: pencil p' = f*Qp + q holds rows (2q, 2q+1)
        //    of field f packed as A + iB (Hermitian extension of the half
        //    spectra; imaginary parts at kz = 0 and nz/2 dropped like a C2R).
        // a kz-only field (is_gz) is M(kz) H(kz) / nz, a ky-only one (is_gy)
        // Yv, which the forward y pass scaled alike: the values the x and y
        // round trip (normalised by 1/ntp) would have produced
        auto load = [&](int pp, int i) -> float2 {
            const int f = pp / Qp, q = pp - f * Qp, o = o0 + f;
            if (RAG && 2 * q >= yv) return make_float2(0.f, 0.f);
            const int kk = i <= n / 2 ? i : n - i;
            const float4 gg = *reinterpret_cast<const float4*>(s_src[o] + spec(k, kk, x, y0 + 2 * q));
            float2 a = make_float2(gg.x, gg.y), b = make_float2(gg.z, gg.w);
            const int kind = s_kind[o];
            if (kind) {
                const float2 m = cscale(tzs[(kind == 1 ? 0 : n) + kk], inv_nz);
                a = cmul(a, m);
                b = cmul(b, m);
            }
            if (kk == 0 || 2 * kk == n) { a.y = 0.f; b.y = 0.f; }
            if (i > n / 2) { a.y = -a.y; b.y = -b.y; }
            return make_float2(a.x - b.y, a.y + b.x);
        };
        auto store = [&](int pp, int i, float2 v) {
            const int f = pp / Qp, q = pp - f * Qp;
            S[(f * P + 2 * q) * np1 + i] = v.x;
            S[(f * P + 2 * q + 1) * np1 + i] = v.y;
        };
        if constexpr (INPLACE) {
            // The last Stockham stage's butterfly writes exactly the indices
            // it read (j + r N/R), so each pencil pair's real rows go back,
            // as one float2, into the slot of the staging tile they came from:
            // every thread overwrites only its own inputs, no barrier or
            // register staging needed.  The update reads them through sval.
            // Two-stage lengths take stage 1's twiddles in stage 0 (PRETW),
            // which keeps the 256-point transform free of register spill;
            // multi-round stages stay loops (ROLL) for the same reason at the
            // lengths with small radices.
            if (REGRP || grp == 0) {
                using F = FftCT<N, 9 * kSigmaRows / 2, NT, kPencil, ct_nst(N) == 2, true>;
                auto keep = [&](int pp, int i, float2 v) { Lb[F::at(pp, i)] = v; };
                F::template run<true>(tw, A, B, load, keep);
            } else {
                using F = FftCT<N, 6 * kSigmaRows / 2, NT, kPencil, ct_nst(N) == 2, true>;
                auto keep = [&](int pp, int i, float2 v) { Lb[F::at(pp, i)] = v; };
                F::template run<true>(tw, A, B, load, keep);
            }
        } else {
            if (grp == 0) fft_any<N, 9 * kSigmaRows / 2, NT, kPencil, true>(k.pz, tw, A, B, npen, 1, npen, load, store);
            else fft_any<N, 6 * kSigmaRows / 2, NT, kPencil, true>(k.pz, tw, A, B, npen, 1, npen, load, store);
        }

        // real value of field f (of this group), row p, height z
        const float* Af = reinterpret_cast<const float*>(Lb);
        auto sval = [&](int f, int p, int z) -> float {
            if constexpr (INPLACE) {
                const int pp = f * Qp + (p >> 1);
                const int slot = (REGRP || grp == 0) ? FftCT<N, 9 * kSigmaRows / 2, NT, kPencil>::at(pp, z)
                                                     : FftCT<N, 6 * kSigmaRows / 2, NT, kPencil>::at(pp, z);
                return Af[2 * slot + (p & 1)];
            } else {
                return S[(f * P + p) * np1 + z];
            }
        };
        // 2. stress update of the group.  Each thread owns kCells cells; all
        //    their streaming inputs are loaded before any store so the loads
        //    are in flight together (the arrays cannot alias, but the
        //    compiler cannot know that through the parameter struct).
        constexpr int kCells = sigma_cells(N);
        static_assert(!REGRP || kCells == 1, "the regrouped updates take one cell per trip");
        for (int t0 = threadIdx.x; t0 < P * n; t0 += kCells * blockDim.x) {
            if (grp == 0) {
                float* __restrict__ s0 = k.s[0];
                float* __restrict__ s1 = k.s[1];
                float* __restrict__ s2 = k.s[2];
                float* __restrict__ q0 = k.Q[0];
                float* __restrict__ q1 = k.Q[1];
                float* __restrict__ q2 = k.Q[2];
                float in[kCells][13];
                int ipv[kCells];
                bool ok[kCells];
#pragma unroll
                for (int u = 0; u < kCells; ++u) {
                    const int t = t0 + u * blockDim.x;
                    ok[u] = t < P * n && (!RAG || t / n < yv);
                    const int p = t / n, z = t - p * n;
                    ipv[u] = cell(k, x, y0 + p, z);
                    if (ok[u]) {
                        const int ip = ipv[u];
                        in[u][0] = s0[ip]; in[u][1] = s1[ip]; in[u][2] = s2[ip];
                        in[u][3] = q0[ip]; in[u][4] = q1[ip]; in[u][5] = q2[ip];
                        in[u][6] = __ldg(k.mrho + ip); in[u][7] = __ldg(k.mgp + ip); in[u][8] = __ldg(k.mgs + ip);
                        in[u][9] = __ldg(k.mc11 + ip); in[u][10] = __ldg(k.mc33 + ip);
                        in[u][11] = __ldg(k.mc13 + ip); in[u][12] = __ldg(k.mcs + ip);
                    }
                }
#pragma unroll
                for (int u = 0; u < kCells; ++u) {
                    if (!ok[u]) continue;
                    const int t = t0 + u * blockDim.x;
                    const int p = t / n, z = t - p * n, y = y0 + p;
                    const int ip = ipv[u];
                    const bool upd = x < nx - 1 && y < ny - 1 && z < n - 1;
                    auto sv = [&](int f) { return sval(f, p, z); };
                    float sxx = in[u][0], syy = in[u][1], szz = in[u][2];
                    if (upd) {
                        float a11[5], a33[5], a13[5], s5[5], a12[5];
                        qset_f(in[u][6], in[u][9], in[u][7], w0, inv_w0, a11);
                        qset_f(in[u][6], in[u][10], in[u][7], w0, inv_w0, a33);
                        qset_f(in[u][6], in[u][11], in[u][7], w0, inv_w0, a13);
                        qset_f(in[u][6], in[u][12], in[u][8], w0, inv_w0, s5);
#pragma unroll
                        for (int j = 0; j < 5; ++j) {
                            a12[j] = a11[j] - 2.0f * s5[j];
                            a13[j] = a13[j] - 2.0f * s5[j];
                        }
                        const float X0 = sv(0), X1 = sv(1), X2 = sv(2);
                        const float Y0 = sv(3), Y1 = sv(4), Y2 = sv(5);
                        const float Z0 = sv(6), Z1 = sv(7), Z2 = sv(8);
#define QD(a, s0_, s1_, s2_) (a[0] * s0_ + a[1] * s1_ + a[2] * s2_)
#define QL(a, s0_, s1_) (a[3] * s0_ + a[4] * s1_)
                        const float d11x = QD(a11, X0, X1, X2), d12x = QD(a12, X0, X1, X2), d13x = QD(a13, X0, X1, X2);
                        const float d12y = QD(a12, Y0, Y1, Y2), d11y = QD(a11, Y0, Y1, Y2), d13y = QD(a13, Y0, Y1, Y2);
                        const float d13z = QD(a13, Z0, Z1, Z2), d33z = QD(a33, Z0, Z1, Z2);
                        const float q11x = QL(a11, X0, X1), q12x = QL(a12, X0, X1), q13x = QL(a13, X0, X1);
                        const float q12y = QL(a12, Y0, Y1), q11y = QL(a11, Y0, Y1), q13y = QL(a13, Y0, Y1);
                        const float q13z = QL(a13, Z0, Z1), q33z = QL(a33, Z0, Z1);
#undef QD
#undef QL
                        // C-PML terms of the slabs this cell is in: every load is
                        // issued before any store (the arrays are distinct, but
                        // through the parameter struct the compiler cannot know)
                        const bool sx = in_slab(x, nx, pml), sy = in_slab(y, ny, pml), sz = in_slab(z, n, pml);
                        float qo[8], po[8];
                        const int isx = sx ? slab_x(k, x, y, z) : 0, isy = sy ? slab_y(k, x, y, z) : 0,
                                  isz = sz ? slab_z(k, x, y, z) : 0;
#pragma unroll
                        for (int m = 0; m < 8; ++m) {
                            const bool on = m < 3 ? sx : (m < 6 ? sy : sz);
                            const int is = m < 3 ? isx : (m < 6 ? isy : isz);
                            qo[m] = on ? k.qn[m][is] : 0.f;
                            po[m] = on ? k.phn[m][is] : 0.f;
                        }
                        // loss: sum_terms tau-coefficient x (S - S_prev)/dt = (Q - Q_prev)/dt
                        const float Qxx = q11x + q12y + q13z, Qyy = q12x + q11y + q13z, Qzz = q13x + q13y + q33z;
                        const float Lxx = (Qxx - in[u][3]) * inv_dt;
                        const float Lyy = (Qyy - in[u][4]) * inv_dt;
                        const float Lzz = (Qzz - in[u][5]) * inv_dt;
                        const float dterm[8] = {d11x, d12x, d13x, d12y, d11y, d13y, d13z, d33z};
                        const float qterm[8] = {q11x, q12x, q13x, q12y, q11y, q13y, q13z, q33z};
                        float ph[8];
#pragma unroll
                        for (int m = 0; m < 8; ++m) {
                            const float a = m < 3 ? axv : (m < 6 ? ty[p] : tz[z]);
                            const float b = m < 3 ? bxv : (m < 6 ? ty[P + p] : tz[n + z]);
                            const float T = dterm[m] + (qterm[m] - qo[m]) * inv_dt;
                            ph[m] = po[m] + dt * (-a * po[m] - b * T);
                        }
                        if (!sx) { ph[0] = ph[1] = ph[2] = 0.f; }
                        if (!sy) { ph[3] = ph[4] = ph[5] = 0.f; }
                        if (!sz) { ph[6] = ph[7] = 0.f; }
                        // ph[6] is phi_vz_zx == phi_vz_zy
                        sxx = sxx + dt * (d11x + d12y + d13z + Lxx + ph[0] + ph[3] + ph[6]);
                        syy = syy + dt * (d12x + d11y + d13z + Lyy + ph[1] + ph[4] + ph[6]);
                        szz = szz + dt * (d13x + d13y + d33z + Lzz + ph[2] + ph[5] + ph[7]);
                        q0[ip] = Qxx; q1[ip] = Qyy; q2[ip] = Qzz;
#pragma unroll
                        for (int m = 0; m < 8; ++m) {
                            const bool on = m < 3 ? sx : (m < 6 ? sy : sz);
                            const int is = m < 3 ? isx : (m < 6 ? isy : isz);
                            if (on) { k.qn[m][is] = qterm[m]; k.phn[m][is] = ph[m]; }
                        }
                    }
                    if (ip == src_ip && it < k.nt_rec) {  // cu:772-777, after the update
                        if (k.src_type == 1) {
                            const float w = k.rik[it];
                            sxx += w; syy += w; szz += w;
                        } else {
                            k.v[0][ip] += k.rik[it];
                        }
                    }
                    if (upd || ip == src_ip) { s0[ip] = sxx; s1[ip] = syy; s2[ip] = szz; }
                    if constexpr (!NOD) D[(0 * P + p) * np1 + z] = szz;
                }
            } else if (!REGRP) {
                const int sidx = grp == 1 ? 4 : grp == 2 ? 3 : 5;  // sxz, sxy, syz in s[]
                float* __restrict__ sg = k.s[sidx];
                float* __restrict__ qg = k.Q[sidx];
                float in[kCells][7];
                int ipv[kCells];
                bool ok[kCells];
#pragma unroll
                for (int u = 0; u < kCells; ++u) {
                    const int t = t0 + u * blockDim.x;
                    ok[u] = t < P * n && (!RAG || t / n < yv);
                    const int p = t / n, z = t - p * n;
                    ipv[u] = cell(k, x, y0 + p, z);
                    if (ok[u]) {
                        const int ip = ipv[u];
                        in[u][0] = sg[ip];
                        in[u][1] = qg[ip];
#pragma unroll
                        for (int j = 0; j < 5; ++j) in[u][2 + j] = __ldg(k.MU[j] + ip);
                    }
                }
#pragma unroll
                for (int u = 0; u < kCells; ++u) {
                    if (!ok[u]) continue;
                    const int t = t0 + u * blockDim.x;
                    const int p = t / n, z = t - p * n, y = y0 + p;
                    const int ip = ipv[u];
                    const bool upd = x < nx - 1 && y < ny - 1 && z < n - 1;
                    auto sv = [&](int f) { return sval(f, p, z); };
                    float sig = in[u][0];
                    if (upd) {
                        const float* mu = &in[u][2];
                        const float A0 = sv(0), A1 = sv(1), A2 = sv(2), B0 = sv(3), B1 = sv(4), B2 = sv(5);
                        const float dA = mu[0] * A0 + mu[1] * A1 + mu[2] * A2, qA = mu[3] * A0 + mu[4] * A1;
                        const float dB = mu[0] * B0 + mu[1] * B1 + mu[2] * B2, qB = mu[3] * B0 + mu[4] * B1;
                        const float Qs = qA + qB;
                        const float L = (Qs - in[u][1]) * inv_dt;
                        // term A: xz vx_z (z slab), xy vx_y (y slab), yz vy_z (z slab)
                        // term B: xz vz_x (x slab), xy vy_x (x slab), yz vz_y (y slab)
                        const int mA = (grp - 1) * 2, mB = mA + 1;
                        const bool onA = grp == 2 ? in_slab(y, ny, pml) : in_slab(z, n, pml);
                        const bool onB = grp == 3 ? in_slab(y, ny, pml) : in_slab(x, nx, pml);
                        // A: z slab (xz, yz) or y slab (xy); B: x slab (xz, xy) or y slab (yz)
                        const int isA = !onA ? 0 : grp == 2 ? slab_y(k, x, y, z) : slab_z(k, x, y, z);
                        const int isB = !onB ? 0 : grp == 3 ? slab_y(k, x, y, z) : slab_x(k, x, y, z);
                        const float qoA = onA ? k.qs[mA][isA] : 0.f, poA = onA ? k.phs[mA][isA] : 0.f;
                        const float qoB = onB ? k.qs[mB][isB] : 0.f, poB = onB ? k.phs[mB][isB] : 0.f;
                        const float aA = grp == 2 ? ty[2 * P + p] : tz[2 * n + z];
                        const float bA = grp == 2 ? ty[3 * P + p] : tz[3 * n + z];
                        const float aB = grp == 3 ? ty[2 * P + p] : axhv, bB = grp == 3 ? ty[3 * P + p] : bxhv;
                        const float TA = dA + (qA - qoA) * inv_dt, TB = dB + (qB - qoB) * inv_dt;
                        const float phA = onA ? poA + dt * (-aA * poA - bA * TA) : 0.f;
                        const float phB = onB ? poB + dt * (-aB * poB - bB * TB) : 0.f;
                        sig = sig + dt * (dA + phA + dB + phB + L);
                        qg[ip] = Qs;
                        sg[ip] = sig;
                        if (onA) { k.qs[mA][isA] = qA; k.phs[mA][isA] = phA; }
                        if (onB) { k.qs[mB][isB] = qB; k.phs[mB][isB] = phB; }
                    }
                    if constexpr (!NOD) {
                        if (grp == 1) D[(1 * P + p) * np1 + z] = sig;
                        if (grp == 3) D[(2 * P + p) * np1 + z] = sig;
                    }
                }
            } else if (grp == 1) {
                // xz, and the A half (dy vx: y slab) of xy: with
                // dt L = ls (Qxy - Qxy_old), sxy_new = sxy + dt (dA + phA) +
                // ls (qA - Qxy_old) + dt (dB + phB) + ls qB and Qxy_new = qA + qB;
                // the A part goes into the stored sxy and Qxy now, the B part
                // in the next group
                float* __restrict__ sg = k.s[4];
                float* __restrict__ qg = k.Q[4];
                float* __restrict__ sxy = k.s[3];
                float* __restrict__ qxy = k.Q[3];
                {
                    const int t = t0;  // one cell per thread and trip (kCells == 1)
                    if (RAG && t / n >= yv) continue;
                    const int p = t / n, z = t - p * n, y = y0 + p;
                    const int ip = cell(k, x, y0 + p, z);
                    const float s_old = sg[ip], q_old = qg[ip], sxy_old = sxy[ip], qxy_old = qxy[ip];
                    float mu[5];
#pragma unroll
                    for (int j = 0; j < 5; ++j) mu[j] = __ldg(k.MU[j] + ip);
                    const bool upd = x < nx - 1 && y < ny - 1 && z < n - 1;
                    auto sv = [&](int f) { return sval(f, p, z); };
                    float sig = s_old;
                    if (upd) {
                        const float A0 = sv(0), A1 = sv(1), A2 = sv(2), B0 = sv(3), B1 = sv(4), B2 = sv(5);
                        const float C0 = sv(6), C1 = sv(7), C2 = sv(8);
                        const float dA = mu[0] * A0 + mu[1] * A1 + mu[2] * A2, qA = mu[3] * A0 + mu[4] * A1;
                        const float dB = mu[0] * B0 + mu[1] * B1 + mu[2] * B2, qB = mu[3] * B0 + mu[4] * B1;
                        const float dC = mu[0] * C0 + mu[1] * C1 + mu[2] * C2, qC = mu[3] * C0 + mu[4] * C1;
                        const float Qs = qA + qB;
                        const float L = (Qs - q_old) * inv_dt;
                        const ShearTerm tA = shear_term(1, false, p, y, z), tB = shear_term(1, true, p, y, z);
                        const ShearTerm tC = shear_term(2, false, p, y, z);
                        const float phA = shear_ph(tA, dA, qA), phB = shear_ph(tB, dB, qB), phC = shear_ph(tC, dC, qC);
                        sig = sig + dt * (dA + phA + dB + phB + L);
                        qg[ip] = Qs;
                        sg[ip] = sig;
                        shear_store(tA, qA, phA);
                        shear_store(tB, qB, phB);
                        shear_store(tC, qC, phC);
                        sxy[ip] = sxy_old + dt * (dC + phC) + ls * (qC - qxy_old);
                        qxy[ip] = qC;
                    }
                    if constexpr (!NOD) D[(1 * P + p) * np1 + z] = sig;
                }
            } else {
                // the B half (dx vy: x slab) of xy, then yz
                float* __restrict__ sxy = k.s[3];
                float* __restrict__ qxy = k.Q[3];
                float* __restrict__ syz = k.s[5];
                float* __restrict__ qyz = k.Q[5];
                {
                    const int t = t0;  // one cell per thread and trip (kCells == 1)
                    if (RAG && t / n >= yv) continue;
                    const int p = t / n, z = t - p * n, y = y0 + p;
                    const int ip = cell(k, x, y0 + p, z);
                    const float sxy_a = sxy[ip], qxy_a = qxy[ip], syz_old = syz[ip], qyz_old = qyz[ip];
                    float mu[5];
#pragma unroll
                    for (int j = 0; j < 5; ++j) mu[j] = __ldg(k.MU[j] + ip);
                    const bool upd = x < nx - 1 && y < ny - 1 && z < n - 1;
                    auto sv = [&](int f) { return sval(f, p, z); };
                    float sig = syz_old;
                    if (upd) {
                        const float B0 = sv(0), B1 = sv(1), B2 = sv(2);
                        const float A0 = sv(3), A1 = sv(4), A2 = sv(5), C0 = sv(6), C1 = sv(7), C2 = sv(8);
                        const float dB = mu[0] * B0 + mu[1] * B1 + mu[2] * B2, qB = mu[3] * B0 + mu[4] * B1;
                        const float dA = mu[0] * A0 + mu[1] * A1 + mu[2] * A2, qA = mu[3] * A0 + mu[4] * A1;
                        const float dC = mu[0] * C0 + mu[1] * C1 + mu[2] * C2, qC = mu[3] * C0 + mu[4] * C1;
                        const float Qyz = qA + qC;
                        const float Lyz = (Qyz - qyz_old) * inv_dt;
                        const ShearTerm tB = shear_term(2, true, p, y, z);
                        const ShearTerm tA = shear_term(3, false, p, y, z), tC = shear_term(3, true, p, y, z);
                        const float phB = shear_ph(tB, dB, qB), phA = shear_ph(tA, dA, qA), phC = shear_ph(tC, dC, qC);
                        const float nxy = sxy_a + dt * (dB + phB) + ls * qB;  // the A part is in sxy_a, qxy_a
                        sig = sig + dt * (dA + phA + dC + phC + Lyz);
                        qxy[ip] = qxy_a + qB;
                        sxy[ip] = nxy;
                        qyz[ip] = Qyz;
                        syz[ip] = sig;
                        shear_store(tB, qB, phB);
                        shear_store(tA, qA, phA);
                        shear_store(tC, qC, phC);
                    }
                    if constexpr (!NOD) D[(2 * P + p) * np1 + z] = sig;
                }
            }
        }
        __syncthreads();
    }

    // 3. z derivatives of the new szz (backward shift -> R_z), sxz (forward ->
    //    R_x), syz (forward -> R_y), batched: pencil p' = f*Qp + q.
    {
        const int npen = 3 * Qp;
        const float inv_n = 1.0f / n;
        auto load = [&](int pp, int i) -> float2 {
            const int f = pp / Qp, q = pp - f * Qp;
            if constexpr (NOD) {
                // the stresses this block stored above (the old value where
                // the update leaves a cell), visible after the barrier that
                // ended the last group
                if (RAG && 2 * q >= yv) return make_float2(0.f, 0.f);
                const float* sf = k.s[f == 0 ? 2 : f == 1 ? 4 : 5];
                const int b = cell(k, x, y0 + 2 * q, i);
                return make_float2(sf[b], sf[b + n]);
            } else {
                return make_float2(D[(f * P + 2 * q) * np1 + i], D[(f * P + 2 * q + 1) * np1 + i]);
            }
        };
        // in place with two stages there is no B: D serves (it is read only by
        // stage 0)
        float2* B2 = (INPLACE && !two_buf) ? reinterpret_cast<float2*>(D) : B;
        float2* Zf = out_any<N, 3 * kSigmaRows / 2, NT, kLinePad>(k.pz, A, B2);
        auto store_f = [&](int pp, int i, float2 v) { Zf[pp * np1 + i] = v; };
        fft_any<N, 3 * kSigmaRows / 2, NT, kLinePad, false, true>(k.pz, tw, A, B2, npen, n + n / 16, 1, load, store_f);
        float2* X1 = Zf == A ? B2 : A;
        auto load_i = [&](int pp, int i) -> float2 {
            const int f = pp / Qp;
            return cmul(Zf[pp * np1 + i], cscale(f == 0 ? tzs[n + i] : tzs[i], inv_n));
        };
        // derivatives parked in D (its stresses were consumed by stage 0 of
        // the forward transform), then written out with all loads first
        auto store_i = [&](int pp, int i, float2 v) {
            const int f = pp / Qp, q = pp - f * Qp;
            D[(f * P + 2 * q) * np1 + i] = v.x;
            D[(f * P + 2 * q + 1) * np1 + i] = v.y;
        };
        fft_any<N, 3 * kSigmaRows / 2, NT, kLinePad, true, true>(k.pz, tw, X1, Zf, npen, n + n / 16, 1, load_i,
                                                                 store_i);
        for (int t = threadIdx.x; t < 3 * P * n; t += blockDim.x) {
            const int i = t % n, fp = t / n, f = fp / P, p = fp - f * P;
            if (RAG && p >= yv) continue;
            const int y = y0 + p;
            const int rc = f == 0 ? 2 : f == 1 ? 0 : 1;
            float* __restrict__ ph = k.php[f == 0 ? 8 : f == 1 ? 2 : 5];  // pzz_z, pxz_z, pyz_z
            const int ip = cell(k, x, y, i);
            const bool slab = in_slab(i, n, pml) && i < n - 1 && x < nx - 1 && y < ny - 1;
            const int is = slab ? slab_z(k, x, y, i) : 0;
            const float old = slab ? ph[is] : 0.f;
            const float part = D[(f * P + p) * np1 + i];
            float r = part;
            if (slab) {
                const float a = f == 0 ? tz[2 * n + i] : tz[i];
                const float b = f == 0 ? tz[3 * n + i] : tz[n + i];
                const float nw = old + dt * (-a * old - b * part);
                ph[is] = nw;
                r += nw;
            }
            k.R[rc][ip] = r;
        }
    }
}

// ------------------------------------------------------------------ k_vy --
// y-derivatives of sxy (+, -> vx), syy (-, -> vy), syz (+, -> vz) for one x
// and P consecutive z; C-PML y terms; accumulate into R.  Each pass parks its
// derivatives in shared memory; the epilogue then loads everything a cell
// needs before storing anything (no store can delay a later load).
template <int N, bool RAG>
__global__ void __launch_bounds__(kThreads) k_vy(KP k, int P_rt)
{
    const int P = N > 0 ? 16 : P_rt;
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    const int n = N > 0 ? N : k.ny, ny = n, pml = k.pml;
    float2* tw = sm;
    float2* tF = tw + n;   // forward shift; the backward one is (-F.x, F.y)
    float2* A = tF + n;
    float2* B = A + (n + n / 16) * P;
    load_table(tw, k.tw_y, n);
    load_table(tF, k.Fy, n);
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *k.d_it += 1;  // step counter
    __syncthreads();
    const int x = blockIdx.y, z0 = blockIdx.x * P;
    const int zv = RAG ? min(P, k.nz - z0) : P;  // rows of the tile inside the grid (even)
    const float dt = k.dt, inv_n = 1.0f / n;
    const bool xin = x < k.nx - 1;
    const float* __restrict__ sxy = k.s[3];
    const float* __restrict__ syy = k.s[1];
    const float* __restrict__ syz = k.s[5];
    float* __restrict__ R0 = k.R[0];
    float* __restrict__ R1 = k.R[1];
    float* __restrict__ R2 = k.R[2];
    float* __restrict__ f1 = k.php[1];  // phi_pxy_y, b_y
    float* __restrict__ f4 = k.php[4];  // phi_pyy_y, averaged b_y
    float* __restrict__ f7 = k.php[7];  // phi_pyz_y, b_y

    // pass 1: sxy + i syy -> dy+ sxy (vx), dy- syy (vy)
    {
        float2* Zf = out_any<N, 16, kThreads, kPencil>(k.py, A, B);
        auto load = [&](int p, int i) -> float2 {
            if (RAG && p >= zv) return make_float2(0.f, 0.f);
            const int ip = cell(k, x, i, z0 + p);
            return make_float2(sxy[ip], syy[ip]);
        };
        auto store = [&](int p, int i, float2 v) { Zf[i * P + p] = v; };
        fft_any<N, 16, kThreads, kPencil, false>(k.py, tw, A, B, P, 1, P, load, store);
        float2* X1 = Zf == A ? B : A;
        // [2][n][P] in the buffer the last stage does not read
        float* D = reinterpret_cast<float*>(out_any<N, 16, kThreads, kPencil>(k.py, X1, Zf));
        auto load_i = [&](int p, int i) -> float2 {
            const int im = i ? n - i : 0;
            return two_shift(Zf[i * P + p], cconj(Zf[im * P + p]), cscale(tF[i], inv_n), 1.0f);
        };
        auto store_i = [&](int p, int i, float2 v) {
            D[i * P + p] = v.x;
            D[(n + i) * P + p] = v.y;
        };
        fft_any<N, 16, kThreads, kPencil, true>(k.py, tw, X1, Zf, P, 1, P, load_i, store_i);
        // kEpi cells per thread and trip: all their loads are in flight at once
        for (int t0 = threadIdx.x; t0 < n * P; t0 += kEpi * blockDim.x) {
            int ipu[kEpi], iu[kEpi], pu[kEpi], isu[kEpi];
            bool ok[kEpi], slab[kEpi];
            float r0[kEpi], r1[kEpi], p1[kEpi], p4[kEpi];
#pragma unroll
            for (int u = 0; u < kEpi; ++u) {
                const int t = t0 + u * blockDim.x;
                pu[u] = t % P;
                iu[u] = t / P;
                ok[u] = t < n * P && (!RAG || pu[u] < zv);
                const int z = z0 + pu[u];
                ipu[u] = cell(k, x, iu[u], z);
                slab[u] = ok[u] && in_slab(iu[u], ny, pml) && xin && iu[u] < ny - 1 && z < k.nz - 1;
                isu[u] = slab[u] ? slab_y(k, x, iu[u], z) : 0;
                r0[u] = ok[u] ? R0[ipu[u]] : 0.f;
                r1[u] = ok[u] ? R1[ipu[u]] : 0.f;
                p1[u] = slab[u] ? f1[isu[u]] : 0.f;
                p4[u] = slab[u] ? f4[isu[u]] : 0.f;
            }
#pragma unroll
            for (int u = 0; u < kEpi; ++u) {
                if (!ok[u]) continue;
                const int i = iu[u], p = pu[u], ip = ipu[u];
                const float dx = D[i * P + p], dy = D[(n + i) * P + p];
                float rx = r0[u] + dx, ry = r1[u] + dy;
                if (slab[u]) {
                    const float q1 = p1[u] + dt * (-k.ay[i] * p1[u] - k.by[i] * dx);
                    const float q4 = p4[u] + dt * (-k.ayh[i] * p4[u] - k.byh[i] * dy);
                    rx += q1;
                    ry += q4;
                    f1[isu[u]] = q1;
                    f4[isu[u]] = q4;
                }
                R0[ip] = rx;
                R1[ip] = ry;
            }
        }
        __syncthreads();
    }
    // pass 2: syz, pencils (2q, 2q+1) -> dy+ syz (vz)
    {
        const int Qp = P / 2;
        float2* Zf = out_any<N, 8, kThreads, kPencil>(k.py, A, B);
        auto load = [&](int q, int i) -> float2 {
            if (RAG && 2 * q >= zv) return make_float2(0.f, 0.f);
            const int ip = cell(k, x, i, z0 + 2 * q);
            return *reinterpret_cast<const float2*>(syz + ip);
        };
        auto store = [&](int q, int i, float2 v) { Zf[i * Qp + q] = v; };
        fft_any<N, 8, kThreads, kPencil, false>(k.py, tw, A, B, Qp, 1, Qp, load, store);
        float2* X1 = Zf == A ? B : A;
        float* D = reinterpret_cast<float*>(out_any<N, 8, kThreads, kPencil>(k.py, X1, Zf));  // [n][P]
        auto load_i = [&](int q, int i) -> float2 { return cmul(Zf[i * Qp + q], cscale(tF[i], inv_n)); };
        auto store_i = [&](int q, int i, float2 v) {
            D[i * P + 2 * q] = v.x;
            D[i * P + 2 * q + 1] = v.y;
        };
        fft_any<N, 8, kThreads, kPencil, true>(k.py, tw, X1, Zf, Qp, 1, Qp, load_i, store_i);
        for (int t0 = threadIdx.x; t0 < n * P; t0 += kEpi * blockDim.x) {
            int ipu[kEpi], iu[kEpi], pu[kEpi], isu[kEpi];
            bool ok[kEpi], slab[kEpi];
            float r2[kEpi], p7[kEpi];
#pragma unroll
            for (int u = 0; u < kEpi; ++u) {
                const int t = t0 + u * blockDim.x;
                pu[u] = t % P;
                iu[u] = t / P;
                ok[u] = t < n * P && (!RAG || pu[u] < zv);
                const int z = z0 + pu[u];
                ipu[u] = cell(k, x, iu[u], z);
                slab[u] = ok[u] && in_slab(iu[u], ny, pml) && xin && iu[u] < ny - 1 && z < k.nz - 1;
                isu[u] = slab[u] ? slab_y(k, x, iu[u], z) : 0;
                r2[u] = ok[u] ? R2[ipu[u]] : 0.f;
                p7[u] = slab[u] ? f7[isu[u]] : 0.f;
            }
#pragma unroll
            for (int u = 0; u < kEpi; ++u) {
                if (!ok[u]) continue;
                const int i = iu[u], ip = ipu[u];
                const float dz = D[i * P + pu[u]];
                float rz = r2[u] + dz;
                if (slab[u]) {
                    const float q7 = p7[u] + dt * (-k.ay[i] * p7[u] - k.by[i] * dz);
                    rz += q7;
                    f7[isu[u]] = q7;
                }
                R2[ip] = rz;
            }
        }
    }
}

// ------------------------------------------------------------------ k_vx --
// x-derivatives of sxx (-, vx), sxy (+, vy), sxz (+, vz); C-PML x terms and
// the velocity update (cuda_kernel_calculate_v, cu:1018-1101); same
// park-then-epilogue structure as k_vy.
template <int N, bool RAG>
__global__ void __launch_bounds__(kThreads) k_vx(KP k, int P_rt)
{
    const int P = N > 0 ? 16 : P_rt;
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    const int n = N > 0 ? N : k.nx, nx = n, pml = k.pml;
    float2* tw = sm;
    float2* tF = tw + n;   // forward shift; the backward one is (-F.x, F.y)
    float2* A = tF + n;
    float2* B = A + (n + n / 16) * P;
    load_table(tw, k.tw_x, n);
    load_table(tF, k.Fx, n);
    __syncthreads();
    const int y = blockIdx.y, z0 = blockIdx.x * P;
    const int zv = RAG ? min(P, k.nz - z0) : P;  // rows of the tile inside the grid (even)
    const float dt = k.dt, inv_n = 1.0f / n;
    const bool yin = y < k.ny - 1;
    const float* __restrict__ sxx = k.s[0];
    const float* __restrict__ sxy = k.s[3];
    const float* __restrict__ sxz = k.s[4];
    float* __restrict__ v0 = k.v[0];
    float* __restrict__ v1 = k.v[1];
    float* __restrict__ v2 = k.v[2];
    const float* __restrict__ R0 = k.R[0];
    const float* __restrict__ R1 = k.R[1];
    const float* __restrict__ R2 = k.R[2];
    const float* __restrict__ ri0 = k.rinv[0];
    const float* __restrict__ ri1 = k.rinv[1];
    const float* __restrict__ ri2 = k.rinv[2];
    float* __restrict__ f0 = k.php[0];  // phi_pxx_x, averaged b_x
    float* __restrict__ f3 = k.php[3];  // phi_pxy_x, b_x
    float* __restrict__ f6 = k.php[6];  // phi_pxz_x, b_x

    // pass 1: sxx + i sxy -> dx- sxx (vx), dx+ sxy (vy)
    {
        float2* Zf = out_any<N, 16, kThreads, kPencil>(k.px, A, B);
        auto load = [&](int p, int i) -> float2 {
            if (RAG && p >= zv) return make_float2(0.f, 0.f);
            const int ip = cell(k, i, y, z0 + p);
            return make_float2(sxx[ip], sxy[ip]);
        };
        auto store = [&](int p, int i, float2 v) { Zf[i * P + p] = v; };
        fft_any<N, 16, kThreads, kPencil, false>(k.px, tw, A, B, P, 1, P, load, store);
        float2* X1 = Zf == A ? B : A;
        float* D = reinterpret_cast<float*>(out_any<N, 16, kThreads, kPencil>(k.px, X1, Zf));  // [2][n][P]
        auto load_i = [&](int p, int i) -> float2 {
            const int im = i ? n - i : 0;
            return two_shift(Zf[i * P + p], cconj(Zf[im * P + p]), cscale(tF[i], inv_n), -1.0f);
        };
        auto store_i = [&](int p, int i, float2 v) {
            D[i * P + p] = v.x;
            D[(n + i) * P + p] = v.y;
        };
        fft_any<N, 16, kThreads, kPencil, true>(k.px, tw, X1, Zf, P, 1, P, load_i, store_i);
        for (int t0 = threadIdx.x; t0 < n * P; t0 += kEpi * blockDim.x) {
            int ipu[kEpi], iu[kEpi], pu[kEpi], isu[kEpi];
            bool ok[kEpi], slab[kEpi];
            float a0[kEpi], a1[kEpi], r0[kEpi], r1[kEpi], w0[kEpi], w1[kEpi], p0[kEpi], p3[kEpi];
#pragma unroll
            for (int u = 0; u < kEpi; ++u) {
                const int t = t0 + u * blockDim.x;
                pu[u] = t % P;
                iu[u] = t / P;
                const int z = z0 + pu[u];
                ok[u] = t < n * P && iu[u] < nx - 1 && yin && z < k.nz - 1;
                ipu[u] = cell(k, iu[u], y, z);
                slab[u] = ok[u] && in_slab(iu[u], nx, pml);
                isu[u] = slab[u] ? slab_x(k, iu[u], y, z) : 0;
                const int ip = ipu[u];
                a0[u] = ok[u] ? v0[ip] : 0.f;
                a1[u] = ok[u] ? v1[ip] : 0.f;
                r0[u] = ok[u] ? R0[ip] : 0.f;
                r1[u] = ok[u] ? R1[ip] : 0.f;
                w0[u] = ok[u] ? ri0[ip] : 0.f;
                w1[u] = ok[u] ? ri1[ip] : 0.f;
                p0[u] = slab[u] ? f0[isu[u]] : 0.f;
                p3[u] = slab[u] ? f3[isu[u]] : 0.f;
            }
#pragma unroll
            for (int u = 0; u < kEpi; ++u) {
                if (!ok[u]) continue;
                const int i = iu[u], p = pu[u], ip = ipu[u];
                float px = D[i * P + p], py = D[(n + i) * P + p];
                if (slab[u]) {
                    const float q0 = p0[u] + dt * (-k.axh[i] * p0[u] - k.bxh[i] * px);
                    const float q3 = p3[u] + dt * (-k.ax[i] * p3[u] - k.bx[i] * py);
                    px += q0;
                    py += q3;
                    f0[isu[u]] = q0;
                    f3[isu[u]] = q3;
                }
                v0[ip] = a0[u] + dt * w0[u] * (px + r0[u]);
                v1[ip] = a1[u] + dt * w1[u] * (py + r1[u]);
            }
        }
        __syncthreads();
    }
    // pass 2: sxz pencils (2q, 2q+1) -> dx+ sxz (vz)
    {
        const int Qp = P / 2;
        float2* Zf = out_any<N, 8, kThreads, kPencil>(k.px, A, B);
        auto load = [&](int q, int i) -> float2 {
            if (RAG && 2 * q >= zv) return make_float2(0.f, 0.f);
            const int ip = cell(k, i, y, z0 + 2 * q);
            return *reinterpret_cast<const float2*>(sxz + ip);
        };
        auto store = [&](int q, int i, float2 v) { Zf[i * Qp + q] = v; };
        fft_any<N, 8, kThreads, kPencil, false>(k.px, tw, A, B, Qp, 1, Qp, load, store);
        float2* X1 = Zf == A ? B : A;
        float* D = reinterpret_cast<float*>(out_any<N, 8, kThreads, kPencil>(k.px, X1, Zf));  // [n][P]
        auto load_i = [&](int q, int i) -> float2 { return cmul(Zf[i * Qp + q], cscale(tF[i], inv_n)); };
        auto store_i = [&](int q, int i, float2 v) {
            D[i * P + 2 * q] = v.x;
            D[i * P + 2 * q + 1] = v.y;
        };
        fft_any<N, 8, kThreads, kPencil, true>(k.px, tw, X1, Zf, Qp, 1, Qp, load_i, store_i);
        for (int t0 = threadIdx.x; t0 < n * P; t0 += kEpi * blockDim.x) {
            int ipu[kEpi], iu[kEpi], pu[kEpi], isu[kEpi];
            bool ok[kEpi], slab[kEpi];
            float a2[kEpi], r2[kEpi], w2[kEpi], p6[kEpi];
#pragma unroll
            for (int u = 0; u < kEpi; ++u) {
                const int t = t0 + u * blockDim.x;
                pu[u] = t % P;
                iu[u] = t / P;
                const int z = z0 + pu[u];
                ok[u] = t < n * P && iu[u] < nx - 1 && yin && z < k.nz - 1;
                ipu[u] = cell(k, iu[u], y, z);
                slab[u] = ok[u] && in_slab(iu[u], nx, pml);
                isu[u] = slab[u] ? slab_x(k, iu[u], y, z) : 0;
                a2[u] = ok[u] ? v2[ipu[u]] : 0.f;
                r2[u] = ok[u] ? R2[ipu[u]] : 0.f;
                w2[u] = ok[u] ? ri2[ipu[u]] : 0.f;
                p6[u] = slab[u] ? f6[isu[u]] : 0.f;
            }
#pragma unroll
            for (int u = 0; u < kEpi; ++u) {
                if (!ok[u]) continue;
                const int i = iu[u], ip = ipu[u];
                float pz = D[i * P + pu[u]];
                if (slab[u]) {
                    const float q6 = p6[u] + dt * (-k.ax[i] * p6[u] - k.bx[i] * pz);
                    pz += q6;
                    f6[isu[u]] = q6;
                }
                v2[ip] = a2[u] + dt * w2[u] * (pz + r2[u]);
            }
        }
    }
}

// ----------------------------------------------------------------- k_rec --
// Receivers (cu:782-791).  With traces to inject (back-propagation of
// recorded data, the adjoint of recording), sample nt - 1 - it of each
// component is first added to that component at the receiver, at the point
// of the step where the source is injected and the records are taken.
__global__ void k_rec(KP k)
{
    const int ir = blockIdx.x * blockDim.x + threadIdx.x;
    const int it = *k.d_it;
    if (ir >= k.rn || it < 0 || it >= k.nt_rec) return;
    const int ip = cell(k, k.r_ix[ir], k.r_iy[ir], k.r_iz);
    if (it < k.inj_nt) {
        const long long o = (long long)(k.inj_nt - 1 - it) * k.rn + ir;
        for (int c = 0; c < 3; ++c)
            if (k.inj[c]) k.v[c][ip] += k.inj[c][o];
    }
    const long long o = (long long)it * k.rn + ir;
    if (k.rec[0]) {
        k.rec[0][o] = k.v[0][ip];
        k.rec[1][o] = k.v[1][ip];
        k.rec[2][o] = k.v[2][ip];
    }
}

// ----------------------------------------------------- setup, FP64 kernels --
// Constant-Q sets (cuviscoelas_3D.cu:195-205) per modulus, FP64:
// c = v cos(pi g / 2); eta1 = -rho c g w0, eta2 = rho c^2, eta3 = rho c^3 g / w0,
// tau1 = rho c g pi, tau2 = rho c^2 g^2 pi / w0 (pi = 3.1415926, cu:15).
__device__ __forceinline__ void qset(double v, double g, double r, double w0, double o[5])
{
    const double pi = 3.1415926;
    const double c = v * cos(g * pi / 2.0);
    o[0] = -r * c * g * w0;
    o[1] = r * c * c;
    o[2] = r * c * c * c * g / w0;
    o[3] = r * c * g * pi;
    o[4] = r * c * c * g * g * pi / w0;
}

// Per-cell coefficient build, FP64.  out[0..7): rho, gamma_p, gamma_s and the
// effective velocities c = v cos(pi gamma / 2) of c11, c33, c13 (gamma_p) and
// c44 (gamma_s); out[7..12): the S set of c44, input of the 8-point average.
// VTI (project extension): c33 = rho vp^2, c44 = c66 = rho vs^2,
// c11 = c33 (1 + 2 eps), c13 = sqrt((c33 - c44)(c33 (1 + 2 delta) - c44)) - c44,
// each modulus taking the constant-Q set of its effective velocity
// (v11 = vp sqrt(1 + 2 eps), v13 = sqrt((c13 + 2 c44)/rho)); the off-diagonal
// sets are P(v) - 2 S(vs), which at eps = delta = 0 is the reference's
// eta_p - 2 eta_s (cu:851-898).
__global__ void k_coef(long long ntp, const float* velp, const float* vels, const float* rho, const float* gp,
                       const float* gs, const float* eps, const float* delta, int vti, double w0, int lossless,
                       float* const* out)
{
    const double pi = 3.1415926;
    for (long long ip = blockIdx.x * (long long)blockDim.x + threadIdx.x; ip < ntp;
         ip += (long long)gridDim.x * blockDim.x) {
        // lossless medium: gamma = 0 (Q infinite), the constant-Q sets reduce
        // to the elastic moduli
        const double r = rho[ip], vp = velp[ip], vs = vels[ip], g_p = lossless ? 0.0 : gp[ip],
                     g_s = lossless ? 0.0 : gs[ip];
        const double cp = cos(g_p * pi / 2.0), cq = cos(g_s * pi / 2.0);
        double v11 = vp, v13 = vp;
        if (vti) {
            const double e = eps[ip], dl = delta[ip];
            const double c33 = r * vp * vp, c44 = r * vs * vs;
            const double c13 = sqrt((c33 - c44) * (c33 * (1.0 + 2.0 * dl) - c44)) - c44;
            v11 = vp * sqrt(1.0 + 2.0 * e);
            v13 = sqrt((c13 + 2.0 * c44) / r);
        }
        out[0][ip] = (float)r;
        out[1][ip] = (float)g_p;
        out[2][ip] = (float)g_s;
        out[3][ip] = (float)(v11 * cp);
        out[4][ip] = (float)(vp * cp);
        out[5][ip] = (float)(v13 * cp);
        out[6][ip] = (float)(vs * cq);
        double s5[5];
        qset(vs, g_s, r, w0, s5);
        for (int j = 0; j < 5; ++j) out[7 + j][ip] = (float)s5[j];
    }
}

// 8-point averaged shear set (cu:956-971) and 1/rho-bar (cu:1077-1092).
struct MuArgs {
    const float* s[5];
    float* mu[5];
    const float* rho;
    float* rinv[3];
};
__global__ void k_mu_rinv(KP k, MuArgs a)
{
    const long long A = (long long)k.ny * k.nz;
    for (long long ip = blockIdx.x * (long long)blockDim.x + threadIdx.x; ip < k.ntp;
         ip += (long long)gridDim.x * blockDim.x) {
        const int z = ip % k.nz, y = (ip / k.nz) % k.ny, x = ip / A;
        const bool in = x < k.nx - 1 && y < k.ny - 1 && z < k.nz - 1;
        for (int j = 0; j < 5; ++j) {
            const float* s = a.s[j];
            double m = 0.0;
            if (in)
                m = 0.125 * ((double)s[ip] + s[ip + 1] + s[ip + k.nz] + s[ip + 1 + k.nz] + s[ip + A] + s[ip + A + 1] +
                             s[ip + A + k.nz] + s[ip + A + 1 + k.nz]);
            a.mu[j][ip] = (float)m;
        }
        const double r0 = a.rho[ip];
        a.rinv[0][ip] = in ? (float)(1.0 / (0.5 * (r0 + a.rho[ip + A]))) : 0.f;
        a.rinv[1][ip] = in ? (float)(1.0 / (0.5 * (r0 + a.rho[ip + k.nz]))) : 0.f;
        a.rinv[2][ip] = in ? (float)(1.0 / (0.5 * (r0 + a.rho[ip + 1]))) : 0.f;
    }
}

// 1D derivative along one axis of a real field (tests / diagnostics): out =
// Re IFFT(T(k)/n * FFT(in)) along `axis`, T the forward or backward shift.
__global__ void k_deriv1d(KP k, int axis, int fwd, const float* in, float* out, int P)
{
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    const FftPlan& pl = axis == 0 ? k.px : axis == 1 ? k.py : k.pz;
    const int n = pl.n;
    const float2* T = axis == 0 ? (fwd ? k.Fx : k.Bx) : axis == 1 ? (fwd ? k.Fy : k.By) : (fwd ? k.Fz : k.Bz);
    const float2* gtw = axis == 0 ? k.tw_x : axis == 1 ? k.tw_y : k.tw_z;
    float2* tw = sm;
    float2* A = tw + n;
    float2* B = A + n * P;
    load_table(tw, gtw, n);
    __syncthreads();
    // pencils: P/2 complex pairs; pencil index pp over the other two axes
    const int Qp = P / 2;
    const long long npen = k.ntp / n;
    const long long pen0 = (long long)blockIdx.x * P;
    auto addr = [&](long long pen, int i) -> long long {
        if (axis == 2) return pen * n + i;
        if (axis == 1) { const long long x = pen / k.nz, z = pen % k.nz; return (x * k.ny + i) * k.nz + z; }
        return (long long)i * k.ny * k.nz + pen;
    };
    float2* Zf = fft_out_buf(pl, A, B);
    auto load = [&](int q, int i) -> float2 {
        const long long p0 = pen0 + 2 * q, p1 = p0 + 1;
        return make_float2(p0 < npen ? in[addr(p0, i)] : 0.f, p1 < npen ? in[addr(p1, i)] : 0.f);
    };
    auto store = [&](int q, int i, float2 v) { Zf[i * Qp + q] = v; };
    fft_run<true>(pl, tw, A, B, Qp, 1, Qp, false, load, store);
    float2* X1 = Zf == A ? B : A;
    const float inv_n = 1.0f / n;
    auto load_i = [&](int q, int i) -> float2 { return cmul(Zf[i * Qp + q], cscale(T[i], inv_n)); };
    auto store_i = [&](int q, int i, float2 v) {
        const long long p0 = pen0 + 2 * q, p1 = p0 + 1;
        if (p0 < npen) out[addr(p0, i)] = v.x;
        if (p1 < npen) out[addr(p1, i)] = v.y;
    };
    fft_run<true>(pl, tw, X1, Zf, Qp, 1, Qp, true, load_i, store_i);
}

// ------------------------------------------- single-field constant-Q field --
// One of the 27 stress-side fields on its own: out = Re IFFT3(|k|^pw T(k_a)
// FFT3(in)) / ntp with T the forward or backward staggered shift along axis
// a (cu:475-744 with the transforms around them).  The half spectrum H[0]
// (kz-major, as in the step) is the scratch; k_fz and k_cy do the z and y
// passes, these two kernels the k-space x pass and the C2R along z.
__global__ void __launch_bounds__(kThreads) kq_mx(KP k, int P, int axis, int fwd, int pw)
{
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    const int n = k.nx;
    float2* tw = sm;
    float2* V = tw + n;   // [n][P]
    float2* A = V + n * P;
    float2* B = A + (n + n / 16) * P;
    load_table(tw, k.tw_x, n);
    __syncthreads();
    const int kz = blockIdx.y, y0 = blockIdx.x * P;
    float2* H = k.H[0];
    auto load = [&](int p, int i) -> float2 { return H[spec(k, kz, i, y0 + p)]; };
    auto store = [&](int p, int i, float2 v) { V[i * P + p] = v; };
    fft_run<true>(k.px, tw, A, B, P, 1, P, false, load, store, 4);
    const float kz2 = k.kz[kz] * k.kz[kz];
    auto load_i = [&](int p, int i) -> float2 {
        const float kyv = k.ky[y0 + p], kxv = k.kx[i];
        const float k2 = fmaxf(kxv * kxv + kyv * kyv + kz2, 1e-10f);
        const float ap = pw == 0 ? 1.0f : (pw < 0 ? 1.0f / sqrtf(k2) : sqrtf(k2));
        float2 T;
        if (axis == 0) T = fwd ? k.Fx[i] : k.Bx[i];
        else if (axis == 1) T = fwd ? k.Fy[y0 + p] : k.By[y0 + p];
        else T = fwd ? k.Fz[kz] : k.Bz[kz];
        return cmul(V[i * P + p], cscale(T, ap * k.inv_ntp));
    };
    auto store_i = [&](int p, int i, float2 v) { H[spec(k, kz, i, y0 + p)] = v; };
    fft_run<true>(k.px, tw, A, B, P, 1, P, true, load_i, store_i, 4);
}

__global__ void __launch_bounds__(kThreads) kq_iz(KP k, int P, float* out)
{
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    const int n = k.nz, Qp = P / 2;
    float2* tw = sm;
    float2* A = tw + n;
    float2* B = A + Qp * (n + n / 16);
    load_table(tw, k.tw_z, n);
    __syncthreads();
    const int x = blockIdx.y, y0 = blockIdx.x * P;
    const float2* g = k.H[0];
    auto load = [&](int q, int i) -> float2 {
        const int kk = i <= n / 2 ? i : n - i;
        const float4 gg = *reinterpret_cast<const float4*>(g + spec(k, kk, x, y0 + 2 * q));
        float2 a = make_float2(gg.x, gg.y), b = make_float2(gg.z, gg.w);
        if (kk == 0 || 2 * kk == n) { a.y = 0.f; b.y = 0.f; }
        if (i > n / 2) { a.y = -a.y; b.y = -b.y; }
        return make_float2(a.x - b.y, a.y + b.x);
    };
    auto store = [&](int q, int i, float2 v) {
        out[cell(k, x, y0 + 2 * q, i)] = v.x;
        out[cell(k, x, y0 + 2 * q + 1, i)] = v.y;
    };
    fft_run<true>(k.pz, tw, A, B, Qp, 1, Qp, true, load, store, 4);
}

// --------------------------------------------------------- tile selection --
int tile_of(int n, int want)
{
    int p = want;
    while (p > 2 && n % p) p >>= 1;
    return p;
}

size_t smem_fz(const KP& k, int P) { return sizeof(float2) * (k.nz + 2 * (P / 2) * (k.nz + k.nz / 16)); }
size_t smem_cy(const KP& k, int L, bool ydv = false)
{
    return sizeof(float2) * (k.ny + 2 * L * (k.ny + k.ny / 16) + (ydv ? (size_t)L * k.ny : 0));
}
size_t smem_mx(const KP& k, int P)
{
    const int nbuf = k.px.nst > 2 ? 2 : 1;
    return sizeof(float2) * (3 * k.nx + k.nx * P + nbuf * (k.nx + k.nx / 16) * P + 2 * P) + sizeof(float) * (k.nx + P);
}
// k_sigma layout: tw[nz] | A | B (only when the z transform has more than two
// stages; otherwise B aliases S, used only by the final z-derivative pass) |
// S[9][P][nz+1] | D[3][P][nz+1] | z tables [4][nz] | y tables [4][P] | Fz, Bz.
// In place (compile-time lengths): tw | A | B (more than two stages) | D |
// tables; the real fields live in the buffer the last C2R stage reads.
// Two-stage lengths (nod) leave D out: the z pass parks its results in A.
// inplace: the compile-time path (sigma_inplace); nod: no z-pass stress buffer
size_t smem_sigma(const KP& k, int P, bool inplace, bool nod = false)
{
    const size_t bufA = (size_t)9 * (P / 2) * (k.nz + k.nz / 16);
    const int nb = k.pz.nst > 2 ? 2 : 1;
    const size_t sreal = inplace ? 0 : (size_t)9 * P * (k.nz + 1);
    const size_t dbuf = nod ? 0 : (size_t)3 * P * (k.nz + 1);
    return sizeof(float2) * (k.nz + nb * bufA + 2 * k.nz) + sizeof(float) * (sreal + dbuf + 4 * k.nz + 4 * P);
}

size_t smem_vyx(int n, int P) { return sizeof(float2) * (2 * n + 2 * (n + n / 16) * P); }

}  // namespace

// Transform lengths with a compile-time path (the even 5-smooth sizes the
// batching and serving workloads draw between 96 and 384, and 64 and 512); a
// kernel takes it when its transform length is listed and its tile fits the
// grid (see launch_step), otherwise the runtime path.
template <class F>
void dispatch_len(int n, F&& f)
{
    switch (n) {
        case 64: f(std::integral_constant<int, 64>{}); break;
        case 96: f(std::integral_constant<int, 96>{}); break;
        case 100: f(std::integral_constant<int, 100>{}); break;
        case 108: f(std::integral_constant<int, 108>{}); break;
        case 120: f(std::integral_constant<int, 120>{}); break;
        case 128: f(std::integral_constant<int, 128>{}); break;
        case 144: f(std::integral_constant<int, 144>{}); break;
        case 150: f(std::integral_constant<int, 150>{}); break;
        case 160: f(std::integral_constant<int, 160>{}); break;
        case 162: f(std::integral_constant<int, 162>{}); break;
        case 180: f(std::integral_constant<int, 180>{}); break;
        case 192: f(std::integral_constant<int, 192>{}); break;
        case 200: f(std::integral_constant<int, 200>{}); break;
        case 216: f(std::integral_constant<int, 216>{}); break;
        case 240: f(std::integral_constant<int, 240>{}); break;
        case 250: f(std::integral_constant<int, 250>{}); break;
        case 256: f(std::integral_constant<int, 256>{}); break;
        case 270: f(std::integral_constant<int, 270>{}); break;
        case 288: f(std::integral_constant<int, 288>{}); break;
        case 300: f(std::integral_constant<int, 300>{}); break;
        case 320: f(std::integral_constant<int, 320>{}); break;
        case 324: f(std::integral_constant<int, 324>{}); break;
        case 360: f(std::integral_constant<int, 360>{}); break;
        case 384: f(std::integral_constant<int, 384>{}); break;
        case 512: f(std::integral_constant<int, 512>{}); break;
        default: f(std::integral_constant<int, 0>{}); break;
    }
}
constexpr int kCtLengths[] = {0, 64, 96, 100, 108, 120, 128, 144, 150, 160, 162, 180, 192, 200, 216, 240, 250, 256, 270, 288, 300, 320, 324, 360, 384, 512};

namespace {

bool ct_length(int n)
{
    for (int c : kCtLengths)
        if (c > 0 && c == n) return true;
    return false;
}
int cdiv(int a, int b) { return (a + b - 1) / b; }

// Tiles of the step's launches.  A kernel whose transform length is compiled
// takes its full tile along the other axis, the last tile ragged (its rows
// or lines past the grid read as zeros and are not written); otherwise the
// runtime path takes the largest power-of-two divisor of the tiled axis up
// to the full tile.  A tile set in KP::tile_rt selects the runtime path with
// that tile.
struct StepTiles {
    int vy, vx, fz, cy, mx, sigma;
    bool rt[kNumTiled];  // runtime path, in the order above
};
StepTiles step_tiles(const KP& k)
{
    StepTiles t;
    auto tile = [&](int i, int len, int tiled, int want) {
        if (k.tile_rt[i] > 0) {
            t.rt[i] = true;
            return k.tile_rt[i];
        }
        t.rt[i] = !ct_length(len);
        return t.rt[i] ? tile_of(tiled, want) : want;
    };
    t.vy = tile(0, k.ny, k.nz, 16);
    t.vx = tile(1, k.nx, k.nz, 16);
    t.fz = tile(2, k.nz, k.ny, 16);
    t.cy = tile(3, k.ny, k.nx, 8);
    t.mx = tile(4, k.nx, k.ny, 16);
    t.sigma = tile(5, k.nz, k.ny, kSigmaRows);
    return t;
}

}  // namespace

int configure_kernels()
{
    const int big = (int)kMaxSmem;  // leaves room for the kernels' small static tables
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* f) {
        cudaError_t r = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        if (r != cudaSuccess) e = r;
    };
    for (int n : kCtLengths)
        dispatch_len(n, [&](auto NN) {
            constexpr int N = decltype(NN)::value;
            set((const void*)k_fz<N>);
            set((const void*)k_cy<N, false>);
            set((const void*)k_cy<N, true>);
            set((const void*)k_mx<N>);
            set((const void*)k_sigma<N, false>);
            if constexpr (N > 0) set((const void*)k_sigma<N, true>);

            set((const void*)k_vy<N, false>);
            set((const void*)k_vx<N, false>);
            if constexpr (N > 0) {
                set((const void*)k_vy<N, true>);
                set((const void*)k_vx<N, true>);
            }
        });
    set((const void*)k_deriv1d);
    set((const void*)kq_mx);
    set((const void*)kq_iz);
    const int et = configure_tc_kernels();
    if (et) e = (cudaError_t)et;
    return (int)e;
}

const char* const kStepKernelNames[kStepKernels] = {"k_vy",  "k_vx",     "k_fz",    "k_cy_fwd",
                                                     "k_mx",  "k_cy_inv", "k_sigma", "k_rec"};

// One time step.  With a profile sink, an event is recorded before the first
// kernel and after every launch, tagged with the launch's kernel index.
void launch_step(const KP& k, cudaStream_t st, StepProfile* prof)
{
    auto mark = [&](int kind) {
        if (prof && prof->n < StepProfile::kMax) {
            cudaEventRecord(prof->ev[prof->n], st);
            prof->kind[prof->n++] = kind;
        }
    };
    // the compile-time path of a kernel fixes its tile: 16 z rows (k_vy,
    // k_vx), 16 y rows (k_fz, k_mx), 8 lines (k_cy), kSigmaRows y rows
    const StepTiles T = step_tiles(k);
    auto len = [&](int i, int n) { return T.rt[i] ? 0 : n; };
    mark(-1);
    // the runtime path's tiles divide the grid; a compiled length may be
    // ragged (a separate instantiation carries the masks)
    dispatch_len(len(0, k.ny), [&](auto NN) {
        constexpr int N = decltype(NN)::value;
        const dim3 grid(cdiv(k.nz, T.vy), k.nx);
        const size_t sm = smem_vyx(k.ny, T.vy);
        if constexpr (N > 0) {
            if (k.nz % T.vy) {
                k_vy<N, true><<<grid, kThreads, sm, st>>>(k, T.vy);
                return;
            }
        }
        k_vy<N, false><<<grid, kThreads, sm, st>>>(k, T.vy);
    });
    mark(0);
    dispatch_len(len(1, k.nx), [&](auto NN) {
        constexpr int N = decltype(NN)::value;
        const dim3 grid(cdiv(k.nz, T.vx), k.ny);
        const size_t sm = smem_vyx(k.nx, T.vx);
        if constexpr (N > 0) {
            if (k.nz % T.vx) {
                k_vx<N, true><<<grid, kThreads, sm, st>>>(k, T.vx);
                return;
            }
        }
        k_vx<N, false><<<grid, kThreads, sm, st>>>(k, T.vx);
    });
    mark(1);
    dispatch_len(len(2, k.nz), [&](auto NN) {
        k_fz<decltype(NN)::value><<<dim3(cdiv(k.ny, T.fz), k.nx, 3), kThreads, smem_fz(k, T.fz), st>>>(k, T.fz);
    });
    mark(2);
    // k-space passes, optionally in batches of kz planes (KP::kz_batch).
    const int L = T.cy, Pm = T.mx;
    const int batch = k.kz_batch > 0 ? k.kz_batch : k.nkz;
    for (int kz0 = 0; kz0 < k.nkz; kz0 += batch) {
        const int nb = kz0 + batch <= k.nkz ? batch : k.nkz - kz0;
        const long long line0 = (long long)kz0 * k.nx, line_end = line0 + (long long)nb * k.nx;
        const int ncy = cdiv(nb * k.nx, L);
        const bool tc = k.form == kFormTc && tc_cy_available(k);
        if (tc) {
            launch_cy_tc(k, false, 3, line0, line_end, st);
        } else {
            dispatch_len(len(3, k.ny), [&](auto NN) {
                k_cy<decltype(NN)::value, false><<<dim3(ncy, 3), kCyThreads, smem_cy(k, L, true), st>>>(k, L, line0,
                                                                                                      line_end);
            });
        }
        mark(3);
        dispatch_len(len(4, k.nx), [&](auto NN) {
            k_mx<decltype(NN)::value><<<dim3(cdiv(k.ny, Pm), nb, 3), kThreads, smem_mx(k, Pm), st>>>(k, Pm, kz0);
        });
        mark(4);
        if (tc) {
            launch_cy_tc(k, true, kNumGxy, line0, line_end, st);
        } else {
            dispatch_len(len(3, k.ny), [&](auto NN) {
                k_cy<decltype(NN)::value, true><<<dim3(ncy, kNumGxy), kCyThreads, smem_cy(k, L), st>>>(k, L, line0,
                                                                                                     line_end);
            });
        }
        mark(5);
    }
    const int Ps = T.sigma;
    dispatch_len(len(5, k.nz), [&](auto NN) {
        constexpr int N = decltype(NN)::value;
        const dim3 grid(cdiv(k.ny, Ps), k.nx);
        const size_t sm = smem_sigma(k, Ps, sigma_inplace(N), sigma_nod_ok(N));
        // the runtime path's tile divides ny; a compiled length may be ragged
        if constexpr (N > 0) {
            if (k.ny % Ps) {
                k_sigma<N, true><<<grid, sigma_threads(N), sm, st>>>(k, Ps);
                return;
            }
        }
        k_sigma<N, false><<<grid, sigma_threads(N), sm, st>>>(k, Ps);
    });
    mark(6);
    if (k.rn > 0) {
        k_rec<<<(k.rn + 255) / 256, 256, 0, st>>>(k);
        mark(7);
    }
}

// Largest dynamic shared memory of the step's launches for this grid.
size_t step_smem_bytes(const KP& k)
{
    const StepTiles T = step_tiles(k);
    size_t m = smem_vyx(k.ny, T.vy);
    m = std::max(m, smem_vyx(k.nx, T.vx));
    m = std::max(m, smem_fz(k, T.fz));
    m = std::max(m, smem_cy(k, T.cy, true));
    m = std::max(m, smem_mx(k, T.mx));
    // the layout launch_step takes: in place and three groups on the
    // compile-time path, without the z pass's stress buffer at two stages
    m = std::max(m, smem_sigma(k, T.sigma, !T.rt[5], !T.rt[5] && k.pz.nst == 2));
    return m;
}

void step_tile_set(const KP& k, int tiles[kNumTiled], int runtime[kNumTiled])
{
    const StepTiles T = step_tiles(k);
    const int t[kNumTiled] = {T.vy, T.vx, T.fz, T.cy, T.mx, T.sigma};
    for (int i = 0; i < kNumTiled; ++i) {
        if (tiles) tiles[i] = t[i];
        if (runtime) runtime[i] = T.rt[i] ? 1 : 0;
    }
}

bool tiles_valid(const KP& k)
{
    // the axis each kernel tiles: z rows (k_vy, k_vx), y rows (k_fz, k_mx,
    // k_sigma); k_cy's lines need not divide anything (a batch's last tile
    // is partial)
    const int axis[kNumTiled] = {k.nz, k.nz, k.ny, 0, k.ny, k.ny};
    for (int i = 0; i < kNumTiled; ++i) {
        const int t = k.tile_rt[i];
        if (t == 0) continue;
        if (t < 2 || t > 32 || (t & 1) || (axis[i] && axis[i] % t)) return false;
    }
    return step_smem_bytes(k) <= kMaxSmem;
}

void launch_coef_build(const KP& k, const float* velp, const float* vels, const float* rho, const float* gp,
                       const float* gs, const float* eps, const float* delta, int vti, float w0, int lossless,
                       float* const* coef_out, cudaStream_t st)
{
    k_coef<<<148 * 8, 256, 0, st>>>(k.ntp, velp, vels, rho, gp, gs, eps, delta, vti, (double)w0, lossless, coef_out);
}

void launch_mu_rinv(const KP& k, const float* rho, const float* const* sset, cudaStream_t st)
{
    MuArgs a;
    for (int j = 0; j < 5; ++j) { a.s[j] = sset[j]; a.mu[j] = const_cast<float*>(k.MU[j]); }
    a.rho = rho;
    for (int c = 0; c < 3; ++c) a.rinv[c] = const_cast<float*>(k.rinv[c]);
    k_mu_rinv<<<148 * 8, 256, 0, st>>>(k, a);
}

// k.v[0] = input field, k.H[0] = k.G[0] = half-spectrum scratch (nkz*nx*ny).
void launch_q_derivative(const KP& k_in, int axis, int fwd, int pw, float* out, cudaStream_t st)
{
    KP k = k_in;
    k.Hy[0] = k.H[0];  // the forward y pass works in place on the one scratch spectrum
    for (int c = 0; c < 3; ++c) k.Yv[c] = nullptr;  // and writes no y derivative
    const int Pz = tile_of(k.ny, 16);
    k_fz<0><<<dim3(k.ny / Pz, k.nx, 1), kThreads, smem_fz(k, Pz), st>>>(k, Pz);
    const int L = tile_of(k.nx, 8);
    k_cy<0, false><<<dim3(k.nkz * k.nx / L, 1), kCyThreads, smem_cy(k, L), st>>>(k, L, 0, (long long)k.nkz * k.nx);
    const int Pm = tile_of(k.ny, 8);
    kq_mx<<<dim3(k.ny / Pm, k.nkz), kThreads, sizeof(float2) * (k.nx + k.nx * Pm + 2 * (k.nx + k.nx / 16) * Pm), st>>>(
        k, Pm, axis, fwd, pw);
    k_cy<0, true><<<dim3(k.nkz * k.nx / L, 1), kCyThreads, smem_cy(k, L), st>>>(k, L, 0, (long long)k.nkz * k.nx);
    const int Pi = tile_of(k.ny, 8);
    kq_iz<<<dim3(k.ny / Pi, k.nx), kThreads, sizeof(float2) * (k.nz + 2 * (Pi / 2) * (k.nz + k.nz / 16)), st>>>(k, Pi,
                                                                                                               out);
}

void launch_derivative_1d(const KP& k, int axis, int fwd, const float* in, float* out, cudaStream_t st)
{
    const int n = axis == 0 ? k.nx : axis == 1 ? k.ny : k.nz;
    const int P = 16;
    const long long npen = k.ntp / n;
    const unsigned nb = (unsigned)((npen + P - 1) / P);
    k_deriv1d<<<nb, kThreads, sizeof(float2) * (n + 2 * n * P), st>>>(k, axis, fwd, in, out, P);
}

}  // namespace qvti
