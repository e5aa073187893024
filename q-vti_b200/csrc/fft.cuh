// Shared-memory mixed-radix FFT building blocks for sm_100a.
//
// The spectral-derivative engine replaces the reference's 63 cuFFT C2C calls
// per step (cuviscoelas_3D.cu:1272-1562) with pencil kernels that transform a
// tile of P pencils of one axis on chip.  A transform of length n = prod(rad)
// runs as a Stockham autosort sequence of radix-2/3/4/5/7/8/16 stages:
//
//   * stage 0 reads its inputs through a caller-supplied `load(p, i)` functor
//     (straight from global memory, or from shared memory with a k-space
//     multiplier applied on the fly),
//   * middle stages ping-pong between two shared-memory buffers,
//   * the last stage hands its outputs to a `store(p, i, v)` functor (to global
//     memory, or into an update epilogue).
//
// so a pencil costs one trip through HBM no matter how many stages it has.
// Element (p, i) of a pencil tile lives at buf[p*ps + i*is]; the thread
// mapping is pencil-fastest (PF) when pencils are contiguous in global memory
// and index-fastest otherwise, so both the global and the shared-memory
// accesses of every stage are coalesced / bank-spread.
//
// Convention: forward e^{-2 pi i k m / n}, inverse e^{+...}, unnormalised,
// matching cuFFT's CUFFT_FORWARD / CUFFT_INVERSE used by the reference.
#pragma once
#include <cuda_runtime.h>

namespace qvti {

constexpr int kMaxStages = 12;

struct FftPlan {
    int n;                   // transform length
    int nst;                 // number of stages (>= 2)
    int rad[kMaxStages];     // radix of each stage, first stage first
};

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b)  // a * conj(b)
{
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// multiply by -i (forward) or +i (inverse)
__device__ __forceinline__ float2 rot(float2 a, bool inv) { return inv ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x); }

// ---------------------------------------------------------------- radix DFTs
template <int R>
struct Dft;

template <>
struct Dft<2> {
    static __device__ __forceinline__ void run(float2* v, bool)
    {
        float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <>
struct Dft<4> {
    static __device__ __forceinline__ void run(float2* v, bool inv)
    {
        float2 s0 = cadd(v[0], v[2]), s1 = csub(v[0], v[2]);
        float2 s2 = cadd(v[1], v[3]), s3 = rot(csub(v[1], v[3]), inv);
        v[0] = cadd(s0, s2);
        v[2] = csub(s0, s2);
        v[1] = cadd(s1, s3);
        v[3] = csub(s1, s3);
    }
};

template <>
struct Dft<8> {
    static __device__ __forceinline__ void run(float2* v, bool inv)
    {
        const float c = 0.70710678118654752f;
        float2 e[4] = {v[0], v[2], v[4], v[6]};
        float2 o[4] = {v[1], v[3], v[5], v[7]};
        Dft<4>::run(e, inv);
        Dft<4>::run(o, inv);
        // o[k] *= W8^k  (W8 = e^{-i pi/4} forward, conjugate inverse)
        float2 t1 = inv ? make_float2(c * (o[1].x - o[1].y), c * (o[1].x + o[1].y))
                        : make_float2(c * (o[1].x + o[1].y), c * (o[1].y - o[1].x));
        float2 t2 = rot(o[2], inv);
        float2 t3 = inv ? make_float2(-c * (o[3].x + o[3].y), c * (o[3].x - o[3].y))
                        : make_float2(c * (o[3].y - o[3].x), -c * (o[3].x + o[3].y));
        v[0] = cadd(e[0], o[0]);
        v[4] = csub(e[0], o[0]);
        v[1] = cadd(e[1], t1);
        v[5] = csub(e[1], t1);
        v[2] = cadd(e[2], t2);
        v[6] = csub(e[2], t2);
        v[3] = cadd(e[3], t3);
        v[7] = csub(e[3], t3);
    }
};

// Odd radices: direct DFT with the roots of unity cos/sin(2 pi k / R).
template <int R>
struct OddRoots;
template <>
struct OddRoots<3> {
    static __device__ __forceinline__ float c(int k) { return k == 0 ? 1.f : -0.5f; }
    static __device__ __forceinline__ float s(int k) { return k == 0 ? 0.f : (k == 1 ? 0.866025404f : -0.866025404f); }
};
template <>
struct OddRoots<5> {
    static __device__ __forceinline__ float c(int k)
    {
        return k == 0 ? 1.f : (k == 1 || k == 4) ? 0.309016994f : -0.809016994f;
    }
    static __device__ __forceinline__ float s(int k)
    {
        return k == 0 ? 0.f : k == 1 ? 0.951056516f : k == 2 ? 0.587785252f : k == 3 ? -0.587785252f : -0.951056516f;
    }
};
template <>
struct OddRoots<7> {
    static __device__ __forceinline__ float c(int k)
    {
        return k == 0 ? 1.f : (k == 1 || k == 6) ? 0.623489802f : (k == 2 || k == 5) ? -0.222520934f : -0.900968868f;
    }
    static __device__ __forceinline__ float s(int k)
    {
        return k == 0 ? 0.f : k == 1 ? 0.781831482f : k == 2 ? 0.974927912f : k == 3 ? 0.433883739f
             : k == 4 ? -0.433883739f : k == 5 ? -0.974927912f : -0.781831482f;
    }
};

template <int R>
struct DftOdd {
    static __device__ __forceinline__ void run(float2* v, bool inv)
    {
        float2 out[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            float2 acc = v[0];
#pragma unroll
            for (int r = 1; r < R; ++r) {
                const int k = (q * r) % R;
                const float c = OddRoots<R>::c(k);
                const float s = inv ? OddRoots<R>::s(k) : -OddRoots<R>::s(k);
                acc.x += v[r].x * c - v[r].y * s;
                acc.y += v[r].x * s + v[r].y * c;
            }
            out[q] = acc;
        }
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = out[q];
    }
};
template <>
struct Dft<3> : DftOdd<3> {};
template <>
struct Dft<5> : DftOdd<5> {};
template <>
struct Dft<7> : DftOdd<7> {};

// Radix 16 in registers as 4 x 4: DFT-4 over n2 of v[n1 + 4 n2], twiddle
// W16^{n1 k2}, DFT-4 over n1; output X[k2 + 4 k1].
__device__ __forceinline__ float2 w16(float2 a, int e, bool inv)
{
    const float c1 = 0.923879533f, s1 = 0.382683432f, r = 0.707106781f;
    float c, s;
    switch (e & 15) {
        case 0: c = 1.f; s = 0.f; break;
        case 1: c = c1; s = s1; break;
        case 2: c = r; s = r; break;
        case 3: c = s1; s = c1; break;
        case 4: c = 0.f; s = 1.f; break;
        case 5: c = -s1; s = c1; break;
        case 6: c = -r; s = r; break;
        case 7: c = -c1; s = s1; break;
        case 8: c = -1.f; s = 0.f; break;
        case 9: c = -c1; s = -s1; break;
        case 10: c = -r; s = -r; break;
        case 11: c = -s1; s = -c1; break;
        case 12: c = 0.f; s = -1.f; break;
        case 13: c = s1; s = -c1; break;
        case 14: c = r; s = -r; break;
        default: c = c1; s = -s1; break;
    }
    // forward W16^e = cos - i sin, inverse its conjugate
    if (!inv) s = -s;
    return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
}

template <>
struct Dft<16> {
    static __device__ __forceinline__ void run(float2* v, bool inv)
    {
        float2 y[16];
#pragma unroll
        for (int n1 = 0; n1 < 4; ++n1) {
            float2 t[4] = {v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12]};
            Dft<4>::run(t, inv);
#pragma unroll
            for (int k2 = 0; k2 < 4; ++k2) y[n1 * 4 + k2] = (n1 && k2) ? w16(t[k2], n1 * k2, inv) : t[k2];
        }
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) {
            float2 t[4] = {y[k2], y[4 + k2], y[8 + k2], y[12 + k2]};
            Dft<4>::run(t, inv);
#pragma unroll
            for (int k1 = 0; k1 < 4; ++k1) v[k2 + 4 * k1] = t[k1];
        }
    }
};

// ------------------------------------------------------------------- stages
// Shared-memory address of element (p, i): p*ps + i*is, plus one extra `is`
// row every 2^padsh indices when padsh > 0 (breaks the bank conflicts of the
// radix-16 stage-0 writes in pencil-fastest tiles).
__device__ __forceinline__ int smem_at(int p, int i, int ps, int is, int padsh)
{
    return p * ps + i * is + (padsh ? (i >> padsh) * is : 0);
}

template <int R, bool PF, class Load, class Store>
__device__ __forceinline__ void fft_stage(int n, int P, int ps, int is, int padsh, int Ns, bool inv, bool first,
                                          bool last, const float2* __restrict__ tw, const float2* src, float2* dst,
                                          Load& load, Store& store)
{
    const int nr = n / R;
    const int total = P * nr;
    const int twstride = n / (Ns * R);
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int p, j;
        if (PF) { p = t % P; j = t / P; }
        else    { j = t % nr; p = t / nr; }
        const int jm = j % Ns;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int idx = j + r * nr;
            v[r] = first ? load(p, idx) : src[smem_at(p, idx, ps, is, padsh)];
        }
        if (jm) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                const float2 w = tw[jm * r * twstride];
                v[r] = inv ? cmulc(v[r], w) : cmul(v[r], w);
            }
        }
        Dft<R>::run(v, inv);
        const int base = (j - jm) * R + jm;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int idx = base + r * Ns;
            if (last) store(p, idx, v[r]);
            else dst[smem_at(p, idx, ps, is, padsh)] = v[r];
        }
    }
}

// Run a full transform of P pencils.  Stage 0 reads through `load`, writes
// bufA; stage s writes buf[s&1] (bufA, bufB alternating); the last stage
// writes through `store`.  Ends with __syncthreads().  Requires nst >= 2.
// Shared buffers must not alias anything `load` reads after stage 0.
template <bool PF, class Load, class Store>
__device__ void fft_run(const FftPlan& pl, const float2* __restrict__ tw, float2* bufA, float2* bufB,
                        int P, int ps, int is, bool inv, Load load, Store store, int padsh = 0)
{
    int Ns = 1;
    for (int s = 0; s < pl.nst; ++s) {
        const bool first = (s == 0), last = (s == pl.nst - 1);
        const float2* src = first ? nullptr : (((s - 1) & 1) ? bufB : bufA);
        float2* dst = (s & 1) ? bufB : bufA;
        switch (pl.rad[s]) {
            case 2: fft_stage<2, PF>(pl.n, P, ps, is, padsh, Ns, inv, first, last, tw, src, dst, load, store); break;
            case 3: fft_stage<3, PF>(pl.n, P, ps, is, padsh, Ns, inv, first, last, tw, src, dst, load, store); break;
            case 4: fft_stage<4, PF>(pl.n, P, ps, is, padsh, Ns, inv, first, last, tw, src, dst, load, store); break;
            case 5: fft_stage<5, PF>(pl.n, P, ps, is, padsh, Ns, inv, first, last, tw, src, dst, load, store); break;
            case 7: fft_stage<7, PF>(pl.n, P, ps, is, padsh, Ns, inv, first, last, tw, src, dst, load, store); break;
            case 16: fft_stage<16, PF>(pl.n, P, ps, is, padsh, Ns, inv, first, last, tw, src, dst, load, store); break;
            default: fft_stage<8, PF>(pl.n, P, ps, is, padsh, Ns, inv, first, last, tw, src, dst, load, store); break;
        }
        __syncthreads();
        Ns *= pl.rad[s];
    }
}

// Buffer that holds the output of fft_run when its store writes "the other"
// buffer of the pair (the one the last stage does not read).
__device__ __forceinline__ float2* fft_out_buf(const FftPlan& pl, float2* bufA, float2* bufB)
{
    return ((pl.nst - 1) & 1) ? bufB : bufA;
}

// Two real pencils a, b packed as z = a + i b and transformed together; this
// recovers A(k) and B(k) from Z(k) and Zc = conj(Z(n-k)).
__device__ __forceinline__ float2 unpack_a(float2 z, float2 zmc) { return make_float2(0.5f * (z.x + zmc.x), 0.5f * (z.y + zmc.y)); }
__device__ __forceinline__ float2 unpack_b(float2 z, float2 zmc)
{
    // (z - zmc) / (2i)
    return make_float2(0.5f * (z.y - zmc.y), -0.5f * (z.x - zmc.x));
}

// For z = a + i b transformed (a, b real), the spectrum of M1 a + i M2 b
// (M1, M2 Hermitian multipliers) is 1/2 [(M1+M2) Z(k) + (M1-M2) Zc] with
// Zc = conj(Z(n-k)).  For the staggered-shift pair of one axis, F = i k
// e^{+i k d/2} and B = i k e^{-i k d/2} satisfy B = (-F.x, F.y) exactly as
// tabulated (the Nyquist bin of both keeps only its real part), so
// (M1, M2) = (F, B) (sgn = 1) or (B, F) (sgn = -1) reduces it to
// i F.y Z + sgn F.x Zc.
__device__ __forceinline__ float2 two_shift(float2 z, float2 zmc, float2 f, float sgn)
{
    const float fx = sgn * f.x;
    return make_float2(fmaf(fx, zmc.x, -f.y * z.y), fmaf(fx, zmc.y, f.y * z.x));
}

}  // namespace qvti

namespace qvti {

// ------------------------------------------------- compile-time transforms --
// The same Stockham sequence with the length, the radix plan, the tile width
// and the block size known at compile time: every index division becomes a
// shift or a multiply, every stage loop has a fixed trip count.  Used for the
// common grid sizes; the runtime fft_run covers the rest.
__host__ __device__ constexpr int ct_nst(int n)
{
    if (n == 16) return 2;
    int m = n, s = 0;
    const int order[7] = {16, 8, 4, 2, 3, 5, 7};
    for (int oi = 0; oi < 7; ++oi)
        while (m % order[oi] == 0) { m /= order[oi]; ++s; }
    return s;
}
__host__ __device__ constexpr int ct_rad(int n, int stage)
{
    if (n == 16) return 4;
    int m = n, s = 0;
    const int order[7] = {16, 8, 4, 2, 3, 5, 7};
    for (int oi = 0; oi < 7; ++oi)
        while (m % order[oi] == 0) {
            if (s == stage) return order[oi];
            m /= order[oi];
            ++s;
        }
    return 1;
}
__host__ __device__ constexpr int ct_ns(int n, int stage)
{
    int p = 1;
    for (int s = 0; s < stage; ++s) p *= ct_rad(n, s);
    return p;
}

// Tile layouts in shared memory (element (p, i) of pencil p, index i):
//   kLine     p (N + 1) + i                  line-major
//   kPencil   p + (i + i/16) P               pencil-fastest, one pad row per 16
//   kLinePad  p (N + N/16) + i + i/16        line-major, one pad per 16
// The thread mapping follows the layout: pencil-fastest tiles put
// consecutive pencils on consecutive lanes (for data whose pencils are
// adjacent in memory), line-major ones consecutive indices (for data whose
// transform axis is contiguous: a half warp then reads 16 consecutive points
// of one line).  With radix-16 first and last stages both padded layouts are
// free of bank conflicts.
constexpr int kLine = 0, kPencil = 1, kLinePad = 2;

// PRETW (two-stage transforms only): stage 0 multiplies its outputs by the
// twiddles stage 1 would apply to them, so stage 1 starts its butterflies
// straight from shared memory.  The products are the same, on the same
// values; what changes is where they are computed: after stage 0's loads are
// consumed, instead of with 16 values and 15 twiddles live in stage 1 (which
// at 256 points spills under a 72-register cap).
// ROLL: a stage of several butterfly rounds per thread (small radices, many
// pencils) stays a loop instead of being unrolled, so the compiler does not
// hoist every round's loads at once; for a kernel already near its register
// cap that is the difference between spilling and not.
template <int N, int P, int NT, int LY, bool PRETW = false, bool ROLL = false>
struct FftCT {
    static constexpr bool PF = LY == kPencil;
    static constexpr int NST = ct_nst(N);
    static constexpr int BUF = LY == kLine ? P * (N + 1) : P * (N + N / 16);  // float2 per buffer

    static constexpr int PSTEP = LY == kPencil ? P : 1;  // distance of consecutive indices
    static_assert(!PRETW || NST == 2, "stage-1 twiddles move into stage 0 only for two-stage transforms");

    static __device__ __forceinline__ int at(int p, int i)
    {
        if constexpr (LY == kPencil) return p + (i + (i >> 4)) * P;
        else if constexpr (LY == kLinePad) return p * (N + N / 16) + i + (i >> 4);
        else return p * (N + 1) + i;
    }

    template <int S, bool INV, class Load, class Store>
    static __device__ __forceinline__ void stage(const float2* __restrict__ tw, float2* A, float2* B, Load& load,
                                                 Store& store)
    {
        constexpr int R = ct_rad(N, S), NS = ct_ns(N, S);
        constexpr bool FIRST = S == 0, LAST = S == NST - 1;
        constexpr int NR = N / R, TOTAL = P * NR, TWS = N / (NS * R);
        const float2* src = ((S - 1) & 1) ? B : A;
        float2* dst = (S & 1) ? B : A;
        constexpr int ITER = (TOTAL + NT - 1) / NT;
        constexpr int UNR = ROLL ? 1 : ITER;
#pragma unroll(UNR)
        for (int it = 0; it < ITER; ++it) {
            const int t = threadIdx.x + it * NT;
            if ((TOTAL % NT) != 0 && t >= TOTAL) break;
            int p, j;
            if (PF) { p = t % P; j = t / P; }
            else    { j = t % NR; p = t / NR; }
            const int jm = j % NS;
            float2 v[R];
            if constexpr (FIRST) {
#pragma unroll
                for (int r = 0; r < R; ++r) v[r] = load(p, j + r * NR);
            } else if constexpr (LY != kLine && NR % 16 == 0) {
                // idx = j + r NR: the pad row advances by NR/16 per r
                const int b = at(p, j);
#pragma unroll
                for (int r = 0; r < R; ++r) v[r] = src[b + r * (NR + NR / 16) * PSTEP];
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) v[r] = src[at(p, j + r * NR)];
            }
            if constexpr (!FIRST && !PRETW) {
                if (jm) {
#pragma unroll
                    for (int r = 1; r < R; ++r) {
                        const float2 w = tw[jm * r * TWS];
                        v[r] = INV ? cmulc(v[r], w) : cmul(v[r], w);
                    }
                }
            }
            Dft<R>::run(v, INV);
            if constexpr (PRETW && FIRST) {
                // two stages (NS = 1 here, R0 = NS of stage 1, TWS of stage 1
                // = 1): output r of butterfly j lands at index j R + r, which
                // stage 1 reads as its butterfly r, element j, with twiddle
                // w^(r j)
                if (j) {
#pragma unroll
                    for (int r = 1; r < R; ++r) {
                        const float2 w = tw[r * j];
                        v[r] = INV ? cmulc(v[r], w) : cmul(v[r], w);
                    }
                }
            }
            const int base = (j - jm) * R + jm;
            if constexpr (LAST) {
#pragma unroll
                for (int r = 0; r < R; ++r) store(p, base + r * NS, v[r]);
            } else if constexpr (LY != kLine && NS % 16 == 0) {
                // idx = base + r NS: the pad row advances by NS/16 per r
                const int b = at(p, base);
#pragma unroll
                for (int r = 0; r < R; ++r) dst[b + r * (NS + NS / 16) * PSTEP] = v[r];
            } else if constexpr (LY != kLine && 16 % (NS * R) == 0) {
                // the R outputs lie in one aligned run of NS R <= 16 indices
                // (base = m NS R + jm, jm < NS): one pad row for all of them
                const int b = at(p, base);
#pragma unroll
                for (int r = 0; r < R; ++r) dst[b + r * NS * PSTEP] = v[r];
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) dst[at(p, base + r * NS)] = v[r];
            }
        }
        __syncthreads();
        if constexpr (!LAST) stage<S + 1, INV>(tw, A, B, load, store);
    }

    // Stage 0 reads `load`, the last stage writes `store`; ends with
    // __syncthreads().  Buffers: A always, B when NST > 2.
    template <bool INV, class Load, class Store>
    static __device__ __forceinline__ void run(const float2* __restrict__ tw, float2* A, float2* B, Load load,
                                               Store store)
    {
        stage<0, INV>(tw, A, B, load, store);
    }

    // The buffer the last stage does not read.
    static __device__ __forceinline__ float2* out_buf(float2* A, float2* B) { return ((NST - 1) & 1) ? B : A; }
};

}  // namespace qvti
