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
#include <cstdio>

#include "engine.cuh"

namespace qvti {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ long long cell(const KP& k, int x, int y, int z)
{
    return ((long long)x * k.ny + y) * k.nz + z;
}
__device__ __forceinline__ long long spec(const KP& k, int kz, int x, int y)
{
    return ((long long)kz * k.nx + x) * k.ny + y;
}
__device__ __forceinline__ bool in_slab(int i, int n, int pml) { return i < pml || i >= n - pml; }

__device__ __forceinline__ void load_table(float2* s, const float2* g, int n)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) s[i] = g[i];
}

// Derivative bookkeeping for the 9 stress-side derivatives d (G index
// o = 3 d + j): component, axis, forward(1)/backward(0) staggered shift.
// d: 0 dx vx, 1 dy vy, 2 dz vz (forward shift, kvx_x kvy_y kvz_z),
//    3 dz vx, 4 dx vz, 5 dy vx, 6 dx vy, 7 dz vy, 8 dy vz (backward shift)
// -- the table assignment of cuviscoelas_3D.cu:1342-1562.
__constant__ int c_comp[9] = {0, 1, 2, 0, 2, 0, 1, 1, 2};
__constant__ int c_axis[9] = {0, 1, 2, 2, 0, 1, 0, 2, 1};
__constant__ int c_fwd[9] = {1, 1, 1, 0, 0, 0, 0, 0, 0};

// ------------------------------------------------------------------ k_fz --
// R2C along z of vx, vy, vz.  Tile: one x, P consecutive y rows (P even);
// rows (2q, 2q+1) share one complex transform.  Output H[f][kz][x][y].
__global__ void __launch_bounds__(kThreads) k_fz(KP k, int P)
{
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    const int n = k.nz, Qp = P / 2, ps = n + 1;
    float2* tw = sm;
    float2* A = tw + n;
    float2* B = A + Qp * ps;
    load_table(tw, k.tw_z, n);
    __syncthreads();
    const int f = blockIdx.z, x = blockIdx.y, y0 = blockIdx.x * P;
    const float* src = k.v[f];
    float2* Z = fft_out_buf(k.pz, A, B);
    auto load = [&](int q, int i) -> float2 {
        const long long b = cell(k, x, y0 + 2 * q, i);
        return make_float2(src[b], src[b + n]);
    };
    auto store = [&](int q, int i, float2 v) { Z[q * ps + i] = v; };
    fft_run<false>(k.pz, tw, A, B, Qp, ps, 1, false, load, store);
    float2* H = k.H[f];
    for (int t = threadIdx.x; t < k.nkz * P; t += blockDim.x) {
        const int p = t % P, kz = t / P, q = p >> 1;
        const float2 z = Z[q * ps + kz];
        const float2 zm = cconj(Z[q * ps + (kz ? n - kz : 0)]);
        H[spec(k, kz, x, y0 + p)] = (p & 1) ? unpack_b(z, zm) : unpack_a(z, zm);
    }
}

// ------------------------------------------------------------------ k_cy --
// C2C along y, in place, on L contiguous y lines per block.  arr selects the
// field (H[0..2] forward or G[0..26] inverse).
template <bool INV>
__global__ void __launch_bounds__(kThreads) k_cy(KP k, int L)
{
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    const int n = k.ny, ps = n + 1;
    float2* tw = sm;
    float2* A = tw + n;
    float2* B = A + L * ps;
    load_table(tw, k.tw_y, n);
    __syncthreads();
    float2* arr = INV ? k.G[blockIdx.y] : k.H[blockIdx.y];
    float2* base = arr + (long long)blockIdx.x * L * n;
    auto load = [&](int p, int i) -> float2 { return base[(long long)p * n + i]; };
    auto store = [&](int p, int i, float2 v) { base[(long long)p * n + i] = v; };
    fft_run<false>(k.py, tw, A, B, L, ps, 1, INV, load, store);
}

// ------------------------------------------------------------------ k_mx --
// x-pencils of the (kz, y-chunk) tile in k-space.
__global__ void __launch_bounds__(kThreads) k_mx(KP k, int P)
{
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    const int n = k.nx;
    float2* tw = sm;
    float2* tFx = tw + n;
    float2* tBx = tFx + n;
    float2* V = tBx + n;            // [3][n][P]
    float2* A = V + 3 * n * P;
    float2* B = A + n * P;
    float* tkx = reinterpret_cast<float*>(B + n * P);
    load_table(tw, k.tw_x, n);
    load_table(tFx, k.Fx, n);
    load_table(tBx, k.Bx, n);
    for (int i = threadIdx.x; i < n; i += blockDim.x) tkx[i] = k.kx[i];
    __syncthreads();
    const int kz = blockIdx.y, y0 = blockIdx.x * P;

    for (int f = 0; f < 3; ++f) {
        const float2* H = k.H[f];
        float2* Vf = V + f * n * P;
        auto load = [&](int p, int i) -> float2 { return H[spec(k, kz, i, y0 + p)]; };
        auto store = [&](int p, int i, float2 v) { Vf[i * P + p] = v; };
        fft_run<true>(k.px, tw, A, B, P, 1, P, false, load, store);
    }

    const float kzv = k.kz[kz];
    const float kz2 = kzv * kzv;
    const float2 tFz = k.Fz[kz], tBz = k.Bz[kz];
    for (int o = 0; o < kNumG; ++o) {
        const int d = o / 3, j = o % 3;
        const int c = c_comp[d], ax = c_axis[d], fw = c_fwd[d];
        const float2* Vc = V + c * n * P;
        float2* G = k.G[o];
        auto load = [&](int p, int i) -> float2 {
            const float kyv = k.ky[y0 + p];
            const float kxv = tkx[i];
            float k2 = kxv * kxv + kyv * kyv + kz2;
            k2 = fmaxf(k2, 1e-10f);  // the reference sets |k|^2 = 1e-10 at DC (cu:74)
            const float ap = j == 1 ? 1.0f : (j == 0 ? 1.0f / sqrtf(k2) : sqrtf(k2));
            float2 T;
            if (ax == 0) T = fw ? tFx[i] : tBx[i];
            else if (ax == 1) T = fw ? k.Fy[y0 + p] : k.By[y0 + p];
            else T = fw ? tFz : tBz;
            return cmul(Vc[i * P + p], cscale(T, ap * k.inv_ntp));
        };
        auto store = [&](int p, int i, float2 v) { G[spec(k, kz, i, y0 + p)] = v; };
        fft_run<true>(k.px, tw, A, B, P, 1, P, true, load, store);
    }
}

// ------------------------------------------------------------------ k_iz --
// z-pencils: C2R of the group's derivative fields, stress update, source
// injection and the z derivative of the updated stress for the next velocity
// update.  GRP 0: sxx syy szz (G 0..8), 1: sxz (G 9..14), 2: sxy (G 15..20),
// 3: syz (G 21..26).
template <int GRP>
__global__ void __launch_bounds__(kThreads) k_iz(KP k, int P)
{
    constexpr int NF = GRP == 0 ? 9 : 6;
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    const int n = k.nz, Qp = P / 2, np1 = n + 1, nx = k.nx, ny = k.ny, pml = k.pml;
    float2* tw = sm;
    float2* A = tw + n;
    float2* B = A + Qp * np1;
    float* S = reinterpret_cast<float*>(B + Qp * np1);  // [NF][P][np1]
    load_table(tw, k.tw_z, n);
    __syncthreads();
    const int x = blockIdx.y, y0 = blockIdx.x * P;
    const int o0 = GRP == 0 ? 0 : 9 + (GRP - 1) * 6;
    const int it = *k.d_it;
    const float dt = k.dt, inv_dt = 1.0f / k.dt;

    // 1. C2R along z: pencils (2q, 2q+1) of the half spectra packed as A + iB.
    for (int f = 0; f < NF; ++f) {
        const float2* g = k.G[o0 + f];
        float* Sf = S + f * P * np1;
        auto load = [&](int q, int i) -> float2 {
            const int kk = i <= n / 2 ? i : n - i;
            const float4 gg = *reinterpret_cast<const float4*>(g + spec(k, kk, x, y0 + 2 * q));
            float2 a = make_float2(gg.x, gg.y), b = make_float2(gg.z, gg.w);
            if (kk == 0 || 2 * kk == n) { a.y = 0.f; b.y = 0.f; }
            if (i > n / 2) { a.y = -a.y; b.y = -b.y; }
            return make_float2(a.x - b.y, a.y + b.x);
        };
        auto store = [&](int q, int i, float2 v) {
            Sf[(2 * q) * np1 + i] = v.x;
            Sf[(2 * q + 1) * np1 + i] = v.y;
        };
        fft_run<true>(k.pz, tw, A, B, Qp, 1, Qp, true, load, store);
    }

    // 2. cell updates.  The updated stress that feeds the z derivative is
    //    parked in S[0] (each cell's S values are read by its own thread only).
    const long long src_ip = (k.s_ix >= 0) ? cell(k, k.s_ix, k.s_iy, k.s_iz) : -1;
    for (int t = threadIdx.x; t < P * n; t += blockDim.x) {
        const int p = t / n, z = t % n, y = y0 + p;
        const long long ip = cell(k, x, y, z);
        const bool upd = x < nx - 1 && y < ny - 1 && z < n - 1;
        auto sv = [&](int f) { return S[(f * P + p) * np1 + z]; };
        float out;
        if constexpr (GRP == 0) {
            float sxx = k.s[0][ip], syy = k.s[1][ip], szz = k.s[2][ip];
            if (upd) {
                float a11[5], a12[5], a13[5], a33[5];
#pragma unroll
                for (int j = 0; j < 5; ++j) {
                    a11[j] = k.K11[j][ip]; a12[j] = k.K12[j][ip];
                    a13[j] = k.K13[j][ip]; a33[j] = k.K33[j][ip];
                }
                const float X0 = sv(0), X1 = sv(1), X2 = sv(2);
                const float Y0 = sv(3), Y1 = sv(4), Y2 = sv(5);
                const float Z0 = sv(6), Z1 = sv(7), Z2 = sv(8);
#define QD(a, s0, s1, s2) (a[0] * s0 + a[1] * s1 + a[2] * s2)
#define QL(a, s0, s1) (a[3] * s0 + a[4] * s1)
                const float d11x = QD(a11, X0, X1, X2), d12x = QD(a12, X0, X1, X2), d13x = QD(a13, X0, X1, X2);
                const float d12y = QD(a12, Y0, Y1, Y2), d11y = QD(a11, Y0, Y1, Y2), d13y = QD(a13, Y0, Y1, Y2);
                const float d13z = QD(a13, Z0, Z1, Z2), d33z = QD(a33, Z0, Z1, Z2);
                const float q11x = QL(a11, X0, X1), q12x = QL(a12, X0, X1), q13x = QL(a13, X0, X1);
                const float q12y = QL(a12, Y0, Y1), q11y = QL(a11, Y0, Y1), q13y = QL(a13, Y0, Y1);
                const float q13z = QL(a13, Z0, Z1), q33z = QL(a33, Z0, Z1);
#undef QD
#undef QL
                const float Qxx = q11x + q12y + q13z, Qyy = q12x + q11y + q13z, Qzz = q13x + q13y + q33z;
                const float Lxx = (Qxx - k.Q[0][ip]) * inv_dt;
                const float Lyy = (Qyy - k.Q[1][ip]) * inv_dt;
                const float Lzz = (Qzz - k.Q[2][ip]) * inv_dt;
                k.Q[0][ip] = Qxx; k.Q[1][ip] = Qyy; k.Q[2][ip] = Qzz;
                float pxx = 0.f, pxy = 0.f, pxz = 0.f, pyx = 0.f, pyy = 0.f, pyz = 0.f, pzxy = 0.f, pzz = 0.f;
                auto mem = [&](int m, float dterm, float qterm, float a, float b) {
                    const float T = dterm + (qterm - k.qn[m][ip]) * inv_dt;
                    k.qn[m][ip] = qterm;
                    float ph = k.phn[m][ip];
                    ph = ph + dt * (-a * ph - b * T);
                    k.phn[m][ip] = ph;
                    return ph;
                };
                if (in_slab(x, nx, pml)) {
                    pxx = mem(0, d11x, q11x, k.ax[x], k.bx[x]);
                    pxy = mem(1, d12x, q12x, k.ax[x], k.bx[x]);
                    pxz = mem(2, d13x, q13x, k.ax[x], k.bx[x]);
                }
                if (in_slab(y, ny, pml)) {
                    pyx = mem(3, d12y, q12y, k.ay[y], k.by[y]);
                    pyy = mem(4, d11y, q11y, k.ay[y], k.by[y]);
                    pyz = mem(5, d13y, q13y, k.ay[y], k.by[y]);
                }
                if (in_slab(z, n, pml)) {
                    pzxy = mem(6, d13z, q13z, k.az[z], k.bz[z]);
                    pzz = mem(7, d33z, q33z, k.az[z], k.bz[z]);
                }
                sxx = sxx + dt * (d11x + d12y + d13z + Lxx + pxx + pyx + pzxy);
                syy = syy + dt * (d12x + d11y + d13z + Lyy + pxy + pyy + pzxy);
                szz = szz + dt * (d13x + d13y + d33z + Lzz + pxz + pyz + pzz);
            }
            if (ip == src_ip && it < k.nt_rec) {
                if (k.src_type == 1) {
                    const float w = k.rik[it];
                    sxx += w; syy += w; szz += w;
                } else {
                    k.v[0][ip] += k.rik[it];
                }
            }
            if (upd || ip == src_ip) { k.s[0][ip] = sxx; k.s[1][ip] = syy; k.s[2][ip] = szz; }
            out = szz;
        } else {
            constexpr int sidx = GRP == 1 ? 4 : GRP == 2 ? 3 : 5;  // sxz, sxy, syz in s[]
            float sig = k.s[sidx][ip];
            if (upd) {
                float mu[5];
#pragma unroll
                for (int j = 0; j < 5; ++j) mu[j] = k.MU[j][ip];
                const float A0 = sv(0), A1 = sv(1), A2 = sv(2), B0 = sv(3), B1 = sv(4), B2 = sv(5);
                const float dA = mu[0] * A0 + mu[1] * A1 + mu[2] * A2, qA = mu[3] * A0 + mu[4] * A1;
                const float dB = mu[0] * B0 + mu[1] * B1 + mu[2] * B2, qB = mu[3] * B0 + mu[4] * B1;
                const float Qs = qA + qB;
                const float L = (Qs - k.Q[sidx][ip]) * inv_dt;
                k.Q[sidx][ip] = Qs;
                // term A: GRP1 vx_z (z slab), GRP2 vx_y (y slab), GRP3 vy_z (z slab)
                // term B: GRP1 vz_x (x slab), GRP2 vy_x (x slab), GRP3 vz_y (y slab)
                const int mA = (GRP - 1) * 2, mB = mA + 1;
                auto mem = [&](int m, float dterm, float qterm, float a, float b) {
                    const float T = dterm + (qterm - k.qs[m][ip]) * inv_dt;
                    k.qs[m][ip] = qterm;
                    float ph = k.phs[m][ip];
                    ph = ph + dt * (-a * ph - b * T);
                    k.phs[m][ip] = ph;
                    return ph;
                };
                float phA = 0.f, phB = 0.f;
                if (GRP == 1) {
                    if (in_slab(z, n, pml)) phA = mem(mA, dA, qA, k.azh[z], k.bzh[z]);
                    if (in_slab(x, nx, pml)) phB = mem(mB, dB, qB, k.axh[x], k.bxh[x]);
                } else if (GRP == 2) {
                    if (in_slab(y, ny, pml)) phA = mem(mA, dA, qA, k.ayh[y], k.byh[y]);
                    if (in_slab(x, nx, pml)) phB = mem(mB, dB, qB, k.axh[x], k.bxh[x]);
                } else {
                    if (in_slab(z, n, pml)) phA = mem(mA, dA, qA, k.azh[z], k.bzh[z]);
                    if (in_slab(y, ny, pml)) phB = mem(mB, dB, qB, k.ayh[y], k.byh[y]);
                }
                sig = sig + dt * (dA + phA + dB + phB + L);
                k.s[sidx][ip] = sig;
            }
            out = sig;
        }
        S[p * np1 + z] = out;  // S[0][p][z]
    }
    if constexpr (GRP == 2) return;
    __syncthreads();

    // 3. z derivative of the updated stress: GRP0 dz- szz -> R_z, GRP1 dz+ sxz
    //    -> R_x, GRP3 dz+ syz -> R_y (cu:1279-1306 partz2, partz1, partz3).
    {
        const float2* T = GRP == 0 ? k.Bz : k.Fz;
        const int rc = GRP == 0 ? 2 : GRP == 1 ? 0 : 1;
        const int phm = GRP == 0 ? 8 : GRP == 1 ? 2 : 5;  // php: pzz_z, pxz_z, pyz_z
        const float inv_n = 1.0f / n;
        auto load = [&](int q, int i) -> float2 { return make_float2(S[(2 * q) * np1 + i], S[(2 * q + 1) * np1 + i]); };
        float2* Zf = fft_out_buf(k.pz, A, B);
        auto store_f = [&](int q, int i, float2 v) { Zf[q * np1 + i] = v; };
        fft_run<false>(k.pz, tw, A, B, Qp, np1, 1, false, load, store_f);
        float2* X1 = Zf == A ? B : A;
        auto load_i = [&](int q, int i) -> float2 { return cmul(Zf[q * np1 + i], cscale(T[i], inv_n)); };
        auto store_i = [&](int q, int i, float2 v) {
            const bool zin = i < n - 1 && x < nx - 1;
            const bool zslab = in_slab(i, n, pml);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int y = y0 + 2 * q + h;
                const long long ip = cell(k, x, y, i);
                const float part = h ? v.y : v.x;
                float r = part;
                if (zslab && zin && y < ny - 1) {
                    float ph = k.php[phm][ip];
                    const float a = GRP == 0 ? k.azh[i] : k.az[i];
                    const float b = GRP == 0 ? k.bzh[i] : k.bz[i];
                    ph = ph + dt * (-a * ph - b * part);
                    k.php[phm][ip] = ph;
                    r += ph;
                }
                k.R[rc][ip] = r;
            }
        };
        fft_run<false>(k.pz, tw, X1, Zf, Qp, np1, 1, true, load_i, store_i);
    }
}

// ------------------------------------------------------------------ k_vy --
// y-derivatives of sxy (+, -> vx), syy (-, -> vy), syz (+, -> vz) for one x
// and P consecutive z; C-PML y terms; accumulate into R.
__global__ void __launch_bounds__(kThreads) k_vy(KP k, int P)
{
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    const int n = k.ny, ny = k.ny, pml = k.pml;
    float2* tw = sm;
    float2* tF = tw + n;
    float2* tB = tF + n;
    float2* A = tB + n;
    float2* B = A + n * P;
    load_table(tw, k.tw_y, n);
    load_table(tF, k.Fy, n);
    load_table(tB, k.By, n);
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *k.d_it += 1;  // step counter
    __syncthreads();
    const int x = blockIdx.y, z0 = blockIdx.x * P;
    const float dt = k.dt, inv_n = 1.0f / n;
    const bool xin = x < k.nx - 1;
    const float* sxy = k.s[3];
    const float* syy = k.s[1];
    const float* syz = k.s[5];

    // pass 1: sxy + i syy
    {
        float2* Zf = fft_out_buf(k.py, A, B);
        auto load = [&](int p, int i) -> float2 {
            const long long ip = cell(k, x, i, z0 + p);
            return make_float2(sxy[ip], syy[ip]);
        };
        auto store = [&](int p, int i, float2 v) { Zf[i * P + p] = v; };
        fft_run<true>(k.py, tw, A, B, P, 1, P, false, load, store);
        float2* X1 = Zf == A ? B : A;
        auto load_i = [&](int p, int i) -> float2 {
            const int im = i ? n - i : 0;
            return two_multiplier(Zf[i * P + p], cconj(Zf[im * P + p]), cscale(tF[i], inv_n), cscale(tB[i], inv_n));
        };
        auto store_i = [&](int p, int i, float2 v) {
            const int z = z0 + p;
            const long long ip = cell(k, x, i, z);
            float rx = v.x, ry = v.y;
            if (in_slab(i, ny, pml) && xin && i < ny - 1 && z < k.nz - 1) {
                float ph = k.php[1][ip];  // phi_pxy_y, b_y
                ph = ph + dt * (-k.ay[i] * ph - k.by[i] * v.x);
                k.php[1][ip] = ph;
                rx += ph;
                float qh = k.php[4][ip];  // phi_pyy_y, averaged b_y
                qh = qh + dt * (-k.ayh[i] * qh - k.byh[i] * v.y);
                k.php[4][ip] = qh;
                ry += qh;
            }
            k.R[0][ip] += rx;
            k.R[1][ip] += ry;
        };
        fft_run<true>(k.py, tw, X1, Zf, P, 1, P, true, load_i, store_i);
    }
    // pass 2: syz, pencils (2q, 2q+1)
    {
        const int Qp = P / 2;
        float2* Zf = fft_out_buf(k.py, A, B);
        auto load = [&](int q, int i) -> float2 {
            const long long ip = cell(k, x, i, z0 + 2 * q);
            return *reinterpret_cast<const float2*>(syz + ip);
        };
        auto store = [&](int q, int i, float2 v) { Zf[i * Qp + q] = v; };
        fft_run<true>(k.py, tw, A, B, Qp, 1, Qp, false, load, store);
        float2* X1 = Zf == A ? B : A;
        auto load_i = [&](int q, int i) -> float2 { return cmul(Zf[i * Qp + q], cscale(tF[i], inv_n)); };
        auto store_i = [&](int q, int i, float2 v) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int z = z0 + 2 * q + h;
                const long long ip = cell(k, x, i, z);
                const float part = h ? v.y : v.x;
                float r = part;
                if (in_slab(i, ny, pml) && xin && i < ny - 1 && z < k.nz - 1) {
                    float ph = k.php[7][ip];  // phi_pyz_y, b_y
                    ph = ph + dt * (-k.ay[i] * ph - k.by[i] * part);
                    k.php[7][ip] = ph;
                    r += ph;
                }
                k.R[2][ip] += r;
            }
        };
        fft_run<true>(k.py, tw, X1, Zf, Qp, 1, Qp, true, load_i, store_i);
    }
}

// ------------------------------------------------------------------ k_vx --
// x-derivatives of sxx (-, vx), sxy (+, vy), sxz (+, vz); C-PML x terms and
// the velocity update (cuda_kernel_calculate_v, cu:1018-1101).
__global__ void __launch_bounds__(kThreads) k_vx(KP k, int P)
{
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    const int n = k.nx, nx = k.nx, pml = k.pml;
    float2* tw = sm;
    float2* tF = tw + n;
    float2* tB = tF + n;
    float2* A = tB + n;
    float2* B = A + n * P;
    load_table(tw, k.tw_x, n);
    load_table(tF, k.Fx, n);
    load_table(tB, k.Bx, n);
    __syncthreads();
    const int y = blockIdx.y, z0 = blockIdx.x * P;
    const float dt = k.dt, inv_n = 1.0f / n;
    const bool yin = y < k.ny - 1;
    const float* sxx = k.s[0];
    const float* sxy = k.s[3];
    const float* sxz = k.s[4];

    // pass 1: sxx + i sxy -> vx, vy
    {
        float2* Zf = fft_out_buf(k.px, A, B);
        auto load = [&](int p, int i) -> float2 {
            const long long ip = cell(k, i, y, z0 + p);
            return make_float2(sxx[ip], sxy[ip]);
        };
        auto store = [&](int p, int i, float2 v) { Zf[i * P + p] = v; };
        fft_run<true>(k.px, tw, A, B, P, 1, P, false, load, store);
        float2* X1 = Zf == A ? B : A;
        auto load_i = [&](int p, int i) -> float2 {
            const int im = i ? n - i : 0;
            return two_multiplier(Zf[i * P + p], cconj(Zf[im * P + p]), cscale(tB[i], inv_n), cscale(tF[i], inv_n));
        };
        auto store_i = [&](int p, int i, float2 v) {
            const int z = z0 + p;
            if (!(i < nx - 1 && yin && z < k.nz - 1)) return;
            const long long ip = cell(k, i, y, z);
            float px = v.x, py = v.y;
            if (in_slab(i, nx, pml)) {
                float ph = k.php[0][ip];  // phi_pxx_x, averaged b_x
                ph = ph + dt * (-k.axh[i] * ph - k.bxh[i] * v.x);
                k.php[0][ip] = ph;
                px += ph;
                float qh = k.php[3][ip];  // phi_pxy_x, b_x
                qh = qh + dt * (-k.ax[i] * qh - k.bx[i] * v.y);
                k.php[3][ip] = qh;
                py += qh;
            }
            k.v[0][ip] += dt * k.rinv[0][ip] * (px + k.R[0][ip]);
            k.v[1][ip] += dt * k.rinv[1][ip] * (py + k.R[1][ip]);
        };
        fft_run<true>(k.px, tw, X1, Zf, P, 1, P, true, load_i, store_i);
    }
    // pass 2: sxz pencils (2q, 2q+1) -> vz
    {
        const int Qp = P / 2;
        float2* Zf = fft_out_buf(k.px, A, B);
        auto load = [&](int q, int i) -> float2 {
            const long long ip = cell(k, i, y, z0 + 2 * q);
            return *reinterpret_cast<const float2*>(sxz + ip);
        };
        auto store = [&](int q, int i, float2 v) { Zf[i * Qp + q] = v; };
        fft_run<true>(k.px, tw, A, B, Qp, 1, Qp, false, load, store);
        float2* X1 = Zf == A ? B : A;
        auto load_i = [&](int q, int i) -> float2 { return cmul(Zf[i * Qp + q], cscale(tF[i], inv_n)); };
        auto store_i = [&](int q, int i, float2 v) {
            if (!(i < nx - 1 && yin)) return;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int z = z0 + 2 * q + h;
                if (z >= k.nz - 1) continue;
                const long long ip = cell(k, i, y, z);
                float part = h ? v.y : v.x;
                if (in_slab(i, nx, pml)) {
                    float ph = k.php[6][ip];  // phi_pxz_x, b_x
                    ph = ph + dt * (-k.ax[i] * ph - k.bx[i] * part);
                    k.php[6][ip] = ph;
                    part += ph;
                }
                k.v[2][ip] += dt * k.rinv[2][ip] * (part + k.R[2][ip]);
            }
        };
        fft_run<true>(k.px, tw, X1, Zf, Qp, 1, Qp, true, load_i, store_i);
    }
}

// ----------------------------------------------------------------- k_rec --
__global__ void k_rec(KP k)
{
    const int ir = blockIdx.x * blockDim.x + threadIdx.x;
    const int it = *k.d_it;
    if (ir >= k.rn || it < 0 || it >= k.nt_rec) return;
    const long long ip = cell(k, k.r_ix[ir], k.r_iy[ir], k.r_iz);
    const long long o = (long long)it * k.rn + ir;
    k.rec[0][o] = k.v[0][ip];
    k.rec[1][o] = k.v[1][ip];
    k.rec[2][o] = k.v[2][ip];
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

// coef layout: [0..5) K11, [5..10) K12, [10..15) K13, [15..20) K33, [20..25) S.
__global__ void k_coef(long long ntp, const float* velp, const float* vels, const float* rho, const float* gp,
                       const float* gs, const float* eps, const float* delta, int vti, double w0, float* const* out)
{
    for (long long ip = blockIdx.x * (long long)blockDim.x + threadIdx.x; ip < ntp;
         ip += (long long)gridDim.x * blockDim.x) {
        const double r = rho[ip], vp = velp[ip], vs = vels[ip], g_p = gp[ip], g_s = gs[ip];
        double s5[5], p33[5], p11[5], p13[5];
        qset(vs, g_s, r, w0, s5);
        qset(vp, g_p, r, w0, p33);
        if (vti) {
            // VTI (project extension): c33 = rho vp^2, c44 = c66 = rho vs^2,
            // c11 = c33 (1 + 2 eps), c13 = sqrt((c33-c44)(c33(1+2 delta)-c44)) - c44;
            // each modulus gets the constant-Q set of its effective velocity.
            const double e = eps[ip], dl = delta[ip];
            const double c33 = r * vp * vp, c44 = r * vs * vs;
            const double c13 = sqrt((c33 - c44) * (c33 * (1.0 + 2.0 * dl) - c44)) - c44;
            qset(vp * sqrt(1.0 + 2.0 * e), g_p, r, w0, p11);
            qset(sqrt((c13 + 2.0 * c44) / r), g_p, r, w0, p13);
        } else {
            for (int j = 0; j < 5; ++j) { p11[j] = p33[j]; p13[j] = p33[j]; }
        }
        for (int j = 0; j < 5; ++j) {
            out[j][ip] = (float)p11[j];
            out[5 + j][ip] = (float)(p11[j] - 2.0 * s5[j]);
            out[10 + j][ip] = (float)(p13[j] - 2.0 * s5[j]);
            out[15 + j][ip] = (float)p33[j];
            out[20 + j][ip] = (float)s5[j];
        }
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

// --------------------------------------------------------- tile selection --
int tile_of(int n, int want)
{
    int p = want;
    while (p > 2 && n % p) p >>= 1;
    return p;
}

size_t smem_fz(const KP& k, int P) { return sizeof(float2) * (k.nz + 2 * (P / 2) * (k.nz + 1)); }
size_t smem_cy(const KP& k, int L) { return sizeof(float2) * (k.ny + 2 * L * (k.ny + 1)); }
size_t smem_mx(const KP& k, int P) { return sizeof(float2) * (3 * k.nx + 5 * k.nx * P) + sizeof(float) * k.nx; }
size_t smem_iz(const KP& k, int P, int nf)
{
    return sizeof(float2) * (k.nz + 2 * (P / 2) * (k.nz + 1)) + sizeof(float) * nf * P * (k.nz + 1);
}
size_t smem_vyx(int n, int P) { return sizeof(float2) * (3 * n + 2 * n * P); }

}  // namespace

int configure_kernels()
{
    const int big = 227 * 1024;
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* f) {
        cudaError_t r = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
        if (r != cudaSuccess) e = r;
    };
    set((const void*)k_fz);
    set((const void*)k_cy<false>);
    set((const void*)k_cy<true>);
    set((const void*)k_mx);
    set((const void*)k_iz<0>);
    set((const void*)k_iz<1>);
    set((const void*)k_iz<2>);
    set((const void*)k_iz<3>);
    set((const void*)k_vy);
    set((const void*)k_vx);
    set((const void*)k_deriv1d);
    return (int)e;
}

void launch_step(const KP& k, cudaStream_t st)
{
    const int Pv = tile_of(k.nz, 16);
    k_vy<<<dim3(k.nz / Pv, k.nx), kThreads, smem_vyx(k.ny, Pv), st>>>(k, Pv);
    k_vx<<<dim3(k.nz / Pv, k.ny), kThreads, smem_vyx(k.nx, Pv), st>>>(k, Pv);
    const int Pz = tile_of(k.ny, 16);
    k_fz<<<dim3(k.ny / Pz, k.nx, 3), kThreads, smem_fz(k, Pz), st>>>(k, Pz);
    const int L = tile_of(k.nkz * k.nx, 8) > 1 ? tile_of(k.nx, 8) : 1;
    k_cy<false><<<dim3(k.nkz * k.nx / L, 3), kThreads, smem_cy(k, L), st>>>(k, L);
    const int Pm = tile_of(k.ny, 8);
    k_mx<<<dim3(k.ny / Pm, k.nkz), kThreads, smem_mx(k, Pm), st>>>(k, Pm);
    k_cy<true><<<dim3(k.nkz * k.nx / L, kNumG), kThreads, smem_cy(k, L), st>>>(k, L);
    const int Pi = tile_of(k.ny, 8);
    k_iz<0><<<dim3(k.ny / Pi, k.nx), kThreads, smem_iz(k, Pi, 9), st>>>(k, Pi);
    k_iz<1><<<dim3(k.ny / Pi, k.nx), kThreads, smem_iz(k, Pi, 6), st>>>(k, Pi);
    k_iz<2><<<dim3(k.ny / Pi, k.nx), kThreads, smem_iz(k, Pi, 6), st>>>(k, Pi);
    k_iz<3><<<dim3(k.ny / Pi, k.nx), kThreads, smem_iz(k, Pi, 6), st>>>(k, Pi);
    if (k.rn > 0) k_rec<<<(k.rn + 255) / 256, 256, 0, st>>>(k);
}

void launch_coef_build(const KP& k, const float* velp, const float* vels, const float* rho, const float* gp,
                       const float* gs, const float* eps, const float* delta, int vti, float w0, float* const* coef_out,
                       cudaStream_t st)
{
    k_coef<<<148 * 8, 256, 0, st>>>(k.ntp, velp, vels, rho, gp, gs, eps, delta, vti, (double)w0, coef_out);
}

void launch_mu_rinv(const KP& k, const float* rho, const float* const* sset, cudaStream_t st)
{
    MuArgs a;
    for (int j = 0; j < 5; ++j) { a.s[j] = sset[j]; a.mu[j] = const_cast<float*>(k.MU[j]); }
    a.rho = rho;
    for (int c = 0; c < 3; ++c) a.rinv[c] = const_cast<float*>(k.rinv[c]);
    k_mu_rinv<<<148 * 8, 256, 0, st>>>(k, a);
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
