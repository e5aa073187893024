// Shared declarations of the B200 viscoelastic pseudospectral engine.
//
// Layout in HBM (one shot, total padded grid nx*ny*nz, z fastest exactly as
// the reference's ip = ix*nty*ntz + iy*ntz + iz, cuviscoelas_3D.cu:176):
//
//   state      v[3], s[6]  (vx vy vz; sxx syy szz sxy sxz syz)      float
//   R[3]       partial right-hand side of the velocity update: the z and y
//              stress derivatives (+ their C-PML memory terms), finished by
//              the x-pencil kernel                                   float
//   Q[6]       loss potentials: sum over terms of tau-coefficient x the
//              |k|^-1 and |k|^0 dispersion fields of the previous step; the
//              reference's spectral time derivative (V - Vprev)/dt
//              (cuviscoelas_3D.cu:514-531) becomes (Q - Qprev)/dt by
//              linearity, saving 18 of its 45 inverse transforms    float
//   C-PML      memory variables and per-term loss potentials, stored for
//              their axis slab only (they are identically zero elsewhere,
//              b = 0 there; see slab_x/slab_y/slab_z)               float
//   coef       rho, gamma_p, gamma_s and the effective velocities of c11,
//              c33, c13, c44 (7; 5 distinct when isotropic), MU (5, the
//              8-point averaged shear set), 1/rho-bar per velocity component;
//              built once per shot in FP64 and rounded              float
//   H[3]       velocity spectra, half along z: [kz][x][y], nkz = nz/2+1 float2
//   Hy[3]      the same, transformed along y too: [kz][x][ky]       float2
//   Yv[3]      dy vy, dy vx, dy vz with the identity dispersion operator,
//              written by the forward y pass: [kz][x][y]            float2
//   G[27]      9 directional derivatives x 3 dispersion operators
//              (|k|^-1, 1, |k|) of the velocity spectra, [kz][x][y]; the
//              six whose multiplier depends on kz or ky alone are not
//              stored: k_sigma forms them from H and Yv               float2
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "fft.cuh"
#include "per_device.h"

namespace qvti {

constexpr int kNumG = 27;
// G indices o = 3 d + j of the z and y derivatives with the identity
// dispersion operator (j = 1; d = 2 dz vz, 3 dz vx, 7 dz vy; d = 1 dy vy,
// 5 dy vx, 8 dy vz): their multiplier i k e^{+-i k h/2} depends on one
// wavenumber, so IFFT3(M FFT3(v)) needs only that axis' transform -- the z
// ones are formed from H in k_sigma, the y ones in the forward y pass, and
// neither goes through the x pass or the inverse y pass.
constexpr int kNumGxy = kNumG - 6;  // fields that go through k_mx and k_cy
__host__ __device__ constexpr bool is_gz(int o) { return o == 7 || o == 10 || o == 22; }
__host__ __device__ constexpr bool is_gy(int o) { return o == 4 || o == 16 || o == 25; }

struct KP {
    int nx, ny, nz, nkz, pml;
    long long ntp;
    float dt, inv_ntp;
    FftPlan px, py, pz;
    // 1D tables (device)
    const float2 *tw_x, *tw_y, *tw_z;             // e^{-2 pi i k/n}
    const float2 *Fx, *Bx, *Fy, *By, *Fz, *Bz;    // staggered-shift derivative multipliers (Nyquist bin real)
    const float *kx, *ky, *kz;                    // |k| per index
    const float *ax, *bx, *axh, *bxh;             // C-PML a, b and their half-point averages
    const float *ay, *by, *ayh, *byh;
    const float *az, *bz, *azh, *bzh;
    // state
    float* v[3];
    float* s[6];
    float* R[3];
    float* Q[6];
    float* php[9];   // velocity-side memory variables, reference order (cu:1049-1074)
    float* phn[8];   // normal-stress memory variables: x_xx x_xy x_xz y_yx y_yy y_yz z_zxy z_zz
    float* qn[8];    // matching per-term loss potentials
    float* phs[6];   // shear memory variables: vx_z vz_x vx_y vy_x vy_z vz_y
    float* qs[6];
    // coefficients (built in FP64 at setup): density, constant-Q exponents and
    // the effective velocities c = v cos(pi gamma / 2) of the moduli c11, c33,
    // c13 (P-type, gamma_p) and c44 = c66 (S-type, gamma_s); the eta/tau sets
    // are rebuilt from them on chip.  MU: 8-point averaged shear set; rinv:
    // 1/rho-bar of vx, vy, vz.
    const float *mrho, *mgp, *mgs, *mc11, *mc33, *mc13, *mcs;
    float w0;
    const float* MU[5];
    const float* rinv[3];
    // spectra
    float2* H[3];
    float2* Hy[3];
    float2* Yv[3];  // null: the forward y pass writes no y derivative
    float2* G[kNumG];
    // source and receivers
    int src_type, s_ix, s_iy, s_iz;
    const float* rik;
    int nt_rec, rn, r_iz;
    const int *r_ix, *r_iy;
    float* rec[3];
    int* d_it;       // current step index, advanced on the device each step
    int kz_batch;    // kz planes per batch of the k-space passes
    // form of the transforms: kFormPlain (FP32 butterflies) or kFormTc (the
    // 256-point y transforms as split-precision tensor-core contractions)
    int form;
    const float* dft16;  // tensor-core DFT matrices (k_dft16_tables), null if unused
    int* err;            // device error flag (a bounded wait that gave up), 0 = ok
    // medium: scale of the constant-Q loss terms (1 viscoelastic, 0
    // dispersion only or lossless, -1 Q-compensated back-propagation)
    float loss_scale;
    // time-reversed traces added at the receivers (nt_inj x rn each; null:
    // none), the adjoint source of back-propagation
    const float* inj[3];
    int inj_nt;
    // tile of each step kernel (k_vy, k_vx, k_fz, k_cy, k_mx, k_sigma):
    // 0 = the default (the compiled kernel's tile, or the runtime kernel's
    // where the length has no compiled kernel); > 0 = the runtime kernel
    // with this tile (qvti_set_tiles, checked by tiles_valid)
    int tile_rt[6];
};
constexpr int kFormPlain = 0, kFormTc = 1;
constexpr int kNumTiled = 6;

// C-PML memory variables are non-zero only inside their axis' slabs (b = 0
// elsewhere, cuviscoelas_3D.cu:291-307), so each is stored for the 2 pml
// planes of its axis only: x-slab [2 pml][ny][nz], y-slab [nx][2 pml][nz],
// z-slab [nx][ny][2 pml], the slab coordinate xs = x for x < pml and
// x - (nx - 2 pml) for x >= nx - pml.  Axis of each variable: php[m] m % 3
// (x, y, z); phn[m], qn[m]: m < 3 x, m < 6 y, else z; phs[m], qs[m]:
// {z, x, y, x, z, y}.
__device__ __forceinline__ int slab_x(const KP& k, int x, int y, int z)
{
    const int xs = x < k.pml ? x : x - k.nx + 2 * k.pml;
    return (xs * k.ny + y) * k.nz + z;
}
__device__ __forceinline__ int slab_y(const KP& k, int x, int y, int z)
{
    const int ys = y < k.pml ? y : y - k.ny + 2 * k.pml;
    return (x * 2 * k.pml + ys) * k.nz + z;
}
__device__ __forceinline__ int slab_z(const KP& k, int x, int y, int z)
{
    const int zs = z < k.pml ? z : z - k.nz + 2 * k.pml;
    return (x * k.ny + y) * 2 * k.pml + zs;
}
constexpr int kPhsAxis[6] = {2, 0, 1, 0, 2, 1};
// Floats in the slab of `axis` (0 x, 1 y, 2 z).
inline long long slab_len(int nx, int ny, int nz, int pml, int axis)
{
    const long long t = 2ll * pml;
    return axis == 0 ? t * ny * nz : axis == 1 ? (long long)nx * t * nz : (long long)nx * ny * t;
}

// Host-side launchers (step_kernels.cu).  All launch on `st`.
constexpr int kStepKernels = 8;
extern const char* const kStepKernelNames[kStepKernels];
struct StepProfile {
    static constexpr int kMax = 1024;
    cudaEvent_t ev[kMax];
    int kind[kMax];   // kernel index of the launch that ends at ev[i]; -1 = start
    int n = 0;
};
void launch_step(const KP& kp, cudaStream_t st, StepProfile* prof = nullptr);
// Largest dynamic shared memory (bytes) one of the step's launches needs.
size_t step_smem_bytes(const KP& kp);
// Tiles the step's launches take (tile_rt applied); runtime[i]: kernel i
// takes its runtime-length path.
void step_tile_set(const KP& kp, int tiles[kNumTiled], int runtime[kNumTiled]);
// Whether kp.tile_rt is a tiling the kernels support for this grid: every
// tile even, at most 32, dividing the axis it tiles (k_cy: any line
// count), and the step's shared memory within kMaxSmem.
bool tiles_valid(const KP& kp);
constexpr size_t kMaxSmem = 226 * 1024;  // dynamic; an SM block takes 227 KB with static
// coef_out: 7 model arrays (rho gp gs c11 c33 c13 cs) then the 5 S-set arrays
// (input of the MU average).
void launch_coef_build(const KP& kp, const float* velp, const float* vels, const float* rho,
                       const float* gp, const float* gs, const float* eps, const float* delta, int vti,
                       float w0, int lossless, float* const* coef_out, cudaStream_t st);
void launch_mu_rinv(const KP& kp, const float* rho, const float* const* sset, cudaStream_t st);
int configure_kernels();   // raise dynamic shared-memory limits, returns cudaError_t
// configure_kernels() once per device (the device must be current); 0 = ok.
int configure_device(int dev);
// Record `code` as the calling thread's last error (qvti_last_error) and
// return it.
int fail(int code);

// Radix plan of a transform length; FP64 build of one axis's 1D tables.
bool make_fft_plan(int n, FftPlan* p);
void launch_axis_tables(int n, double d, double f0, int pml, float2* tw, float* kmag, float2* F, float2* B,
                        float* a, float* b, float* ah, float* bh, cudaStream_t st);

// Tensor-core form (tc_dft.cu): 256-point y transforms on tcgen05.
bool tc_cy_available(const KP& k);
size_t tc_cy_smem();
int configure_tc_kernels();
void launch_dft16_tables(float* out, cudaStream_t st);  // 4096 floats
// A bounded wait that runs out after limit_cycles and records QVTI_ERR_TIMEOUT in *err.
void launch_wait_probe(int* err, long long limit_cycles, cudaStream_t st);
void launch_cy_tc(const KP& k, bool inv, int nfield, long long line0, long long line_end, cudaStream_t st);

// Individual stages, exposed for unit tests through the C ABI.
void launch_q_derivative(const KP& kp, int axis, int fwd, int pw, float* out, cudaStream_t st);
void launch_derivative_1d(const KP& kp, int axis, int fwd_shift, const float* in, float* out, cudaStream_t st);

}  // namespace qvti
