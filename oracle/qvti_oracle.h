/* FP64 CPU oracle for the 3D viscoelastic pseudospectral step.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py as the checker.  The product never links it.
 *
 * A line-by-line restatement, in double precision, of the reference's
 * cuviscoelas_3D.cu:22-1134 with the call order of its time loop
 * (cuviscoelas_3D.cu:1255-1630): 6 forward C2C FFTs of the stresses, 9
 * staggered derivatives for the velocity update, 3 forward FFTs of the
 * velocities, 45 constant-Q derivative fields (3 dispersion + 2 loss operators
 * for each of 9 directional derivatives), the stress update with C-PML memory
 * variables, source injection and receiver sampling.  Quirks are kept: the
 * real part of C2C output, unnormalised inverse with /ntp in the updates, the
 * last plane of every axis never updated, the 8-point averaged shear
 * coefficients, the backward-difference spectral time derivative with a zero
 * previous spectrum at step 0, velp_max forced to 5000 in the C-PML profile
 * and pi truncated to 3.1415926.
 *
 * Project extension (no reference counterpart): VTI media (Thomsen eps/delta,
 * c66 = c44) and an explosive source.  With eps = delta = 0 the VTI stiffness
 * sets reduce to the isotropic ones formula for formula.
 */
#ifndef QVTI_ORACLE_H
#define QVTI_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int ntx, nty, ntz, pml, nt;
    float dx, dy, dz, dt, f0;
    int vti;        /* 0 isotropic, 1 VTI (eps/delta used)                   */
    int src_type;   /* 0 point force on vx, 1 explosive on pxx/pyy/pzz       */
    int s_ix, s_iy, s_iz;   /* injection cell (padded indices, no offset)    */
    int r_iz, rn;   /* receiver depth index and receiver count               */
    int nthreads;   /* OpenMP threads, 0 = runtime default                   */
} qo_params;

/* Run one shot.  Records are [it][ir] (nt*rn floats each).  snaps receives
 * vx,vy,vz after each step listed in snap_steps (nsnap*3*ntp floats, the
 * state after k steps).  state_out (optional) receives the 9 final fields
 * vx,vy,vz,pxx,pyy,pzz,pxy,pxz,pyz in double.  Returns 0 on success. */
int qo_run(const qo_params* p, const float* rik,
           const float* velp, const float* vels, const float* rho,
           const float* gama_p, const float* gama_s,
           const float* eps, const float* delta,
           const int* r_ix, const int* r_iy,
           float* rec_vx, float* rec_vy, float* rec_vz,
           int nsnap, const int* snap_steps, float* snaps, double* state_out);

/* In-place unnormalised 3D C2C FFT of interleaved complex doubles laid out
 * [n0][n1][n2] (n2 fastest); sign -1 forward, +1 inverse. */
void qo_fft3d(int n0, int n1, int n2, double* data, int sign);

/* 1D staggered-shift derivative multipliers along one axis
 * (cuviscoelas_3D.cu:76-151): fwd = i k e^{+i k d/2}, bwd = i k e^{-i k d/2},
 * signed k with the Nyquist bin on the positive branch.  2n doubles each. */
void qo_shift_tables(int n, float d, double* fwd, double* bwd);

/* Non-negative wavenumber magnitudes (cuviscoelas_3D.cu:54-67). */
void qo_wavenumbers(int n, float d, double* k);

/* Constant-Q coefficients (cuviscoelas_3D.cu:195-205) for ncell cells:
 * out[0..5*ncell) = eta1, eta2, eta3, tau1, tau2 (each ncell long). */
void qo_q_coeffs(int ncell, const float* vel, const float* gam, const float* rho, float f0, double* out);

/* C-PML damping a(i), b(i) along one axis (cuviscoelas_3D.cu:213-309). */
void qo_pml_profile(int n, int pml, float d, float f0, double* a, double* b);

#ifdef __cplusplus
}
#endif
#endif
