/* FP64 CPU oracle -- see qvti_oracle.h.  TEST INFRASTRUCTURE ONLY.
 *
 * Every function cites the reference lines it restates (file:line within the
 * reference project).  Arrays are [ix][iy][iz], z fastest, as in the
 * reference (ip = ix*nty*ntz + iy*ntz + iz, cuviscoelas_3D.cu:176).
 */
#include "qvti_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI_REF 3.1415926 /* cuviscoelas_3D.cu:15, viscoelas_3D.cpp:14 */
#define TWO_PI 6.283185307179586476925286766559

/* ------------------------------------------------------------------ FFT --
 * Mixed-radix Stockham autosort FFT (any length; radix 4, 2, 3, 5 and a
 * direct DFT for other primes).  Plays the role of cuFFT's C2C transform
 * (cuviscoelas_3D.cu:1703-1704): unnormalised, forward e^{-i}, inverse e^{+i}. */

typedef struct { double re, im; } cplx;

typedef struct {
    int n, nf, f[40];
} plan1d;

static void plan_make(int n, plan1d* p)
{
    int m = n;
    p->n = n;
    p->nf = 0;
    while (m % 4 == 0) { p->f[p->nf++] = 4; m /= 4; }
    while (m % 2 == 0) { p->f[p->nf++] = 2; m /= 2; }
    for (int r = 3; m > 1; r += 2)
        while (m % r == 0) { p->f[p->nf++] = r; m /= r; }
}

/* One radix-R DFT of v[0..R) in place: v'[q] = sum_r v[r] e^{sign 2 pi i q r/R}. */
static void dft_small(int R, cplx* v, int sign, cplx* scratch)
{
    if (R == 2) {
        cplx a = v[0], b = v[1];
        v[0].re = a.re + b.re; v[0].im = a.im + b.im;
        v[1].re = a.re - b.re; v[1].im = a.im - b.im;
        return;
    }
    if (R == 4) {
        cplx a = v[0], b = v[1], c = v[2], d = v[3];
        cplx s0 = {a.re + c.re, a.im + c.im}, s1 = {a.re - c.re, a.im - c.im};
        cplx s2 = {b.re + d.re, b.im + d.im}, s3 = {b.re - d.re, b.im - d.im};
        /* multiply s3 by sign*i */
        cplx t3 = {-sign * s3.im, sign * s3.re};
        v[0].re = s0.re + s2.re; v[0].im = s0.im + s2.im;
        v[2].re = s0.re - s2.re; v[2].im = s0.im - s2.im;
        v[1].re = s1.re + t3.re; v[1].im = s1.im + t3.im;
        v[3].re = s1.re - t3.re; v[3].im = s1.im - t3.im;
        return;
    }
    for (int q = 0; q < R; ++q) {
        double sr = 0, si = 0;
        for (int r = 0; r < R; ++r) {
            double ang = sign * TWO_PI * (double)((long)q * r % R) / R;
            double c = cos(ang), s = sin(ang);
            sr += v[r].re * c - v[r].im * s;
            si += v[r].re * s + v[r].im * c;
        }
        scratch[q].re = sr;
        scratch[q].im = si;
    }
    memcpy(v, scratch, sizeof(cplx) * R);
}

/* Stockham autosort: x (length n) -> natural-order DFT in x; y is scratch. */
static void fft1d(const plan1d* p, cplx* x, cplx* y, int sign)
{
    int n = p->n, ns = 1;
    cplx *in = x, *out = y;
    cplx v[64], scr[64];
    for (int s = 0; s < p->nf; ++s) {
        int R = p->f[s];
        int nr = n / R;
        for (int j = 0; j < nr; ++j) {
            int jm = j % ns;
            double ang = sign * TWO_PI * jm / (double)(ns * R);
            for (int r = 0; r < R; ++r) {
                cplx a = in[j + r * nr];
                if (r && jm) {
                    double c = cos(ang * r), sn = sin(ang * r);
                    cplx b = {a.re * c - a.im * sn, a.re * sn + a.im * c};
                    a = b;
                }
                v[r] = a;
            }
            dft_small(R, v, sign, scr);
            int base = (j / ns) * ns * R + jm;
            for (int r = 0; r < R; ++r) out[base + r * ns] = v[r];
        }
        ns *= R;
        cplx* t = in; in = out; out = t;
    }
    if (in != x) memcpy(x, in, sizeof(cplx) * n);
}

/* transform every line along one axis of an [n0][n1][n2] complex array */
static void fft_axis(cplx* a, int n0, int n1, int n2, int axis, int sign)
{
    int n = axis == 0 ? n0 : axis == 1 ? n1 : n2;
    long stride = axis == 0 ? (long)n1 * n2 : axis == 1 ? n2 : 1;
    long nlines = (long)n0 * n1 * n2 / n;
    plan1d p;
    plan_make(n, &p);
#pragma omp parallel
    {
        cplx* buf = (cplx*)malloc(sizeof(cplx) * n);
        cplx* scr = (cplx*)malloc(sizeof(cplx) * n);
#pragma omp for schedule(static)
        for (long l = 0; l < nlines; ++l) {
            long base;
            if (axis == 2) base = l * n2;
            else if (axis == 1) base = (l / n2) * (long)n1 * n2 + (l % n2);
            else base = l;
            for (int i = 0; i < n; ++i) buf[i] = a[base + i * stride];
            fft1d(&p, buf, scr, sign);
            for (int i = 0; i < n; ++i) a[base + i * stride] = buf[i];
        }
        free(buf);
        free(scr);
    }
}

static void fft3(cplx* a, int n0, int n1, int n2, int sign)
{
    fft_axis(a, n0, n1, n2, 2, sign);
    fft_axis(a, n0, n1, n2, 1, sign);
    fft_axis(a, n0, n1, n2, 0, sign);
}

void qo_fft3d(int n0, int n1, int n2, double* data, int sign)
{
    fft3((cplx*)data, n0, n1, n2, sign);
}

/* ------------------------------------------------------- k-space tables -- */

/* cuviscoelas_3D.cu:54-67: |k| per index, Nyquist on the positive branch. */
void qo_wavenumbers(int n, float d, double* k)
{
    for (int i = 0; i < n; ++i) {
        int m = i <= n / 2 ? i : n - i;
        k[i] = 2.0 * PI_REF / n / d * m;
    }
}

/* cuviscoelas_3D.cu:76-151.  Forward tables (kvx_x, kvy_y, kvz_z) are
 * i k e^{+i k d/2}; backward tables (the other six) are i k e^{-i k d/2}. */
void qo_shift_tables(int n, float d, double* fwd, double* bwd)
{
    double dk = 1.0 / n / d;
    double tmp = 2.0 * PI_REF * dk;
    for (int i = 0; i < n; ++i) {
        if (i <= n / 2) {
            double s = sin(i * PI_REF / n), c = cos(i * PI_REF / n);
            fwd[2 * i] = -tmp * i * s;  fwd[2 * i + 1] = tmp * i * c;   /* :80-81 */
            bwd[2 * i] = tmp * i * s;   bwd[2 * i + 1] = tmp * i * c;   /* :83-84 */
        } else {
            int m = n - i;
            double s = sin(m * PI_REF / n), c = cos(m * PI_REF / n);
            fwd[2 * i] = -tmp * m * s;  fwd[2 * i + 1] = -tmp * m * c;  /* :93-94 */
            bwd[2 * i] = tmp * m * s;   bwd[2 * i + 1] = -tmp * m * c;  /* :96-97 */
        }
    }
}

/* cuviscoelas_3D.cu:195-205 with c = v cos(gamma pi/2). */
static void q_set(double v, double g, double r, double w0, double out[5])
{
    double c = v * cos(g * PI_REF / 2.0);
    out[0] = -r * c * g * w0;            /* eta1: multiplies |k|^-1 */
    out[1] = r * c * c;                  /* eta2: multiplies 1      */
    out[2] = r * c * c * c * g / w0;     /* eta3: multiplies |k|    */
    out[3] = r * c * g * PI_REF;         /* tau1: |k|^-1 on d/dt    */
    out[4] = r * c * c * g * g * PI_REF / w0; /* tau2: 1 on d/dt    */
}

static double w0_of(float f0)
{
    return (double)(float)(2 * PI_REF * f0); /* viscoelas_3D.cpp:109, a float */
}

void qo_q_coeffs(int ncell, const float* vel, const float* gam, const float* rho, float f0, double* out)
{
    double w0 = w0_of(f0);
    for (int i = 0; i < ncell; ++i) {
        double s[5];
        q_set(vel[i], gam[i], rho[i], w0, s);
        for (int j = 0; j < 5; ++j) out[(long)j * ncell + i] = s[j];
    }
}

/* cuviscoelas_3D.cu:213-309, gamma = 1, n1=2, n2=1, n3=2, R=1e-2, and
 * velp_max forced to 5000 (:235).  Interior: alpha = pi f0, Omega = 0. */
void qo_pml_profile(int n, int pml, float d, float f0, double* a, double* b)
{
    double alpha_max = PI_REF * (double)f0;
    double om_max = (1 + 2 + 1) * 5000.0 * log(1.0 / (double)1e-2f) / ((2 + 1 - 1) * pml * (double)d);
    for (int i = 0; i < n; ++i) { a[i] = alpha_max; b[i] = 0.0; }
    for (int i = 0; i < pml; ++i) {
        double al = alpha_max * pow((double)i / (pml - 1), 2);
        double om = om_max * pow((double)(pml - 1 - i) / pml, 3);
        a[i] = al + om; b[i] = om;
        a[n - 1 - i] = al + om; b[n - 1 - i] = om;
    }
}

/* ------------------------------------------------------------ the step -- */

typedef struct {
    double* c[5]; /* eta1 eta2 eta3 tau1 tau2 */
} qset;

static void qset_alloc(qset* q, long n)
{
    for (int j = 0; j < 5; ++j) q->c[j] = (double*)malloc(sizeof(double) * n);
}

static void qset_free(qset* q)
{
    for (int j = 0; j < 5; ++j) free(q->c[j]);
}

static inline double qdot(const qset* q, long ip, double* const S[5])
{
    return q->c[0][ip] * S[0][ip] + q->c[1][ip] * S[1][ip] + q->c[2][ip] * S[2][ip] +
           q->c[3][ip] * S[3][ip] + q->c[4][ip] * S[4][ip];
}

/* Re IFFT(M(k) * X(k)) for a multiplier that depends on one axis (table T)
 * times an optional |k|^pw factor; result scaled later by 1/ntp like the
 * reference.  X may be formed from (V - Vprev)/dt when prev != NULL. */
static void spectral_apply(int ntx, int nty, int ntz, const cplx* X, const cplx* prev, double dt,
                           int axis, const double* T, int pw, const double* kx, const double* ky,
                           const double* kz, cplx* work, double* out_re)
{
    long ntp = (long)ntx * nty * ntz;
#pragma omp parallel for schedule(static)
    for (long ip = 0; ip < ntp; ++ip) {
        int iz = ip % ntz, iy = (ip / ntz) % nty, ix = ip / ((long)nty * ntz);
        cplx x = X[ip];
        if (prev) { /* cuviscoelas_3D.cu:514-519: (out - dv)/dt */
            x.re = (x.re - prev[ip].re) / dt;
            x.im = (x.im - prev[ip].im) / dt;
        }
        int it = axis == 0 ? ix : axis == 1 ? iy : iz;
        double tr = T[2 * it], ti = T[2 * it + 1];
        double k2 = 1.0;
        if (pw != 0) {
            k2 = kx[ix] * kx[ix] + ky[iy] * ky[iy] + kz[iz] * kz[iz];
            if (ip == 0) k2 = 1e-10; /* cuviscoelas_3D.cu:74 */
            k2 = pw < 0 ? 1.0 / sqrt(k2) : sqrt(k2); /* Ap1, Ap3 (:188-190) */
        }
        work[ip].re = k2 * (tr * x.re - ti * x.im);
        work[ip].im = k2 * (tr * x.im + ti * x.re);
    }
    fft3(work, ntx, nty, ntz, +1);
#pragma omp parallel for schedule(static)
    for (long ip = 0; ip < ntp; ++ip) out_re[ip] = work[ip].re;
}

static void to_complex(long n, const double* r, cplx* c)
{
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) { c[i].re = r[i]; c[i].im = 0.0; }
}

int qo_run(const qo_params* p, const float* rik,
           const float* velp, const float* vels, const float* rho,
           const float* gama_p, const float* gama_s,
           const float* eps, const float* delta,
           const int* r_ix, const int* r_iy,
           float* rec_vx, float* rec_vy, float* rec_vz,
           int nsnap, const int* snap_steps, float* snaps, double* state_out)
{
    const int ntx = p->ntx, nty = p->nty, ntz = p->ntz;
    const long ntp = (long)ntx * nty * ntz;
    const long A = (long)nty * ntz;
    const double dt = p->dt;
    const double inv = 1.0 / (double)ntp;
    if (ntx < 4 || nty < 4 || ntz < 4 || p->pml < 2 || p->nt < 0) return 1;
    if (p->vti && (!eps || !delta)) return 2;
#ifdef _OPENMP
    if (p->nthreads > 0) omp_set_num_threads(p->nthreads);
#endif

    /* ---- setup: k-space (cu:22-152), Q sets (cu:155-210), C-PML (cu:213-309) */
    double *kx = malloc(sizeof(double) * ntx), *ky = malloc(sizeof(double) * nty), *kz = malloc(sizeof(double) * ntz);
    double *Fx = malloc(sizeof(double) * 2 * ntx), *Bx = malloc(sizeof(double) * 2 * ntx);
    double *Fy = malloc(sizeof(double) * 2 * nty), *By = malloc(sizeof(double) * 2 * nty);
    double *Fz = malloc(sizeof(double) * 2 * ntz), *Bz = malloc(sizeof(double) * 2 * ntz);
    qo_wavenumbers(ntx, p->dx, kx); qo_wavenumbers(nty, p->dy, ky); qo_wavenumbers(ntz, p->dz, kz);
    qo_shift_tables(ntx, p->dx, Fx, Bx); qo_shift_tables(nty, p->dy, Fy, By); qo_shift_tables(ntz, p->dz, Fz, Bz);
    double *ax = malloc(sizeof(double) * ntx), *bx = malloc(sizeof(double) * ntx);
    double *ay = malloc(sizeof(double) * nty), *by = malloc(sizeof(double) * nty);
    double *az = malloc(sizeof(double) * ntz), *bz = malloc(sizeof(double) * ntz);
    qo_pml_profile(ntx, p->pml, p->dx, p->f0, ax, bx);
    qo_pml_profile(nty, p->pml, p->dy, p->f0, ay, by);
    qo_pml_profile(ntz, p->pml, p->dz, p->f0, az, bz);

    /* Stiffness sets.  Isotropic (cu:879-898): K11 = K33 = P(vp, gp),
     * K12 = K13 = P - 2 S, shear S(vs, gs).  VTI (project extension):
     * c33 = rho vp^2, c44 = c66 = rho vs^2, c11 = c33 (1 + 2 eps),
     * c13 = sqrt((c33 - c44)(c33 (1 + 2 delta) - c44)) - c44;
     * K11 = P(vp sqrt(1+2eps)), K33 = P(vp), K12 = K11 - 2 S,
     * K13 = P(sqrt((c13 + 2 c44)/rho)) - 2 S. */
    qset K11, K33, K12, K13, S;
    qset_alloc(&K11, ntp); qset_alloc(&K33, ntp); qset_alloc(&K12, ntp); qset_alloc(&K13, ntp); qset_alloc(&S, ntp);
    const double w0 = w0_of(p->f0);
#pragma omp parallel for schedule(static)
    for (long ip = 0; ip < ntp; ++ip) {
        double r = rho[ip], vp = velp[ip], vs = vels[ip], gp = gama_p[ip], gs = gama_s[ip];
        double s5[5], p11[5], p33[5], p13[5];
        q_set(vs, gs, r, w0, s5);
        q_set(vp, gp, r, w0, p33);
        if (p->vti) {
            double e = eps[ip], dl = delta[ip];
            double c33 = r * vp * vp, c44 = r * vs * vs;
            double c13 = sqrt((c33 - c44) * (c33 * (1.0 + 2.0 * dl) - c44)) - c44;
            q_set(vp * sqrt(1.0 + 2.0 * e), gp, r, w0, p11);
            q_set(sqrt((c13 + 2.0 * c44) / r), gp, r, w0, p13);
        } else {
            memcpy(p11, p33, sizeof p11);
            memcpy(p13, p33, sizeof p13);
        }
        for (int j = 0; j < 5; ++j) {
            S.c[j][ip] = s5[j];
            K33.c[j][ip] = p33[j];
            K11.c[j][ip] = p11[j];
            K12.c[j][ip] = p11[j] - 2.0 * s5[j];
            K13.c[j][ip] = p13[j] - 2.0 * s5[j];
        }
    }

    /* ---- state (cu:312-410 zero-initialisation) */
    double* F[9]; /* vx vy vz pxx pyy pzz pxy pxz pyz */
    for (int f = 0; f < 9; ++f) F[f] = calloc(ntp, sizeof(double));
    double *vx = F[0], *vy = F[1], *vz = F[2], *pxx = F[3], *pyy = F[4], *pzz = F[5], *pxy = F[6], *pxz = F[7], *pyz = F[8];
    /* velocity-side memory variables (cu:1049-1074) */
    enum { P_XX_X, P_XY_Y, P_XZ_Z, P_XY_X, P_YY_Y, P_YZ_Z, P_XZ_X, P_YZ_Y, P_ZZ_Z, NPHIP };
    double* phip[NPHIP];
    for (int f = 0; f < NPHIP; ++f) phip[f] = calloc(ntp, sizeof(double));
    /* stress-side memory variables (cu:846-877, 902-954) */
    enum { V_X_XX, V_Z_ZX, V_Y_YX, V_X_XY, V_Z_ZY, V_Y_YY, V_X_XZ, V_Z_ZZ, V_Y_YZ,
           V_X_Z, V_Z_X, V_X_Y, V_Y_X, V_Y_Z, V_Z_Y, NPHIV };
    double* phiv[NPHIV];
    for (int f = 0; f < NPHIV; ++f) phiv[f] = calloc(ntp, sizeof(double));

    cplx* SP[6];
    for (int f = 0; f < 6; ++f) SP[f] = malloc(sizeof(cplx) * ntp);
    cplx *V[3], *dV[3];
    for (int f = 0; f < 3; ++f) { V[f] = malloc(sizeof(cplx) * ntp); dV[f] = calloc(ntp, sizeof(cplx)); }
    cplx* work = malloc(sizeof(cplx) * ntp);
    double* part[9];
    for (int f = 0; f < 9; ++f) part[f] = malloc(sizeof(double) * ntp);
    double* pv[9][5];
    for (int d = 0; d < 9; ++d)
        for (int j = 0; j < 5; ++j) pv[d][j] = malloc(sizeof(double) * ntp);

    int ok = 1;
    for (int f = 0; f < 9 && ok; ++f) ok = F[f] && part[f];
    if (!ok || !work) return 3;

    const int rn = p->rn;
    int isnap = 0;

    for (int it = 0; it < p->nt; ++it) {
        /* -- stress spectra (cu:1265-1277) */
        for (int f = 0; f < 6; ++f) { to_complex(ntp, F[3 + f], SP[f]); fft3(SP[f], ntx, nty, ntz, -1); }
        /* SP order: xx yy zz xy xz yz */
        /* -- stress divergence (cu:1279-1306) */
        spectral_apply(ntx, nty, ntz, SP[0], NULL, dt, 0, Bx, 0, kx, ky, kz, work, part[0]); /* partx1 = dx- pxx */
        spectral_apply(ntx, nty, ntz, SP[3], NULL, dt, 1, Fy, 0, kx, ky, kz, work, part[1]); /* party1 = dy+ pxy */
        spectral_apply(ntx, nty, ntz, SP[4], NULL, dt, 2, Fz, 0, kx, ky, kz, work, part[2]); /* partz1 = dz+ pxz */
        spectral_apply(ntx, nty, ntz, SP[4], NULL, dt, 0, Fx, 0, kx, ky, kz, work, part[3]); /* partx2 = dx+ pxz */
        spectral_apply(ntx, nty, ntz, SP[5], NULL, dt, 1, Fy, 0, kx, ky, kz, work, part[4]); /* party2 = dy+ pyz */
        spectral_apply(ntx, nty, ntz, SP[2], NULL, dt, 2, Bz, 0, kx, ky, kz, work, part[5]); /* partz2 = dz- pzz */
        spectral_apply(ntx, nty, ntz, SP[3], NULL, dt, 0, Fx, 0, kx, ky, kz, work, part[6]); /* partx3 = dx+ pxy */
        spectral_apply(ntx, nty, ntz, SP[1], NULL, dt, 1, By, 0, kx, ky, kz, work, part[7]); /* party3 = dy- pyy */
        spectral_apply(ntx, nty, ntz, SP[5], NULL, dt, 2, Fz, 0, kx, ky, kz, work, part[8]); /* partz3 = dz+ pyz */

        /* -- velocity update with C-PML (cu:1018-1101) */
        double *px1 = part[0], *py1 = part[1], *pz1 = part[2], *px2 = part[3], *py2 = part[4], *pz2 = part[5],
               *px3 = part[6], *py3 = part[7], *pz3 = part[8];
#pragma omp parallel for schedule(static)
        for (long ip = 0; ip < ntp; ++ip) {
            int iz = ip % ntz, iy = (ip / ntz) % nty, ix = ip / A;
            if (!(iz < ntz - 1 && ix < ntx - 1 && iy < nty - 1)) continue;
            double axh = 0.5 * (ax[ix] + ax[ix + 1]), bxh = 0.5 * (bx[ix] + bx[ix + 1]);
            double ayh = 0.5 * (ay[iy] + ay[iy + 1]), byh = 0.5 * (by[iy] + by[iy + 1]);
            double azh = 0.5 * (az[iz] + az[iz + 1]), bzh = 0.5 * (bz[iz] + bz[iz + 1]);
            double* q = NULL;
            q = phip[P_XX_X]; q[ip] += dt * (-axh * q[ip] - bxh * px1[ip] * inv);
            q = phip[P_XY_Y]; q[ip] += dt * (-ay[iy] * q[ip] - by[iy] * py1[ip] * inv);
            q = phip[P_XZ_Z]; q[ip] += dt * (-az[iz] * q[ip] - bz[iz] * pz1[ip] * inv);
            q = phip[P_XY_X]; q[ip] += dt * (-ax[ix] * q[ip] - bx[ix] * px3[ip] * inv);
            q = phip[P_YY_Y]; q[ip] += dt * (-ayh * q[ip] - byh * py3[ip] * inv);
            q = phip[P_YZ_Z]; q[ip] += dt * (-az[iz] * q[ip] - bz[iz] * pz3[ip] * inv);
            q = phip[P_XZ_X]; q[ip] += dt * (-ax[ix] * q[ip] - bx[ix] * px2[ip] * inv);
            q = phip[P_YZ_Y]; q[ip] += dt * (-ay[iy] * q[ip] - by[iy] * py2[ip] * inv);
            q = phip[P_ZZ_Z]; q[ip] += dt * (-azh * q[ip] - bzh * pz2[ip] * inv);
            vx[ip] += dt / (0.5 * (rho[ip] + rho[ip + A])) *
                      (px1[ip] * inv + phip[P_XX_X][ip] + py1[ip] * inv + phip[P_XY_Y][ip] + pz1[ip] * inv + phip[P_XZ_Z][ip]);
            vy[ip] += dt / (0.5 * (rho[ip] + rho[ip + ntz])) *
                      (px3[ip] * inv + phip[P_XY_X][ip] + py3[ip] * inv + phip[P_YY_Y][ip] + pz3[ip] * inv + phip[P_YZ_Z][ip]);
            vz[ip] += dt / (0.5 * (rho[ip] + rho[ip + 1])) *
                      (px2[ip] * inv + phip[P_XZ_X][ip] + py2[ip] * inv + phip[P_YZ_Y][ip] + pz2[ip] * inv + phip[P_ZZ_Z][ip]);
        }

        /* -- velocity spectra (cu:1331-1338) */
        for (int f = 0; f < 3; ++f) { to_complex(ntp, F[f], V[f]); fft3(V[f], ntx, nty, ntz, -1); }

        /* -- 45 constant-Q derivative fields (cu:1342-1562).  Index d:
         * 0 vx_x(F), 1 vy_y(F), 2 vz_z(F), 3 vx_z(B), 4 vz_x(B), 5 vx_y(B),
         * 6 vy_x(B), 7 vy_z(B), 8 vz_y(B); j: 0..2 dispersion with |k|^-1, 1,
         * |k|; 3..4 loss with |k|^-1, 1 on (V - Vprev)/dt. */
        static const int comp[9] = {0, 1, 2, 0, 2, 0, 1, 1, 2};
        static const int axis[9] = {0, 1, 2, 2, 0, 1, 0, 2, 1};
        static const int fwd[9] = {1, 1, 1, 0, 0, 0, 0, 0, 0};
        for (int d = 0; d < 9; ++d) {
            const double* T = axis[d] == 0 ? (fwd[d] ? Fx : Bx) : axis[d] == 1 ? (fwd[d] ? Fy : By) : (fwd[d] ? Fz : Bz);
            static const int pw[5] = {-1, 0, 1, -1, 0};
            for (int j = 0; j < 5; ++j)
                spectral_apply(ntx, nty, ntz, V[comp[d]], j >= 3 ? dV[comp[d]] : NULL, dt, axis[d], T, pw[j],
                               kx, ky, kz, work, pv[d][j]);
        }
        for (int d = 0; d < 9; ++d)
            for (int j = 0; j < 5; ++j) {
                double* a = pv[d][j];
#pragma omp parallel for schedule(static)
                for (long ip = 0; ip < ntp; ++ip) a[ip] *= inv;
            }

        /* -- stress update with constant-Q and C-PML (cu:800-1015) */
#pragma omp parallel for schedule(static)
        for (long ip = 0; ip < ntp; ++ip) {
            int iz = ip % ntz, iy = (ip / ntz) % nty, ix = ip / A;
            if (!(iz < ntz - 1 && ix < ntx - 1 && iy < nty - 1)) continue;
            double *Sxx[5], *Syy[5], *Szz[5];
            for (int j = 0; j < 5; ++j) { Sxx[j] = pv[0][j]; Syy[j] = pv[1][j]; Szz[j] = pv[2][j]; }
            double k11x = qdot(&K11, ip, Sxx), k12x = qdot(&K12, ip, Sxx), k13x = qdot(&K13, ip, Sxx);
            double k12y = qdot(&K12, ip, Syy), k11y = qdot(&K11, ip, Syy), k13y = qdot(&K13, ip, Syy);
            double k13z = qdot(&K13, ip, Szz), k33z = qdot(&K33, ip, Szz);
            double* q;
            q = phiv[V_X_XX]; q[ip] += dt * (-ax[ix] * q[ip] - bx[ix] * k11x);
            q = phiv[V_Z_ZX]; q[ip] += dt * (-az[iz] * q[ip] - bz[iz] * k13z);
            q = phiv[V_Y_YX]; q[ip] += dt * (-ay[iy] * q[ip] - by[iy] * k12y);
            q = phiv[V_Z_ZZ]; q[ip] += dt * (-az[iz] * q[ip] - bz[iz] * k33z);
            q = phiv[V_X_XZ]; q[ip] += dt * (-ax[ix] * q[ip] - bx[ix] * k13x);
            q = phiv[V_Y_YZ]; q[ip] += dt * (-ay[iy] * q[ip] - by[iy] * k13y);
            q = phiv[V_Y_YY]; q[ip] += dt * (-ay[iy] * q[ip] - by[iy] * k11y);
            q = phiv[V_X_XY]; q[ip] += dt * (-ax[ix] * q[ip] - bx[ix] * k12x);
            q = phiv[V_Z_ZY]; q[ip] += dt * (-az[iz] * q[ip] - bz[iz] * k13z);
            pxx[ip] += dt * (k11x + k12y + k13z + phiv[V_X_XX][ip] + phiv[V_Y_YX][ip] + phiv[V_Z_ZX][ip]);
            pyy[ip] += dt * (k12x + k11y + k13z + phiv[V_X_XY][ip] + phiv[V_Y_YY][ip] + phiv[V_Z_ZY][ip]);
            pzz[ip] += dt * (k13x + k13y + k33z + phiv[V_X_XZ][ip] + phiv[V_Y_YZ][ip] + phiv[V_Z_ZZ][ip]);

            /* 8-point averaged shear coefficients (cu:956-971) */
            double mu[5];
            for (int j = 0; j < 5; ++j) {
                const double* s = S.c[j];
                mu[j] = 0.125 * (s[ip] + s[ip + 1] + s[ip + ntz] + s[ip + 1 + ntz] + s[ip + A] + s[ip + A + 1] +
                                 s[ip + A + ntz] + s[ip + A + 1 + ntz]);
            }
#define MDOT(d) (mu[0] * pv[d][0][ip] + mu[1] * pv[d][1][ip] + mu[2] * pv[d][2][ip] + mu[3] * pv[d][3][ip] + mu[4] * pv[d][4][ip])
            double m_vx_z = MDOT(3), m_vz_x = MDOT(4), m_vx_y = MDOT(5), m_vy_x = MDOT(6), m_vy_z = MDOT(7), m_vz_y = MDOT(8);
#undef MDOT
            double azh = 0.5 * (az[iz] + az[iz + 1]), bzh = 0.5 * (bz[iz] + bz[iz + 1]);
            double axh = 0.5 * (ax[ix] + ax[ix + 1]), bxh = 0.5 * (bx[ix] + bx[ix + 1]);
            double ayh = 0.5 * (ay[iy] + ay[iy + 1]), byh = 0.5 * (by[iy] + by[iy + 1]);
            q = phiv[V_X_Z]; q[ip] += dt * (-azh * q[ip] - bzh * m_vx_z);
            q = phiv[V_Z_X]; q[ip] += dt * (-axh * q[ip] - bxh * m_vz_x);
            q = phiv[V_X_Y]; q[ip] += dt * (-ayh * q[ip] - byh * m_vx_y);
            q = phiv[V_Y_X]; q[ip] += dt * (-axh * q[ip] - bxh * m_vy_x);
            q = phiv[V_Y_Z]; q[ip] += dt * (-azh * q[ip] - bzh * m_vy_z);
            q = phiv[V_Z_Y]; q[ip] += dt * (-ayh * q[ip] - byh * m_vz_y);
            pxz[ip] += dt * (m_vx_z + phiv[V_X_Z][ip] + m_vz_x + phiv[V_Z_X][ip]);
            pyz[ip] += dt * (m_vy_z + phiv[V_Y_Z][ip] + m_vz_y + phiv[V_Z_Y][ip]);
            pxy[ip] += dt * (m_vx_y + phiv[V_X_Y][ip] + m_vy_x + phiv[V_Y_X][ip]);
        }

        /* -- source and receivers (cu:747-797) */
        {
            long is = (long)p->s_ix * A + (long)p->s_iy * ntz + p->s_iz;
            if (p->s_ix >= 0 && p->s_ix < ntx && p->s_iy >= 0 && p->s_iy < nty && p->s_iz >= 0 && p->s_iz < ntz) {
                if (p->src_type == 1) { pxx[is] += rik[it]; pyy[is] += rik[it]; pzz[is] += rik[it]; }
                else vx[is] += rik[it];
            }
            for (int ir = 0; ir < rn; ++ir) {
                long ipr = (long)r_ix[ir] * A + (long)r_iy[ir] * ntz + p->r_iz;
                if (rec_vx) rec_vx[(long)it * rn + ir] = (float)vx[ipr];
                if (rec_vy) rec_vy[(long)it * rn + ir] = (float)vy[ipr];
                if (rec_vz) rec_vz[(long)it * rn + ir] = (float)vz[ipr];
            }
        }
        /* -- previous spectra for the loss term (cu:1105-1134) */
        for (int f = 0; f < 3; ++f) memcpy(dV[f], V[f], sizeof(cplx) * ntp);

        while (isnap < nsnap && snap_steps[isnap] == it + 1) {
            for (int f = 0; f < 3; ++f)
                for (long ip = 0; ip < ntp; ++ip) snaps[((long)isnap * 3 + f) * ntp + ip] = (float)F[f][ip];
            ++isnap;
        }
    }
    if (state_out)
        for (int f = 0; f < 9; ++f) memcpy(state_out + (long)f * ntp, F[f], sizeof(double) * ntp);

    for (int f = 0; f < 9; ++f) { free(F[f]); free(part[f]); }
    for (int f = 0; f < NPHIP; ++f) free(phip[f]);
    for (int f = 0; f < NPHIV; ++f) free(phiv[f]);
    for (int f = 0; f < 6; ++f) free(SP[f]);
    for (int f = 0; f < 3; ++f) { free(V[f]); free(dV[f]); }
    for (int d = 0; d < 9; ++d)
        for (int j = 0; j < 5; ++j) free(pv[d][j]);
    free(work);
    qset_free(&K11); qset_free(&K33); qset_free(&K12); qset_free(&K13); qset_free(&S);
    free(kx); free(ky); free(kz); free(Fx); free(Bx); free(Fy); free(By); free(Fz); free(Bz);
    free(ax); free(bx); free(ay); free(by); free(az); free(bz);
    return 0;
}
