/* Myfunctions.h -- drop-in replacement for the reference's C ABI header
 * (Myfunctions.h:1-113 of the reference project).
 *
 * Same function names, argument lists and call semantics, so a host driver
 * written against the reference (viscoelas_3D.cpp) recompiles against this
 * header and links libqvti.so instead of the cuFFT object:
 *
 *   getdevice                 Myfunctions.h:3-4     (impl. cuviscoelas_3D.cu:2144-2148)
 *   struct Source             Myfunctions.h:6-10    unchanged layout
 *   struct MultiGPU           Myfunctions.h:12-75   the caller-visible members
 *                             record/record2/record3 are kept; the reference's
 *                             ~140 device pointers become one opaque handle
 *   cuda_forward_acoustic_3D  Myfunctions.h:77-85   (cuviscoelas_3D.cu:1137-1652)
 *   cuda_Host_initialization  Myfunctions.h:88-89   (cuviscoelas_3D.cu:1658-1683)
 *   cuda_Device_malloc        Myfunctions.h:91-96   (cuviscoelas_3D.cu:1689-1916)
 *   cuda_Device_free          Myfunctions.h:98-102  (cuviscoelas_3D.cu:1922-2141)
 *
 * The functions stay void like the reference's; a failure is reported by
 * qvti_last_error() (include/qvti.h).  Behaviour kept: force source added to
 * vx at (s_ix, s_iy, s_iz + 10) (cuviscoelas_3D.cu:772), receivers
 * ir = ix*rny_max + iy at depth r_iz, records [it][ir] in pinned host memory,
 * w0 taken from the caller, synchronous return after the seismograms are on
 * the host.
 */
#ifndef QVTI_MYFUNCTIONS_H
#define QVTI_MYFUNCTIONS_H

#include "qvti.h"

#ifdef __cplusplus
extern "C" {
#endif

void getdevice(int* GPU_N);

struct Source {
    int s_iz, s_ix, s_iy, r_iz, *r_ix, *r_iy, r_n;
};

struct MultiGPU {
    /* seismograms in pinned host memory, nt*rnmax floats each ([it][ir]) */
    float *record, *record2, *record3;
    /* engine state (opaque) and the sizes cuda_Device_malloc was given */
    qvti_sim* sim;
    int ntx, nty, ntz, nt, rnmax;
};

void cuda_forward_acoustic_3D(int myid, int is, int nt, int ntx, int nty, int ntz, int ntp, int nx, int ny, int nz,
                              int pml, float dx, float dy, float dz, float dt, float f0, float w0, float velp_max,
                              float* rik, float* velp, float* gama_p, float* vels, float* gama_s, float* rho,
                              struct Source ss[], struct MultiGPU plan[], int GPU_N, int rnmax, int rnx_max,
                              int rny_max, int dr);

void cuda_Host_initialization(int ntp, int nt, int rnmax, struct MultiGPU plan[], int GPU_N);

void cuda_Device_malloc(int ntx, int nty, int ntz, int ntp, int nx, int ny, int nz, int nt, int rnmax,
                        struct MultiGPU plan[], int GPU_N);

void cuda_Device_free(struct MultiGPU plan[], int GPU_N);

/* host-driver helpers (implemented by the host driver, viscoelas_3D.cpp:494-693) */
void getrik(int nt, float dt, float f0, float* rik);
void get_velQ(int pml, int ntx, int nty, int ntz, int ntp, int nx, int ny, int nz, float* velp, float* Qp,
              float* vels, float* Qs, float* rho);

#ifdef __cplusplus
}
#endif
#endif
