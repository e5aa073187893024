// Test harness around the reference's own CUDA build (cuFFT path).
//
// TEST INFRASTRUCTURE ONLY.  This file is compiled together with the
// reference's unmodified cuviscoelas_3D.cu (by oracle/Makefile, target
// `ref`, into oracle/_ref/libqvti_ref.so) and drives the reference through
// its own C ABI exactly the way its host driver does:
//
//   cuda_Device_malloc        (Myfunctions.h:91-96,  cuviscoelas_3D.cu:1689-1916)
//   cuda_Host_initialization  (Myfunctions.h:88-89,  cuviscoelas_3D.cu:1658-1683)
//   cuda_forward_acoustic_3D  (Myfunctions.h:77-85,  cuviscoelas_3D.cu:1137-1652)
//   cuda_Device_free          (Myfunctions.h:98-102, cuviscoelas_3D.cu:1922-2141)
//
// with the call sequence of viscoelas_3D.cpp:337-338, 398-405, 452.  The only
// addition is read-back of the final wavefield through the device pointers
// the reference stores in `struct MultiGPU` (d_vx ... d_pyz), which is how
// snapshots are taken without patching the reference: a snapshot at step k is
// the final state of a run with nt = k.
//
// It is used by tests/golden/make_golden.py to produce golden fixtures and by
// the GPU parity tests.  Nothing in the product links or loads it.
#include <cstdio>
#include <cstring>
#include <chrono>
#include <vector>
#include <cuda_runtime.h>
#include "Myfunctions.h"

#define QREF_PI 3.1415926   // the reference's truncated pi (viscoelas_3D.cpp:14)

extern "C" int qref_run(int ntx, int nty, int ntz, int pml, int nt,
                        float dx, float dy, float dz, float dt, float f0,
                        const float* rik, const float* velp, const float* gama_p,
                        const float* vels, const float* gama_s, const float* rho,
                        int s_ix, int s_iy, int s_iz, int r_iz,
                        const int* r_ix, const int* r_iy, int rnx_max, int rny_max,
                        float* rec_vx, float* rec_vy, float* rec_vz,
                        float* out_fields, double* elapsed_ms)
{
    const int ntp = ntx * nty * ntz;
    const int nx = ntx - 2 * pml, ny = nty - 2 * pml, nz = ntz - 2 * pml;
    const int rnmax = rnx_max * rny_max;
    const float w0 = 2 * QREF_PI * f0;          // viscoelas_3D.cpp:109
    const float velp_max = 5000.0f;             // overwritten on device anyway (cu:235)

    std::vector<int> rix(r_ix, r_ix + rnmax), riy(r_iy, r_iy + rnmax);
    std::vector<float> h_rik(rik, rik + nt);
    std::vector<float> h_velp(velp, velp + ntp), h_gp(gama_p, gama_p + ntp),
        h_vels(vels, vels + ntp), h_gs(gama_s, gama_s + ntp), h_rho(rho, rho + ntp);

    struct Source ss[1];
    ss[0].s_ix = s_ix; ss[0].s_iy = s_iy; ss[0].s_iz = s_iz; ss[0].r_iz = r_iz;
    ss[0].r_ix = rix.data(); ss[0].r_iy = riy.data(); ss[0].r_n = rnmax;

    struct MultiGPU plan[1];
    memset(plan, 0, sizeof(plan));
    cuda_Device_malloc(ntx, nty, ntz, ntp, nx, ny, nz, nt, rnmax, plan, 1);
    cuda_Host_initialization(ntp, nt, rnmax, plan, 1);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) { fprintf(stderr, "qref: malloc: %s\n", cudaGetErrorString(e)); return 1; }

    auto t0 = std::chrono::steady_clock::now();
    cuda_forward_acoustic_3D(0, 0, nt, ntx, nty, ntz, ntp, nx, ny, nz, pml,
                             dx, dy, dz, dt, f0, w0, velp_max,
                             h_rik.data(), h_velp.data(), h_gp.data(), h_vels.data(), h_gs.data(), h_rho.data(),
                             ss, plan, 1, rnmax, rnx_max, rny_max, 1);
    e = cudaDeviceSynchronize();
    auto t1 = std::chrono::steady_clock::now();
    if (elapsed_ms) *elapsed_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    if (e != cudaSuccess) { fprintf(stderr, "qref: run: %s\n", cudaGetErrorString(e)); return 2; }

    const size_t nrec = (size_t)nt * rnmax;
    if (rec_vx) memcpy(rec_vx, plan[0].record, nrec * sizeof(float));
    if (rec_vy) memcpy(rec_vy, plan[0].record2, nrec * sizeof(float));
    if (rec_vz) memcpy(rec_vz, plan[0].record3, nrec * sizeof(float));
    if (out_fields) {
        float* dev[9] = {plan[0].d_vx, plan[0].d_vy, plan[0].d_vz, plan[0].d_pxx, plan[0].d_pyy,
                         plan[0].d_pzz, plan[0].d_pxy, plan[0].d_pxz, plan[0].d_pyz};
        for (int f = 0; f < 9; ++f)
            cudaMemcpy(out_fields + (size_t)f * ntp, dev[f], (size_t)ntp * sizeof(float), cudaMemcpyDeviceToHost);
    }
    e = cudaDeviceSynchronize();
    cuda_Device_free(plan, 1);
    cudaDeviceSynchronize();
    return e == cudaSuccess ? 0 : 3;
}
