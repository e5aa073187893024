// The reference's void C ABI (include/Myfunctions.h) on top of the qvti_*
// entry points.  Call sequence and semantics follow viscoelas_3D.cpp:337-338,
// 398-405, 452 and cuviscoelas_3D.cu:1137-1652, 1658-1683, 1689-1916, 1922-2141.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cuda_runtime.h>

#include "../../include/Myfunctions.h"

extern "C" void getdevice(int* GPU_N)
{
    if (!GPU_N) return;
    if (cudaGetDeviceCount(GPU_N) != cudaSuccess) *GPU_N = 0;
}

// Allocation needs the grid only; the engine itself is created on the first
// shot, when pml, spacing, dt and f0 are known (the reference passes them to
// cuda_forward_acoustic_3D, not to cuda_Device_malloc), and kept for the
// following shots while those stay the same.
extern "C" void cuda_Device_malloc(int ntx, int nty, int ntz, int ntp, int nx, int ny, int nz, int nt, int rnmax,
                                   struct MultiGPU plan[], int GPU_N)
{
    (void)ntp; (void)nx; (void)ny; (void)nz;
    for (int i = 0; i < GPU_N; ++i) {
        cudaSetDevice(i);
        std::memset(&plan[i], 0, sizeof(plan[i]));
        plan[i].ntx = ntx; plan[i].nty = nty; plan[i].ntz = ntz; plan[i].nt = nt; plan[i].rnmax = rnmax;
        const size_t b = sizeof(float) * (size_t)rnmax * nt;
        cudaMallocHost((void**)&plan[i].record, b);
        cudaMallocHost((void**)&plan[i].record2, b);
        cudaMallocHost((void**)&plan[i].record3, b);
    }
}

extern "C" void cuda_Host_initialization(int ntp, int nt, int rnmax, struct MultiGPU plan[], int GPU_N)
{
    (void)ntp;
    for (int i = 0; i < GPU_N; ++i) {
        const size_t b = sizeof(float) * (size_t)rnmax * nt;
        if (plan[i].record) std::memset(plan[i].record, 0, b);
        if (plan[i].record2) std::memset(plan[i].record2, 0, b);
        if (plan[i].record3) std::memset(plan[i].record3, 0, b);
    }
}

namespace {
// Everything qvti_create fixes: the same values let a simulation run the next shot.
bool same_engine(const qvti_config& a, const qvti_config& b)
{
    return a.ntx == b.ntx && a.nty == b.nty && a.ntz == b.ntz && a.pml == b.pml && a.dx == b.dx && a.dy == b.dy &&
           a.dz == b.dz && a.dt == b.dt && a.f0 == b.f0 && a.w0 == b.w0 && a.vti == b.vti && a.device == b.device;
}
}  // namespace

extern "C" void cuda_forward_acoustic_3D(int myid, int is, int nt, int ntx, int nty, int ntz, int ntp, int nx,
                                         int ny, int nz, int pml, float dx, float dy, float dz, float dt, float f0,
                                         float w0, float velp_max, float* rik, float* velp, float* gama_p,
                                         float* vels, float* gama_s, float* rho, struct Source ss[],
                                         struct MultiGPU plan[], int GPU_N, int rnmax, int rnx_max, int rny_max,
                                         int dr)
{
    (void)myid; (void)ntp; (void)nx; (void)ny; (void)nz; (void)velp_max; (void)dr; (void)rnmax;
    const int rn = rnx_max * rny_max;  // receiver ir = ix*rny_max + iy (cu:787)
    // launch every device's shot, then collect (the reference interleaves its
    // GPUs step by step, cu:1255-1630; independent shots, same result)
    for (int i = 0; i < GPU_N; ++i) {
        MultiGPU& p = plan[i];
        const Source& s = ss[is + i];
        qvti_config cfg;
        std::memset(&cfg, 0, sizeof(cfg));
        cfg.ntx = ntx; cfg.nty = nty; cfg.ntz = ntz; cfg.pml = pml;
        cfg.dx = dx; cfg.dy = dy; cfg.dz = dz; cfg.dt = dt; cfg.f0 = f0; cfg.w0 = w0;
        cfg.vti = 0; cfg.device = i;
        // the engine allocated for the previous shot is kept when this shot
        // has the same grid and constants (the reference allocates once in
        // cuda_Device_malloc and reuses its buffers for every shot,
        // viscoelas_3D.cpp:355-405); model, source and receivers are set again
        if (p.sim) {
            qvti_config have;
            if (qvti_get_config(p.sim, &have) || !same_engine(have, cfg)) {
                qvti_destroy(p.sim);
                p.sim = nullptr;
            }
        }
        if (!p.sim && qvti_create(&cfg, &p.sim)) continue;
        if (qvti_set_model(p.sim, velp, vels, rho, gama_p, gama_s, nullptr, nullptr, 0)) continue;
        if (qvti_set_receivers(p.sim, s.r_iz, s.r_ix, s.r_iy, rn)) continue;
        if (qvti_set_source(p.sim, QVTI_SRC_FORCE_X, s.s_ix, s.s_iy, s.s_iz + 10, rik, nt)) continue;
        if (qvti_reset(p.sim)) continue;
        qvti_step(p.sim, nt);
    }
    for (int i = 0; i < GPU_N; ++i)
        if (plan[i].sim) qvti_get_records(plan[i].sim, plan[i].record, plan[i].record2, plan[i].record3);
}

extern "C" void cuda_Device_free(struct MultiGPU plan[], int GPU_N)
{
    for (int i = 0; i < GPU_N; ++i) {
        cudaSetDevice(i);
        if (plan[i].sim) qvti_destroy(plan[i].sim);
        plan[i].sim = nullptr;
        if (plan[i].record) cudaFreeHost(plan[i].record);
        if (plan[i].record2) cudaFreeHost(plan[i].record2);
        if (plan[i].record3) cudaFreeHost(plan[i].record3);
        plan[i].record = plan[i].record2 = plan[i].record3 = nullptr;
    }
}

// ---------------------------------------------------------------------------
// Host-driver helpers of the reference's header (implemented in its
// viscoelas_3D.cpp); provided here so a driver written against the
// reference links unchanged.

// Ricker wavelet (1 - 2 tau) e^{-tau}, tau = (pi f0 (it dt - 1/f0))^2 with
// pi = 3.1415926 (viscoelas_3D.cpp:494-502).
extern "C" void getrik(int nt, float dt, float f0, float* rik)
{
    const double pi_ref = 3.1415926;
    for (int it = 0; it < nt; ++it) {
        const float t = it * dt - 1 / f0;
        const double tmp = (pi_ref * f0 * (double)t) * (pi_ref * f0 * (double)t);
        rik[it] = (float)((1.0 - 2.0 * tmp) * std::exp(-tmp));
    }
}

// P-velocity model: raw float32 [ix][iy][iz] interior read from the file named
// by $QVTI_VELP_FILE (default ./input/vpnew19_455_505.bin, the reference's
// hard-coded name, viscoelas_3D.cpp:541), edge-replicated into the C-PML
// (z, then y, then x; viscoelas_3D.cpp:576-655), then vs = vp/1.5, Qp = 200,
// Qs = 150, rho = 1800 everywhere (viscoelas_3D.cpp:658-677).  Missing or
// short file: the interior keeps whatever velp held (the reference reads
// without checking); a message goes to stderr.
extern "C" void get_velQ(int pml, int ntx, int nty, int ntz, int ntp, int nx, int ny, int nz, float* velp, float* Qp,
                         float* vels, float* Qs, float* rho)
{
    (void)ntp; (void)nx; (void)ny; (void)nz;
    const char* path = std::getenv("QVTI_VELP_FILE");
    if (!path) path = "./input/vpnew19_455_505.bin";
    FILE* fp = std::fopen(path, "rb");
    if (!fp) std::fprintf(stderr, "get_velQ: cannot open %s\n", path);
    auto at = [&](int ix, int iy, int iz) -> float& { return velp[((size_t)ix * nty + iy) * ntz + iz]; };
    if (fp) {
        size_t got = 0, want = 0;
        for (int ix = pml; ix < ntx - pml; ix++)
            for (int iy = pml; iy < nty - pml; iy++)
                for (int iz = pml; iz < ntz - pml; iz++) {
                    ++want;
                    got += std::fread(&at(ix, iy, iz), sizeof(float), 1, fp);
                }
        std::fclose(fp);
        if (got != want) std::fprintf(stderr, "get_velQ: %s holds %zu of %zu values\n", path, got, want);
    }
    for (int ix = pml; ix < ntx - pml; ix++)
        for (int iy = pml; iy < nty - pml; iy++) {
            for (int iz = 0; iz < pml; iz++) at(ix, iy, iz) = at(ix, iy, pml);
            for (int iz = ntz - pml; iz < ntz; iz++) at(ix, iy, iz) = at(ix, iy, ntz - pml - 1);
        }
    for (int iz = 0; iz < ntz; iz++)
        for (int ix = pml; ix < ntx - pml; ix++) {
            for (int iy = 0; iy < pml; iy++) at(ix, iy, iz) = at(ix, pml, iz);
            for (int iy = nty - pml; iy < nty; iy++) at(ix, iy, iz) = at(ix, nty - pml - 1, iz);
        }
    for (int iz = 0; iz < ntz; iz++)
        for (int iy = 0; iy < nty; iy++) {
            for (int ix = 0; ix < pml; ix++) at(ix, iy, iz) = at(pml, iy, iz);
            for (int ix = ntx - pml; ix < ntx; ix++) at(ix, iy, iz) = at(ntx - pml - 1, iy, iz);
        }
    const size_t n = (size_t)ntx * nty * ntz;
    for (size_t ip = 0; ip < n; ++ip) {
        vels[ip] = velp[ip] / 1.5f;
        Qp[ip] = 200.0f;
        Qs[ip] = 150.0f;
        rho[ip] = 1800.0f;
    }
}
