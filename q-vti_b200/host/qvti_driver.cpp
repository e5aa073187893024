// Host driver with the reference's surface (viscoelas_3D.cpp:16-491):
// model and parameter inputs, observation system, seismogram output files and
// binary formats, calling the GPU through the drop-in C ABI (Myfunctions.h).
//
//   qvti_driver [run-description file]
//
// The run description is "key = value" lines; every key defaults to the
// reference's hard-coded value (viscoelas_3D.cpp:82-112, 146-186), except the
// grid, which defaults to 256x256x64 (interior 226x226x34): the reference's 535x485x49
// has prime factors 107 and 97 that the engine's FFTs do not support).
//
//   nx ny nz pml nt      interior size, C-PML cells, steps
//   dx dy dz dt f0       spacing (m), step (s), Ricker / reference frequency
//   nsx nsy dsx dsy      shot grid and spacing (cells)
//   nsx0 nsy0 depth dr   first-shot offset, source/receiver depth, receiver step
//   velp_file            raw float32 [ix][iy][iz] interior P velocity (the
//                        reference's ./input/vpnew19_455_505.bin); when absent a
//                        homogeneous model velp_const is used
//   velp_const           m/s (default 2500)
//   vs_ratio qp qs rho   vs = vp/vs_ratio, constant Q and density (reference:
//                        1.5, 200, 150, 1800 -- viscoelas_3D.cpp:667-673)
//   snap_every           > 0: write vx/vy/vz interior snapshots every k steps
//                        (the reference's commented snapshot block,
//                        cuviscoelas_3D.cu:1611-1627) to ./output/shot%dsnap%d_v?.bin
//   outdir recdir        output directories (default ./output, ./record)
//   log                  JSON-lines run log, one line per shot (default
//                        <outdir>/run.jsonl; "none" disables): shot index,
//                        wall seconds, Gcell-steps/s, status and, for
//                        stepped runs (snap_every > 0), the FP64 sums of
//                        squares of the nine wavefields after the last step
//                        and whether any value was non-finite
//
// Outputs (formats of viscoelas_3D.cpp:188-199, 416-435):
//   <outdir>/source_xy.txt, <outdir>/source_trnum.txt       text
//   <recdir>/Q1dep_v{x,y,z}_small_shot%d.bin                raw float32 [it][ir]
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "Myfunctions.h"
#include "qvti.h"

namespace {

std::map<std::string, std::string> read_params(const char* path)
{
    std::map<std::string, std::string> kv;
    if (!path) return kv;
    std::ifstream in(path);
    if (!in) {
        std::fprintf(stderr, "cannot read %s\n", path);
        std::exit(2);
    }
    std::string line;
    while (std::getline(in, line)) {
        auto h = line.find('#');
        if (h != std::string::npos) line.resize(h);
        auto e = line.find('=');
        if (e == std::string::npos) continue;
        std::string k = line.substr(0, e), v = line.substr(e + 1);
        auto trim = [](std::string s) {
            size_t a = s.find_first_not_of(" \t\r"), b = s.find_last_not_of(" \t\r");
            return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
        };
        kv[trim(k)] = trim(v);
    }
    return kv;
}

struct P {
    std::map<std::string, std::string> kv;
    double num(const char* k, double d) const
    {
        auto it = kv.find(k);
        return it == kv.end() ? d : std::atof(it->second.c_str());
    }
    std::string str(const char* k, const char* d) const
    {
        auto it = kv.find(k);
        return it == kv.end() ? std::string(d) : it->second;
    }
};

void write_raw(const std::string& path, const float* a, size_t n)
{
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) {
        std::fprintf(stderr, "cannot write %s\n", path.c_str());
        return;
    }
    std::fwrite(a, sizeof(float), n, f);
    std::fclose(f);
}

}  // namespace

int main(int argc, char** argv)
{
    P p{read_params(argc > 1 ? argv[1] : nullptr)};
    const int nx = (int)p.num("nx", 226), ny = (int)p.num("ny", 226), nz = (int)p.num("nz", 34);
    const int pml = (int)p.num("pml", 15), nt = (int)p.num("nt", 3000);
    const int nsx = (int)p.num("nsx", 1), nsy = (int)p.num("nsy", 1);
    const int dsx = (int)p.num("dsx", 30), dsy = (int)p.num("dsy", 30);
    const int nsx0 = (int)p.num("nsx0", nx / 2), nsy0 = (int)p.num("nsy0", ny / 2);
    const int depth = (int)p.num("depth", 1), dr = (int)p.num("dr", 1);
    const float dx = (float)p.num("dx", 20.0), dy = (float)p.num("dy", 20.0), dz = (float)p.num("dz", 20.0);
    const float dt = (float)p.num("dt", 0.0008), f0 = (float)p.num("f0", 20.0);
    const float w0 = (float)(2 * 3.1415926 * f0);  // viscoelas_3D.cpp:109
    const int snap_every = (int)p.num("snap_every", 0);
    const std::string outdir = p.str("outdir", "./output"), recdir = p.str("recdir", "./record");
    const std::string log_path = p.str("log", (outdir + "/run.jsonl").c_str());
    const int ntx = nx + 2 * pml, nty = ny + 2 * pml, ntz = nz + 2 * pml;  // viscoelas_3D.cpp:117-119
    const int ntp = ntx * nty * ntz;
    mkdir(outdir.c_str(), 0755);
    mkdir(recdir.c_str(), 0755);
    std::printf("ntx=%d, nty=%d, ntz=%d\nnx=%d,  ny=%d,  nz=%d,  nt=%d,  ns=%d\n", ntx, nty, ntz, nx, ny, nz, nt,
                nsx * nsy);

    int GPU_N = 0;
    getdevice(&GPU_N);
    GPU_N = 1;  // viscoelas_3D.cpp:101

    std::vector<float> rik(nt);
    getrik(nt, dt, f0, rik.data());

    // observation system (viscoelas_3D.cpp:146-186)
    const int ns = nsx * nsy, rnx_max = nx / dr, rny_max = ny / dr;
    int rnmax = 0;
    std::vector<Source> ss(ns);
    for (int isx = 0; isx < nsx; isx++)
        for (int isy = 0; isy < nsy; isy++) {
            const int is = isx * nsy + isy;
            ss[is].s_ix = isx * dsx + pml + nsx0;
            ss[is].s_iy = isy * dsy + pml + nsy0;
            ss[is].s_iz = pml + depth;
            ss[is].r_iz = pml + depth;
            ss[is].r_n = rnx_max * rny_max;
            if (rnmax < ss[is].r_n) rnmax = ss[is].r_n;
        }
    std::vector<std::vector<int>> rix(ns, std::vector<int>(rnmax)), riy(ns, std::vector<int>(rnmax));
    for (int is = 0; is < ns; is++) {
        for (int ip = 0; ip < rnmax; ip++) {
            rix[is][ip] = pml + ip / rny_max * dr;
            riy[is][ip] = pml + ip % rny_max * dr;
        }
        ss[is].r_ix = rix[is].data();
        ss[is].r_iy = riy[is].data();
    }
    {
        FILE* fp = std::fopen((outdir + "/source_xy.txt").c_str(), "wt");
        if (fp) {
            for (int is = 0; is < ns; is++) std::fprintf(fp, "%10d %10d\r\n", ss[is].s_ix - pml, ss[is].s_iy - pml);
            std::fclose(fp);
        }
        fp = std::fopen((outdir + "/source_trnum.txt").c_str(), "wt");
        if (fp) {
            for (int is = 0; is < ns; is++) std::fprintf(fp, "%d\r\n", ss[is].r_n);
            std::fclose(fp);
        }
    }

    // model (viscoelas_3D.cpp:281-289, 537-693)
    std::vector<float> velp(ntp, (float)p.num("velp_const", 2500.0)), Qp(ntp), vels(ntp), Qs(ntp), rho(ntp),
        gama_p(ntp), gama_s(ntp);
    const std::string vf = p.str("velp_file", "");
    if (!vf.empty()) {
        setenv("QVTI_VELP_FILE", vf.c_str(), 1);
        get_velQ(pml, ntx, nty, ntz, ntp, nx, ny, nz, velp.data(), Qp.data(), vels.data(), Qs.data(), rho.data());
    }
    const float vs_ratio = (float)p.num("vs_ratio", 1.5), qp = (float)p.num("qp", 200), qs = (float)p.num("qs", 150);
    const float rho0 = (float)p.num("rho", 1800);
    for (int ip = 0; ip < ntp; ip++) {
        vels[ip] = velp[ip] / vs_ratio;
        Qp[ip] = qp;
        Qs[ip] = qs;
        rho[ip] = rho0;
        gama_p[ip] = (float)(std::atan(1.0 / Qp[ip]) / 3.1415926);
        gama_s[ip] = (float)(std::atan(1.0 / Qs[ip]) / 3.1415926);
    }

    std::vector<MultiGPU> plan(GPU_N);
    cuda_Device_malloc(ntx, nty, ntz, ntp, nx, ny, nz, nt, rnmax, plan.data(), GPU_N);
    cuda_Host_initialization(ntp, nt, rnmax, plan.data(), GPU_N);

    FILE* log = log_path == "none" ? nullptr : std::fopen(log_path.c_str(), "w");
    if (!log && log_path != "none") std::fprintf(stderr, "cannot write %s\n", log_path.c_str());
    int status = 0;
    for (int is = 0; is < ns; is += GPU_N) {
        const auto t0 = std::chrono::steady_clock::now();
        int shot_rc = 0;
        double norms[9];
        int nonfinite = -1;  // -1: not measured (a whole-shot ABI call)
        if (snap_every > 0) {
            // stepped run through the extended ABI to take snapshots
            qvti_config cfg{};
            cfg.ntx = ntx; cfg.nty = nty; cfg.ntz = ntz; cfg.pml = pml;
            cfg.dx = dx; cfg.dy = dy; cfg.dz = dz; cfg.dt = dt; cfg.f0 = f0; cfg.w0 = w0;
            qvti_sim* sim = nullptr;
            int rc = qvti_create(&cfg, &sim);
            if (!rc) rc = qvti_set_model(sim, velp.data(), vels.data(), rho.data(), gama_p.data(), gama_s.data(),
                                         nullptr, nullptr, 0);
            if (!rc) rc = qvti_set_receivers(sim, ss[is].r_iz, ss[is].r_ix, ss[is].r_iy, rnx_max * rny_max);
            if (!rc) rc = qvti_set_source(sim, QVTI_SRC_FORCE_X, ss[is].s_ix, ss[is].s_iy, ss[is].s_iz + 10,
                                          rik.data(), nt);
            if (!rc) rc = qvti_reset(sim);
            std::vector<float> f((size_t)3 * ntp), crop((size_t)nx * ny * nz);
            for (int it = 0; !rc && it < nt; it += snap_every) {
                const int k = std::min(snap_every, nt - it);
                rc = qvti_step(sim, k);
                if (!rc) rc = qvti_get_fields(sim, 0, 3, f.data());
                for (int c = 0; !rc && c < 3; ++c) {
                    size_t o = 0;
                    for (int ix = pml; ix < ntx - pml; ix++)
                        for (int iy = pml; iy < nty - pml; iy++)
                            for (int iz = pml; iz < ntz - pml; iz++)
                                crop[o++] = f[(size_t)c * ntp + ((size_t)ix * nty + iy) * ntz + iz];
                    char name[64];
                    std::snprintf(name, sizeof name, "/shot%dsnap%d_v%c.bin", is, it + k, "xyz"[c]);
                    write_raw(outdir + name, crop.data(), crop.size());
                }
            }
            if (!rc) rc = qvti_get_records(sim, plan[0].record, plan[0].record2, plan[0].record3);
            if (!rc) {
                const int nrc = qvti_field_norms(sim, norms, &nonfinite);
                if (nrc && nrc != QVTI_ERR_NONFINITE) rc = nrc;
            }
            if (sim) qvti_destroy(sim);
            if (rc) {
                std::fprintf(stderr, "shot %d failed: %s\n", is, qvti_error_string(rc));
                status = 1;
            }
            shot_rc = rc;
        } else {
            cuda_forward_acoustic_3D(0, is, nt, ntx, nty, ntz, ntp, nx, ny, nz, pml, dx, dy, dz, dt, f0, w0, 5000.0f,
                                     rik.data(), velp.data(), gama_p.data(), vels.data(), gama_s.data(), rho.data(),
                                     ss.data(), plan.data(), GPU_N, rnmax, rnx_max, rny_max, dr);
            shot_rc = qvti_last_error();
            if (shot_rc) {
                std::fprintf(stderr, "shot %d failed: %s\n", is, qvti_error_string(shot_rc));
                status = 1;
            }
        }
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (log) {
            std::fprintf(log, "{\"shot\": %d, \"seconds\": %.6f, \"gcell_steps_per_s\": %.6f, \"status\": \"%s\"", is,
                         sec, (double)ntp * nt / sec / 1e9, shot_rc ? qvti_error_string(shot_rc) : "ok");
            if (nonfinite >= 0) {
                std::fprintf(log, ", \"nonfinite\": %s, \"energy\": [", nonfinite ? "true" : "false");
                for (int f = 0; f < 9; ++f) std::fprintf(log, "%s%.17g", f ? ", " : "", norms[f]);
                std::fprintf(log, "]");
            }
            std::fprintf(log, "}\n");
            std::fflush(log);
        }
        for (int i = 0; i < GPU_N && is + i < ns; i++) {
            const char* comp[3] = {"vx", "vy", "vz"};
            float* rec[3] = {plan[i].record, plan[i].record2, plan[i].record3};
            for (int c = 0; c < 3; ++c) {
                char name[96];
                std::snprintf(name, sizeof name, "/Q1dep_%s_small_shot%d.bin", comp[c], is + i);
                write_raw(recdir + name, rec[c], (size_t)rnmax * nt);
            }
        }
        std::printf("shot %d done\n", is);
    }
    cuda_Device_free(plan.data(), GPU_N);
    if (log) std::fclose(log);
    return status;
}
