// Host side of the engine: allocation, FP64 setup on the GPU, CUDA-graph
// replay of the step, and the qvti_* C ABI (include/qvti.h).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <mutex>
#include <new>
#include <vector>

#include "engine.cuh"
#include "../../include/qvti.h"

namespace qvti {

thread_local int g_last_error = QVTI_OK;

int fail(int code)
{
    g_last_error = code;
    return code;
}

// Kernel attributes (the large dynamic shared-memory limits) are per device:
// each device is configured once, the first time a simulation or a stage
// entry point uses it, with that device current.
namespace {
PerDeviceOnce<kMaxDevices> g_configured;
std::atomic<long long> g_sims_created{0};
}  // namespace

int configure_device(int dev)
{
    return g_configured.run(dev, [] { return configure_kernels(); });
}

namespace {

#define QV_CUDA(call)                                                                        \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            fprintf(stderr, "qvti: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(e_), \
                    __FILE__, __LINE__);                                                     \
            return fail(e_ == cudaErrorMemoryAllocation ? QVTI_ERR_OOM : QVTI_ERR_CUDA);     \
        }                                                                                    \
    } while (0)

bool smooth(int n)
{
    for (int r : {2, 3, 5, 7})
        while (n % r == 0) n /= r;
    return n == 1;
}

// Radix schedule: radix 16 first, then 8, 4, 2 and the odd radices (256 is
// two radix-16 stages: one shared-memory exchange per transform).
bool make_plan(int n, FftPlan* p)
{
    p->n = n;
    p->nst = 0;
    int m = n;
    while (m % 16 == 0 && p->nst < kMaxStages) { p->rad[p->nst++] = 16; m /= 16; }
    while (m % 8 == 0 && p->nst < kMaxStages) { p->rad[p->nst++] = 8; m /= 8; }
    while (m % 4 == 0 && p->nst < kMaxStages) { p->rad[p->nst++] = 4; m /= 4; }
    while (m % 2 == 0 && p->nst < kMaxStages) { p->rad[p->nst++] = 2; m /= 2; }
    for (int r : {3, 5, 7})
        while (m % r == 0 && p->nst < kMaxStages) { p->rad[p->nst++] = r; m /= r; }
    if (m != 1) return false;
    if (p->nst == 1 && p->rad[0] == 16) {  // n = 16: two radix-4 stages
        p->rad[0] = 4;
        p->rad[1] = 4;
        p->nst = 2;
    }
    if (p->nst < 2) return false;
    // the compile-time transforms (and the shared-memory sizes derived from
    // them) use the same radix sequence
    if (p->nst != ct_nst(n)) return false;
    for (int st = 0; st < p->nst; ++st)
        if (p->rad[st] != ct_rad(n, st)) return false;
    return true;
}

// FP64 construction of the 1D tables of one axis on the GPU:
// twiddles e^{-2 pi i k/n}; |k| (cuviscoelas_3D.cu:54-67); staggered-shift
// multipliers i k e^{+-i k d/2} (cu:76-151) with the Nyquist bin reduced to
// its real part -- the Hermitian part of the multiplier, which is what the
// real part of the reference's C2C output sees; C-PML a, b (cu:213-309,
// velp_max forced to 5000, R = 1e-2, pi = 3.1415926) and their half-point
// averages 0.5 (v[i] + v[i+1]); with a == nullptr the C-PML outputs are not
// written (a, b, ah, bh may all be null then).
__global__ void k_axis_tables(int n, double d, double f0, int pml, float2* tw, float* kmag, float2* F, float2* B,
                              float* a, float* b, float* ah, float* bh)
{
    const double pi_ref = 3.1415926;
    for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < n; i += blockDim.x * gridDim.x) {
        double s, c;
        sincospi(-2.0 * i / n, &s, &c);
        tw[i] = make_float2((float)c, (float)s);
        const int m = i <= n / 2 ? i : n - i;
        const double tmp = 2.0 * pi_ref / n / d;
        kmag[i] = (float)(tmp * m);
        const double sn = sin(m * pi_ref / n), cs = cos(m * pi_ref / n);
        double fr, fi, br, bi;
        if (i <= n / 2) { fr = -tmp * m * sn; fi = tmp * m * cs; br = tmp * m * sn; bi = tmp * m * cs; }
        else            { fr = -tmp * m * sn; fi = -tmp * m * cs; br = tmp * m * sn; bi = -tmp * m * cs; }
        if (2 * i == n) { fi = 0.0; bi = 0.0; }
        F[i] = make_float2((float)fr, (float)fi);
        B[i] = make_float2((float)br, (float)bi);
        if (!a) continue;  // no C-PML profiles wanted (spectral stages only)
        auto prof = [&](int j, double* av, double* bv) {
            const double alpha_max = pi_ref * f0;
            const double om_max = 4.0 * 5000.0 * log(1.0 / (double)1e-2f) / (2.0 * pml * d);
            int jj = j < pml ? j : (j >= n - pml ? n - 1 - j : -1);
            if (jj < 0) { *av = alpha_max; *bv = 0.0; return; }
            const double al = alpha_max * pow((double)jj / (pml - 1), 2.0);
            const double om = om_max * pow((double)(pml - 1 - jj) / pml, 3.0);
            *av = al + om;
            *bv = om;
        };
        double a0, b0, a1, b1;
        prof(i, &a0, &b0);
        prof(i + 1 < n ? i + 1 : i, &a1, &b1);
        a[i] = (float)a0;
        b[i] = (float)b0;
        ah[i] = (float)(0.5 * (a0 + a1));
        bh[i] = (float)(0.5 * (b0 + b1));
    }
}

__global__ void k_norms(long long ntp, const float* f, double* out, int* nonfinite)
{
    double acc = 0.0;
    int bad = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ntp; i += (long long)gridDim.x * blockDim.x) {
        const float v = f[i];
        if (!isfinite(v)) bad = 1;
        else acc += (double)v * v;
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    __shared__ double red[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) red[w] = acc;
    bad = __syncthreads_or(bad);
    if (w == 0) {
        acc = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
        for (int o = 16; o; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) atomicAdd(out, acc);
    }
    if (threadIdx.x == 0 && bad) atomicOr(nonfinite, 1);
}

// Any non-finite value among 4 n4 floats of each of three fields sets *flag
// (float4 loads; every grid axis is even, so ntp is a multiple of 4).  x * 0
// is +-0 for finite x and NaN for Inf or NaN, so a sum of such products is
// zero exactly when every value is finite (a sum of the values themselves
// could overflow).
__global__ void k_finite3(long long n4, const float4* a, const float4* b, const float4* c, int* flag)
{
    int bad = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
        const float4 x = a[i], y = b[i], z = c[i];
        const float s = (x.x * 0.f + x.y * 0.f + x.z * 0.f + x.w * 0.f) + (y.x * 0.f + y.y * 0.f + y.z * 0.f + y.w * 0.f) +
                        (z.x * 0.f + z.y * 0.f + z.z * 0.f + z.w * 0.f);
        bad |= !(s == 0.f);
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

}  // namespace

bool make_fft_plan(int n, FftPlan* p) { return make_plan(n, p); }

void launch_axis_tables(int n, double d, double f0, int pml, float2* tw, float* kmag, float2* F, float2* B,
                        float* a, float* b, float* ah, float* bh, cudaStream_t st)
{
    k_axis_tables<<<4, 256, 0, st>>>(n, d, f0, pml, tw, kmag, F, B, a, b, ah, bh);
}

struct Sim {
    qvti_config cfg{};
    int nx = 0, ny = 0, nz = 0, nkz = 0;
    long long ntp = 0;
    cudaStream_t st = nullptr;
    KP kp{};
    std::vector<void*> allocs;
    float* coef[12] = {};
    int* d_it = nullptr;
    float* d_rik = nullptr;
    int* d_rix = nullptr;
    int* d_riy = nullptr;
    float* d_rec[3] = {};
    size_t rik_cap = 0, rix_cap = 0, rec_cap = 0;  // element capacities of the buffers above
    float** d_coefp = nullptr;  // device copy of coef[] (the coefficient build's outputs)
    size_t coefp_cap = 0;
    double* d_norm = nullptr;
    int* d_bad = nullptr;
    int* d_err = nullptr;  // set by a kernel whose bounded wait gave up
    int media = QVTI_MEDIA_VISCOELASTIC;
    float* d_inj[3] = {};  // time-reversed traces (qvti_set_injection)
    size_t inj_cap[3] = {};
    int* d_nonfinite = nullptr;  // set by qvti_check_finite_async
    int nt = 0, rn = 0;
    bool have_model = false, have_src = false;
    int steps = 0;
    // the step loop as CUDA graphs: one step, and kGraphSteps steps (built
    // when a call first asks for that many); both rebuilt after any change
    // to the launch parameters
    cudaGraphExec_t gexec = nullptr, gexec_n = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    void drop_graphs()
    {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (gexec_n) cudaGraphExecDestroy(gexec_n);
        gexec = gexec_n = nullptr;
    }

    // Device arrays come from the stream-ordered allocator on the
    // simulation's own stream: creating or freeing a simulation then orders
    // only against that stream, where cudaMalloc/cudaFree may wait for the
    // work of every stream on the device (other shots in flight).
    template <class T>
    int alloc(T** p, size_t count)
    {
        void* q = nullptr;
        cudaError_t e = cudaMallocAsync(&q, count * sizeof(T) > 0 ? count * sizeof(T) : 16, st);
        if (e != cudaSuccess) return fail(e == cudaErrorMemoryAllocation ? QVTI_ERR_OOM : QVTI_ERR_CUDA);
        allocs.push_back(q);
        *p = static_cast<T*>(q);
        return QVTI_OK;
    }
    void release(void* p)
    {
        for (auto& q : allocs)
            if (q == p) { cudaFreeAsync(q, st); q = nullptr; }
    }
    // Grow-only buffer: reallocated only when `count` exceeds its capacity,
    // so a simulation reused shot after shot keeps its buffers.
    template <class T>
    int ensure(T** p, size_t* cap, size_t count)
    {
        if (*p && count <= *cap) return QVTI_OK;
        if (*p) { release(*p); *p = nullptr; *cap = 0; }
        const int rc = alloc(p, count);
        if (rc == QVTI_OK) *cap = count;
        return rc;
    }
    ~Sim()
    {
        drop_graphs();
        for (void* p : allocs)
            if (p) cudaFreeAsync(p, st);
        if (st) cudaStreamSynchronize(st);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (st) cudaStreamDestroy(st);
    }
};

namespace {

// A device buffer freed when it goes out of scope (error returns included).
struct DevBuf {
    void* p = nullptr;
    float* f() const { return static_cast<float*>(p); }
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
};

// Number of full-grid float arrays (v, s, R, Q, coefficients, MU, 1/rho),
// of C-PML slab arrays per axis (x, y, z) and of half-spectrum complex arrays.
constexpr int kRealArrays = 3 + 6 + 3 + 6 + 12 + 5 + 3;
constexpr int kSlabArrays[3] = {13, 13, 11};  // php 3/3/3, phn 3/3/2, qn 3/3/2, phs 2/2/2, qs 2/2/2
constexpr int kSpecArrays = 3 + 3 + 3 + kNumGxy;  // H, Hy, Yv, G without the one-axis fields

// Every C-PML slab array of a simulation with its length in floats.
int slab_arrays(const KP& k, float** out, size_t* len)
{
    int n = 0;
    auto add = [&](float* p, int axis) {
        out[n] = p;
        len[n++] = (size_t)slab_len(k.nx, k.ny, k.nz, k.pml, axis);
    };
    for (int c = 0; c < 9; ++c) add(k.php[c], c % 3);
    for (int c = 0; c < 8; ++c) add(k.phn[c], c < 3 ? 0 : c < 6 ? 1 : 2);
    for (int c = 0; c < 8; ++c) add(k.qn[c], c < 3 ? 0 : c < 6 ? 1 : 2);
    for (int c = 0; c < 6; ++c) add(k.phs[c], kPhsAxis[c]);
    for (int c = 0; c < 6; ++c) add(k.qs[c], kPhsAxis[c]);
    return n;
}
constexpr int kNumSlab = 9 + 8 + 8 + 6 + 6;

// Steps per multi-step graph: 16 steps are 128 kernel nodes, and a chunk of
// the scheduler (32 steps) is two launches.
constexpr int kGraphSteps = 16;

// Captures `nsteps` steps into *out (the step counter lives on the device,
// so every replay advances it).
int build_graph(Sim* s, int nsteps, cudaGraphExec_t* out)
{
    if (*out) { cudaGraphExecDestroy(*out); *out = nullptr; }
    cudaGraph_t g = nullptr;
    QV_CUDA(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < nsteps; ++i) launch_step(s->kp, s->st);
    QV_CUDA(cudaStreamEndCapture(s->st, &g));
    cudaError_t e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    QV_CUDA(e);
    return QVTI_OK;
}
int build_graph(Sim* s) { return build_graph(s, 1, &s->gexec); }

}  // namespace
}  // namespace qvti

using qvti::Sim;
using qvti::fail;

struct qvti_sim : qvti::Sim {};

extern "C" size_t qvti_footprint_bytes(int ntx, int nty, int ntz, int pml, int vti)
{
    (void)vti;
    const size_t ntp = (size_t)ntx * nty * ntz;
    const size_t nspec = (size_t)(ntz / 2 + 1) * ntx * nty;
    size_t slab = 0;
    for (int a = 0; a < 3; ++a) slab += (size_t)qvti::kSlabArrays[a] * (size_t)qvti::slab_len(ntx, nty, ntz, pml, a);
    return ntp * sizeof(float) * qvti::kRealArrays + slab * sizeof(float) + nspec * sizeof(float2) * qvti::kSpecArrays;
}

extern "C" int qvti_create(const qvti_config* cfg, qvti_sim** out)
{
    using namespace qvti;
    if (!cfg || !out) return fail(QVTI_ERR_ARG);
    *out = nullptr;
    const int nx = cfg->ntx, ny = cfg->nty, nz = cfg->ntz;
    if (nx < 16 || ny < 16 || nz < 16 || nx > 1024 || ny > 1024 || nz > 1024) return fail(QVTI_ERR_UNSUPPORTED);
    if ((nx | ny | nz) & 1) return fail(QVTI_ERR_UNSUPPORTED);
    if (!smooth(nx) || !smooth(ny) || !smooth(nz)) return fail(QVTI_ERR_UNSUPPORTED);
    if (cfg->pml < 2 || 2 * cfg->pml >= nx || 2 * cfg->pml >= ny || 2 * cfg->pml >= nz) return fail(QVTI_ERR_ARG);
    if (!(cfg->dx > 0 && cfg->dy > 0 && cfg->dz > 0 && cfg->dt > 0 && cfg->f0 > 0)) return fail(QVTI_ERR_ARG);
    FftPlan px, py, pz;
    if (!make_plan(nx, &px) || !make_plan(ny, &py) || !make_plan(nz, &pz)) return fail(QVTI_ERR_UNSUPPORTED);

    QV_CUDA(cudaSetDevice(cfg->device));
    if (configure_device(cfg->device)) return fail(QVTI_ERR_CUDA);

    Sim* s = new (std::nothrow) qvti_sim();
    if (!s) return fail(QVTI_ERR_OOM);
    s->cfg = *cfg;
    s->nx = nx; s->ny = ny; s->nz = nz; s->nkz = nz / 2 + 1;
    s->ntp = (long long)nx * ny * nz;
    auto bail = [&](int code) { delete s; return fail(code); };
    if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) return bail(QVTI_ERR_CUDA);
    if (cudaEventCreate(&s->ev0) != cudaSuccess || cudaEventCreate(&s->ev1) != cudaSuccess) return bail(QVTI_ERR_CUDA);

    KP& k = s->kp;
    k.nx = nx; k.ny = ny; k.nz = nz; k.nkz = s->nkz; k.pml = cfg->pml;
    k.ntp = s->ntp;
    k.dt = cfg->dt;
    k.inv_ntp = (float)(1.0 / (double)s->ntp);
    k.px = px; k.py = py; k.pz = pz;
    // every launch of the step must fit the shared memory of one block
    // (e.g. nz = 512 needs more for its z tiles than an SM offers)
    if (step_smem_bytes(k) > kMaxSmem) return bail(QVTI_ERR_UNSUPPORTED);
    const long long ntp = s->ntp, nspec = (long long)s->nkz * nx * ny;

    // 1D tables
    float2 *twx, *twy, *twz, *Fx, *Bx, *Fy, *By, *Fz, *Bz;
    float *kx, *ky, *kz, *t[12];
    int rc = 0;
    rc |= s->alloc(&twx, nx); rc |= s->alloc(&twy, ny); rc |= s->alloc(&twz, nz);
    rc |= s->alloc(&Fx, nx); rc |= s->alloc(&Bx, nx); rc |= s->alloc(&Fy, ny); rc |= s->alloc(&By, ny);
    rc |= s->alloc(&Fz, nz); rc |= s->alloc(&Bz, nz);
    rc |= s->alloc(&kx, nx); rc |= s->alloc(&ky, ny); rc |= s->alloc(&kz, nz);
    for (int a = 0; a < 3; ++a)
        for (int j = 0; j < 4; ++j) rc |= s->alloc(&t[a * 4 + j], a == 0 ? nx : a == 1 ? ny : nz);
    if (rc) return bail(g_last_error);
    k.tw_x = twx; k.tw_y = twy; k.tw_z = twz;
    k.Fx = Fx; k.Bx = Bx; k.Fy = Fy; k.By = By; k.Fz = Fz; k.Bz = Bz;
    k.kx = kx; k.ky = ky; k.kz = kz;
    k.ax = t[0]; k.bx = t[1]; k.axh = t[2]; k.bxh = t[3];
    k.ay = t[4]; k.by = t[5]; k.ayh = t[6]; k.byh = t[7];
    k.az = t[8]; k.bz = t[9]; k.azh = t[10]; k.bzh = t[11];
    k_axis_tables<<<4, 256, 0, s->st>>>(nx, cfg->dx, cfg->f0, cfg->pml, twx, kx, Fx, Bx, t[0], t[1], t[2], t[3]);
    k_axis_tables<<<4, 256, 0, s->st>>>(ny, cfg->dy, cfg->f0, cfg->pml, twy, ky, Fy, By, t[4], t[5], t[6], t[7]);
    k_axis_tables<<<4, 256, 0, s->st>>>(nz, cfg->dz, cfg->f0, cfg->pml, twz, kz, Fz, Bz, t[8], t[9], t[10], t[11]);

    // full-grid arrays
    for (int c = 0; c < 3; ++c) rc |= s->alloc(&k.v[c], ntp);
    for (int c = 0; c < 6; ++c) rc |= s->alloc(&k.s[c], ntp);
    for (int c = 0; c < 3; ++c) rc |= s->alloc(&k.R[c], ntp);
    for (int c = 0; c < 6; ++c) rc |= s->alloc(&k.Q[c], ntp);
    // C-PML memory variables: slab storage (engine.cuh, slab_x/y/z)
    const int pml = cfg->pml;
    auto slab = [&](int axis) { return (size_t)slab_len(nx, ny, nz, pml, axis); };
    for (int c = 0; c < 9; ++c) rc |= s->alloc(&k.php[c], slab(c % 3));
    for (int c = 0; c < 8; ++c) rc |= s->alloc(&k.phn[c], slab(c < 3 ? 0 : c < 6 ? 1 : 2));
    for (int c = 0; c < 8; ++c) rc |= s->alloc(&k.qn[c], slab(c < 3 ? 0 : c < 6 ? 1 : 2));
    for (int c = 0; c < 6; ++c) rc |= s->alloc(&k.phs[c], slab(kPhsAxis[c]));
    for (int c = 0; c < 6; ++c) rc |= s->alloc(&k.qs[c], slab(kPhsAxis[c]));
    if (rc) return bail(g_last_error);
    float* mu[5];
    float* rinv[3];
    for (int c = 0; c < 5; ++c) rc |= s->alloc(&mu[c], ntp);
    for (int c = 0; c < 3; ++c) rc |= s->alloc(&rinv[c], ntp);
    for (int c = 0; c < 12; ++c) rc |= s->alloc(&s->coef[c], ntp);
    for (int c = 0; c < 3; ++c) rc |= s->alloc(&k.H[c], nspec);
    for (int c = 0; c < 3; ++c) rc |= s->alloc(&k.Hy[c], nspec);
    for (int c = 0; c < kNumG; ++c) {
        k.G[c] = nullptr;
        if (!is_gz(c)) rc |= s->alloc(&k.G[c], nspec);
    }
    // the y derivatives live where the x/y pipeline would have put them
    k.Yv[0] = k.G[16];  // dy vx
    k.Yv[1] = k.G[4];   // dy vy
    k.Yv[2] = k.G[25];  // dy vz
    rc |= s->alloc(&s->d_it, 1);
    rc |= s->alloc(&s->d_norm, 16);
    rc |= s->alloc(&s->d_bad, 4);
    rc |= s->alloc(&s->d_err, 1);
    rc |= s->alloc(&s->d_nonfinite, 1);
    float* dft16 = nullptr;
    rc |= s->alloc(&dft16, 4096);
    if (rc) return bail(g_last_error);
    launch_dft16_tables(dft16, s->st);
    if (cudaMemsetAsync(s->d_err, 0, sizeof(int), s->st) != cudaSuccess ||
        cudaMemsetAsync(s->d_nonfinite, 0, sizeof(int), s->st) != cudaSuccess)
        return bail(QVTI_ERR_CUDA);
    k.dft16 = dft16;
    k.err = s->d_err;
    k.form = kFormPlain;
    k.loss_scale = 1.0f;
    k.inj[0] = k.inj[1] = k.inj[2] = nullptr;
    k.inj_nt = 0;


    for (int j = 0; j < 5; ++j) k.MU[j] = mu[j];
    k.mrho = s->coef[0]; k.mgp = s->coef[1]; k.mgs = s->coef[2];
    k.mc33 = s->coef[4]; k.mcs = s->coef[6];
    // isotropic: c11 = c13 = c33, read from one array
    k.mc11 = cfg->vti ? s->coef[3] : s->coef[4];
    k.mc13 = cfg->vti ? s->coef[5] : s->coef[4];
    k.w0 = cfg->w0 > 0 ? cfg->w0 : (float)(2 * 3.1415926 * cfg->f0);  // viscoelas_3D.cpp:109
    // kz planes per batch of the k-space passes (k_cy fwd, k_mx, k_cy inv).
    // Batches of ~48 MB of spectra would keep a batch in L2 between k_mx and
    // the inverse y pass, but the small grids cost more than the saved HBM
    // traffic (measured at 256^3), so the default is one batch;
    // QVTI_KZ_BATCH overrides it for tuning.
    {
        int b = s->nkz;
        if (const char* e = getenv("QVTI_KZ_BATCH")) b = atoi(e);
        k.kz_batch = b < 1 ? 1 : (b > s->nkz ? s->nkz : b);
    }
    for (int c = 0; c < 3; ++c) k.rinv[c] = rinv[c];
    k.d_it = s->d_it;
    k.src_type = 0; k.s_ix = -1; k.s_iy = 0; k.s_iz = 0;
    k.rik = nullptr; k.nt_rec = 0; k.rn = 0; k.r_iz = 0; k.r_ix = nullptr; k.r_iy = nullptr;
    for (int c = 0; c < 3; ++c) k.rec[c] = nullptr;
    if (cudaStreamSynchronize(s->st) != cudaSuccess || cudaGetLastError() != cudaSuccess) return bail(QVTI_ERR_CUDA);
    *out = static_cast<qvti_sim*>(s);
    g_sims_created.fetch_add(1);
    return QVTI_OK;
}

extern "C" long long qvti_sims_created(void) { return qvti::g_sims_created.load(); }

extern "C" int qvti_get_config(const qvti_sim* s, qvti_config* cfg)
{
    if (!s || !cfg) return fail(QVTI_ERR_ARG);
    *cfg = s->cfg;
    return QVTI_OK;
}

extern "C" int qvti_destroy(qvti_sim* sim)
{
    if (!sim) return fail(QVTI_ERR_ARG);
    cudaSetDevice(sim->cfg.device);
    cudaStreamSynchronize(sim->st);
    delete sim;
    return QVTI_OK;
}

namespace qvti {
// The model upload and coefficient build, queued on the simulation's stream.
// Host arrays are staged in spectrum scratch arrays (G), which hold nothing
// between steps and are at least ntp floats each, so no device memory is
// allocated.  sync: return once the host arrays have been read (the
// contract of qvti_set_model); without it the caller keeps them valid until
// the stream has passed the upload.
int set_model_impl(Sim* s, const float* const host[7], int on_device, bool sync)
{
    QV_CUDA(cudaSetDevice(s->cfg.device));
    const size_t bytes = sizeof(float) * s->ntp;
    const int nin = s->cfg.vti ? 7 : 5;
    const float* dev[7] = {};
    if (on_device) {
        for (int i = 0; i < nin; ++i) dev[i] = host[i];
    } else {
        int o = 0;
        for (int i = 0; i < nin; ++i) {
            while (is_gz(o)) ++o;  // the kz-only fields have no G array
            float* stage = reinterpret_cast<float*>(s->kp.G[o++]);
            QV_CUDA(cudaMemcpyAsync(stage, host[i], bytes, cudaMemcpyHostToDevice, s->st));
            dev[i] = stage;
        }
    }
    if (s->ensure(&s->d_coefp, &s->coefp_cap, 12)) return g_last_error;
    QV_CUDA(cudaMemcpyAsync(s->d_coefp, s->coef, sizeof(float*) * 12, cudaMemcpyHostToDevice, s->st));
    launch_coef_build(s->kp, dev[0], dev[1], dev[2], dev[3], dev[4], s->cfg.vti ? dev[5] : nullptr,
                      s->cfg.vti ? dev[6] : nullptr, s->cfg.vti, s->kp.w0, s->media == QVTI_MEDIA_LOSSLESS,
                      s->d_coefp, s->st);
    launch_mu_rinv(s->kp, dev[2], s->coef + 7, s->st);
    QV_CUDA(cudaGetLastError());
    if (sync) QV_CUDA(cudaStreamSynchronize(s->st));
    s->have_model = true;
    return QVTI_OK;
}
}  // namespace qvti

extern "C" int qvti_set_model(qvti_sim* s, const float* velp, const float* vels, const float* rho, const float* gama_p,
                              const float* gama_s, const float* eps, const float* delta, int on_device)
{
    using namespace qvti;
    if (!s || !velp || !vels || !rho || !gama_p || !gama_s) return fail(QVTI_ERR_ARG);
    if (s->cfg.vti && (!eps || !delta)) return fail(QVTI_ERR_ARG);
    const float* host[7] = {velp, vels, rho, gama_p, gama_s, eps, delta};
    return set_model_impl(s, host, on_device, true);
}

extern "C" int qvti_set_source(qvti_sim* s, int type, int s_ix, int s_iy, int s_iz, const float* wavelet, int nt)
{
    using namespace qvti;
    if (!s || !wavelet || nt <= 0 || (type != QVTI_SRC_FORCE_X && type != QVTI_SRC_EXPLOSIVE)) return fail(QVTI_ERR_ARG);
    QV_CUDA(cudaSetDevice(s->cfg.device));
    QV_CUDA(cudaStreamSynchronize(s->st));
    if (s->ensure(&s->d_rik, &s->rik_cap, nt)) return g_last_error;
    // every upload and clear goes through the simulation's stream: it does not
    // synchronise with the legacy stream, and a pageable upload may return
    // before its transfer has landed
    QV_CUDA(cudaMemcpyAsync(s->d_rik, wavelet, sizeof(float) * nt, cudaMemcpyHostToDevice, s->st));
    s->nt = nt;
    KP& k = s->kp;
    k.src_type = type;
    const bool inside = s_ix >= 0 && s_ix < s->nx && s_iy >= 0 && s_iy < s->ny && s_iz >= 0 && s_iz < s->nz;
    k.s_ix = inside ? s_ix : -1;
    k.s_iy = s_iy;
    k.s_iz = s_iz;
    k.rik = s->d_rik;
    k.nt_rec = nt;
    for (int c = 0; c < 3; ++c) k.rec[c] = nullptr;
    if (s->rn > 0) {
        size_t cap = s->rec_cap;
        for (int c = 0; c < 3; ++c) {
            cap = s->rec_cap;
            if (s->ensure(&s->d_rec[c], &cap, (size_t)nt * s->rn)) return g_last_error;
            QV_CUDA(cudaMemsetAsync(s->d_rec[c], 0, sizeof(float) * (size_t)nt * s->rn, s->st));
            k.rec[c] = s->d_rec[c];
        }
        s->rec_cap = cap;
    }
    s->have_src = true;
    s->drop_graphs();
    return QVTI_OK;
}

extern "C" int qvti_set_receivers(qvti_sim* s, int r_iz, const int* r_ix, const int* r_iy, int rn)
{
    using namespace qvti;
    if (!s || rn < 0 || (rn > 0 && (!r_ix || !r_iy)) || r_iz < 0 || r_iz >= s->nz) return fail(QVTI_ERR_ARG);
    for (int i = 0; i < rn; ++i)
        if (r_ix[i] < 0 || r_ix[i] >= s->nx || r_iy[i] < 0 || r_iy[i] >= s->ny) return fail(QVTI_ERR_ARG);
    QV_CUDA(cudaSetDevice(s->cfg.device));
    QV_CUDA(cudaStreamSynchronize(s->st));
    KP& k = s->kp;
    s->rn = rn;
    k.rn = rn;
    k.r_iz = r_iz;
    if (rn > 0) {
        size_t cap = s->rix_cap;
        if (s->ensure(&s->d_rix, &cap, rn)) return g_last_error;
        cap = s->rix_cap;
        if (s->ensure(&s->d_riy, &cap, rn)) return g_last_error;
        s->rix_cap = cap;
        QV_CUDA(cudaMemcpyAsync(s->d_rix, r_ix, sizeof(int) * rn, cudaMemcpyHostToDevice, s->st));
        QV_CUDA(cudaMemcpyAsync(s->d_riy, r_iy, sizeof(int) * rn, cudaMemcpyHostToDevice, s->st));
    }
    k.r_ix = s->d_rix;
    k.r_iy = s->d_riy;
    for (int c = 0; c < 3; ++c) k.rec[c] = nullptr;
    if (rn > 0 && s->nt > 0) {
        size_t cap = s->rec_cap;
        for (int c = 0; c < 3; ++c) {
            cap = s->rec_cap;
            if (s->ensure(&s->d_rec[c], &cap, (size_t)s->nt * rn)) return g_last_error;
            QV_CUDA(cudaMemsetAsync(s->d_rec[c], 0, sizeof(float) * (size_t)s->nt * rn, s->st));
            k.rec[c] = s->d_rec[c];
        }
        s->rec_cap = cap;
    }
    s->drop_graphs();
    return QVTI_OK;
}

namespace qvti {
// State cleared on the simulation's stream; sync: wait for it.
int reset_impl(Sim* s, bool sync)
{
    QV_CUDA(cudaSetDevice(s->cfg.device));
    KP& k = s->kp;
    const size_t b = sizeof(float) * s->ntp;
    for (int c = 0; c < 3; ++c) QV_CUDA(cudaMemsetAsync(k.v[c], 0, b, s->st));
    for (int c = 0; c < 6; ++c) QV_CUDA(cudaMemsetAsync(k.s[c], 0, b, s->st));
    for (int c = 0; c < 3; ++c) QV_CUDA(cudaMemsetAsync(k.R[c], 0, b, s->st));
    for (int c = 0; c < 6; ++c) QV_CUDA(cudaMemsetAsync(k.Q[c], 0, b, s->st));
    float* sl[kNumSlab];
    size_t sn[kNumSlab];
    slab_arrays(k, sl, sn);
    for (int c = 0; c < kNumSlab; ++c) QV_CUDA(cudaMemsetAsync(sl[c], 0, sizeof(float) * sn[c], s->st));
    const int minus1 = -1;
    QV_CUDA(cudaMemcpyAsync(s->d_it, &minus1, sizeof(int), cudaMemcpyHostToDevice, s->st));
    QV_CUDA(cudaMemsetAsync(s->d_err, 0, sizeof(int), s->st));
    QV_CUDA(cudaMemsetAsync(s->d_nonfinite, 0, sizeof(int), s->st));
    for (int c = 0; c < 3; ++c)
        if (s->d_rec[c]) QV_CUDA(cudaMemsetAsync(s->d_rec[c], 0, sizeof(float) * (size_t)s->nt * s->rn, s->st));
    if (sync) QV_CUDA(cudaStreamSynchronize(s->st));
    s->steps = 0;
    return QVTI_OK;
}
}  // namespace qvti

extern "C" int qvti_reset(qvti_sim* s)
{
    using namespace qvti;
    if (!s) return fail(QVTI_ERR_ARG);
    return reset_impl(s, true);
}

extern "C" int qvti_step(qvti_sim* s, int nsteps)
{
    using namespace qvti;
    if (!s || nsteps < 0) return fail(QVTI_ERR_ARG);
    if (!s->have_model || !s->have_src) return fail(QVTI_ERR_STATE);
    if (s->steps + nsteps > s->nt) return fail(QVTI_ERR_ARG);  // wavelet / record capacity
    QV_CUDA(cudaSetDevice(s->cfg.device));
    int left = nsteps;
    if (left >= kGraphSteps) {
        if (!s->gexec_n) {
            int rc = build_graph(s, kGraphSteps, &s->gexec_n);
            if (rc) return rc;
        }
        for (; left >= kGraphSteps; left -= kGraphSteps) QV_CUDA(cudaGraphLaunch(s->gexec_n, s->st));
    }
    if (left > 0 && !s->gexec) {
        int rc = build_graph(s);
        if (rc) return rc;
    }
    for (; left > 0; --left) QV_CUDA(cudaGraphLaunch(s->gexec, s->st));
    s->steps += nsteps;
    return QVTI_OK;
}

extern "C" int qvti_step_timed(qvti_sim* s, int nsteps, float* ms)
{
    using namespace qvti;
    if (!s || !ms) return fail(QVTI_ERR_ARG);
    QV_CUDA(cudaSetDevice(s->cfg.device));
    // both graphs the call replays are built before the first event
    if (s->have_model && s->have_src) {
        if (!s->gexec) {
            int rc = build_graph(s);
            if (rc) return rc;
        }
        if (nsteps >= kGraphSteps && !s->gexec_n) {
            int rc = build_graph(s, kGraphSteps, &s->gexec_n);
            if (rc) return rc;
        }
    }
    QV_CUDA(cudaStreamSynchronize(s->st));
    QV_CUDA(cudaEventRecord(s->ev0, s->st));
    int rc = qvti_step(s, nsteps);
    if (rc) return rc;
    QV_CUDA(cudaEventRecord(s->ev1, s->st));
    QV_CUDA(cudaEventSynchronize(s->ev1));
    QV_CUDA(cudaEventElapsedTime(ms, s->ev0, s->ev1));
    return QVTI_OK;
}

namespace qvti {
// After the simulation's stream is idle: a kernel that gave up a bounded wait
// left a status in the device error flag.
int device_status(Sim* s)
{
    int e = 0;
    QV_CUDA(cudaMemcpy(&e, s->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    return e ? fail(e) : QVTI_OK;
}
}  // namespace qvti

extern "C" int qvti_sync(qvti_sim* s)
{
    using namespace qvti;
    if (!s) return fail(QVTI_ERR_ARG);
    QV_CUDA(cudaSetDevice(s->cfg.device));
    QV_CUDA(cudaStreamSynchronize(s->st));
    return device_status(s);
}

extern "C" int qvti_steps_done(const qvti_sim* s) { return s ? s->steps : -1; }

extern "C" int qvti_get_records(qvti_sim* s, float* vx, float* vy, float* vz)
{
    using namespace qvti;
    if (!s) return fail(QVTI_ERR_ARG);
    QV_CUDA(cudaSetDevice(s->cfg.device));
    QV_CUDA(cudaStreamSynchronize(s->st));
    float* dst[3] = {vx, vy, vz};
    const size_t n = (size_t)s->steps * s->rn;
    for (int c = 0; c < 3; ++c)
        if (dst[c] && n && s->d_rec[c]) QV_CUDA(cudaMemcpy(dst[c], s->d_rec[c], n * sizeof(float), cudaMemcpyDeviceToHost));
    return device_status(s);
}

static float* field_ptr(qvti_sim* s, int which)
{
    if (which < 3) return s->kp.v[which];
    static const int smap[6] = {0, 1, 2, 3, 4, 5};  // pxx pyy pzz pxy pxz pyz
    return s->kp.s[smap[which - 3]];
}

extern "C" int qvti_get_fields(qvti_sim* s, int first, int count, float* out)
{
    using namespace qvti;
    if (!s || !out || first < 0 || count < 0 || first + count > 9) return fail(QVTI_ERR_ARG);
    QV_CUDA(cudaSetDevice(s->cfg.device));
    QV_CUDA(cudaStreamSynchronize(s->st));
    for (int f = 0; f < count; ++f)
        QV_CUDA(cudaMemcpy(out + (size_t)f * s->ntp, field_ptr(s, first + f), sizeof(float) * s->ntp,
                           cudaMemcpyDeviceToHost));
    return QVTI_OK;
}

extern "C" int qvti_device_field(qvti_sim* s, int which, float** p)
{
    if (!s || !p || which < 0 || which > 8) return qvti::fail(QVTI_ERR_ARG);
    *p = field_ptr(s, which);
    return QVTI_OK;
}

extern "C" int qvti_check_finite_async(qvti_sim* s, int* host_flag)
{
    using namespace qvti;
    if (!s) return fail(QVTI_ERR_ARG);
    QV_CUDA(cudaSetDevice(s->cfg.device));
    k_finite3<<<148 * 4, 256, 0, s->st>>>(s->ntp / 4, reinterpret_cast<const float4*>(s->kp.v[0]),
                                          reinterpret_cast<const float4*>(s->kp.v[1]),
                                          reinterpret_cast<const float4*>(s->kp.v[2]), s->d_nonfinite);
    QV_CUDA(cudaGetLastError());
    if (host_flag)
        QV_CUDA(cudaMemcpyAsync(host_flag, s->d_nonfinite, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    return QVTI_OK;
}

extern "C" int qvti_field_norms(qvti_sim* s, double* norms9, int* nonfinite)
{
    using namespace qvti;
    if (!s || !norms9) return fail(QVTI_ERR_ARG);
    QV_CUDA(cudaSetDevice(s->cfg.device));
    int bad_all = 0;
    for (int f = 0; f < 9; ++f) {
        QV_CUDA(cudaMemsetAsync(s->d_norm, 0, sizeof(double), s->st));
        QV_CUDA(cudaMemsetAsync(s->d_bad, 0, sizeof(int), s->st));
        k_norms<<<148 * 4, 256, 0, s->st>>>(s->ntp, field_ptr(s, f), s->d_norm, s->d_bad);
        double acc = 0;
        int bad = 0;
        QV_CUDA(cudaMemcpyAsync(&acc, s->d_norm, sizeof(double), cudaMemcpyDeviceToHost, s->st));
        QV_CUDA(cudaMemcpyAsync(&bad, s->d_bad, sizeof(int), cudaMemcpyDeviceToHost, s->st));
        QV_CUDA(cudaStreamSynchronize(s->st));
        norms9[f] = acc;
        bad_all |= bad;
    }
    if (nonfinite) *nonfinite = bad_all;
    return bad_all ? fail(QVTI_ERR_NONFINITE) : QVTI_OK;
}

// ------------------------------------------------------ checkpoint / resume --
namespace {

// Snapshot layout: this header, then kStateArrays float arrays in
// state_arrays() order (18 full-grid arrays, then the 37 C-PML slab arrays,
// each its own length), then the records of the steps done (vx, vy, vz, each
// [step][receiver]).  Grid, spacing, dt, C-PML width and medium type are in
// the header so a snapshot cannot resume a different simulation.
struct StateHeader {
    char magic[8];
    int32_t ntx, nty, ntz, pml;
    int32_t vti, n_arrays, steps, rn;
    float dx, dy, dz, dt;
    uint64_t array_bytes, total_bytes;  // all state arrays together; the whole snapshot
};
static_assert(sizeof(StateHeader) == 72, "snapshot header layout");
constexpr char kStateMagic[8] = {'Q', 'V', 'T', 'I', 'S', 'T', '0', '2'};
constexpr int kStateArrays = 3 + 6 + 3 + 6 + qvti::kNumSlab;

int state_arrays(Sim* s, float** out, size_t* bytes)
{
    qvti::KP& k = s->kp;
    int n = 0;
    const size_t full = sizeof(float) * (size_t)s->ntp;
    for (float* p : k.v) { out[n] = p; bytes[n++] = full; }
    for (float* p : k.s) { out[n] = p; bytes[n++] = full; }
    for (float* p : k.R) { out[n] = p; bytes[n++] = full; }
    for (float* p : k.Q) { out[n] = p; bytes[n++] = full; }
    size_t len[qvti::kNumSlab];
    const int ns = qvti::slab_arrays(k, out + n, len);
    for (int i = 0; i < ns; ++i) bytes[n + i] = sizeof(float) * len[i];
    return n + ns;
}

StateHeader state_header(Sim* s)
{
    StateHeader h{};
    memcpy(h.magic, kStateMagic, sizeof(h.magic));
    h.ntx = s->nx; h.nty = s->ny; h.ntz = s->nz; h.pml = s->cfg.pml;
    h.vti = s->cfg.vti ? 1 : 0;
    h.n_arrays = kStateArrays;
    h.steps = s->steps;
    h.rn = s->rn;
    h.dx = s->cfg.dx; h.dy = s->cfg.dy; h.dz = s->cfg.dz; h.dt = s->cfg.dt;
    float* arr[kStateArrays];
    size_t b[kStateArrays];
    state_arrays(s, arr, b);
    h.array_bytes = 0;
    for (size_t x : b) h.array_bytes += x;
    const uint64_t rec = s->rn > 0 && s->d_rec[0] ? 3ull * s->steps * s->rn * sizeof(float) : 0;
    h.total_bytes = sizeof(StateHeader) + h.array_bytes + rec;
    return h;
}

}  // namespace

extern "C" int qvti_state_bytes(qvti_sim* s, size_t* bytes)
{
    if (!s || !bytes) return fail(QVTI_ERR_ARG);
    *bytes = (size_t)state_header(s).total_bytes;
    return QVTI_OK;
}

extern "C" int qvti_save_state(qvti_sim* s, void* host, size_t bytes)
{
    using namespace qvti;
    if (!s || !host) return fail(QVTI_ERR_ARG);
    const StateHeader h = state_header(s);
    if (bytes < h.total_bytes) return fail(QVTI_ERR_ARG);
    QV_CUDA(cudaSetDevice(s->cfg.device));
    char* dst = static_cast<char*>(host);
    memcpy(dst, &h, sizeof(h));
    dst += sizeof(h);
    float* arr[kStateArrays];
    size_t ab[kStateArrays];
    state_arrays(s, arr, ab);
    for (int i = 0; i < kStateArrays; ++i) {
        QV_CUDA(cudaMemcpyAsync(dst, arr[i], ab[i], cudaMemcpyDeviceToHost, s->st));
        dst += ab[i];
    }
    const size_t rec = sizeof(float) * (size_t)h.steps * h.rn;
    if (h.total_bytes > sizeof(h) + h.array_bytes)
        for (int c = 0; c < 3; ++c) {
            QV_CUDA(cudaMemcpyAsync(dst, s->d_rec[c], rec, cudaMemcpyDeviceToHost, s->st));
            dst += rec;
        }
    QV_CUDA(cudaStreamSynchronize(s->st));
    return QVTI_OK;
}

extern "C" int qvti_load_state(qvti_sim* s, const void* host, size_t bytes)
{
    using namespace qvti;
    if (!s || !host || bytes < sizeof(StateHeader)) return fail(QVTI_ERR_ARG);
    if (!s->have_src) return fail(QVTI_ERR_STATE);
    StateHeader h;
    memcpy(&h, host, sizeof(h));
    const StateHeader mine = state_header(s);
    const bool same = memcmp(h.magic, kStateMagic, sizeof(h.magic)) == 0 && h.ntx == mine.ntx &&
                      h.nty == mine.nty && h.ntz == mine.ntz && h.pml == mine.pml && h.vti == mine.vti &&
                      h.n_arrays == kStateArrays && h.array_bytes == mine.array_bytes &&
                      memcmp(&h.dx, &mine.dx, 4 * sizeof(float)) == 0;
    if (!same || h.steps < 0 || h.steps > s->nt || h.rn != s->rn) return fail(QVTI_ERR_ARG);
    const uint64_t rec = sizeof(float) * (uint64_t)h.steps * h.rn;
    const bool with_rec = h.rn > 0 && s->d_rec[0];
    const uint64_t want = sizeof(h) + h.array_bytes + (with_rec ? 3 * rec : 0);
    if (h.total_bytes != want || bytes < want) return fail(QVTI_ERR_ARG);
    QV_CUDA(cudaSetDevice(s->cfg.device));
    const char* src = static_cast<const char*>(host) + sizeof(h);
    float* arr[kStateArrays];
    size_t ab[kStateArrays];
    state_arrays(s, arr, ab);
    for (int i = 0; i < kStateArrays; ++i) {
        QV_CUDA(cudaMemcpyAsync(arr[i], src, ab[i], cudaMemcpyHostToDevice, s->st));
        src += ab[i];
    }
    if (with_rec) {
        const size_t all = sizeof(float) * (size_t)s->nt * s->rn;
        for (int c = 0; c < 3; ++c) {
            QV_CUDA(cudaMemsetAsync(s->d_rec[c], 0, all, s->st));
            if (rec) QV_CUDA(cudaMemcpyAsync(s->d_rec[c], src, rec, cudaMemcpyHostToDevice, s->st));
            src += rec;
        }
    }
    // the step kernels advance the counter first: after n steps it holds n - 1
    const int it = h.steps - 1;
    QV_CUDA(cudaMemcpyAsync(s->d_it, &it, sizeof(int), cudaMemcpyHostToDevice, s->st));
    QV_CUDA(cudaStreamSynchronize(s->st));
    s->steps = h.steps;
    return QVTI_OK;
}

extern "C" int qvti_forward_shot(qvti_sim* s, const float* velp, const float* vels, const float* rho,
                                 const float* gama_p, const float* gama_s, const float* eps, const float* delta,
                                 int src_type, int s_ix, int s_iy, int s_iz, const float* wavelet, int nt, int r_iz,
                                 const int* r_ix, const int* r_iy, int rn, float* rec_vx, float* rec_vy, float* rec_vz)
{
    using namespace qvti;
    if (!s || !velp || !vels || !rho || !gama_p || !gama_s) return fail(QVTI_ERR_ARG);
    if (s->cfg.vti && (!eps || !delta)) return fail(QVTI_ERR_ARG);
    int rc;
    // receivers and source first (each waits for the stream to be idle);
    // then the model upload and the state clear are queued without a wait,
    // so the step graphs are built on the host while the copy engines move
    // the model; the host arrays stay valid until this call returns
    if ((rc = qvti_set_receivers(s, r_iz, r_ix, r_iy, rn))) return rc;
    if ((rc = qvti_set_source(s, src_type, s_ix, s_iy, s_iz, wavelet, nt))) return rc;
    const float* host[7] = {velp, vels, rho, gama_p, gama_s, eps, delta};
    if ((rc = set_model_impl(s, host, 0, false))) return rc;
    if ((rc = reset_impl(s, false))) return rc;
    if ((rc = qvti_step(s, nt))) return rc;
    return qvti_get_records(s, rec_vx, rec_vy, rec_vz);
}

extern "C" int qvti_derivative_1d(qvti_sim* s, int axis, int fwd, const float* in, float* out)
{
    using namespace qvti;
    if (!s || !in || !out || axis < 0 || axis > 2) return fail(QVTI_ERR_ARG);
    QV_CUDA(cudaSetDevice(s->cfg.device));
    const size_t b = sizeof(float) * s->ntp;
    DevBuf din, dout;  // freed on every return
    QV_CUDA(cudaMalloc(&din.p, b));
    QV_CUDA(cudaMalloc(&dout.p, b));
    QV_CUDA(cudaMemcpyAsync(din.p, in, b, cudaMemcpyHostToDevice, s->st));  // ordered before the launches
    launch_derivative_1d(s->kp, axis, fwd, din.f(), dout.f(), s->st);
    QV_CUDA(cudaGetLastError());
    QV_CUDA(cudaStreamSynchronize(s->st));
    QV_CUDA(cudaMemcpy(out, dout.p, b, cudaMemcpyDeviceToHost));
    return QVTI_OK;
}

// Algorithmic HBM bytes of each step kernel: the reads and writes its job
// needs once each (full-grid fields, half spectra, C-PML variables in their
// slabs only), no re-reads.
static void kernel_bytes(const qvti_sim* s, double* b)
{
    const double F = 4.0 * s->ntp, S = 8.0 * s->nkz * (double)s->nx * s->ny;
    const int pml = s->cfg.pml;
    auto slab = [&](int n) { int c = 0; for (int i = 0; i < n - 1; ++i) c += (i < pml || i >= n - pml); return (double)c; };
    const double gx = s->nx - 1, gy = s->ny - 1, gz = s->nz - 1;
    const double cx = slab(s->nx) * gy * gz, cy = slab(s->ny) * gx * gz, cz = slab(s->nz) * gx * gy;
    const double model = (s->cfg.vti ? 7 : 5) * F;
    b[0] = 3 * F + 6 * F + 24 * cy;                                        // k_vy
    b[1] = 3 * F + 6 * F + 3 * F + 3 * F + 24 * cx;                        // k_vx
    b[2] = 3 * F + 3 * S;                                                  // k_fz
    b[3] = 3 * 3 * S;                                                      // k_cy_fwd (H -> Hy, Yv)
    b[4] = 3 * S + qvti::kNumGxy * S;                                      // k_mx
    b[5] = qvti::kNumGxy * 2 * S;                                          // k_cy_inv
    // k_sigma: 27 half spectra (21 G, 3 H, 3 Yv), 6 stresses and 6 loss potentials read+written,
    // model + MU, 3 R written, C-PML variables in their slabs
    b[6] = qvti::kNumG * S + 12 * F + 12 * F + model + 5 * F + 3 * F + 3 * 8 * cz +
           (48 + 16 + 16) * cx + (48 + 16 + 16) * cy + (32 + 16 + 16) * cz;
    b[7] = s->rn * (3 * 4.0 * 2 + 8.0);                                    // k_rec
}

// Per-kernel device time of the step (CUDA events between the kernels of
// nrep consecutive steps on the simulation's stream; the steps advance the
// state like qvti_step).  names: maxk*32 chars; ms, bytes: maxk each;
// *nkernels receives the number of kernels per step.
extern "C" int qvti_profile_step(qvti_sim* s, int nrep, int maxk, int* nkernels, char* names, float* ms,
                                 double* bytes)
{
    using namespace qvti;
    if (!s || nrep <= 0 || maxk < kStepKernels) return fail(QVTI_ERR_ARG);
    if (!s->have_model || !s->have_src) return fail(QVTI_ERR_STATE);
    if (s->steps + nrep > s->nt) return fail(QVTI_ERR_ARG);
    QV_CUDA(cudaSetDevice(s->cfg.device));
    StepProfile* prof = new StepProfile();
    for (auto& e : prof->ev) QV_CUDA(cudaEventCreate(&e));
    std::vector<double> acc(kStepKernels, 0.0);
    int rc = QVTI_OK;
    for (int r = 0; r < nrep && rc == QVTI_OK; ++r) {
        prof->n = 0;
        launch_step(s->kp, s->st, prof);
        if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(prof->ev[prof->n - 1]) != cudaSuccess) {
            rc = fail(QVTI_ERR_CUDA);
            break;
        }
        for (int i = 1; i < prof->n; ++i) {
            float t = 0;
            cudaEventElapsedTime(&t, prof->ev[i - 1], prof->ev[i]);
            if (prof->kind[i] >= 0 && prof->kind[i] < kStepKernels) acc[prof->kind[i]] += t;
        }
        s->steps += 1;
    }
    for (auto& e : prof->ev) cudaEventDestroy(e);
    delete prof;
    if (rc) return rc;
    double b[kStepKernels];
    kernel_bytes(s, b);
    for (int i = 0; i < kStepKernels; ++i) {
        if (names) { std::strncpy(names + 32 * i, kStepKernelNames[i], 31); names[32 * i + 31] = 0; }
        if (ms) ms[i] = (float)(acc[i] / nrep);
        if (bytes) bytes[i] = b[i];
    }
    if (nkernels) *nkernels = kStepKernels;
    return QVTI_OK;
}

extern "C" int qvti_q_derivative(qvti_sim* s, int axis, int fwd, int power, const float* in, float* out)
{
    using namespace qvti;
    if (!s || !in || !out || axis < 0 || axis > 2 || power < -1 || power > 1) return fail(QVTI_ERR_ARG);
    QV_CUDA(cudaSetDevice(s->cfg.device));
    QV_CUDA(cudaStreamSynchronize(s->st));
    const size_t b = sizeof(float) * s->ntp;
    DevBuf din, dout;  // freed on every return
    QV_CUDA(cudaMalloc(&din.p, b));
    QV_CUDA(cudaMalloc(&dout.p, b));
    QV_CUDA(cudaMemcpyAsync(din.p, in, b, cudaMemcpyHostToDevice, s->st));  // ordered before the launches
    KP k = s->kp;
    k.v[0] = din.f();
    k.H[0] = s->kp.G[0];  // scratch: rewritten by every time step anyway
    k.G[0] = s->kp.G[0];
    launch_q_derivative(k, axis, fwd, power, dout.f(), s->st);
    QV_CUDA(cudaGetLastError());
    QV_CUDA(cudaStreamSynchronize(s->st));
    QV_CUDA(cudaMemcpy(out, dout.p, b, cudaMemcpyDeviceToHost));
    return QVTI_OK;
}

extern "C" int qvti_get_stream(qvti_sim* s, void** stream)
{
    if (!s || !stream) return qvti::fail(QVTI_ERR_ARG);
    *stream = static_cast<void*>(s->st);
    return QVTI_OK;
}

extern "C" int qvti_set_kz_batch(qvti_sim* s, int kz_batch)
{
    using namespace qvti;
    if (!s || kz_batch < 1 || kz_batch > s->nkz) return fail(QVTI_ERR_ARG);
    if (s->kp.kz_batch != kz_batch) {
        s->kp.kz_batch = kz_batch;
        s->drop_graphs();
    }
    return QVTI_OK;
}

extern "C" int qvti_set_media(qvti_sim* s, int media)
{
    using namespace qvti;
    if (!s || media < QVTI_MEDIA_VISCOELASTIC || media > QVTI_MEDIA_Q_COMPENSATED) return fail(QVTI_ERR_ARG);
    s->media = media;
    const float ls = media == QVTI_MEDIA_VISCOELASTIC ? 1.0f : media == QVTI_MEDIA_Q_COMPENSATED ? -1.0f : 0.0f;
    if (s->kp.loss_scale != ls) {
        s->kp.loss_scale = ls;
        s->drop_graphs();
    }
    // the lossless medium's coefficients are built without gamma: a model
    // set before this call is out of date
    s->have_model = false;
    return QVTI_OK;
}

extern "C" int qvti_set_injection(qvti_sim* s, const float* vx, const float* vy, const float* vz, int nt)
{
    using namespace qvti;
    if (!s || nt < 0 || (nt > 0 && !vx && !vy && !vz)) return fail(QVTI_ERR_ARG);
    if (nt > 0 && s->rn <= 0) return fail(QVTI_ERR_STATE);  // injected at the receivers
    QV_CUDA(cudaSetDevice(s->cfg.device));
    QV_CUDA(cudaStreamSynchronize(s->st));
    const float* host[3] = {vx, vy, vz};
    KP& k = s->kp;
    for (int c = 0; c < 3; ++c) {
        k.inj[c] = nullptr;
        if (nt == 0 || !host[c]) continue;
        const size_t n = (size_t)nt * s->rn;
        if (s->ensure(&s->d_inj[c], &s->inj_cap[c], n)) return g_last_error;
        QV_CUDA(cudaMemcpyAsync(s->d_inj[c], host[c], sizeof(float) * n, cudaMemcpyHostToDevice, s->st));
        k.inj[c] = s->d_inj[c];
    }
    k.inj_nt = nt;
    QV_CUDA(cudaStreamSynchronize(s->st));
    s->drop_graphs();
    return QVTI_OK;
}

extern "C" int qvti_set_form(qvti_sim* s, int form)
{
    using namespace qvti;
    if (!s || (form != QVTI_FORM_PLAIN && form != QVTI_FORM_TC)) return fail(QVTI_ERR_ARG);
    KP probe = s->kp;
    probe.form = form == QVTI_FORM_TC ? kFormTc : kFormPlain;
    if (form == QVTI_FORM_TC && !tc_cy_available(probe)) return fail(QVTI_ERR_UNSUPPORTED);
    if (s->kp.form != probe.form) {
        s->kp.form = probe.form;
        s->drop_graphs();
    }
    return QVTI_OK;
}

extern "C" int qvti_set_tiles(qvti_sim* s, const int tiles[QVTI_NUM_TILES])
{
    using namespace qvti;
    static_assert(QVTI_NUM_TILES == kNumTiled, "one tile per step kernel");
    if (!s || !tiles) return fail(QVTI_ERR_ARG);
    KP probe = s->kp;
    bool same = true;
    for (int i = 0; i < kNumTiled; ++i) {
        probe.tile_rt[i] = tiles[i];
        same = same && tiles[i] == s->kp.tile_rt[i];
    }
    if (!tiles_valid(probe)) return fail(QVTI_ERR_UNSUPPORTED);
    if (!same) {
        s->kp = probe;
        s->drop_graphs();
    }
    return QVTI_OK;
}

extern "C" int qvti_get_tiles(qvti_sim* s, int tiles[QVTI_NUM_TILES], int runtime[QVTI_NUM_TILES])
{
    using namespace qvti;
    if (!s) return fail(QVTI_ERR_ARG);
    step_tile_set(s->kp, tiles, runtime);
    return QVTI_OK;
}

extern "C" int qvti_autotune_tiles(qvti_sim* s, int probe_steps, int best[QVTI_NUM_TILES], float ms_out[QVTI_NUM_TILES])
{
    using namespace qvti;
    if (!s || probe_steps < 1) return fail(QVTI_ERR_ARG);
    if (!s->have_model || !s->have_src) return fail(QVTI_ERR_STATE);
    if (s->nt < probe_steps + 1) return fail(QVTI_ERR_ARG);
    // the step kernels' profile slots each tile setting times: k_vy, k_vx,
    // k_fz, k_cy (forward + inverse), k_mx, k_sigma
    auto kernel_ms = [](int i, const float* ms) {
        switch (i) {
            case 0: return ms[0];
            case 1: return ms[1];
            case 2: return ms[2];
            case 3: return ms[3] + ms[5];
            case 4: return ms[4];
            default: return ms[6];
        }
    };
    int chosen[kNumTiled] = {};
    float chosen_ms[kNumTiled] = {};
    auto time_of = [&](int i, const int* tiles, float* t) -> int {
        float ms[kStepKernels];
        int rc;
        if ((rc = qvti_set_tiles(s, tiles)) || (rc = qvti_reset(s)) ||
            (rc = qvti_profile_step(s, 1, kStepKernels, nullptr, nullptr, ms, nullptr)) ||
            (rc = qvti_profile_step(s, probe_steps, kStepKernels, nullptr, nullptr, ms, nullptr)))
            return rc;
        *t = kernel_ms(i, ms);
        return QVTI_OK;
    };
    int saved[kNumTiled];
    std::memcpy(saved, s->kp.tile_rt, sizeof saved);
    int rc = QVTI_OK;
    for (int i = 0; i < kNumTiled && rc == QVTI_OK; ++i) {
        int cand[kNumTiled];
        std::memcpy(cand, chosen, sizeof cand);
        cand[i] = 0;
        float t_def = 0.f;
        if ((rc = time_of(i, cand, &t_def))) break;
        float t_best = t_def;
        for (int t : {2, 4, 8, 16, 32}) {
            cand[i] = t;
            KP probe = s->kp;
            std::memcpy(probe.tile_rt, cand, sizeof cand);
            if (!tiles_valid(probe)) continue;
            float tt = 0.f;
            if ((rc = time_of(i, cand, &tt))) break;
            if (tt < 0.97f * t_def && tt < t_best) {
                t_best = tt;
                chosen[i] = t;
            }
        }
        chosen_ms[i] = t_best;
    }
    if (rc) {
        qvti_set_tiles(s, saved);
        qvti_reset(s);
        return rc;
    }
    if ((rc = qvti_set_tiles(s, chosen)) || (rc = qvti_reset(s))) return rc;
    for (int i = 0; i < kNumTiled; ++i) {
        if (best) best[i] = chosen[i];
        if (ms_out) ms_out[i] = chosen_ms[i];
    }
    return QVTI_OK;
}

extern "C" int qvti_probe_bounded_wait(qvti_sim* s, double seconds)
{
    using namespace qvti;
    if (!s || !(seconds > 0.0 && seconds <= 2.0)) return fail(QVTI_ERR_ARG);
    QV_CUDA(cudaSetDevice(s->cfg.device));
    int clock_khz = 0;
    QV_CUDA(cudaDeviceGetAttribute(&clock_khz, cudaDevAttrClockRate, s->cfg.device));
    launch_wait_probe(s->d_err, (long long)(seconds * 1e3 * clock_khz), s->st);
    QV_CUDA(cudaGetLastError());
    return QVTI_OK;
}

extern "C" int qvti_last_error(void) { return qvti::g_last_error; }

extern "C" const char* qvti_error_string(int code)
{
    switch (code) {
        case QVTI_OK: return "ok";
        case QVTI_ERR_ARG: return "invalid argument";
        case QVTI_ERR_CUDA: return "CUDA runtime error";
        case QVTI_ERR_UNSUPPORTED: return "unsupported grid size or option";
        case QVTI_ERR_STATE: return "call out of order";
        case QVTI_ERR_OOM: return "device allocation failed";
        case QVTI_ERR_NONFINITE: return "non-finite value detected";
        case QVTI_ERR_TIMEOUT: return "wait timed out";
        default: return "unknown error";
    }
}
