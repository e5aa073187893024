// qvti_q_derivative_noalloc: one constant-Q derivative field for callers that
// cannot allocate device memory.
//
// Some callers own every byte of device memory through their own budget --
// a serving process whose footprint is fixed at start-up, a host framework
// that hands libraries pre-planned buffers from its own pool, or a latency-
// critical loop that cannot absorb the implicit device-wide synchronisation
// of cudaMalloc/cudaFree.  They cannot use qvti_q_derivative, which allocates
// device copies of its host arrays and a simulation's spectra as scratch.
// This variant takes device pointers for the input and output and keeps its
// scratch (the half spectrum) and its 1D tables in file-scope __device__
// arrays of a fixed maximum size, so a call allocates nothing.
#include <cstdio>
#include <mutex>

#include "engine.cuh"
#include "../../include/qvti.h"

namespace qvti {
namespace {

// Largest half spectrum (nz/2 + 1) * nx * ny the static scratch holds:
// 2^19 complex values = 4 MiB (e.g. 96^3, 64 x 64 x 128, 128 x 128 x 60).
constexpr long long kNoAllocSpectrum = 1ll << 19;
constexpr int kNoAllocAxis = 1024;  // longest axis the static tables hold

// Held by every GPU that loads the library, until the process exits.
static __device__ __align__(256) float2 g_na_scratch[kNoAllocSpectrum];
static __device__ __align__(256) float2 g_na_tw[3][kNoAllocAxis];
static __device__ __align__(256) float2 g_na_F[3][kNoAllocAxis];
static __device__ __align__(256) float2 g_na_B[3][kNoAllocAxis];
static __device__ __align__(256) float g_na_k[3][kNoAllocAxis];

// Device addresses of the arrays above, looked up once per device with that
// device current (a host-side use of the array names would not be a device
// address).
struct NoAllocDev {
    bool ready = false;
    float2 *scratch = nullptr, *tw = nullptr, *F = nullptr, *B = nullptr;
    float* k = nullptr;
};
NoAllocDev g_na_dev[kMaxDevices];
std::mutex g_na_mu;

int setup_device(int dev, NoAllocDev** out)
{
    if (dev < 0 || dev >= kMaxDevices) return QVTI_ERR_ARG;
    std::lock_guard<std::mutex> lk(g_na_mu);
    NoAllocDev& d = g_na_dev[dev];
    if (!d.ready) {
        cudaError_t e = cudaSuccess;
        auto addr = [&](void** p, const void* sym) {
            const cudaError_t r = cudaGetSymbolAddress(p, sym);
            if (r != cudaSuccess) e = r;
        };
        addr((void**)&d.scratch, g_na_scratch);
        addr((void**)&d.tw, g_na_tw);
        addr((void**)&d.F, g_na_F);
        addr((void**)&d.B, g_na_B);
        addr((void**)&d.k, g_na_k);
        if (e != cudaSuccess) {
            fprintf(stderr, "qvti_q_derivative_noalloc: cudaGetSymbolAddress: %s\n", cudaGetErrorString(e));
            return QVTI_ERR_CUDA;
        }
        if (configure_device(dev) != 0) return QVTI_ERR_CUDA;  // shared-memory limits of this device
        d.ready = true;
    }
    *out = &d;
    return QVTI_OK;
}

bool smooth_even(int n)
{
    if (n < 16 || n > kNoAllocAxis || (n & 1)) return false;
    int m = n;
    for (int r : {2, 3, 5, 7})
        while (m % r == 0) m /= r;
    return m == 1;
}

}  // namespace
}  // namespace qvti

extern "C" int qvti_q_derivative_noalloc(const float* d_in, float* d_out, int ntx, int nty, int ntz, float dx,
                                         float dy, float dz, int axis, int fwd, int power, void* stream)
{
    using namespace qvti;
    if (!d_in || !d_out || axis < 0 || axis > 2 || power < -1 || power > 1 || !(dx > 0 && dy > 0 && dz > 0))
        return fail(QVTI_ERR_ARG);
    if (!smooth_even(ntx) || !smooth_even(nty) || !smooth_even(ntz)) return fail(QVTI_ERR_UNSUPPORTED);
    const long long nkz = ntz / 2 + 1;
    if (nkz * ntx * nty > kNoAllocSpectrum) {
        fprintf(stderr,
                "qvti_q_derivative_noalloc: grid %dx%dx%d needs %lld spectrum values, the static scratch holds %lld\n",
                ntx, nty, ntz, nkz * ntx * nty, kNoAllocSpectrum);
        return fail(QVTI_ERR_UNSUPPORTED);
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(QVTI_ERR_CUDA);
    NoAllocDev* d = nullptr;
    int rc = setup_device(dev, &d);
    if (rc) return fail(rc);

    KP k{};
    k.nx = ntx; k.ny = nty; k.nz = ntz; k.nkz = (int)nkz; k.pml = 2;
    k.ntp = (long long)ntx * nty * ntz;
    k.inv_ntp = (float)(1.0 / (double)k.ntp);
    if (!make_fft_plan(ntx, &k.px) || !make_fft_plan(nty, &k.py) || !make_fft_plan(ntz, &k.pz))
        return fail(QVTI_ERR_UNSUPPORTED);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int n[3] = {ntx, nty, ntz};
    const float h[3] = {dx, dy, dz};
    for (int a = 0; a < 3; ++a)  // twiddles, |k| and shift multipliers; no C-PML profiles
        launch_axis_tables(n[a], h[a], 1.0, 2, d->tw + (size_t)a * kNoAllocAxis, d->k + (size_t)a * kNoAllocAxis,
                           d->F + (size_t)a * kNoAllocAxis, d->B + (size_t)a * kNoAllocAxis, nullptr, nullptr,
                           nullptr, nullptr, st);
    k.tw_x = d->tw; k.tw_y = d->tw + kNoAllocAxis; k.tw_z = d->tw + 2 * kNoAllocAxis;
    k.Fx = d->F; k.Fy = d->F + kNoAllocAxis; k.Fz = d->F + 2 * kNoAllocAxis;
    k.Bx = d->B; k.By = d->B + kNoAllocAxis; k.Bz = d->B + 2 * kNoAllocAxis;
    k.kx = d->k; k.ky = d->k + kNoAllocAxis; k.kz = d->k + 2 * kNoAllocAxis;
    k.v[0] = const_cast<float*>(d_in);
    k.H[0] = d->scratch;  // every stage overwrites what it reads: nothing needs clearing
    k.G[0] = d->scratch;
    launch_q_derivative(k, axis, fwd, power, d_out, st);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "qvti_q_derivative_noalloc: launch: %s\n", cudaGetErrorString(e));
        return fail(QVTI_ERR_CUDA);
    }
    return QVTI_OK;
}
