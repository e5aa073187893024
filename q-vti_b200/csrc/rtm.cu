// Reverse-time migration of one shot (qvti_rtm_shot) on top of the stepper.
//
// The reference's host program is titled "3D viscoacoustic reverse time
// migration" (viscoelas_3D.cpp:1-3) and declares its options -- RTM type,
// imaging condition, media type, checkpoints (:42-65, :223-229) -- without
// implementing any of them.  Here:
//
//   1. the source wavefield runs forward in the chosen medium; after every
//      snap_every-th step its three velocities are copied, on the
//      simulation's stream, into a device buffer (one slot per kept step);
//   2. the observed records run backward: a simulation without a source
//      injects them time-reversed at the receivers (qvti_set_injection);
//      after the back-propagation step that reaches time t of a kept step,
//      k_image accumulates the zero-lag cross-correlation sum_c S_c(t) R_c(t)
//      and the illumination sum_c S_c(t)^2 at every cell;
//   3. the source-normalised image divides by the illumination plus
//      illum_eps times its maximum.
//
// Q compensation (QVTI_MEDIA_Q_COMPENSATED) reverses the sign of the loss
// terms in both propagations, restoring the amplitude attenuation removed;
// the lossless medium sets Q infinite; dispersion-only drops the loss terms.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/qvti.h"

namespace {

// image += sum_c s_c r_c, illum += sum_c s_c^2 over n cells (float4 loads;
// every grid axis is even, so n is a multiple of 4).
__global__ void k_image(long long n4, const float4* s0, const float4* s1, const float4* s2, const float4* r0,
                        const float4* r1, const float4* r2, float4* image, float4* illum)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
        const float4 a = s0[i], b = s1[i], c = s2[i], x = r0[i], y = r1[i], z = r2[i];
        float4 im = image[i], il = illum[i];
        im.x += a.x * x.x + b.x * y.x + c.x * z.x;
        im.y += a.y * x.y + b.y * y.y + c.y * z.y;
        im.z += a.z * x.z + b.z * y.z + c.z * z.z;
        im.w += a.w * x.w + b.w * y.w + c.w * z.w;
        il.x += a.x * a.x + b.x * b.x + c.x * c.x;
        il.y += a.y * a.y + b.y * b.y + c.y * c.y;
        il.z += a.z * a.z + b.z * b.z + c.z * c.z;
        il.w += a.w * a.w + b.w * b.w + c.w * c.w;
        image[i] = im;
        illum[i] = il;
    }
}

// A simulation freed on every return.
struct SimGuard {
    qvti_sim* s = nullptr;
    ~SimGuard()
    {
        if (s) qvti_destroy(s);
    }
};

struct DeviceBuf {
    void* p = nullptr;
    ~DeviceBuf()
    {
        if (p) cudaFree(p);
    }
};

#define RTM_TRY(x)                 \
    do {                           \
        const int rc_ = (x);       \
        if (rc_) return rc_;       \
    } while (0)

// QVTI_ERR_NONFINITE when a propagation blew up -- the Q-compensated medium
// amplifies what attenuation would remove and, over long paths through
// strong attenuation, the high wavenumbers with it -- instead of an image of
// NaN.
int finite_or_fail(qvti_sim* s)
{
    double norms[9];
    int bad = 0;
    const int rc = qvti_field_norms(s, norms, &bad);  // QVTI_ERR_NONFINITE when bad
    return rc ? rc : bad ? QVTI_ERR_NONFINITE : QVTI_OK;
}

int prepare(const qvti_config* cfg, int media, const float* const* model, int r_iz, const int* r_ix, const int* r_iy,
            int rn, qvti_sim** out)
{
    RTM_TRY(qvti_create(cfg, out));
    RTM_TRY(qvti_set_media(*out, media));
    RTM_TRY(qvti_set_model(*out, model[0], model[1], model[2], model[3], model[4], model[5], model[6], 0));
    return qvti_set_receivers(*out, r_iz, r_ix, r_iy, rn);
}

}  // namespace

extern "C" int qvti_rtm_shot(const qvti_config* cfg, const float* velp, const float* vels, const float* rho,
                             const float* gama_p, const float* gama_s, const float* eps, const float* delta,
                             int src_type, int s_ix, int s_iy, int s_iz, const float* wavelet, int nt, int r_iz,
                             const int* r_ix, const int* r_iy, int rn, const float* obs_vx, const float* obs_vy,
                             const float* obs_vz, const qvti_rtm_opts* opts, float* image_xcorr, float* image_norm)
{
    if (!cfg || !opts || !wavelet || nt <= 0 || rn <= 0 || opts->snap_every < 1 || !(opts->illum_eps >= 0.f) ||
        (!obs_vx && !obs_vy && !obs_vz))
        return QVTI_ERR_ARG;
    const long long ntp = (long long)cfg->ntx * cfg->nty * cfg->ntz;
    const int K = opts->snap_every;
    const int nsnap = nt / K;  // kept steps t = K - 1, 2K - 1, ...: after step t with (t + 1) % K == 0
    if (nsnap < 1) return QVTI_ERR_ARG;
    if (cudaSetDevice(cfg->device) != cudaSuccess) return QVTI_ERR_CUDA;
    const float* model[7] = {velp, vels, rho, gama_p, gama_s, eps, delta};
    const size_t fbytes = sizeof(float) * (size_t)ntp;

    DeviceBuf snaps, acc;
    if (cudaMalloc(&snaps.p, 3 * fbytes * (size_t)nsnap) != cudaSuccess) return QVTI_ERR_OOM;
    if (cudaMalloc(&acc.p, 2 * fbytes) != cudaSuccess) return QVTI_ERR_OOM;
    float* S = static_cast<float*>(snaps.p);
    float* image = static_cast<float*>(acc.p);
    float* illum = image + ntp;

    // 1. source wavefield, forward
    {
        SimGuard src;
        RTM_TRY(prepare(cfg, opts->media, model, r_iz, r_ix, r_iy, rn, &src.s));
        RTM_TRY(qvti_set_source(src.s, src_type, s_ix, s_iy, s_iz, wavelet, nt));
        RTM_TRY(qvti_reset(src.s));
        void* stv = nullptr;
        RTM_TRY(qvti_get_stream(src.s, &stv));
        cudaStream_t st = static_cast<cudaStream_t>(stv);
        float* v[3];
        for (int c = 0; c < 3; ++c) RTM_TRY(qvti_device_field(src.s, c, &v[c]));
        for (int i = 0; i < nsnap; ++i) {
            RTM_TRY(qvti_step(src.s, K));
            for (int c = 0; c < 3; ++c)
                if (cudaMemcpyAsync(S + ((size_t)i * 3 + c) * ntp, v[c], fbytes, cudaMemcpyDeviceToDevice, st) !=
                    cudaSuccess)
                    return QVTI_ERR_CUDA;
        }
        RTM_TRY(qvti_sync(src.s));
        RTM_TRY(finite_or_fail(src.s));
    }

    // 2. receiver wavefield, backward in time, imaged at the kept steps
    SimGuard rcv;
    RTM_TRY(prepare(cfg, opts->media, model, r_iz, r_ix, r_iy, rn, &rcv.s));
    std::vector<float> silent(nt, 0.f);
    RTM_TRY(qvti_set_source(rcv.s, src_type, -1, -1, -1, silent.data(), nt));  // outside the grid: no source
    RTM_TRY(qvti_set_injection(rcv.s, obs_vx, obs_vy, obs_vz, nt));
    RTM_TRY(qvti_reset(rcv.s));
    void* stv = nullptr;
    RTM_TRY(qvti_get_stream(rcv.s, &stv));
    cudaStream_t st = static_cast<cudaStream_t>(stv);
    float* r[3];
    for (int c = 0; c < 3; ++c) RTM_TRY(qvti_device_field(rcv.s, c, &r[c]));
    if (cudaMemsetAsync(image, 0, 2 * fbytes, st) != cudaSuccess) return QVTI_ERR_CUDA;
    // back-propagation step j reaches time t = nt - 1 - j; kept step i has
    // t = (i + 1) K - 1
    int done = 0;
    for (int i = nsnap - 1; i >= 0; --i) {
        const int j = nt - (i + 1) * K;
        RTM_TRY(qvti_step(rcv.s, j + 1 - done));
        done = j + 1;
        const float* s = S + (size_t)i * 3 * ntp;
        k_image<<<148 * 4, 256, 0, st>>>(ntp / 4, reinterpret_cast<const float4*>(s),
                                         reinterpret_cast<const float4*>(s + ntp),
                                         reinterpret_cast<const float4*>(s + 2 * ntp),
                                         reinterpret_cast<const float4*>(r[0]), reinterpret_cast<const float4*>(r[1]),
                                         reinterpret_cast<const float4*>(r[2]), reinterpret_cast<float4*>(image),
                                         reinterpret_cast<float4*>(illum));
        if (cudaGetLastError() != cudaSuccess) return QVTI_ERR_CUDA;
    }
    RTM_TRY(qvti_sync(rcv.s));
    RTM_TRY(finite_or_fail(rcv.s));

    // 3. outputs
    if (image_xcorr && cudaMemcpy(image_xcorr, image, fbytes, cudaMemcpyDeviceToHost) != cudaSuccess)
        return QVTI_ERR_CUDA;
    if (image_norm) {
        std::vector<float> im(ntp), il(ntp);
        if (cudaMemcpy(im.data(), image, fbytes, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(il.data(), illum, fbytes, cudaMemcpyDeviceToHost) != cudaSuccess)
            return QVTI_ERR_CUDA;
        const float mx = *std::max_element(il.begin(), il.end());
        const float stab = opts->illum_eps * mx;
        for (long long i = 0; i < ntp; ++i) image_norm[i] = il[i] + stab > 0.f ? im[i] / (il[i] + stab) : 0.f;
    }
    return QVTI_OK;
}
