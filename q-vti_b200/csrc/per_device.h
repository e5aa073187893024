// Once-per-device initialisation.  CUDA kernel attributes such as the
// dynamic shared-memory limit, and symbol addresses of __device__ arrays, are
// properties of one device: a process that uses several devices has to set
// them up on each.  run(dev, f) calls f() the first time device `dev` is
// seen (the caller makes `dev` current), remembers success, and retries after
// a failure; concurrent callers are serialised.  Plain C++ (no CUDA headers),
// so the logic is testable without a GPU.
#pragma once
#include <mutex>

namespace qvti {

constexpr int kMaxDevices = 64;

template <int N>
class PerDeviceOnce {
public:
    // Returns f()'s status (0 = success) the first time, 0 afterwards, and
    // -1 for a device ordinal outside [0, N).
    template <class F>
    int run(int dev, F&& f)
    {
        if (dev < 0 || dev >= N) return -1;
        std::lock_guard<std::mutex> lk(mu_);
        if (done_[dev]) return 0;
        const int rc = f();
        if (rc == 0) done_[dev] = true;
        return rc;
    }
    bool done(int dev)
    {
        std::lock_guard<std::mutex> lk(mu_);
        return dev >= 0 && dev < N && done_[dev];
    }

private:
    std::mutex mu_;
    bool done_[N] = {};
};

}  // namespace qvti
