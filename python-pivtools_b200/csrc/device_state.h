// device_state.h -- host-side state kept per CUDA device.
//
// The libraries hold a little state across calls: the SM count, each kernel's
// resident CTAs per SM (after raising its dynamic shared-memory limit, which is a
// per-device attribute) and the staging workspace of the host-pointer entry
// points.  All of it is indexed by the device current at the call, so a process
// that drives several GPUs from one or more host threads sets every device up
// on its own.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <mutex>

namespace piv {

constexpr int kMaxDevices = 64;

// The current device, or -1 (no device, or an index beyond the tables).
inline int current_device()
{
    int d = -1;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kMaxDevices) return -1;
    return d;
}

// SM count of `dev`, queried once per device.
inline int device_sms(int dev)
{
    static std::atomic<int> sms[kMaxDevices];
    int v = sms[dev].load(std::memory_order_acquire);
    if (v > 0) return v;
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        n = 148;
    }
    sms[dev].store(n, std::memory_order_release);
    return n;
}

// A non-negative value computed once per device by a set-up function (called with
// that device current, under a lock); a negative result (failure) is not cached.
struct PerDeviceOnce {
    std::atomic<int> v[kMaxDevices];
    std::mutex mu;
    PerDeviceOnce()
    {
        for (auto &x : v) x.store(-1, std::memory_order_relaxed);
    }
    template <class F>
    int get(int dev, F &&setup)
    {
        int x = v[dev].load(std::memory_order_acquire);
        if (x >= 0) return x;
        std::lock_guard<std::mutex> lock(mu);
        x = v[dev].load(std::memory_order_relaxed);
        if (x >= 0) return x;
        x = setup();
        if (x >= 0) v[dev].store(x, std::memory_order_release);
        return x;
    }
};

}  // namespace piv
