// Launch figures (SM count, resident blocks per SM, function attributes) of
// the current device, computed once per device.
#pragma once

#include <cuda_runtime.h>

#include <mutex>

namespace grrt_b200 {

constexpr int kMaxLaunchDevices = 64;

// The Shape of the current device, filled by fill(device) the first time
// that device asks. Every call site is its own template instance (its lambda
// has its own type), with its own lock held around the check and the fill:
// host threads whose first renders start together wait for one fill, and
// contexts on different devices each get the figures of their own device.
template <typename Shape, typename Fill>
const Shape& per_device_shape(Fill fill) {
    static std::mutex m;
    static Shape shapes[kMaxLaunchDevices];
    static bool ready[kMaxLaunchDevices] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxLaunchDevices) {
        cudaGetLastError();
        dev = 0;
    }
    std::lock_guard<std::mutex> lk(m);
    if (!ready[dev]) {
        shapes[dev] = fill(dev);
        ready[dev] = true;
    }
    return shapes[dev];
}

}  // namespace grrt_b200
