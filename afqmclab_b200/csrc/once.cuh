// One-time set-up per device.
//
// Kernel attributes such as the dynamic shared-memory limit belong to the
// context of the device that is current when they are set, so a process that
// launches on several devices has to set them on each one.  first_on_device
// returns true the first time it is called for `flags` with a given device
// current (devices 0..63), false afterwards.
#pragma once
#include <atomic>
#include <cuda_runtime.h>

inline bool first_on_device(std::atomic<unsigned long long> &flags)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return true;
    const unsigned long long bit = 1ull << dev;
    return (flags.fetch_or(bit) & bit) == 0;
}
