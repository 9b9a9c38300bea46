// Allocation-free population configuration.
//
// Some callers cannot allocate device memory at the point where they need a
// population-control table: a host framework that owns the GPU's memory
// through its own pooled allocator and forbids plugins from calling the CUDA
// allocator, an application whose device memory budget is fixed at start-up,
// or a latency-critical loop where the implicit synchronisation of an
// allocation is not acceptable.  afqmc_pop_configuration_noalloc_dev serves
// them: its only scratch (the per-walker copy counts) lives in a file-scope
// device array that the library reserves once when it is loaded, on every
// GPU that loads it, and keeps until the process exits.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/afqmc_b200.h"
#include "engine_internal.cuh"
#include "walker_kernels.cuh"

// Scratch for the copy counts of up to AFQMC_NOALLOC_MAX_WALKERS walkers
// (256 KB on every device that loads the library).
static __device__ __align__(256) int g_pop_scratch[AFQMC_NOALLOC_MAX_WALKERS];

namespace {

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
int *g_scratch_ptr[MAX_DEVICES] = {};

// The host-side name g_pop_scratch is not a device address; the device
// address is looked up once per device, with that device current.
int scratch_for_current_device(int **out)
{
    int dev = 0;
    cudaError_t r = cudaGetDevice(&dev);
    if (r != cudaSuccess)
        return engine_fail(AFQMC_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(r));
    if (dev < 0 || dev >= MAX_DEVICES) return engine_fail(AFQMC_ERR_ARG, "device index out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        r = cudaGetSymbolAddress(&p, g_pop_scratch);
        if (r != cudaSuccess || !p)
            return engine_fail(AFQMC_ERR_CUDA,
                               std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(r));
        g_scratch_ptr[dev] = (int *)p;
    }
    *out = g_scratch_ptr[dev];
    return AFQMC_OK;
}

}  // namespace

extern "C" int afqmc_pop_configuration_noalloc_dev(int W, const double *weights, const double *uniforms,
                                                   int *table, void *stream)
{
    if (W <= 0 || !weights || !uniforms || !table) return engine_fail(AFQMC_ERR_ARG, "bad argument");
    if (W > AFQMC_NOALLOC_MAX_WALKERS)
        return engine_fail(AFQMC_ERR_ARG, "afqmc_pop_configuration_noalloc_dev: W = " + std::to_string(W) +
                                              " exceeds the scratch limit of " +
                                              std::to_string(AFQMC_NOALLOC_MAX_WALKERS) + " walkers");
    int *scratch = nullptr;
    int r = scratch_for_current_device(&scratch);
    if (r != AFQMC_OK) return r;
    launch_pop_comb_scratch(W, weights, uniforms, scratch, table, (cudaStream_t)stream);
    return engine_check_launch();
}
