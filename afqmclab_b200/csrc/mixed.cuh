// Mixed-precision form of the walker step (tensor-core contractions; FP64
// LU/log-determinant, phases, weights and re-orthonormalisation).
#pragma once
struct afqmc_engine;
struct MixedState;

int mixed_create(afqmc_engine *e);
void mixed_destroy(afqmc_engine *e);
int mixed_project_dtk_dtv(afqmc_engine *e);
int mixed_modify_gm(afqmc_engine *e);
int mixed_add_measurement(afqmc_engine *e);
int mixed_update_operators(afqmc_engine *e);
// keep the FP64 walker copy and the reduced-precision working copy in step
int mixed_sync_to_fp64(afqmc_engine *e);
int mixed_sync_from_fp64(afqmc_engine *e);
// The phaseless mixed form can take a population (FP64, reference layout) into
// its fp32 walkers directly from another device buffer; the FP64 copy is
// refreshed from the fp32 walkers before any FP64 use.
bool mixed_can_load_direct(const afqmc_engine *e);
// the walkers from a device buffer already in the phaseless mixed form's
// fp32 planar layout (2 n ncol floats per walker: real plane, imaginary plane)
int mixed_load_f32(afqmc_engine *e, const float *src);
int mixed_load_direct(afqmc_engine *e, const zd *src);
int mixed_status(afqmc_engine *e);
int mixed_pop_control(afqmc_engine *e);
// overlaps, population-control weights and the log-weight shift, as the
// mixed form's population control computes them (no comb)
int mixed_pop_weights(afqmc_engine *e);
int mixed_exchange(afqmc_engine *e);

// tcgen05 exchange kernel (exchange_tc.cu)
#include <cuda_bf16.h>
#include "common.cuh"
int exchange_tc_supported(int n, int Ns);
int exchange_tc_launch(cudaStream_t s, int G, int W, int Ns, int n, const __nv_bfloat16 *A2r,
                       const __nv_bfloat16 *A2i, const __nv_bfloat16 *Theta, long long tOff,
                       long long Ktot, const int *alive, zd *ex, int *err, bool realA);
__global__ void build_a2_kernel(int G, int Ns, int n, long long Ktot, long long tOff, const zd *Aall,
                                __nv_bfloat16 *A2r, __nv_bfloat16 *A2i);
