// Mixed-precision form of the constrained-path (Hubbard) walker step:
// tcgen05 kind::tf32 contractions with compensated (hi + lo) operands
// (propagation, and the measurement's half step and overlap), FP64
// LU/log-determinant, weights, re-orthonormalisation and the rest of the
// measurement.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "common.cuh"

struct afqmc_engine;
struct CpMixedState;

bool cp_mixed_supported(int L, int N, std::string *why);
int cp_mixed_create(afqmc_engine *e);
void cp_mixed_destroy(afqmc_engine *e);
int cp_mixed_project_dtk_dtv(afqmc_engine *e);
int cp_mixed_modify_gm(afqmc_engine *e);
int cp_mixed_pop_control(afqmc_engine *e);
int cp_mixed_pop_weights(afqmc_engine *e);
int cp_mixed_sync_to_fp64(afqmc_engine *e);
int cp_mixed_sync_from_fp64(afqmc_engine *e);
int cp_mixed_status(afqmc_engine *e);
// the measurement's half step and overlap on the tensor cores (S in e->S,
// the FP64 walkers after the half step in e->wfTmp); *done false when the
// half-step operator is not real (the FP64 measurement runs then)
int cp_mixed_measure_prep(afqmc_engine *e, bool *done);

// Shared tf32 tensor-core pieces (also used by the phaseless mixed form):
// (E - I) of a real n x n operator E (host, column-major) as tf32 high/low
// parts, row-major; -1 when E has an imaginary part
int tf32_split_operator(const zd *E, int n, std::vector<float> &hi, std::vector<float> &lo);
// x -> (tf32 high part, fp32 remainder), elementwise
int split_f32_launch(cudaStream_t s, long long count, const float *x, float *hi, float *lo);
// phi' = phi + (E - I) phi for fp32 planar walkers (2 ncol columns of n
// per walker) given as hi + lo; output hi/lo (olo != NULL) or fp32 into ohi
int onebody_tf32_launch(cudaStream_t s, int n, int ncol, int W, const float *Ehi, const float *Elo,
                        const float *rhi, const float *rlo, float *ohi, float *olo, int *err);
