// Compensated tf32 tensor-core overlap S_b = phiT_b^H phi from fp32 planar
// walkers (overlap_tc.cu).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"

// nb (1 or 2) spin blocks sharing the walker's leading columns, 2 sum Ns <= 128
bool overlap_tc_supported(int n, int nb, const int *Ns);
// host: the stacked 2 sum Ns x 2 n operator rows (tf32 high / low parts) of the
// trial blocks T_b (n x Ns_b)
int overlap_tc_build(int nb, const zd *const *Thost, int n, const int *Ns, std::vector<float> &hi,
                     std::vector<float> &lo);
// S[w * sStride + sOff[b] + a + Ns[b] * c] of every block for every walker w of
// the fp32 population w32
int overlap_tc_launch(cudaStream_t s, int n, int ncol, int nb, const int *Ns, int W, const float *Ohi,
                      const float *Olo, const float *w32, zd *S, long long sStride, const long long *sOff,
                      int *err);

// Half-step one-body of the mixed estimator: out = phi + (E - I) phi for every
// column of the fp32 population w32 (W walkers, 2 ncol columns of n sites
// each), (E - I) given as tf32 high / low parts (n x n row-major); n in {64, 128}
bool onebody_split_supported(int n);
int onebody_split_launch(cudaStream_t s, int n, int ncol, int W, const float *Ehi, const float *Elo,
                         const float *w32, float *out, int *err);
