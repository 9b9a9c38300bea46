// Compensated tf32 tensor-core overlap S_b = phiT_b^H phi from fp32 planar
// walkers (overlap_tc.cu).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"

bool overlap_tc_supported(int n, int Ns);
// host: the 2 Ns x 2 n operator rows (tf32 high / low parts) of the trial block T (n x Ns)
int overlap_tc_build(const zd *Thost, int n, int Ns, std::vector<float> &hi, std::vector<float> &lo);
// S[w * sStride + sOff + a + Ns * c] for every walker w of the fp32 population w32
int overlap_tc_launch(cudaStream_t s, int n, int ncol, int Ns, int W, const float *Ohi, const float *Olo,
                      const float *w32, double *S, long long sStride, long long sOff, int *err);
