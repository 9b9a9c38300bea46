// theta_b = phi_b S_b^{-1} on the tcgen05 tensor cores from fp32 planar
// walkers (theta_tc.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.cuh"

// nb (1 or 2) spin blocks sharing the walker's leading columns; n in {64, 128},
// 2 nb round16(max Ns) <= 128; s32 = floats per walker of the fp32 inverse
// slots (a multiple of 4)
bool theta_tc_supported(int n, int nb, const int *Ns, long long s32);
// theta_b = phi S_b^{-1} for every block b and walker from the fp32 inverse
// planes [re | im] at Sinv32 + w s32 + 2 sOff[b] (walkers outside `mask` give
// theta = 0): bf16 planar Theta (+ w * thetaStride + tOff[b], im plane `plane`
// elements after re; element (i, a) at i + n a) and, when thetaZ is given, the
// FP64 copy (+ w * zStride + tOff[b]); compensated tf32 products
int theta_tc_launch(cudaStream_t s, int n, int ncol, int nb, const int *Ns, int W, const float *w32,
                    const float *Sinv32, long long s32, const long long *sOff, const int *mask,
                    __nv_bfloat16 *Theta, long long thetaStride, long long plane, const long long *tOff,
                    zd *thetaZ, long long zStride, int *err);
