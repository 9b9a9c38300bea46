// theta_b = phi_b S_b^{-1} on the tcgen05 tensor cores from fp32 planar
// walkers (theta_tc.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.cuh"

bool theta_tc_supported(int n, int Ns);
// floats of one B scratch array (hi or lo) for W walkers
size_t theta_tc_bscratch(int W, int Ns);
// Builds the S^{-1} operand (walkers outside `mask` give theta = 0) and runs
// the product: bf16 planar Theta (+ w * thetaStride + tOff, im plane `plane`
// elements after re; element (i, a) at i + n a) and, when thetaZ is given,
// the FP64 copy (+ w * zStride + tOff).  comp = 1 single tf32 product,
// comp = 3 compensated.
int theta_tc_launch(cudaStream_t s, int n, int ncol, int Ns, int W, const float *w32, const zd *Sinv,
                    long long sStride, long long sOff, const int *mask, int comp, float *Bh, float *Bl,
                    __nv_bfloat16 *Theta, long long thetaStride, long long plane, long long tOff, zd *thetaZ,
                    long long zStride, int *err);
