// Exchange of the phaseless mixed estimator as dense tensor-core GEMMs for
// real half-rotated Cholesky vectors (exchange_gemm.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.cuh"

struct afqmc_engine;

struct ExGemmBlock {
    int Ns = 0;
    long long K = 0, tOff = 0;
    __nv_bfloat16 *V = nullptr;   // K x K, sum_g A_g (x) A_g in the u-index order
};

struct ExGemmScratch {
    __nv_bfloat16 *Bt = nullptr;   // K x 2W
    __nv_bfloat16 *Av = nullptr;   // [Ar; Ai], 2K x 2W
    __nv_bfloat16 *Rt = nullptr;   // 2K x K
    float *Y = nullptr;                                          // 2K per vector
    float *Z = nullptr;                                          // K x 2W
    double *shift = nullptr;   // max Re logov of the alive walkers
};

bool exchange_gemm_supported(int n, int Ns, int W, int G);
// V of spin block b from the engine's FP64 half-rotated vectors (set-up)
int exchange_gemm_build(afqmc_engine *e, int b, ExGemmBlock &blk);
int exchange_gemm_alloc(afqmc_engine *e, long long Kmax, ExGemmScratch &s);
// exTot[w] (= or +=) sum_g ex[g, w] of this block; exNum[g] += sum_w den_w ex[g, w]
// (den_w = exp(logov_w) of the alive walkers); A2r = the block's real A rows
// (g, a) x i, Theta = the bf16 theta planes of the population; both sums
// are counted `mult` times (a block standing for two identical spin blocks).
// Launches on the engine's stream.
int exchange_gemm_run(afqmc_engine *e, const ExGemmBlock &blk, const __nv_bfloat16 *A2r,
                      const __nv_bfloat16 *Theta, const ExGemmScratch &s, bool accumulate, int mult,
                      zd *exTot, zd *exNum, int *err);
