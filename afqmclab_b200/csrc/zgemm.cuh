// Batched complex FP64 GEMM used by the plain (FP64) form of the walker step.
// C_b = alpha * op(A_b) * op(B_b) + beta * C_b for every batch entry b,
// column-major operands, op in {N, T, C}; A or B may be real (double).
// This is the B200 replacement for the reference's gmm_cpu/zgemm calls
// (common/tensorHao/source/tensor_2d_bl_cpu.cpp:61-75) and its zgemv
// (tensor_1d_bl_cpu.cpp:50-107), batched over the walker population.
#pragma once
#include "common.cuh"

enum { OP_N = 0, OP_T = 1, OP_C = 2 };
// operand storage kinds
enum { ST_Z64 = 0, ST_R64 = 1, ST_C32P = 2 };  // complex f64 | real f64 | complex f32 planar
// output modes
enum { OUT_Z64 = 1, OUT_BF16P = 2, OUT_C32P = 4 };

struct ZGemmArgs {
    int m = 0, n = 0, k = 0;
    int opA = OP_N, opB = OP_N;
    int a_real = 0, b_real = 0;   // operand stored as double instead of double2
    zd alpha = {1.0, 0.0}, beta = {0.0, 0.0};
    const void *A = nullptr; long long lda = 0, strideA = 0;
    const void *B = nullptr; long long ldb = 0, strideB = 0;
    zd *C = nullptr; long long ldc = 0, strideC = 0;
    int batch = 1;
    const int *mask = nullptr;     // skip batch b when mask[b] == 0
    const int *skip = nullptr;     // skip batch b when skip[b] != 0
    // symmetric product (m = n): only output tiles that meet the lower
    // triangle (row >= column) are computed; tiles above it are not written
    int lower = 0;
    // complex f32 planar operands: imaginary plane at +planeA/+planeB floats
    // (set a_real/b_real = 2 to select them; 1 = real f64 as before)
    long long planeA = 0, planeB = 0;
    // extra outputs: bits of OUT_* besides the f64 complex C (OUT_Z64 is implied
    // when C != nullptr); C2 receives bf16 planar (imag plane at +plane2),
    // C3 complex f32 planar (imag plane at +plane3); same ldc / strideC.
    int outMode = OUT_Z64;
    void *C2 = nullptr; long long plane2 = 0, strideC2 = 0, ldc2 = 0;
    float *C3 = nullptr; long long plane3 = 0, strideC3 = 0, ldc3 = 0;
};

// Launches on `stream`; returns cudaGetLastError().
cudaError_t zgemm_batched(const ZGemmArgs &a, cudaStream_t stream);

// Autotuner switch (process-wide) and the cached choice for a shape (-1: none).
void zgemm_set_autotune(int on);
int zgemm_tuned_choice(const ZGemmArgs &a);
