// tcgen05 BF16 GEMM with TMA operand loads (mixed-precision form).
//   C[m, n] = alpha * sum_k A[m, k] * B[n, k]
// A (M x K) and B (N x K) are K-major bf16 (row pitch lda / ldb elements,
// 16-byte multiples); C is column-major (element (m, n) at m + n * ldc),
// fp32 or bf16.  With splits > 1 the K range is cut into `splits` chunks of
// a multiple of 64 and chunk s writes its partial product to C + s * splitStride.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

enum { TC_OUT_F32 = 0, TC_OUT_BF16 = 1 };

struct TcGemmArgs {
    int M = 0, N = 0, K = 0;
    const __nv_bfloat16 *A = nullptr; long long lda = 0;
    const __nv_bfloat16 *B = nullptr; long long ldb = 0;
    void *C = nullptr; long long ldc = 0; int outType = TC_OUT_F32;
    int splits = 1; long long splitStride = 0;
    float alpha = 1.0f;
    int *err = nullptr;        // set to a non-zero code when a wait times out
    // exchanged store (bf16, persistent form only): with permN = n > 0 and
    // M = 2 permK, N = permK, element (p permK + i + n b, j + n a) goes to
    // C[(p permK + j + n b) permK + i + n a] (ldc unused)
    int permN = 0; long long permK = 0;
};

// Returns 0 on success, a cudaError_t / CUresult value otherwise.
int tc_gemm_bf16(const TcGemmArgs &a, cudaStream_t s);

// Bounded-wait self-check (one CTA, waits that nothing completes, limit in
// SM cycles); writes the bits of the waits that gave up to *errDev.
constexpr long long TC_WAIT_LIMIT_CYCLES = 2000000000LL;
int tc_bounded_wait_check(long long limitCycles, int *errDev, cudaStream_t s);

// Builds a 2-D bf16 tensor map (inner extent `inner`, `rows` rows, row pitch
// `pitch` elements) with a 64 x boxRows box and 128-byte swizzle.
int tc_make_map_bf16(void *map, const void *base, long long inner, long long rows, long long pitch,
                     int boxRows);
