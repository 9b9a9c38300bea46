// tcgen05 BF16 GEMM: one 128 x BN output tile per CTA, warp-specialised.
//   warp 0 lane 0 : TMA producer (A 128x64, B BNx64 per stage, 128B swizzle)
//   warp 1        : TMEM allocation; lane 0 issues the UMMAs and commits
//   warps 2..5    : epilogue, TMEM -> registers -> global (coalesced along m)
// Every wait is bounded (tc_common.cuh); on a timeout the kernel records an
// error code, skips the remaining work and still releases its TMEM.
#include <cudaTypedefs.h>

#include <atomic>
#include <mutex>

#include "tc_common.cuh"
#include "tc_gemm.cuh"

extern std::atomic<long long> g_launch_count;

namespace {

constexpr int TC_BM = 128;
constexpr int TC_BK = 64;
constexpr int A_STAGE_BYTES = TC_BM * TC_BK * 2;

template <int BN>
__host__ __device__ constexpr int stages_for() { return BN >= 256 ? 4 : 6; }

template <int BN>
__host__ __device__ constexpr size_t smem_bytes()
{
    return 1024 + (size_t)stages_for<BN>() * (A_STAGE_BYTES + BN * TC_BK * 2) + 256;
}

template <int BN, int OUT>
__global__ void __launch_bounds__(192, 1)
tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
               int M, int N, int K, int kSplit, void *C, long long ldc, long long splitStride,
               float alpha, int *err)
{
    constexpr int STAGES = stages_for<BN>();
    constexpr int B_STAGE_BYTES = BN * TC_BK * 2;
    constexpr uint32_t IDESC = idesc_bf16(TC_BM, BN);
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t *sA = base;
    uint8_t *sB = base + STAGES * A_STAGE_BYTES;
    uint64_t *full = (uint64_t *)(sB + STAGES * B_STAGE_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *tmemFull = empty + STAGES;
    uint32_t *tmemSlot = (uint32_t *)(tmemFull + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * TC_BM, n0 = blockIdx.y * BN;
    const int k0 = blockIdx.z * kSplit;
    const int kEnd = min(K, k0 + kSplit);
    const int KT = (kEnd - k0 + TC_BK - 1) / TC_BK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        mbar_init(tmemFull, 1);
        fence_mbar_init();
        tma_prefetch_desc(&tmA);
        tma_prefetch_desc(&tmB);
    }
    if (warp == 1) { tmem_alloc(tmemSlot, BN); tmem_relinquish(); }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmemSlot;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {
            for (int kt = 0; kt < KT && ok; ++kt) {
                const int s = kt % STAGES;
                if (kt >= STAGES) ok = mbar_wait(&empty[s], ((kt / STAGES) - 1) & 1);
                if (!ok) break;
                mbar_arrive_expect_tx(&full[s], A_STAGE_BYTES + B_STAGE_BYTES);
                tma_load_2d(sA + s * A_STAGE_BYTES, &tmA, &full[s], k0 + kt * TC_BK, m0);
                tma_load_2d(sB + s * B_STAGE_BYTES, &tmB, &full[s], k0 + kt * TC_BK, n0);
            }
            // drain: the last stages' UMMAs must finish reading before exit
            for (int kt = max(KT, STAGES); kt < KT + STAGES && ok; ++kt) {
                const int s = kt % STAGES;
                ok = mbar_wait(&empty[s], ((kt / STAGES) - 1) & 1);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            for (int kt = 0; kt < KT && ok; ++kt) {
                const int s = kt % STAGES;
                ok = mbar_wait(&full[s], (kt / STAGES) & 1);
                if (!ok) break;
                tc_fence_after();
                const uint32_t a0 = smem_u32(sA + s * A_STAGE_BYTES);
                const uint32_t b0 = smem_u32(sB + s * B_STAGE_BYTES);
#pragma unroll
                for (int kk = 0; kk < TC_BK / 16; ++kk)
                    umma_bf16(tmem, desc_k_sw128(a0 + kk * 32), desc_k_sw128(b0 + kk * 32), IDESC,
                              (kt > 0 || kk > 0) ? 1u : 0u);
                umma_commit(&empty[s]);
            }
            umma_commit(tmemFull);
        }
        __syncwarp();
    } else {
        ok = mbar_wait(tmemFull, 0);
        tc_fence_after();
        if (ok && KT > 0) {
            const int q = warp & 3;
            const int row = m0 + q * 32 + lane;
            const size_t off = (size_t)blockIdx.z * splitStride;
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 32) {
                float v[32];
                tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + c0, v);
                if (row < M) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const int col = n0 + c0 + j;
                        if (col < N) {
                            size_t idx = off + (size_t)row + (size_t)col * ldc;
                            if (OUT == TC_OUT_F32) ((float *)C)[idx] = alpha * v[j];
                            else ((__nv_bfloat16 *)C)[idx] = __float2bfloat16_rn(alpha * v[j]);
                        }
                    }
                }
            }
        }
    }
    if (!ok && err) atomicExch(err, 1);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) tmem_dealloc(tmem, BN);
}

PFN_cuTensorMapEncodeTiled_v12000 get_encode()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

template <int BN, int OUT>
int launch_bn(const TcGemmArgs &a, cudaStream_t s)
{
    CUtensorMap ma, mb;
    int r = tc_make_map_bf16(&ma, a.A, a.K, a.M, a.lda, TC_BM);
    if (r) return r;
    r = tc_make_map_bf16(&mb, a.B, a.K, a.N, a.ldb, BN);
    if (r) return r;
    const size_t smem = smem_bytes<BN>();
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(tc_gemm_kernel<BN, OUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    int kSplit = a.K;
    if (a.splits > 1) kSplit = ((a.K + a.splits - 1) / a.splits + TC_BK - 1) / TC_BK * TC_BK;
    dim3 grid((a.M + TC_BM - 1) / TC_BM, (a.N + BN - 1) / BN, a.splits > 1 ? a.splits : 1);
    tc_gemm_kernel<BN, OUT><<<grid, 192, smem, s>>>(ma, mb, a.M, a.N, a.K, kSplit, a.C, a.ldc,
                                                     a.splitStride, a.alpha, a.err);
    return (int)cudaGetLastError();
}

}  // namespace

int tc_make_map_bf16(void *map, const void *base, long long inner, long long rows, long long pitch,
                     int boxRows)
{
    auto enc = get_encode();
    if (!enc) return (int)cudaErrorNotSupported;
    if (((uintptr_t)base & 15) || ((pitch * 2) & 15)) return (int)cudaErrorMisalignedAddress;
    cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(pitch * 2)};
    cuuint32_t box[2] = {64u, (cuuint32_t)boxRows};
    cuuint32_t estr[2] = {1u, 1u};
    CUresult r = enc((CUtensorMap *)map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims,
                     strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : (int)r + 10000;
}

int tc_gemm_bf16(const TcGemmArgs &a, cudaStream_t s)
{
    g_launch_count++;
    if (a.M <= 0 || a.N <= 0 || a.K <= 0) return 0;
    if (a.N >= 192) {
        if (a.outType == TC_OUT_F32) return launch_bn<256, TC_OUT_F32>(a, s);
        return launch_bn<256, TC_OUT_BF16>(a, s);
    }
    if (a.outType == TC_OUT_F32) return launch_bn<128, TC_OUT_F32>(a, s);
    return launch_bn<128, TC_OUT_BF16>(a, s);
}
