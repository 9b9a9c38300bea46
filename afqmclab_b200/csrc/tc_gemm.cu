// tcgen05 BF16 GEMM in two forms, both warp-specialised:
//   - tc_gemm_t_kernel (large outputs, at least one tile per SM): persistent,
//     the product formed transposed so a TMEM lane holds an output column,
//     double-buffered accumulators, 16-byte column stores;
//   - tc_gemm_kernel (small outputs): one 128 x BN output tile per CTA.
// In the second form:
//   warp 0 lane 0 : TMA producer (A 128x64, B BNx64 per stage, 128B swizzle)
//   warp 1        : TMEM allocation; lane 0 issues the UMMAs and commits
//   warps 2..5    : epilogue, TMEM -> registers -> global (coalesced along m)
// Every wait is bounded (tc_common.cuh); on a timeout the kernel records an
// error code, skips the remaining work and still releases its TMEM.
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "tc_common.cuh"
#include "tc_gemm.cuh"
#include "once.cuh"

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

// ---------------------------------------------------------------------------
// Persistent form for large outputs: the product is formed transposed,
// D[n][m] = sum_k B[n, k] A[m, k], so a TMEM lane holds one output column
// (128 consecutive m of it per epilogue thread) and writes it with 16-byte
// stores.  Tiles of 128 n x 256 m, double-buffered TMEM (2 x 256 columns) so
// the epilogue of one tile overlaps the MMAs of the next.
//   warp 0 lane 0 : TMA producer      warp 1 : TMEM owner, UMMA issuer
//   warps 2..9    : epilogue (lane quarter = warp % 4, column half = (warp - 2) / 4)
// ---------------------------------------------------------------------------
constexpr int TT_BN = 128, TT_BM = 256, TT_STAGES = 4, TT_THREADS = 320;
constexpr int TT_A_BYTES = TT_BM * TC_BK * 2, TT_B_BYTES = TT_BN * TC_BK * 2;
constexpr size_t TT_SMEM = 1024 + (size_t)TT_STAGES * (TT_A_BYTES + TT_B_BYTES) + 256;

template <int OUT>
__global__ void __launch_bounds__(TT_THREADS, 1)
tc_gemm_t_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int M,
                 int N, int K, int kSplit, int splits, void *C, long long ldc, long long splitStride,
                 float alpha, int *err, int permN, long long permK)
{
    constexpr uint32_t IDESC = idesc_bf16(TT_BN, TT_BM);
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t *sA = base;
    uint8_t *sB = base + TT_STAGES * TT_A_BYTES;
    uint64_t *full = (uint64_t *)(sB + TT_STAGES * TT_B_BYTES);
    uint64_t *empty = full + TT_STAGES;
    uint64_t *tfull = empty + TT_STAGES;   // 2
    uint64_t *tempty = tfull + 2;          // 2
    uint32_t *tmemSlot = (uint32_t *)(tempty + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int MT = (M + TT_BM - 1) / TT_BM, NTn = (N + TT_BN - 1) / TT_BN;
    const int tiles = MT * NTn * splits;
    auto tile_kt = [&](int t, int &m0, int &n0, int &k0) {
        const int z = t / (MT * NTn), r = t - z * (MT * NTn);
        m0 = (r % MT) * TT_BM;
        n0 = (r / MT) * TT_BN;
        k0 = z * kSplit;
        const int kEnd = min(K, k0 + kSplit);
        return kEnd > k0 ? (kEnd - k0 + TC_BK - 1) / TC_BK : 0;
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < TT_STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        for (int b = 0; b < 2; ++b) { mbar_init(&tfull[b], 1); mbar_init(&tempty[b], 256); }
        fence_mbar_init();
        tma_prefetch_desc(&tmA);
        tma_prefetch_desc(&tmB);
    }
    if (warp == 1) { tmem_alloc(tmemSlot, 512); tmem_relinquish(); }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmemSlot;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {
            int it = 0;
            for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
                int m0, n0, k0;
                const int KT = tile_kt(t, m0, n0, k0);
                for (int kt = 0; kt < KT && ok; ++kt, ++it) {
                    const int s = it % TT_STAGES;
                    if (it >= TT_STAGES) ok = mbar_wait_sleep(&empty[s], ((it / TT_STAGES) - 1) & 1);
                    if (!ok) break;
                    mbar_arrive_expect_tx(&full[s], TT_A_BYTES + TT_B_BYTES);
                    tma_load_2d(sA + s * TT_A_BYTES, &tmA, &full[s], k0 + kt * TC_BK, m0);
                    tma_load_2d(sB + s * TT_B_BYTES, &tmB, &full[s], k0 + kt * TC_BK, n0);
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int it = 0, tc = 0;
            for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x, ++tc) {
                int m0, n0, k0;
                const int KT = tile_kt(t, m0, n0, k0);
                const int buf = tc & 1;
                if (tc >= 2) ok = mbar_wait_sleep(&tempty[buf], ((tc >> 1) - 1) & 1);
                if (!ok) break;
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(buf * TT_BM);
                for (int kt = 0; kt < KT && ok; ++kt, ++it) {
                    const int s = it % TT_STAGES;
                    ok = mbar_wait_sleep(&full[s], (it / TT_STAGES) & 1);
                    if (!ok) break;
                    tc_fence_after();
                    const uint32_t a0 = smem_u32(sA + s * TT_A_BYTES);
                    const uint32_t b0 = smem_u32(sB + s * TT_B_BYTES);
#pragma unroll
                    for (int kk = 0; kk < TC_BK / 16; ++kk)
                        umma_bf16(d, desc_k_sw128(b0 + kk * 32), desc_k_sw128(a0 + kk * 32), IDESC,
                                  (kt > 0 || kk > 0) ? 1u : 0u);
                    umma_commit(&empty[s]);
                }
                umma_commit(&tfull[buf]);
            }
        }
        __syncwarp();
    } else {
        const int q = warp & 3, half = (warp - 2) >> 2;
        int tc = 0;
        for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x, ++tc) {
            int m0, n0, k0;
            const int KT = tile_kt(t, m0, n0, k0);
            const int buf = tc & 1;
            ok = mbar_wait_sleep(&tfull[buf], (tc >> 1) & 1);
            if (!ok) break;
            tc_fence_after();
            const int n = n0 + q * 32 + lane;
            const size_t colOff = (size_t)(t / (MT * NTn)) * splitStride + (size_t)n * ldc;
            const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * TT_BM);
#pragma unroll 1
            for (int c0 = half * 128; c0 < half * 128 + 128; c0 += 32) {
                float v[32];
                tmem_ld32(trow + (uint32_t)c0, v);
                if (KT == 0) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) v[j] = 0.f;
                }
                const int mb = m0 + c0;
                if (n < N) {
                    if (OUT == TC_OUT_BF16) {
                        __nv_bfloat16 *dst = (__nv_bfloat16 *)C + colOff + mb;
                        if (permN > 0) {
                            // exchanged store: (p K + i + n b, j + n a) -> row p K + j + n b,
                            // column i + n a of a K-pitched output (32 rows never cross b or p)
                            const int p = mb >= permK ? 1 : 0;
                            const long long r = mb - p * permK;
                            const long long i0 = r % permN, b = r / permN;
                            const long long j = n % permN, a = n / permN;
                            dst = (__nv_bfloat16 *)C + ((p * permK + j + permN * b) * permK + permN * a + i0);
                        }
#pragma unroll
                        for (int j = 0; j < 32; j += 8) {
                            if (mb + j + 8 <= M) {
                                uint4 pk;
                                __nv_bfloat162 h0 = __floats2bfloat162_rn(alpha * v[j], alpha * v[j + 1]);
                                __nv_bfloat162 h1 = __floats2bfloat162_rn(alpha * v[j + 2], alpha * v[j + 3]);
                                __nv_bfloat162 h2 = __floats2bfloat162_rn(alpha * v[j + 4], alpha * v[j + 5]);
                                __nv_bfloat162 h3 = __floats2bfloat162_rn(alpha * v[j + 6], alpha * v[j + 7]);
                                pk.x = *(uint32_t *)&h0; pk.y = *(uint32_t *)&h1;
                                pk.z = *(uint32_t *)&h2; pk.w = *(uint32_t *)&h3;
                                *(uint4 *)(dst + j) = pk;
                            } else {
                                for (int u = 0; u < 8; ++u)
                                    if (mb + j + u < M) dst[j + u] = __float2bfloat16_rn(alpha * v[j + u]);
                            }
                        }
                    } else {
                        float *dst = (float *)C + colOff + mb;
#pragma unroll
                        for (int j = 0; j < 32; j += 4) {
                            if (mb + j + 4 <= M) {
                                *(float4 *)(dst + j) =
                                    make_float4(alpha * v[j], alpha * v[j + 1], alpha * v[j + 2], alpha * v[j + 3]);
                            } else {
                                for (int u = 0; u < 4; ++u)
                                    if (mb + j + u < M) dst[j + u] = alpha * v[j + u];
                            }
                        }
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(&tempty[buf]);
        }
    }
    if (!ok && err) atomicExch(err, 1);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) tmem_dealloc(tmem, 512);
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
    static std::atomic<unsigned long long> attr{0};
    if (first_on_device(attr)) {
        cudaFuncSetAttribute(tc_gemm_kernel<BN, OUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
    int kSplit = a.K;
    if (a.splits > 1) kSplit = ((a.K + a.splits - 1) / a.splits + TC_BK - 1) / TC_BK * TC_BK;
    dim3 grid((a.M + TC_BM - 1) / TC_BM, (a.N + BN - 1) / BN, a.splits > 1 ? a.splits : 1);
    tc_gemm_kernel<BN, OUT><<<grid, 192, smem, s>>>(ma, mb, a.M, a.N, a.K, kSplit, a.C, a.ldc,
                                                     a.splitStride, a.alpha, a.err);
    return (int)cudaGetLastError();
}

template <int OUT>
int launch_t(const TcGemmArgs &a, cudaStream_t s)
{
    CUtensorMap ma, mb;
    int r = tc_make_map_bf16(&ma, a.A, a.K, a.M, a.lda, TT_BM);
    if (r) return r;
    r = tc_make_map_bf16(&mb, a.B, a.K, a.N, a.ldb, TT_BN);
    if (r) return r;
    static std::atomic<unsigned long long> attr{0};
    if (first_on_device(attr)) {
        cudaFuncSetAttribute(tc_gemm_t_kernel<OUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TT_SMEM);
    }
    const int splits = a.splits > 1 ? a.splits : 1;
    int kSplit = a.K;
    if (splits > 1) kSplit = ((a.K + splits - 1) / splits + TC_BK - 1) / TC_BK * TC_BK;
    const long long tiles = (long long)((a.M + TT_BM - 1) / TT_BM) * ((a.N + TT_BN - 1) / TT_BN) * splits;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = (int)std::min<long long>(tiles, sms);
    tc_gemm_t_kernel<OUT><<<grid, TT_THREADS, TT_SMEM, s>>>(ma, mb, a.M, a.N, a.K, kSplit, splits, a.C, a.ldc,
                                                            a.splitStride, a.alpha, a.err, a.permN, a.permK);
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
    if (a.permN > 0) {
        // exchanged bf16 store of the persistent form: M = 2 permK, N = permK,
        // 32-row runs inside one orbital run, 16-byte aligned destinations
        if (a.outType != TC_OUT_BF16 || a.splits > 1 || a.permN % 32 != 0 || a.permK % TT_BM != 0 ||
            a.permK % a.permN != 0 || a.M != 2 * a.permK || a.N != a.permK || ((uintptr_t)a.C % 16) != 0)
            return (int)cudaErrorInvalidValue;
        return launch_t<TC_OUT_BF16>(a, s);
    }
    // large outputs: the persistent transposed form, when its 16-byte column
    // stores are aligned
    {
        const int es = a.outType == TC_OUT_F32 ? 4 : 2;
        const bool aligned = ((uintptr_t)a.C % 16 == 0) && ((a.ldc * es) % 16 == 0) &&
                             (a.splits <= 1 || (a.splitStride * es) % 16 == 0);
        const long long tiles = (long long)((a.M + TT_BM - 1) / TT_BM) * ((a.N + TT_BN - 1) / TT_BN);
        if (aligned && a.M >= TT_BM && a.N >= TT_BN && tiles * (a.splits > 1 ? a.splits : 1) >= 148) {
            if (a.outType == TC_OUT_F32) return launch_t<TC_OUT_F32>(a, s);
            return launch_t<TC_OUT_BF16>(a, s);
        }
    }
    if (a.N >= 192) {
        if (a.outType == TC_OUT_F32) return launch_bn<256, TC_OUT_F32>(a, s);
        return launch_bn<256, TC_OUT_BF16>(a, s);
    }
    if (a.outType == TC_OUT_F32) return launch_bn<128, TC_OUT_F32>(a, s);
    return launch_bn<128, TC_OUT_BF16>(a, s);
}

// ---------------------------------------------------------------------------
// Self-check of the bounded waits.  One CTA holds a TMEM allocation (as the
// tensor-core kernels do) and waits, with the same two wait helpers those
// kernels use, on two mbarriers that nothing arrives at.  Each wait must give
// up after `limit` SM cycles; the CTA then records which ones did (bit 0: the
// spinning wait, bit 1: the suspending wait), completes both phases itself,
// frees its TMEM and returns.  Nothing is in flight while it waits.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(64, 1) bounded_wait_check_kernel(long long limit, int *err)
{
    __shared__ uint64_t bars[2];
    __shared__ uint32_t tmemSlot;
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    if (warp == 1) { tmem_alloc(&tmemSlot, 32); tmem_relinquish(); }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x == 0) {
        int bits = 0;
        if (!mbar_wait(&bars[0], 0, limit)) bits |= 1;
        if (!mbar_wait_sleep(&bars[1], 0, 1000, limit)) bits |= 2;
        // complete both phases so that no wait is left pending
        mbar_arrive(&bars[0]);
        mbar_arrive(&bars[1]);
        *err = bits;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) tmem_dealloc(tmemSlot, 32);
}

static_assert(TC_WAIT_LIMIT_CYCLES == TC_WAIT_LIMIT, "one wait limit for the kernels and the check");

int tc_bounded_wait_check(long long limitCycles, int *errDev, cudaStream_t s)
{
    g_launch_count++;
    bounded_wait_check_kernel<<<1, 64, 0, s>>>(limitCycles, errDev);
    return (int)cudaGetLastError();
}
