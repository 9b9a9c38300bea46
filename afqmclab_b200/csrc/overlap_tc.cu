// Overlap S_b = phiT_b^H phi of every walker on the tcgen05 tensor cores from
// fp32 walkers (planar [re n x ncol | im n x ncol] per walker), compensated:
// each fp32 walker tile is split in shared memory into a tf32 high part and
// the fp32 remainder, and the trial operator into tf32 high and low parts, so
//   S = O_hi phi_hi + O_lo phi_hi + O_hi phi_lo
// carries about 22 significant bits (kind::tf32, fp32 accumulation); the
// result is written in FP64 for the LU / log-determinant.
// Replaces SDSDOperation / SD2sSD2isOperation's overlap gmm
// (SDSDOperation.cpp:154-164, SD2sSD2isOperation.cpp:84-94) in the
// mixed-precision form.
//
// The spin blocks share the walker (SD2is: both use its leading columns), so
// their operators are stacked into one A operand of at most 128 rows and a
// walker tile is read once for both: block b occupies rows from 2 sum_{b'<b}
// Ns_b', row 2a = [Re T(:,a) | Im T(:,a)], row 2a+1 = [-Im T(:,a) | Re T(:,a)],
// so the real and imaginary parts of S(a, c) land in neighbouring TMEM lanes.
//
// Persistent CTAs over tiles of BN walker columns (whole walkers), K = 2n in
// chunks of 32:
//   warp 0 lane 0 : TMA producer (O_hi, O_lo chunks; raw fp32 walker chunks)
//   warp 1        : TMEM owner; lane 0 issues the UMMAs (double-buffered TMEM)
//   warps 2..5    : split each walker chunk in place (hi) and beside it (lo)
//   warps 6..9    : epilogue (TMEM lane quarter = warp % 4), one complex
//                   double per lane and column pair after a lane-pair exchange
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <string>
#include <vector>

#include "engine_internal.cuh"
#include "overlap_tc.cuh"
#include "tc_common.cuh"
#include "once.cuh"

extern std::atomic<long long> g_launch_count;

namespace {

constexpr int BM = 128, BK = 32, BN = 128, STAGES = 3, NT = 320;
constexpr int A_BYTES = BM * BK * 4;
constexpr int B_BYTES = BN * BK * 4;
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
constexpr size_t SMEM = 1024 + (size_t)STAGES * STAGE_BYTES + 256;

struct OvArgs {
    int n, W, kbA, bnw, wpt, tiles, rows;
    int nb, Ns[2], rowBase[2];
    long long sOff[2];
    uint32_t idesc;
    double2 *S;
    long long sStride;
    int *err;
};

__global__ void __launch_bounds__(NT, 1)
ov_split_kernel(const __grid_constant__ CUtensorMap tAh, const __grid_constant__ CUtensorMap tAl,
                const __grid_constant__ CUtensorMap tB, OvArgs p)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = (uint64_t *)(base + STAGES * STAGE_BYTES);
    uint64_t *split = full + STAGES;
    uint64_t *empty = split + STAGES;
    uint64_t *tfull = empty + STAGES;   // 2
    uint64_t *tempty = tfull + 2;       // 2
    uint32_t *tmemSlot = (uint32_t *)(tempty + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int KT = 2 * p.kbA;
    const int ncols = p.wpt * p.bnw;
    const uint32_t bBytes = (uint32_t)(ncols * BK * 4);
    const int myTiles = (p.tiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&split[s], 128);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) { mbar_init(&tfull[b], 1); mbar_init(&tempty[b], 128); }
        fence_mbar_init();
        tma_prefetch_desc(&tAh);
        tma_prefetch_desc(&tAl);
        tma_prefetch_desc(&tB);
    }
    if (warp == 1) { tmem_alloc(tmemSlot, 2 * BN); tmem_relinquish(); }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmemSlot;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {
            int it = 0;
            for (int ti = 0; ti < myTiles && ok; ++ti) {
                const int t = (int)blockIdx.x + ti * (int)gridDim.x;
                for (int kt = 0; kt < KT && ok; ++kt, ++it) {
                    const int s = it % STAGES;
                    if (it >= STAGES) ok = mbar_wait(&empty[s], ((it / STAGES) - 1) & 1);
                    if (!ok) break;
                    const int plane = kt / p.kbA, kk = (kt % p.kbA) * BK;
                    uint8_t *st = base + s * STAGE_BYTES;
                    // walkers past W are not loaded (their columns are never written)
                    const int nv = min(p.wpt, p.W - t * p.wpt);
                    mbar_arrive_expect_tx(&full[s], 2 * A_BYTES + (uint32_t)(nv * p.bnw * BK * 4));
                    tma_load_2d(st, &tAh, &full[s], plane * p.n + kk, 0);
                    tma_load_2d(st + A_BYTES, &tAl, &full[s], plane * p.n + kk, 0);
                    for (int j = 0; j < nv; ++j)
                        tma_load_3d(st + 2 * A_BYTES + j * p.bnw * BK * 4, &tB, &full[s], kk, 0,
                                    2 * (t * p.wpt + j) + plane);
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int it = 0;
            for (int ti = 0; ti < myTiles && ok; ++ti) {
                const int buf = ti & 1;
                if (ti >= 2) ok = mbar_wait(&tempty[buf], ((ti >> 1) - 1) & 1);
                if (!ok) break;
                const uint32_t d = tmem + (uint32_t)(buf * BN);
                for (int kt = 0; kt < KT && ok; ++kt, ++it) {
                    const int s = it % STAGES;
                    ok = mbar_wait(&split[s], (it / STAGES) & 1);
                    if (!ok) break;
                    tc_fence_after();
                    const uint32_t st = smem_u32(base + s * STAGE_BYTES);
                    const uint32_t ah = st, al = st + A_BYTES, bh = st + 2 * A_BYTES, bl = bh + B_BYTES;
#pragma unroll
                    for (int k8 = 0; k8 < BK / 8; ++k8) {
                        const uint32_t acc0 = (kt > 0 || k8 > 0) ? 1u : 0u;
                        umma_tf32(d, desc_k_sw128(ah + k8 * 32), desc_k_sw128(bh + k8 * 32), p.idesc, acc0);
                        umma_tf32(d, desc_k_sw128(al + k8 * 32), desc_k_sw128(bh + k8 * 32), p.idesc, 1u);
                        umma_tf32(d, desc_k_sw128(ah + k8 * 32), desc_k_sw128(bl + k8 * 32), p.idesc, 1u);
                    }
                    umma_commit(&empty[s]);
                }
                if (ok) umma_commit(&tfull[buf]);
            }
        }
        __syncwarp();
    } else if (warp < 6) {
        // split the raw walker chunk: hi in place, lo in the slot beside it
        const int t = threadIdx.x - 64;
        const int n4 = (int)(bBytes / 16);
        const int items = myTiles * KT;
        for (int it = 0; it < items && ok; ++it) {
            const int s = it % STAGES;
            ok = mbar_wait(&full[s], (it / STAGES) & 1);
            if (!ok) break;
            float4 *bh = (float4 *)(base + s * STAGE_BYTES + 2 * A_BYTES);
            float4 *bl = (float4 *)(base + s * STAGE_BYTES + 2 * A_BYTES + B_BYTES);
            for (int i = t; i < n4; i += 128) {
                const float4 x = bh[i];
                float4 h, l;
                h.x = tf32_round(x.x); l.x = x.x - h.x;
                h.y = tf32_round(x.y); l.y = x.y - h.y;
                h.z = tf32_round(x.z); l.z = x.z - h.z;
                h.w = tf32_round(x.w); l.w = x.w - h.w;
                bh[i] = h;
                bl[i] = l;
            }
            fence_proxy_async();
            mbar_arrive(&split[s]);
        }
    } else {
        const int q = warp & 3;
        const int row = q * 32 + lane;
        const int b = (p.nb > 1 && row >= p.rowBase[1]) ? 1 : 0;
        const int rr = row - (b ? p.rowBase[1] : 0);
        const int a = rr >> 1;
        const int Ns = b ? p.Ns[1] : p.Ns[0];
        const long long sOff = b ? p.sOff[1] : p.sOff[0];
        const bool rowOK = row < p.rows;
        const int odd = lane & 1;
        for (int ti = 0; ti < myTiles && ok; ++ti) {
            const int buf = ti & 1;
            ok = mbar_wait(&tfull[buf], (ti >> 1) & 1);
            if (!ok) break;
            tc_fence_after();
            const int t = (int)blockIdx.x + ti * (int)gridDim.x;
            const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * BN);
#pragma unroll 1
            for (int c0 = 0; c0 < ncols; c0 += 32) {
                float v[32];
                tmem_ld32(trow + (uint32_t)c0, v);
#pragma unroll
                for (int j = 0; j < 32; j += 2) {
                    // even lane: Re S(a, col j) and Re S(a, col j+1); odd lane: the Im parts
                    const float send = odd ? v[j] : v[j + 1];
                    const float recv = __shfl_xor_sync(0xffffffffu, send, 1);
                    const int col = c0 + j + odd;
                    const int wj = col / p.bnw, c = col - wj * p.bnw;
                    const int w = t * p.wpt + wj;
                    if (rowOK && a < Ns && c < Ns && w < p.W)
                        p.S[(size_t)w * p.sStride + sOff + a + (size_t)Ns * c] =
                            odd ? make_double2((double)recv, (double)v[j + 1]) : make_double2((double)v[j], (double)recv);
                }
            }
            tc_fence_before();
            mbar_arrive(&tempty[buf]);
        }
    }
    if (!ok && p.err) atomicExch(p.err, 1);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) tmem_dealloc(tmem, 2 * BN);
}

// ---------------------------------------------------------------------------
// One-body product of the measurement's half step on the tensor cores:
//   out = phi + (E - I) phi   for every column of the fp32 population
// (columns (walker, plane, orbital), n sites each), compensated tf32:
// (E - I) is held resident in shared memory as tf32 high and low parts, each
// raw walker chunk is split in place into high part and remainder, and
//   phi_hi (E-I)_hi + phi_lo (E-I)_hi + phi_hi (E-I)_lo
// is accumulated in fp32.  The product is formed transposed (TMEM lane =
// population column, TMEM column = site), so each epilogue thread adds its
// column's fp32 residual and writes the column with 16-byte stores.
// Replaces Hop2isSD2isOperation::applyToRight (hop2isSD2isOperation.cpp:14-19)
// for the half step of the mixed estimator.
//   warp 0 lane 0 : TMA producer (the operator once, then walker chunks)
//   warp 1        : TMEM owner, UMMA issuer (double-buffered accumulators)
//   warps 2..5    : in-place split of each walker chunk
//   warps 6..9    : epilogue
// ---------------------------------------------------------------------------
constexpr int OB_STAGES = 3, OB_TILE = 128, OB_KC = 32;
constexpr int OB_CHUNK_BYTES = OB_TILE * OB_KC * 4;   // 16 KB: 128 columns x 32 sites

struct ObArgs {
    int n, nkc;
    long long cols, tiles;
    uint32_t idesc;
    const float *res;    // the walkers (residual)
    float *out;
    int *err;
};

__global__ void __launch_bounds__(320, 1)
ob_split_kernel(const __grid_constant__ CUtensorMap tEh, const __grid_constant__ CUtensorMap tEl,
                const __grid_constant__ CUtensorMap tP, ObArgs p)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const uint32_t eBytes = (uint32_t)p.n * 128;          // one k chunk of (E - I): n rows x 32 sites
    uint8_t *sEh = base;                                   // nkc chunks
    uint8_t *sEl = sEh + (size_t)p.nkc * eBytes;
    uint8_t *stg = sEl + (size_t)p.nkc * eBytes;           // OB_STAGES x (raw->hi | lo)
    uint64_t *full = (uint64_t *)(stg + (size_t)OB_STAGES * 2 * OB_CHUNK_BYTES);
    uint64_t *split = full + OB_STAGES;
    uint64_t *empty = split + OB_STAGES;
    uint64_t *eFull = empty + OB_STAGES;
    uint64_t *tfull = eFull + 1;    // 2
    uint64_t *tempty = tfull + 2;   // 2
    uint32_t *tmemSlot = (uint32_t *)(tempty + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long myTiles = (p.tiles - (long long)blockIdx.x + gridDim.x - 1) / gridDim.x;
    const int KT = p.nkc;

    if (threadIdx.x == 0) {
        for (int s = 0; s < OB_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&split[s], 128);
            mbar_init(&empty[s], 1);
        }
        mbar_init(eFull, 1);
        for (int b = 0; b < 2; ++b) { mbar_init(&tfull[b], 1); mbar_init(&tempty[b], 128); }
        fence_mbar_init();
        tma_prefetch_desc(&tEh);
        tma_prefetch_desc(&tEl);
        tma_prefetch_desc(&tP);
    }
    if (warp == 1) { tmem_alloc(tmemSlot, 256); tmem_relinquish(); }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmemSlot;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {
            mbar_arrive_expect_tx(eFull, 2 * KT * eBytes);
            for (int kc = 0; kc < KT; ++kc) {
                tma_load_2d(sEh + kc * eBytes, &tEh, eFull, kc * OB_KC, 0);
                tma_load_2d(sEl + kc * eBytes, &tEl, eFull, kc * OB_KC, 0);
            }
            long long it = 0;
            for (long long ti = 0; ti < myTiles && ok; ++ti) {
                const long long t = blockIdx.x + ti * gridDim.x;
                for (int kc = 0; kc < KT && ok; ++kc, ++it) {
                    const int s = (int)(it % OB_STAGES);
                    if (it >= OB_STAGES) ok = mbar_wait_sleep(&empty[s], (uint32_t)(((it / OB_STAGES) - 1) & 1));
                    if (!ok) break;
                    mbar_arrive_expect_tx(&full[s], OB_CHUNK_BYTES);
                    tma_load_2d(stg + (size_t)s * 2 * OB_CHUNK_BYTES, &tP, &full[s], kc * OB_KC, (int)(t * OB_TILE));
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            ok = mbar_wait_sleep(eFull, 0);
            long long it = 0;
            for (long long ti = 0; ti < myTiles && ok; ++ti) {
                const int buf = (int)(ti & 1);
                if (ti >= 2) ok = mbar_wait_sleep(&tempty[buf], (uint32_t)(((ti >> 1) - 1) & 1));
                if (!ok) break;
                const uint32_t d = tmem + (uint32_t)(buf * 128);
                for (int kc = 0; kc < KT && ok; ++kc, ++it) {
                    const int s = (int)(it % OB_STAGES);
                    ok = mbar_wait_sleep(&split[s], (uint32_t)((it / OB_STAGES) & 1));
                    if (!ok) break;
                    tc_fence_after();
                    const uint32_t ph = smem_u32(stg + (size_t)s * 2 * OB_CHUNK_BYTES), pl = ph + OB_CHUNK_BYTES;
                    const uint32_t eh = smem_u32(sEh + kc * eBytes), el = smem_u32(sEl + kc * eBytes);
#pragma unroll
                    for (int k8 = 0; k8 < OB_KC / 8; ++k8) {
                        const uint32_t acc0 = (kc > 0 || k8 > 0) ? 1u : 0u;
                        umma_tf32(d, desc_k_sw128(ph + k8 * 32), desc_k_sw128(eh + k8 * 32), p.idesc, acc0);
                        umma_tf32(d, desc_k_sw128(pl + k8 * 32), desc_k_sw128(eh + k8 * 32), p.idesc, 1u);
                        umma_tf32(d, desc_k_sw128(ph + k8 * 32), desc_k_sw128(el + k8 * 32), p.idesc, 1u);
                    }
                    umma_commit(&empty[s]);
                }
                if (ok) umma_commit(&tfull[buf]);
            }
        }
        __syncwarp();
    } else if (warp < 6) {
        const int t = threadIdx.x - 64;
        const long long items = myTiles * KT;
        for (long long it = 0; it < items && ok; ++it) {
            const int s = (int)(it % OB_STAGES);
            ok = mbar_wait_sleep(&full[s], (uint32_t)((it / OB_STAGES) & 1));
            if (!ok) break;
            float4 *bh = (float4 *)(stg + (size_t)s * 2 * OB_CHUNK_BYTES);
            float4 *bl = (float4 *)(stg + (size_t)s * 2 * OB_CHUNK_BYTES + OB_CHUNK_BYTES);
#pragma unroll 4
            for (int i = t; i < OB_CHUNK_BYTES / 16; i += 128) {
                const float4 x = bh[i];
                float4 h, l;
                h.x = tf32_round(x.x); l.x = x.x - h.x;
                h.y = tf32_round(x.y); l.y = x.y - h.y;
                h.z = tf32_round(x.z); l.z = x.z - h.z;
                h.w = tf32_round(x.w); l.w = x.w - h.w;
                bh[i] = h;
                bl[i] = l;
            }
            fence_proxy_async();
            mbar_arrive(&split[s]);
        }
    } else {
        const int q = warp & 3;
        const int r = q * 32 + lane;
        for (long long ti = 0; ti < myTiles && ok; ++ti) {
            const int buf = (int)(ti & 1);
            const long long t = blockIdx.x + ti * gridDim.x;
            const long long col = t * OB_TILE + r;
            const float *rc = p.res + col * p.n;
            float *oc = p.out + col * p.n;
            // the first 32 sites of this column's residual are loaded while
            // the tile's products are still running
            float4 x0[8];
            if (col < p.cols) {
#pragma unroll
                for (int j = 0; j < 8; ++j) x0[j] = *(const float4 *)(rc + 4 * j);
            }
            ok = mbar_wait_sleep(&tfull[buf], (uint32_t)((ti >> 1) & 1));
            if (!ok) break;
            tc_fence_after();
            const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * 128);
            for (int c0 = 0; c0 < p.n; c0 += 32) {
                float v[32];
                tmem_ld32(trow + (uint32_t)c0, v);
                if (col < p.cols) {
                    // the next 32 sites' residual loads issue before this chunk's stores
                    float4 x1[8];
                    const bool more = c0 + 32 < p.n;
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                        if (more) x1[j] = *(const float4 *)(rc + c0 + 32 + 4 * j);
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                        *(float4 *)(oc + c0 + 4 * j) = make_float4(x0[j].x + v[4 * j], x0[j].y + v[4 * j + 1],
                                                                   x0[j].z + v[4 * j + 2], x0[j].w + v[4 * j + 3]);
#pragma unroll
                    for (int j = 0; j < 8; ++j) x0[j] = x1[j];
                }
            }
            tc_fence_before();
            mbar_arrive(&tempty[buf]);
        }
    }
    if (!ok && p.err) atomicExch(p.err, 1);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) tmem_dealloc(tmem, 256);
}

PFN_cuTensorMapEncodeTiled_v12000 encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool done = false;
    if (!done) {
        cudaDriverEntryPointQueryResult q;
        void *f = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)f;
        done = true;
    }
    return fn;
}

int map_f32(CUtensorMap *map, const float *ptr, int rank, const cuuint64_t *dims, const cuuint64_t *pitch,
            const cuuint32_t *box)
{
    auto enc = encoder();
    if (!enc) return (int)cudaErrorNotSupported;
    if ((uintptr_t)ptr & 15) return (int)cudaErrorMisalignedAddress;
    for (int i = 0; i + 1 < rank; ++i)
        if (pitch[i] & 15) return (int)cudaErrorMisalignedAddress;
    cuuint32_t es[3] = {1u, 1u, 1u};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, const_cast<float *>(ptr), dims, pitch, box,
                     es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : (int)r + 10000;
}

float tf32_host(float x)
{
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7F800000u) != 0x7F800000u) { u += 0x1000u; u &= 0xFFFFE000u; }
    std::memcpy(&x, &u, 4);
    return x;
}

}  // namespace

bool overlap_tc_supported(int n, int nb, const int *Ns)
{
    if (n % 4 != 0 || nb < 1 || nb > 2) return false;
    int rows = 0;
    for (int b = 0; b < nb; ++b) {
        if (Ns[b] < 0 || Ns[b] > 64) return false;
        rows += 2 * Ns[b];
    }
    return rows >= 2 && rows <= BM;
}

// rows of block b from 2 sum_{b' < b} Ns_b': 2a -> [Re T(:,a) | Im T(:,a)],
// 2a + 1 -> [-Im T(:,a) | Re T(:,a)]; tf32 high parts and the tf32 remainders
int overlap_tc_build(int nb, const zd *const *Thost, int n, const int *Ns, std::vector<float> &hi,
                     std::vector<float> &lo)
{
    int rows = 0;
    for (int b = 0; b < nb; ++b) rows += 2 * Ns[b];
    hi.assign((size_t)rows * 2 * n, 0.f);
    lo.assign((size_t)rows * 2 * n, 0.f);
    auto put = [&](size_t idx, double v) {
        const float h = tf32_host((float)v);
        hi[idx] = h;
        lo[idx] = tf32_host((float)(v - (double)h));
    };
    int r0 = 0;
    for (int b = 0; b < nb; ++b) {
        for (int a = 0; a < Ns[b]; ++a)
            for (int i = 0; i < n; ++i) {
                const zd t = Thost[b][i + (size_t)n * a];
                const size_t re = (size_t)(r0 + 2 * a) * 2 * n, im = re + 2 * n;
                put(re + i, t.x);
                put(re + n + i, t.y);
                put(im + i, -t.y);
                put(im + n + i, t.x);
            }
        r0 += 2 * Ns[b];
    }
    return 0;
}

int overlap_tc_launch(cudaStream_t s, int n, int ncol, int nb, const int *Ns, int W, const float *Ohi,
                      const float *Olo, const float *w32, zd *S, long long sStride, const long long *sOff,
                      int *err)
{
    if (!overlap_tc_supported(n, nb, Ns)) return (int)cudaErrorInvalidValue;
    static std::atomic<unsigned long long> attr{0};
    if (first_on_device(attr)) {
        cudaFuncSetAttribute(ov_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
    }
    OvArgs a{};
    a.n = n; a.W = W; a.nb = nb;
    int rows = 0, maxNs = 0;
    for (int b = 0; b < 2; ++b) {
        a.Ns[b] = b < nb ? Ns[b] : 0;
        a.sOff[b] = b < nb ? sOff[b] : 0;
        a.rowBase[b] = rows;
        rows += 2 * a.Ns[b];
        maxNs = std::max(maxNs, a.Ns[b]);
    }
    a.rows = rows;
    CUtensorMap ah, al, b;
    cuuint64_t da[2] = {(cuuint64_t)2 * n, (cuuint64_t)rows}, pa[1] = {(cuuint64_t)2 * n * 4};
    cuuint32_t boxA[2] = {BK, BM};
    int r = map_f32(&ah, Ohi, 2, da, pa, boxA);
    if (!r) r = map_f32(&al, Olo, 2, da, pa, boxA);
    const int bnw = (maxNs + 15) / 16 * 16;
    cuuint64_t db[3] = {(cuuint64_t)n, (cuuint64_t)ncol, (cuuint64_t)2 * W};
    cuuint64_t pb[2] = {(cuuint64_t)n * 4, (cuuint64_t)n * ncol * 4};
    cuuint32_t boxB[3] = {BK, (cuuint32_t)bnw, 1u};
    if (!r) r = map_f32(&b, w32, 3, db, pb, boxB);
    if (r) return r;
    a.kbA = (n + BK - 1) / BK;
    a.bnw = bnw;
    a.wpt = std::max(1, BN / bnw);
    a.tiles = (W + a.wpt - 1) / a.wpt;
    a.idesc = idesc_tf32(BM, a.wpt * bnw);
    a.S = S; a.sStride = sStride; a.err = err;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    g_launch_count++;
    ov_split_kernel<<<std::min(a.tiles, sms), NT, SMEM, s>>>(ah, al, b, a);
    return (int)cudaGetLastError();
}

bool onebody_split_supported(int n) { return n == 64 || n == 128; }

int onebody_split_launch(cudaStream_t s, int n, int ncol, int W, const float *Ehi, const float *Elo,
                         const float *w32, float *out, int *err)
{
    if (!onebody_split_supported(n)) return (int)cudaErrorInvalidValue;
    const int nkc = n / OB_KC;
    const size_t smem = 1024 + (size_t)2 * nkc * n * 128 + (size_t)OB_STAGES * 2 * OB_CHUNK_BYTES + 256;
    static std::atomic<unsigned long long> attr{0};
    if (first_on_device(attr)) {
        cudaFuncSetAttribute(ob_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    }
    CUtensorMap eh, el, pm;
    cuuint64_t de[2] = {(cuuint64_t)n, (cuuint64_t)n}, pe[1] = {(cuuint64_t)n * 4};
    cuuint32_t be[2] = {(cuuint32_t)OB_KC, (cuuint32_t)n};
    int r = map_f32(&eh, Ehi, 2, de, pe, be);
    if (!r) r = map_f32(&el, Elo, 2, de, pe, be);
    const long long cols = 2LL * ncol * W;
    cuuint64_t dp[2] = {(cuuint64_t)n, (cuuint64_t)cols}, pp[1] = {(cuuint64_t)n * 4};
    cuuint32_t bp[2] = {(cuuint32_t)OB_KC, (cuuint32_t)OB_TILE};
    if (!r) r = map_f32(&pm, w32, 2, dp, pp, bp);
    if (r) return r;
    ObArgs a{};
    a.n = n; a.nkc = nkc; a.cols = cols;
    a.tiles = (cols + OB_TILE - 1) / OB_TILE;
    a.idesc = idesc_tf32(OB_TILE, n);
    a.res = w32; a.out = out; a.err = err;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    g_launch_count++;
    ob_split_kernel<<<(unsigned)std::min<long long>(a.tiles, sms), 320, smem, s>>>(eh, el, pm, a);
    return (int)cudaGetLastError();
}
