// theta_b = phi_b S_b^{-1} (n x Ns per walker and spin block) on the tcgen05
// tensor cores (kind::tf32, fp32 accumulation), from the fp32 planar walkers
// and the FP64 inverse overlaps.  The walker tile arrives by TMA with the
// sites contiguous and is rewritten in shared memory as a K-major operand
// (128-byte swizzle); S^{-1} is the K-major B operand:
//   theta_re = phi_re S_re - phi_im S_im,  theta_im = phi_re S_im + phi_im S_re
// as one real product over K = (re part, im part) x electrons, N = (re, im)
// output columns.  The walker values are rounded to tf32 when they are
// rewritten; with `comp` = 3 both operands are split into tf32 high and low
// parts (A in shared memory, B when it is built) and
// A_hi B_hi + A_lo B_hi + A_hi B_lo is accumulated (about 22 significant
// bits), for the measurement; the force uses a single product.
// Replaces the zgetrs('T') solve of SDSDOperation.cpp:166-173 /
// SD2sSD2isOperation.cpp:187-198 in the mixed-precision form.
//
// Persistent CTAs, one walker at a time, two pipeline items per walker (the
// re and im halves of K):
//   warp 0 lane 0 : TMA producer        warp 1     : TMEM owner, UMMA issuer
//   warps 2..5    : rewrite of A (K-major, hi/lo)   warps 6..9 : epilogue (double-buffered TMEM)
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <string>

#include "engine_internal.cuh"
#include "tc_common.cuh"
#include "theta_tc.cuh"

extern std::atomic<long long> g_launch_count;

namespace {

constexpr int BK = 32;
constexpr int NT = 320;

struct ThArgs {
    int n, Ns, Nsp, W, nchunk, nkb, comp, stages;
    uint32_t rawBytes, aBytes, bBytes, stageBytes, idesc;
    __nv_bfloat16 *Theta;  // + w * thetaStride + tOff, planes Ktot apart
    long long thetaStride, plane, tOff;
    zd *thetaZ;            // optional FP64 copy, + w * zStride + tOff
    long long zStride;
    int *err;
};

__global__ void __launch_bounds__(NT, 1)
theta_tc_kernel(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tBh,
                const __grid_constant__ CUtensorMap tBl, ThArgs p)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    // stage: [raw A | A hi | A lo | B hi | B lo]
    uint64_t *full = (uint64_t *)(base + (size_t)p.stages * p.stageBytes);
    uint64_t *split = full + p.stages;
    uint64_t *empty = split + p.stages;
    uint64_t *tfull = empty + p.stages;   // 2
    uint64_t *tempty = tfull + 2;         // 2
    uint32_t *tmemSlot = (uint32_t *)(tempty + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nw = (p.W - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;   // walkers of this CTA
    const int items = 2 * nw;

    if (threadIdx.x == 0) {
        for (int s = 0; s < p.stages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&split[s], 128);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) { mbar_init(&tfull[b], 1); mbar_init(&tempty[b], 128); }
        fence_mbar_init();
        tma_prefetch_desc(&tA);
        tma_prefetch_desc(&tBh);
    }
    if (warp == 1) { tmem_alloc(tmemSlot, 256); tmem_relinquish(); }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmemSlot;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {
            for (int it = 0; it < items && ok; ++it) {
                const int s = it % p.stages;
                if (it >= p.stages) ok = mbar_wait(&empty[s], ((it / p.stages) - 1) & 1);
                if (!ok) break;
                const int w = (int)blockIdx.x + (it >> 1) * (int)gridDim.x, part = it & 1;
                uint8_t *st = base + (size_t)s * p.stageBytes;
                mbar_arrive_expect_tx(&full[s], p.rawBytes + (p.comp == 3 ? 2u : 1u) * p.bBytes);
                for (int c = 0; c < p.nchunk; ++c)
                    tma_load_3d(st + c * p.Nsp * 128, &tA, &full[s], c * 32, 0, 2 * w + part);
                uint8_t *bh = st + p.rawBytes + 2 * p.aBytes;
                for (int kb = 0; kb < p.nkb; ++kb) {
                    tma_load_2d(bh + kb * 2 * p.Nsp * 128, &tBh, &full[s], part * p.Nsp + kb * BK, w * 2 * p.Nsp);
                    if (p.comp == 3)
                        tma_load_2d(bh + p.bBytes + kb * 2 * p.Nsp * 128, &tBl, &full[s], part * p.Nsp + kb * BK,
                                    w * 2 * p.Nsp);
                }
            }
            for (int it = max(items, p.stages); it < items + p.stages && ok; ++it) {
                const int s = it % p.stages;
                ok = mbar_wait(&empty[s], ((it / p.stages) - 1) & 1);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            for (int it = 0; it < items && ok; ++it) {
                const int s = it % p.stages, lw = it >> 1, part = it & 1, buf = lw & 1;
                if (part == 0 && lw >= 2) {
                    ok = mbar_wait(&tempty[buf], ((lw >> 1) - 1) & 1);
                    if (!ok) break;
                }
                ok = mbar_wait(&split[s], (it / p.stages) & 1);
                if (!ok) break;
                tc_fence_after();
                const uint32_t st = smem_u32(base + (size_t)s * p.stageBytes);
                const uint32_t ah = st + p.rawBytes, al = ah + p.aBytes, bh = al + p.aBytes, bl = bh + p.bBytes;
                const uint32_t d = tmem + (uint32_t)(buf * 128);
                for (int kk = 0; kk < p.Nsp / 8; ++kk) {
                    const uint32_t aoff = (uint32_t)((kk >> 2) * 128 * 128 + (kk & 3) * 32);
                    const uint32_t boff = (uint32_t)((kk >> 2) * 2 * p.Nsp * 128 + (kk & 3) * 32);
                    const uint32_t acc0 = (part > 0 || kk > 0) ? 1u : 0u;
                    umma_tf32(d, desc_k_sw128(ah + aoff), desc_k_sw128(bh + boff), p.idesc, acc0);
                    if (p.comp == 3) {
                        umma_tf32(d, desc_k_sw128(al + aoff), desc_k_sw128(bh + boff), p.idesc, 1u);
                        umma_tf32(d, desc_k_sw128(ah + aoff), desc_k_sw128(bl + boff), p.idesc, 1u);
                    }
                }
                umma_commit(&empty[s]);
                if (part == 1) umma_commit(&tfull[buf]);
            }
        }
        __syncwarp();
    } else if (warp < 6) {
        // rewrite the raw tile (Nsp rows of 32 sites per 32-site chunk) as a
        // K-major, 128-byte-swizzled operand: row = site, 16-byte chunk
        // (k % 32) / 4 stored at chunk ^ (site % 8) of the 128-byte row
        const int t = threadIdx.x - 64;
        const int units = 128 * (p.Nsp / 4);
        for (int it = 0; it < items && ok; ++it) {
            const int s = it % p.stages;
            ok = mbar_wait(&full[s], (it / p.stages) & 1);
            if (!ok) break;
            const uint8_t *raw = base + (size_t)s * p.stageBytes;
            uint8_t *ah = base + (size_t)s * p.stageBytes + p.rawBytes;
            uint8_t *al = ah + p.aBytes;
            for (int u = t; u < units; u += 128) {
                const int i = u & 127, k4 = u >> 7;
                float x[4];
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    x[j] = i < p.n ? *(const float *)(raw + (i >> 5) * p.Nsp * 128 + (4 * k4 + j) * 128 + (i & 31) * 4)
                                   : 0.f;
                float4 h, l;
                h.x = tf32_round(x[0]); l.x = x[0] - h.x;
                h.y = tf32_round(x[1]); l.y = x[1] - h.y;
                h.z = tf32_round(x[2]); l.z = x[2] - h.z;
                h.w = tf32_round(x[3]); l.w = x[3] - h.w;
                const int kb = k4 >> 3, c16 = (k4 & 7) ^ (i & 7);
                const size_t off = (size_t)kb * 128 * 128 + (size_t)i * 128 + c16 * 16;
                *(float4 *)(ah + off) = h;
                if (p.comp == 3) *(float4 *)(al + off) = l;
            }
            fence_proxy_async();
            mbar_arrive(&split[s]);
        }
    } else {
        const int q = warp & 3;
        const int row = q * 32 + lane;
        const int Ns = p.Ns, Nsp = p.Nsp, n = p.n;
        for (int lw = 0; lw < nw && ok; ++lw) {
            const int buf = lw & 1;
            ok = mbar_wait(&tfull[buf], (lw >> 1) & 1);
            if (!ok) break;
            tc_fence_after();
            const int w = (int)blockIdx.x + lw * (int)gridDim.x;
            const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * 128);
            __nv_bfloat16 *th = p.Theta + (size_t)w * p.thetaStride + p.tOff;
            zd *tz = p.thetaZ ? p.thetaZ + (size_t)w * p.zStride + p.tOff : nullptr;
            double *tzd = (double *)tz;
            for (int c0 = 0; c0 < 2 * Nsp; c0 += 32) {
                float v[32];
                tmem_ld32(trow + (uint32_t)c0, v);
                if (row < n) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const int col = c0 + j;
                        const int im = col >= Nsp ? 1 : 0;
                        const int a = col - im * Nsp;
                        if (a < Ns) {
                            const size_t o = (size_t)row + (size_t)n * a;
                            th[o + im * p.plane] = __float2bfloat16_rn(v[j]);
                            if (tzd) tzd[2 * o + im] = (double)v[j];
                        }
                    }
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

// B rows of walker w (K-major, 2 Nsp values each): row a (< Nsp): [Re S(b, a) | -Im S(b, a)],
// row Nsp + a: [Im S(b, a) | Re S(b, a)], b over Nsp (zero beyond Ns); hi and
// (with comp = 3) lo tf32 parts.  Walkers outside `mask` get zeros.
__global__ void build_b_kernel(int W, int Ns, int Nsp, const zd *Sinv, long long sStride, long long sOff,
                               const int *mask, int comp, float *Bh, float *Bl)
{
    const int w = blockIdx.x;
    const bool on = mask == nullptr || mask[w] != 0;
    const int K2 = 2 * Nsp;
    float *bh = Bh + (size_t)w * K2 * K2;
    float *bl = comp == 3 ? Bl + (size_t)w * K2 * K2 : nullptr;
    const zd *S = Sinv + (size_t)w * sStride + sOff;
    for (int e = threadIdx.x; e < Nsp * Nsp; e += blockDim.x) {
        const int b = e % Nsp, a = e / Nsp;
        zd v = make_double2(0.0, 0.0);
        if (on && a < Ns && b < Ns) v = S[b + (size_t)Ns * a];
        const double vals[4] = {v.x, -v.y, v.y, v.x};
        const size_t idx[4] = {(size_t)a * K2 + b, (size_t)a * K2 + Nsp + b, (size_t)(Nsp + a) * K2 + b,
                               (size_t)(Nsp + a) * K2 + Nsp + b};
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const float h = tf32_round((float)vals[t]);
            bh[idx[t]] = h;
            if (bl) bl[idx[t]] = tf32_round((float)(vals[t] - (double)h));
        }
    }
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
            const cuuint32_t *box, CUtensorMapSwizzle swz = CU_TENSOR_MAP_SWIZZLE_128B)
{
    auto enc = encoder();
    if (!enc) return (int)cudaErrorNotSupported;
    if ((uintptr_t)ptr & 15) return (int)cudaErrorMisalignedAddress;
    for (int i = 0; i + 1 < rank; ++i)
        if (pitch[i] & 15) return (int)cudaErrorMisalignedAddress;
    cuuint32_t es[3] = {1u, 1u, 1u};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, const_cast<float *>(ptr), dims, pitch, box,
                     es, CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : (int)r + 10000;
}

}  // namespace

bool theta_tc_supported(int n, int Ns) { return (n == 64 || n == 128) && Ns >= 1 && Ns <= 64; }

size_t theta_tc_bscratch(int W, int Ns)
{
    const int Nsp = (Ns + 15) / 16 * 16;
    return (size_t)W * 4 * Nsp * Nsp;
}

int theta_tc_launch(cudaStream_t s, int n, int ncol, int Ns, int W, const float *w32, const zd *Sinv,
                    long long sStride, long long sOff, const int *mask, int comp, float *Bh, float *Bl,
                    __nv_bfloat16 *Theta, long long thetaStride, long long plane, long long tOff, zd *thetaZ,
                    long long zStride, int *err)
{
    if (!theta_tc_supported(n, Ns) || (comp != 1 && comp != 3)) return (int)cudaErrorInvalidValue;
    const int Nsp = (Ns + 15) / 16 * 16;
    g_launch_count++;
    build_b_kernel<<<W, 256, 0, s>>>(W, Ns, Nsp, Sinv, sStride, sOff, mask, comp, Bh, Bl);
    cudaError_t ce = cudaGetLastError();
    if (ce != cudaSuccess) return (int)ce;

    ThArgs a{};
    a.n = n; a.Ns = Ns; a.Nsp = Nsp; a.W = W; a.comp = comp;
    a.nchunk = n / 32;
    a.nkb = (Nsp + BK - 1) / BK;
    a.rawBytes = (uint32_t)(a.nchunk * Nsp * 128);
    a.aBytes = (uint32_t)(a.nkb * 128 * 128);
    a.bBytes = (uint32_t)(a.nkb * 2 * Nsp * 128);
    a.stageBytes = a.rawBytes + 2 * a.aBytes + 2 * a.bBytes;
    const size_t budget = 200 * 1024;
    a.stages = (int)std::max<size_t>(1, std::min<size_t>(4, budget / a.stageBytes));
    a.idesc = idesc_tf32(128, 2 * Nsp);
    a.Theta = Theta; a.thetaStride = thetaStride; a.plane = plane; a.tOff = tOff;
    a.thetaZ = thetaZ; a.zStride = zStride; a.err = err;

    CUtensorMap mA, mBh, mBl;
    cuuint64_t dA[3] = {(cuuint64_t)n, (cuuint64_t)ncol, (cuuint64_t)2 * W};
    cuuint64_t pA[2] = {(cuuint64_t)n * 4, (cuuint64_t)n * ncol * 4};
    cuuint32_t bA[3] = {32u, (cuuint32_t)Nsp, 1u};
    int r = map_f32(&mA, w32, 3, dA, pA, bA, CU_TENSOR_MAP_SWIZZLE_NONE);
    cuuint64_t dB[2] = {(cuuint64_t)2 * Nsp, (cuuint64_t)2 * Nsp * W};
    cuuint64_t pB[1] = {(cuuint64_t)2 * Nsp * 4};
    cuuint32_t bB[2] = {(cuuint32_t)BK, (cuuint32_t)(2 * Nsp)};
    if (!r) r = map_f32(&mBh, Bh, 2, dB, pB, bB);
    if (!r) r = map_f32(&mBl, comp == 3 ? Bl : Bh, 2, dB, pB, bB);
    if (r) return r;
    const size_t smem = 1024 + (size_t)a.stages * a.stageBytes + 256;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(theta_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr = true;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = std::min(W, sms);
    g_launch_count++;
    theta_tc_kernel<<<grid, NT, smem, s>>>(mA, mBh, mBl, a);
    return (int)cudaGetLastError();
}
