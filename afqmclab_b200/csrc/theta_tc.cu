// theta_b = phi S_b^{-1} (n x Ns_b per walker and spin block) on the tcgen05
// tensor cores (kind::tf32, fp32 accumulation), from the fp32 planar walkers
// and the inverse overlaps (fp32 planes written by the LU).  The spin blocks
// share the walker (SD2is: both use its leading columns), so one walker
// operand serves both: the walker tile arrives by TMA with the sites
// contiguous and is rewritten in shared memory as a K-major operand P
// (row = site, 128-byte swizzle), and the operand X stacks the blocks'
// S^{-1} rows (block, column a, re/im):
//   theta_re = phi_re S_re - phi_im S_im,  theta_im = phi_re S_im + phi_im S_re
// as one real product X P^T over K = (re part, im part) x electrons.  Both
// operands are split into tf32 high and low parts and
// X_hi P_hi + X_lo P_hi + X_hi P_lo is accumulated (about 22 significant
// bits).  Replaces the zgetrs('T') solve of SDSDOperation.cpp:166-173 /
// SD2sSD2isOperation.cpp:187-198 in the mixed-precision form.
//
// Persistent CTAs, one walker at a time, two items per walker (the re and im
// halves of K).  Three rings keep the loads ahead of the work: raw walker
// chunks (TMA, per item), the walker's inverse slot (bulk copy, per walker)
// and the split operands (per item).
//   warp 0 lane 0 : producer (TMA walker chunks, bulk copy of the inverses)
//   warp 1        : TMEM owner, UMMA issuer
//   warps 2..9    : rewrite of P (K-major, hi/lo) and build of X (hi/lo)
//   warps 10..13  : epilogue (double-buffered TMEM): TMEM lane = output
//                   column, so each thread writes its column over the sites
//                   with 16-byte stores
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <string>

#include "engine_internal.cuh"
#include "tc_common.cuh"
#include "theta_tc.cuh"
#include "once.cuh"

extern std::atomic<long long> g_launch_count;

namespace {

constexpr int NCONV = 256;                 // converter threads (warps 2..9)
constexpr int NT = 64 + NCONV + 128;       // + producer, MMA warps and 4 epilogue warps
constexpr int MAX_RS = 4, MAX_XS = 2, MAX_OS = 2;
constexpr size_t SMEM_CAP = 227 * 1024;

struct ThArgs {
    int n, Nsp, W, nchunk, nkb, nb;
    int RS, XS, OS;
    int Ns[2];
    long long sOff[2], tOff[2];
    uint32_t rawBytes, xBytes, opBytes, idesc;
    const float *Sinv32;   // fp32 planes [re | im] of S_b^{-1} at + w s32 + 2 sOff[b]
    long long s32;
    const int *mask;
    __nv_bfloat16 *Theta;  // + w * thetaStride + tOff[b], planes `plane` apart
    long long thetaStride, plane;
    zd *thetaZ;            // optional FP64 copy, + w * zStride + tOff[b]
    long long zStride;
    int *err;
};

__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// element (row, k) of a K-major, 128-byte-swizzled fp32 operand of 128 rows
__device__ __forceinline__ uint32_t sw_off(int row, int k)
{
    return (uint32_t)((k >> 5) * 128 * 128 + row * 128 + ((((k & 31) >> 2) ^ (row & 7)) << 4) + (k & 3) * 4);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *(const uint32_t *)&h;
}

// four fp32 values as tf32 high parts and tf32-rounded remainders (16-byte stores)
__device__ __forceinline__ void store_split(uint8_t *hi, uint8_t *lo, uint32_t off, const float *v)
{
    float4 h, l;
    h.x = tf32_round(v[0]); l.x = tf32_round(v[0] - h.x);
    h.y = tf32_round(v[1]); l.y = tf32_round(v[1] - h.y);
    h.z = tf32_round(v[2]); l.z = tf32_round(v[2] - h.z);
    h.w = tf32_round(v[3]); l.w = tf32_round(v[3] - h.w);
    *(float4 *)(hi + off) = h;
    *(float4 *)(lo + off) = l;
}

template <int NSP>
__global__ void __launch_bounds__(NT, 1)
theta_tc_kernel(const __grid_constant__ CUtensorMap tA, ThArgs p)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    // [OS operand stages: P hi | P lo | X hi | X lo][RS raw chunks][XS inverse slots][barriers]
    uint8_t *ops = base;
    uint8_t *raws = ops + (size_t)p.OS * p.opBytes;
    uint8_t *xsl = raws + (size_t)p.RS * p.rawBytes;
    uint64_t *rawFull = (uint64_t *)(xsl + (size_t)p.XS * p.xBytes);
    uint64_t *rawEmpty = rawFull + MAX_RS;
    uint64_t *xFull = rawEmpty + MAX_RS;
    uint64_t *xEmpty = xFull + MAX_XS;
    uint64_t *opFull = xEmpty + MAX_XS;
    uint64_t *opEmpty = opFull + MAX_OS;
    uint64_t *tfull = opEmpty + MAX_OS;   // 2
    uint64_t *tempty = tfull + 2;         // 2
    uint32_t *tmemSlot = (uint32_t *)(tempty + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nw = (p.W - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;   // walkers of this CTA
    const int items = 2 * nw;
    const uint32_t pBytes = (uint32_t)p.nkb * 128 * 128;   // one of P hi, P lo, X hi, X lo

    if (threadIdx.x == 0) {
        for (int s = 0; s < p.RS; ++s) { mbar_init(&rawFull[s], 1); mbar_init(&rawEmpty[s], NCONV); }
        for (int s = 0; s < p.XS; ++s) { mbar_init(&xFull[s], 1); mbar_init(&xEmpty[s], NCONV); }
        for (int s = 0; s < p.OS; ++s) { mbar_init(&opFull[s], NCONV); mbar_init(&opEmpty[s], 1); }
        for (int b = 0; b < 2; ++b) { mbar_init(&tfull[b], 1); mbar_init(&tempty[b], 128); }
        fence_mbar_init();
        tma_prefetch_desc(&tA);
    }
    if (warp == 1) { tmem_alloc(tmemSlot, 256); tmem_relinquish(); }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmemSlot;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {
            for (int lw = 0; lw < nw && ok; ++lw) {
                const int w = (int)blockIdx.x + lw * (int)gridDim.x;
                const int xs = lw % p.XS;
                if (lw >= p.XS) ok = mbar_wait_sleep(&xEmpty[xs], ((lw / p.XS) - 1) & 1);
                if (!ok) break;
                mbar_arrive_expect_tx(&xFull[xs], p.xBytes);
                bulk_load(xsl + (size_t)xs * p.xBytes, p.Sinv32 + (size_t)w * p.s32, p.xBytes, &xFull[xs]);
                for (int part = 0; part < 2 && ok; ++part) {
                    const int it = 2 * lw + part, rs = it % p.RS;
                    if (it >= p.RS) ok = mbar_wait_sleep(&rawEmpty[rs], ((it / p.RS) - 1) & 1);
                    if (!ok) break;
                    uint8_t *dst = raws + (size_t)rs * p.rawBytes;
                    mbar_arrive_expect_tx(&rawFull[rs], p.rawBytes);
                    for (int c = 0; c < p.nchunk; ++c)
                        tma_load_3d(dst + c * p.Nsp * 128, &tA, &rawFull[rs], c * 32, 0, 2 * w + part);
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            for (int it = 0; it < items && ok; ++it) {
                const int os = it % p.OS, lw = it >> 1, part = it & 1, buf = lw & 1;
                if (part == 0 && lw >= 2) {
                    ok = mbar_wait_sleep(&tempty[buf], ((lw >> 1) - 1) & 1);
                    if (!ok) break;
                }
                ok = mbar_wait_sleep(&opFull[os], (it / p.OS) & 1);
                if (!ok) break;
                tc_fence_after();
                const uint32_t st = smem_u32(ops + (size_t)os * p.opBytes);
                const uint32_t ph = st, pl = st + pBytes, xh = st + 2 * pBytes, xl = st + 3 * pBytes;
                const uint32_t d = tmem + (uint32_t)(buf * 128);
#pragma unroll
                for (int kk = 0; kk < NSP / 8; ++kk) {
                    // D (rows = block, column, re/im; columns = sites) = X P^T
                    const uint32_t off = (uint32_t)((kk >> 2) * 128 * 128 + (kk & 3) * 32);
                    const uint32_t acc0 = (part > 0 || kk > 0) ? 1u : 0u;
                    umma_tf32(d, desc_k_sw128(xh + off), desc_k_sw128(ph + off), p.idesc, acc0);
                    umma_tf32(d, desc_k_sw128(xl + off), desc_k_sw128(ph + off), p.idesc, 1u);
                    umma_tf32(d, desc_k_sw128(xh + off), desc_k_sw128(pl + off), p.idesc, 1u);
                }
                umma_commit(&opEmpty[os]);
                if (part == 1) umma_commit(&tfull[buf]);
            }
        }
        __syncwarp();
    } else if (warp < 2 + NCONV / 32) {
        const int t = threadIdx.x - 64;
        constexpr int Nsp = NSP, G4 = NSP / 4;
        constexpr int units = 128 * G4;
        const int tasks = p.nb * Nsp * G4;   // (block, column a, group of 4 electrons c)
        for (int it = 0; it < items && ok; ++it) {
            const int lw = it >> 1, part = it & 1;
            const int w = (int)blockIdx.x + lw * (int)gridDim.x;
            const int rs = it % p.RS, os = it % p.OS, xs = lw % p.XS;
            const bool on = p.mask == nullptr || p.mask[w] != 0;
            ok = mbar_wait_sleep(&rawFull[rs], (it / p.RS) & 1);
            if (ok && it >= p.OS) ok = mbar_wait_sleep(&opEmpty[os], ((it / p.OS) - 1) & 1);
            if (ok) ok = mbar_wait_sleep(&xFull[xs], (lw / p.XS) & 1);
            if (!ok) break;
            const uint8_t *raw = raws + (size_t)rs * p.rawBytes;
            const float *xsrc = (const float *)(xsl + (size_t)xs * p.xBytes);
            uint8_t *ph = ops + (size_t)os * p.opBytes;
            uint8_t *pl = ph + pBytes, *xh = ph + 2 * pBytes, *xl = ph + 3 * pBytes;
            // P: the raw chunks (Nsp rows of 32 sites each) as K-major rows
            // (row = site), split into hi and lo
#pragma unroll
            for (int u = t; u < units; u += NCONV) {
                const int i = u & 127, k4 = u >> 7;
                float x[4];
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    x[j] = i < p.n ? *(const float *)(raw + (i >> 5) * Nsp * 128 + (4 * k4 + j) * 128 + (i & 31) * 4)
                                   : 0.f;
                float4 h, l;
                h.x = tf32_round(x[0]); l.x = x[0] - h.x;
                h.y = tf32_round(x[1]); l.y = x[1] - h.y;
                h.z = tf32_round(x[2]); l.z = x[2] - h.z;
                h.w = tf32_round(x[3]); l.w = x[3] - h.w;
                const uint32_t off = sw_off(i, 4 * k4);
                *(float4 *)(ph + off) = h;
                *(float4 *)(pl + off) = l;
            }
            mbar_arrive(&rawEmpty[rs]);
            // X: rows 2 Nsp b + 2 a (theta_re) and 2 Nsp b + 2 a + 1 (theta_im);
            // K = electron c of this item's part:
            //   re part: [S_re(c, a) ; S_im(c, a)],  im part: [-S_im(c, a) ; S_re(c, a)]
#pragma unroll 2
            for (int q = t; q < tasks; q += NCONV) {
                const int g = q % G4, a = (q / G4) % Nsp, b = q / (G4 * Nsp);
                const int Ns = b ? p.Ns[1] : p.Ns[0];
                const long long so = 2 * (b ? p.sOff[1] : p.sOff[0]);
                float xr[4] = {0.f, 0.f, 0.f, 0.f}, xi[4] = {0.f, 0.f, 0.f, 0.f};
                if (on && a < Ns) {
                    const float *Xr = xsrc + so + (size_t)Ns * a, *Xi = Xr + (size_t)Ns * Ns;
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        if (4 * g + j < Ns) { xr[j] = Xr[4 * g + j]; xi[j] = Xi[4 * g + j]; }
                }
                float vre[4], vim[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    vre[j] = part ? -xi[j] : xr[j];
                    vim[j] = part ? xr[j] : xi[j];
                }
                const int rRe = 2 * Nsp * b + 2 * a;
                store_split(xh, xl, sw_off(rRe, 4 * g), vre);
                store_split(xh, xl, sw_off(rRe + 1, 4 * g), vim);
            }
            if (part == 1) mbar_arrive(&xEmpty[xs]);
            fence_proxy_async();
            mbar_arrive(&opFull[os]);
        }
    } else {
        // lane r of the accumulator = (block b, column a, re/im): theta_b(:, a)
        // of one part over the sites, contiguous in Theta and thetaZ
        const int q = warp & 3;
        const int r = q * 32 + lane;
        constexpr int Nsp = NSP;
        const int n = p.n;
        const int b = r / (2 * Nsp), rr = r - b * 2 * Nsp, a = rr >> 1, im = rr & 1;
        const int Ns = b == 0 ? p.Ns[0] : (b == 1 ? p.Ns[1] : 0);
        const bool valid = b < p.nb && a < Ns;
        const long long tOff = b ? p.tOff[1] : p.tOff[0];
        for (int lw = 0; lw < nw && ok; ++lw) {
            const int buf = lw & 1;
            ok = mbar_wait_sleep(&tfull[buf], (lw >> 1) & 1);
            if (!ok) break;
            tc_fence_after();
            const int w = (int)blockIdx.x + lw * (int)gridDim.x;
            const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * 128);
            __nv_bfloat16 *th = p.Theta + (size_t)w * p.thetaStride + tOff + (size_t)im * p.plane + (size_t)n * a;
            double2 *tz = p.thetaZ ? (double2 *)(p.thetaZ + (size_t)w * p.zStride + tOff + (size_t)n * a) : nullptr;
            for (int c0 = 0; c0 < n; c0 += 32) {
                float v[32];
                tmem_ld32(trow + (uint32_t)c0, v);
                if (valid) {
#pragma unroll
                    for (int j = 0; j < 32; j += 8) {
                        uint4 pk;
                        pk.x = pack_bf16x2(v[j], v[j + 1]);
                        pk.y = pack_bf16x2(v[j + 2], v[j + 3]);
                        pk.z = pack_bf16x2(v[j + 4], v[j + 5]);
                        pk.w = pack_bf16x2(v[j + 6], v[j + 7]);
                        *(uint4 *)(th + c0 + j) = pk;
                    }
                }
                if (tz) {
                    // the re lane keeps sites c0..c0+15, the im lane c0+16..c0+31
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const float send = im ? v[j] : v[16 + j];
                        const float recv = __shfl_xor_sync(0xffffffffu, send, 1);
                        if (valid) {
                            if (im) tz[c0 + 16 + j] = make_double2((double)recv, (double)v[16 + j]);
                            else tz[c0 + j] = make_double2((double)v[j], (double)recv);
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
            const cuuint32_t *box, CUtensorMapSwizzle swz)
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

struct Plan {
    int Nsp, nkb, nchunk, RS, XS, OS;
    uint32_t rawBytes, xBytes, opBytes;
    size_t smem;
};

// ring depths: the deepest (operand stages, raw chunks, inverse slots) that fits
bool make_plan(int n, int nb, const int *Ns, long long s32, Plan &pl)
{
    if ((n != 64 && n != 128) || nb < 1 || nb > 2 || s32 <= 0 || (s32 & 3)) return false;
    int maxNs = 0;
    for (int b = 0; b < nb; ++b) {
        if (Ns[b] < 1 || Ns[b] > 64) return false;
        maxNs = std::max(maxNs, Ns[b]);
    }
    pl.Nsp = (maxNs + 15) / 16 * 16;
    if (2 * nb * pl.Nsp > 128) return false;
    pl.nkb = (pl.Nsp + 31) / 32;
    pl.nchunk = n / 32;
    pl.rawBytes = (uint32_t)(pl.nchunk * pl.Nsp * 128);
    pl.xBytes = (uint32_t)(s32 * 4);
    pl.opBytes = (uint32_t)(4 * pl.nkb * 128 * 128);
    const int tries[][3] = {{2, 4, 2}, {2, 3, 2}, {2, 2, 2}, {2, 2, 1}, {1, 4, 2}, {1, 2, 2}, {1, 2, 1}, {1, 1, 1}};
    for (const auto &t : tries) {
        const size_t smem = 1024 + (size_t)t[0] * pl.opBytes + (size_t)t[1] * pl.rawBytes + (size_t)t[2] * pl.xBytes + 256;
        if (smem <= SMEM_CAP) {
            pl.OS = t[0]; pl.RS = t[1]; pl.XS = t[2]; pl.smem = smem;
            return true;
        }
    }
    return false;
}

}  // namespace

bool theta_tc_supported(int n, int nb, const int *Ns, long long s32)
{
    Plan pl;
    return make_plan(n, nb, Ns, s32, pl);
}

int theta_tc_launch(cudaStream_t s, int n, int ncol, int nb, const int *Ns, int W, const float *w32,
                    const float *Sinv32, long long s32, const long long *sOff, const int *mask,
                    __nv_bfloat16 *Theta, long long thetaStride, long long plane, const long long *tOff,
                    zd *thetaZ, long long zStride, int *err)
{
    Plan pl;
    if (!make_plan(n, nb, Ns, s32, pl)) return (int)cudaErrorInvalidValue;
    if ((uintptr_t)Sinv32 & 15) return (int)cudaErrorMisalignedAddress;
    ThArgs a{};
    a.n = n; a.Nsp = pl.Nsp; a.W = W; a.nb = nb;
    a.nchunk = pl.nchunk; a.nkb = pl.nkb;
    a.RS = pl.RS; a.XS = pl.XS; a.OS = pl.OS;
    for (int b = 0; b < 2; ++b) {
        a.Ns[b] = b < nb ? Ns[b] : 0;
        a.sOff[b] = b < nb ? sOff[b] : 0;
        a.tOff[b] = b < nb ? tOff[b] : 0;
    }
    a.rawBytes = pl.rawBytes; a.xBytes = pl.xBytes; a.opBytes = pl.opBytes;
    a.idesc = idesc_tf32(128, 128);
    a.Sinv32 = Sinv32; a.s32 = s32; a.mask = mask;
    a.Theta = Theta; a.thetaStride = thetaStride; a.plane = plane;
    a.thetaZ = thetaZ; a.zStride = zStride; a.err = err;

    CUtensorMap mA;
    cuuint64_t dA[3] = {(cuuint64_t)n, (cuuint64_t)ncol, (cuuint64_t)2 * W};
    cuuint64_t pA[2] = {(cuuint64_t)n * 4, (cuuint64_t)n * ncol * 4};
    cuuint32_t bA[3] = {32u, (cuuint32_t)pl.Nsp, 1u};
    int r = map_f32(&mA, w32, 3, dA, pA, bA, CU_TENSOR_MAP_SWIZZLE_NONE);
    if (r) return r;
    static std::atomic<unsigned long long> attr{0};
    if (first_on_device(attr)) {
        cudaFuncSetAttribute(theta_tc_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_CAP);
        cudaFuncSetAttribute(theta_tc_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_CAP);
        cudaFuncSetAttribute(theta_tc_kernel<48>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_CAP);
        cudaFuncSetAttribute(theta_tc_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_CAP);
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = std::min(W, sms);
    g_launch_count++;
    switch (pl.Nsp) {
    case 16: theta_tc_kernel<16><<<grid, NT, pl.smem, s>>>(mA, a); break;
    case 32: theta_tc_kernel<32><<<grid, NT, pl.smem, s>>>(mA, a); break;
    case 48: theta_tc_kernel<48><<<grid, NT, pl.smem, s>>>(mA, a); break;
    default: theta_tc_kernel<64><<<grid, NT, pl.smem, s>>>(mA, a); break;
    }
    return (int)cudaGetLastError();
}
