// Mixed-precision form of the phaseless walker step.
//
// Walkers are stored as complex fp32 (planar: real plane then imaginary
// plane, each n x ncol column-major).  The dense contractions run on the
// tcgen05 tensor cores in bf16 with fp32 accumulation:
//   force      xbar = A^T Theta            (calculateCholeskyBg, :237-256)
//   two-body   M = sqrt(-dt) sum_g x_g L_g (CholeskyReal::setTwoBodySampleMatrix)
//   Taylor     exp(M) phi, all orders in one kernel (LogHop2isSD2isOperation)
//   one-body   exp(-dt K) phi = phi + (exp(-dt K) - 1) phi
// while the overlap matrices, their LU / log-determinant / inverse, the phase
// and cos projections, the weights, population control and the Gram-Schmidt
// re-orthonormalisation stay in FP64 (FP64 arithmetic on the fp32 walker).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "engine_internal.cuh"
#include "mixed.cuh"
#include "cp_mixed.cuh"
#include "exchange_gemm.cuh"
#include "overlap_tc.cuh"
#include "theta_tc.cuh"
#include "tc_common.cuh"
#include "tc_gemm.cuh"
#include "once.cuh"

struct MixedState {
    float *wf32 = nullptr, *tmp32 = nullptr;
    __nv_bfloat16 *Theta = nullptr, *Abig = nullptr, *Y = nullptr, *Lt = nullptr, *Mbuf = nullptr,
                  *Et = nullptr;
    float *xbarp = nullptr;
    zd *wfDaggerTm = nullptr;
    __nv_bfloat16 *A2r[2] = {nullptr, nullptr}, *A2i[2] = {nullptr, nullptr};
    bool realA = false;   // every A_g has a zero imaginary part (real trial, real Cholesky vectors)
    zd *ex2 = nullptr;
    // exchange as GEMMs (real A): per-block V, scratch, per-walker sum over g
    bool exGemm = false;
    ExGemmBlock exg[2];
    ExGemmScratch exs;
    zd *exTot = nullptr;
    // spin-restricted: the two spin blocks have the same trial and (nup = ndn)
    // the same walker columns, so every per-spin quantity of block 1 equals
    // block 0's; bl1 lists block 0 alone with log-det multiplicity 2 and the
    // force, exchange and kinetic sums of block 0 are doubled
    bool restricted = false;
    Blocks bl1{};
    float *Ohi[2] = {nullptr, nullptr}, *Olo[2] = {nullptr, nullptr};   // overlap operators
    bool ovStacked = false;   // Ohi[0]/Olo[0] hold both blocks' operators
    float *Sinv32 = nullptr;   // S^{-1} as fp32 planes [re | im] per block slot
    float *E1h = nullptr, *E1l = nullptr; // exp(+dt/2 K) - I, tf32 high/low (measurement)
    float *sh = nullptr, *sl = nullptr;   // walkers split into tf32 high/low parts
    int *err = nullptr;
    int splits = 1;
    long long ws32 = 0;  // floats per walker (2 n ncol)
    bool ready = false;
};

namespace {

#define MTRY(expr)                   \
    do {                             \
        int _r = (expr);             \
        if (_r != AFQMC_OK) return _r; \
    } while (0)

int cuda_check(cudaError_t r, const char *what)
{
    if (r != cudaSuccess) return engine_fail(AFQMC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(r));
    return AFQMC_OK;
}

// ------------------------------------------------------------ setup kernels
// Force operand, K-major rows: [Re; Im] outputs x [Re; Im] inputs of the
// complex product xbar_g = sum_k A_gk Theta_k with Theta stored per spin as
// theta(i, b) at tOff + i + n b (b = electron, i = orbital).
__global__ void build_abig_kernel(int G, long long Ktot, int n, Blocks bl, const zd *Aall,
                                  __nv_bfloat16 *Abig)
{
    const long long K2 = 2 * Ktot;
    const long long total = (long long)G * Ktot;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int g = (int)(e / Ktot);
        long long kap = e % Ktot;
        int b = bl.nblk > 1 && kap >= bl.tOff[1] ? 1 : 0;
        long long r = kap - bl.tOff[b];
        int Ns = bl.Ns[b];
        int i = (int)(r % n), bb = (int)(r / n);
        zd a = Aall[(size_t)g * Ktot + bl.tOff[b] + bb + (size_t)Ns * i];
        Abig[(size_t)g * K2 + kap] = __double2bfloat16(a.x);
        Abig[(size_t)g * K2 + Ktot + kap] = __double2bfloat16(-a.y);
        Abig[(size_t)(G + g) * K2 + kap] = __double2bfloat16(a.y);
        Abig[(size_t)(G + g) * K2 + Ktot + kap] = __double2bfloat16(a.x);
    }
}

// L_g transposed to K-major rows: Lt[m * G + g] = chol[m + n^2 g]
__global__ void build_lt_kernel(long long n2, int G, const double *chol, __nv_bfloat16 *Lt)
{
    const long long total = n2 * G;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        long long m = e / G;
        int g = (int)(e % G);
        Lt[e] = __double2bfloat16(chol[m + n2 * g]);
    }
}

// (exp(-dt K) - 1) as a K-major bf16 operand: Et[i n + j] = E(i, j) - delta_ij
__global__ void build_et_kernel(int n, const zd *E, __nv_bfloat16 *Et)
{
    const int total = n * n;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        int i = e / n, j = e % n;
        double v = E[i + (size_t)n * j].x - (i == j ? 1.0 : 0.0);
        Et[e] = __double2bfloat16(v);
    }
}

// wfDaggerT permuted from the (b + Ns i) to the (i + n b) layout of each block
__global__ void permute_wdt_kernel(int n, Blocks bl, const zd *src, zd *dst)
{
    for (int b = 0; b < bl.nblk; ++b) {
        int Ns = bl.Ns[b];
        for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < Ns * n; e += gridDim.x * blockDim.x) {
            int i = e % n, bb = e / n;
            dst[bl.tOff[b] + e] = src[bl.tOff[b] + bb + (size_t)Ns * i];
        }
    }
}

// ---------------------------------------------------------- walker storage
__global__ void wf_to_f32p_kernel(int W, long long wsize, const zd *wf, float *w32, const int *mask)
{
    const int w = blockIdx.x;
    if (mask && !mask[w]) return;
    for (long long e = threadIdx.x; e < wsize; e += blockDim.x) {
        zd v = wf[(size_t)w * wsize + e];
        w32[(size_t)w * 2 * wsize + e] = (float)v.x;
        w32[(size_t)w * 2 * wsize + wsize + e] = (float)v.y;
    }
}
__global__ void f32p_to_wf_kernel(int W, long long wsize, const float *w32, zd *wf, const int *mask)
{
    const int w = blockIdx.x;
    if (mask && !mask[w]) return;
    for (long long e = threadIdx.x; e < wsize; e += blockDim.x)
        wf[(size_t)w * wsize + e] = make_double2(w32[(size_t)w * 2 * wsize + e],
                                                 w32[(size_t)w * 2 * wsize + wsize + e]);
}

// populationControl<T> in-place copies of fp32 walkers (populationControl.h:110-117)
__global__ void gather32_kernel(int W, long long ws32, const int *table, float *w32, zd *logw)
{
    const int i = blockIdx.x;
    const int j = table[i];
    if (j == i || j < 0) return;
    const float4 *src = (const float4 *)(w32 + (size_t)j * ws32);
    float4 *dst = (float4 *)(w32 + (size_t)i * ws32);
    for (long long e = threadIdx.x; e < ws32 / 4; e += blockDim.x) dst[e] = src[e];
    if (threadIdx.x == 0) logw[i] = logw[j];
}

// Gram-Schmidt (SD2is::stabilize, SD2is.cpp:48-76) on an fp32 walker: norms,
// projections and updates in FP64, the columns kept in fp32 between updates
// (the walker's own precision), which halves the shared memory per walker.
// n <= 128 (the mixed form runs n = 64 or 128).
__global__ void __launch_bounds__(256, 5)
mgs32_kernel(int W, int n, int ncol, int nup, int ndn, float *w32, zd *logw, const int *alive,
             int *status)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[32];
    const int w = blockIdx.x;
    if (alive && !alive[w]) return;
    float2 *A = (float2 *)smem_raw;   // the walker, fp32 (columns stored between FP64 updates)
    float *g = w32 + (size_t)w * 2 * n * ncol;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
    const long long ws = (long long)n * ncol;
    for (long long e = tid; e < ws; e += nt) A[e] = make_float2(g[e], g[ws + e]);
    __syncthreads();
    const int nmin = nup < ndn ? nup : ndn;
    double logR = 0.0, logRmin = 0.0;
    int bad = 0;
    for (int j = 0; j < ncol; ++j) {
        double s = 0.0;
        for (int i = tid; i < n; i += nt) {
            const float2 v = A[i + (size_t)n * j];
            s += (double)v.x * v.x + (double)v.y * v.y;
        }
        s = block_sum(s, red);
        double r = sqrt(s);
        if (r == 0.0) bad = 1;
        double inv = r > 0.0 ? 1.0 / r : 0.0;
        for (int i = tid; i < n; i += nt) {
            const float2 v = A[i + (size_t)n * j];
            A[i + (size_t)n * j] = make_float2((float)(v.x * inv), (float)(v.y * inv));
        }
        if (tid == 0) {
            double lr = log(r);
            logR += lr;
            if (j < nmin) logRmin += lr;
        }
        __syncthreads();
        // This lane's rows i = lane + 32 r of column j (n <= 128: at most four),
        // converted to FP64 once per column; each column c's rows are converted
        // once and kept for both the projection and the update (the fp32 <->
        // FP64 conversions, not the FMAs, bound this loop).
        zd qv[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int i = lane + 32 * r;
            const float2 q = i < n ? A[i + (size_t)n * j] : make_float2(0.f, 0.f);
            qv[r] = make_double2(q.x, q.y);
        }
        for (int c = j + 1 + wid; c < ncol; c += nw) {
            zd d = make_double2(0.0, 0.0);
            zd vv[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int i = lane + 32 * r;
                const float2 v = i < n ? A[i + (size_t)n * c] : make_float2(0.f, 0.f);
                vv[r] = make_double2(v.x, v.y);
                if (i < n) zfma(d, make_double2(qv[r].x, -qv[r].y), vv[r]);
            }
            d.x = warp_sum(d.x);
            d.y = warp_sum(d.y);
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int i = lane + 32 * r;
                if (i < n) {
                    const double vx = vv[r].x - (d.x * qv[r].x - d.y * qv[r].y);
                    const double vy = vv[r].y - (d.x * qv[r].y + d.y * qv[r].x);
                    A[i + (size_t)n * c] = make_float2((float)vx, (float)vy);
                }
            }
        }
        __syncthreads();
    }
    for (long long e = tid; e < ws; e += nt) { g[e] = A[e].x; g[ws + e] = A[e].y; }
    if (tid == 0) {
        zd lw = logw[w];
        if (nup == ndn) lw.x += 2.0 * logR;
        else lw.x += logR + logRmin;
        logw[w] = lw;
        if (bad && status) atomicOr(status + w, (int)ST_ZERO_NORM);
    }
}

// Phaseless force from the tensor-core xbar partials, aux sampling, sample
// log-weight and second cos projection (same arithmetic as the FP64 form),
// writing y = sqrt(-dt) x as the bf16 operand of the two-body GEMM.  One warp
// per walker (four walkers per block): a walker's sums need no block barrier
// and more walkers are in flight per SM.  Each lane takes its fields two at a
// time (g and g + 32): both fields' loads and Gaussians are issued before the
// first field's stores, and the sums still run in field order.
__global__ void __launch_bounds__(128, 4)
mixed_sample_warp_kernel(int W, CholDev c, const float *xbarp, int splits, long long splitStride,
                         int *surv, int *alive, const unsigned long long *offs, uint64_t seed,
                         __nv_bfloat16 *Y, zd *logw, double dtET, zd hopLogw)
{
    const int lane = threadIdx.x & 31;
    const int w = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (w >= W || !surv[w]) return;
    const int G = c.G;
    const unsigned long long off = offs[w];
    zd f2 = make_double2(0, 0), xf = make_double2(0, 0), xb = make_double2(0, 0);
    for (int g0 = lane; g0 < G; g0 += 64) {
        const int nf = g0 + 32 < G ? 2 : 1;
        double xr[2] = {0.0, 0.0}, xi[2] = {0.0, 0.0}, bgv[2] = {0.0, 0.0}, gs[2] = {0.0, 0.0};
        zd cf[2] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            if (u < nf) {
                const int g = g0 + 32 * u;
                bgv[u] = c.bg[g];
                if (c.constForce) {
                    cf[u] = c.constForce[g];
                } else {
                    for (int s = 0; s < splits; ++s) {
                        xr[u] += xbarp[s * splitStride + g + (size_t)2 * G * w];
                        xi[u] += xbarp[s * splitStride + G + g + (size_t)2 * G * w];
                    }
                }
            }
        }
#pragma unroll
        for (int u = 0; u < 2; ++u)
            if (u < nf) gs[u] = rng_gaussian(seed, off + 2ULL * (g0 + 32 * u));
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            if (u < nf) {
                const int g = g0 + 32 * u;
                zd f;
                if (c.constForce) {
                    f = cf[u];
                } else {
                    double a = xr[u] - bgv[u], b = xi[u];
                    f = make_double2(-b * c.sqrtMinusDtIm, a * c.sqrtMinusDtIm);
                    double af = zabs(f);
                    if (af > c.forceCap) f = make_double2(f.x * c.forceCap / af, f.y * c.forceCap / af);
                }
                zd x = make_double2(gs[u] + f.x, f.y);
                Y[(size_t)(2 * w) * G + g] = __double2bfloat16(-c.sqrtMinusDtIm * x.y);
                Y[(size_t)(2 * w + 1) * G + g] = __double2bfloat16(c.sqrtMinusDtIm * x.x);
                zfma(f2, f, f);
                zfma(xf, x, f);
                zfma(xb, x, make_double2(bgv[u], 0.0));
            }
        }
    }
    f2.x = warp_sum(f2.x); f2.y = warp_sum(f2.y);
    xf.x = warp_sum(xf.x); xf.y = warp_sum(xf.y);
    xb.x = warp_sum(xb.x); xb.y = warp_sum(xb.y);
    if (lane == 0) {
        double phase = xf.y;
        double cs = cos(phase);
        if (cs <= 0.0) {
            alive[w] = 0; surv[w] = 0;
        } else {
            zd lw = logw[w];
            lw.x += log(cs);
            zd smp = zsub(zscale(f2, 0.5), xf);
            smp = zsub(smp, make_double2(-c.sqrtMinusDtIm * xb.y, c.sqrtMinusDtIm * xb.x));
            zd t = zadd(smp, lw);
            t.x += dtET;
            logw[w] = zadd(hopLogw, t);
        }
    }
}

// ex += ex2 (the second spin block's exchange plane)
__global__ void add_planes_kernel(long long count, const zd *src, zd *dst)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
         e += (long long)gridDim.x * blockDim.x)
        dst[e] = zadd(dst[e], src[e]);
}

// sum of the xbar partials -> FP64 complex xbar (G x W), for the measurement
__global__ void xbar_combine_kernel(int G, int W, const float *xbarp, int splits,
                                    long long splitStride, zd *xbar)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)G * W;
         e += (long long)gridDim.x * blockDim.x) {
        int g = (int)(e % G), w = (int)(e / G);
        double xr = 0.0, xi = 0.0;
        for (int s = 0; s < splits; ++s) {
            xr += xbarp[s * splitStride + g + (size_t)2 * G * w];
            xi += xbarp[s * splitStride + G + g + (size_t)2 * G * w];
        }
        xbar[e] = make_double2(xr, xi);
    }
}

// ------------------------------------------------------------ Taylor kernel
// One walker at a time per CTA (persistent over walkers).  The walker's
// row i lives in thread i (fp32 accumulators); the current Taylor term is
// the bf16 B operand in shared memory (K-major core matrices), M (bf16
// planes, 128B-swizzled by TMA) the A operand; the complex product uses two
// TMEM accumulators (real / imaginary rows) and the descriptor's A-negate
// bit for -Im(M) Im(term).  After the series converges the one-body
// operator (exp(-dt K) - 1, real) is applied the same way and the walker is
// written back in place.  Rows beyond n (n = 64) are padding.
// Shared memory of the Taylor kernel: M (re, im planes; the one-body
// operator E - I is loaded into the re plane after the series) and the bf16
// operand (re, im planes) holding the current term, K-major with the
// 128-byte swizzle (NC rows of n).  Two CTAs fit on an SM for n = 128, NC <= 32.
template <int NC>
struct TaylorSmem {
    static constexpr size_t m_bytes(int n) { return (size_t)2 * (n / 64) * 16384; }
    static constexpr size_t b_plane(int n) { return (size_t)(n / 64) * NC * 128; }
    static constexpr size_t bytes(int n) { return 1024 + m_bytes(n) + 2 * b_plane(n) + 64; }
};

// element (a, i) of a K-major, 128-byte-swizzled bf16 operand of NC rows
template <int NC>
__device__ __forceinline__ void store_b_sw(uint8_t *sB, int a, int i, float v)
{
    const uint32_t off = (uint32_t)(i >> 6) * (NC * 128) + (uint32_t)a * 128u +
                         (uint32_t)((((i & 63) >> 3) ^ (a & 7)) << 4) + (uint32_t)(i & 7) * 2u;
    *(__nv_bfloat16 *)(sB + off) = __float2bfloat16_rn(v);
}

// Taylor series of exp(M) phi (M = sqrt(-dt) sum_g x_g L_g, bf16 operands,
// fp32 accumulation) for one walker at a time, then the one-body factor:
//   phi' = S + (E - I) S,  S = sum_k M^k phi / k!
// NT = 128 or 256 threads.  Thread t keeps row t % 128 of the running sum S
// in registers for its share of the NC columns (all of them with 128
// threads, one half each with 256: warps w and w + 4 read the same TMEM
// lanes, so the column halves split between them; 256 threads measured
// 9 % slower at 32 columns and is not launched), reads the product
// accumulators back 16 columns at a time and writes its part of each term
// back as the next bf16 operand.  The order stops at k >= checkFrom once
// max |term| <= acc (the dynamicOrder rule of the reference's Taylor
// expansion, CholeskyRealSampleSDOperation / applyToRight with taylor
// accuracy 1e-10) or at kmax.
template <int NC, int NT>
__global__ void __launch_bounds__(NT, NT == 256 ? 2 : 1)
taylor_onebody_kernel(const __grid_constant__ CUtensorMap tmM, const __grid_constant__ CUtensorMap tmE,
                      int W, int n, float *w32, const int *surv, int *order, long long *stats, int kmax,
                      float acc, float relTol, int checkFrom, int doOneBody, int *status, int *err)
{
    static_assert(NT == 128 || NT == 256, "128 or 256 threads");
    constexpr int NG = NT / 128;          // column groups
    constexpr int NCH = NC / NG;          // columns of one thread
    constexpr int NW = NT / 32;           // warps
    static_assert(NCH % 16 == 0, "16-column TMEM reads");
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int KB = n / 64;
    uint8_t *sMr = base;
    uint8_t *sMi = base + KB * 16384;
    uint8_t *sBr = base + 2 * KB * 16384;
    uint8_t *sBi = sBr + (size_t)KB * NC * 128;
    uint64_t *bars = (uint64_t *)(sBi + (size_t)KB * NC * 128);   // [0] M, [1] MMA, [2] E
    uint32_t *tslot = (uint32_t *)(bars + 3);
    __shared__ float red[NW], red0[NW];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int row = tid & 127;
    const int col0 = (tid >> 7) * NCH;    // first column of this thread
    const bool rowOK = row < n;
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init(&bars[2], 1);
        fence_mbar_init();
        tma_prefetch_desc(&tmM);
        tma_prefetch_desc(&tmE);
    }
    if (warp == 0) { tmem_alloc(tslot, 128); tmem_relinquish(); }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tm = *tslot;
    const uint32_t lanebase = (uint32_t)((warp & 3) * 32) << 16;
    const uint32_t tCr = tm, tCi = tm + 64;
    constexpr uint32_t IDESC = idesc_bf16(128, NC);
    constexpr uint32_t IDESCN = idesc_bf16(128, NC, true);
    uint32_t phL = 0, phD = 0;
    bool ok = true;
    uint32_t phE = 0;

    auto issue = [&](const uint8_t *Ar, const uint8_t *Ai) {
        // C_r (+)= Ar Br - Ai Bi ; C_i (+)= Ai Br + Ar Bi  (Ai absent for the real one-body)
        tc_fence_after();
        // descriptors of K step kk = the base descriptor + the step's byte
        // offset / 16 (the start-address field; no carry for shared addresses)
        const uint64_t aR0 = desc_k_sw128(smem_u32(Ar)), bR0 = desc_k_sw128(smem_u32(sBr)),
                       bI0 = desc_k_sw128(smem_u32(sBi)), aI0 = Ai ? desc_k_sw128(smem_u32(Ai)) : 0;
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
            if (kk < n / 16) {
                const uint64_t oa = (uint64_t)(((kk >> 2) * 16384 + (kk & 3) * 32) >> 4);
                const uint64_t ob = (uint64_t)(((kk >> 2) * NC * 128 + (kk & 3) * 32) >> 4);
                umma_bf16(tCr, aR0 + oa, bR0 + ob, IDESC, kk > 0 ? 1u : 0u);
                umma_bf16(tCi, aR0 + oa, bI0 + ob, IDESC, kk > 0 ? 1u : 0u);
                if (Ai) {
                    umma_bf16(tCr, aI0 + oa, bI0 + ob, IDESCN, 1u);
                    umma_bf16(tCi, aI0 + oa, bR0 + ob, IDESC, 1u);
                }
            }
        }
        umma_commit(&bars[1]);
    };
    auto block_max = [&](float v, float *buf) {
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) buf[warp] = v;
    };
    auto read_max = [&](const float *buf) {
        float m = buf[0];
#pragma unroll
        for (int q = 1; q < NW; ++q) m = fmaxf(m, buf[q]);
        return m;
    };

    // Walkers of this CTA: blockIdx.x, +gridDim.x, ... skipping the dead ones.
    auto next_walker = [&](int w) {
        while (w < W && !surv[w]) w += gridDim.x;
        return w;
    };
    // M of the first walker; later walkers' M planes are prefetched while the
    // previous walker finishes (imaginary plane once the series has converged,
    // real plane once the one-body product is done).
    int w = next_walker(blockIdx.x);
    bool mPending = false;
    if (w < W) {
        if (tid == 0) {
            mbar_arrive_expect_tx(&bars[0], (uint32_t)(2 * KB * 16384));
            for (int kb = 0; kb < KB; ++kb) {
                tma_load_2d(sMr + kb * 16384, &tmM, &bars[0], kb * 64, (2 * w) * n);
                tma_load_2d(sMi + kb * 16384, &tmM, &bars[0], kb * 64, (2 * w + 1) * n);
            }
        }
        mPending = true;
    }
    while (w < W) {
        const int wn = next_walker(w + gridDim.x);
        float *gw = w32 + (size_t)w * 2 * n * NC;
        // the next walker's fp32 planes (2 n NC floats, contiguous) are
        // pulled into L2 while this walker's series runs
        if (tid == 0 && wn < W) bulk_prefetch_l2(w32 + (size_t)wn * 2 * n * NC, (uint32_t)(2 * n * NC * sizeof(float)));
        // order 0: S = phi, operand = bf16(phi); all loads issue before the stores
        float pr[NCH], pi[NCH];
#pragma unroll
        for (int a = 0; a < NCH; ++a) {
            pr[a] = rowOK ? gw[row + (size_t)n * (col0 + a)] : 0.f;
            pi[a] = rowOK ? gw[(size_t)n * NC + row + (size_t)n * (col0 + a)] : 0.f;
        }
        float s2 = 0.f;
        if (rowOK) {
#pragma unroll
            for (int a = 0; a < NCH; ++a) {
                store_b_sw<NC>(sBr, col0 + a, row, pr[a]);
                store_b_sw<NC>(sBi, col0 + a, row, pi[a]);
                s2 = fmaxf(s2, pr[a] * pr[a] + pi[a] * pi[a]);
            }
        }
        block_max(s2, red0);
        fence_proxy_async();
        tc_fence_before();
        __syncthreads();
        // terms below fp32 resolution of the walker's largest entry cannot
        // change the fp32 sum: the series stops there (or at acc)
        const float tol = fmaxf(acc, relTol * sqrtf(read_max(red0)));
        ok = __syncthreads_and(mbar_wait(&bars[0], phL)) != 0;
        phL ^= 1;
        mPending = false;
        if (!ok) break;
        int k = 0;
        while (true) {
            ++k;
            if (tid == 0) issue(sMr, sMi);
            ok = __syncthreads_and(mbar_wait(&bars[1], phD)) != 0;
            phD ^= 1;
            if (!ok) break;
            tc_fence_after();
            const float inv = 1.0f / (float)k;
            float mx = 0.f;
            // Accumulator columns come out of TMEM in chunks of up to 32: all
            // loads of a chunk are issued before the one completion wait.
            constexpr int CH = (NCH % 32 == 0) ? 32 : 16;
#pragma unroll
            for (int cb = 0; cb < NCH; cb += CH) {
                uint32_t cr[CH], ci[CH];
#pragma unroll
                for (int c1 = 0; c1 < CH; c1 += 16) {
                    tmem_ld16_nw(tCr + lanebase + col0 + cb + c1, cr + c1);
                    tmem_ld16_nw(tCi + lanebase + col0 + cb + c1, ci + c1);
                }
                tmem_wait_ld();
#pragma unroll
                for (int c1 = 0; c1 < CH; c1 += 16) {
                    const int c0 = cb + c1;
#pragma unroll
                    for (int a = 0; a < 16; ++a) {
                        const float tr = __uint_as_float(cr[c1 + a]) * inv, ti = __uint_as_float(ci[c1 + a]) * inv;
                        pr[c0 + a] += tr;
                        pi[c0 + a] += ti;
                        if (rowOK) {
                            mx = fmaxf(mx, tr * tr + ti * ti);
                            store_b_sw<NC>(sBr, col0 + c0 + a, row, tr);
                            store_b_sw<NC>(sBi, col0 + c0 + a, row, ti);
                        }
                    }
                }
            }
            block_max(mx, red);
            fence_proxy_async();
            tc_fence_before();
            __syncthreads();
            const bool conv = (k >= checkFrom) && (sqrtf(read_max(red)) <= tol);
            if (conv || k >= kmax) {
                if (!conv && tid == 0 && status) atomicOr(status + w, (int)ST_TAYLOR_CAP);
                break;
            }
            // red[] is next written after the following order's
            // __syncthreads_and, which every thread reaches after reading it
        }
        if (!ok) break;
        // Every MMA of the series has completed: the M planes are free.
        if (wn < W) {
            if (tid == 0) {
                mbar_arrive_expect_tx(&bars[0], (uint32_t)(2 * KB * 16384));
                for (int kb = 0; kb < KB; ++kb)
                    tma_load_2d(sMi + kb * 16384, &tmM, &bars[0], kb * 64, (2 * wn + 1) * n);
                if (!doOneBody)
                    for (int kb = 0; kb < KB; ++kb)
                        tma_load_2d(sMr + kb * 16384, &tmM, &bars[0], kb * 64, (2 * wn) * n);
            }
            mPending = true;
        }
        if (doOneBody) {
            // E - I into the real M plane, operand = bf16(S)
            if (tid == 0) {
                mbar_arrive_expect_tx(&bars[2], (uint32_t)(KB * 16384));
                for (int kb = 0; kb < KB; ++kb) tma_load_2d(sMr + kb * 16384, &tmE, &bars[2], kb * 64, 0);
            }
            if (rowOK) {
#pragma unroll
                for (int a = 0; a < NCH; ++a) {
                    store_b_sw<NC>(sBr, col0 + a, row, pr[a]);
                    store_b_sw<NC>(sBi, col0 + a, row, pi[a]);
                }
            }
            fence_proxy_async();
            tc_fence_before();
            __syncthreads();
            ok = __syncthreads_and(mbar_wait(&bars[2], phE)) != 0;
            phE ^= 1;
            if (!ok) break;
            if (tid == 0) issue(sMr, nullptr);
            ok = __syncthreads_and(mbar_wait(&bars[1], phD)) != 0;
            phD ^= 1;
            if (!ok) break;
            tc_fence_after();
            // the one-body product has read E: the real plane of the next M may land
            if (wn < W && tid == 0)
                for (int kb = 0; kb < KB; ++kb)
                    tma_load_2d(sMr + kb * 16384, &tmM, &bars[0], kb * 64, (2 * wn) * n);
#pragma unroll
            for (int c0 = 0; c0 < NCH; c0 += 16) {
                uint32_t vr[16], vi[16];
                tmem_ld16_nw(tCr + lanebase + col0 + c0, vr);
                tmem_ld16_nw(tCi + lanebase + col0 + c0, vi);
                tmem_wait_ld();
#pragma unroll
                for (int a = 0; a < 16; ++a) { pr[c0 + a] += __uint_as_float(vr[a]); pi[c0 + a] += __uint_as_float(vi[a]); }
            }
        }
        if (rowOK) {
#pragma unroll
            for (int a = 0; a < NCH; ++a) {
                gw[row + (size_t)n * (col0 + a)] = pr[a];
                gw[(size_t)n * NC + row + (size_t)n * (col0 + a)] = pi[a];
            }
        }
        if (tid == 0) {
            order[w] = k;
            // order statistics: calls, total order, min, max (integer
            // atomics, so the result does not depend on the walker order)
            if (stats) {
                atomicAdd((unsigned long long *)&stats[0], 1ULL);
                atomicAdd((unsigned long long *)&stats[1], (unsigned long long)k);
                atomicMin(&stats[2], (long long)k);
                atomicMax(&stats[3], (long long)k);
            }
        }
        tc_fence_before();
        __syncthreads();
        w = wn;
    }
    // An abandoned prefetch still lands in this CTA's shared memory: wait
    // (bounded) for it before the CTA exits.
    if (!ok && mPending) (void)mbar_wait(&bars[0], phL);
    if (!ok && err) atomicExch(err, 2);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tm, 128);
}

template <int NC>
int launch_taylor(afqmc_engine *e, const CUtensorMap &mM, const CUtensorMap &mE, int doOneBody)
{
    const size_t smem = TaylorSmem<NC>::bytes(e->n);
    static std::atomic<unsigned long long> attr{0};
    if (first_on_device(attr)) {
        cudaFuncSetAttribute(taylor_onebody_kernel<NC, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)TaylorSmem<NC>::bytes(128));
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int perSm = TaylorSmem<NC>::bytes(e->n) <= 112 * 1024 ? 2 : 1;
    int grid = std::min(e->W, perSm * sms);
    taylor_onebody_kernel<NC, 128><<<grid, 128, smem, e->stream>>>(
        mM, mE, e->W, e->n, e->mx->wf32, e->surv, e->order, e->tstats, 30, 1e-10f, 5.9604645e-8f, 4, doOneBody,
        e->status, e->mx->err);
    return engine_check_launch();
}

// Taylor kernel with M in tensor memory (NC = 16 or 32 columns).
//
// The A operand of every order's product is the walker's M, the same for all
// orders; held in shared memory it is re-read by each MMA (4 KB per K step
// and MMA against 1 KB of the term), and at N = 32 those operand reads, not
// the multiply, set the MMA rate.  Here M's two bf16 planes live in tensor
// memory (row i in lane i, 128 columns), loaded once per walker by the
// threads with tcgen05.st, and each K step is two MMAs with A read from
// tensor memory and one B window of N = 2 NC rows from shared memory (the
// term's real rows, then its imaginary rows):
//   D1 = Re(M) [Re t; Im t],  D2 = Im(M) [Re t; Im t]
//   Re(M t) = D1[re] - D2[im],  Im(M t) = D1[im] + D2[re].
// The one-body operator E - I stays resident in shared memory for the
// kernel's life.  M reaches tensor memory one plane at a time through a
// shared-memory staging buffer: a TMA load of the plane (128-byte swizzle),
// then tcgen05.cp of each K step's 128 x 16 slab, all issued by one thread
// and asynchronous to the others.  The next walker's real plane is loaded
// while the current series runs and copied in once the series has finished
// reading M; its imaginary plane is loaded during the one-body product and
// copied in ahead of the next walker's first MMA.
// Tensor memory per CTA: M 128 columns, D1 and D2 2 NC each (256 allocated),
// and shared memory (E, the term, the staging buffer; 81 KB at n = 128)
// keeps at most two CTAs on an SM, so the allocation never waits.
template <int NC>
struct TaylorTsSmem {
    static constexpr size_t e_bytes(int n) { return (size_t)(n / 64) * 16384; }
    static constexpr size_t b_bytes(int n) { return (size_t)(n / 64) * 2 * NC * 128; }
    static constexpr size_t bytes(int n)
    {
        return std::max((size_t)80 * 1024, (size_t)1024 + 2 * e_bytes(n) + b_bytes(n) + 64);
    }
};

// Fragment access of a 16-lane slab of tensor memory (tcgen05.ld .16x256b):
// with G column groups of 8, register 4m + q of thread t holds lane
// (base + t/4 + 8 (q >> 1)), column 8m + 2 (t % 4) + (q & 1) -- the layout
// stmatrix takes, so a term goes from tensor memory to the next MMA's B
// operand as bf16 pairs and one transposing stmatrix per four 8x8 tiles.
template <int G>
__device__ __forceinline__ void tmem_ld_frag(uint32_t taddr, uint32_t *r);
template <>
__device__ __forceinline__ void tmem_ld_frag<2>(uint32_t taddr, uint32_t *r)
{
    asm volatile("tcgen05.ld.sync.aligned.16x256b.x2.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr)
                 : "memory");
}
template <>
__device__ __forceinline__ void tmem_ld_frag<4>(uint32_t taddr, uint32_t *r)
{
    asm volatile(
        "tcgen05.ld.sync.aligned.16x256b.x4.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}
template <>
__device__ __forceinline__ void tmem_ld_frag<8>(uint32_t taddr, uint32_t *r)
{
    asm volatile(
        "tcgen05.ld.sync.aligned.16x256b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
          "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
          "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
}
// four 8x8 b16 tiles, each stored transposed: lane 8j + c gives the address
// of stored row c of tile j, which receives column c of the thread fragment
__device__ __forceinline__ void stmatrix_x4_trans(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
    asm volatile("stmatrix.sync.aligned.m8n8.x4.trans.shared.b16 [%0], {%1,%2,%3,%4};" ::"r"(addr), "r"(a), "r"(b),
                 "r"(c), "r"(d)
                 : "memory");
}
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi)
{
    __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&p);
}

template <int NC, int NN>
__global__ void __launch_bounds__(128, 2)
taylor_ts_kernel(const __grid_constant__ CUtensorMap tmM, const __grid_constant__ CUtensorMap tmE, int W,
                 float *w32,
                 const int *surv, int *order, long long *stats, int kmax, float acc, float relTol,
                 int checkFrom, int *status, int *err)
{
    constexpr int n = NN;        // walker rows: 64 or 128 (all addressing compile-time)
    constexpr int NB = 2 * NC;   // MMA N: the term's real rows, then its imaginary rows
    constexpr int G = NC / 8;    // 8-column groups of the real (or imaginary) part
    constexpr int NE = 8 * G;    // complex elements of a thread: 2 slabs x G groups x 4
    static_assert(G == 2 || G == 4, "16 or 32 columns");
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    constexpr int KB = n / 64;
    uint8_t *sE = base;
    uint8_t *sB = base + KB * 16384;
    uint8_t *sS = sB + (size_t)KB * NB * 128;                      // M plane staging
    uint64_t *bars = (uint64_t *)(sS + (size_t)KB * 16384);   // [0] E, [1] MMA, [2] staged, [3] copied
    uint32_t *tslot = (uint32_t *)(bars + 4);
    __shared__ float red[4], red0[4];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // Rows: warp w owns rows 32w..32w+31 (its lane quarter of tensor memory),
    // as two 16-row slabs h; within slab h thread t holds rows
    // 32w + 16h + t/4 (+8) and columns 8m + 2 (t % 4) (+1) of each group m.
    const bool warpOK = 32 * warp < n;   // n = 64 or 128: rows of the warp exist
    const int r0 = 32 * warp + (lane >> 2), c0 = 2 * (lane & 3);
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init(&bars[2], 1);
        mbar_init(&bars[3], 1);
        fence_mbar_init();
        tma_prefetch_desc(&tmE);
        tma_prefetch_desc(&tmM);
    }
    if (warp == 0) { tmem_alloc(tslot, 256); tmem_relinquish(); }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tm = *tslot;
    const uint32_t tMr = tm, tMi = tm + 64, tD1 = tm + 128, tD2 = tm + 128 + NB;
    constexpr uint32_t IDESC = idesc_bf16(128, NB);
    const uint64_t bB0 = desc_k_sw128(smem_u32(sB));   // K step kk: + its byte offset / 16
    // stmatrix addresses of this lane for slabs 0 and 1 (real rows; the
    // imaginary rows are NC B rows further): one stmatrix covers two column
    // groups of the slab, tile j = lane / 8 = (group 2p + j / 2, slab rows
    // 8 (j % 2) .. +7), stored row c = lane % 8 = B row 16p + 8 (j / 2) + c,
    // holding the K chunk of those 8 rows (128-byte swizzle: chunk ^ (row & 7))
    uint32_t stAddr[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int j = lane >> 3, c = lane & 7;
        const int brow = 8 * (j >> 1) + c;
        const int i0 = 32 * warp + 16 * h + 8 * (j & 1);
        stAddr[h] = smem_u32(sB) + (uint32_t)((i0 >> 6) * NB * 128 + brow * 128 + ((((i0 & 63) >> 3) ^ c) << 4));
    }
    if (tid == 0) {
        mbar_arrive_expect_tx(&bars[0], (uint32_t)(KB * 16384));
        for (int kb = 0; kb < KB; ++kb) tma_load_2d(sE + kb * 16384, &tmE, &bars[0], kb * 64, 0);
    }
    uint32_t phD = 0;
    bool ok = true, eReady = false;

    auto block_max = [&](float v, float *buf) {
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) buf[warp] = v;
    };
    auto read_max = [&](const float *buf) { return fmaxf(fmaxf(buf[0], buf[1]), fmaxf(buf[2], buf[3])); };
    auto next_walker = [&](int w) {
        while (w < W && !surv[w]) w += gridDim.x;
        return w;
    };
    // element e = 4 G h + 4 m + q of this thread: row and column
    auto erow = [&](int e) { return r0 + 16 * (e / (4 * G)) + 8 * ((e & 3) >> 1); };
    auto ecol = [&](int e) { return 8 * ((e / 4) % G) + c0 + (e & 1); };
    // B operand rows of slab h from 4 G values of the slab (one part: real
    // rows at B row 0, imaginary rows at B row NC)
    auto stage_part = [&](int h, int part, const float *v) {
        const uint32_t a0 = stAddr[h] + (uint32_t)(part * NC * 128);
#pragma unroll
        for (int p = 0; p < G / 2; ++p)
            stmatrix_x4_trans(a0 + (uint32_t)(p * 2048), pack_bf16x2(v[8 * p], v[8 * p + 1]),
                              pack_bf16x2(v[8 * p + 2], v[8 * p + 3]), pack_bf16x2(v[8 * p + 4], v[8 * p + 5]),
                              pack_bf16x2(v[8 * p + 6], v[8 * p + 7]));
    };
    auto stage = [&](const float *vr, const float *vi) {
        if (!warpOK) return;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            stage_part(h, 0, vr + 4 * G * h);
            stage_part(h, 1, vi + 4 * G * h);
        }
    };
    // The M staging pipeline (thread 0 only): plane p of walker w into the
    // staging buffer by TMA, the staged plane into tensor memory by
    // tcgen05.cp (ordered before the MMAs this thread issues later), and the
    // wait for the copy to finish reading the buffer.  A failed wait clears
    // ok0, which the next block-wide check reads.
    // thread 0's pipeline state, kept in shared memory (no registers for the
    // other 127 threads): parities of bars[2] and bars[3], loads / copies in
    // flight, and whether every wait so far succeeded
    __shared__ uint32_t pipe[5];   // phS, phC, pendS, pendC, ok0
    if (tid == 0) { pipe[0] = 0; pipe[1] = 0; pipe[2] = 0; pipe[3] = 0; pipe[4] = 1; }
    auto stage_plane = [&](int w, int p) {
        mbar_arrive_expect_tx(&bars[2], (uint32_t)(KB * 16384));
        for (int kb = 0; kb < KB; ++kb) tma_load_2d(sS + kb * 16384, &tmM, &bars[2], kb * 64, (2 * w + p) * n);
        pipe[2] = 1;
    };
    auto copy_plane = [&](uint32_t tDst) {
        if (!mbar_wait(&bars[2], pipe[0])) pipe[4] = 0;
        pipe[0] ^= 1;
        pipe[2] = 0;
        tc_fence_after();
        const uint64_t sS0 = desc_k_sw128(smem_u32(sS));
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
            if (kk < n / 16) {
                const uint64_t sd = sS0 + (uint64_t)(((kk >> 2) * 16384 + (kk & 3) * 32) >> 4);
                asm volatile("tcgen05.cp.cta_group::1.128x256b [%0], %1;" ::"r"(tDst + kk * 8), "l"(sd) : "memory");
            }
        }
        umma_commit(&bars[3]);
        pipe[3] = 1;
    };
    auto staging_free = [&]() {
        if (!mbar_wait(&bars[3], pipe[1])) pipe[4] = 0;
        pipe[1] ^= 1;
        pipe[3] = 0;
    };

    int w = next_walker(blockIdx.x);
    if (tid == 0 && w < W) {
        stage_plane(w, 0);
        copy_plane(tMr);
        staging_free();
        stage_plane(w, 1);
    }
    while (w < W) {
        const int wn = next_walker(w + gridDim.x);
        float *gw = w32 + (size_t)w * 2 * n * NC;
        if (tid == 0 && wn < W) {
            bulk_prefetch_l2(w32 + (size_t)wn * 2 * n * NC, (uint32_t)(2 * n * NC * sizeof(float)));
        }
        // order 0: S = phi, operand = bf16(phi)
        float pr[NE], pi[NE];
        float s2 = 0.f;
#pragma unroll
        for (int e = 0; e < NE; ++e) {
            const size_t off = (size_t)erow(e) + (size_t)n * ecol(e);
            pr[e] = warpOK ? gw[off] : 0.f;
            pi[e] = warpOK ? gw[(size_t)n * NC + off] : 0.f;
            s2 = fmaxf(s2, pr[e] * pr[e] + pi[e] * pi[e]);
        }
        stage(pr, pi);
        block_max(s2, red0);
        fence_proxy_async();
        tc_fence_before();
        __syncthreads();
        const float tol = fmaxf(acc, relTol * sqrtf(read_max(red0)));
        if (!eReady) {
            ok = __syncthreads_and(mbar_wait(&bars[0], 0)) != 0;
            eReady = ok;
            if (!ok) break;
        }
        int k = 0;
        while (true) {
            ++k;
            if (tid == 0) {
                if (k == 1) copy_plane(tMi);   // this walker's imaginary plane, staged meanwhile
                tc_fence_after();
#pragma unroll
                for (int kk = 0; kk < 8; ++kk) {
                    if (kk < n / 16) {
                        const uint64_t bd = bB0 + (uint64_t)(((kk >> 2) * NB * 128 + (kk & 3) * 32) >> 4);
                        umma_bf16_ts(tD1, tMr + kk * 8, bd, IDESC, kk > 0 ? 1u : 0u);
                        umma_bf16_ts(tD2, tMi + kk * 8, bd, IDESC, kk > 0 ? 1u : 0u);
                    }
                }
                umma_commit(&bars[1]);
                if (k == 1) {
                    // the next walker's real plane goes into the freed staging buffer
                    staging_free();
                    if (wn < W) stage_plane(wn, 0);
                }
            }
            ok = __syncthreads_and(mbar_wait(&bars[1], phD) && (tid != 0 || pipe[4])) != 0;
            phD ^= 1;
            if (!ok) break;
            tc_fence_after();
            const float inv = 1.0f / (float)k;
            float mx = 0.f;
            if (warpOK) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    // D1 = Re M [Re t; Im t], D2 = Im M [Re t; Im t] over this slab:
                    // Re t' = (D1 re - D2 im) / k first, then Im t' = (D1 im + D2 re) / k
                    const uint32_t lo = (uint32_t)(32 * warp + 16 * h) << 16;
                    float tr[4 * G];
                    {
                        uint32_t a[4 * G], b[4 * G];
                        tmem_ld_frag<G>(tD1 + lo, a);
                        tmem_ld_frag<G>(tD2 + lo + NC, b);
                        tmem_wait_ld();
#pragma unroll
                        for (int x = 0; x < 4 * G; ++x) {
                            tr[x] = (__uint_as_float(a[x]) - __uint_as_float(b[x])) * inv;
                            pr[4 * G * h + x] += tr[x];
                        }
                    }
                    stage_part(h, 0, tr);
                    float ti[4 * G];
                    {
                        uint32_t a[4 * G], b[4 * G];
                        tmem_ld_frag<G>(tD1 + lo + NC, a);
                        tmem_ld_frag<G>(tD2 + lo, b);
                        tmem_wait_ld();
#pragma unroll
                        for (int x = 0; x < 4 * G; ++x) {
                            ti[x] = (__uint_as_float(a[x]) + __uint_as_float(b[x])) * inv;
                            pi[4 * G * h + x] += ti[x];
                            mx = fmaxf(mx, fmaf(tr[x], tr[x], ti[x] * ti[x]));
                        }
                    }
                    stage_part(h, 1, ti);
                }
            }
            block_max(mx, red);
            fence_proxy_async();
            tc_fence_before();
            __syncthreads();
            const bool conv = (k >= checkFrom) && (sqrtf(read_max(red)) <= tol);
            if (conv || k >= kmax) {
                if (!conv && tid == 0 && status) atomicOr(status + w, (int)ST_TAYLOR_CAP);
                break;
            }
        }
        if (!ok) break;
        // one-body: phi' = S + (E - I) S, the operand = bf16(S)
        stage(pr, pi);
        fence_proxy_async();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint64_t bE0 = desc_k_sw128(smem_u32(sE));
#pragma unroll
            for (int kk = 0; kk < 8; ++kk) {
                if (kk < n / 16) {
                    const uint64_t oe = (uint64_t)(((kk >> 2) * 16384 + (kk & 3) * 32) >> 4);
                    const uint64_t ob = (uint64_t)(((kk >> 2) * NB * 128 + (kk & 3) * 32) >> 4);
                    umma_bf16(tD1, bE0 + oe, bB0 + ob, IDESC, kk > 0 ? 1u : 0u);
                }
            }
            umma_commit(&bars[1]);
            // the series has finished reading M: the next walker's real plane goes in
            if (wn < W) copy_plane(tMr);
        }
        ok = __syncthreads_and(mbar_wait(&bars[1], phD) && (tid != 0 || pipe[4])) != 0;
        phD ^= 1;
        if (!ok) break;
        tc_fence_after();
        if (warpOK) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint32_t a[4 * G], b[4 * G];
                const uint32_t lo = (uint32_t)(32 * warp + 16 * h) << 16;
                tmem_ld_frag<G>(tD1 + lo, a);
                tmem_ld_frag<G>(tD1 + lo + NC, b);
                tmem_wait_ld();
#pragma unroll
                for (int x = 0; x < 4 * G; ++x) {
                    pr[4 * G * h + x] += __uint_as_float(a[x]);
                    pi[4 * G * h + x] += __uint_as_float(b[x]);
                }
            }
#pragma unroll
            for (int e = 0; e < NE; ++e) {
                const size_t off = (size_t)erow(e) + (size_t)n * ecol(e);
                gw[off] = pr[e];
                gw[(size_t)n * NC + off] = pi[e];
            }
        }
        if (tid == 0) {
            if (wn < W) {
                // the next walker's imaginary plane, copied in before its first MMA
                staging_free();
                stage_plane(wn, 1);
            }
            order[w] = k;
            if (stats) {
                atomicAdd((unsigned long long *)&stats[0], 1ULL);
                atomicAdd((unsigned long long *)&stats[1], (unsigned long long)k);
                atomicMin(&stats[2], (long long)k);
                atomicMax(&stats[3], (long long)k);
            }
        }
        tc_fence_before();
        __syncthreads();
        w = wn;
    }
    // a failed wait: let the loads and copies this CTA issued finish before it exits
    if (!ok && !eReady) (void)mbar_wait(&bars[0], 0);
    if (tid == 0) {
        if (pipe[2]) (void)mbar_wait(&bars[2], pipe[0]);
        if (pipe[3]) (void)mbar_wait(&bars[3], pipe[1]);
    }
    if (!ok && err) atomicExch(err, 2);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tm, 256);
}

template <int NC>
int launch_taylor_ts(afqmc_engine *e, const CUtensorMap &mM, const CUtensorMap &mE)
{
    const size_t smem = TaylorTsSmem<NC>::bytes(e->n);
    static std::atomic<unsigned long long> attr{0};
    if (first_on_device(attr)) {
        cudaFuncSetAttribute(taylor_ts_kernel<NC, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)TaylorTsSmem<NC>::bytes(128));
        cudaFuncSetAttribute(taylor_ts_kernel<NC, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)TaylorTsSmem<NC>::bytes(64));
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = std::min(e->W, 2 * sms);
    auto kern = e->n == 128 ? taylor_ts_kernel<NC, 128> : taylor_ts_kernel<NC, 64>;
    kern<<<grid, 128, smem, e->stream>>>(
        mM, mE, e->W, e->mx->wf32, e->surv, e->order, e->tstats, 30, 1e-10f, 5.9604645e-8f, 4,
        e->status, e->mx->err);
    return engine_check_launch();
}

int run_taylor(afqmc_engine *e)
{
    MixedState *m = e->mx;
    CUtensorMap mM, mE;
    int r = tc_make_map_bf16(&mM, m->Mbuf, e->n, (long long)2 * e->W * e->n, e->n, 128);
    if (r) return engine_fail(AFQMC_ERR_CUDA, "tensor map (M): " + std::to_string(r));
    r = tc_make_map_bf16(&mE, m->Et, e->n, e->n, e->n, 128);
    if (r) return engine_fail(AFQMC_ERR_CUDA, "tensor map (E): " + std::to_string(r));
    switch (e->ncol) {
    case 16: return launch_taylor_ts<16>(e, mM, mE);
    case 32: return launch_taylor_ts<32>(e, mM, mE);
    case 48: return launch_taylor<48>(e, mM, mE, 1);
    case 64: return launch_taylor<64>(e, mM, mE, 1);
    default: return engine_fail(AFQMC_ERR_UNSUPPORTED, "mixed Taylor kernel needs 16, 32, 48 or 64 columns");
    }
}

int tc(afqmc_engine *e, TcGemmArgs a)
{
    a.err = e->mx->err;
    int r = tc_gemm_bf16(a, e->stream);
    if (r) return engine_fail(AFQMC_ERR_CUDA, "tcgen05 gemm: " + std::to_string(r));
    return AFQMC_OK;
}

// the spin blocks the mixed form computes (block 0 alone when restricted)
const Blocks &mbl(const afqmc_engine *e) { return e->mx->restricted ? e->mx->bl1 : e->bl; }

// S_b = phiT_b^H phi_b from the fp32 walkers (compensated tf32 tensor-core
// product, FP64 result); every walker's slot is written
int overlap32(afqmc_engine *e, const float *w32, const int *mask)
{
    (void)mask;
    MixedState *m = e->mx;
    const Blocks &bl = mbl(e);
    int nb = 0, Ns[2];
    long long sOff[2];
    for (int b = 0; b < bl.nblk; ++b)
        if (bl.Ns[b] > 0) { Ns[nb] = bl.Ns[b]; sOff[nb] = bl.sOff[b]; ++nb; }
    if (nb == 0) return AFQMC_OK;
    if (m->ovStacked) {
        const int r = overlap_tc_launch(e->stream, e->n, e->ncol, nb, Ns, e->W, m->Ohi[0], m->Olo[0], w32, e->S,
                                        e->bl.sStride, sOff, m->err);
        if (r) return engine_fail(AFQMC_ERR_CUDA, "overlap launch: " + std::to_string(r));
        return AFQMC_OK;
    }
    for (int b = 0; b < nb; ++b) {
        const int r = overlap_tc_launch(e->stream, e->n, e->ncol, 1, Ns + b, e->W, m->Ohi[b], m->Olo[b], w32,
                                        e->S, e->bl.sStride, sOff + b, m->err);
        if (r) return engine_fail(AFQMC_ERR_CUDA, "overlap launch: " + std::to_string(r));
    }
    return AFQMC_OK;
}

// theta_b = phi_b S_b^{-1} (n x Ns) -> bf16 planar Theta (+ FP64 copy when
// thetaZ): compensated tcgen05 tf32 product, so that the bf16 Theta rounds
// from a value good to about 22 bits
int theta32(afqmc_engine *e, const float *w32, const int *mask, zd *thetaZ)
{
    MixedState *m = e->mx;
    const Blocks &bl = mbl(e);
    int nb = 0, Ns[2];
    long long sOff[2], tOff[2];
    for (int b = 0; b < bl.nblk; ++b)
        if (bl.Ns[b] > 0) { Ns[nb] = bl.Ns[b]; sOff[nb] = bl.sOff[b]; tOff[nb] = bl.tOff[b]; ++nb; }
    if (nb == 0) return AFQMC_OK;
    const long long s32 = sinv32_stride(bl);
    // both blocks in one pass when they fit, else one pass per block
    const int groups = theta_tc_supported(e->n, nb, Ns, s32) ? 1 : nb;
    for (int gi = 0; gi < groups; ++gi) {
        const int nbg = groups == 1 ? nb : 1;
        const int r = theta_tc_launch(e->stream, e->n, e->ncol, nbg, Ns + gi, e->W, w32, m->Sinv32, s32,
                                      sOff + gi, mask, m->Theta, 2 * e->Ktot, e->Ktot, tOff + gi, thetaZ,
                                      e->bl.tStride, m->err);
        if (r) return engine_fail(AFQMC_ERR_CUDA, "theta launch: " + std::to_string(r));
    }
    return AFQMC_OK;
}

int force_tc(afqmc_engine *e)
{
    MixedState *m = e->mx;
    TcGemmArgs a;
    if (m->realA) {
        // real A_g: xbar_re = A theta_re, xbar_im = A theta_im as one real
        // product over the theta planes (column 2w + p = plane p of walker w),
        // which lands in the same layout as the complex form
        // (restricted: block 0's columns only, doubled exactly by alpha)
        a.M = e->G; a.N = 2 * e->W; a.K = (int)(m->restricted ? e->bl.tOff[1] : e->Ktot);
        a.A = m->Abig; a.lda = 2 * e->Ktot;
        a.B = m->Theta; a.ldb = e->Ktot;
        a.C = m->xbarp; a.ldc = e->G;
        a.alpha = m->restricted ? 2.0f : 1.0f;
    } else {
        a.M = 2 * e->G; a.N = e->W; a.K = (int)(2 * e->Ktot);
        a.A = m->Abig; a.lda = 2 * e->Ktot;
        a.B = m->Theta; a.ldb = 2 * e->Ktot;
        a.C = m->xbarp; a.ldc = 2 * e->G;
    }
    a.outType = TC_OUT_F32;
    a.splits = m->splits; a.splitStride = (long long)2 * e->G * e->W;
    return tc(e, a);
}

int check_err(afqmc_engine *e)
{
    (void)e;
    return engine_check_launch();
}

}  // namespace

// flag = 1 when any element of A has a nonzero imaginary part
__global__ void any_imag_kernel(long long count, const zd *A, int *flag)
{
    bool any = false;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count; e += (long long)gridDim.x * blockDim.x)
        any = any || A[e].y != 0.0;
    if (__syncthreads_or(any) && threadIdx.x == 0) atomicOr(flag, 1);
}

int mixed_create(afqmc_engine *e)
{
    if (e->kind == KIND_CP) return cp_mixed_create(e);
    if (e->n != 64 && e->n != 128) return engine_fail(AFQMC_ERR_UNSUPPORTED, "mixed precision form needs n = 64 or 128");
    if (e->ncol % 16 != 0 || e->ncol > 64) return engine_fail(AFQMC_ERR_UNSUPPORTED, "mixed precision form needs 16..64 columns in steps of 16");
    if (e->G % 64 != 0) return engine_fail(AFQMC_ERR_UNSUPPORTED, "mixed precision form needs G a multiple of 64");
    if (e->useLog || !e->expK[0]) return engine_fail(AFQMC_ERR_UNSUPPORTED, "mixed precision form needs the dense exp(-dt K) operator");
    MixedState *m = new MixedState();
    e->mx = m;
    const int W = e->W, n = e->n, G = e->G;
    m->ws32 = (long long)2 * n * e->ncol;
    const long long Ktot = e->Ktot;
    m->splits = (2 * Ktot) % (64 * 4) == 0 ? 4 : 1;
    MTRY(engine_dalloc(e, &m->wf32, (size_t)W * m->ws32));
    MTRY(engine_dalloc(e, &m->tmp32, (size_t)W * m->ws32));
    MTRY(engine_dalloc(e, (unsigned short **)&m->Theta, (size_t)W * 2 * Ktot));
    MTRY(engine_dalloc(e, (unsigned short **)&m->Abig, (size_t)2 * G * 2 * Ktot));
    MTRY(engine_dalloc(e, (unsigned short **)&m->Y, (size_t)2 * W * G));
    MTRY(engine_dalloc(e, (unsigned short **)&m->Lt, (size_t)n * n * G));
    MTRY(engine_dalloc(e, (unsigned short **)&m->Mbuf, (size_t)2 * W * n * n));
    MTRY(engine_dalloc(e, (unsigned short **)&m->Et, (size_t)n * n));
    MTRY(engine_dalloc(e, &m->xbarp, (size_t)m->splits * 2 * G * W));
    MTRY(engine_dalloc(e, &m->wfDaggerTm, (size_t)Ktot));
    MTRY(engine_dalloc(e, &m->err, 1));
    MTRY(engine_dalloc(e, &m->ex2, (size_t)G * W));
    for (int b = 0; b < e->bl.nblk; ++b) {
        const int Ns = e->bl.Ns[b];
        if (Ns == 0 || !(exchange_tc_supported(n, Ns) || exchange_gemm_supported(n, Ns, W, G))) continue;
        MTRY(engine_dalloc(e, (unsigned short **)&m->A2r[b], (size_t)G * Ns * n));
        MTRY(engine_dalloc(e, (unsigned short **)&m->A2i[b], (size_t)G * Ns * n));
        build_a2_kernel<<<1184, 256, 0, e->stream>>>(G, Ns, n, Ktot, e->bl.tOff[b], e->Aall, m->A2r[b],
                                                     m->A2i[b]);
    }
    {
        // exact test on the FP64 half-rotated vectors
        MTRY(cuda_check(cudaMemsetAsync(m->err, 0, sizeof(int), e->stream), "memset"));
        any_imag_kernel<<<592, 256, 0, e->stream>>>((long long)G * Ktot, e->Aall, m->err);
        int h = 1;
        MTRY(cuda_check(cudaMemcpyAsync(&h, m->err, sizeof(int), cudaMemcpyDeviceToHost, e->stream), "copy"));
        MTRY(cuda_check(cudaStreamSynchronize(e->stream), "sync"));
        MTRY(cuda_check(cudaMemsetAsync(m->err, 0, sizeof(int), e->stream), "memset"));
        m->realA = (h == 0);
    }
    // with real A the exchange runs as dense GEMMs over K = Ns n
    if (m->realA) {
        bool ok = true;
        long long Kmax = 0;
        for (int b = 0; b < e->bl.nblk; ++b) {
            if (e->bl.Ns[b] == 0) continue;
            ok = ok && exchange_gemm_supported(n, e->bl.Ns[b], W, G);
            Kmax = std::max(Kmax, (long long)n * e->bl.Ns[b]);
        }
        if (ok && Kmax > 0) {
            // spin-restricted when both blocks carry the same trial bit for bit
            if (e->bl.nblk == 2 && e->nup == e->ndn && e->nup > 0) {
                std::vector<zd> t0((size_t)n * e->nup), t1((size_t)n * e->ndn);
                MTRY(cuda_check(cudaMemcpy(t0.data(), e->phiT[0], sizeof(zd) * t0.size(), cudaMemcpyDeviceToHost),
                                "copy"));
                MTRY(cuda_check(cudaMemcpy(t1.data(), e->phiT[1], sizeof(zd) * t1.size(), cudaMemcpyDeviceToHost),
                                "copy"));
                if (std::memcmp(t0.data(), t1.data(), sizeof(zd) * t0.size()) == 0) {
                    m->restricted = true;
                    m->bl1 = e->bl;
                    m->bl1.nblk = 1;
                    m->bl1.Ns[1] = 0;
                    m->bl1.mult = 2;
                }
            }
            for (int b = 0; b < (m->restricted ? 1 : e->bl.nblk); ++b)
                if (e->bl.Ns[b] > 0) MTRY(exchange_gemm_build(e, b, m->exg[b]));
            MTRY(exchange_gemm_alloc(e, Kmax, m->exs));
            MTRY(engine_dalloc(e, &m->exTot, (size_t)W));
            m->exGemm = true;
        }
    }
    build_abig_kernel<<<1184, 256, 0, e->stream>>>(G, Ktot, n, e->bl, e->Aall, m->Abig);
    build_lt_kernel<<<1184, 256, 0, e->stream>>>((long long)n * n, G, e->chol, m->Lt);
    build_et_kernel<<<64, 256, 0, e->stream>>>(n, e->expK[0], m->Et);
    permute_wdt_kernel<<<64, 256, 0, e->stream>>>(n, e->bl, e->wfDaggerT, m->wfDaggerTm);
    MTRY(engine_check_launch());
    // the dense one-body operator must be real for the bf16 one-body path
    std::vector<zd> h((size_t)n * n);
    MTRY(cuda_check(cudaMemcpyAsync(h.data(), e->expK[0], sizeof(zd) * n * n, cudaMemcpyDeviceToHost, e->stream), "copy"));
    MTRY(cuda_check(cudaStreamSynchronize(e->stream), "sync"));
    for (const zd &v : h)
        if (v.y != 0.0) return engine_fail(AFQMC_ERR_UNSUPPORTED, "mixed precision one-body needs a real exp(-dt K)");
    // exp(+dt/2 K) of the measurement's half step on the tensor cores
    {
        std::vector<zd> E1((size_t)n * n);
        MTRY(cuda_check(cudaMemcpy(E1.data(), e->expK[1], sizeof(zd) * E1.size(), cudaMemcpyDeviceToHost), "copy"));
        std::vector<float> eh, el;
        if (tf32_split_operator(E1.data(), n, eh, el))
            return engine_fail(AFQMC_ERR_UNSUPPORTED, "mixed precision one-body needs a real exp(dt/2 K)");
        MTRY(engine_dalloc(e, &m->E1h, eh.size()));
        MTRY(engine_dalloc(e, &m->E1l, el.size()));
        MTRY(cuda_check(cudaMemcpy(m->E1h, eh.data(), 4 * eh.size(), cudaMemcpyHostToDevice), "upload"));
        MTRY(cuda_check(cudaMemcpy(m->E1l, el.data(), 4 * el.size(), cudaMemcpyHostToDevice), "upload"));
        MTRY(engine_dalloc(e, &m->sh, (size_t)W * m->ws32));
        MTRY(engine_dalloc(e, &m->sl, (size_t)W * m->ws32));
    }
    // S^{-1} of the theta product, fp32 planes written by the LU
    MTRY(engine_dalloc(e, &m->Sinv32, (size_t)W * sinv32_stride(e->bl)));
    for (int b = 0; b < e->bl.nblk; ++b)
        if (e->bl.Ns[b] > 0 && !theta_tc_supported(n, 1, &e->bl.Ns[b], sinv32_stride(e->bl)))
            return engine_fail(AFQMC_ERR_UNSUPPORTED, "theta block too wide for the mixed form");
    // compensated tf32 overlap operator of the spin blocks, stacked
    {
        int nb = 0, Ns[2];
        std::vector<zd> T[2];
        const zd *Tp[2];
        const Blocks &bl = mbl(e);
        for (int b = 0; b < bl.nblk; ++b) {
            if (bl.Ns[b] == 0) continue;
            Ns[nb] = bl.Ns[b];
            T[nb].resize((size_t)n * Ns[nb]);
            MTRY(cuda_check(cudaMemcpy(T[nb].data(), e->phiT[b], sizeof(zd) * T[nb].size(), cudaMemcpyDeviceToHost),
                            "copy"));
            Tp[nb] = T[nb].data();
            ++nb;
        }
        // one operator for both blocks when it fits the 128 rows of a tile,
        // else one per block
        m->ovStacked = nb > 0 && overlap_tc_supported(n, nb, Ns);
        const int nop = m->ovStacked ? 1 : nb;
        for (int o = 0; o < nop; ++o) {
            const int nbo = m->ovStacked ? nb : 1;
            if (!overlap_tc_supported(n, nbo, Ns + o))
                return engine_fail(AFQMC_ERR_UNSUPPORTED, "overlap block too wide for the mixed form");
            std::vector<float> oh, ol;
            overlap_tc_build(nbo, Tp + o, n, Ns + o, oh, ol);
            MTRY(engine_dalloc(e, &m->Ohi[o], oh.size()));
            MTRY(engine_dalloc(e, &m->Olo[o], ol.size()));
            MTRY(cuda_check(cudaMemcpy(m->Ohi[o], oh.data(), 4 * oh.size(), cudaMemcpyHostToDevice), "upload"));
            MTRY(cuda_check(cudaMemcpy(m->Olo[o], ol.data(), 4 * ol.size(), cudaMemcpyHostToDevice), "upload"));
        }
    }
    m->ready = true;
    return AFQMC_OK;
}

void mixed_destroy(afqmc_engine *e)
{
    if (e->cpm) cp_mixed_destroy(e);
    delete e->mx;
    e->mx = nullptr;
}

int mixed_update_operators(afqmc_engine *e)
{
    if (e->kind == KIND_CP) return AFQMC_OK;
    build_et_kernel<<<64, 256, 0, e->stream>>>(e->n, e->expK[0], e->mx->Et);
    return engine_check_launch();
}

int mixed_sync_to_fp64(afqmc_engine *e)
{
    if (e->kind == KIND_CP) return cp_mixed_sync_to_fp64(e);
    f32p_to_wf_kernel<<<e->W, 256, 0, e->stream>>>(e->W, e->wsize, e->mx->wf32, e->wf, nullptr);
    return engine_check_launch();
}

int mixed_sync_from_fp64(afqmc_engine *e)
{
    if (e->kind == KIND_CP) return cp_mixed_sync_from_fp64(e);
    wf_to_f32p_kernel<<<e->W, 256, 0, e->stream>>>(e->W, e->wsize, e->wf, e->mx->wf32, nullptr);
    return engine_check_launch();
}

bool mixed_can_load_direct(const afqmc_engine *e) { return e->kind != KIND_CP; }

int mixed_load_f32(afqmc_engine *e, const float *src)
{
    const cudaError_t r = cudaMemcpyAsync(e->mx->wf32, src, sizeof(float) * (size_t)e->W * e->mx->ws32,
                                          cudaMemcpyDeviceToDevice, e->stream);
    if (r != cudaSuccess) return engine_fail(AFQMC_ERR_CUDA, std::string("installing fp32 walkers: ") + cudaGetErrorString(r));
    return AFQMC_OK;
}

int mixed_load_direct(afqmc_engine *e, const zd *src)
{
    wf_to_f32p_kernel<<<e->W, 256, 0, e->stream>>>(e->W, e->wsize, src, e->mx->wf32, nullptr);
    return engine_check_launch();
}

int mixed_status(afqmc_engine *e)
{
    if (e->kind == KIND_CP) return cp_mixed_status(e);
    int h = 0;
    cudaMemcpy(&h, e->mx->err, sizeof(int), cudaMemcpyDeviceToHost);
    return h ? 32 : 0;
}

int mixed_project_dtk_dtv(afqmc_engine *e)
{
    if (e->kind == KIND_CP) return cp_mixed_project_dtk_dtv(e);
    MixedState *m = e->mx;
    const int W = e->W;
    cudaStream_t s = e->stream;
    const bool needTheta = (e->forceType == AFQMC_DYNAMIC_FORCE);
    { PHASE(AFQMC_PH_OVERLAP); MTRY(overlap32(e, m->wf32, e->alive)); }
    {
        PHASE(AFQMC_PH_LU);
        launch_lu_logdet_inverse32(W, mbl(e), e->S, e->Sinv, m->Sinv32, e->alive, e->logw, make_double2(0, 0),
                                   e->logwT, e->logov, e->alive, e->surv, e->logw, nullptr, e->status,
                                   LU_PROJECT, needTheta, s);
        MTRY(engine_check_launch());
    }
    if (needTheta) {
        { PHASE(AFQMC_PH_THETA); MTRY(theta32(e, m->wf32, e->surv, nullptr)); }
        { PHASE(AFQMC_PH_FORCE); MTRY(force_tc(e)); }
    }
    {
        PHASE(AFQMC_PH_SAMPLE);
        launch_rng_scan(W, e->surv, 2 * e->G, e->counter, e->offs, s);
        mixed_sample_warp_kernel<<<(W + 3) / 4, 128, 0, s>>>(W, e->cdv, m->xbarp, m->splits,
                                                            (long long)2 * e->G * W, e->surv, e->alive,
                                                            e->offs, e->seed, m->Y, e->logw, e->dt * e->ET,
                                                            engine_one_body_logw(e, 0));
        MTRY(engine_check_launch());
    }
    {
        PHASE(AFQMC_PH_MBUILD);
        TcGemmArgs a;
        a.M = e->n * e->n; a.N = 2 * W; a.K = e->G;
        a.A = m->Lt; a.lda = e->G;
        a.B = m->Y; a.ldb = e->G;
        a.C = m->Mbuf; a.ldc = (long long)e->n * e->n; a.outType = TC_OUT_BF16;
        MTRY(tc(e, a));
    }
    {
        PHASE(AFQMC_PH_TAYLOR);
        MTRY(run_taylor(e));
    }
    return check_err(e);
}

int mixed_modify_gm(afqmc_engine *e)
{
    if (e->kind == KIND_CP) return cp_mixed_modify_gm(e);
    // columns in registers (FP64) where the shape fits one CTA of 512 lanes
    if (launch_mgs_col(e->W, e->n, e->ncol, e->nup, e->ndn, 1, e->mx->wf32, true, e->logw, e->alive,
                       e->status, e->stream))
        return engine_check_launch();
    const size_t bytes = (size_t)e->n * e->ncol * sizeof(float2);
    static std::atomic<unsigned long long> attr{0};
    if (first_on_device(attr)) {
        cudaFuncSetAttribute(mgs32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    }
    if (bytes > 160 * 1024) return engine_fail(AFQMC_ERR_UNSUPPORTED, "walker too large for the fp32 stabiliser");
    mgs32_kernel<<<e->W, 256, bytes, e->stream>>>(e->W, e->n, e->ncol, e->nup, e->ndn, e->mx->wf32,
                                                  e->logw, e->alive, e->status);
    return engine_check_launch();
}

int mixed_pop_weights(afqmc_engine *e)
{
    if (e->kind == KIND_CP) return cp_mixed_pop_weights(e);
    MTRY(overlap32(e, e->mx->wf32, e->alive));
    launch_lu_logdet_inverse(e->W, mbl(e), e->S, nullptr, e->alive, e->logw, make_double2(0, 0),
                             e->logwT, e->logov, e->alive, nullptr, e->logw, e->weight, e->status,
                             LU_POPWEIGHT, false, e->stream);
    return engine_check_launch();
}

int mixed_pop_control(afqmc_engine *e)
{
    if (e->kind == KIND_CP) return cp_mixed_pop_control(e);
    MixedState *m = e->mx;
    MTRY(mixed_pop_weights(e));
    launch_pop_comb(e->W, e->weight, nullptr, e->seed, e->counter, e->number, e->table,
                    e->status + e->W, e->stream);
    gather32_kernel<<<e->W, 256, 0, e->stream>>>(e->W, m->ws32, e->table, m->wf32, e->logw);
    return engine_check_launch();
}

// Exchange term of the mixed estimator.  Real A: quadratic forms as dense
// GEMMs (exchange_gemm.cu; per-walker sum over g and the den-weighted
// per-vector sums, both written here).  Complex A: tcgen05 kernel per spin
// block (bf16 operands: A2 planes, Theta) writing ex[g, w], FP64 CUDA-core
// kernel for block widths that do not divide 32.
int mixed_exchange(afqmc_engine *e)
{
    MixedState *m = e->mx;
    if (m->exGemm) {
        // exTot[w] = sum over blocks and g of ex; exNum[g] += sum_w den_w ex[g, w]
        // (restricted: block 0 counted twice)
        const Blocks &bl = mbl(e);
        bool first = true;
        for (int b = 0; b < bl.nblk; ++b) {
            if (bl.Ns[b] == 0) continue;
            MTRY(exchange_gemm_run(e, m->exg[b], m->A2r[b], m->Theta, m->exs, !first, bl.mult, m->exTot,
                                   e->exNum, m->err));
            first = false;
        }
        return AFQMC_OK;
    }
    bool allTc = true;
    for (int b = 0; b < e->bl.nblk; ++b)
        if (e->bl.Ns[b] > 0 && !exchange_tc_supported(e->n, e->bl.Ns[b])) allTc = false;
    if (!allTc) {
        if (launch_pl_exchange(e->W, e->n, e->G, e->bl, e->Aall, e->Ktot, e->thetaT, e->alive, e->ex,
                               e->stream, 1))
            return engine_fail(AFQMC_ERR_UNSUPPORTED, "exchange kernel supports at most 64 electrons per spin");
        return engine_check_launch();
    }
    int nb = 0;
    for (int b = 0; b < e->bl.nblk; ++b) {
        if (e->bl.Ns[b] == 0) continue;
        zd *out = nb == 0 ? e->ex : m->ex2;
        int r = exchange_tc_launch(e->stream, e->G, e->W, e->bl.Ns[b], e->n, m->A2r[b], m->A2i[b],
                                   m->Theta, e->bl.tOff[b], e->Ktot, e->alive, out, m->err, m->realA);
        if (r) return engine_fail(AFQMC_ERR_CUDA, "exchange launch: " + std::to_string(r));
        ++nb;
    }
    if (nb == 2) add_planes_kernel<<<592, 256, 0, e->stream>>>((long long)e->G * e->W, m->ex2, e->ex);
    return engine_check_launch();
}

int mixed_add_measurement(afqmc_engine *e)
{
    MixedState *m = e->mx;
    const int W = e->W;
    cudaStream_t s = e->stream;
    {
        PHASE(AFQMC_PH_MEASURE);
        // walkerTemp = exp(dt/2 K) walker: compensated tf32 tensor-core
        // product phi + (E - I) phi, fp32 result
        int r = 0;
        if (onebody_split_supported(e->n)) {
            r = onebody_split_launch(s, e->n, e->ncol, W, m->E1h, m->E1l, m->wf32, m->tmp32, m->err);
        } else {
            r = split_f32_launch(s, (long long)W * m->ws32, m->wf32, m->sh, m->sl);
            if (!r) r = onebody_tf32_launch(s, e->n, e->ncol, W, m->E1h, m->E1l, m->sh, m->sl, m->tmp32, nullptr, m->err);
        }
        if (r) return engine_fail(AFQMC_ERR_CUDA, "measurement one-body: " + std::to_string(r));
        MTRY(overlap32(e, m->tmp32, e->alive));
        launch_lu_logdet_inverse32(W, mbl(e), e->S, e->Sinv, m->Sinv32, e->alive, e->logw,
                                   engine_one_body_logw(e, 1), e->logwT, e->logov, e->alive, nullptr, nullptr,
                                   nullptr, e->status, LU_PLAIN, true, s);
        MTRY(engine_check_launch());
        MTRY(theta32(e, m->tmp32, e->alive, e->thetaT));
        MTRY(force_tc(e));
        xbar_combine_kernel<<<592, 256, 0, s>>>(e->G, W, m->xbarp, m->splits, (long long)2 * e->G * W, e->xbar);
        MTRY(engine_check_launch());
    }
    {
        PHASE(AFQMC_PH_EXCHANGE);
        MTRY(mixed_exchange(e));
    }
    {
        PHASE(AFQMC_PH_MEASURE);
        launch_pl_energy(W, e->G, e->Ktot, m->wfDaggerTm, e->thetaT, e->xbar, e->ex, e->alive,
                         e->logov, e->eloc, e->den, e->parts, s, m->exGemm ? m->exTot : nullptr,
                         m->restricted ? e->bl.tOff[1] : e->Ktot, mbl(e).mult);
        launch_measure_reduce(W, e->alive, e->eloc, e->den, e->parts, 1, e->acc, e->G, e->xbar,
                              m->exGemm ? nullptr : e->ex, e->bgNum, e->exNum, s);
    }
    return engine_check_launch();
}
