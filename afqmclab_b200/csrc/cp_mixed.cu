// Mixed-precision form of the constrained-path (Hubbard) walker step.
//
// Walkers live as two fp32 arrays per population, hi and lo, in the planar
// layout [re n x N | im n x N] per walker; hi holds tf32-representable values
// and the walker is hi + lo (an fp32 value).  The contractions run on the
// tcgen05 tensor cores with kind::tf32 and fp32 accumulation:
//   overlap   S = phiT^H phi: 3-term compensated product
//             (T_hi phi_hi + T_lo phi_hi + T_hi phi_lo), written as FP64 for the
//             LU/log-determinant (FP64, shared with the plain form);
//   one-body  phi' = phi + (exp(-dtK) - I) phi, again 3-term compensated;
//   force     the Green's function entries the force needs,
//             G(p, q) = sum_a phi(p, a) D(q, a) with D = conj(phiT) S^{-T},
//             one tf32 product (the force only steers importance sampling).
// The aux-field sampling, the weight/phase bookkeeping, the modified
// Gram-Schmidt re-orthonormalisation (on an FP64 copy) and population
// control stay in FP64.  The measurement takes its half step exp(+dtK/2) and
// the overlap on the tensor cores (as the propagation) and the LU, Green's
// function and energy in FP64 on a copy of the half-stepped walkers.
//
// Reference step being replaced: afqmcConstraintPathProjection.cpp:40-86
// (projectExpMinusDtKExpMinusDtV) with HubbardSOCSDOperation /
// NiupNidnSDOperation applied per walker.
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <complex>
#include <cstring>
#include <string>
#include <vector>

#include "cp_mixed.cuh"
#include "engine_internal.cuh"
#include "tc_common.cuh"
#include "once.cuh"

extern std::atomic<long long> g_launch_count;

struct CpMixedState {
    float *hi = nullptr, *lo = nullptr;     // walkers
    float *thi = nullptr, *tlo = nullptr;   // after the two-body sample
    float *Ehi = nullptr, *Elo = nullptr;   // exp(-dtK) - I, n x n row-major
    float *Hhi = nullptr, *Hlo = nullptr;   // exp(+dtK/2) - I (the measurement's half step), when real
    float *Ohi = nullptr, *Olo = nullptr;   // overlap operator, 2N x 2n row-major
    float *Ag = nullptr;                    // [Re phiT | Im phiT], n x K2 row-major
    float *Bg = nullptr;                    // per walker 2N x K2: S^{-1} rows, re/im interleaved
    float2 *gd = nullptr;                   // G(partner(q), q), W x n
    int *err = nullptr;
    long long ws = 0;                       // floats per walker and array (2 n N)
    int K2 = 0;                             // 2N rounded up to a multiple of 4
    int bnw = 0, wptO = 0;                  // overlap: columns per walker, walkers per tile
    int wptG = 0;                           // force: walkers per tile
};

namespace {

constexpr int BM = 128;
constexpr int BK = 32;                    // fp32 elements per 128-byte swizzle row
constexpr int BN = 256;
constexpr int STAGES = 2;   // two CTAs per SM: one epilogue overlaps the other's K loop
constexpr int A_BYTES = BM * BK * 4;
constexpr int B_BYTES = BN * BK * 4;
constexpr size_t SMEM = 1024 + (size_t)STAGES * (A_BYTES + B_BYTES) + 256;
constexpr int RES_BUFS = 3;
constexpr int RES_BYTES = 2 * BM * 32 * 4;   // hi and lo of 32 columns
static_assert(RES_BUFS * RES_BYTES <= STAGES * (A_BYTES + B_BYTES), "residual buffers exceed the stages");

enum { CPM_ONEBODY = 0, CPM_OVERLAP = 1, CPM_GDIAG = 2 };

struct CpTcArgs {
    int n, N, W, L, decomp;
    int kbA, nseg;       // k-blocks per segment, segments
    long long cols;      // one-body: columns of the walker population (2 N W)
    int bnw, wpt;        // walkers per tile (overlap, force), columns per walker (overlap)
    uint32_t idesc;
    const float *rhi, *rlo;
    float *ohi, *olo;
    double *S;
    long long sStride;
    const float *phi;
    float2 *gd;
    int *err;
};

// One 128 x 256 (at most) fp32 output tile per CTA.
//   warp 0 lane 0 : TMA producer      warp 1 : TMEM owner, lane 0 issues the UMMAs
//   warps 2..5    : epilogue (TMEM lane quarter = warp % 4)
template <int MODE>
__global__ void __launch_bounds__(192, 2)
cpm_tc_kernel(const __grid_constant__ CUtensorMap tA0, const __grid_constant__ CUtensorMap tA1,
              const __grid_constant__ CUtensorMap tB0, const __grid_constant__ CUtensorMap tB1,
              const __grid_constant__ CUtensorMap tR0, const __grid_constant__ CUtensorMap tR1, CpTcArgs p)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t *sA = base;
    uint8_t *sB = base + STAGES * A_BYTES;
    uint64_t *full = (uint64_t *)(sB + STAGES * B_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *tmemFull = empty + STAGES;
    // one-body: the residual columns in three 32 KB buffers over the freed stages
    uint64_t *resFull = tmemFull + 1;
    uint64_t *resEmpty = resFull + RES_BUFS;
    uint32_t *tmemSlot = (uint32_t *)(resEmpty + RES_BUFS);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * BM;
    const int tile = blockIdx.y;
    const int KT = p.kbA * p.nseg;
    uint32_t bBytes;
    if (MODE == CPM_ONEBODY) bBytes = B_BYTES;
    else if (MODE == CPM_OVERLAP) bBytes = (uint32_t)(p.wpt * p.bnw * BK * 4);
    else bBytes = (uint32_t)(p.wpt * 2 * p.N * BK * 4);

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        mbar_init(tmemFull, 1);
        for (int b = 0; b < RES_BUFS; ++b) { mbar_init(&resFull[b], 1); mbar_init(&resEmpty[b], 4); }
        fence_mbar_init();
        tma_prefetch_desc(&tA0);
        tma_prefetch_desc(&tB0);
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
                const int seg = kt / p.kbA, kk = (kt % p.kbA) * BK;
                mbar_arrive_expect_tx(&full[s], A_BYTES + bBytes);
                uint8_t *a = sA + s * A_BYTES, *b = sB + s * B_BYTES;
                if (MODE == CPM_ONEBODY) {
                    // segments: (E_hi, phi_hi), (E_lo, phi_hi), (E_hi, phi_lo)
                    tma_load_2d(a, seg == 1 ? &tA1 : &tA0, &full[s], kk, m0);
                    tma_load_2d(b, seg == 2 ? &tB1 : &tB0, &full[s], kk, tile * BN);
                } else if (MODE == CPM_OVERLAP) {
                    // segments: term (O_hi phi_hi, O_lo phi_hi, O_hi phi_lo) x plane (re, im)
                    const int term = seg >> 1, plane = seg & 1;
                    tma_load_2d(a, term == 1 ? &tA1 : &tA0, &full[s], plane * p.n + kk, m0);
                    const CUtensorMap *mb = term == 2 ? &tB1 : &tB0;
                    for (int j = 0; j < p.wpt; ++j)
                        tma_load_3d(b + j * p.bnw * BK * 4, mb, &full[s], kk, 0, 2 * (tile * p.wpt + j) + plane);
                } else {
                    tma_load_2d(a, &tA0, &full[s], kk, m0);
                    tma_load_2d(b, &tB0, &full[s], kk, tile * p.wpt * 2 * p.N);
                }
            }
            for (int kt = max(KT, STAGES); kt < KT + STAGES && ok; ++kt) {
                const int s = kt % STAGES;
                ok = mbar_wait(&empty[s], ((kt / STAGES) - 1) & 1);
            }
            if (MODE == CPM_ONEBODY) {
                // the MMAs have read the stages: the residual phi = hi + lo of
                // the tile's columns, 32 at a time, by TMA into the freed space
                int issued = 0;
                for (int ch = 0; ch < BN / 32 && ok; ++ch) {
                    const int b = ch % RES_BUFS;
                    if (ch >= RES_BUFS) ok = mbar_wait(&resEmpty[b], ((ch / RES_BUFS) - 1) & 1);
                    if (!ok) break;
                    uint8_t *buf = base + b * RES_BYTES;
                    mbar_arrive_expect_tx(&resFull[b], RES_BYTES);
                    tma_load_2d(buf, &tR0, &resFull[b], m0, tile * BN + ch * 32);
                    tma_load_2d(buf + RES_BYTES / 2, &tR1, &resFull[b], m0, tile * BN + ch * 32);
                    ++issued;
                }
                // the copies land before this CTA can leave
                for (int ch = issued - RES_BUFS < 0 ? 0 : issued - RES_BUFS; ch < issued; ++ch)
                    (void)mbar_wait(&resFull[ch % RES_BUFS], (ch / RES_BUFS) & 1);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            for (int kt = 0; kt < KT && ok; ++kt) {
                const int s = kt % STAGES;
                ok = mbar_wait(&full[s], (kt / STAGES) & 1);
                if (!ok) break;
                tc_fence_after();
                const uint32_t a0 = smem_u32(sA + s * A_BYTES);
                const uint32_t b0 = smem_u32(sB + s * B_BYTES);
#pragma unroll
                for (int k8 = 0; k8 < BK / 8; ++k8)
                    umma_tf32(tmem, desc_k_sw128(a0 + k8 * 32), desc_k_sw128(b0 + k8 * 32), p.idesc,
                              (kt > 0 || k8 > 0) ? 1u : 0u);
                umma_commit(&empty[s]);
            }
            umma_commit(tmemFull);
        }
        __syncwarp();
    } else {
        ok = mbar_wait(tmemFull, 0);
        tc_fence_after();
        const int q = warp & 3;
        const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16);
        const int row = m0 + q * 32 + lane;
        if (ok && MODE == CPM_ONEBODY) {
            // phi' = (E - I) phi + phi: the residual phi = hi + lo comes by
            // TMA, 32 columns per buffer, smem [column][row]
            const int n = p.n;
            const long long col0 = (long long)tile * BN;
            const int ncols = (int)(p.cols - col0 < BN ? p.cols - col0 : BN);
            const size_t rbase = (size_t)row + (size_t)n * col0;
            float *oh = p.ohi + rbase;
            float *ol = p.olo ? p.olo + rbase : nullptr;
            const bool rowOK = row < n;
            const int rl = q * 32 + lane;
#pragma unroll 1
            for (int ch = 0; ch < BN / 32; ++ch) {
                const int b = ch % RES_BUFS;
                ok = __all_sync(0xffffffffu, mbar_wait(&resFull[b], (ch / RES_BUFS) & 1)) != 0;
                if (!ok) break;
                float v[32];
                tmem_ld32(trow + ch * 32, v);
                const float *hb = (const float *)(base + b * RES_BYTES), *lb = hb + BM * 32;
                if (rowOK) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const int c = ch * 32 + j;
                        if (c < ncols) {
                            const float res = hb[j * BM + rl] + lb[j * BM + rl];
                            const float x = v[j] + res;
                            if (ol) {
                                const float h = tf32_round(x);
                                oh[n * c] = h;
                                ol[n * c] = x - h;
                            } else {
                                oh[n * c] = x;
                            }
                        }
                    }
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&resEmpty[b]);
            }
        } else if (ok && MODE == CPM_OVERLAP) {
            const int N = p.N;
            const int part = row >= N ? 1 : 0, a = row - part * N;
            const int ncols = p.wpt * p.bnw;
#pragma unroll 1
            for (int c0 = 0; c0 < ncols; c0 += 32) {
                float v[32];
                tmem_ld32(trow + c0, v);
                if (row < 2 * N) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const int col = c0 + j;
                        const int wj = col / p.bnw, c = col - wj * p.bnw;
                        const int w = tile * p.wpt + wj;
                        if (col < ncols && c < N && w < p.W)
                            p.S[2 * ((size_t)w * p.sStride + a + (size_t)N * c) + part] = (double)v[j];
                    }
                }
            }
        } else if (ok && MODE == CPM_GDIAG) {
            const int N = p.N, L = p.L, n = p.n;
            const int two = 2 * N;
            const int ncols = p.wpt * two;
            const int prow = p.decomp <= 1 ? row : (row < L ? row + L : row - L);
            float gr = 0.f, gi = 0.f;
            int cur = 0;
#pragma unroll 1
            for (int c0 = 0; c0 < ncols; c0 += 32) {
                // this chunk's walker entries first, all loads in flight
                // before the accumulator is read (and ahead of the stores)
                float fr[16], fi[16];
#pragma unroll
                for (int t = 0; t < 16; ++t) {
                    const int col = c0 + 2 * t;
                    const int j = col / two, a = (col - j * two) >> 1;
                    const int w = tile * p.wpt + j;
                    if (col < ncols && row < n && w < p.W) {
                        const float *ph = p.phi + (size_t)w * 2 * n * N + prow + (size_t)n * a;
                        fr[t] = ph[0];
                        fi[t] = ph[(size_t)n * N];
                    } else {
                        fr[t] = 0.f;
                        fi[t] = 0.f;
                    }
                }
                float v[32];
                tmem_ld32(trow + c0, v);
#pragma unroll
                for (int t = 0; t < 16; ++t) {
                    const int col = c0 + 2 * t;
                    if (col < ncols) {
                        const int j = col / two;
                        if (j != cur) {
                            const int w = tile * p.wpt + cur;
                            if (row < n && w < p.W) p.gd[(size_t)w * n + row] = make_float2(gr, gi);
                            gr = gi = 0.f;
                            cur = j;
                        }
                        gr += fr[t] * v[2 * t] - fi[t] * v[2 * t + 1];
                        gi += fr[t] * v[2 * t + 1] + fi[t] * v[2 * t];
                    }
                }
            }
            const int w = tile * p.wpt + cur;
            if (row < n && w < p.W) p.gd[(size_t)w * n + row] = make_float2(gr, gi);
        }
    }
    if (!ok && p.err) atomicExch(p.err, 1);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) tmem_dealloc(tmem, BN);
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

// fp32 tensor map, 128-byte swizzle, box of 32 elements along dim 0.
int make_map_f32(CUtensorMap *map, const float *base, int rank, const long long *dims,
                 const long long *pitchBytes, const int *box, bool swizzle128 = true)
{
    auto enc = encoder();
    if (!enc) return (int)cudaErrorNotSupported;
    if ((uintptr_t)base & 15) return (int)cudaErrorMisalignedAddress;
    cuuint64_t d[3];
    cuuint64_t st[2];
    cuuint32_t bx[3], es[3] = {1u, 1u, 1u};
    for (int i = 0; i < rank; ++i) { d[i] = (cuuint64_t)dims[i]; bx[i] = (cuuint32_t)box[i]; }
    for (int i = 0; i + 1 < rank; ++i) {
        if (pitchBytes[i] & 15) return (int)cudaErrorMisalignedAddress;
        st[i] = (cuuint64_t)pitchBytes[i];
    }
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, const_cast<float *>(base), d, st, bx, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE,
                     swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : (int)r + 10000;
}

// the one-body's residual walker columns: box of BM rows x 32 columns, no
// swizzle (smem [column][row])
int make_res_map(CUtensorMap *map, const float *base, int n, long long cols)
{
    long long d[2] = {n, cols}, pch[1] = {(long long)n * 4};
    int box[2] = {BM, 32};
    return make_map_f32(map, base, 2, d, pch, box, false);
}

template <int MODE>
int launch_tc_stream(cudaStream_t s, dim3 grid, const CUtensorMap &a0, const CUtensorMap &a1,
                     const CUtensorMap &b0, const CUtensorMap &b1, const CUtensorMap &r0, const CUtensorMap &r1,
                     const CpTcArgs &args)
{
    static std::atomic<unsigned long long> attr{0};
    if (first_on_device(attr)) {
        cudaFuncSetAttribute(cpm_tc_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
    }
    g_launch_count++;
    cpm_tc_kernel<MODE><<<grid, 192, SMEM, s>>>(a0, a1, b0, b1, r0, r1, args);
    return (int)cudaGetLastError();
}

template <int MODE>
int launch_tc(afqmc_engine *e, dim3 grid, const CUtensorMap &a0, const CUtensorMap &a1, const CUtensorMap &b0,
              const CUtensorMap &b1, const CUtensorMap &r0, const CUtensorMap &r1, const CpTcArgs &args)
{
    launch_tc_stream<MODE>(e->stream, grid, a0, a1, b0, b1, r0, r1, args);
    return engine_check_launch();
}

CpTcArgs base_args(afqmc_engine *e)
{
    CpTcArgs a{};
    a.n = e->n; a.N = e->ncol; a.W = e->W; a.L = e->L; a.decomp = e->decomp;
    a.err = e->cpm->err;
    return a;
}

#define CTRY(x) do { int r_ = (x); if (r_) return engine_fail(AFQMC_ERR_CUDA, std::string("tensor map: ") + std::to_string(r_)); } while (0)

// S = phiT^H phi for every walker (3-term compensated tf32), FP64 result in e->S
int overlap_tc(afqmc_engine *e, const float *hi, const float *lo)
{
    CpMixedState *m = e->cpm;
    const int n = e->n, N = e->ncol, W = e->W;
    CUtensorMap a0, a1, b0, b1;
    long long da[2] = {2LL * n, 2LL * N}, pa[1] = {2LL * n * 4};
    int boxA[2] = {BK, BM};
    CTRY(make_map_f32(&a0, m->Ohi, 2, da, pa, boxA));
    CTRY(make_map_f32(&a1, m->Olo, 2, da, pa, boxA));
    long long db[3] = {n, N, 2LL * W}, pb[2] = {(long long)n * 4, (long long)n * N * 4};
    int boxB[3] = {BK, m->bnw, 1};
    CTRY(make_map_f32(&b0, hi, 3, db, pb, boxB));
    CTRY(make_map_f32(&b1, lo, 3, db, pb, boxB));
    CpTcArgs a = base_args(e);
    a.kbA = (n + BK - 1) / BK; a.nseg = 6;
    a.bnw = m->bnw; a.wpt = m->wptO;
    a.idesc = idesc_tf32(BM, m->wptO * m->bnw);
    a.S = (double *)e->S; a.sStride = e->bl.sStride;
    dim3 grid((2 * N + BM - 1) / BM, (W + m->wptO - 1) / m->wptO);
    return launch_tc<CPM_OVERLAP>(e, grid, a0, a1, b0, b1, a0, a1, a);
}

// Green's function entries for the force: gd[w][q] = G(partner(q), q)
int gdiag_tc(afqmc_engine *e)
{
    CpMixedState *m = e->cpm;
    const int n = e->n, N = e->ncol, W = e->W;
    CUtensorMap a0, b0;
    long long da[2] = {2LL * N, n}, pa[1] = {(long long)m->K2 * 4};
    int boxA[2] = {BK, BM};
    CTRY(make_map_f32(&a0, m->Ag, 2, da, pa, boxA));
    long long db[2] = {2LL * N, 2LL * N * W}, pb[1] = {(long long)m->K2 * 4};
    int boxB[2] = {BK, m->wptG * 2 * N};
    CTRY(make_map_f32(&b0, m->Bg, 2, db, pb, boxB));
    CpTcArgs a = base_args(e);
    a.kbA = (2 * N + BK - 1) / BK; a.nseg = 1;
    a.wpt = m->wptG;
    a.idesc = idesc_tf32(BM, (m->wptG * 2 * N + 15) / 16 * 16);
    a.phi = m->hi; a.gd = m->gd;
    dim3 grid((n + BM - 1) / BM, (W + m->wptG - 1) / m->wptG);
    return launch_tc<CPM_GDIAG>(e, grid, a0, a0, b0, b0, a0, a0, a);
}

// out <- in + (O - I) in for a one-body operator given as O - I (hi, lo)
int onebody_tc_op(afqmc_engine *e, const float *Ohi, const float *Olo, const float *inHi, const float *inLo,
                  float *outHi, float *outLo)
{
    const int n = e->n, N = e->ncol, W = e->W;
    CUtensorMap a0, a1, b0, b1;
    long long da[2] = {n, n}, pa[1] = {(long long)n * 4};
    int boxA[2] = {BK, BM};
    CTRY(make_map_f32(&a0, Ohi, 2, da, pa, boxA));
    CTRY(make_map_f32(&a1, Olo, 2, da, pa, boxA));
    const long long cols = 2LL * N * W;
    long long db[2] = {n, cols}, pb[1] = {(long long)n * 4};
    int boxB[2] = {BK, BN};
    CTRY(make_map_f32(&b0, inHi, 2, db, pb, boxB));
    CTRY(make_map_f32(&b1, inLo, 2, db, pb, boxB));
    CUtensorMap r0, r1;
    CTRY(make_res_map(&r0, inHi, n, cols));
    CTRY(make_res_map(&r1, inLo, n, cols));
    CpTcArgs a = base_args(e);
    a.kbA = (n + BK - 1) / BK; a.nseg = 3;
    a.cols = cols;
    a.idesc = idesc_tf32(BM, BN);
    a.rhi = inHi; a.rlo = inLo; a.ohi = outHi; a.olo = outLo;
    dim3 grid((n + BM - 1) / BM, (unsigned)((cols + BN - 1) / BN));
    return launch_tc<CPM_ONEBODY>(e, grid, a0, a1, b0, b1, r0, r1, a);
}

// phi <- phi + (exp(-dtK) - I) phi from (thi, tlo) into (hi, lo)
int onebody_tc(afqmc_engine *e)
{
    CpMixedState *m = e->cpm;
    return onebody_tc_op(e, m->Ehi, m->Elo, m->thi, m->tlo, m->hi, m->lo);
}

// Bg rows of walker w: row 2a = [Re Sinv(a, :) | Im Sinv(a, :)],
// row 2a+1 = [Im Sinv(a, :) | -Re Sinv(a, :)]  (tf32-rounded)
__global__ void build_bg_kernel(int W, int N, int K2, const zd *Sinv, long long sStride, const int *surv,
                                float *Bg)
{
    const int w = blockIdx.x;
    if (!surv[w]) return;
    const zd *S = Sinv + (size_t)w * sStride;
    float *B = Bg + (size_t)w * 2 * N * K2;
    for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
        const int b = e % N, a = e / N;
        const zd s = S[a + (size_t)N * b];
        const float sr = tf32_round((float)s.x), si = tf32_round((float)s.y);
        float *r0 = B + (size_t)(2 * a) * K2, *r1 = r0 + K2;
        r0[b] = sr; r0[N + b] = si;
        r1[b] = si; r1[N + b] = -sr;
    }
}

__device__ __forceinline__ zd zexp_d(zd z)
{
    double s, c;
    sincos(z.y, &s, &c);
    const double r = exp(z.x);
    return make_double2(r * c, r * s);
}

// Force from the Green's function entries, aux-field sampling, sample
// log-weight and the aux-field two-body application; same arithmetic and
// random stream as the FP64 kernels (NiupNidn::sampleAuxFromForce,
// NiupNidn.cpp:66-84; getTwoBodySampleFromAuxForce :100-142;
// NiupNidnSampleSDOperation::applyToRight, NiupNidnSDOperation.cpp:15-41;
// HubbardSOCMeasureFixedSDSD force, HubbardSOCMeasureFixedSDSD.cpp:95-130).
__global__ void __launch_bounds__(256)
cpm_sample_apply_kernel(int W, HubbardDev h, const float2 *gd, const int *surv, const unsigned long long *offs,
                        uint64_t seed, const float *hi, const float *lo, float *thi, float *tlo, zd *logw,
                        double dtET, zd hopLogw, int *auxOut)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int w = blockIdx.x;
    if (!surv[w]) return;
    const int L = h.L, N = h.N, n = h.n;
    // layout: 16-byte entries first, so every array is aligned for any L
    zd *gxS = (zd *)smem_raw;                        // per site: gamma x
    float2 *d = (float2 *)(gxS + L);                 // 4 L entries: d00, d01, d10, d11
    int *aux = (int *)(d + 4 * L);
    double *lpS = (double *)(aux + L + (L & 1));     // per site: x f - log(e^f + e^-f)
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
        double f;
        if (h.constForce) {
            f = h.constForce[i];
        } else {
            const float2 ga = gd[(size_t)w * n + i], gb = gd[(size_t)w * n + i + L];
            zd a = make_double2(ga.x, ga.y), b = make_double2(gb.x, gb.y), bgv;
            if (h.decomp == 0) bgv = make_double2(a.x + b.x - 1.0, a.y + b.y);
            else if (h.decomp == 2) bgv = zadd(a, b);
            else bgv = zsub(a, b);
            f = zmul(h.gamma[i], bgv).x;
            f = fmin(fmax(f, -h.forceCap), h.forceCap);
        }
        const double em = exp(-f), ep = exp(f);
        const int x = (rng_uniform(seed, offs[w] + (unsigned long long)i) < em / (em + ep)) ? -1 : 1;
        aux[i] = x;
        if (auxOut) auxOut[(size_t)w * L + i] = x;
        lpS[i] = x * f - log(ep + em);
        const zd ga = zscale(h.gamma[i], (double)x);
        gxS[i] = ga;
        zd a00, a01, a10, a11;
        if (h.decomp == 0) {
            const zd ex = zexp_d(ga);
            a00 = zmul(ex, h.cd00[i]); a10 = zmul(ex, h.cd10[i]); a01 = zmul(ex, h.cd01[i]); a11 = zmul(ex, h.cd11[i]);
        } else if (h.decomp == 1) {
            const zd ex = zexp_d(ga), ei = zexp_d(zneg(ga));
            a00 = zmul(ex, h.cd00[i]); a10 = zmul(ei, h.cd10[i]); a01 = zmul(ex, h.cd01[i]); a11 = zmul(ei, h.cd11[i]);
        } else {
            const zd ep2 = zexp_d(ga), em2 = zexp_d(zneg(ga));
            zd c, s;
            if (h.decomp == 2) {
                c = zscale(zadd(ep2, em2), 0.5); s = zscale(zsub(ep2, em2), 0.5);
            } else {
                // cos / sin of the complex argument
                double sn, cs;
                sincos(ga.x, &sn, &cs);
                c = make_double2(cs * cosh(ga.y), -sn * sinh(ga.y));
                s = make_double2(sn * cosh(ga.y), cs * sinh(ga.y));
            }
            const zd sa = h.decomp == 2 ? s : zneg(s);
            a00 = zadd(zmul(c, h.cd00[i]), zmul(s, h.cd10[i]));
            a10 = zadd(zmul(sa, h.cd00[i]), zmul(c, h.cd10[i]));
            a01 = zadd(zmul(c, h.cd01[i]), zmul(s, h.cd11[i]));
            a11 = zadd(zmul(sa, h.cd01[i]), zmul(c, h.cd11[i]));
        }
        d[i] = make_float2((float)a00.x, (float)a00.y);
        d[L + i] = make_float2((float)a01.x, (float)a01.y);
        d[2 * L + i] = make_float2((float)a10.x, (float)a10.y);
        d[3 * L + i] = make_float2((float)a11.x, (float)a11.y);
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        // the walker's sample log-weight: the per-site terms summed by warp 0
        // in a fixed order (lane-strided partial sums, then a shuffle tree)
        const int lane = threadIdx.x;
        double lp = 0.0;
        zd gsum = make_double2(0.0, 0.0);
        for (int i = lane; i < L; i += 32) {
            lp += lpS[i];
            gsum = zadd(gsum, gxS[i]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lp += __shfl_xor_sync(0xffffffffu, lp, o);
            gsum.x += __shfl_xor_sync(0xffffffffu, gsum.x, o);
            gsum.y += __shfl_xor_sync(0xffffffffu, gsum.y, o);
        }
        if (lane == 0) {
            zd lw;
            if (h.decomp == 0) lw = zsub(make_double2(log(0.5) * L + h.dtUSum * 0.5, 0.0), gsum);
            else lw = make_double2(log(0.5) * L, 0.0);
            lw.x -= lp;
            zd t = zadd(lw, logw[w]);
            t.x += dtET;
            logw[w] = zadd(hopLogw, t);
        }
    }
    const size_t base = (size_t)w * 2 * n * N, plane = (size_t)n * N;
    for (int e = threadIdx.x; e < L * N; e += blockDim.x) {
        const int i = e % L, j = e / L;
        const size_t ia = base + i + (size_t)n * j, ib = ia + L;
        const float ar = hi[ia] + lo[ia], ai = hi[ia + plane] + lo[ia + plane];
        const float br = hi[ib] + lo[ib], bi = hi[ib + plane] + lo[ib + plane];
        const float2 d00 = d[i], d01 = d[L + i], d10 = d[2 * L + i], d11 = d[3 * L + i];
        const float r0r = d00.x * ar - d00.y * ai + d01.x * br - d01.y * bi;
        const float r0i = d00.x * ai + d00.y * ar + d01.x * bi + d01.y * br;
        const float r1r = d10.x * ar - d10.y * ai + d11.x * br - d11.y * bi;
        const float r1i = d10.x * ai + d10.y * ar + d11.x * bi + d11.y * br;
        float h0 = tf32_round(r0r); thi[ia] = h0; tlo[ia] = r0r - h0;
        h0 = tf32_round(r0i); thi[ia + plane] = h0; tlo[ia + plane] = r0i - h0;
        h0 = tf32_round(r1r); thi[ib] = h0; tlo[ib] = r1r - h0;
        h0 = tf32_round(r1i); thi[ib + plane] = h0; tlo[ib + plane] = r1i - h0;
    }
}

// FP64 walkers <-> (hi, lo) fp32 planar walkers
__global__ void split_kernel(int W, int n, int N, const zd *wf, float *hi, float *lo)
{
    const int w = blockIdx.x;
    const size_t nN = (size_t)n * N;
    const zd *src = wf + (size_t)w * nN;
    float *h = hi + (size_t)w * 2 * nN, *l = lo + (size_t)w * 2 * nN;
    for (size_t e = threadIdx.x; e < nN; e += blockDim.x) {
        const zd v = src[e];
        const float xr = (float)v.x, xi = (float)v.y;
        const float hr = tf32_round(xr), hi_ = tf32_round(xi);
        h[e] = hr; l[e] = xr - hr;
        h[e + nN] = hi_; l[e + nN] = xi - hi_;
    }
}

__global__ void combine_kernel(int W, int n, int N, const float *hi, const float *lo, zd *wf)
{
    const int w = blockIdx.x;
    const size_t nN = (size_t)n * N;
    zd *dst = wf + (size_t)w * nN;
    const float *h = hi + (size_t)w * 2 * nN, *l = lo + (size_t)w * 2 * nN;
    for (size_t e = threadIdx.x; e < nN; e += blockDim.x)
        dst[e] = make_double2((double)(h[e] + l[e]), (double)(h[e + nN] + l[e + nN]));
}

__global__ void split_f32_kernel(long long count, const float *x, float *hi, float *lo)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
         e += (long long)gridDim.x * blockDim.x) {
        const float v = x[e], h = tf32_round(v);
        hi[e] = h;
        lo[e] = v - h;
    }
}

__global__ void gather_kernel(int W, long long ws, const int *table, float *hi, float *lo, zd *logw)
{
    const int i = blockIdx.x;
    const int j = table[i];
    if (j == i || j < 0) return;
    const float4 *sh = (const float4 *)(hi + (size_t)j * ws), *sl = (const float4 *)(lo + (size_t)j * ws);
    float4 *dh = (float4 *)(hi + (size_t)i * ws), *dl = (float4 *)(lo + (size_t)i * ws);
    for (long long e = threadIdx.x; e < ws / 4; e += blockDim.x) { dh[e] = sh[e]; dl[e] = sl[e]; }
    if (threadIdx.x == 0) logw[i] = logw[j];
}

float tf32_host(float x)
{
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7F800000u) != 0x7F800000u) {
        u += 0x1000u;
        u &= 0xFFFFE000u;
    }
    std::memcpy(&x, &u, 4);
    return x;
}

void split_host(double v, float &h, float &l)
{
    h = tf32_host((float)v);
    l = tf32_host((float)(v - (double)h));
}

}  // namespace

int tf32_split_operator(const zd *E, int n, std::vector<float> &hi, std::vector<float> &lo)
{
    hi.assign((size_t)n * n, 0.f);
    lo.assign((size_t)n * n, 0.f);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k) {
            const zd v = E[i + (size_t)n * k];
            if (v.y != 0.0) return -1;
            split_host(v.x - (i == k ? 1.0 : 0.0), hi[(size_t)i * n + k], lo[(size_t)i * n + k]);
        }
    return 0;
}

int split_f32_launch(cudaStream_t s, long long count, const float *x, float *hi, float *lo)
{
    g_launch_count++;
    split_f32_kernel<<<1184, 256, 0, s>>>(count, x, hi, lo);
    return (int)cudaGetLastError();
}

int onebody_tf32_launch(cudaStream_t s, int n, int ncol, int W, const float *Ehi, const float *Elo,
                        const float *rhi, const float *rlo, float *ohi, float *olo, int *err)
{
    CUtensorMap a0, a1, b0, b1;
    long long da[2] = {n, n}, pa[1] = {(long long)n * 4};
    int boxA[2] = {BK, BM};
    int r = make_map_f32(&a0, Ehi, 2, da, pa, boxA);
    if (!r) r = make_map_f32(&a1, Elo, 2, da, pa, boxA);
    const long long cols = 2LL * ncol * W;
    long long db[2] = {n, cols}, pb[1] = {(long long)n * 4};
    int boxB[2] = {BK, BN};
    if (!r) r = make_map_f32(&b0, rhi, 2, db, pb, boxB);
    if (!r) r = make_map_f32(&b1, rlo, 2, db, pb, boxB);
    CUtensorMap r0, r1;
    if (!r) r = make_res_map(&r0, rhi, n, cols);
    if (!r) r = make_res_map(&r1, rlo, n, cols);
    if (r) return r;
    CpTcArgs a{};
    a.n = n; a.N = ncol; a.W = W;
    a.kbA = (n + BK - 1) / BK; a.nseg = 3;
    a.cols = cols;
    a.idesc = idesc_tf32(BM, BN);
    a.rhi = rhi; a.rlo = rlo; a.ohi = ohi; a.olo = olo;
    a.err = err;
    dim3 grid((n + BM - 1) / BM, (unsigned)((cols + BN - 1) / BN));
    return launch_tc_stream<CPM_ONEBODY>(s, grid, a0, a1, b0, b1, r0, r1, a);
}

bool cp_mixed_supported(int L, int N, std::string *why)
{
    const int n = 2 * L;
    if (n % 4 != 0) { if (why) *why = "mixed constrained-path form needs an even number of sites"; return false; }
    if (N > 128) { if (why) *why = "mixed constrained-path form needs at most 128 electrons"; return false; }
    return true;
}

int cp_mixed_create(afqmc_engine *e)
{
    std::string why;
    if (!cp_mixed_supported(e->L, e->ncol, &why)) return engine_fail(AFQMC_ERR_UNSUPPORTED, why);
    const int n = e->n, N = e->ncol, W = e->W;
    std::vector<zd> E((size_t)n * n), T((size_t)n * N), H((size_t)n * n);
    if (cudaMemcpy(E.data(), e->expK[0], sizeof(zd) * E.size(), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(H.data(), e->expK[1], sizeof(zd) * H.size(), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(T.data(), e->phiT[0], sizeof(zd) * T.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
        return engine_fail(AFQMC_ERR_CUDA, "reading operators for the mixed form");
    for (const zd &v : E)
        if (v.y != 0.0) return engine_fail(AFQMC_ERR_UNSUPPORTED, "mixed constrained-path form needs a real exp(-dt K)");
    CpMixedState *m = new CpMixedState();
    e->cpm = m;
    m->ws = 2LL * n * N;
    m->K2 = (2 * N + 3) / 4 * 4;
    m->bnw = (N + 15) / 16 * 16;
    m->wptO = std::max(1, BN / m->bnw);
    m->wptG = std::max(1, BN / (2 * N));
#define CM(x) do { int r_ = (x); if (r_ != AFQMC_OK) return r_; } while (0)
    CM(engine_dalloc(e, &m->hi, (size_t)W * m->ws));
    CM(engine_dalloc(e, &m->lo, (size_t)W * m->ws));
    CM(engine_dalloc(e, &m->thi, (size_t)W * m->ws));
    CM(engine_dalloc(e, &m->tlo, (size_t)W * m->ws));
    CM(engine_dalloc(e, &m->Ehi, (size_t)n * n));
    CM(engine_dalloc(e, &m->Elo, (size_t)n * n));
    CM(engine_dalloc(e, &m->Ohi, (size_t)4 * N * n));
    CM(engine_dalloc(e, &m->Olo, (size_t)4 * N * n));
    CM(engine_dalloc(e, &m->Ag, (size_t)n * m->K2));
    CM(engine_dalloc(e, &m->Bg, (size_t)W * 2 * N * m->K2));
    CM(engine_dalloc(e, (float **)&m->gd, (size_t)2 * W * n));
    CM(engine_dalloc(e, &m->err, 1));
    // E - I, row-major (row i = output site, contiguous over k)
    std::vector<float> eh((size_t)n * n), el((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k)
            split_host(E[i + (size_t)n * k].x - (i == k ? 1.0 : 0.0), eh[(size_t)i * n + k], el[(size_t)i * n + k]);
    // overlap operator rows: a -> [Re T(:,a) | Im T(:,a)], N + a -> [-Im T(:,a) | Re T(:,a)]
    std::vector<float> oh((size_t)4 * N * n), ol((size_t)4 * N * n);
    for (int a = 0; a < N; ++a)
        for (int i = 0; i < n; ++i) {
            const zd t = T[i + (size_t)n * a];
            const size_t r0 = (size_t)a * 2 * n, r1 = (size_t)(N + a) * 2 * n;
            split_host(t.x, oh[r0 + i], ol[r0 + i]);
            split_host(t.y, oh[r0 + n + i], ol[r0 + n + i]);
            split_host(-t.y, oh[r1 + i], ol[r1 + i]);
            split_host(t.x, oh[r1 + n + i], ol[r1 + n + i]);
        }
    std::vector<float> ag((size_t)n * m->K2, 0.f);
    for (int q = 0; q < n; ++q)
        for (int b = 0; b < N; ++b) {
            const zd t = T[q + (size_t)n * b];
            ag[(size_t)q * m->K2 + b] = tf32_host((float)t.x);
            ag[(size_t)q * m->K2 + N + b] = tf32_host((float)t.y);
        }
    // the measurement's half step exp(+dtK/2) - I on the tensor cores when it is real
    bool hReal = true;
    for (const zd &v : H) hReal = hReal && v.y == 0.0;
    if (hReal) {
        std::vector<float> hh((size_t)n * n), hl((size_t)n * n);
        for (int i = 0; i < n; ++i)
            for (int k = 0; k < n; ++k)
                split_host(H[i + (size_t)n * k].x - (i == k ? 1.0 : 0.0), hh[(size_t)i * n + k], hl[(size_t)i * n + k]);
        CM(engine_dalloc(e, &m->Hhi, (size_t)n * n));
        CM(engine_dalloc(e, &m->Hlo, (size_t)n * n));
        if (cudaMemcpy(m->Hhi, hh.data(), 4 * hh.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(m->Hlo, hl.data(), 4 * hl.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            return engine_fail(AFQMC_ERR_CUDA, "uploading the mixed-form half-step operator");
    }
    if (cudaMemcpy(m->Ehi, eh.data(), 4 * eh.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(m->Elo, el.data(), 4 * el.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(m->Ohi, oh.data(), 4 * oh.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(m->Olo, ol.data(), 4 * ol.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(m->Ag, ag.data(), 4 * ag.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return engine_fail(AFQMC_ERR_CUDA, "uploading mixed-form operators");
    if (cudaMemset(m->Bg, 0, sizeof(float) * (size_t)W * 2 * N * m->K2) != cudaSuccess ||
        cudaMemset(m->err, 0, sizeof(int)) != cudaSuccess)
        return engine_fail(AFQMC_ERR_CUDA, "clearing mixed-form buffers");
    return AFQMC_OK;
}

void cp_mixed_destroy(afqmc_engine *e)
{
    delete e->cpm;
    e->cpm = nullptr;
}

int cp_mixed_sync_to_fp64(afqmc_engine *e)
{
    g_launch_count++;
    combine_kernel<<<e->W, 256, 0, e->stream>>>(e->W, e->n, e->ncol, e->cpm->hi, e->cpm->lo, e->wf);
    return engine_check_launch();
}

int cp_mixed_sync_from_fp64(afqmc_engine *e)
{
    g_launch_count++;
    split_kernel<<<e->W, 256, 0, e->stream>>>(e->W, e->n, e->ncol, e->wf, e->cpm->hi, e->cpm->lo);
    return engine_check_launch();
}

// The measurement's half step and overlap on the tensor cores: (thi, tlo) <-
// the walkers after exp(+dtK/2) (compensated tf32, as the propagation),
// S = phiT^H of them (FP64 result in e->S), and their FP64 copy in e->wfTmp
// for the Green's function.  *done is false (nothing launched) where the
// half-step operator is not real; the FP64 measurement runs then.
int cp_mixed_measure_prep(afqmc_engine *e, bool *done)
{
    CpMixedState *m = e->cpm;
    *done = false;
    if (!m->Hhi) return AFQMC_OK;
    CM(onebody_tc_op(e, m->Hhi, m->Hlo, m->hi, m->lo, m->thi, m->tlo));
    CM(overlap_tc(e, m->thi, m->tlo));
    g_launch_count++;
    combine_kernel<<<e->W, 256, 0, e->stream>>>(e->W, e->n, e->ncol, m->thi, m->tlo, e->wfTmp);
    CM(engine_check_launch());
    *done = true;
    return AFQMC_OK;
}

int cp_mixed_status(afqmc_engine *e)
{
    int h = 0;
    cudaMemcpy(&h, e->cpm->err, sizeof(int), cudaMemcpyDeviceToHost);
    return h ? 32 : 0;
}

int cp_mixed_project_dtk_dtv(afqmc_engine *e)
{
    CpMixedState *m = e->cpm;
    const int W = e->W;
    cudaStream_t s = e->stream;
    const bool needG = (e->forceType == AFQMC_DYNAMIC_FORCE);
    { PHASE(AFQMC_PH_OVERLAP); CM(overlap_tc(e, m->hi, m->lo)); }
    {
        PHASE(AFQMC_PH_LU);
        launch_lu_logdet_inverse(W, e->bl, e->S, e->Sinv, e->alive, e->logw, make_double2(0, 0),
                                 e->logwT, e->logov, e->alive, e->surv, e->logw, nullptr, e->status,
                                 LU_PROJECT, needG, s);
        CM(engine_check_launch());
    }
    if (needG) {
        PHASE(AFQMC_PH_FORCE);
        g_launch_count++;
        build_bg_kernel<<<W, 256, 0, s>>>(W, e->ncol, m->K2, e->Sinv, e->bl.sStride, e->surv, m->Bg);
        CM(engine_check_launch());
        CM(gdiag_tc(e));
    }
    {
        PHASE(AFQMC_PH_SAMPLE);
        launch_rng_scan(W, e->surv, e->L, e->counter, e->offs, s);
        const int L = e->L;
        const size_t smem = sizeof(float2) * 4 * L + sizeof(int) * (L + (L & 1)) + sizeof(double) * L + sizeof(zd) * L;
        g_launch_count++;
        cpm_sample_apply_kernel<<<W, 256, smem, s>>>(W, e->hd, m->gd, e->surv, e->offs, e->seed, m->hi, m->lo,
                                                     m->thi, m->tlo, e->logw, e->dt * e->ET,
                                                     engine_one_body_logw(e, 0), nullptr);
        CM(engine_check_launch());
    }
    { PHASE(AFQMC_PH_ONEBODY); CM(onebody_tc(e)); }
    return engine_check_launch();
}

int cp_mixed_modify_gm(afqmc_engine *e)
{
    CM(cp_mixed_sync_to_fp64(e));
    launch_mgs(e->W, e->n, e->ncol, e->nup, e->ndn, 0, e->wf, e->logw, e->alive, e->status, e->stream);
    CM(engine_check_launch());
    return cp_mixed_sync_from_fp64(e);
}

int cp_mixed_pop_weights(afqmc_engine *e)
{
    CpMixedState *m = e->cpm;
    CM(overlap_tc(e, m->hi, m->lo));
    launch_lu_logdet_inverse(e->W, e->bl, e->S, nullptr, e->alive, e->logw, make_double2(0, 0),
                             e->logwT, e->logov, e->alive, nullptr, e->logw, e->weight, e->status,
                             LU_POPWEIGHT, false, e->stream);
    return engine_check_launch();
}

int cp_mixed_pop_control(afqmc_engine *e)
{
    CpMixedState *m = e->cpm;
    CM(cp_mixed_pop_weights(e));
    launch_pop_comb(e->W, e->weight, nullptr, e->seed, e->counter, e->number, e->table,
                    e->status + e->W, e->stream);
    g_launch_count++;
    gather_kernel<<<e->W, 256, 0, e->stream>>>(e->W, m->ws, e->table, m->hi, m->lo, e->logw);
    return engine_check_launch();
}
