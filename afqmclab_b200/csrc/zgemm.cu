// Batched complex FP64 GEMM (plain form).  B200 has no FP64 tcgen05 path, and
// its FP64 DMMA rate equals its DFMA rate, so this kernel register-tiles the
// complex multiply-adds on the FP64 pipe: each thread owns a TMxTN block of
// the output, operand tiles are staged through shared memory (double
// buffered), and column-major stores are coalesced along the row index.
#include "zgemm.cuh"

#include <cuda_bf16.h>

#include <atomic>
#include <map>
#include <mutex>
#include <tuple>

extern std::atomic<long long> g_launch_count;

namespace {

constexpr int BK = 8;

template <int OP>
__device__ __forceinline__ zd load_op(const void *P, long long ld, int i, int l, int kind,
                                      long long plane)
{
    // element (i, l) of op(P) where P is column-major with leading dimension ld
    long long idx = (OP == OP_N) ? (long long)i + (long long)l * ld : (long long)l + (long long)i * ld;
    zd v;
    if (kind == ST_R64) v = make_double2(__ldg((const double *)P + idx), 0.0);
    else if (kind == ST_C32P) v = make_double2((double)__ldg((const float *)P + idx),
                                               (double)__ldg((const float *)P + plane + idx));
    else v = __ldg((const zd *)P + idx);
    if (OP == OP_C) v.y = -v.y;
    return v;
}

// REAL: 0 both operands complex (a real operand is loaded as complex with a
// zero imaginary part), 1 A real, 2 B real, 3 both real; a real operand
// takes one FP64 multiply-add per real product instead of the complex four.
template <int BM, int BN, int TM, int TN, int OPA, int OPB, int REAL>
__global__ void __launch_bounds__((BM / TM) * (BN / TN), TM * TN > 16 ? 1 : 2)
zgemm_kernel(ZGemmArgs a)
{
    constexpr int NTX = BM / TM;           // threads along rows
    constexpr int NT = (BM / TM) * (BN / TN);
    const int b = blockIdx.z;
    if (a.mask && a.mask[b] == 0) return;
    if (a.skip && a.skip[b] != 0) return;
    const int tileM = blockIdx.x * BM, tileN = blockIdx.y * BN;
    if (tileM >= a.m || tileN >= a.n) return;
    if (a.lower && tileM + BM <= tileN) return;

    const size_t esA = a.a_real == ST_R64 ? sizeof(double) : a.a_real == ST_C32P ? sizeof(float) : sizeof(zd);
    const size_t esB = a.b_real == ST_R64 ? sizeof(double) : a.b_real == ST_C32P ? sizeof(float) : sizeof(zd);
    const char *Ab = (const char *)a.A + (size_t)b * a.strideA * esA;
    const char *Bb = (const char *)a.B + (size_t)b * a.strideB * esB;
    zd *Cb = a.C ? a.C + (size_t)b * a.strideC : nullptr;

    __shared__ zd As[2][BK][BM];
    __shared__ zd Bs[2][BK][BN];

    const int tid = threadIdx.x;
    // a warp covers 8 row and 4 column positions of the 16 x 16 thread grid,
    // so each operand fragment load touches 8 (A) or 4 (B) distinct 16-byte
    // words: one shared-memory wavefront each
    static_assert(NTX == 16 && NT == 256, "16 x 16 thread grid");
    const int warp = tid >> 5, lane = tid & 31;
    const int tx = (warp & 1) * 8 + (lane & 7), ty = (warp >> 1) * 4 + (lane >> 3);

    zd acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = make_double2(0.0, 0.0);

    // real-operand forms (half the multiply-adds per K-step) fetch the next
    // K-step's tiles into registers before this step's products and store them
    // to shared memory after, so the global loads' latency overlaps the
    // multiply-adds; the complex form has the registers for neither and
    // stores them before its products
    constexpr bool STAGE = REAL != 0;
    constexpr int LA = (BM * BK + NT - 1) / NT, LB = (BN * BK + NT - 1) / NT;
    zd pa[LA], pb[LB];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int t = 0; t < LA; ++t) {
            const int e = tid + t * NT;
            int i, l;
            if (OPA == OP_N) { i = e % BM; l = e / BM; } else { l = e % BK; i = e / BK; }
            const int gi = tileM + i, gl = k0 + l;
            zd v = make_double2(0.0, 0.0);
            if (e < BM * BK && gi < a.m && gl < a.k) v = load_op<OPA>(Ab, a.lda, gi, gl, a.a_real, a.planeA);
            pa[t] = v;
        }
#pragma unroll
        for (int t = 0; t < LB; ++t) {
            const int e = tid + t * NT;
            int l, j;
            if (OPB == OP_N) { l = e % BK; j = e / BK; } else { j = e % BN; l = e / BN; }
            const int gl = k0 + l, gj = tileN + j;
            zd v = make_double2(0.0, 0.0);
            if (e < BN * BK && gl < a.k && gj < a.n) v = load_op<OPB>(Bb, a.ldb, gl, gj, a.b_real, a.planeB);
            pb[t] = v;
        }
    };
    auto commit = [&](int buf) {
#pragma unroll
        for (int t = 0; t < LA; ++t) {
            const int e = tid + t * NT;
            int i, l;
            if (OPA == OP_N) { i = e % BM; l = e / BM; } else { l = e % BK; i = e / BK; }
            if (e < BM * BK) As[buf][l][i] = pa[t];
        }
#pragma unroll
        for (int t = 0; t < LB; ++t) {
            const int e = tid + t * NT;
            int l, j;
            if (OPB == OP_N) { l = e % BK; j = e / BK; } else { j = e % BN; l = e / BN; }
            if (e < BN * BK) Bs[buf][l][j] = pb[t];
        }
    };

    auto load_tiles = [&](int buf, int k0) {
        for (int e = tid; e < BM * BK; e += NT) {
            int i, l;
            if (OPA == OP_N) { i = e % BM; l = e / BM; } else { l = e % BK; i = e / BK; }
            int gi = tileM + i, gl = k0 + l;
            zd v = make_double2(0.0, 0.0);
            if (gi < a.m && gl < a.k) v = load_op<OPA>(Ab, a.lda, gi, gl, a.a_real, a.planeA);
            As[buf][l][i] = v;
        }
        for (int e = tid; e < BN * BK; e += NT) {
            int l, j;
            if (OPB == OP_N) { l = e % BK; j = e / BK; } else { j = e % BN; l = e / BN; }
            int gl = k0 + l, gj = tileN + j;
            zd v = make_double2(0.0, 0.0);
            if (gl < a.k && gj < a.n) v = load_op<OPB>(Bb, a.ldb, gl, gj, a.b_real, a.planeB);
            Bs[buf][l][j] = v;
        }
    };

    int buf = 0;
    if (STAGE) {
        fetch(0);
        commit(0);
    } else {
        load_tiles(0, 0);
    }
    __syncthreads();
    for (int k0 = 0; k0 < a.k; k0 += BK) {
        const bool more = k0 + BK < a.k;
        if (STAGE && more) fetch(k0 + BK);
        if (!STAGE && more) load_tiles(buf ^ 1, k0 + BK);
#pragma unroll
        for (int l = 0; l < BK; ++l) {
            zd ra[TM], rb[TN];
#pragma unroll
            for (int i = 0; i < TM; ++i) ra[i] = As[buf][l][tx + i * NTX];
#pragma unroll
            for (int j = 0; j < TN; ++j) rb[j] = Bs[buf][l][ty + j * (BN / TN)];
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) {
                    if (REAL == 0) {
                        zfma(acc[i][j], ra[i], rb[j]);
                    } else if (REAL == 1) {
                        acc[i][j].x = fma(ra[i].x, rb[j].x, acc[i][j].x);
                        acc[i][j].y = fma(ra[i].x, rb[j].y, acc[i][j].y);
                    } else if (REAL == 2) {
                        acc[i][j].x = fma(ra[i].x, rb[j].x, acc[i][j].x);
                        acc[i][j].y = fma(ra[i].y, rb[j].x, acc[i][j].y);
                    } else {
                        acc[i][j].x = fma(ra[i].x, rb[j].x, acc[i][j].x);
                    }
                }
        }
        if (STAGE && more) commit(buf ^ 1);
        __syncthreads();
        buf ^= 1;
    }

    const bool beta0 = (a.beta.x == 0.0 && a.beta.y == 0.0);
#pragma unroll
    for (int j = 0; j < TN; ++j) {
        int gj = tileN + ty + j * (BN / TN);
        if (gj >= a.n) continue;
#pragma unroll
        for (int i = 0; i < TM; ++i) {
            int gi = tileM + tx + i * NTX;
            if (gi >= a.m) continue;
            zd v = zmul(a.alpha, acc[i][j]);
            if (Cb) {
                zd *c = Cb + gi + (size_t)gj * a.ldc;
                if (!beta0) zfma(v, a.beta, *c);
                *c = v;
            }
            if (a.outMode & OUT_BF16P) {
                __nv_bfloat16 *c2 = (__nv_bfloat16 *)a.C2 + (size_t)b * a.strideC2 + gi + (size_t)gj * a.ldc2;
                c2[0] = __double2bfloat16(v.x);
                c2[a.plane2] = __double2bfloat16(v.y);
            }
            if (a.outMode & OUT_C32P) {
                float *c3 = a.C3 + (size_t)b * a.strideC3 + gi + (size_t)gj * a.ldc3;
                c3[0] = (float)v.x;
                c3[a.plane3] = (float)v.y;
            }
        }
    }
}

template <int BM, int BN, int TM, int TN, int OPA, int OPB, int REAL = 0>
cudaError_t launch3(const ZGemmArgs &a, cudaStream_t s)
{
    dim3 grid((a.m + BM - 1) / BM, (a.n + BN - 1) / BN, a.batch);
    dim3 block((BM / TM) * (BN / TN));
    zgemm_kernel<BM, BN, TM, TN, OPA, OPB, REAL><<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

template <int BM, int BN, int TM, int TN, int OPA, int OPB>
cudaError_t launch_real(const ZGemmArgs &a, cudaStream_t s)
{
    const int real = (a.a_real == ST_R64 ? 1 : 0) | (a.b_real == ST_R64 ? 2 : 0);
    if (real == 1) return launch3<BM, BN, TM, TN, OPA, OPB, 1>(a, s);
    if (real == 2) return launch3<BM, BN, TM, TN, OPA, OPB, 2>(a, s);
    if (real == 3) return launch3<BM, BN, TM, TN, OPA, OPB, 3>(a, s);
    return launch3<BM, BN, TM, TN, OPA, OPB, 0>(a, s);
}

template <int BM, int BN, int TM, int TN>
cudaError_t launch2(const ZGemmArgs &a, cudaStream_t s)
{
    // the operator pairs that real operands come with take the real forms
    if (a.opA == OP_N && a.opB == OP_N) return launch_real<BM, BN, TM, TN, OP_N, OP_N>(a, s);
    if (a.opA == OP_N && a.opB == OP_T) return launch_real<BM, BN, TM, TN, OP_N, OP_T>(a, s);
    if (a.opA == OP_C && a.opB == OP_N) return launch_real<BM, BN, TM, TN, OP_C, OP_N>(a, s);
    if (a.opA == OP_T && a.opB == OP_N) return launch_real<BM, BN, TM, TN, OP_T, OP_N>(a, s);
#define ZG_CASE(OA, OB) \
    if (a.opA == OA && a.opB == OB) return launch3<BM, BN, TM, TN, OA, OB>(a, s);
    ZG_CASE(OP_N, OP_N) ZG_CASE(OP_N, OP_T) ZG_CASE(OP_N, OP_C)
    ZG_CASE(OP_T, OP_N) ZG_CASE(OP_T, OP_T) ZG_CASE(OP_T, OP_C)
    ZG_CASE(OP_C, OP_N) ZG_CASE(OP_C, OP_T) ZG_CASE(OP_C, OP_C)
#undef ZG_CASE
    return cudaErrorInvalidValue;
}

}  // namespace

// ----------------------------------------------------------- autotuner
// Candidate tile shapes; the default rule picks one by size, the autotuner
// (when enabled) times every candidate once per problem shape and keeps the
// fastest.  Timing runs are synchronous, so shapes are tuned on first use
// outside stream capture; captured launches reuse the cached choice.
namespace {

constexpr int NCAND = 5;

int real_form(const ZGemmArgs &a)
{
    if (a.opA != OP_N || (a.opB != OP_N && a.opB != OP_T)) return 0;
    return (a.a_real == ST_R64 ? 1 : 0) | (a.b_real == ST_R64 ? 2 : 0);
}

// Wide thread tiles for one real operand: a thread's A (B) values cost four
// shared-memory wavefronts per complex and two per real value and K-column,
// so 4 x 8 (complex A, real B) and 8 x 4 (real A, complex B) give 64 FP64
// FMAs per 32 wavefronts, twice the 4 x 4 form's 32 per 24.
cudaError_t launch_wide_real(const ZGemmArgs &a, cudaStream_t s)
{
    const int real = real_form(a);
    if (real == 2) {
        if (a.opB == OP_N) return launch3<64, 128, 4, 8, OP_N, OP_N, 2>(a, s);
        return launch3<64, 128, 4, 8, OP_N, OP_T, 2>(a, s);
    }
    if (real == 1) {
        if (a.opB == OP_N) return launch3<128, 64, 8, 4, OP_N, OP_N, 1>(a, s);
        return launch3<128, 64, 8, 4, OP_N, OP_T, 1>(a, s);
    }
    return launch2<64, 64, 4, 4>(a, s);
}

cudaError_t launch_cand(int c, const ZGemmArgs &a, cudaStream_t s)
{
    switch (c) {
    case 0: return launch2<32, 32, 2, 2>(a, s);
    case 1: return launch2<32, 64, 2, 4>(a, s);
    case 2: return launch2<64, 64, 4, 4>(a, s);
    case 3: return launch2<128, 32, 8, 2>(a, s);
    default: return launch_wide_real(a, s);
    }
}

int default_cand(const ZGemmArgs &a)
{
    if (a.m <= 32 && a.n <= 32) return 0;
    if (a.m <= 32) return 1;
    const int real = real_form(a);
    if ((real == 1 || real == 2) && a.m >= 128 && a.n >= 128) return 4;
    return 2;
}

std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int, int, int, int>, int> g_tuned;
std::atomic<int> g_autotune{0};

}  // namespace

void zgemm_set_autotune(int on) { g_autotune = on; }

int zgemm_tuned_choice(const ZGemmArgs &a)
{
    auto key = std::make_tuple(a.m, a.n, a.k, a.opA, a.opB, a.a_real, a.b_real, a.batch);
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tuned.find(key);
    return it == g_tuned.end() ? -1 : it->second;
}

cudaError_t zgemm_batched(const ZGemmArgs &a, cudaStream_t stream)
{
    g_launch_count++;
    if (a.m <= 0 || a.n <= 0 || a.batch <= 0) return cudaSuccess;
    if (a.k <= 0) return cudaErrorInvalidValue;
    const auto key = std::make_tuple(a.m, a.n, a.k, a.opA, a.opB, a.a_real, a.b_real, a.batch);
    int choice = -1;
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) choice = it->second;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(stream, &cs);
    if (choice < 0 && g_autotune && cs == cudaStreamCaptureStatusNone && a.beta.x == 0.0 &&
        a.beta.y == 0.0) {
        // time every candidate (the output is simply rewritten each time)
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        float best = 1e30f;
        for (int c = 0; c < NCAND; ++c) {
            if (launch_cand(c, a, stream) != cudaSuccess) { cudaGetLastError(); continue; }
            cudaEventRecord(e0, stream);
            for (int r = 0; r < 3; ++r) launch_cand(c, a, stream);
            cudaEventRecord(e1, stream);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) { best = ms; choice = c; }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tuned[key] = choice;
    }
    if (choice < 0) choice = default_cand(a);
    return launch_cand(choice, a, stream);
}
