// AFQMC walker-step engine: host-side sequencing of the sm_100a kernels and
// the extern "C" entry points declared in include/afqmc_b200.h.
//
// The population (W walkers) lives in device memory as one strided batch:
// walker w's n x ncol column-major matrix starts at w * n * ncol, its log
// weight, alive flag and random-stream offset sit in per-walker arrays.
// The step order is the reference drivers' per-walker loop body
// (tutorials/afqmcConstraintPath/source/afqmcConstraintPathProjection.cpp:37-74,
//  tutorials/afqmcPhaseless/source/afqmcPhaselessProjection.cpp:75-121),
// executed population-wide, kernel by kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/afqmc_b200.h"
#include "common.cuh"
#include "cp_mixed.cuh"
#include "engine_internal.cuh"
#include "exchange_f64.cuh"
#include "mixed.cuh"
#include "tc_gemm.cuh"
#include "walker_kernels.cuh"
#include "zgemm.cuh"

#include <atomic>
#include <mutex>
extern std::atomic<long long> g_launch_count;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

#define CUDA_TRY(expr)                                                                        \
    do {                                                                                      \
        cudaError_t _e = (expr);                                                              \
        if (_e != cudaSuccess)                                                                \
            return fail(AFQMC_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
    } while (0)

#define TRY(expr)                   \
    do {                            \
        int _r = (expr);            \
        if (_r != AFQMC_OK) return _r; \
    } while (0)

constexpr int TAYLOR_KMAX = 30;
constexpr int TAYLOR_BASE = 3;          // baseTaylorOrder default (logHop2isSD2isOperation.h:31)
constexpr double TAYLOR_ACC = 1e-10;    // accuracy default

typedef std::complex<double> cd;

// ------------------------------------------------ NiupNidn constants (host)
// The Hubbard-Stratonovich coupling gamma solves cosh(gamma) = e^y
// (solveCoshxEqExpy) or cos(gamma) = e^y (solveCosxEqExpy), and the
// field-dependent on-site factor is the exponential of a Hermitian 2x2 matrix
// (exp2by2Matrix), common/mathHao/source/simple_fun.cpp:7-91.  The root is
// either purely real or purely imaginary; the reference's choice of branch
// (negative root for the cosh form, e^y > 1; negative imaginary root
// otherwise) fixes the sign convention of the sampled fields, so it is kept.
cd solve_cosh_eq_exp(double y)
{
    const double ey = std::exp(y);
    if (ey >= 1.0) return cd(-std::acosh(ey), 0.0);   // cosh(-a) = e^y, a >= 0
    return cd(0.0, -std::acos(ey));                    // cosh(-i b) = cos(b) = e^y
}
cd solve_cos_eq_exp(double y)
{
    const double ey = std::exp(y);
    if (ey <= 1.0) return cd(std::acos(ey), 0.0);      // cos(a) = e^y, a in [0, pi/2]
    return cd(0.0, -std::acosh(ey));                   // cos(-i b) = cosh(b) = e^y
}
// exp(H) for H = [[a, conj(c)], [c, b]] (a, b real): with m = (a+b)/2 and
// r = sqrt(((a-b)/2)^2 + |c|^2), (H - m I)^2 = r^2 I, so
//   exp(H) = e^m [cosh(r) I + sinh(r)/r (H - m I)].
// On return a, b hold the diagonal and c the lower off-diagonal entry.
void exp2by2(double &a, double &b, cd &c)
{
    const double m = 0.5 * (a + b), h = 0.5 * (a - b);
    const double r = std::sqrt(h * h + std::norm(c));
    const double em = std::exp(m);
    // sinh(r)/r, by its series where r is small enough for the series to be exact in FP64
    const double shr = (r < 1e-4) ? 1.0 + r * r / 6.0 : std::sinh(r) / r;
    const double ch = std::cosh(r);
    a = em * (ch + shr * h);
    b = em * (ch - shr * h);
    c = em * shr * c;
}

zd tozd(cd z) { return make_double2(z.real(), z.imag()); }

// One device int per device for the error word of the stand-alone
// tensor-core entry points (allocated the first time each device needs it).
int device_error_word(int **out)
{
    static int *words[64] = {};
    static std::mutex mu;
    int dev = 0;
    cudaError_t r = cudaGetDevice(&dev);
    if (r != cudaSuccess) return fail(AFQMC_ERR_CUDA, cudaGetErrorString(r));
    if (dev < 0 || dev >= 64) return fail(AFQMC_ERR_UNSUPPORTED, "device index above 63");
    std::lock_guard<std::mutex> lock(mu);
    if (!words[dev]) {
        r = cudaMalloc(&words[dev], sizeof(int));
        if (r != cudaSuccess) { words[dev] = nullptr; return fail(AFQMC_ERR_CUDA, cudaGetErrorString(r)); }
    }
    *out = words[dev];
    return AFQMC_OK;
}

}  // namespace

// Back-propagation state of a constrained-path engine
// (tutorials/afqmcConstraintPathBP: afqmcConstraintPath.h members
// walkerBackup, walkerBPMeasure, twoBodyAuxBackup, twoBodyAuxBPMeasure,
// tablePerThreadBackup, isBP, BPIndex).  Field records are [step][walker][site]
// ints, validity flags [step][walker] (the walker was sampled at that step),
// tables [step][walker]; tableValid[i] says a population control ran at step i.
struct BPState {
    int steps = 0, skip = 0, index = 0, cap = 0;
    bool active = false;
    int *aux = nullptr, *auxMeas = nullptr, *valid = nullptr, *validMeas = nullptr, *table = nullptr;
    int *ones = nullptr;
    std::vector<char> tableValid;
    zd *wfBackup = nullptr, *logwBackup = nullptr, *wfMeas = nullptr, *logwMeas = nullptr;
    zd *left = nullptr, *leftTmp = nullptr, *right = nullptr, *logwL = nullptr, *logovBP = nullptr;
};

namespace {

template <class T>
int dalloc(afqmc_engine *e, T **p, size_t count)
{
    if (count == 0) count = 1;
    void *q = nullptr;
    cudaError_t r = cudaMalloc(&q, count * sizeof(T));
    if (r != cudaSuccess)
        return fail(AFQMC_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(r));
    r = cudaMemset(q, 0, count * sizeof(T));
    if (r != cudaSuccess) return fail(AFQMC_ERR_CUDA, cudaGetErrorString(r));
    e->allocs.push_back(q);
    *p = (T *)q;
    return AFQMC_OK;
}

template <class T>
int dupload(afqmc_engine *e, T **p, const void *host, size_t count)
{
    TRY(dalloc(e, p, count));
    if (host) CUDA_TRY(cudaMemcpy(*p, host, count * sizeof(T), cudaMemcpyHostToDevice));
    return AFQMC_OK;
}

int check_launch()
{
    cudaError_t r = cudaGetLastError();
    if (r != cudaSuccess) return fail(AFQMC_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(r));
    return AFQMC_OK;
}

int gemm(const ZGemmArgs &a, cudaStream_t s)
{
    cudaError_t r = zgemm_batched(a, s);
    if (r != cudaSuccess) return fail(AFQMC_ERR_CUDA, std::string("zgemm: ") + cudaGetErrorString(r));
    return AFQMC_OK;
}

// common allocations for both engines
int alloc_population(afqmc_engine *e)
{
    const int W = e->W;
    e->wsize = (long long)e->n * e->ncol;
    TRY(dalloc(e, &e->wf, (size_t)W * e->wsize));
    TRY(dalloc(e, &e->wfTmp, (size_t)W * e->wsize));
    TRY(dalloc(e, &e->term[0], (size_t)W * e->wsize));
    TRY(dalloc(e, &e->term[1], (size_t)W * e->wsize));
    TRY(dalloc(e, &e->logw, W));
    TRY(dalloc(e, &e->logov, W));
    TRY(dalloc(e, &e->S, (size_t)W * e->bl.sStride));
    TRY(dalloc(e, &e->Sinv, (size_t)W * e->bl.sStride));
    TRY(dalloc(e, &e->thetaT, (size_t)W * e->bl.tStride));
    TRY(dalloc(e, &e->alive, W));
    TRY(dalloc(e, &e->surv, W));
    TRY(dalloc(e, &e->status, W + 1));
    TRY(dalloc(e, &e->done, W));
    TRY(dalloc(e, &e->order, W));
    TRY(dalloc(e, &e->table, W));
    TRY(dalloc(e, &e->number, W));
    TRY(dalloc(e, &e->counter, 1));
    TRY(dalloc(e, &e->offs, W));
    TRY(dalloc(e, &e->weight, W));
    TRY(dalloc(e, &e->tstats, 4));
    long long init[4] = {0, 0, 1LL << 40, 0};
    CUDA_TRY(cudaMemcpy(e->tstats, init, sizeof(init), cudaMemcpyHostToDevice));
    TRY(dalloc(e, &e->acc, 8));
    TRY(dalloc(e, &e->eloc, W));
    TRY(dalloc(e, &e->den, W));
    TRY(dalloc(e, &e->parts, (size_t)3 * W));
    CUDA_TRY(cudaStreamCreateWithFlags(&e->own, cudaStreamNonBlocking));
    e->stream = e->own;
    return AFQMC_OK;
}

void set_blocks(afqmc_engine *e)
{
    Blocks &b = e->bl;
    if (e->kind == KIND_CP) {
        b.nblk = 1; b.Ns[0] = e->ncol; b.Ns[1] = 0;
        b.sOff[0] = 0; b.tOff[0] = 0; b.sOff[1] = 0; b.tOff[1] = 0;
        b.sStride = (long long)e->ncol * e->ncol;
        b.tStride = (long long)e->ncol * e->n;
    } else {
        b.nblk = e->ndn > 0 ? 2 : 1;
        b.Ns[0] = e->nup; b.Ns[1] = e->ndn;
        b.sOff[0] = 0; b.sOff[1] = (long long)e->nup * e->nup;
        b.tOff[0] = 0; b.tOff[1] = (long long)e->nup * e->n;
        b.sStride = (long long)e->nup * e->nup + (long long)e->ndn * e->ndn;
        b.tStride = (long long)(e->nup + e->ndn) * e->n;
    }
}

// ---------------------------------------------------------------- pieces
// S_b = phiT_b^H phi (SDSDOperation.cpp:154-164, gmm 'C')
// The spin blocks the FP64 step computes: block 0 alone (counted twice) for a
// closed-shell trial, both otherwise.
const Blocks &fbl(const afqmc_engine *e)
{
    return (e->exf && e->exf->restricted) ? e->exf->bl1 : e->bl;
}

int overlap_gemm(afqmc_engine *e, const zd *wf, const int *mask, const Blocks &bl)
{
    for (int b = 0; b < bl.nblk; ++b) {
        int Ns = bl.Ns[b];
        if (Ns == 0) continue;
        ZGemmArgs g;
        g.m = Ns; g.n = Ns; g.k = e->n;
        g.opA = OP_C; g.opB = OP_N;
        g.A = e->phiT[b]; g.lda = e->n; g.strideA = 0;
        g.B = wf; g.ldb = e->n; g.strideB = e->wsize;
        g.C = e->S + bl.sOff[b]; g.ldc = Ns; g.strideC = bl.sStride;
        g.batch = e->W; g.mask = mask;
        TRY(gemm(g, e->stream));
    }
    return AFQMC_OK;
}

// thetaT_b = (S_b^{-1})^T phi_b^T  (zgetrs 'T', SDSDOperation.cpp:166-173)
int theta_gemm(afqmc_engine *e, const zd *wf, const int *mask, const Blocks &bl)
{
    for (int b = 0; b < bl.nblk; ++b) {
        int Ns = bl.Ns[b];
        if (Ns == 0) continue;
        ZGemmArgs g;
        g.m = Ns; g.n = e->n; g.k = Ns;
        g.opA = OP_T; g.opB = OP_T;
        g.A = e->Sinv + bl.sOff[b]; g.lda = Ns; g.strideA = bl.sStride;
        g.B = wf; g.ldb = e->n; g.strideB = e->wsize;
        g.C = e->thetaT + bl.tOff[b]; g.ldc = Ns; g.strideC = bl.tStride;
        g.batch = e->W; g.mask = mask;
        TRY(gemm(g, e->stream));
    }
    return AFQMC_OK;
}

// phaseless xbar = A^T thetaT for every walker (calculateCholeskyBg, :237-256);
// a closed-shell block list sums block 0's rows and doubles them
int xbar_gemm(afqmc_engine *e, const Blocks &bl)
{
    // real half-rotated vectors: the exchange's real X (K x G per block) in
    // place of the complex-typed Aall, one real x complex product per block
    if (e->exf && e->exf->gemm) return exf64_force(e, bl);
    ZGemmArgs g;
    g.m = e->G; g.n = e->W; g.k = (int)(bl.mult == 2 ? bl.tOff[1] : e->Ktot);
    g.alpha = make_double2((double)bl.mult, 0.0);
    g.opA = OP_T; g.opB = OP_N;
    g.A = e->Aall; g.lda = e->Ktot;
    g.B = e->thetaT; g.ldb = e->bl.tStride;
    g.C = e->xbar; g.ldc = e->G;
    g.batch = 1;
    return gemm(g, e->stream);
}

// dst = exp(M) src via the dynamicOrder Taylor series
// (LogHop2isSD2isOperation::applyToRight, logHop2isSD2isOperation.cpp:38-45,159-195).
// Mstride = 0 for a shared matrix (one-body LogHop2is), n*n per walker otherwise.
int taylor_apply(afqmc_engine *e, const zd *M, long long Mstride, const zd *src, zd *dst,
                 const int *mask, bool stats)
{
    const int W = e->W;
    launch_copy_masked(W, e->wsize, src, dst, mask, e->stream);
    CUDA_TRY(cudaMemsetAsync(e->done, 0, sizeof(int) * W, e->stream));
    const zd *old = src;
    for (int k = 1; k <= TAYLOR_KMAX; ++k) {
        zd *nw = e->term[(k - 1) & 1];
        ZGemmArgs g;
        g.m = e->n; g.n = e->ncol; g.k = e->n;
        g.A = M; g.lda = e->n; g.strideA = Mstride;
        g.B = old; g.ldb = e->n; g.strideB = e->wsize;
        g.C = nw; g.ldc = e->n; g.strideC = e->wsize;
        g.alpha = make_double2(1.0 / k, 0.0);
        g.batch = W; g.mask = mask; g.skip = e->done;
        TRY(gemm(g, e->stream));
        launch_taylor_accum(W, e->wsize, nw, dst, mask, e->done, e->order, k, TAYLOR_BASE + 1,
                            TAYLOR_ACC, k == TAYLOR_KMAX ? 1 : 0, e->status, e->stream);
        old = nw;
    }
    if (stats) launch_taylor_stats(W, mask, e->order, e->tstats, e->stream);
    return check_launch();
}

// one-body operator `which` applied to src -> dst for masked walkers
int one_body(afqmc_engine *e, int which, const zd *src, zd *dst, const int *mask)
{
    if (e->useLog && e->kind == KIND_PL) {
        const zd *Mx = which == 0 ? e->logK : e->expK[which];
        return taylor_apply(e, Mx, 0, src, dst, mask, false);
    }
    ZGemmArgs g;
    g.m = e->n; g.n = e->ncol; g.k = e->n;
    g.A = e->expK[which]; g.lda = e->n; g.strideA = 0;
    g.B = src; g.ldb = e->n; g.strideB = e->wsize;
    g.C = dst; g.ldc = e->n; g.strideC = e->wsize;
    g.batch = e->W; g.mask = mask;
    return gemm(g, e->stream);
}

zd one_body_logw(afqmc_engine *e, int which)
{
    if (e->useLog && e->kind == KIND_PL && which == 0) return e->logKLogw;
    return e->expLogw[which];
}

// --------------------------------------------------- projectExpMinusDtKExpMinusDtV
int project_dtk_dtv(afqmc_engine *e)
{
    const int W = e->W;
    cudaStream_t s = e->stream;
    if (e->precision == AFQMC_MIXED) return mixed_project_dtk_dtv(e);
    const bool needTheta = (e->forceType == AFQMC_DYNAMIC_FORCE);
    // overlap, log-determinant, first cos projection
    const Blocks &bl = fbl(e);
    { PHASE(AFQMC_PH_OVERLAP); TRY(overlap_gemm(e, e->wf, e->alive, bl)); }
    {
        PHASE(AFQMC_PH_LU);
        launch_lu_logdet_inverse(W, bl, e->S, e->Sinv, e->alive, e->logw, make_double2(0, 0),
                                 e->logwT, e->logov, e->alive, e->surv, e->logw, nullptr, e->status,
                                 LU_PROJECT, needTheta, s);
        TRY(check_launch());
    }
    if (needTheta) { PHASE(AFQMC_PH_THETA); TRY(theta_gemm(e, e->wf, e->surv, bl)); }
    zd hop = one_body_logw(e, 0);
    if (e->kind == KIND_CP) {
        if (needTheta) {
            PHASE(AFQMC_PH_FORCE);
            launch_cp_force(W, e->hd, e->thetaT, e->bl.tStride, e->surv, e->forceCP, s);
        }
        {
            PHASE(AFQMC_PH_SAMPLE);
            launch_rng_scan(W, e->surv, e->L, e->counter, e->offs, s);
            BPState *bp = (e->bp && e->bp->active) ? e->bp : nullptr;
            // back-propagation: this step's fields and which walkers drew them
            // (twoBodyAuxBackup[i][BPIndex], afqmcConstraintPathProjection.cpp:73)
            int *auxOut = bp ? bp->aux + (size_t)bp->index * W * e->L : nullptr;
            launch_cp_sample_apply(W, e->hd, e->forceCP, e->surv, e->offs, e->seed, e->wf, e->wfTmp,
                                   e->logw, e->dt * e->ET, hop, auxOut, s);
            TRY(check_launch());
            if (bp)
                CUDA_TRY(cudaMemcpyAsync(bp->valid + (size_t)bp->index * W, e->surv, sizeof(int) * W,
                                         cudaMemcpyDeviceToDevice, s));
        }
        { PHASE(AFQMC_PH_ONEBODY); TRY(one_body(e, 0, e->wfTmp, e->wf, e->surv)); }
    } else {
        if (needTheta) { PHASE(AFQMC_PH_FORCE); TRY(xbar_gemm(e, bl)); }
        {
            PHASE(AFQMC_PH_SAMPLE);
            launch_rng_scan(W, e->surv, 2 * e->G, e->counter, e->offs, s);
            launch_pl_sample(W, e->cdv, e->xbar, e->surv, e->surv, e->alive, e->offs, e->seed,
                             e->aux, e->forcePL, e->logw, e->dt * e->ET, hop, s);
            TRY(check_launch());
        }
        {
            // M = sqrt(-dt) sum_g aux_g L_g  (choleskyReal.cpp:160-169), all walkers in one GEMM
            PHASE(AFQMC_PH_MBUILD);
            ZGemmArgs g;
            g.m = e->n * e->n; g.n = W; g.k = e->G;
            g.a_real = 1;
            g.A = e->chol; g.lda = (long long)e->n * e->n;
            g.B = e->aux; g.ldb = e->G;
            g.C = e->M; g.ldc = (long long)e->n * e->n;
            g.alpha = make_double2(0.0, e->cdv.sqrtMinusDtIm);
            TRY(gemm(g, s));
        }
        {
            PHASE(AFQMC_PH_TAYLOR);
            TRY(taylor_apply(e, e->M, (long long)e->n * e->n, e->wf, e->wfTmp, e->surv, true));
        }
        { PHASE(AFQMC_PH_ONEBODY); TRY(one_body(e, 0, e->wfTmp, e->wf, e->surv)); }
    }
    return check_launch();
}

int modify_gm(afqmc_engine *e)
{
    PHASE(AFQMC_PH_STABILIZE);
    if (e->precision == AFQMC_MIXED) return mixed_modify_gm(e);
    launch_mgs(e->W, e->n, e->ncol, e->nup, e->ndn, e->kind == KIND_PL ? 1 : 0, e->wf, e->logw,
               e->alive, e->status, e->stream);
    return check_launch();
}

int pop_control(afqmc_engine *e)
{
    PHASE(AFQMC_PH_POPCONTROL);
    if (e->precision == AFQMC_MIXED) return mixed_pop_control(e);
    TRY(overlap_gemm(e, e->wf, e->alive, fbl(e)));
    launch_lu_logdet_inverse(e->W, fbl(e), e->S, nullptr, e->alive, e->logw, make_double2(0, 0),
                             e->logwT, e->logov, e->alive, nullptr, e->logw, e->weight, e->status,
                             LU_POPWEIGHT, false, e->stream);
    launch_pop_comb(e->W, e->weight, nullptr, e->seed, e->counter, e->number, e->table,
                    e->status + e->W, e->stream);
    launch_pop_gather(e->W, e->wsize, e->table, e->wf, e->logw, e->stream);
    if (e->bp && e->bp->active) {
        // tablePerThreadBackup[BPIndex] (afqmcConstraintPathProjection.cpp:161-170)
        BPState *bp = e->bp;
        CUDA_TRY(cudaMemcpyAsync(bp->table + (size_t)bp->index * e->W, e->table, sizeof(int) * e->W,
                                 cudaMemcpyDeviceToDevice, e->stream));
        bp->tableValid[bp->index] = 1;
    }
    return check_launch();
}

int project_one_step_direct(afqmc_engine *e)
{
    TRY(project_dtk_dtv(e));
    e->mgsIndex++;
    if (e->mgsIndex == e->mgsStep) { TRY(modify_gm(e)); e->mgsIndex = 0; }
    e->popIndex++;
    if (e->popIndex == e->popStep) { TRY(pop_control(e)); e->popIndex = 0; }
    return AFQMC_OK;
}

void drop_graphs(afqmc_engine *e)
{
    for (auto &g : e->graphExec)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    e->graphWarm = false;
    e->measWarm = false;
}

// Records the kernels that `body` issues on the engine stream into a graph.
// The launches issued while capturing are counted as the graph's kernel
// nodes and credited to the launch counter each time the graph is replayed.
template <class F>
int capture(afqmc_engine *e, cudaGraphExec_t *out, long long *kernels, F body)
{
    cudaGraph_t g = nullptr;
    CUDA_TRY(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    const long long c0 = g_launch_count.load();
    int r = body();
    *kernels = g_launch_count.load() - c0;
    g_launch_count -= *kernels;
    cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
    if (r != AFQMC_OK) { if (g) cudaGraphDestroy(g); return r; }
    if (ce != cudaSuccess) return fail(AFQMC_ERR_CUDA, std::string("stream capture: ") + cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return fail(AFQMC_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
    return AFQMC_OK;
}

// projectOneStep: with graphs on, the step's kernels (and the cadence
// operations due at this step) replay as one graph launch.  The first step
// runs directly so that every launcher's one-time setup happens outside
// capture; the profiler needs direct launches.
int project_one_step(afqmc_engine *e)
{
    if (e->bp && e->bp->active) {
        // recording a back-propagation window: direct launches (the record
        // offsets move every step), BPIndex++ after the step
        BPState *bp = e->bp;
        if (bp->index >= bp->steps)
            return fail(AFQMC_ERR_STATE, "back-propagation window is full: measure it first");
        bp->tableValid[bp->index] = 0;
        TRY(project_one_step_direct(e));
        bp->index++;
        return AFQMC_OK;
    }
    if (!e->useGraphs || e->prof || !e->graphWarm) {
        int r = project_one_step_direct(e);
        if (r == AFQMC_OK && e->useGraphs) e->graphWarm = true;
        return r;
    }
    const bool doMgs = (e->mgsIndex + 1 == e->mgsStep);
    const bool doPop = (e->popIndex + 1 == e->popStep);
    const int key = (doMgs ? 1 : 0) | (doPop ? 2 : 0);
    if (!e->graphExec[key]) {
        TRY(capture(e, &e->graphExec[key], &e->graphKernels[key], [&]() {
            TRY(project_dtk_dtv(e));
            if (doMgs) TRY(modify_gm(e));
            if (doPop) TRY(pop_control(e));
            return AFQMC_OK;
        }));
    }
    CUDA_TRY(cudaGraphLaunch(e->graphExec[key], e->stream));
    g_launch_count += e->graphKernels[key];
    e->mgsIndex = doMgs ? 0 : e->mgsIndex + 1;
    e->popIndex = doPop ? 0 : e->popIndex + 1;
    return AFQMC_OK;
}

int add_mixed_measurement_direct(afqmc_engine *e);

int add_mixed_measurement(afqmc_engine *e)
{
    if (!e->useGraphs || e->prof || !e->measWarm) {
        int r = add_mixed_measurement_direct(e);
        if (r == AFQMC_OK && e->useGraphs) e->measWarm = true;
        return r;
    }
    if (!e->graphExec[4])
        TRY(capture(e, &e->graphExec[4], &e->graphKernels[4], [&]() { return add_mixed_measurement_direct(e); }));
    CUDA_TRY(cudaGraphLaunch(e->graphExec[4], e->stream));
    g_launch_count += e->graphKernels[4];
    return AFQMC_OK;
}

int add_mixed_measurement_direct(afqmc_engine *e)
{
    if (e->precision == AFQMC_MIXED && e->kind == KIND_PL) return mixed_add_measurement(e);
    const int W = e->W;
    cudaStream_t s = e->stream;
    {
        PHASE(AFQMC_PH_MEASURE);
        // constrained-path mixed form: the half step and the overlap on the
        // tensor cores, the rest on an FP64 copy of the half-stepped walkers;
        // the FP64 form (or a complex half-step operator) runs both in FP64
        bool tcPrep = false;
        if (e->precision == AFQMC_MIXED) TRY(cp_mixed_measure_prep(e, &tcPrep));
        if (!tcPrep) {
            if (e->precision == AFQMC_MIXED) TRY(mixed_sync_to_fp64(e));
            TRY(one_body(e, 1, e->wf, e->wfTmp, e->alive));
            TRY(overlap_gemm(e, e->wfTmp, e->alive, fbl(e)));
        }
        launch_lu_logdet_inverse(W, fbl(e), e->S, e->Sinv, e->alive, e->logw, one_body_logw(e, 1),
                                 e->logwT, e->logov, e->alive, nullptr, nullptr, nullptr,
                                 e->status, LU_PLAIN, true, s);
        TRY(check_launch());
        TRY(theta_gemm(e, e->wfTmp, e->alive, fbl(e)));
    }
    if (e->kind == KIND_CP) {
        PHASE(AFQMC_PH_MEASURE);
        launch_cp_energy(W, e->hd, e->wfDaggerK, e->thetaT, e->bl.tStride, e->U, e->mu, e->hx,
                         e->hy, e->hz, e->alive, e->logov, e->eloc, e->den, e->parts, e->sites, s);
        launch_measure_reduce(W, e->alive, e->eloc, e->den, e->parts, 3, e->acc, 4 * e->L, e->sites,
                              nullptr, e->siteNum, nullptr, s);
        if (e->observe) {
            // G = conj(phiT) thetaT per walker (SDSDOperation::returnGreenMatrix), then
            // the observe estimator's sums
            ZGemmArgs g;
            g.m = e->n; g.n = e->n; g.k = e->ncol;
            g.A = e->phiTc; g.lda = e->n; g.strideA = 0;
            g.B = e->thetaT; g.ldb = e->ncol; g.strideB = e->bl.tStride;
            g.C = e->Gfull; g.ldc = e->n; g.strideC = (long long)e->n * e->n;
            g.batch = W; g.mask = e->alive;
            TRY(gemm(g, s));
            launch_cp_observe(W, e->L, e->Gfull, e->den, e->alive, e->obs, s);
        }
    } else {
        const Blocks &bl = fbl(e);
        const bool exg = e->exf && e->exf->gemm;
        { PHASE(AFQMC_PH_MEASURE); TRY(xbar_gemm(e, bl)); }
        {
            PHASE(AFQMC_PH_EXCHANGE);
            if (exg) {
                // real A: quadratic forms as FP64 GEMMs (exchange_f64.cu); exNum is
                // accumulated there, the per-walker totals go to the energy
                bool first = true;
                for (int b = 0; b < bl.nblk; ++b) {
                    if (bl.Ns[b] == 0) continue;
                    TRY(exf64_run(e, e->exf->blk[b], !first, bl.mult));
                    first = false;
                }
            } else if (launch_pl_exchange(W, e->n, e->G, e->bl, e->Aall, e->Ktot, e->thetaT, e->alive, e->ex, s)) {
                return fail(AFQMC_ERR_UNSUPPORTED, "exchange kernel supports at most 64 electrons per spin");
            }
        }
        {
            PHASE(AFQMC_PH_MEASURE);
            launch_pl_energy(W, e->G, e->Ktot, e->wfDaggerT, e->thetaT, e->xbar, e->ex, e->alive,
                             e->logov, e->eloc, e->den, e->parts, s, exg ? e->exf->exTot : nullptr,
                             bl.mult == 2 ? bl.tOff[1] : e->Ktot, bl.mult);
            launch_measure_reduce(W, e->alive, e->eloc, e->den, e->parts, 1, e->acc, e->G, e->xbar,
                                  exg ? nullptr : e->ex, e->bgNum, e->exNum, s);
        }
    }
    return check_launch();
}

int create_common_checks(int W, int precision)
{
    if (W <= 0) return fail(AFQMC_ERR_ARG, "walker count must be positive");
    if (precision != AFQMC_FP64 && precision != AFQMC_MIXED) return fail(AFQMC_ERR_ARG, "unknown precision");
    return AFQMC_OK;
}

// Runs after every argument check, so that argument errors are reported as
// such on a machine without a GPU too.
int create_device_check()
{
    int dev = 0;
    cudaError_t r = cudaGetDevice(&dev);
    if (r != cudaSuccess) return fail(AFQMC_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(r));
    return AFQMC_OK;
}

void free_engine(afqmc_engine *e)
{
    if (!e) return;
    drop_graphs(e);
    if (e->mx || e->cpm) mixed_destroy(e);
    delete e->exf;
    e->exf = nullptr;
    delete e->bp;
    e->bp = nullptr;
    prof_resolve(e);
    for (cudaEvent_t ev : e->evpool) cudaEventDestroy(ev);
    if (e->upStream) cudaStreamSynchronize(e->upStream);
    for (int k = 0; k < 2; ++k) {
        if (e->upReady[k]) cudaEventDestroy(e->upReady[k]);
        if (e->upFree[k]) cudaEventDestroy(e->upFree[k]);
    }
    if (e->upStream) cudaStreamDestroy(e->upStream);
    for (void *p : e->allocs) cudaFree(p);
    if (e->own) cudaStreamDestroy(e->own);
    delete e;
}

}  // namespace

// Mixed-estimator ingredients at the current walkers, without the one-body
// half step of addMixedMeasurement: logov, Sinv, thetaT, xbar, ex, eloc, den
// (FP64 arithmetic; the mixed form's fp32 walkers are read through the FP64
// copy).  Used by the adjoint.
// exchange: PL_EX_BLOCKWISE the per-walker kernel over both spin blocks;
// PL_EX_GEMM_ONE the FP64 GEMM form over block 0 counted twice (a restricted
// trial); PL_EX_GEMM_ALL the GEMM form over every block.
int engine_pl_local_energy(afqmc_engine *e, int exchange)
{
    const int W = e->W;
    cudaStream_t s = e->stream;
    if (e->precision == AFQMC_MIXED) TRY(mixed_sync_to_fp64(e));
    TRY(overlap_gemm(e, e->wf, e->alive, e->bl));
    launch_lu_logdet_inverse(W, e->bl, e->S, e->Sinv, e->alive, e->logw, make_double2(0, 0),
                             e->logwT, e->logov, e->alive, nullptr, nullptr, nullptr, e->status,
                             LU_PLAIN, true, s);
    TRY(check_launch());
    TRY(theta_gemm(e, e->wf, e->alive, e->bl));
    TRY(xbar_gemm(e, e->bl));
    if (exchange != PL_EX_BLOCKWISE) {
        if (!e->exf || !e->exf->gemm) return fail(AFQMC_ERR_STATE, "GEMM exchange not set up");
        const bool one = exchange == PL_EX_GEMM_ONE;
        if (one && !e->exf->restricted) return fail(AFQMC_ERR_STATE, "trial is not spin-restricted");
        const int nb = one ? 1 : e->bl.nblk, mult = one ? 2 : 1;
        bool first = true;
        for (int b = 0; b < nb; ++b) {
            if (e->bl.Ns[b] == 0) continue;
            TRY(exf64_walker_totals(e, exf64_block(e, b), !first, mult));
            first = false;
        }
        launch_pl_energy(W, e->G, e->Ktot, e->wfDaggerT, e->thetaT, e->xbar, e->ex, e->alive, e->logov,
                         e->eloc, e->den, e->parts, s, e->exf->exTot, one ? e->bl.tOff[1] : e->Ktot, mult);
        return check_launch();
    }
    if (launch_pl_exchange(W, e->n, e->G, e->bl, e->Aall, e->Ktot, e->thetaT, e->alive, e->ex, s))
        return fail(AFQMC_ERR_UNSUPPORTED, "exchange kernel supports at most 64 electrons per spin");
    launch_pl_energy(W, e->G, e->Ktot, e->wfDaggerT, e->thetaT, e->xbar, e->ex, e->alive, e->logov,
                     e->eloc, e->den, e->parts, s);
    return check_launch();
}

// FP64 form, real half-rotated vectors (real trial and Cholesky vectors,
// tested exactly): the exchange runs as FP64 GEMMs, and a closed-shell trial
// (equal spin blocks, bit for bit) computes block 0 alone and counts it
// twice, as the mixed form does.  Complex A keeps the blockwise kernel.
int fp64_exchange_setup(afqmc_engine *e)
{
    std::vector<zd> a((size_t)e->Ktot * e->G);
    CUDA_TRY(cudaMemcpyAsync(a.data(), e->Aall, sizeof(zd) * a.size(), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    for (const zd &v : a)
        if (v.y != 0.0) return AFQMC_OK;
    e->exf = new ExF64Scratch();
    ExF64Scratch &x = *e->exf;
    if (e->bl.nblk == 2 && e->nup == e->ndn && e->nup > 0) {
        const size_t cnt = (size_t)e->n * e->nup;
        std::vector<zd> t0(cnt), t1(cnt);
        CUDA_TRY(cudaMemcpy(t0.data(), e->phiT[0], sizeof(zd) * cnt, cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(t1.data(), e->phiT[1], sizeof(zd) * cnt, cudaMemcpyDeviceToHost));
        if (std::memcmp(t0.data(), t1.data(), sizeof(zd) * cnt) == 0) {
            x.restricted = true;
            x.bl1 = e->bl;
            x.bl1.nblk = 1;
            x.bl1.Ns[1] = 0;
            x.bl1.mult = 2;
        }
    }
    long long Kmax = 0;
    for (int b = 0; b < e->bl.nblk; ++b) Kmax = std::max(Kmax, (long long)e->bl.Ns[b] * e->n);
    TRY(exf64_alloc(e, Kmax, x));
    const Blocks &bl = fbl(e);
    for (int b = 0; b < bl.nblk; ++b)
        if (bl.Ns[b] > 0) TRY(exf64_build(e, b, x.blk[b]));
    x.gemm = true;
    return check_launch();
}

int engine_fail(int code, const std::string &msg) { return fail(code, msg); }
int engine_check_launch() { return check_launch(); }
int engine_gemm(const ZGemmArgs &a, cudaStream_t s) { return gemm(a, s); }
template <class T> int engine_dalloc(afqmc_engine *e, T **p, size_t count) { return dalloc(e, p, count); }
template int engine_dalloc<float>(afqmc_engine *, float **, size_t);
template int engine_dalloc<int>(afqmc_engine *, int **, size_t);
template int engine_dalloc<zd>(afqmc_engine *, zd **, size_t);
template int engine_dalloc<double>(afqmc_engine *, double **, size_t);
template int engine_dalloc<unsigned short>(afqmc_engine *, unsigned short **, size_t);
zd engine_one_body_logw(afqmc_engine *e, int which) { return one_body_logw(e, which); }

// =========================================================== C ABI
extern "C" {

const char *afqmc_last_error(void) { return g_err.c_str(); }
const char *afqmc_version(void) { return "afqmclab_b200 0.1 (sm_100a)"; }

int afqmc_cp_create(int L, int N, int W, int decomp, int force_type, double dt, double ET,
                    double force_cap, int mgs_step, int pop_control_step, int precision,
                    const double *K, const double *expMinusDtK, const double *expHalfDtK,
                    const double *expMinusHalfDtK, const double *U, const double *mu,
                    const double *hx, const double *hy, const double *hz,
                    const double *const_force, const double *phiT, double logwT_re,
                    double logwT_im, unsigned long long seed, afqmc_engine **out)
{
    if (!out) return fail(AFQMC_ERR_ARG, "out is NULL");
    *out = nullptr;
    TRY(create_common_checks(W, precision));
    if (L <= 0 || N <= 0 || N > 2 * L) return fail(AFQMC_ERR_ARG, "need 0 < N <= 2L");
    if (decomp < 0 || decomp > 3) return fail(AFQMC_ERR_ARG, "unknown decomposition");
    if (!K || !expMinusDtK || !expHalfDtK || !U || !mu || !hx || !hy || !hz || !phiT)
        return fail(AFQMC_ERR_ARG, "missing model array");
    if (mgs_step <= 0 || pop_control_step <= 0) return fail(AFQMC_ERR_ARG, "cadence must be positive");
    if (force_type != AFQMC_DYNAMIC_FORCE && force_type != AFQMC_CONST_FORCE)
        return fail(AFQMC_ERR_ARG, "unknown force type");
    TRY(create_device_check());
    afqmc_engine *e = new afqmc_engine();
    e->kind = KIND_CP; e->L = L; e->n = 2 * L; e->ncol = N; e->nup = N; e->ndn = 0; e->W = W;
    e->precision = precision; e->decomp = decomp; e->forceType = force_type;
    e->dt = dt; e->ET = ET; e->forceCap = force_cap; e->mgsStep = mgs_step; e->popStep = pop_control_step;
    e->seed = seed; e->logwT = make_double2(logwT_re, logwT_im);
    set_blocks(e);
    int r = alloc_population(e);
    const int n = e->n;
#define CK(x) do { r = (x); if (r != AFQMC_OK) { free_engine(e); return r; } } while (0)
    CK(r);
    CK(dupload(e, &e->phiT[0], phiT, (size_t)n * N));
    CK(dupload(e, &e->expK[0], expMinusDtK, (size_t)n * n));
    CK(dupload(e, &e->expK[1], expHalfDtK, (size_t)n * n));
    CK(dupload(e, &e->expK[2], expMinusHalfDtK ? expMinusHalfDtK : expHalfDtK, (size_t)n * n));
    CK(dupload(e, &e->U, U, L)); CK(dupload(e, &e->mu, mu, L)); CK(dupload(e, &e->hx, hx, L));
    CK(dupload(e, &e->hy, hy, L)); CK(dupload(e, &e->hz, hz, L));
    // NiupNidn constants (NiupNidn.cpp:12-26, setGamma :223-250, setConstDiag :252-270)
    std::vector<zd> gam(L), c00(L), c01(L), c10(L), c11(L);
    double usum = 0;
    for (int i = 0; i < L; ++i) usum += U[i];
    for (int i = 0; i < L; ++i) {
        double dtU = dt * U[i];
        cd g;
        if (decomp == AFQMC_DENSITY_CHARGE) g = solve_cosh_eq_exp(-dtU * 0.5);
        else if (decomp == AFQMC_HOP_SPIN) g = solve_cos_eq_exp(dtU * 0.5);
        else g = solve_cosh_eq_exp(dtU * 0.5);
        double a = -dt * (U[i] * 0.5 - mu[i] + hz[i] * 0.5);
        double b = -dt * (U[i] * 0.5 - mu[i] - hz[i] * 0.5);
        cd c = -dt * 0.5 * cd(hx[i], hy[i]);
        exp2by2(a, b, c);
        gam[i] = tozd(g); c00[i] = make_double2(a, 0); c01[i] = tozd(std::conj(c));
        c10[i] = tozd(c); c11[i] = make_double2(b, 0);
    }
    CK(dupload(e, &e->gamma, gam.data(), L));
    CK(dupload(e, &e->cdiag[0], c00.data(), L)); CK(dupload(e, &e->cdiag[1], c01.data(), L));
    CK(dupload(e, &e->cdiag[2], c10.data(), L)); CK(dupload(e, &e->cdiag[3], c11.data(), L));
    if (const_force) CK(dupload(e, &e->constForceCP, const_force, L));
    CK(dalloc(e, &e->forceCP, (size_t)W * L));
    CK(dalloc(e, &e->sites, (size_t)W * 4 * L));
    CK(dalloc(e, &e->siteNum, (size_t)4 * L));
    e->hd.L = L; e->hd.N = N; e->hd.n = n; e->hd.decomp = decomp;
    e->hd.gamma = e->gamma; e->hd.cd00 = e->cdiag[0]; e->hd.cd01 = e->cdiag[1];
    e->hd.cd10 = e->cdiag[2]; e->hd.cd11 = e->cdiag[3];
    e->hd.dtUSum = dt * usum; e->hd.forceCap = force_cap;
    e->hd.constForce = (force_type == AFQMC_CONST_FORCE)
                           ? (e->constForceCP ? e->constForceCP : nullptr) : nullptr;
    if (force_type == AFQMC_CONST_FORCE && !e->constForceCP) {
        CK(dalloc(e, &e->constForceCP, L));
        e->hd.constForce = e->constForceCP;
    }
    e->hd.phiT = e->phiT[0];
    // wfDaggerK = phiT^H K (HubbardSOCMeasureFixedSDSD::initWfDaggerK, :160-167)
    zd *Kd = nullptr;
    CK(dupload(e, &Kd, K, (size_t)n * n));
    e->Kmat = Kd;
    CK(dalloc(e, &e->wfDaggerK, (size_t)N * n));
    {
        ZGemmArgs g;
        g.m = N; g.n = n; g.k = n; g.opA = OP_C;
        g.A = e->phiT[0]; g.lda = n; g.B = Kd; g.ldb = n; g.C = e->wfDaggerK; g.ldc = N;
        CK(gemm(g, e->stream));
    }
    if (precision == AFQMC_MIXED) CK(mixed_create(e));
    cudaError_t ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) { free_engine(e); return fail(AFQMC_ERR_CUDA, cudaGetErrorString(ce)); }
#undef CK
    *out = e;
    return AFQMC_OK;
}

int afqmc_pl_create(int n, int Nup, int Ndn, int G, int W, int force_type, double dt, double ET,
                    double force_cap, int mgs_step, int pop_control_step, int precision,
                    const double *chol, const double *bg, const double *t,
                    const double *expMinusDtK, double logwExpMinusDtK, const double *expHalfDtK,
                    double logwExpHalfDtK, const double *expMinusHalfDtK,
                    double logwExpMinusHalfDtK, const double *logExpMinusDtK,
                    double logwLogExpMinusDtK, const double *const_force, const double *phiTUp,
                    const double *phiTDn, double logwT_re, double logwT_im,
                    unsigned long long seed, afqmc_engine **out)
{
    if (!out) return fail(AFQMC_ERR_ARG, "out is NULL");
    *out = nullptr;
    TRY(create_common_checks(W, precision));
    if (n <= 0 || Nup <= 0 || Ndn < 0 || Nup > n || Ndn > n || G <= 0)
        return fail(AFQMC_ERR_ARG, "bad sizes");
    if (!chol || !bg || !t || !phiTUp || (Ndn > 0 && !phiTDn) || !expHalfDtK)
        return fail(AFQMC_ERR_ARG, "missing model array");
    if (!expMinusDtK && !logExpMinusDtK) return fail(AFQMC_ERR_ARG, "need expMinusDtK or logExpMinusDtK");
    if (mgs_step <= 0 || pop_control_step <= 0) return fail(AFQMC_ERR_ARG, "cadence must be positive");
    if (force_type != AFQMC_DYNAMIC_FORCE && force_type != AFQMC_CONST_FORCE)
        return fail(AFQMC_ERR_ARG, "unknown force type");
    TRY(create_device_check());
    afqmc_engine *e = new afqmc_engine();
    e->kind = KIND_PL; e->n = n; e->nup = Nup; e->ndn = Ndn; e->ncol = std::max(Nup, Ndn);
    e->G = G; e->W = W; e->precision = precision; e->forceType = force_type;
    e->dt = dt; e->ET = ET; e->forceCap = force_cap; e->mgsStep = mgs_step; e->popStep = pop_control_step;
    e->seed = seed; e->logwT = make_double2(logwT_re, logwT_im);
    set_blocks(e);
    int r = alloc_population(e);
#define CK(x) do { r = (x); if (r != AFQMC_OK) { free_engine(e); return r; } } while (0)
    CK(r);
    const size_t n2 = (size_t)n * n;
    CK(dupload(e, &e->phiT[0], phiTUp, (size_t)n * Nup));
    if (Ndn > 0) CK(dupload(e, &e->phiT[1], phiTDn, (size_t)n * Ndn));
    e->useLog = (expMinusDtK == nullptr);
    if (!e->useLog) CK(dupload(e, &e->expK[0], expMinusDtK, n2));
    else CK(dupload(e, &e->logK, logExpMinusDtK, n2));
    CK(dupload(e, &e->expK[1], expHalfDtK, n2));
    CK(dupload(e, &e->expK[2], expMinusHalfDtK ? expMinusHalfDtK : expHalfDtK, n2));
    e->expLogw[0] = make_double2(logwExpMinusDtK, 0);
    e->expLogw[1] = make_double2(logwExpHalfDtK, 0);
    e->expLogw[2] = make_double2(logwExpMinusHalfDtK, 0);
    e->logKLogw = make_double2(logwLogExpMinusDtK, 0);
    CK(dupload(e, &e->chol, chol, n2 * G));
    CK(dupload(e, &e->bg, bg, G));
    if (const_force) CK(dupload(e, &e->constForcePL, const_force, G));
    else if (force_type == AFQMC_CONST_FORCE) CK(dalloc(e, &e->constForcePL, G));
    e->Ktot = (long long)(Nup + Ndn) * n;
    CK(dalloc(e, &e->Aall, (size_t)e->Ktot * G));
    CK(dalloc(e, &e->wfDaggerT, (size_t)e->Ktot));
    double *td = nullptr;
    CK(dupload(e, &td, t, n2));
    e->tdev = td;
    // A_g,sigma = phiT_sigma^H L_g (initWfDaggerCholeskyVecs, :165-186) and
    // wfDaggerT = phiT_sigma^H t (initWfDaggerT, :148-163), stacked up/down
    for (int b = 0; b < e->bl.nblk; ++b) {
        int Ns = e->bl.Ns[b];
        ZGemmArgs g;
        g.m = Ns; g.n = n; g.k = n; g.opA = OP_C; g.b_real = 1;
        g.A = e->phiT[b]; g.lda = n; g.strideA = 0;
        g.B = e->chol; g.ldb = n; g.strideB = (long long)n2;
        g.C = e->Aall + e->bl.tOff[b]; g.ldc = Ns; g.strideC = e->Ktot;
        g.batch = G;
        CK(gemm(g, e->stream));
        ZGemmArgs h = g;
        h.B = td; h.strideB = 0; h.C = e->wfDaggerT + e->bl.tOff[b]; h.strideC = 0; h.batch = 1;
        CK(gemm(h, e->stream));
    }
    CK(dalloc(e, &e->xbar, (size_t)G * W));
    CK(dalloc(e, &e->forcePL, (size_t)G * W));
    CK(dalloc(e, &e->aux, (size_t)G * W));
    CK(dalloc(e, &e->ex, (size_t)G * W));
    CK(dalloc(e, &e->bgNum, G));
    CK(dalloc(e, &e->exNum, G));
    if (precision == AFQMC_FP64) CK(dalloc(e, &e->M, n2 * W));
    e->cdv.n = n; e->cdv.G = G; e->cdv.bg = e->bg; e->cdv.forceCap = force_cap;
    e->cdv.sqrtMinusDtIm = -std::sqrt(dt);
    e->cdv.constForce = (force_type == AFQMC_CONST_FORCE) ? e->constForcePL : nullptr;
    if (precision == AFQMC_MIXED) CK(mixed_create(e));
    else CK(fp64_exchange_setup(e));
    cudaError_t ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) { free_engine(e); return fail(AFQMC_ERR_CUDA, cudaGetErrorString(ce)); }
#undef CK
    *out = e;
    return AFQMC_OK;
}

int afqmc_destroy(afqmc_engine *e)
{
    if (!e) return AFQMC_OK;
    cudaStreamSynchronize(e->stream);
    free_engine(e);
    return AFQMC_OK;
}

int afqmc_set_stream(afqmc_engine *e, void *cuda_stream)
{
    if (!e) return fail(AFQMC_ERR_ARG, "null engine");
    cudaStream_t ns = cuda_stream ? (cudaStream_t)cuda_stream : e->own;
    if (ns != e->stream) drop_graphs(e);
    e->stream = ns;
    return AFQMC_OK;
}

int afqmc_synchronize(afqmc_engine *e)
{
    if (!e) return fail(AFQMC_ERR_ARG, "null engine");
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return AFQMC_OK;
}

int afqmc_set_walkers(afqmc_engine *e, const double *wf, const double *logw, const int *alive)
{
    if (!e || !wf || !logw || !alive) return fail(AFQMC_ERR_ARG, "null argument");
    CUDA_TRY(cudaMemcpyAsync(e->wf, wf, sizeof(zd) * e->wsize * e->W, cudaMemcpyHostToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync(e->logw, logw, sizeof(zd) * e->W, cudaMemcpyHostToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync(e->alive, alive, sizeof(int) * e->W, cudaMemcpyHostToDevice, e->stream));
    if (e->precision == AFQMC_MIXED) TRY(mixed_sync_from_fp64(e));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return AFQMC_OK;
}

namespace {

// the copy stream, its events and the log-weight / alive staging slots,
// made by the first asynchronous upload
int upload_init(afqmc_engine *e)
{
    if (e->upStream) return AFQMC_OK;
    CUDA_TRY(cudaStreamCreateWithFlags(&e->upStream, cudaStreamNonBlocking));
    for (int k = 0; k < 2; ++k) {
        CUDA_TRY(cudaEventCreateWithFlags(&e->upReady[k], cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&e->upFree[k], cudaEventDisableTiming));
        CUDA_TRY(cudaEventRecord(e->upFree[k], e->stream));
        TRY(dalloc(e, &e->stgLw[k], (size_t)e->W));
        TRY(dalloc(e, &e->stgAl[k], (size_t)e->W));
    }
    return AFQMC_OK;
}

}  // namespace

int afqmc_set_walkers_async(afqmc_engine *e, const double *wf, const double *logw, const int *alive)
{
    if (!e || !wf || !logw || !alive) return fail(AFQMC_ERR_ARG, "null argument");
    TRY(upload_init(e));
    if (!e->stgWf[0])
        for (int k = 0; k < 2; ++k) TRY(dalloc(e, &e->stgWf[k], (size_t)e->wsize * e->W));
    const int k = e->upNext;
    e->upNext ^= 1;
    // the slot's previous contents must have been installed first
    CUDA_TRY(cudaStreamWaitEvent(e->upStream, e->upFree[k], 0));
    CUDA_TRY(cudaMemcpyAsync(e->stgWf[k], wf, sizeof(zd) * e->wsize * e->W, cudaMemcpyHostToDevice, e->upStream));
    CUDA_TRY(cudaMemcpyAsync(e->stgLw[k], logw, sizeof(zd) * e->W, cudaMemcpyHostToDevice, e->upStream));
    CUDA_TRY(cudaMemcpyAsync(e->stgAl[k], alive, sizeof(int) * e->W, cudaMemcpyHostToDevice, e->upStream));
    CUDA_TRY(cudaEventRecord(e->upReady[k], e->upStream));
    // installed on the work stream after everything enqueued before this call
    CUDA_TRY(cudaStreamWaitEvent(e->stream, e->upReady[k], 0));
    CUDA_TRY(cudaMemcpyAsync(e->logw, e->stgLw[k], sizeof(zd) * e->W, cudaMemcpyDeviceToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync(e->alive, e->stgAl[k], sizeof(int) * e->W, cudaMemcpyDeviceToDevice, e->stream));
    if (e->precision == AFQMC_MIXED && mixed_can_load_direct(e)) {
        TRY(mixed_load_direct(e, e->stgWf[k]));
    } else {
        CUDA_TRY(cudaMemcpyAsync(e->wf, e->stgWf[k], sizeof(zd) * e->wsize * e->W, cudaMemcpyDeviceToDevice,
                                 e->stream));
        if (e->precision == AFQMC_MIXED) TRY(mixed_sync_from_fp64(e));
    }
    CUDA_TRY(cudaEventRecord(e->upFree[k], e->stream));
    return AFQMC_OK;
}

int afqmc_set_walkers_f32_async(afqmc_engine *e, const float *wf32, const double *logw, const int *alive)
{
    if (!e || !wf32 || !logw || !alive) return fail(AFQMC_ERR_ARG, "null argument");
    if (e->precision != AFQMC_MIXED || !mixed_can_load_direct(e))
        return fail(AFQMC_ERR_UNSUPPORTED, "fp32 walker upload is for the phaseless mixed form");
    TRY(upload_init(e));
    const size_t count = (size_t)2 * e->wsize * e->W;   // [re | im] planes per walker
    if (!e->stgWf32[0])
        for (int k = 0; k < 2; ++k) TRY(dalloc(e, &e->stgWf32[k], count));
    const int k = e->upNext;
    e->upNext ^= 1;
    CUDA_TRY(cudaStreamWaitEvent(e->upStream, e->upFree[k], 0));
    CUDA_TRY(cudaMemcpyAsync(e->stgWf32[k], wf32, sizeof(float) * count, cudaMemcpyHostToDevice, e->upStream));
    CUDA_TRY(cudaMemcpyAsync(e->stgLw[k], logw, sizeof(zd) * e->W, cudaMemcpyHostToDevice, e->upStream));
    CUDA_TRY(cudaMemcpyAsync(e->stgAl[k], alive, sizeof(int) * e->W, cudaMemcpyHostToDevice, e->upStream));
    CUDA_TRY(cudaEventRecord(e->upReady[k], e->upStream));
    CUDA_TRY(cudaStreamWaitEvent(e->stream, e->upReady[k], 0));
    CUDA_TRY(cudaMemcpyAsync(e->logw, e->stgLw[k], sizeof(zd) * e->W, cudaMemcpyDeviceToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync(e->alive, e->stgAl[k], sizeof(int) * e->W, cudaMemcpyDeviceToDevice, e->stream));
    TRY(mixed_load_f32(e, e->stgWf32[k]));
    CUDA_TRY(cudaEventRecord(e->upFree[k], e->stream));
    return AFQMC_OK;
}

int afqmc_upload_wait(afqmc_engine *e)
{
    if (!e) return fail(AFQMC_ERR_ARG, "null engine");
    if (e->upStream) CUDA_TRY(cudaStreamSynchronize(e->upStream));
    return AFQMC_OK;
}

int afqmc_get_walkers(afqmc_engine *e, double *wf, double *logw, int *alive)
{
    if (!e) return fail(AFQMC_ERR_ARG, "null engine");
    if (e->precision == AFQMC_MIXED) TRY(mixed_sync_to_fp64(e));
    if (wf) CUDA_TRY(cudaMemcpyAsync(wf, e->wf, sizeof(zd) * e->wsize * e->W, cudaMemcpyDeviceToHost, e->stream));
    if (logw) CUDA_TRY(cudaMemcpyAsync(logw, e->logw, sizeof(zd) * e->W, cudaMemcpyDeviceToHost, e->stream));
    if (alive) CUDA_TRY(cudaMemcpyAsync(alive, e->alive, sizeof(int) * e->W, cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return AFQMC_OK;
}

int afqmc_set_rng(afqmc_engine *e, unsigned long long seed, unsigned long long counter)
{
    if (!e) return fail(AFQMC_ERR_ARG, "null engine");
    if (seed != e->seed) drop_graphs(e);
    e->seed = seed;
    CUDA_TRY(cudaMemcpyAsync(e->counter, &counter, sizeof(counter), cudaMemcpyHostToDevice, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return AFQMC_OK;
}

int afqmc_get_rng(afqmc_engine *e, unsigned long long *seed, unsigned long long *counter)
{
    if (!e) return fail(AFQMC_ERR_ARG, "null engine");
    if (seed) *seed = e->seed;
    if (counter) {
        CUDA_TRY(cudaMemcpyAsync(counter, e->counter, sizeof(*counter), cudaMemcpyDeviceToHost, e->stream));
        CUDA_TRY(cudaStreamSynchronize(e->stream));
    }
    return AFQMC_OK;
}

int afqmc_set_ET(afqmc_engine *e, double ET)
{
    if (!e) return fail(AFQMC_ERR_ARG, "null engine");
    if (ET != e->ET) drop_graphs(e);
    e->ET = ET;
    return AFQMC_OK;
}

int afqmc_set_cadence(afqmc_engine *e, int mgs_index, int pop_control_index)
{
    if (!e) return fail(AFQMC_ERR_ARG, "null engine");
    e->mgsIndex = mgs_index;
    e->popIndex = pop_control_index;
    return AFQMC_OK;
}

int afqmc_project_one_step(afqmc_engine *e, int nsteps)
{
    if (!e) return fail(AFQMC_ERR_ARG, "null engine");
    for (int i = 0; i < nsteps; ++i) TRY(project_one_step(e));
    return AFQMC_OK;
}

int afqmc_project_half(afqmc_engine *e, int which)
{
    if (!e || (which != -1 && which != 1)) return fail(AFQMC_ERR_ARG, "which must be -1 or +1");
    if (e->precision == AFQMC_MIXED) TRY(mixed_sync_to_fp64(e));
    int idx = which < 0 ? 2 : 1;
    TRY(one_body(e, idx, e->wf, e->wfTmp, e->alive));
    launch_copy_masked(e->W, e->wsize, e->wfTmp, e->wf, e->alive, e->stream);
    TRY(check_launch());
    // walkerNew.logw = oneBody.logw + walker.logw for alive walkers
    std::vector<zd> lw(e->W);
    std::vector<int> al(e->W);
    CUDA_TRY(cudaMemcpyAsync(lw.data(), e->logw, sizeof(zd) * e->W, cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaMemcpyAsync(al.data(), e->alive, sizeof(int) * e->W, cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    zd add = one_body_logw(e, idx);
    for (int w = 0; w < e->W; ++w)
        if (al[w]) lw[w] = zadd(add, lw[w]);
    CUDA_TRY(cudaMemcpyAsync(e->logw, lw.data(), sizeof(zd) * e->W, cudaMemcpyHostToDevice, e->stream));
    if (e->precision == AFQMC_MIXED) TRY(mixed_sync_from_fp64(e));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return AFQMC_OK;
}

int afqmc_modify_gm(afqmc_engine *e)
{
    if (!e) return fail(AFQMC_ERR_ARG, "null engine");
    return modify_gm(e);
}

int afqmc_pop_control(afqmc_engine *e, int *table_out, double *weight_out)
{
    if (!e) return fail(AFQMC_ERR_ARG, "null engine");
    TRY(pop_control(e));
    if (table_out) CUDA_TRY(cudaMemcpyAsync(table_out, e->table, sizeof(int) * e->W, cudaMemcpyDeviceToHost, e->stream));
    if (weight_out) CUDA_TRY(cudaMemcpyAsync(weight_out, e->weight, sizeof(double) * e->W, cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return AFQMC_OK;
}

int afqmc_reset_measurement(afqmc_engine *e)
{
    if (!e) return fail(AFQMC_ERR_ARG, "null engine");
    CUDA_TRY(cudaMemsetAsync(e->acc, 0, sizeof(zd) * 8, e->stream));
    if (e->bgNum) CUDA_TRY(cudaMemsetAsync(e->bgNum, 0, sizeof(zd) * e->G, e->stream));
    if (e->exNum) CUDA_TRY(cudaMemsetAsync(e->exNum, 0, sizeof(zd) * e->G, e->stream));
    if (e->siteNum) CUDA_TRY(cudaMemsetAsync(e->siteNum, 0, sizeof(zd) * 4 * e->L, e->stream));
    if (e->obs)
        CUDA_TRY(cudaMemsetAsync(e->obs, 0, sizeof(zd) * (8LL * e->L * e->L + 3LL * e->L * e->L), e->stream));
    return AFQMC_OK;
}

int afqmc_cp_set_observables(afqmc_engine *e, int on)
{
    if (!e || e->kind != KIND_CP) return fail(AFQMC_ERR_ARG, "constrained-path engine required");
    drop_graphs(e);
    if (on && !e->Gfull) {
        const int n = e->n, N = e->ncol, L = e->L;
        std::vector<zd> t((size_t)n * N);
        CUDA_TRY(cudaMemcpyAsync(t.data(), e->phiT[0], sizeof(zd) * t.size(), cudaMemcpyDeviceToHost, e->stream));
        CUDA_TRY(cudaStreamSynchronize(e->stream));
        for (zd &v : t) v.y = -v.y;
        TRY(dupload(e, &e->phiTc, t.data(), t.size()));
        TRY(dalloc(e, &e->Gfull, (size_t)e->W * n * n));
        TRY(dalloc(e, &e->obs, (size_t)8 * L * L + (size_t)3 * L * L));
    }
    e->observe = on != 0;
    return AFQMC_OK;
}

int afqmc_get_observables(afqmc_engine *e, double *greenNum, double *densityDensityNum, double *splusSminusNum,
                          double *sminusSplusNum, double *spairSpairNum)
{
    if (!e || e->kind != KIND_CP || !e->obs) return fail(AFQMC_ERR_STATE, "observables are not enabled");
    const size_t n2 = 4ULL * e->L * e->L, l2 = (size_t)e->L * e->L;
    double *dst[5] = {greenNum, densityDensityNum, splusSminusNum, sminusSplusNum, spairSpairNum};
    const size_t off[5] = {0, n2, 2 * n2, 2 * n2 + l2, 2 * n2 + 2 * l2};
    const size_t cnt[5] = {n2, n2, l2, l2, l2};
    for (int k = 0; k < 5; ++k)
        if (dst[k]) CUDA_TRY(cudaMemcpyAsync(dst[k], e->obs + off[k], sizeof(zd) * cnt[k], cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return AFQMC_OK;
}

// ------------------------------------------------------------ back-propagation
// The back-propagated estimator of tutorials/afqmcConstraintPathBP
// (afqmcConstraintPathBackPropagation.cpp, afqmcConstraintPathMeasure.cpp:
// addMeasurement): the fields and population-control tables of a window of
// `steps` steps are recorded; at measurement the window-start walkers are
// resampled by the recorded tables, the trial is propagated leftwards through
// each walker's recorded fields, and the observe estimator (energies from the
// full Green's matrix, HubbardSOCMeasureCommuteSDSD::addEnergy, and the
// observables) is accumulated for the pair (left: back-propagated trial,
// right: window-start walker), weighted by the current walker's overlap.

int afqmc_cp_bp_begin(afqmc_engine *e, int steps, int measure_skip)
{
    if (!e || e->kind != KIND_CP) return fail(AFQMC_ERR_ARG, "constrained-path engine required");
    if (e->precision != AFQMC_FP64) return fail(AFQMC_ERR_UNSUPPORTED, "back-propagation runs in the FP64 form");
    if (steps <= 0 || measure_skip <= 0) return fail(AFQMC_ERR_ARG, "steps and measure_skip must be positive");
    if (!e->observe) return fail(AFQMC_ERR_STATE, "back-propagation measures the observe estimator: enable it first");
    const int W = e->W, L = e->L;
    const size_t ws = (size_t)e->wsize;
    if (!e->bp) e->bp = new BPState();
    BPState *bp = e->bp;
    if (!bp->wfBackup) {
        TRY(dalloc(e, &bp->wfBackup, ws * W)); TRY(dalloc(e, &bp->wfMeas, ws * W));
        TRY(dalloc(e, &bp->left, ws * W)); TRY(dalloc(e, &bp->leftTmp, ws * W)); TRY(dalloc(e, &bp->right, ws * W));
        TRY(dalloc(e, &bp->logwBackup, W)); TRY(dalloc(e, &bp->logwMeas, W)); TRY(dalloc(e, &bp->logwL, W));
        TRY(dalloc(e, &bp->logovBP, W));
        TRY(dalloc(e, &bp->ones, W));
        launch_set_int(bp->ones, 1, W, e->stream);
    }
    if (steps > bp->cap) {
        TRY(dalloc(e, &bp->aux, (size_t)steps * W * L)); TRY(dalloc(e, &bp->auxMeas, (size_t)steps * W * L));
        TRY(dalloc(e, &bp->valid, (size_t)steps * W)); TRY(dalloc(e, &bp->validMeas, (size_t)steps * W));
        TRY(dalloc(e, &bp->table, (size_t)steps * W));
        bp->cap = steps;
    }
    drop_graphs(e);
    // prepareBackPropagation: the window starts from the current walkers
    CUDA_TRY(cudaMemcpyAsync(bp->wfBackup, e->wf, sizeof(zd) * ws * W, cudaMemcpyDeviceToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync(bp->logwBackup, e->logw, sizeof(zd) * W, cudaMemcpyDeviceToDevice, e->stream));
    CUDA_TRY(cudaMemsetAsync(bp->valid, 0, sizeof(int) * (size_t)steps * W, e->stream));
    bp->steps = steps;
    bp->skip = measure_skip;
    bp->index = 0;
    bp->tableValid.assign((size_t)steps, 0);
    bp->active = true;
    return check_launch();
}

int afqmc_cp_bp_state(afqmc_engine *e, int *active, int *index)
{
    if (!e) return fail(AFQMC_ERR_ARG, "null engine");
    const bool on = e->bp && e->bp->active;
    if (active) *active = on ? 1 : 0;
    if (index) *index = on ? e->bp->index : 0;
    return AFQMC_OK;
}

namespace {

// generateWalkerBackupFromWalkerBPMeasure
// (afqmcConstraintPathBackPropagation.cpp:78-97): the next window's start
// walkers = the resampled window-start walkers propagated over the first
// measure_skip recorded steps (walkers without a record at a step are not
// propagated at it), normalised (logw reset to 0) at every step j with
// j % mgsStep == 0.
int bp_regenerate_backup(afqmc_engine *e)
{
    BPState *bp = e->bp;
    const int W = e->W, L = e->L;
    const size_t ws = (size_t)e->wsize;
    cudaStream_t s = e->stream;
    CUDA_TRY(cudaMemcpyAsync(bp->wfBackup, bp->wfMeas, sizeof(zd) * ws * W, cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(bp->logwBackup, bp->logwMeas, sizeof(zd) * W, cudaMemcpyDeviceToDevice, s));
    for (int j = 0; j < bp->skip; ++j) {
        const int *valid = bp->validMeas + (size_t)j * W;
        launch_cp_aux_apply(W, e->hd, bp->auxMeas + (size_t)j * W * L, valid, bp->wfBackup, bp->leftTmp,
                            bp->logwBackup, false, e->expLogw[0], s);
        ZGemmArgs g;
        g.m = e->n; g.n = e->ncol; g.k = e->n;
        g.A = e->expK[0]; g.lda = e->n;
        g.B = bp->leftTmp; g.ldb = e->n; g.strideB = e->wsize;
        g.C = bp->wfBackup; g.ldc = e->n; g.strideC = e->wsize;
        g.batch = W; g.mask = valid;
        TRY(gemm(g, s));
        if (j % e->mgsStep == 0) {
            launch_mgs(W, e->n, e->ncol, e->nup, e->ndn, 0, bp->wfBackup, bp->logwBackup, bp->ones, e->status, s);
            CUDA_TRY(cudaMemsetAsync(bp->logwBackup, 0, sizeof(zd) * W, s));
        }
    }
    return check_launch();
}

// one-body operator k applied from the left, K^H phi (HopSDOperation::
// applyToLeft, hopSDOperation.cpp:21-26), to every alive walker of src
// (srcStride 0: the same matrix for all) into dst
int left_one_body(afqmc_engine *e, int k, const zd *src, long long srcStride, zd *dst)
{
    ZGemmArgs g;
    g.m = e->n; g.n = e->ncol; g.k = e->n;
    g.opA = OP_C;
    g.A = e->expK[k]; g.lda = e->n;
    g.B = src; g.ldb = e->n; g.strideB = srcStride;
    g.C = dst; g.ldc = e->n; g.strideC = e->wsize;
    g.batch = e->W; g.mask = e->alive;
    return gemm(g, e->stream);
}

}  // namespace

int afqmc_cp_bp_measure(afqmc_engine *e)
{
    if (!e || e->kind != KIND_CP) return fail(AFQMC_ERR_ARG, "constrained-path engine required");
    BPState *bp = e->bp;
    if (!bp || !bp->active || bp->index != bp->steps)
        return fail(AFQMC_ERR_STATE, "no complete back-propagation window to measure");
    const int W = e->W, L = e->L, steps = bp->steps, skip = bp->skip;
    const size_t ws = (size_t)e->wsize;
    cudaStream_t s = e->stream;
    PHASE(AFQMC_PH_MEASURE);
    // prepareBackPropagationMeasAndNextBackup (afqmcConstraintPathBackPropagation.cpp:22-76)
    std::swap(bp->wfMeas, bp->wfBackup);
    std::swap(bp->logwMeas, bp->logwBackup);
    if (steps >= skip) {
        CUDA_TRY(cudaMemcpyAsync(bp->auxMeas, bp->aux, sizeof(int) * (size_t)steps * W * L, cudaMemcpyDeviceToDevice, s));
        CUDA_TRY(cudaMemcpyAsync(bp->validMeas, bp->valid, sizeof(int) * (size_t)steps * W, cudaMemcpyDeviceToDevice, s));
    } else {
        std::swap(bp->auxMeas, bp->aux);
        std::swap(bp->validMeas, bp->valid);
    }
    for (int i = 0; i < steps; ++i) {
        if (bp->tableValid[i]) {
            const int *tab = bp->table + (size_t)i * W;
            launch_pop_gather(W, e->wsize, tab, bp->wfMeas, bp->logwMeas, s);
            launch_bp_gather_rows(W, L, i + 1, tab, bp->auxMeas, s);
            launch_bp_gather_rows(W, 1, i + 1, tab, bp->validMeas, s);
        }
        if (i + 1 == skip) TRY(bp_regenerate_backup(e));
    }
    if (steps >= skip) {
        // the window slides by measure_skip steps: records skip..steps-1 move
        // to 0..steps-skip-1 (in increasing order, so no source is overwritten
        // before it is read), their old slots are left without a table
        for (int i = 0; i + skip < steps; ++i) {
            CUDA_TRY(cudaMemcpyAsync(bp->aux + (size_t)i * W * L, bp->aux + (size_t)(i + skip) * W * L,
                                     sizeof(int) * (size_t)W * L, cudaMemcpyDeviceToDevice, s));
            CUDA_TRY(cudaMemcpyAsync(bp->valid + (size_t)i * W, bp->valid + (size_t)(i + skip) * W,
                                     sizeof(int) * W, cudaMemcpyDeviceToDevice, s));
            CUDA_TRY(cudaMemcpyAsync(bp->table + (size_t)i * W, bp->table + (size_t)(i + skip) * W,
                                     sizeof(int) * W, cudaMemcpyDeviceToDevice, s));
            bp->tableValid[i] = bp->tableValid[i + skip];
            bp->tableValid[i + skip] = 0;
        }
        bp->index = steps - skip;
    } else {
        bp->active = false;
    }

    // addMeasurement (afqmcConstraintPathMeasure.cpp:47-78) for the alive walkers.
    // The weight: the current walker's overlap with the trial after exp(dt/2 K).
    TRY(one_body(e, 1, e->wf, e->wfTmp, e->alive));
    TRY(overlap_gemm(e, e->wfTmp, e->alive, fbl(e)));
    launch_lu_logdet_inverse(W, fbl(e), e->S, nullptr, e->alive, e->logw, one_body_logw(e, 1), e->logwT,
                             e->logov, e->alive, nullptr, nullptr, nullptr, e->status, LU_PLAIN, false, s);
    // left: exp(-dt/2 K)^H phiT, then for j = steps..1 the recorded fields and
    // exp(-dt K) from the left, normalised when (steps - j + 1) % mgsStep == 0,
    // then exp(dt/2 K)^H
    TRY(left_one_body(e, 2, e->phiT[0], 0, bp->left));
    CUDA_TRY(cudaMemsetAsync(bp->logwL, 0, sizeof(zd) * W, s));
    const zd noLogw = make_double2(0.0, 0.0);
    for (int j = steps; j > 0; --j) {
        launch_cp_aux_apply(W, e->hd, bp->auxMeas + (size_t)(j - 1) * W * L, e->alive, bp->left, bp->leftTmp,
                            bp->logwL, true, noLogw, s);
        TRY(left_one_body(e, 0, bp->leftTmp, e->wsize, bp->left));
        if ((steps - j + 1) % e->mgsStep == 0)
            launch_mgs(W, e->n, e->ncol, e->nup, e->ndn, 0, bp->left, bp->logwL, e->alive, e->status, s);
    }
    TRY(left_one_body(e, 1, bp->left, e->wsize, bp->leftTmp));
    // right: exp(dt/2 K) times the window-start walker
    TRY(one_body(e, 1, bp->wfMeas, bp->right, e->alive));
    // S = left^H right, its inverse, thetaT = S^-T right^T, G = conj(left) thetaT
    // (SDSDOperation.cpp:52-186 for the pair)
    {
        ZGemmArgs g;
        g.m = e->ncol; g.n = e->ncol; g.k = e->n;
        g.opA = OP_C;
        g.A = bp->leftTmp; g.lda = e->n; g.strideA = e->wsize;
        g.B = bp->right; g.ldb = e->n; g.strideB = e->wsize;
        g.C = e->S; g.ldc = e->ncol; g.strideC = e->bl.sStride;
        g.batch = W; g.mask = e->alive;
        TRY(gemm(g, s));
    }
    CUDA_TRY(cudaMemsetAsync(bp->logwL, 0, sizeof(zd) * W, s));
    launch_lu_logdet_inverse(W, e->bl, e->S, e->Sinv, e->alive, bp->logwL, noLogw, noLogw, bp->logovBP, e->alive,
                             nullptr, nullptr, nullptr, e->status, LU_PLAIN, true, s);
    TRY(theta_gemm(e, bp->right, e->alive, e->bl));
    launch_zconj((long long)ws * W, bp->leftTmp, bp->left, s);
    {
        ZGemmArgs g;
        g.m = e->n; g.n = e->n; g.k = e->ncol;
        g.A = bp->left; g.lda = e->n; g.strideA = e->wsize;
        g.B = e->thetaT; g.ldb = e->ncol; g.strideB = e->bl.tStride;
        g.C = e->Gfull; g.ldc = e->n; g.strideC = (long long)e->n * e->n;
        g.batch = W; g.mask = e->alive;
        TRY(gemm(g, s));
    }
    launch_cp_commute_energy(W, L, e->Gfull, e->Kmat, e->U, e->mu, e->hx, e->hy, e->hz, e->alive, e->logov,
                             e->eloc, e->den, e->parts, s);
    launch_measure_reduce(W, e->alive, e->eloc, e->den, e->parts, 3, e->acc, 0, nullptr, nullptr, nullptr,
                          nullptr, s);
    launch_cp_observe(W, L, e->Gfull, e->den, e->alive, e->obs, s);
    return check_launch();
}

int afqmc_add_mixed_measurement(afqmc_engine *e)
{
    if (!e) return fail(AFQMC_ERR_ARG, "null engine");
    return add_mixed_measurement(e);
}

int afqmc_get_measurement(afqmc_engine *e, double *out)
{
    if (!e || !out) return fail(AFQMC_ERR_ARG, "null argument");
    zd a[8];
    CUDA_TRY(cudaMemcpyAsync(a, e->acc, sizeof(a), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    for (int i = 0; i < 5; ++i) { out[2 * i] = a[i].x; out[2 * i + 1] = a[i].y; }
    if (e->kind == KIND_PL) { out[6] = out[7] = out[8] = out[9] = 0.0; }
    return AFQMC_OK;
}

int afqmc_get_site_nums(afqmc_engine *e, double *NupNum, double *NdnNum, double *SplusNum,
                        double *SminusNum)
{
    if (!e || e->kind != KIND_CP) return fail(AFQMC_ERR_ARG, "constrained-path engine required");
    const int L = e->L;
    std::vector<zd> h((size_t)4 * L);
    CUDA_TRY(cudaMemcpyAsync(h.data(), e->siteNum, sizeof(zd) * 4 * L, cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    double *dst[4] = {NupNum, NdnNum, SplusNum, SminusNum};
    for (int k = 0; k < 4; ++k)
        if (dst[k]) std::memcpy(dst[k], h.data() + (size_t)k * L, sizeof(zd) * L);
    return AFQMC_OK;
}

int afqmc_get_cholesky_nums(afqmc_engine *e, double *bgNum, double *exNum)
{
    if (!e || e->kind != KIND_PL) return fail(AFQMC_ERR_ARG, "phaseless engine required");
    if (bgNum) CUDA_TRY(cudaMemcpyAsync(bgNum, e->bgNum, sizeof(zd) * e->G, cudaMemcpyDeviceToHost, e->stream));
    if (exNum) CUDA_TRY(cudaMemcpyAsync(exNum, e->exNum, sizeof(zd) * e->G, cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return AFQMC_OK;
}

int afqmc_pl_update_background(afqmc_engine *e, const double *bg, const double *expMinusDtK,
                               double logwExpMinusDtK, const double *expHalfDtK,
                               double logwExpHalfDtK, const double *expMinusHalfDtK,
                               double logwExpMinusHalfDtK)
{
    if (!e || e->kind != KIND_PL || !bg) return fail(AFQMC_ERR_ARG, "phaseless engine and bg required");
    const size_t n2 = (size_t)e->n * e->n;
    // In the Taylor (LogHop2is) form the half-step slots hold log-form
    // matrices; switching to dense operators has to replace all three.
    if (e->useLog && expMinusDtK && (!expHalfDtK || !expMinusHalfDtK))
        return fail(AFQMC_ERR_ARG, "switching from the Taylor one-body form to dense operators needs "
                                   "expMinusDtK, expHalfDtK and expMinusHalfDtK");
    drop_graphs(e);
    CUDA_TRY(cudaMemcpyAsync(e->bg, bg, sizeof(double) * e->G, cudaMemcpyHostToDevice, e->stream));
    if (expMinusDtK) {
        if (!e->expK[0]) TRY(dalloc(e, &e->expK[0], n2));
        CUDA_TRY(cudaMemcpyAsync(e->expK[0], expMinusDtK, sizeof(zd) * n2, cudaMemcpyHostToDevice, e->stream));
        e->expLogw[0] = make_double2(logwExpMinusDtK, 0);
        e->useLog = false;
    }
    if (expHalfDtK) {
        CUDA_TRY(cudaMemcpyAsync(e->expK[1], expHalfDtK, sizeof(zd) * n2, cudaMemcpyHostToDevice, e->stream));
        e->expLogw[1] = make_double2(logwExpHalfDtK, 0);
    }
    if (expMinusHalfDtK) {
        CUDA_TRY(cudaMemcpyAsync(e->expK[2], expMinusHalfDtK, sizeof(zd) * n2, cudaMemcpyHostToDevice, e->stream));
        e->expLogw[2] = make_double2(logwExpMinusHalfDtK, 0);
    }
    if (e->precision == AFQMC_MIXED) TRY(mixed_update_operators(e));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return AFQMC_OK;
}

namespace {

// RealMaterialMolecule::setKp (realMaterialMolecule.cpp:155-166): Kp = K +
// sum_g bg_g L_g (the gemv of the reference, accumulated over g in order),
// one thread per matrix entry.
__global__ void kp_build_kernel(long long n2, int G, const double *K, const double *chol, const double *bg,
                                zd *Kp)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n2;
         i += (long long)gridDim.x * blockDim.x) {
        double s = K[i];
        for (int g = 0; g < G; ++g) s = fma(chol[i + n2 * g], bg[g], s);
        Kp[i] = make_double2(s, 0.0);
    }
}

// out[0] = max_j sum_i |Kp(i, j)| (the 1-norm, for the scaling of the series),
// out[1] = sum_g bg_g^2 in the reference's order (the propagators' logw).
__global__ void kp_norms_kernel(int n, const zd *Kp, int G, const double *bg, double *out)
{
    __shared__ double red[256];
    double m = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double c = 0.0;
        for (int i = 0; i < n; ++i) c += fabs(Kp[i + (size_t)n * j].x);
        m = fmax(m, c);
    }
    red[threadIdx.x] = m;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int g = 0; g < G; ++g) b += bg[g] * bg[g];
        out[0] = red[0];
        out[1] = b;
    }
}

// dst = scale * src + diag * I (n x n, column-major); src may be null (zero)
__global__ void scaled_plus_identity_kernel(int n, const zd *src, double scale, double diag, zd *dst)
{
    const long long n2 = (long long)n * n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n2;
         i += (long long)gridDim.x * blockDim.x) {
        zd v = src ? make_double2(scale * src[i].x, scale * src[i].y) : make_double2(0.0, 0.0);
        if (i % (n + 1) == 0) v.x += diag;
        dst[i] = v;
    }
}

// exp(-alpha Kp) into dst: the series of B = -alpha Kp / 2^s to order 16 by
// Horner's rule (X <- I + B X / j), then s squarings, with s the smallest
// power that brings ||B||_1 to 0.5 or below, where the truncated term is
// below 1e-19 relative.  The same matrix function as the reference's
// V exp(-alpha lambda) V^T from the eigensystem of Kp (returnExpMinusAlphaK,
// realMaterialMolecule.cpp:117-131), computed with GEMMs instead of an
// eigensolver.
int expm_series(afqmc_engine *e, const zd *Kp, double alpha, double kpNorm1, zd *dst, zd *B, zd *X, zd *Y)
{
    const int n = e->n;
    cudaStream_t s = e->stream;
    int sq = 0;
    while (std::fabs(alpha) * kpNorm1 > 0.5 * std::ldexp(1.0, sq) && sq < 60) ++sq;
    const int blocks = (int)std::min<long long>(1024, ((long long)n * n + 255) / 256);
    constexpr int ORDER = 16;
    g_launch_count += 2;
    scaled_plus_identity_kernel<<<blocks, 256, 0, s>>>(n, Kp, -alpha / std::ldexp(1.0, sq), 0.0, B);
    scaled_plus_identity_kernel<<<blocks, 256, 0, s>>>(n, B, 1.0 / ORDER, 1.0, X);
    TRY(check_launch());
    for (int j = ORDER - 1; j >= 1; --j) {
        g_launch_count++;
        scaled_plus_identity_kernel<<<blocks, 256, 0, s>>>(n, nullptr, 0.0, 1.0, Y);
        TRY(check_launch());
        ZGemmArgs g;
        g.m = n; g.n = n; g.k = n;
        g.alpha = make_double2(1.0 / j, 0.0); g.beta = make_double2(1.0, 0.0);
        g.A = B; g.lda = n; g.B = X; g.ldb = n; g.C = Y; g.ldc = n;
        TRY(gemm(g, s));
        std::swap(X, Y);
    }
    for (int q = 0; q < sq; ++q) {
        ZGemmArgs g;
        g.m = n; g.n = n; g.k = n;
        g.A = X; g.lda = n; g.B = X; g.ldb = n; g.C = Y; g.ldc = n;
        TRY(gemm(g, s));
        std::swap(X, Y);
    }
    CUDA_TRY(cudaMemcpyAsync(dst, X, sizeof(zd) * n * n, cudaMemcpyDeviceToDevice, s));
    return AFQMC_OK;
}

}  // namespace

int afqmc_pl_rebuild_propagators(afqmc_engine *e, const double *K)
{
    if (!e || e->kind != KIND_PL || !K) return fail(AFQMC_ERR_ARG, "phaseless engine and K required");
    const int n = e->n, G = e->G;
    const size_t n2 = (size_t)n * n;
    if (!e->kin) TRY(dalloc(e, &e->kin, n2));
    if (!e->propScratch) TRY(dalloc(e, &e->propScratch, 4 * n2));
    if (!e->propNorms) TRY(dalloc(e, &e->propNorms, 2));
    if (!e->expK[0]) TRY(dalloc(e, &e->expK[0], n2));
    drop_graphs(e);
    cudaStream_t s = e->stream;
    CUDA_TRY(cudaMemcpyAsync(e->kin, K, sizeof(double) * n2, cudaMemcpyHostToDevice, s));
    zd *Kp = e->propScratch, *B = Kp + n2, *X = B + n2, *Y = X + n2;
    g_launch_count += 2;
    kp_build_kernel<<<(int)std::min<size_t>(1024, (n2 + 255) / 256), 256, 0, s>>>((long long)n2, G, e->kin,
                                                                                  e->chol, e->bg, Kp);
    kp_norms_kernel<<<1, 256, 0, s>>>(n, Kp, G, e->bg, e->propNorms);
    TRY(check_launch());
    double h[2] = {0.0, 0.0};
    CUDA_TRY(cudaMemcpyAsync(h, e->propNorms, sizeof(h), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (!std::isfinite(h[0]) || !std::isfinite(h[1])) return fail(AFQMC_ERR_ARG, "non-finite K + sum_g bg_g L_g");
    // afqmcPhaseless.cpp:151-177: expMinusDtK, expMinusHalfDtK and expHalfDtK,
    // each with logw = alpha * 0.5 * sum bg^2
    const double alphas[3] = {e->dt, -0.5 * e->dt, 0.5 * e->dt};   // slots 0, 1 (expHalfDtK), 2
    for (int k = 0; k < 3; ++k) {
        TRY(expm_series(e, Kp, alphas[k], h[0], e->expK[k], B, X, Y));
        e->expLogw[k] = make_double2(alphas[k] * 0.5 * h[1], 0.0);
    }
    e->useLog = false;
    if (e->precision == AFQMC_MIXED) TRY(mixed_update_operators(e));
    CUDA_TRY(cudaStreamSynchronize(s));
    return AFQMC_OK;
}

int afqmc_log_overlaps(afqmc_engine *e, double *out)
{
    if (!e || !out) return fail(AFQMC_ERR_ARG, "null argument");
    if (e->precision == AFQMC_MIXED) TRY(mixed_sync_to_fp64(e));
    TRY(overlap_gemm(e, e->wf, nullptr, e->bl));
    launch_lu_logdet_inverse(e->W, e->bl, e->S, nullptr, nullptr, e->logw, make_double2(0, 0),
                             e->logwT, e->logov, nullptr, nullptr, nullptr, nullptr, nullptr,
                             LU_PLAIN, false, e->stream);
    TRY(check_launch());
    CUDA_TRY(cudaMemcpyAsync(out, e->logov, sizeof(zd) * e->W, cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return AFQMC_OK;
}

int afqmc_green_matrix(afqmc_engine *e, int walker, int spin, double *out)
{
    if (!e || !out || walker < 0 || walker >= e->W) return fail(AFQMC_ERR_ARG, "bad argument");
    if (spin < 0 || spin >= e->bl.nblk) return fail(AFQMC_ERR_ARG, "bad spin");
    if (e->precision == AFQMC_MIXED) TRY(mixed_sync_to_fp64(e));
    TRY(overlap_gemm(e, e->wf, nullptr, e->bl));
    launch_lu_logdet_inverse(e->W, e->bl, e->S, e->Sinv, nullptr, e->logw, make_double2(0, 0),
                             e->logwT, e->logov, nullptr, nullptr, nullptr, nullptr, nullptr,
                             LU_PLAIN, true, e->stream);
    TRY(check_launch());
    TRY(theta_gemm(e, e->wf, nullptr, e->bl));
    // G^T = thetaT^T phiT^H, i.e. G = conj(phiT) thetaT transposed back on the host
    const int n = e->n, Ns = e->bl.Ns[spin];
    std::vector<zd> h((size_t)n * n);
    zd *scratch = nullptr;
    TRY(dalloc(e, &scratch, (size_t)n * n));
    ZGemmArgs g;
    g.m = n; g.n = n; g.k = Ns; g.opA = OP_T; g.opB = OP_C;
    g.A = e->thetaT + (size_t)walker * e->bl.tStride + e->bl.tOff[spin]; g.lda = Ns;
    g.B = e->phiT[spin]; g.ldb = n;
    g.C = scratch; g.ldc = n;
    TRY(gemm(g, e->stream));
    CUDA_TRY(cudaMemcpyAsync(h.data(), scratch, sizeof(zd) * n * n, cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    cudaFree(scratch);
    e->allocs.pop_back();
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            zd v = h[j + (size_t)n * i];
            out[2 * (i + (size_t)n * j)] = v.x;
            out[2 * (i + (size_t)n * j) + 1] = v.y;
        }
    return AFQMC_OK;
}

int afqmc_taylor_stats(afqmc_engine *e, long long *calls, long long *total, int *min_order,
                       int *max_order)
{
    if (!e) return fail(AFQMC_ERR_ARG, "null engine");
    long long s[4];
    CUDA_TRY(cudaMemcpyAsync(s, e->tstats, sizeof(s), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    if (calls) *calls = s[0];
    if (total) *total = s[1];
    if (min_order) *min_order = (int)std::min<long long>(s[2], 1 << 30);
    if (max_order) *max_order = (int)s[3];
    return AFQMC_OK;
}

int afqmc_status(afqmc_engine *e, int *status_or)
{
    if (!e || !status_or) return fail(AFQMC_ERR_ARG, "null argument");
    std::vector<int> st(e->W + 1);
    CUDA_TRY(cudaMemcpyAsync(st.data(), e->status, sizeof(int) * (e->W + 1), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    int o = 0;
    for (int v : st) o |= v;
    if (e->mx || e->cpm) o |= mixed_status(e);
    *status_or = o;
    return AFQMC_OK;
}

long long afqmc_launch_count(void) { return g_launch_count.load(); }

int afqmc_set_graphs(afqmc_engine *e, int enable)
{
    if (!e) return fail(AFQMC_ERR_ARG, "null engine");
    if (!enable) drop_graphs(e);
    e->useGraphs = enable != 0;
    return AFQMC_OK;
}

int afqmc_profile_enable(afqmc_engine *e, int on)
{
    if (!e) return fail(AFQMC_ERR_ARG, "null engine");
    prof_resolve(e);
    e->prof = on != 0;
    for (int i = 0; i < AFQMC_NPHASES; ++i) { e->profMs[i] = 0.0; e->profCount[i] = 0; }
    return AFQMC_OK;
}

int afqmc_profile_get(afqmc_engine *e, double *ms, long long *counts)
{
    if (!e) return fail(AFQMC_ERR_ARG, "null engine");
    prof_resolve(e);
    for (int i = 0; i < AFQMC_NPHASES; ++i) {
        if (ms) ms[i] = e->profMs[i];
        if (counts) counts[i] = e->profCount[i];
    }
    return AFQMC_OK;
}

int afqmc_gemm_bf16_dev(int M, int N, int K, const void *A, long long lda, const void *B,
                        long long ldb, void *C, long long ldc, int out_bf16, int splits,
                        long long split_stride, float alpha, void *stream)
{
    if (M < 0 || N < 0 || K <= 0 || !A || !B || !C || splits < 1) return fail(AFQMC_ERR_ARG, "bad argument");
    if (splits > 1 && (K % (64 * splits)) != 0) return fail(AFQMC_ERR_ARG, "K must split into multiples of 64");
    int *derr = nullptr;
    TRY(device_error_word(&derr));
    cudaStream_t s = (cudaStream_t)stream;
    CUDA_TRY(cudaMemsetAsync(derr, 0, sizeof(int), s));
    TcGemmArgs a;
    a.M = M; a.N = N; a.K = K;
    a.A = (const __nv_bfloat16 *)A; a.lda = lda;
    a.B = (const __nv_bfloat16 *)B; a.ldb = ldb;
    a.C = C; a.ldc = ldc; a.outType = out_bf16 ? TC_OUT_BF16 : TC_OUT_F32;
    a.splits = splits; a.splitStride = split_stride; a.alpha = alpha; a.err = derr;
    int r = tc_gemm_bf16(a, s);
    if (r) return fail(AFQMC_ERR_CUDA, "tcgen05 gemm launch failed: " + std::to_string(r));
    int h = 0;
    CUDA_TRY(cudaMemcpyAsync(&h, derr, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (h) return fail(AFQMC_ERR_CUDA, "tcgen05 gemm: barrier wait timed out");
    return AFQMC_OK;
}

int afqmc_bounded_wait_check(long long limit_cycles, int *error_word, void *stream)
{
    if (!error_word) return fail(AFQMC_ERR_ARG, "null argument");
    if (limit_cycles < 1000) limit_cycles = 1000;
    if (limit_cycles > TC_WAIT_LIMIT_CYCLES) limit_cycles = TC_WAIT_LIMIT_CYCLES;
    int *derr = nullptr;
    TRY(device_error_word(&derr));
    cudaStream_t s = (cudaStream_t)stream;
    CUDA_TRY(cudaMemsetAsync(derr, 0, sizeof(int), s));
    int r = tc_bounded_wait_check(limit_cycles, derr, s);
    if (r) return fail(AFQMC_ERR_CUDA, "bounded-wait check launch failed: " + std::to_string(r));
    CUDA_TRY(cudaMemcpyAsync(error_word, derr, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return AFQMC_OK;
}

int afqmc_set_autotune(int enable)
{
    zgemm_set_autotune(enable);
    return AFQMC_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ batches
// Several engines (e.g. lattices of different size and filling) advanced
// together: each step is one graph with one branch per engine, each branch
// on that engine's stream, forked from and joined to the batch stream.
struct afqmc_batch {
    std::vector<afqmc_engine *> engines;
    std::vector<cudaEvent_t> joins;
    cudaEvent_t fork = nullptr;
    cudaStream_t stream = nullptr, own = nullptr;
    cudaGraphExec_t exec[4] = {nullptr, nullptr, nullptr, nullptr};
    long long kernels[4] = {0, 0, 0, 0};
    bool warm = false;
};

namespace {
void batch_drop(afqmc_batch *b)
{
    for (auto &g : b->exec)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    b->warm = false;
}
}  // namespace

extern "C" {

int afqmc_batch_create(afqmc_engine **engines, int count, afqmc_batch **out)
{
    if (!engines || count <= 0 || !out) return fail(AFQMC_ERR_ARG, "bad argument");
    for (int i = 0; i < count; ++i) {
        if (!engines[i]) return fail(AFQMC_ERR_ARG, "null engine in batch");
        if (engines[i]->mgsStep != engines[0]->mgsStep || engines[i]->popStep != engines[0]->popStep ||
            engines[i]->mgsIndex != engines[0]->mgsIndex || engines[i]->popIndex != engines[0]->popIndex)
            return fail(AFQMC_ERR_ARG, "engines of a batch must share the stabilisation and population-control cadence");
    }
    afqmc_batch *b = new afqmc_batch();
    b->engines.assign(engines, engines + count);
    cudaError_t r = cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking);
    b->stream = b->own;
    if (r == cudaSuccess) r = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    b->joins.resize(count, nullptr);
    for (int i = 0; i < count && r == cudaSuccess; ++i)
        r = cudaEventCreateWithFlags(&b->joins[i], cudaEventDisableTiming);
    if (r != cudaSuccess) { delete b; return fail(AFQMC_ERR_CUDA, cudaGetErrorString(r)); }
    *out = b;
    return AFQMC_OK;
}

int afqmc_batch_destroy(afqmc_batch *b)
{
    if (!b) return AFQMC_OK;
    cudaStreamSynchronize(b->stream);
    batch_drop(b);
    for (cudaEvent_t ev : b->joins) if (ev) cudaEventDestroy(ev);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->own) cudaStreamDestroy(b->own);
    delete b;
    return AFQMC_OK;
}

int afqmc_batch_step(afqmc_batch *b, int nsteps)
{
    if (!b) return fail(AFQMC_ERR_ARG, "null batch");
    for (int s = 0; s < nsteps; ++s) {
        afqmc_engine *e0 = b->engines[0];
        const bool doMgs = (e0->mgsIndex + 1 == e0->mgsStep);
        const bool doPop = (e0->popIndex + 1 == e0->popStep);
        const int key = (doMgs ? 1 : 0) | (doPop ? 2 : 0);
        bool profiling = false;
        for (auto *e : b->engines) profiling |= e->prof;
        if (!b->warm || profiling) {
            // first step direct: one-time launcher setup and autotuning happen
            // here; the profiler also needs direct launches
            for (size_t i = 0; i < b->engines.size(); ++i) {
                afqmc_engine *e = b->engines[i];
                CUDA_TRY(cudaEventRecord(b->fork, b->stream));
                CUDA_TRY(cudaStreamWaitEvent(e->stream, b->fork, 0));
                TRY(project_one_step_direct(e));
                CUDA_TRY(cudaEventRecord(b->joins[i], e->stream));
                CUDA_TRY(cudaStreamWaitEvent(b->stream, b->joins[i], 0));
            }
            if (!b->warm)
                for (auto *e : b->engines) CUDA_TRY(cudaStreamSynchronize(e->stream));
            b->warm = true;
            continue;
        }
        if (!b->exec[key]) {
            cudaGraph_t g = nullptr;
            CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            const long long c0 = g_launch_count.load();
            int r = AFQMC_OK;
            cudaEventRecord(b->fork, b->stream);
            for (size_t i = 0; i < b->engines.size() && r == AFQMC_OK; ++i) {
                afqmc_engine *e = b->engines[i];
                cudaStreamWaitEvent(e->stream, b->fork, 0);
                r = project_dtk_dtv(e);
                if (r == AFQMC_OK && doMgs) r = modify_gm(e);
                if (r == AFQMC_OK && doPop) r = pop_control(e);
                cudaEventRecord(b->joins[i], e->stream);
                cudaStreamWaitEvent(b->stream, b->joins[i], 0);
            }
            b->kernels[key] = g_launch_count.load() - c0;
            g_launch_count -= b->kernels[key];
            cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
            if (r != AFQMC_OK) { if (g) cudaGraphDestroy(g); return r; }
            if (ce != cudaSuccess) return fail(AFQMC_ERR_CUDA, std::string("batch capture: ") + cudaGetErrorString(ce));
            ce = cudaGraphInstantiate(&b->exec[key], g, 0);
            cudaGraphDestroy(g);
            if (ce != cudaSuccess) return fail(AFQMC_ERR_CUDA, std::string("batch instantiate: ") + cudaGetErrorString(ce));
        }
        // order the graph after work already queued on the engines' streams,
        // and later work on those streams after the graph
        for (size_t i = 0; i < b->engines.size(); ++i) {
            CUDA_TRY(cudaEventRecord(b->joins[i], b->engines[i]->stream));
            CUDA_TRY(cudaStreamWaitEvent(b->stream, b->joins[i], 0));
        }
        CUDA_TRY(cudaGraphLaunch(b->exec[key], b->stream));
        g_launch_count += b->kernels[key];
        CUDA_TRY(cudaEventRecord(b->fork, b->stream));
        for (auto *e : b->engines) CUDA_TRY(cudaStreamWaitEvent(e->stream, b->fork, 0));
        for (auto *e : b->engines) {
            e->mgsIndex = doMgs ? 0 : e->mgsIndex + 1;
            e->popIndex = doPop ? 0 : e->popIndex + 1;
        }
    }
    return AFQMC_OK;
}

int afqmc_batch_set_stream(afqmc_batch *b, void *cuda_stream)
{
    if (!b) return fail(AFQMC_ERR_ARG, "null batch");
    if (!cuda_stream) return fail(AFQMC_ERR_ARG, "null stream");
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    if (b->own) { cudaStreamDestroy(b->own); b->own = nullptr; }
    b->stream = (cudaStream_t)cuda_stream;
    return AFQMC_OK;
}

int afqmc_batch_synchronize(afqmc_batch *b)
{
    if (!b) return fail(AFQMC_ERR_ARG, "null batch");
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    for (auto *e : b->engines) CUDA_TRY(cudaStreamSynchronize(e->stream));
    return AFQMC_OK;
}

int afqmc_pop_configuration_host(int L, int size, const double *weight, const double *uniforms,
                                 int *table)
{
    if (L <= 0 || size <= 0 || L % size != 0 || !weight || !uniforms || !table)
        return fail(AFQMC_ERR_ARG, "need L > 0 divisible by size and non-null arrays");
    const int Lc = L / size;
    double sum = 0.0;
    for (int i = 0; i < L; ++i) sum += weight[i];
    std::vector<int> number(L, 0);
    int index_old = 0;
    double prob_sum_old = weight[0] / sum;
    for (int i = 0; i < L; ++i) {
        double prob_sum_new = (i + uniforms[i]) / (L * 1.0);
        while (prob_sum_new > prob_sum_old && index_old < L - 1) {
            index_old++;
            prob_sum_old += weight[index_old] / sum;
        }
        number[index_old]++;
    }
    for (int i = 0; i < L; ++i) table[i] = number[i] != 0 ? i : -1;
    auto fill = [&](int lo, int hi) {
        int zero_i = lo, one_i = lo;
        while (zero_i < hi && number[zero_i] != 0) zero_i++;
        while (one_i < hi && number[one_i] <= 1) one_i++;
        while (zero_i < hi && one_i < hi) {
            table[zero_i] = one_i; number[zero_i]++; number[one_i]--;
            while (zero_i < hi && number[zero_i] != 0) zero_i++;
            while (one_i < hi && number[one_i] <= 1) one_i++;
        }
    };
    for (int c = 0; c < size; ++c) fill(Lc * c, Lc * (c + 1));
    if (size > 1) fill(0, L);
    for (int i = 0; i < L; ++i)
        if (number[i] != 1) return fail(AFQMC_ERR_STATE, "population configuration left a slot unfilled");
    return AFQMC_OK;
}

int afqmc_pop_weights(afqmc_engine *e, double *weight_out)
{
    if (!e || !weight_out) return fail(AFQMC_ERR_ARG, "null argument");
    if (e->precision == AFQMC_MIXED) {
        TRY(mixed_pop_weights(e));
    } else {
        TRY(overlap_gemm(e, e->wf, e->alive, fbl(e)));
        launch_lu_logdet_inverse(e->W, fbl(e), e->S, nullptr, e->alive, e->logw, make_double2(0, 0),
                                 e->logwT, e->logov, e->alive, nullptr, e->logw, e->weight, e->status,
                                 LU_POPWEIGHT, false, e->stream);
        TRY(check_launch());
    }
    CUDA_TRY(cudaMemcpyAsync(weight_out, e->weight, sizeof(double) * e->W, cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return AFQMC_OK;
}

long long afqmc_walker_bytes(afqmc_engine *e)
{
    if (!e) return -1;
    return (long long)sizeof(zd) * (e->wsize + 1);
}

int afqmc_copy_walker_out(afqmc_engine *e, int w, void *dst_dev)
{
    if (!e || !dst_dev || w < 0 || w >= e->W) return fail(AFQMC_ERR_ARG, "bad argument");
    if (e->precision == AFQMC_MIXED) TRY(mixed_sync_to_fp64(e));
    CUDA_TRY(cudaMemcpyAsync(dst_dev, e->wf + (size_t)w * e->wsize, sizeof(zd) * e->wsize,
                             cudaMemcpyDeviceToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync((zd *)dst_dev + e->wsize, e->logw + w, sizeof(zd), cudaMemcpyDeviceToDevice,
                             e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return AFQMC_OK;
}

int afqmc_copy_walker_in(afqmc_engine *e, int w, const void *src_dev)
{
    if (!e || !src_dev || w < 0 || w >= e->W) return fail(AFQMC_ERR_ARG, "bad argument");
    if (e->precision == AFQMC_MIXED) TRY(mixed_sync_to_fp64(e));
    CUDA_TRY(cudaMemcpyAsync(e->wf + (size_t)w * e->wsize, src_dev, sizeof(zd) * e->wsize,
                             cudaMemcpyDeviceToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync(e->logw + w, (const zd *)src_dev + e->wsize, sizeof(zd), cudaMemcpyDeviceToDevice,
                             e->stream));
    if (e->precision == AFQMC_MIXED) TRY(mixed_sync_from_fp64(e));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return AFQMC_OK;
}

namespace {
int walker_xfer(afqmc_engine *e, int count, const int *idx, zd *buf, bool unpack)
{
    if (!e || count < 0 || (count > 0 && (!idx || !buf)) || count > e->W) return fail(AFQMC_ERR_ARG, "bad argument");
    if (count == 0) return AFQMC_OK;
    std::vector<char> seen(e->W, 0);
    for (int k = 0; k < count; ++k) {
        if (idx[k] < 0 || idx[k] >= e->W) return fail(AFQMC_ERR_ARG, "walker index out of range");
        if (unpack && seen[idx[k]]++) return fail(AFQMC_ERR_ARG, "a slot appears twice in the unpack list");
    }
    CUDA_TRY(cudaMemcpyAsync(e->table, idx, sizeof(int) * count, cudaMemcpyHostToDevice, e->stream));
    if (e->precision == AFQMC_MIXED) TRY(mixed_sync_to_fp64(e));
    launch_walker_xfer(count, e->wsize, e->table, e->wf, e->logw, buf, unpack, e->stream);
    TRY(check_launch());
    if (unpack && e->precision == AFQMC_MIXED) TRY(mixed_sync_from_fp64(e));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return AFQMC_OK;
}
}  // namespace

int afqmc_pack_walkers(afqmc_engine *e, int count, const int *idx, void *dst_dev)
{
    return walker_xfer(e, count, idx, (zd *)dst_dev, false);
}

int afqmc_unpack_walkers(afqmc_engine *e, int count, const int *slots, const void *src_dev)
{
    return walker_xfer(e, count, slots, (zd *)const_cast<void *>(src_dev), true);
}

int afqmc_apply_table(afqmc_engine *e, const int *table)
{
    if (!e || !table) return fail(AFQMC_ERR_ARG, "null argument");
    for (int i = 0; i < e->W; ++i)
        if (table[i] < 0 || table[i] >= e->W) return fail(AFQMC_ERR_ARG, "table entry out of range");
    CUDA_TRY(cudaMemcpyAsync(e->table, table, sizeof(int) * e->W, cudaMemcpyHostToDevice, e->stream));
    if (e->precision == AFQMC_MIXED) {
        TRY(mixed_sync_to_fp64(e));
        launch_pop_gather(e->W, e->wsize, e->table, e->wf, e->logw, e->stream);
        TRY(mixed_sync_from_fp64(e));
    } else {
        launch_pop_gather(e->W, e->wsize, e->table, e->wf, e->logw, e->stream);
    }
    TRY(check_launch());
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return AFQMC_OK;
}

int afqmc_pop_configuration_dev(int W, const double *weights, const double *uniforms, int *table,
                                void *stream)
{
    if (W <= 0 || !weights || !uniforms || !table) return fail(AFQMC_ERR_ARG, "bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    int *number = nullptr;
    CUDA_TRY(cudaMallocAsync(&number, sizeof(int) * W, s));
    launch_pop_comb(W, weights, uniforms, 0, nullptr, number, table, nullptr, s);
    int r = check_launch();
    CUDA_TRY(cudaFreeAsync(number, s));
    return r;
}

}  // extern "C"
