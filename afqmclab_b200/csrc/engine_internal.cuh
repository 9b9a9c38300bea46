// Internal state of an engine handle (shared by engine.cu and mixed.cu).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/afqmc_b200.h"
#include "common.cuh"
#include "walker_kernels.cuh"
#include "zgemm.cuh"

struct MixedState;
struct CpMixedState;
struct ExF64Scratch;
struct BPState;

enum { KIND_CP = 0, KIND_PL = 1 };

struct afqmc_engine {
    int kind = 0;
    int n = 0, ncol = 0, nup = 0, ndn = 0, W = 0, L = 0, G = 0;
    int precision = AFQMC_FP64;
    int decomp = 0, forceType = 0;
    double dt = 0, ET = 0, forceCap = 0;
    int mgsStep = 1, popStep = 1, mgsIndex = 0, popIndex = 0;
    uint64_t seed = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    // asynchronous population upload: copy stream, two device staging slots
    cudaStream_t upStream = nullptr;
    cudaEvent_t upReady[2] = {nullptr, nullptr}, upFree[2] = {nullptr, nullptr};
    zd *stgWf[2] = {nullptr, nullptr}, *stgLw[2] = {nullptr, nullptr};
    float *stgWf32[2] = {nullptr, nullptr};   // fp32 walkers of the phaseless mixed form
    int *stgAl[2] = {nullptr, nullptr};
    int upNext = 0;
    Blocks bl{};
    long long wsize = 0;
    zd logwT{0, 0};
    zd *phiT[2] = {nullptr, nullptr};
    // population and workspaces
    zd *wf = nullptr, *wfTmp = nullptr, *term[2] = {nullptr, nullptr}, *logw = nullptr,
       *logov = nullptr, *S = nullptr, *Sinv = nullptr, *thetaT = nullptr;
    int *alive = nullptr, *surv = nullptr, *status = nullptr, *done = nullptr, *order = nullptr,
        *table = nullptr, *number = nullptr;
    unsigned long long *counter = nullptr, *offs = nullptr;
    double *weight = nullptr;
    long long *tstats = nullptr;
    // one-body operators: 0 exp(-dt K), 1 exp(+dt/2 K), 2 exp(-dt/2 K)
    zd *expK[3] = {nullptr, nullptr, nullptr};
    zd expLogw[3] = {{0, 0}, {0, 0}, {0, 0}};
    bool useLog = false;
    zd *logK = nullptr;
    // propagator rebuild on the GPU: K (n x n), scratch Kp and three Taylor
    // matrices (n x n each), the 1-norm of Kp and sum bg^2
    double *kin = nullptr, *propNorms = nullptr;
    zd *propScratch = nullptr;
    zd logKLogw{0, 0};
    // Hubbard
    HubbardDev hd{};
    zd *gamma = nullptr, *cdiag[4] = {nullptr, nullptr, nullptr, nullptr};
    double *U = nullptr, *mu = nullptr, *hx = nullptr, *hy = nullptr, *hz = nullptr,
           *constForceCP = nullptr, *forceCP = nullptr;
    zd *wfDaggerK = nullptr;
    // phaseless
    CholDev cdv{};
    double *chol = nullptr, *bg = nullptr, *tdev = nullptr;
    zd *Aall = nullptr, *wfDaggerT = nullptr, *xbar = nullptr, *forcePL = nullptr, *aux = nullptr,
       *M = nullptr, *ex = nullptr, *constForcePL = nullptr;
    long long Ktot = 0;
    // measurement
    zd *acc = nullptr, *bgNum = nullptr, *exNum = nullptr, *eloc = nullptr, *den = nullptr,
       *parts = nullptr;
    // constrained path: per-walker site terms (G_ii up, G_ii down, the two
    // spin-flip off-diagonals; W x 4L) and their den-weighted sums (4L)
    zd *sites = nullptr, *siteNum = nullptr;
    // constrained path, observe estimator (off unless enabled): each walker's
    // full Green's matrix (W x n x n), conj(phiT) and the den-weighted sums
    // (greenMatrixNum, densityDensityNum: n x n; S+S-, S-S+, pair: L x L)
    bool observe = false;
    zd *Gfull = nullptr, *phiTc = nullptr, *obs = nullptr;
    // back-propagation (constrained path, FP64 form; off unless begun) and the
    // model's K (2L x 2L), which the back-propagated estimator needs
    BPState *bp = nullptr;
    zd *Kmat = nullptr;
    // FP64 form: closed-shell single block and GEMM exchange (real A)
    ExF64Scratch *exf = nullptr;
    // mixed-precision state
    MixedState *mx = nullptr;
    CpMixedState *cpm = nullptr;   // constrained-path mixed form
    // phase profiler (CUDA events on the engine stream; off unless enabled)
    bool prof = false;
    struct Mark { int phase; cudaEvent_t a, b; };
    std::vector<Mark> marks;
    std::vector<cudaEvent_t> evpool;
    double profMs[AFQMC_NPHASES] = {};
    long long profCount[AFQMC_NPHASES] = {};
    // CUDA graphs of the step, one per cadence variant (bit 0: modifyGM,
    // bit 1: popControl), and of the measurement (index 4)
    bool useGraphs = false;
    bool graphWarm = false, measWarm = false;
    cudaGraphExec_t graphExec[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    long long graphKernels[5] = {0, 0, 0, 0, 0};  // kernel nodes per graph
    std::vector<void *> allocs;
};

// Phase timing: record an event pair around a phase when profiling is on.
struct PhaseScope {
    afqmc_engine *e; int phase; cudaEvent_t a = nullptr;
    PhaseScope(afqmc_engine *e_, int p) : e(e_), phase(p)
    {
        if (!e->prof) return;
        if (e->evpool.empty()) cudaEventCreate(&a); else { a = e->evpool.back(); e->evpool.pop_back(); }
        cudaEventRecord(a, e->stream);
    }
    ~PhaseScope()
    {
        if (!e->prof) return;
        cudaEvent_t b;
        if (e->evpool.empty()) cudaEventCreate(&b); else { b = e->evpool.back(); e->evpool.pop_back(); }
        cudaEventRecord(b, e->stream);
        e->marks.push_back({phase, a, b});
    }
};
#define PHASE(p) PhaseScope _ps_##p(e, p)

inline void prof_resolve(afqmc_engine *e)
{
    if (e->marks.empty()) return;
    cudaStreamSynchronize(e->stream);
    for (auto &m : e->marks) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, m.a, m.b);
        e->profMs[m.phase] += ms;
        e->profCount[m.phase] += 1;
        e->evpool.push_back(m.a);
        e->evpool.push_back(m.b);
    }
    e->marks.clear();
}


// helpers implemented in engine.cu
int engine_fail(int code, const std::string &msg);
int engine_check_launch();
int engine_gemm(const ZGemmArgs &a, cudaStream_t s);
template <class T> int engine_dalloc(afqmc_engine *e, T **p, size_t count);
zd engine_one_body_logw(afqmc_engine *e, int which);
// Local energy of the phaseless engine at the current walkers (logov, Sinv,
// thetaT, xbar, eloc, den); the exchange form is one of PL_EX_*.
enum { PL_EX_BLOCKWISE = 0, PL_EX_GEMM_ONE = 1, PL_EX_GEMM_ALL = 2 };
int engine_pl_local_energy(afqmc_engine *e, int exchange);
