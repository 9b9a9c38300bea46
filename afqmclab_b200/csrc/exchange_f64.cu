// Exchange term of the phaseless mixed estimator in FP64 as dense GEMMs, for
// real half-rotated Cholesky vectors A_g (real trial, real L_g): the FP64
// form of the quadratic-form algorithm of exchange_gemm.cu, so that the two
// precision forms compute the same thing the same way.  Per spin block
// (Ns electrons, n orbitals, K = Ns n) and walker w, in the thetaT index
// order q = a + Ns i, with u_w(q) = thetaT_w(a, i) and x_g(q) = A_g(a, i):
//
//   sum_g ex[g, w] = sum_g tr(D_gw D_gw) = u_w^T V u_w,
//       V(b + Ns i, a + Ns j) = sum_g A_g(a, i) A_g(b, j) = C(a + Ns i, b + Ns j),
//       C = X X^T (K x K, real, built once)
//   exNum[g] += sum_w den_w ex[g, w] = x_g^T R x_g,
//       R(a + Ns i, b + Ns j) = M(b + Ns i, a + Ns j),  M = sum_w den_w u_w u_w^T
//
// calculateCholeskyEx (afqmc/model/realMaterialMolecule/source/
// realMaterialMoleculeMeasureFixedSD2sSD2is.cpp:258-284) forms D_gw block by
// block; the energy needs only the sum over g and the per-vector
// accumulator only the den-weighted sum over walkers.  Three FP64 GEMMs per
// block: Z = V U (real x complex, K x W), M = U_den U^T (complex, K x K) and
// Y = R X (complex x real, K x G), each followed by a dot.
#include <algorithm>
#include <atomic>
#include <string>

#include "engine_internal.cuh"
#include "exchange_f64.cuh"
#include "zgemm.cuh"

extern std::atomic<long long> g_launch_count;

namespace {

// X(q, g) = Re A_g(a, i), q = a + Ns i (the block's rows of Aall, column g)
__global__ void xf64_kernel(long long K, int G, long long Ktot, long long tOff, const zd *Aall, double *X)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < K * G;
         e += (long long)gridDim.x * blockDim.x) {
        const long long q = e % K, g = e / K;
        X[e] = Aall[(size_t)g * Ktot + tOff + q].x;
    }
}

// V(q1, q2) = Re C(a + Ns i, b + Ns j) with q1 = b + Ns i, q2 = a + Ns j
__global__ void vf64_kernel(long long K, int Ns, const zd *C, double *V)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < K * K;
         e += (long long)gridDim.x * blockDim.x) {
        const long long q1 = e % K, q2 = e / K;
        const long long b = q1 % Ns, i = q1 / Ns, a = q2 % Ns, j = q2 / Ns;
        V[e] = C[(size_t)(a + Ns * i) + (size_t)K * (b + Ns * j)].x;
    }
}

// exTot[w] (+)= mult sum_q u_w(q) Z(q, w) for alive walkers
__global__ void __launch_bounds__(256)
ex_walker_dot_kernel(long long K, const zd *U, long long ldu, const zd *Z, const int *alive, int mult,
                     int accumulate, zd *exTot)
{
    __shared__ double red[32];
    const int w = blockIdx.x;
    if (!alive[w]) return;
    const zd *u = U + (size_t)w * ldu;
    const zd *z = Z + (size_t)w * K;
    zd s = make_double2(0.0, 0.0);
    for (long long q = threadIdx.x; q < K; q += blockDim.x) zfma(s, u[q], z[q]);
    s = block_zsum(s, red);
    if (threadIdx.x == 0) {
        s = zscale(s, (double)mult);
        exTot[w] = accumulate ? zadd(exTot[w], s) : s;
    }
}

// Uden(:, w) = exp(logov_w) u_w for alive walkers, 0 otherwise
__global__ void __launch_bounds__(256)
ex_scale_kernel(long long K, const zd *U, long long ldu, const zd *logov, const int *alive, zd *Uden)
{
    const int w = blockIdx.x;
    const zd d = alive[w] ? zexp(logov[w]) : make_double2(0.0, 0.0);
    const zd *u = U + (size_t)w * ldu;
    zd *o = Uden + (size_t)w * K;
    for (long long q = threadIdx.x; q < K; q += blockDim.x) o[q] = zmul(d, u[q]);
}

// R(a + Ns i, b + Ns j) = M(b + Ns i, a + Ns j); M is symmetric and only its
// lower triangle (row >= column) is read
__global__ void ex_exchange_kernel(long long K, int Ns, const zd *M, zd *R)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < K * K;
         e += (long long)gridDim.x * blockDim.x) {
        const long long q1 = e % K, q2 = e / K;
        const long long a = q1 % Ns, i = q1 / Ns, b = q2 % Ns, j = q2 / Ns;
        const long long r = b + Ns * i, c = a + Ns * j;
        R[e] = r >= c ? M[(size_t)r + (size_t)K * c] : M[(size_t)c + (size_t)K * r];
    }
}

// exNum[g] += mult sum_q x_g(q) Y(q, g)
__global__ void __launch_bounds__(256)
ex_vector_dot_kernel(long long K, const double *X, const zd *Y, int mult, zd *exNum)
{
    __shared__ double red[32];
    const int g = blockIdx.x;
    const double *x = X + (size_t)g * K;
    const zd *y = Y + (size_t)g * K;
    zd s = make_double2(0.0, 0.0);
    for (long long q = threadIdx.x; q < K; q += blockDim.x) {
        s.x = fma(x[q], y[q].x, s.x);
        s.y = fma(x[q], y[q].y, s.y);
    }
    s = block_zsum(s, red);
    if (threadIdx.x == 0) exNum[g] = zadd(exNum[g], zscale(s, (double)mult));
}

// xbar = alpha sum_s P_s (+ xbar when accumulating); P_s consecutive G x W blocks
__global__ void ex_force_sum_kernel(long long count, int S, const zd *P, zd alpha, int accumulate, zd *xbar)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
         e += (long long)gridDim.x * blockDim.x) {
        zd v = P[e];
        for (int s = 1; s < S; ++s) v = zadd(v, P[(size_t)s * count + e]);
        v = zmul(alpha, v);
        xbar[e] = accumulate ? zadd(xbar[e], v) : v;
    }
}

int gemm_check(const ZGemmArgs &a, cudaStream_t s)
{
    cudaError_t r = zgemm_batched(a, s);
    if (r != cudaSuccess) return engine_fail(AFQMC_ERR_CUDA, std::string("FP64 exchange GEMM: ") + cudaGetErrorString(r));
    return AFQMC_OK;
}

}  // namespace

int exf64_build(afqmc_engine *e, int b, ExF64 &x)
{
    const int Ns = e->bl.Ns[b], G = e->G;
    const long long K = (long long)Ns * e->n;
    x.b = b; x.Ns = Ns; x.K = K;
    int r;
    if ((r = engine_dalloc(e, &x.X, (size_t)K * G))) return r;
    if ((r = engine_dalloc(e, &x.V, (size_t)K * K))) return r;
    g_launch_count++;
    xf64_kernel<<<592, 256, 0, e->stream>>>(K, G, e->Ktot, e->bl.tOff[b], e->Aall, x.X);
    // C = X X^T into the shared K x K scratch, then V from it
    ZGemmArgs g;
    g.m = (int)K; g.n = (int)K; g.k = G;
    g.opA = OP_N; g.opB = OP_T; g.a_real = 1; g.b_real = 1;
    g.A = x.X; g.lda = K; g.B = x.X; g.ldb = K;
    g.C = e->exf->M; g.ldc = K;
    if ((r = gemm_check(g, e->stream))) return r;
    g_launch_count++;
    vf64_kernel<<<1184, 256, 0, e->stream>>>(K, Ns, e->exf->M, x.V);
    return engine_check_launch();
}

int exf64_alloc(afqmc_engine *e, long long Kmax, ExF64Scratch &s)
{
    int r;
    if ((r = engine_dalloc(e, &s.Z, (size_t)Kmax * e->W))) return r;
    if ((r = engine_dalloc(e, &s.M, (size_t)Kmax * Kmax))) return r;
    if ((r = engine_dalloc(e, &s.R, (size_t)Kmax * Kmax))) return r;
    if ((r = engine_dalloc(e, &s.Y, (size_t)Kmax * e->G))) return r;
    if ((r = engine_dalloc(e, &s.exTot, (size_t)e->W))) return r;
    // the force's output (G x W) may be too few 64 x 64 tiles for the SMs:
    // about four CTA slots' worth of work in partial products over K
    const long long tiles = (long long)((e->G + 63) / 64) * ((e->W + 63) / 64);
    int S = 1;
    while (S < 8 && tiles * S < 592) S *= 2;
    s.xsplit = S;
    if (S > 1 && (r = engine_dalloc(e, &s.xp, (size_t)S * e->G * e->W))) return r;
    return AFQMC_OK;
}

int exf64_force(afqmc_engine *e, const Blocks &bl)
{
    ExF64Scratch &s = *e->exf;
    const int G = e->G, W = e->W;
    bool first = true;
    int r;
    for (int b = 0; b < bl.nblk; ++b) {
        if (bl.Ns[b] == 0) continue;
        const ExF64 x = exf64_block(e, b);
        int S = s.xsplit;
        while (S > 1 && x.K % S) S /= 2;
        ZGemmArgs g;
        g.m = G; g.n = W; g.k = (int)(x.K / S);
        g.opA = OP_T; g.opB = OP_N; g.a_real = ST_R64;
        g.A = x.X; g.lda = x.K; g.strideA = x.K / S;
        g.B = e->thetaT + e->bl.tOff[b]; g.ldb = e->bl.tStride; g.strideB = x.K / S;
        const zd mult = make_double2((double)bl.mult, 0.0);
        if (S == 1) {
            g.C = e->xbar; g.ldc = G;
            g.alpha = mult;
            g.beta = first ? make_double2(0.0, 0.0) : make_double2(1.0, 0.0);
            if ((r = gemm_check(g, e->stream))) return r;
        } else {
            g.C = s.xp; g.ldc = G; g.strideC = (long long)G * W;
            g.batch = S;
            if ((r = gemm_check(g, e->stream))) return r;
            g_launch_count++;
            ex_force_sum_kernel<<<296, 256, 0, e->stream>>>((long long)G * W, S, s.xp, mult, first ? 0 : 1,
                                                           e->xbar);
            if ((r = engine_check_launch())) return r;
        }
        first = false;
    }
    return AFQMC_OK;
}

ExF64 exf64_block(const afqmc_engine *e, int b)
{
    ExF64 x = e->exf->blk[e->exf->restricted ? 0 : b];
    x.b = b;
    return x;
}

int exf64_walker_totals(afqmc_engine *e, const ExF64 &x, bool accumulate, int mult)
{
    ExF64Scratch &s = *e->exf;
    const long long K = x.K;
    const int W = e->W;
    const zd *U = e->thetaT + e->bl.tOff[x.b];
    const long long ldu = e->bl.tStride;
    cudaStream_t st = e->stream;
    int r;
    // Z = V U
    ZGemmArgs z;
    z.m = (int)K; z.n = W; z.k = (int)K; z.a_real = 1;
    z.A = x.V; z.lda = K; z.B = U; z.ldb = ldu; z.C = s.Z; z.ldc = K;
    if ((r = gemm_check(z, st))) return r;
    g_launch_count++;
    ex_walker_dot_kernel<<<W, 256, 0, st>>>(K, U, ldu, s.Z, e->alive, mult, accumulate ? 1 : 0, s.exTot);
    return engine_check_launch();
}

int exf64_pair_matrix(afqmc_engine *e, const ExF64 &x, const zd *Uden, const zd *Um)
{
    ExF64Scratch &s = *e->exf;
    const long long K = x.K;
    ZGemmArgs m;
    m.m = (int)K; m.n = (int)K; m.k = e->W; m.opA = OP_N; m.opB = OP_T;
    m.A = Uden; m.lda = K; m.B = Um; m.ldb = K; m.C = s.M; m.ldc = K;
    m.lower = 1;   // M = sum_w den_w u_w u_w^T is symmetric
    int r = gemm_check(m, e->stream);
    if (r) return r;
    g_launch_count++;
    ex_exchange_kernel<<<1184, 256, 0, e->stream>>>(K, x.Ns, s.M, s.R);
    return engine_check_launch();
}

int exf64_run(afqmc_engine *e, const ExF64 &x, bool accumulate, int mult)
{
    ExF64Scratch &s = *e->exf;
    const long long K = x.K;
    const int W = e->W, G = e->G;
    const zd *U = e->thetaT + e->bl.tOff[x.b];
    const long long ldu = e->bl.tStride;
    cudaStream_t st = e->stream;
    int r;
    if ((r = exf64_walker_totals(e, x, accumulate, mult))) return r;
    // M = U_den U^T  (U_den into Z)
    g_launch_count++;
    ex_scale_kernel<<<W, 256, 0, st>>>(K, U, ldu, e->logov, e->alive, s.Z);
    ZGemmArgs m;
    m.m = (int)K; m.n = (int)K; m.k = W; m.opA = OP_N; m.opB = OP_T;
    m.A = s.Z; m.lda = K; m.B = U; m.ldb = ldu; m.C = s.M; m.ldc = K;
    m.lower = 1;   // M = sum_w den_w u_w u_w^T is symmetric
    if ((r = gemm_check(m, st))) return r;
    g_launch_count++;
    ex_exchange_kernel<<<1184, 256, 0, st>>>(K, x.Ns, s.M, s.R);
    // Y = R X, exNum_g += x_g^T Y_g
    ZGemmArgs y;
    y.m = (int)K; y.n = G; y.k = (int)K; y.b_real = 1;
    y.A = s.R; y.lda = K; y.B = x.X; y.ldb = K; y.C = s.Y; y.ldc = K;
    if ((r = gemm_check(y, st))) return r;
    g_launch_count++;
    ex_vector_dot_kernel<<<G, 256, 0, st>>>(K, x.X, s.Y, mult, e->exNum);
    return engine_check_launch();
}
