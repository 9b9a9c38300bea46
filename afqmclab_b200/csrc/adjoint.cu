// Adjoint of the phaseless mixed estimator and of the mean log-overlap with
// respect to the one-body matrix t, the Cholesky vectors L_g and the trial
// orbitals (FP64, the current walkers held fixed).
//
// With theta_s = phi_s S_s^{-1} (S_s = phiT_s^H phi_s), Gamma_s = theta_s phiT_s^H
// (the transpose of the reference's mixed Green's function G_s,
// SDSDOperation.cpp:74-89), D_gs = A_gs theta_s (A_gs = phiT_s^H L_g) and
//   E_w = sum_s tr(t Gamma_s) + 1/2 sum_g [ xbar_g^2 - sum_s tr(D_gs D_gs) ]
//   E   = sum_w den_w E_w / sum_w den_w,  den_w = <phiT|phi_w>
// (RealMaterialMoleculeMeasureFixedSD2sSD2is::addEnergy, :197-284):
//   dE/dt      = [ sum_s R_s phiT_s^H ]^T / sum den,        R_s = sum_w den_w theta_s
//   dE/dL_g    = [ sum_s conj(phiT_s) Y_gs^T ] / sum den,
//                Y_gs = sum_w den_w theta_s Z_gs,  Z_gs = xbar_g I - D_gs
//   dE/dconj(phiT_s) = sum_w den_w [ V - theta (phiT^H V) + (E_w - E) theta ] / sum den,
//                V = t theta + sum_g L_g theta Z_g
//   d mean(log <phiT|phi_w>) / dconj(phiT_s) = mean_w theta_s
// E is a function of conj(phiT) only, so the orbital gradient is the
// conjugate Wirtinger derivative.  theta, S and D_g are recomputed for the
// current walkers instead of being stored from the propagation.
//
// Two forms compute these sums.
//
// GEMM form (real half-rotated vectors A_g, the FP64 exchange's operands of
// exchange_f64.cu): with u_w(b + Ns i) = theta_w(i, b), X(b + Ns i, g) =
// A_g(b, i), V = perm(X X^T) and R = perm(sum_w den_w u_w u_w^T) (the
// exchange's permutations), every sum over g or over walkers is one large
// GEMM:
//   Z = V U                     Z(b + Ns i, w)   = (sum_g D_gw A_g)(b, i)
//   phiT^H V_w = H_w theta_w,   H_w = phiT^H t + sum_g xbar_gw A_g - reshape(Z_w)
//   Y(b + Ns i, g) = Y_g(i, b) = (Uden xbar^T - R X)(b + Ns i, g)
//   sum_w den_w V_w = t R_s + sum_g L_g Y_g   (one split-K GEMM, K = n G)
//   sum_w den_w theta_w (phiT^H V_w) = sum_w theta_w (den_w H_w theta_w)
// about K^2 (3W + 2G) flops per block (K = Ns n) against the per-walker
// form's 4 W G n Ns (2 Ns + n).  A spin-restricted trial (both blocks the same
// orbitals; a walker's one orbital matrix serves both spins) computes block
// 0 alone and counts it twice, as the FP64 step does.
//
// Per-walker form (complex A): batched FP64 GEMMs over the G Cholesky
// vectors, one walker and spin at a time, working set O(G n Ns):
//   D_g (Ns x Ns)  = A_g theta                    batch over g
//   Z_g            = xbar_g I - D_g               elementwise
//   theta Z_g      -> Y'' ((g, i), b) rows        batch over g, then Y += den Y''
//   V partials     = L_g (theta Z_g)              batch over g, summed in g order
//   V             += t theta;  C = phiT^H V;  U = den [V - theta C + (E_w - E) theta]
// and, after the walkers, dE/dL_g = conj(phiT) Y_g^T for every g (one batch).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "engine_internal.cuh"
#include "exchange_f64.cuh"

namespace {

// R^T_s += den_w thetaT_s, the unweighted sum (log-overlap) and
// Et = sum_w den_w (E_w - E) thetaT_w
__global__ void adj_r_kernel(int W, long long Ktot, long long tStride, const zd *thetaT,
                             const int *alive, const zd *den, const zd *eloc, zd Emix, zd *Rt, zd *St,
                             zd *Et)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < Ktot;
         e += (long long)gridDim.x * blockDim.x) {
        zd r = make_double2(0, 0), q = make_double2(0, 0), t = make_double2(0, 0);
        for (int w = 0; w < W; ++w) {
            if (!alive[w]) continue;
            const zd x = thetaT[(size_t)w * tStride + e];
            zfma(r, den[w], x);
            q = zadd(q, x);
            zfma(t, zmul(den[w], zsub(eloc[w], Emix)), x);
        }
        Rt[e] = r;
        St[e] = q;
        Et[e] = t;
    }
}

// Um(:, w) = u_w, Uden(:, w) = den_w u_w for alive walkers, zero columns otherwise
__global__ void adj_mask_kernel(long long K, int W, const zd *U, long long ldu, const int *alive,
                                const zd *den, zd *Um, zd *Uden)
{
    const long long total = K * W;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int w = (int)(e / K);
        const long long q = e % K;
        zd u = make_double2(0, 0), d = make_double2(0, 0);
        if (alive[w]) {
            u = U[(size_t)w * ldu + q];
            d = zmul(den[w], u);
        }
        Um[e] = u;
        Uden[e] = d;
    }
}

// xbm(g, w) = xbar(g, w) for alive walkers, 0 otherwise (G x W)
__global__ void adj_xbm_kernel(long long count, int G, const zd *xbar, const int *alive, zd *xbm)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
         e += (long long)gridDim.x * blockDim.x)
        xbm[e] = alive[e / G] ? xbar[e] : make_double2(0, 0);
}

// H(q, w) = den_w [Tt(q) + XB(q, w) - Z(q, w)] in place of XB (0 for dead walkers)
__global__ void adj_h_kernel(long long K, int W, const zd *Tt, const zd *Z, const int *alive, const zd *den,
                             zd *XB)
{
    const long long total = K * W;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int w = (int)(e / K);
        zd h = make_double2(0, 0);
        if (alive[w]) h = zmul(den[w], zsub(zadd(Tt[e % K], XB[e]), Z[e]));
        XB[e] = h;
    }
}

// gradT(b + Ns i) = [sum_s Vp_s + TR - sum_w P_w](i, b) + Et(b + Ns i); the
// n x Ns matrices are column-major, the gradient in the thetaT layout
__global__ void adj_grad_kernel(int n, int Ns, int S, const zd *Vp, const zd *TR, int W, const zd *Pw,
                                const int *alive, const zd *Et, double *grad)
{
    const long long cnt = (long long)n * Ns;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < cnt;
         e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % n), b = (int)(e / n);
        zd v = TR[e];
        for (int s = 0; s < S; ++s) v = zadd(v, Vp[(size_t)s * cnt + e]);
        for (int w = 0; w < W; ++w)
            if (alive[w]) v = zsub(v, Pw[(size_t)w * cnt + e]);
        const size_t t = (size_t)b + (size_t)Ns * i;
        v = zadd(v, Et[t]);
        grad[2 * t] = v.x;
        grad[2 * t + 1] = v.y;
    }
}

// D_g <- xbar_g I - D_g for the G blocks (Ns x Ns, column-major) of one walker
__global__ void adj_z_kernel(int G, int Ns, const zd *xg, zd *D)
{
    const long long total = (long long)G * Ns * Ns;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long r = e % ((long long)Ns * Ns);
        const int g = (int)(e / ((long long)Ns * Ns));
        const int a = (int)(r % Ns), b = (int)(r / Ns);
        zd v = zneg(D[e]);
        if (a == b) v = zadd(v, xg[g]);
        D[e] = v;
    }
}

// Y += alpha X
__global__ void adj_axpy_kernel(long long count, zd alpha, const zd *X, zd *Y)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
         e += (long long)gridDim.x * blockDim.x)
        zfma(Y[e], alpha, X[e]);
}

// V += sum_g P_g (P_g consecutive blocks of `count` values), summed in g order
__global__ void adj_vsum_kernel(long long count, int G, const zd *P, zd *V)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
         e += (long long)gridDim.x * blockDim.x) {
        zd v = V[e];
        for (int g = 0; g < G; ++g) v = zadd(v, P[(size_t)g * count + e]);
        V[e] = v;
    }
}

// gradT(b + Ns i) += den [V - theta C + (E_w - E) theta](i, b); V and TC are
// n x Ns column-major, theta is read in the thetaT layout (b + Ns i)
__global__ void adj_u_kernel(int n, int Ns, const zd *V, const zd *TC, const zd *thetaTw, zd den, zd dE,
                             double *grad)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * Ns; e += gridDim.x * blockDim.x) {
        const int i = e % n, b = e / n;
        const size_t t = (size_t)b + (size_t)Ns * i;
        zd u = zsub(V[e], TC[e]);
        zfma(u, dE, thetaTw[t]);
        u = zmul(den, u);
        grad[2 * t] += u.x;
        grad[2 * t + 1] += u.y;
    }
}

__global__ void adj_conj_kernel(long long count, const zd *src, zd *dst)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
         e += (long long)gridDim.x * blockDim.x)
        dst[e] = zconj(src[e]);
}

// Device scratch of one adjoint evaluation, freed on every return path
// (cudaFree waits for the work in flight).
struct DevBufs {
    std::vector<void *> p;
    ~DevBufs()
    {
        for (void *q : p) cudaFree(q);
    }
    template <class T> cudaError_t get(T **out, size_t count)
    {
        *out = nullptr;
        cudaError_t c = cudaMalloc((void **)out, sizeof(T) * std::max<size_t>(count, 1));
        if (c == cudaSuccess) p.push_back((void *)*out);
        return c;
    }
};

// what both forms share
struct AdjCtx {
    afqmc_engine *e = nullptr;
    cudaStream_t s = nullptr;
    zd Emix{}, invDen{};
    const std::vector<zd> *den = nullptr, *eloc = nullptr;
    const std::vector<int> *al = nullptr;
    const zd *Rt = nullptr, *Et = nullptr;
    zd *dchol = nullptr;      // n x n x G, or null
    double *gradT = nullptr;  // thetaT layout, 2 doubles per entry
    DevBufs *bufs = nullptr;
};

#define ACK(x) do { cudaError_t _c = (x); if (_c != cudaSuccess) return engine_fail(AFQMC_ERR_CUDA, cudaGetErrorString(_c)); } while (0)
#define AGM(g) do { int _r = engine_gemm((g), s); if (_r) return _r; } while (0)

// Per-walker form: batched over the G Cholesky vectors, one walker and spin at
// a time; gradT accumulates every term, dchol every block.
int adjoint_per_walker(AdjCtx &c)
{
    afqmc_engine *e = c.e;
    cudaStream_t s = c.s;
    const int W = e->W, n = e->n, G = e->G;
    const long long Ktot = e->Ktot;
    const int maxNs = std::max(e->bl.Ns[0], e->bl.Ns[1]);
    const long long gnN = (long long)G * n * maxNs;
    zd *Dz, *Ypp, *Yacc, *Vp, *V, *Cs, *TC, *cT;
    ACK(c.bufs->get(&Dz, (size_t)G * maxNs * maxNs));
    ACK(c.bufs->get(&Ypp, (size_t)gnN));
    ACK(c.bufs->get(&Yacc, (size_t)gnN));
    ACK(c.bufs->get(&Vp, (size_t)gnN));
    ACK(c.bufs->get(&V, (size_t)n * maxNs));
    ACK(c.bufs->get(&Cs, (size_t)maxNs * maxNs));
    ACK(c.bufs->get(&TC, (size_t)n * maxNs));
    ACK(c.bufs->get(&cT, (size_t)n * maxNs));
    ACK(cudaMemsetAsync(c.gradT, 0, sizeof(double) * 2 * Ktot, s));
    const std::vector<zd> &den = *c.den, &eloc = *c.eloc;
    bool first = true;
    for (int sb = 0; sb < e->bl.nblk; ++sb) {
        const int Ns = e->bl.Ns[sb];
        if (Ns == 0) continue;
        const long long tOff = e->bl.tOff[sb];
        const long long cnt = (long long)G * n * Ns;
        ACK(cudaMemsetAsync(Yacc, 0, sizeof(zd) * (size_t)cnt, s));
        adj_conj_kernel<<<64, 256, 0, s>>>((long long)n * Ns, e->phiT[sb], cT);
        ACK(cudaGetLastError());
        for (int w = 0; w < W; ++w) {
            if (!(*c.al)[w]) continue;
            const zd *thw = e->thetaT + (size_t)w * e->bl.tStride + tOff;   // theta(i, b) at b + Ns i
            // D_g = A_g theta (Ns x Ns), all g
            {
                ZGemmArgs g;
                g.m = Ns; g.n = Ns; g.k = n; g.opA = OP_N; g.opB = OP_T;
                g.A = e->Aall + tOff; g.lda = Ns; g.strideA = Ktot;
                g.B = thw; g.ldb = Ns; g.strideB = 0;
                g.C = Dz; g.ldc = Ns; g.strideC = (long long)Ns * Ns;
                g.batch = G;
                AGM(g);
            }
            adj_z_kernel<<<296, 256, 0, s>>>(G, Ns, e->xbar + (size_t)G * w, Dz);
            ACK(cudaGetLastError());
            // Y''((g, i), b) = (theta Z_g)(i, b): block g at row g n of a (G n) x Ns matrix
            {
                ZGemmArgs g;
                g.m = n; g.n = Ns; g.k = Ns; g.opA = OP_T; g.opB = OP_N;
                g.A = thw; g.lda = Ns; g.strideA = 0;
                g.B = Dz; g.ldb = Ns; g.strideB = (long long)Ns * Ns;
                g.C = Ypp; g.ldc = (long long)G * n; g.strideC = n;
                g.batch = G;
                AGM(g);
            }
            adj_axpy_kernel<<<592, 256, 0, s>>>(cnt, den[w], Ypp, Yacc);
            ACK(cudaGetLastError());
            // V = t theta + sum_g L_g (theta Z_g)
            {
                ZGemmArgs g;
                g.m = n; g.n = Ns; g.k = n; g.opA = OP_N; g.opB = OP_N; g.a_real = ST_R64;
                g.A = e->chol; g.lda = n; g.strideA = (long long)n * n;
                g.B = Ypp; g.ldb = (long long)G * n; g.strideB = n;
                g.C = Vp; g.ldc = n; g.strideC = (long long)n * Ns;
                g.batch = G;
                AGM(g);
            }
            {
                ZGemmArgs g;
                g.m = n; g.n = Ns; g.k = n; g.opA = OP_N; g.opB = OP_T; g.a_real = ST_R64;
                g.A = e->tdev; g.lda = n;
                g.B = thw; g.ldb = Ns;
                g.C = V; g.ldc = n;
                AGM(g);
            }
            adj_vsum_kernel<<<64, 256, 0, s>>>((long long)n * Ns, G, Vp, V);
            ACK(cudaGetLastError());
            // C = phiT^H V (Ns x Ns); TC = theta C (n x Ns)
            {
                ZGemmArgs g;
                g.m = Ns; g.n = Ns; g.k = n; g.opA = OP_C; g.opB = OP_N;
                g.A = e->phiT[sb]; g.lda = n;
                g.B = V; g.ldb = n;
                g.C = Cs; g.ldc = Ns;
                AGM(g);
            }
            {
                ZGemmArgs g;
                g.m = n; g.n = Ns; g.k = Ns; g.opA = OP_T; g.opB = OP_N;
                g.A = thw; g.lda = Ns;
                g.B = Cs; g.ldb = Ns;
                g.C = TC; g.ldc = n;
                AGM(g);
            }
            adj_u_kernel<<<64, 256, 0, s>>>(n, Ns, V, TC, thw, den[w], zsub(eloc[w], c.Emix),
                                            c.gradT + 2 * tOff);
            ACK(cudaGetLastError());
        }
        // dE/dL_g (n x n) += conj(phiT) Y_g^T / sum den, all g
        if (c.dchol) {
            ZGemmArgs g;
            g.m = n; g.n = n; g.k = Ns; g.opA = OP_N; g.opB = OP_T;
            g.A = cT; g.lda = n; g.strideA = 0;
            g.B = Yacc; g.ldb = (long long)G * n; g.strideB = n;
            g.C = c.dchol; g.ldc = n; g.strideC = (long long)n * n;
            g.alpha = c.invDen;
            g.beta = first ? make_double2(0.0, 0.0) : make_double2(1.0, 0.0);
            g.batch = G;
            AGM(g);
        }
        first = false;
    }
    return AFQMC_OK;
}

// GEMM form over the blocks `nb` (block 0 counted `mult` times); writes
// gradT's slots of those blocks and dchol.
int adjoint_gemm(AdjCtx &c, int nb, int mult)
{
    afqmc_engine *e = c.e;
    cudaStream_t s = c.s;
    ExF64Scratch &xs = *e->exf;
    const int W = e->W, n = e->n, G = e->G;
    const int maxNs = std::max(e->bl.Ns[0], e->bl.Ns[1]);
    const long long Kmax = (long long)maxNs * n, ldu = e->bl.tStride;
    // split of sum_g L_g Y_g into chunks of gper vectors: about four CTAs of
    // 64 x 64 output tiles per SM in all
    const int tiles = ((n + 63) / 64) * ((maxNs + 63) / 64);
    const int gper = std::max(1, G / std::max(1, 592 / tiles));
    const int S = G / gper, rem = G - S * gper, slots = S + (rem > 0 ? 1 : 0);
    zd *Um, *Uden, *XB, *xbm, *Cw, *Pw, *Vp, *TR, *Tt, *cT;
    ACK(c.bufs->get(&Um, (size_t)Kmax * W));
    ACK(c.bufs->get(&Uden, (size_t)Kmax * W));
    ACK(c.bufs->get(&XB, (size_t)Kmax * W));
    ACK(c.bufs->get(&xbm, (size_t)G * W));
    ACK(c.bufs->get(&Cw, (size_t)maxNs * maxNs * W));
    ACK(c.bufs->get(&Pw, (size_t)Kmax * W));
    ACK(c.bufs->get(&Vp, (size_t)Kmax * slots));
    ACK(c.bufs->get(&TR, (size_t)Kmax));
    ACK(c.bufs->get(&Tt, (size_t)Kmax));
    ACK(c.bufs->get(&cT, (size_t)Kmax));
    adj_xbm_kernel<<<296, 256, 0, s>>>((long long)G * W, G, e->xbar, e->alive, xbm);
    ACK(cudaGetLastError());
    // the local energy left Z = V U of its last block in the scratch; the
    // blocks run in reverse order so that the first one reuses it
    int zBlock = -1;
    for (int b = 0; b < nb; ++b)
        if (e->bl.Ns[b] > 0) zBlock = b;
    bool first = true;
    for (int b = nb - 1; b >= 0; --b) {
        const int Ns = e->bl.Ns[b];
        if (Ns == 0) continue;
        const ExF64 x = exf64_block(e, b);
        const long long K = x.K, tOff = e->bl.tOff[b];
        const zd *U = e->thetaT + tOff;
        if (b != zBlock) {
            ZGemmArgs g;
            g.m = (int)K; g.n = W; g.k = (int)K; g.a_real = ST_R64;
            g.A = x.V; g.lda = K; g.B = U; g.ldb = ldu; g.C = xs.Z; g.ldc = K;
            AGM(g);
        }
        adj_mask_kernel<<<592, 256, 0, s>>>(K, W, U, ldu, e->alive, e->den, Um, Uden);
        ACK(cudaGetLastError());
        // Tt = phiT^H t (Ns x n)
        {
            ZGemmArgs g;
            g.m = Ns; g.n = n; g.k = n; g.opA = OP_C; g.b_real = ST_R64;
            g.A = e->phiT[b]; g.lda = n; g.B = e->tdev; g.ldb = n; g.C = Tt; g.ldc = Ns;
            AGM(g);
        }
        // XB = X xbar (K x W), then H_w = den_w [Tt + XB_w - Z_w] in its place
        {
            ZGemmArgs g;
            g.m = (int)K; g.n = W; g.k = G; g.a_real = ST_R64;
            g.A = x.X; g.lda = K; g.B = xbm; g.ldb = G; g.C = XB; g.ldc = K;
            AGM(g);
        }
        adj_h_kernel<<<592, 256, 0, s>>>(K, W, Tt, xs.Z, e->alive, e->den, XB);
        ACK(cudaGetLastError());
        // C_w = H_w theta_w (Ns x Ns), P_w = theta_w C_w (n x Ns)
        {
            ZGemmArgs g;
            g.m = Ns; g.n = Ns; g.k = n; g.opA = OP_N; g.opB = OP_T;
            g.A = XB; g.lda = Ns; g.strideA = K;
            g.B = U; g.ldb = Ns; g.strideB = ldu;
            g.C = Cw; g.ldc = Ns; g.strideC = (long long)Ns * Ns;
            g.batch = W; g.mask = e->alive;
            AGM(g);
        }
        {
            ZGemmArgs g;
            g.m = n; g.n = Ns; g.k = Ns; g.opA = OP_T; g.opB = OP_N;
            g.A = U; g.lda = Ns; g.strideA = ldu;
            g.B = Cw; g.ldb = Ns; g.strideB = (long long)Ns * Ns;
            g.C = Pw; g.ldc = n; g.strideC = K;
            g.batch = W; g.mask = e->alive;
            AGM(g);
        }
        // R = perm(Uden Um^T); Y = Uden xbar^T - R X (K x G)
        {
            int r = exf64_pair_matrix(e, x, Uden, Um);
            if (r) return r;
        }
        {
            ZGemmArgs g;
            g.m = (int)K; g.n = G; g.k = W; g.opA = OP_N; g.opB = OP_T;
            g.A = Uden; g.lda = K; g.B = xbm; g.ldb = G; g.C = xs.Y; g.ldc = K;
            AGM(g);
        }
        {
            ZGemmArgs g;
            g.m = (int)K; g.n = G; g.k = (int)K; g.b_real = ST_R64;
            g.A = xs.R; g.lda = K; g.B = x.X; g.ldb = K; g.C = xs.Y; g.ldc = K;
            g.alpha = make_double2(-1.0, 0.0); g.beta = make_double2(1.0, 0.0);
            AGM(g);
        }
        // dE/dL_g (n x n) (+)= mult conj(phiT) Y_g^T / sum den, all g
        if (c.dchol) {
            adj_conj_kernel<<<64, 256, 0, s>>>((long long)n * Ns, e->phiT[b], cT);
            ACK(cudaGetLastError());
            ZGemmArgs g;
            g.m = n; g.n = n; g.k = Ns;
            g.A = cT; g.lda = n; g.strideA = 0;
            g.B = xs.Y; g.ldb = Ns; g.strideB = K;
            g.C = c.dchol; g.ldc = n; g.strideC = (long long)n * n;
            g.alpha = zscale(c.invDen, (double)mult);
            g.beta = first ? make_double2(0.0, 0.0) : make_double2(1.0, 0.0);
            g.batch = G;
            AGM(g);
        }
        // sum_g L_g Y_g: chol (n x n G) times the (n G) x Ns stack of Y_g, in
        // `slots` partial products over consecutive vectors
        {
            ZGemmArgs g;
            g.m = n; g.n = Ns; g.k = gper * n; g.opA = OP_N; g.opB = OP_T; g.a_real = ST_R64;
            g.A = e->chol; g.lda = n; g.strideA = (long long)gper * n * n;
            g.B = xs.Y; g.ldb = Ns; g.strideB = (long long)gper * K;
            g.C = Vp; g.ldc = n; g.strideC = K;
            g.batch = S;
            AGM(g);
            if (rem > 0) {
                g.k = rem * n;
                g.A = e->chol + (size_t)S * gper * n * n;
                g.B = xs.Y + (size_t)S * gper * K;
                g.C = Vp + (size_t)S * K;
                g.batch = 1;
                AGM(g);
            }
        }
        // TR = t R_s (n x Ns; R_s^T is Rt's block in the thetaT layout)
        {
            ZGemmArgs g;
            g.m = n; g.n = Ns; g.k = n; g.opA = OP_N; g.opB = OP_T; g.a_real = ST_R64;
            g.A = e->tdev; g.lda = n; g.B = c.Rt + tOff; g.ldb = Ns; g.C = TR; g.ldc = n;
            AGM(g);
        }
        adj_grad_kernel<<<(int)std::min<long long>((K + 255) / 256, 1184), 256, 0, s>>>(
            n, Ns, slots, Vp, TR, W, Pw, e->alive, c.Et + tOff, c.gradT + 2 * tOff);
        ACK(cudaGetLastError());
        first = false;
    }
    return AFQMC_OK;
}

#undef ACK
#undef AGM

}  // namespace

extern "C" int afqmc_pl_adjoint(afqmc_engine *e, double *energy, double *mean_logov, double *dE_dt,
                                double *dE_dchol, double *dE_dconj_phiT_up,
                                double *dE_dconj_phiT_dn, double *dLogov_dconj_phiT_up,
                                double *dLogov_dconj_phiT_dn)
{
    if (!e || e->kind != KIND_PL) return engine_fail(AFQMC_ERR_ARG, "phaseless engine required");
    const int W = e->W, n = e->n, G = e->G;
    cudaStream_t s = e->stream;
    DevBufs bufs;
#define ACK(x) do { cudaError_t _c = (x); if (_c != cudaSuccess) return engine_fail(AFQMC_ERR_CUDA, cudaGetErrorString(_c)); } while (0)
    // the GEMM form for real half-rotated vectors; block 0 alone, counted
    // twice, for a spin-restricted trial (the walker's one orbital matrix
    // serves both spins, so the two blocks are the same)
    int form = PL_EX_BLOCKWISE;
    if (e->exf && e->exf->gemm) form = e->exf->restricted ? PL_EX_GEMM_ONE : PL_EX_GEMM_ALL;
    int r = engine_pl_local_energy(e, form);  // logov, Sinv, thetaT, xbar, eloc, den at the walkers
    if (r) return r;
    // host reductions of E and the mean log-overlap
    std::vector<zd> den(W), eloc(W), lo(W);
    std::vector<int> al(W);
    ACK(cudaMemcpyAsync(den.data(), e->den, sizeof(zd) * W, cudaMemcpyDeviceToHost, s));
    ACK(cudaMemcpyAsync(eloc.data(), e->eloc, sizeof(zd) * W, cudaMemcpyDeviceToHost, s));
    ACK(cudaMemcpyAsync(lo.data(), e->logov, sizeof(zd) * W, cudaMemcpyDeviceToHost, s));
    ACK(cudaMemcpyAsync(al.data(), e->alive, sizeof(int) * W, cudaMemcpyDeviceToHost, s));
    ACK(cudaStreamSynchronize(s));
    zd sd = make_double2(0, 0), sh = make_double2(0, 0), sl = make_double2(0, 0);
    int nal = 0;
    for (int w = 0; w < W; ++w) {
        if (!al[w]) continue;
        sd = zadd(sd, den[w]);
        sh = zadd(sh, zmul(den[w], eloc[w]));
        sl = zadd(sl, lo[w]);
        ++nal;
    }
    if (nal == 0) return engine_fail(AFQMC_ERR_STATE, "no alive walkers");
    const zd Emix = zdiv(sh, sd);
    const zd invDen = zdiv(make_double2(1, 0), sd);
    if (energy) { energy[0] = Emix.x; energy[1] = Emix.y; }
    if (mean_logov) { mean_logov[0] = sl.x / nal; mean_logov[1] = sl.y / nal; }

    const long long Ktot = e->Ktot;
    zd *Rt, *St, *Et, *dchol = nullptr;
    double *gradT;
    ACK(bufs.get(&Rt, (size_t)Ktot));
    ACK(bufs.get(&St, (size_t)Ktot));
    ACK(bufs.get(&Et, (size_t)Ktot));
    ACK(bufs.get(&gradT, (size_t)2 * Ktot));
    // dE_dchol in device memory of this GPU takes the gradient directly
    bool cholDev = false;
    if (dE_dchol) {
        cudaPointerAttributes pa{};
        int dev = -1;
        ACK(cudaGetDevice(&dev));
        if (cudaPointerGetAttributes(&pa, dE_dchol) == cudaSuccess) {
            if (pa.type == cudaMemoryTypeDevice && pa.device != dev)
                return engine_fail(AFQMC_ERR_ARG, "dE_dchol is device memory of another GPU");
            cholDev = pa.type == cudaMemoryTypeDevice;
        } else {
            cudaGetLastError();
        }
        if (cholDev) dchol = (zd *)dE_dchol;
        else ACK(bufs.get(&dchol, (size_t)n * n * G));
    }
    adj_r_kernel<<<256, 256, 0, s>>>(W, Ktot, e->bl.tStride, e->thetaT, e->alive, e->den, e->eloc, Emix,
                                     Rt, St, Et);
    ACK(cudaGetLastError());
    AdjCtx c;
    c.e = e; c.s = s; c.Emix = Emix; c.invDen = invDen;
    c.den = &den; c.eloc = &eloc; c.al = &al;
    c.Rt = Rt; c.Et = Et; c.dchol = dchol; c.gradT = gradT; c.bufs = &bufs;
    if (form == PL_EX_BLOCKWISE) r = adjoint_per_walker(c);
    else if (form == PL_EX_GEMM_ONE) r = adjoint_gemm(c, 1, 2);
    else r = adjoint_gemm(c, e->bl.nblk, 1);
    if (r) return r;
    // dE/dt = sum_s conj(phiT_s) R_s^T / sum den (n x n; R_s^T is Rt's block)
    zd *dEdt = nullptr;
    if (dE_dt) {
        zd *cT;
        ACK(bufs.get(&dEdt, (size_t)n * n));
        ACK(bufs.get(&cT, (size_t)n * std::max(e->bl.Ns[0], e->bl.Ns[1])));
        bool first = true;
        for (int sb = 0; sb < e->bl.nblk; ++sb) {
            const int Ns = e->bl.Ns[sb];
            if (Ns == 0) continue;
            adj_conj_kernel<<<64, 256, 0, s>>>((long long)n * Ns, e->phiT[sb], cT);
            ACK(cudaGetLastError());
            ZGemmArgs g;
            g.m = n; g.n = n; g.k = Ns;
            g.A = cT; g.lda = n; g.B = Rt + e->bl.tOff[sb]; g.ldb = Ns; g.C = dEdt; g.ldc = n;
            g.alpha = invDen;
            g.beta = first ? make_double2(0.0, 0.0) : make_double2(1.0, 0.0);
            r = engine_gemm(g, s);
            if (r) return r;
            first = false;
        }
        if (first) ACK(cudaMemsetAsync(dEdt, 0, sizeof(zd) * (size_t)n * n, s));
    }

    // gradients to the host
    std::vector<zd> hS(Ktot);
    std::vector<double> hG(2 * Ktot);
    ACK(cudaMemcpyAsync(hS.data(), St, sizeof(zd) * Ktot, cudaMemcpyDeviceToHost, s));
    ACK(cudaMemcpyAsync(hG.data(), gradT, sizeof(double) * 2 * Ktot, cudaMemcpyDeviceToHost, s));
    if (dEdt) ACK(cudaMemcpyAsync(dE_dt, dEdt, sizeof(zd) * (size_t)n * n, cudaMemcpyDeviceToHost, s));
    if (dchol && !cholDev)
        ACK(cudaMemcpyAsync(dE_dchol, dchol, sizeof(zd) * (size_t)n * n * G, cudaMemcpyDeviceToHost, s));
    ACK(cudaStreamSynchronize(s));
#undef ACK
    // orbital gradients: transpose the (N x n) accumulators to n x N; with
    // block 0 counted twice, block 1's energy gradient is block 0's
    double *outE[2] = {dE_dconj_phiT_up, dE_dconj_phiT_dn};
    double *outL[2] = {dLogov_dconj_phiT_up, dLogov_dconj_phiT_dn};
    for (int sb = 0; sb < e->bl.nblk; ++sb) {
        const int Ns = e->bl.Ns[sb];
        const long long gOff = form == PL_EX_GEMM_ONE ? e->bl.tOff[0] : e->bl.tOff[sb];
        for (int b = 0; b < Ns; ++b)
            for (int i = 0; i < n; ++i) {
                const size_t src = e->bl.tOff[sb] + b + (size_t)Ns * i, dst = i + (size_t)n * b;
                const size_t gsrc = gOff + b + (size_t)Ns * i;
                if (outE[sb]) {
                    zd v = zmul(make_double2(hG[2 * gsrc], hG[2 * gsrc + 1]), invDen);
                    outE[sb][2 * dst] = v.x;
                    outE[sb][2 * dst + 1] = v.y;
                }
                if (outL[sb]) {
                    outL[sb][2 * dst] = hS[src].x / nal;
                    outL[sb][2 * dst + 1] = hS[src].y / nal;
                }
            }
    }
    return AFQMC_OK;
}
