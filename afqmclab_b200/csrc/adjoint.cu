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
// Every contraction is a batched FP64 GEMM over the G Cholesky vectors, one
// walker and spin at a time, so the working set is O(G n Ns) whatever the
// walker size: per walker and spin
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

namespace {

// R^T_s += den_w thetaT_s (and the unweighted sum for the log-overlap)
__global__ void adj_r_kernel(int W, long long Ktot, long long tStride, const zd *thetaT,
                             const int *alive, const zd *den, zd *Rt, zd *St)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < Ktot;
         e += (long long)gridDim.x * blockDim.x) {
        zd r = make_double2(0, 0), q = make_double2(0, 0);
        for (int w = 0; w < W; ++w) {
            if (!alive[w]) continue;
            const zd x = thetaT[(size_t)w * tStride + e];
            zfma(r, den[w], x);
            q = zadd(q, x);
        }
        Rt[e] = r;
        St[e] = q;
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

}  // namespace

int engine_pl_local_energy(afqmc_engine *e);

extern "C" int afqmc_pl_adjoint(afqmc_engine *e, double *energy, double *mean_logov, double *dE_dt,
                                double *dE_dchol, double *dE_dconj_phiT_up,
                                double *dE_dconj_phiT_dn, double *dLogov_dconj_phiT_up,
                                double *dLogov_dconj_phiT_dn)
{
    if (!e || e->kind != KIND_PL) return engine_fail(AFQMC_ERR_ARG, "phaseless engine required");
    const int W = e->W, n = e->n, G = e->G;
    cudaStream_t s = e->stream;
    int r = engine_pl_local_energy(e);  // logov, Sinv, thetaT, xbar, ex, eloc, den at the walkers
    if (r) return r;
    // host reductions of E and the mean log-overlap
    std::vector<zd> den(W), eloc(W), lo(W);
    std::vector<int> al(W);
    cudaMemcpyAsync(den.data(), e->den, sizeof(zd) * W, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(eloc.data(), e->eloc, sizeof(zd) * W, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(lo.data(), e->logov, sizeof(zd) * W, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(al.data(), e->alive, sizeof(int) * W, cudaMemcpyDeviceToHost, s);
    cudaError_t ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return engine_fail(AFQMC_ERR_CUDA, cudaGetErrorString(ce));
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
    const int maxNs = std::max(e->bl.Ns[0], e->bl.Ns[1]);
    const long long gnN = (long long)G * n * maxNs;
    zd *Rt = nullptr, *St = nullptr, *Dz = nullptr, *Ypp = nullptr, *Yacc = nullptr, *Vp = nullptr,
       *V = nullptr, *Cs = nullptr, *TC = nullptr, *cT = nullptr, *dchol = nullptr;
    double *gradT = nullptr;
    auto cleanup = [&]() {
        for (void *p : {(void *)Rt, (void *)St, (void *)Dz, (void *)Ypp, (void *)Yacc, (void *)Vp, (void *)V,
                        (void *)Cs, (void *)TC, (void *)cT, (void *)dchol, (void *)gradT})
            if (p) cudaFree(p);
    };
#define ACK(x) do { cudaError_t _c = (x); if (_c != cudaSuccess) { cleanup(); return engine_fail(AFQMC_ERR_CUDA, cudaGetErrorString(_c)); } } while (0)
#define AGM(g) do { int _r = engine_gemm((g), s); if (_r) { cleanup(); return _r; } } while (0)
    ACK(cudaMalloc(&Rt, sizeof(zd) * Ktot));
    ACK(cudaMalloc(&St, sizeof(zd) * Ktot));
    ACK(cudaMalloc(&Dz, sizeof(zd) * (size_t)G * maxNs * maxNs));
    ACK(cudaMalloc(&Ypp, sizeof(zd) * (size_t)gnN));
    ACK(cudaMalloc(&Yacc, sizeof(zd) * (size_t)gnN));
    ACK(cudaMalloc(&Vp, sizeof(zd) * (size_t)gnN));
    ACK(cudaMalloc(&V, sizeof(zd) * (size_t)n * maxNs));
    ACK(cudaMalloc(&Cs, sizeof(zd) * (size_t)maxNs * maxNs));
    ACK(cudaMalloc(&TC, sizeof(zd) * (size_t)n * maxNs));
    ACK(cudaMalloc(&cT, sizeof(zd) * (size_t)n * maxNs));
    if (dE_dchol) ACK(cudaMalloc(&dchol, sizeof(zd) * (size_t)n * n * G));
    ACK(cudaMalloc(&gradT, sizeof(double) * 2 * Ktot));
    ACK(cudaMemsetAsync(gradT, 0, sizeof(double) * 2 * Ktot, s));
    adj_r_kernel<<<256, 256, 0, s>>>(W, Ktot, e->bl.tStride, e->thetaT, e->alive, e->den, Rt, St);
    ACK(cudaGetLastError());

    for (int sb = 0; sb < e->bl.nblk; ++sb) {
        const int Ns = e->bl.Ns[sb];
        if (Ns == 0) continue;
        const long long tOff = e->bl.tOff[sb];
        const long long cnt = (long long)G * n * Ns;
        ACK(cudaMemsetAsync(Yacc, 0, sizeof(zd) * (size_t)cnt, s));
        adj_conj_kernel<<<64, 256, 0, s>>>((long long)n * Ns, e->phiT[sb], cT);
        ACK(cudaGetLastError());
        for (int w = 0; w < W; ++w) {
            if (!al[w]) continue;
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
            adj_u_kernel<<<64, 256, 0, s>>>(n, Ns, V, TC, thw, den[w], zsub(eloc[w], Emix), gradT + 2 * tOff);
            ACK(cudaGetLastError());
        }
        // dE/dL_g (n x n) += conj(phiT) Y_g^T / sum den, all g
        if (dchol) {
            ZGemmArgs g;
            g.m = n; g.n = n; g.k = Ns; g.opA = OP_N; g.opB = OP_T;
            g.A = cT; g.lda = n; g.strideA = 0;
            g.B = Yacc; g.ldb = (long long)G * n; g.strideB = n;
            g.C = dchol; g.ldc = n; g.strideC = (long long)n * n;
            g.alpha = invDen;
            g.beta = sb > 0 ? make_double2(1.0, 0.0) : make_double2(0.0, 0.0);
            g.batch = G;
            AGM(g);
        }
    }
    // gradients to the host
    std::vector<zd> hR(Ktot), hS(Ktot), hpT0((size_t)n * e->bl.Ns[0]), hpT1;
    std::vector<double> hG(2 * Ktot);
    ACK(cudaMemcpyAsync(hR.data(), Rt, sizeof(zd) * Ktot, cudaMemcpyDeviceToHost, s));
    ACK(cudaMemcpyAsync(hS.data(), St, sizeof(zd) * Ktot, cudaMemcpyDeviceToHost, s));
    ACK(cudaMemcpyAsync(hG.data(), gradT, sizeof(double) * 2 * Ktot, cudaMemcpyDeviceToHost, s));
    ACK(cudaMemcpyAsync(hpT0.data(), e->phiT[0], sizeof(zd) * hpT0.size(), cudaMemcpyDeviceToHost, s));
    if (e->bl.nblk > 1) {
        hpT1.resize((size_t)n * e->bl.Ns[1]);
        ACK(cudaMemcpyAsync(hpT1.data(), e->phiT[1], sizeof(zd) * hpT1.size(), cudaMemcpyDeviceToHost, s));
    }
    if (dchol) ACK(cudaMemcpyAsync(dE_dchol, dchol, sizeof(zd) * (size_t)n * n * G, cudaMemcpyDeviceToHost, s));
    ACK(cudaStreamSynchronize(s));
    cleanup();
#undef ACK
#undef AGM
    const std::vector<zd> *pT[2] = {&hpT0, &hpT1};
    // dE/dt(i,j) = sum_s sum_b R_s(j,b) conj(phiT_s(i,b)) / sum den   (R_s(j,b) = Rt(b,j))
    if (dE_dt) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                zd v = make_double2(0, 0);
                for (int sb = 0; sb < e->bl.nblk; ++sb) {
                    const int Ns = e->bl.Ns[sb];
                    for (int b = 0; b < Ns; ++b)
                        zfma(v, hR[e->bl.tOff[sb] + b + (size_t)Ns * j], zconj((*pT[sb])[i + (size_t)n * b]));
                }
                v = zmul(v, invDen);
                dE_dt[2 * (i + (size_t)n * j)] = v.x;
                dE_dt[2 * (i + (size_t)n * j) + 1] = v.y;
            }
    }
    // orbital gradients: transpose the (N x n) accumulators to n x N
    double *outE[2] = {dE_dconj_phiT_up, dE_dconj_phiT_dn};
    double *outL[2] = {dLogov_dconj_phiT_up, dLogov_dconj_phiT_dn};
    for (int sb = 0; sb < e->bl.nblk; ++sb) {
        const int Ns = e->bl.Ns[sb];
        for (int b = 0; b < Ns; ++b)
            for (int i = 0; i < n; ++i) {
                const size_t src = e->bl.tOff[sb] + b + (size_t)Ns * i, dst = i + (size_t)n * b;
                if (outE[sb]) {
                    zd v = zmul(make_double2(hG[2 * src], hG[2 * src + 1]), invDen);
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
