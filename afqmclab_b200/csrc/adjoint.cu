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
//   dE/dL_g    = [ sum_s (Q_gs - P_gs) phiT_s^H ]^T / sum den,
//                Q_gs = sum_w den_w xbar_gw theta_s,  P_gs = sum_w den_w theta_s D_gs
//   dE/dconj(phiT_s) = sum_w den_w [ V - theta (phiT^H V) + (E_w - E) theta ] / sum den,
//                V = t theta + sum_g L_g theta (xbar_g - D_g)
//   d mean(log <phiT|phi_w>) / dconj(phiT_s) = mean_w theta_s
// E is a function of conj(phiT) only, so the orbital gradient is the
// conjugate Wirtinger derivative.  Per-walker determinants and D_g are
// recomputed here instead of being stored.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "engine_internal.cuh"

namespace {

// P_g^T (N x n) += den_w D^T theta^T accumulated over walkers; one CTA per
// (g, spin).  Dynamic smem: A (N x n), T (N x n), D (N x N), acc (N x n).
__global__ void __launch_bounds__(256)
adj_p_kernel(int W, int n, int G, Blocks bl, long long Ktot, const zd *Aall, const zd *thetaT,
             const int *alive, const zd *den, zd *Pt)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int g = blockIdx.x, s = blockIdx.y;
    const int Ns = bl.Ns[s];
    if (Ns == 0) return;
    zd *A = (zd *)smem_raw;
    zd *T = A + (size_t)Ns * n;
    zd *D = T + (size_t)Ns * n;
    zd *acc = D + (size_t)Ns * Ns;
    const int tid = threadIdx.x, nt = blockDim.x;
    const zd *Ag = Aall + (size_t)g * Ktot + bl.tOff[s];
    for (int e = tid; e < Ns * n; e += nt) { A[e] = Ag[e]; acc[e] = make_double2(0, 0); }
    for (int w = 0; w < W; ++w) {
        if (!alive[w]) continue;
        __syncthreads();
        const zd *th = thetaT + (size_t)w * bl.tStride + bl.tOff[s];
        for (int e = tid; e < Ns * n; e += nt) T[e] = th[e];
        __syncthreads();
        // D(a,b) = sum_i A(a,i) thetaT(b,i)
        for (int e = tid; e < Ns * Ns; e += nt) {
            const int a = e % Ns, b = e / Ns;
            zd d = make_double2(0, 0);
            for (int i = 0; i < n; ++i) zfma(d, A[a + (size_t)Ns * i], T[b + (size_t)Ns * i]);
            D[e] = d;
        }
        __syncthreads();
        const zd dw = den[w];
        // P^T(b,i) += den * sum_a D(a,b) thetaT(a,i)
        for (int e = tid; e < Ns * n; e += nt) {
            const int b = e % Ns, i = e / Ns;
            zd v = make_double2(0, 0);
            for (int a = 0; a < Ns; ++a) zfma(v, D[a + (size_t)Ns * b], T[a + (size_t)Ns * i]);
            zfma(acc[e], dw, v);
        }
    }
    __syncthreads();
    const int maxNs = bl.Ns[0] > bl.Ns[1] ? bl.Ns[0] : bl.Ns[1];
    zd *out = Pt + ((size_t)s * G + g) * (size_t)maxNs * n;
    for (int e = tid; e < Ns * n; e += nt) out[e] = acc[e];
}

// Per (walker, spin): V = t theta + sum_g L_g theta (xbar_g - D_g), then
// U = den [V - theta (phiT^H V) + (E_w - E) theta] added to the orbital
// gradient accumulator (transposed: U^T is N x n, like thetaT).
// Dynamic smem: T (N x n), A (N x n), D (N x N), Wt (N x n), Vt (N x n).
__global__ void __launch_bounds__(256)
adj_v_kernel(int W, int n, int G, Blocks bl, long long Ktot, const zd *Aall, const double *chol,
             const double *t, const zd *phiT0, const zd *phiT1, const zd *thetaT, const zd *xbar,
             const int *alive, const zd *den, const zd *eloc, zd Emix, double *gradT)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int w = blockIdx.x, s = blockIdx.y;
    const int Ns = bl.Ns[s];
    if (Ns == 0 || !alive[w]) return;
    const int tid = threadIdx.x, nt = blockDim.x;
    zd *T = (zd *)smem_raw;
    zd *A = T + (size_t)Ns * n;
    zd *D = A + (size_t)Ns * n;
    zd *Wt = D + (size_t)Ns * Ns;
    zd *Vt = Wt + (size_t)Ns * n;
    const zd *th = thetaT + (size_t)w * bl.tStride + bl.tOff[s];
    for (int e = tid; e < Ns * n; e += nt) T[e] = th[e];
    __syncthreads();
    // Vt(b,i) = sum_j t(i,j) thetaT(b,j)   [(t theta)^T]
    for (int e = tid; e < Ns * n; e += nt) {
        const int b = e % Ns, i = e / Ns;
        zd v = make_double2(0, 0);
        for (int j = 0; j < n; ++j) {
            const double tij = t[i + (size_t)n * j];
            const zd x = T[b + (size_t)Ns * j];
            v.x += tij * x.x; v.y += tij * x.y;
        }
        Vt[e] = v;
    }
    for (int g = 0; g < G; ++g) {
        __syncthreads();
        const zd *Ag = Aall + (size_t)g * Ktot + bl.tOff[s];
        for (int e = tid; e < Ns * n; e += nt) A[e] = Ag[e];
        __syncthreads();
        for (int e = tid; e < Ns * Ns; e += nt) {
            const int a = e % Ns, b = e / Ns;
            zd d = make_double2(0, 0);
            for (int i = 0; i < n; ++i) zfma(d, A[a + (size_t)Ns * i], T[b + (size_t)Ns * i]);
            D[e] = d;
        }
        __syncthreads();
        const zd xg = xbar[g + (size_t)G * w];
        // Wt(b,i) = [theta (xbar - D)]^T (b,i) = xbar thetaT(b,i) - sum_a D(a,b) thetaT(a,i)
        for (int e = tid; e < Ns * n; e += nt) {
            const int b = e % Ns, i = e / Ns;
            zd v = zmul(xg, T[b + (size_t)Ns * i]);
            for (int a = 0; a < Ns; ++a) {
                const zd d = D[a + (size_t)Ns * b], x = T[a + (size_t)Ns * i];
                v.x -= d.x * x.x - d.y * x.y;
                v.y -= d.x * x.y + d.y * x.x;
            }
            Wt[e] = v;
        }
        __syncthreads();
        // Vt(b,i) += sum_j L_g(i,j) Wt(b,j)
        const double *Lg = chol + (size_t)g * n * n;
        for (int e = tid; e < Ns * n; e += nt) {
            const int b = e % Ns, i = e / Ns;
            zd v = Vt[e];
            for (int j = 0; j < n; ++j) {
                const double l = Lg[i + (size_t)n * j];
                const zd x = Wt[b + (size_t)Ns * j];
                v.x += l * x.x; v.y += l * x.y;
            }
            Vt[e] = v;
        }
    }
    __syncthreads();
    // C(a,b) = (phiT^H V)(a,b) = sum_i conj(phiT(i,a)) V(i,b)   (reuse D)
    const zd *pT = s == 0 ? phiT0 : phiT1;
    for (int e = tid; e < Ns * Ns; e += nt) {
        const int a = e % Ns, b = e / Ns;
        zd c = make_double2(0, 0);
        for (int i = 0; i < n; ++i) zfma(c, zconj(pT[i + (size_t)n * a]), Vt[b + (size_t)Ns * i]);
        D[e] = c;
    }
    __syncthreads();
    const zd dw = den[w];
    const zd de = zsub(eloc[w], Emix);
    // U^T(b,i) = den [ Vt(b,i) - sum_a C(a,b) thetaT(a,i) + (E_w - E) thetaT(b,i) ]
    double *out = gradT + 2 * (size_t)bl.tOff[s];
    for (int e = tid; e < Ns * n; e += nt) {
        const int b = e % Ns, i = e / Ns;
        zd u = Vt[e];
        for (int a = 0; a < Ns; ++a) {
            const zd c = D[a + (size_t)Ns * b], x = T[a + (size_t)Ns * i];
            u.x -= c.x * x.x - c.y * x.y;
            u.y -= c.x * x.y + c.y * x.x;
        }
        zfma(u, de, T[e]);
        u = zmul(dw, u);
        atomicAdd(out + 2 * e, u.x);
        atomicAdd(out + 2 * e + 1, u.y);
    }
}

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

// Xd(g, w) = den_w xbar_gw
__global__ void adj_xd_kernel(int G, int W, const zd *xbar, const zd *den, const int *alive, zd *Xd)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)G * W;
         e += (long long)gridDim.x * blockDim.x) {
        const int w = (int)(e / G);
        Xd[e] = alive[w] ? zmul(den[w], xbar[e]) : make_double2(0, 0);
    }
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
    const int N0 = std::max(e->bl.Ns[0], e->bl.Ns[1]);  // block stride of the P accumulators
    zd *Rt = nullptr, *St = nullptr, *Xd = nullptr, *Q = nullptr, *Pt = nullptr, *RG = nullptr;
    double *gradT = nullptr;
    auto cleanup = [&]() {
        for (void *p : {(void *)Rt, (void *)St, (void *)Xd, (void *)Q, (void *)Pt, (void *)RG, (void *)gradT})
            if (p) cudaFree(p);
    };
#define ACK(x) do { cudaError_t _c = (x); if (_c != cudaSuccess) { cleanup(); return engine_fail(AFQMC_ERR_CUDA, cudaGetErrorString(_c)); } } while (0)
    ACK(cudaMalloc(&Rt, sizeof(zd) * Ktot));
    ACK(cudaMalloc(&St, sizeof(zd) * Ktot));
    ACK(cudaMalloc(&Xd, sizeof(zd) * (size_t)G * W));
    ACK(cudaMalloc(&Q, sizeof(zd) * (size_t)Ktot * G));
    ACK(cudaMalloc(&Pt, sizeof(zd) * (size_t)2 * G * N0 * n));
    ACK(cudaMalloc(&RG, sizeof(zd) * (size_t)n * n * (G + 1)));
    ACK(cudaMalloc(&gradT, sizeof(double) * 2 * Ktot));
    ACK(cudaMemsetAsync(gradT, 0, sizeof(double) * 2 * Ktot, s));
    ACK(cudaMemsetAsync(Pt, 0, sizeof(zd) * (size_t)2 * G * N0 * n, s));
    adj_r_kernel<<<256, 256, 0, s>>>(W, Ktot, e->bl.tStride, e->thetaT, e->alive, e->den, Rt, St);
    adj_xd_kernel<<<256, 256, 0, s>>>(G, W, e->xbar, e->den, e->alive, Xd);
    // Q^T (Ktot x G) = thetaT (Ktot x W) Xd^T
    {
        ZGemmArgs g;
        g.m = (int)Ktot; g.n = G; g.k = W; g.opA = OP_N; g.opB = OP_T;
        g.A = e->thetaT; g.lda = e->bl.tStride; g.B = Xd; g.ldb = G; g.C = Q; g.ldc = Ktot;
        r = engine_gemm(g, s);
        if (r) { cleanup(); return r; }
    }
    const int maxNs = N0;
    size_t smP = ((size_t)3 * maxNs * n + (size_t)maxNs * maxNs) * sizeof(zd);
    size_t smV = ((size_t)4 * maxNs * n + (size_t)maxNs * maxNs) * sizeof(zd);
    if (smV > 200 * 1024) { cleanup(); return engine_fail(AFQMC_ERR_UNSUPPORTED, "adjoint: walker block too large for shared memory"); }
    cudaFuncSetAttribute(adj_p_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(adj_v_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    adj_p_kernel<<<dim3(G, e->bl.nblk), 256, smP, s>>>(W, n, G, e->bl, Ktot, e->Aall, e->thetaT, e->alive, e->den, Pt);
    const double *tdev = e->tdev;
    adj_v_kernel<<<dim3(W, e->bl.nblk), 256, smV, s>>>(W, n, G, e->bl, Ktot, e->Aall, e->chol, tdev,
                                                         e->phiT[0], e->phiT[1], e->thetaT, e->xbar,
                                                         e->alive, e->den, e->eloc, Emix, gradT);
    r = engine_check_launch();
    if (r) { cleanup(); return r; }
    // (Q - P)_g per spin, and the gradient assembly on the host
    std::vector<zd> hQ((size_t)Ktot * G), hP((size_t)2 * G * N0 * n), hR(Ktot), hS(Ktot), hpT0((size_t)n * e->bl.Ns[0]), hpT1;
    std::vector<double> hG(2 * Ktot);
    ACK(cudaMemcpyAsync(hQ.data(), Q, sizeof(zd) * hQ.size(), cudaMemcpyDeviceToHost, s));
    ACK(cudaMemcpyAsync(hP.data(), Pt, sizeof(zd) * hP.size(), cudaMemcpyDeviceToHost, s));
    ACK(cudaMemcpyAsync(hR.data(), Rt, sizeof(zd) * Ktot, cudaMemcpyDeviceToHost, s));
    ACK(cudaMemcpyAsync(hS.data(), St, sizeof(zd) * Ktot, cudaMemcpyDeviceToHost, s));
    ACK(cudaMemcpyAsync(hG.data(), gradT, sizeof(double) * 2 * Ktot, cudaMemcpyDeviceToHost, s));
    ACK(cudaMemcpyAsync(hpT0.data(), e->phiT[0], sizeof(zd) * hpT0.size(), cudaMemcpyDeviceToHost, s));
    if (e->bl.nblk > 1) {
        hpT1.resize((size_t)n * e->bl.Ns[1]);
        ACK(cudaMemcpyAsync(hpT1.data(), e->phiT[1], sizeof(zd) * hpT1.size(), cudaMemcpyDeviceToHost, s));
    }
    ACK(cudaStreamSynchronize(s));
    cleanup();
#undef ACK
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
    // dE/dL_g(i,j) = sum_s sum_b (Q - P)_gs(j,b) conj(phiT_s(i,b)) / sum den
    if (dE_dchol) {
        for (int g = 0; g < G; ++g)
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                    zd v = make_double2(0, 0);
                    for (int sb = 0; sb < e->bl.nblk; ++sb) {
                        const int Ns = e->bl.Ns[sb];
                        const zd *Qg = hQ.data() + (size_t)g * Ktot + e->bl.tOff[sb];
                        const zd *Pg = hP.data() + ((size_t)sb * G + g) * (size_t)N0 * n;
                        for (int b = 0; b < Ns; ++b) {
                            zd qp = zsub(Qg[b + (size_t)Ns * j], Pg[b + (size_t)Ns * j]);
                            zfma(v, qp, zconj((*pT[sb])[i + (size_t)n * b]));
                        }
                    }
                    v = zmul(v, invDen);
                    size_t o = 2 * (i + (size_t)n * j + (size_t)n * n * g);
                    dE_dchol[o] = v.x;
                    dE_dchol[o + 1] = v.y;
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
