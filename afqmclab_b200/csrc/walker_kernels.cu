// AFQMC walker-step kernels other than the GEMMs (plain FP64 form).
// Each kernel cites the reference function it replaces.
#include "walker_kernels.cuh"

#include <atomic>

std::atomic<long long> g_launch_count{0};

#include <stdio.h>
#include <cooperative_groups.h>
#include "once.cuh"

namespace cg = cooperative_groups;

namespace {

constexpr int LU_SMEM_MAX_NS = 64;

// ---------------------------------------------------------------------------
// LU with partial pivoting + log-determinant (+ inverse) of every overlap
// block of a walker; one CTA per walker.
// Replaces SDSDOperation::calculateLUOverlap/returnLogOverlap
// (SDSDOperation.cpp:65-72,154-164), SD2sSD2isOperation (:84-94,187-198),
// LUconstruct_cpu (tensor_2d_bl_cpu.cpp:145-167, zgetrf) and
// logDeterminant (tensor_2d_common_fun.cpp:75-105).  Pivoting follows
// zgetf2: first row of maximal |re|+|im|, reciprocal scaling of the column.
// The first cos projection of the driver step
// (afqmcConstraintPathProjection.cpp:45-48, afqmcPhaselessProjection.cpp:85-88)
// and the population-control weights (afqmcConstraintPathProjection.cpp:108-122)
// are fused into the epilogue.
// ---------------------------------------------------------------------------
template <bool SMEM>
__global__ void __launch_bounds__(256)
lu_kernel(int W, Blocks bl, zd *S, zd *Sinv, const int *active, const zd *logw, zd logwAdd,
          zd logwT, zd *logov, int *alive, int *surv, zd *logwOut, double *weight, int *status,
          int mode, int wantInverse, int maxNs)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int w = blockIdx.x;
    const int tid = threadIdx.x, nt = blockDim.x;
    zd *sA = (zd *)smem_raw;
    zd *sX = sA + (SMEM ? maxNs * maxNs : 0);
    int *piv = (int *)(sX + (SMEM ? maxNs * maxNs : 0));
    __shared__ int sFlag, sBlk;   // singular anywhere / in the current block

    const bool act = (active == nullptr) || active[w] != 0;
    if (!act) {
        if (tid == 0) {
            if (mode == LU_PROJECT) surv[w] = 0;
            if (mode == LU_POPWEIGHT) { weight[w] = 0.0; alive[w] = 1; }
        }
        return;
    }
    if (tid == 0) sFlag = 0;
    zd logdetSum = make_double2(0.0, 0.0);

    for (int b = 0; b < bl.nblk; ++b) {
        const int Ns = bl.Ns[b];
        if (Ns == 0) continue;
        zd *Sg = S + (size_t)w * bl.sStride + bl.sOff[b];
        zd *Xg = Sinv ? Sinv + (size_t)w * bl.sStride + bl.sOff[b] : nullptr;
        zd *A = SMEM ? sA : Sg;
        zd *X = SMEM ? sX : Xg;
        if (SMEM)
            for (int e = tid; e < Ns * Ns; e += nt) A[e] = Sg[e];
        if (tid == 0) sBlk = 0;
        __syncthreads();
        for (int j = 0; j < Ns; ++j) {
            if (tid < 32) {
                double best = -1.0; int bi = Ns;
                for (int i = j + tid; i < Ns; i += 32) {
                    double v = zcabs1(A[i + (size_t)j * Ns]);
                    if (v > best) { best = v; bi = i; }
                }
                for (int o = 16; o > 0; o >>= 1) {
                    double ov = __shfl_xor_sync(0xffffffffu, best, o);
                    int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                    if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
                }
                if (tid == 0) piv[j] = bi;
            }
            __syncthreads();
            const int p = piv[j];
            if (p != j)
                for (int c = tid; c < Ns; c += nt) {
                    zd t = A[j + (size_t)c * Ns];
                    A[j + (size_t)c * Ns] = A[p + (size_t)c * Ns];
                    A[p + (size_t)c * Ns] = t;
                }
            __syncthreads();
            const zd d = A[j + (size_t)j * Ns];
            if (!zeq0(d)) {
                zd inv = zdiv(make_double2(1.0, 0.0), d);
                for (int i = j + 1 + tid; i < Ns; i += nt) A[i + (size_t)j * Ns] = zmul(A[i + (size_t)j * Ns], inv);
            } else if (tid == 0) {
                sFlag = 1;
                sBlk = 1;
            }
            __syncthreads();
            const int r = Ns - j - 1;
            for (int e = tid; e < r * r; e += nt) {
                int i = j + 1 + e % r, c = j + 1 + e / r;
                zd u = A[j + (size_t)c * Ns];
                zd l = A[i + (size_t)j * Ns];
                zd v = A[i + (size_t)c * Ns];
                v.x -= l.x * u.x - l.y * u.y;
                v.y -= l.x * u.y + l.y * u.x;
                A[i + (size_t)c * Ns] = v;
            }
            __syncthreads();
        }
        // log determinant with pivot signs; a singular block contributes
        // lognorm -1e300 and phase 1 (lognormPhaseDeterminant,
        // tensor_2d_common_fun.cpp:75-84), and the blocks' log-dets add up
        // (SD2sSD2isOperation.cpp:84-94)
        if (tid == 0) {
            if (sBlk) {
                logdetSum = zadd(logdetSum, make_double2(-1e300, 0.0));
            } else {
                double lognorm = 0.0; zd phase = make_double2(1.0, 0.0);
                for (int j = 0; j < Ns; ++j) {
                    zd u = A[j + (size_t)j * Ns];
                    double a = zabs(u);
                    lognorm += log(a);
                    zd f = (piv[j] != j) ? zneg(u) : u;
                    phase = zmul(phase, make_double2(f.x / a, f.y / a));
                }
                zd ld = zadd(make_double2(lognorm, 0.0), zlog(phase));
                logdetSum = zadd(logdetSum, ld);
            }
        }
        // inverse: X = A^{-1} column by column (P, unit-L forward, U backward)
        if (wantInverse && Xg) {
            for (int c = tid; c < Ns; c += nt) {
                zd *x = X + (size_t)c * Ns;
                for (int i = 0; i < Ns; ++i) x[i] = make_double2(i == c ? 1.0 : 0.0, 0.0);
                for (int i = 0; i < Ns; ++i) {
                    int pi = piv[i];
                    if (pi != i) { zd t = x[i]; x[i] = x[pi]; x[pi] = t; }
                }
                for (int i = 0; i < Ns; ++i) {
                    zd s = x[i];
                    for (int k = 0; k < i; ++k) {
                        zd l = A[i + (size_t)k * Ns], xk = x[k];
                        s.x -= l.x * xk.x - l.y * xk.y;
                        s.y -= l.x * xk.y + l.y * xk.x;
                    }
                    x[i] = s;
                }
                for (int i = Ns - 1; i >= 0; --i) {
                    zd s = x[i];
                    for (int k = i + 1; k < Ns; ++k) {
                        zd u = A[i + (size_t)k * Ns], xk = x[k];
                        s.x -= u.x * xk.x - u.y * xk.y;
                        s.y -= u.x * xk.y + u.y * xk.x;
                    }
                    x[i] = zdiv(s, A[i + (size_t)i * Ns]);
                }
            }
            __syncthreads();
            if (SMEM)
                for (int e = tid; e < Ns * Ns; e += nt) Xg[e] = X[e];
        }
        __syncthreads();
    }

    if (tid == 0) {
        zd lwR = zadd(logwAdd, logw[w]);
        if (bl.mult == 2) logdetSum = zadd(logdetSum, logdetSum);
        zd lo = zadd(zadd(zconj(logwT), lwR), logdetSum);
        logov[w] = lo;
        if (sFlag && status) atomicOr(status + w, (int)ST_SINGULAR);
        if (!(isfinite(lo.x) && isfinite(lo.y)) && status && !sFlag) atomicOr(status + w, (int)ST_NONFINITE);
        if (mode == LU_PROJECT) {
            double phase = lo.y;
            double c = cos(phase);
            if (c <= 0.0) {
                alive[w] = 0; surv[w] = 0;
            } else {
                zd lw = logw[w];
                lw = zadd(lw, make_double2(log(c), -phase));
                logwOut[w] = lw;
                surv[w] = 1;
            }
        } else if (mode == LU_POPWEIGHT) {
            zd e = zexp(lo);
            double ov = e.x;
            if (ov <= 0.0) {
                weight[w] = 0.0;
            } else {
                weight[w] = ov;
                logwOut[w] = zsub(logw[w], lo);
            }
            alive[w] = 1;
        }
    }
}

// ---------------------------------------------------------------------------
// Same contract as lu_kernel for blocks of 33..GJ_CTA_MAX_NS columns, one CTA
// per walker, the block resident in shared memory (column-major, as in S).
// Warp w owns the columns c = w (mod warps); lane l holds rows l, l+32, ...
// With the inverse requested: Gauss-Jordan elimination in place (zgetf2 pivot
// choice, row interchanges undone as column swaps at the end).  Without it:
// the LU elimination of the trailing block only.  Per column j, two barriers:
//   A  every warp interchanges rows j and p and scales row j in its columns;
//      the owner of column j gathers that column (and rewrites it);
//   B  every warp applies the rank-1 update to its columns; the owner of
//      column j+1 updates it first and finds the next pivot and its
//      reciprocal, so the search overlaps the other warps' updates.
// The pivots are the U diagonal of zgetrf; the log-determinant is summed from
// them at the end with the interchange signs, as logDeterminant does
// (tensor_2d_common_fun.cpp:75-105).
// ---------------------------------------------------------------------------
constexpr int GJ_CTA_MAX_NS = 120;

// column buffer: ns complex values during the elimination, then the pivot
// list, the column permutation and the log-determinant partial sums
__host__ __device__ constexpr size_t gj_cta_col_bytes(int ns)
{
    return (((size_t)16 * ns > (size_t)8 * ns + 400 ? (size_t)16 * ns : (size_t)8 * ns + 400) + 15) / 16 * 16;
}
__host__ __device__ constexpr size_t gj_cta_smem(int ns)
{
    return (size_t)ns * ns * sizeof(zd) + gj_cta_col_bytes(ns) + 3 * sizeof(zd);
}

// pivot of column j (rows >= j) by one warp whose lanes hold rows lane + 32 r;
// lane 0 publishes (1/pivot, (row, zero flag), pivot)
template <int RPL>
__device__ __forceinline__ void gj_cta_pivot(const zd *A, int Ns, int j, int lane, zd *sc)
{
    double best = -1.0;
    int bi = Ns;
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
        const int i = lane + 32 * r;
        if (i >= j && i < Ns) {
            const double v = zcabs1(A[i + (size_t)Ns * j]);
            if (v > best) { best = v; bi = i; }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
    }
    if (lane == 0) {
        const zd d = A[bi + (size_t)Ns * j];
        const bool z = zeq0(d);
        sc[0] = z ? make_double2(0.0, 0.0) : zdiv(make_double2(1.0, 0.0), d);
        sc[1] = make_double2((double)bi, z ? 1.0 : 0.0);
        sc[2] = d;
    }
}

template <int NT, int RPL>
__global__ void __launch_bounds__(NT)
gj_cta_kernel(int W, Blocks bl, const zd *S, zd *Sinv, const int *active, const zd *logw,
              zd logwAdd, zd logwT, zd *logov, int *alive, int *surv, zd *logwOut, double *weight,
              int *status, int mode, int wantInverse, int maxNs)
{
    constexpr int NW = NT / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    zd *A = (zd *)smem_raw;
    zd *col = A + (size_t)maxNs * maxNs;
    // [0] 1 / pivot, [1] (pivot row, zero pivot flag), [2] pivot
    zd *sc = (zd *)((unsigned char *)col + gj_cta_col_bytes(maxNs));
    const int w = blockIdx.x, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool act = (active == nullptr) || active[w] != 0;
    if (!act) {
        if (tid == 0) {
            if (mode == LU_PROJECT) surv[w] = 0;
            if (mode == LU_POPWEIGHT) { weight[w] = 0.0; alive[w] = 1; }
        }
        return;
    }
    bool singular = false;
    zd logdetSum = make_double2(0.0, 0.0);
    for (int b = 0; b < bl.nblk; ++b) {
        const int Ns = bl.Ns[b];
        if (Ns == 0) continue;
        const zd *Sg = S + (size_t)w * bl.sStride + bl.sOff[b];
        zd *Xg = (wantInverse && Sinv) ? Sinv + (size_t)w * bl.sStride + bl.sOff[b] : nullptr;
        const bool inv = Xg != nullptr;
        __syncthreads();
        for (int e = tid; e < Ns * Ns; e += NT) A[e] = Sg[e];
        __syncthreads();
        if (warp == 0) gj_cta_pivot<RPL>(A, Ns, 0, lane, sc);
        __syncthreads();
        int myPiv = tid;   // thread k keeps the pivot row and value of column k
        zd myD = make_double2(1.0, 0.0);
        bool sing = false;
        for (int j = 0; j < Ns; ++j) {
            const int p = (int)sc[1].x;
            if (sc[1].y != 0.0) sing = true;
            const zd dinv = sc[0];
            if (tid == j) { myPiv = p; myD = sc[2]; }
            // A: interchange + row scaling in this warp's columns (one lane per column)
            for (int c = warp + NW * lane; c < Ns; c += NW * 32) {
                const zd a = A[j + (size_t)Ns * c], bq = A[p + (size_t)Ns * c];
                if (p != j) A[p + (size_t)Ns * c] = a;
                A[j + (size_t)Ns * c] = (c == j) ? bq : zmul(bq, dinv);
            }
            if (warp == j % NW) {
                __syncwarp();
                // column j after the interchange: gather, then its final values
#pragma unroll
                for (int r = 0; r < RPL; ++r) {
                    const int i = lane + 32 * r;
                    if (i < Ns && i != j) {
                        const zd f = A[i + (size_t)Ns * j];
                        col[i] = f;
                        if (inv) A[i + (size_t)Ns * j] = zneg(zmul(f, dinv));
                    }
                }
                if (inv && lane == 0) A[j + (size_t)Ns * j] = dinv;
            }
            __syncthreads();
            // B: rank-1 update of this warp's columns; column j+1 first
            zd f[RPL];
            bool mine[RPL];
#pragma unroll
            for (int r = 0; r < RPL; ++r) {
                const int i = lane + 32 * r;
                mine[r] = i < Ns && i != j && (inv || i > j);
                f[r] = mine[r] ? col[i] : make_double2(0.0, 0.0);
            }
            const int cn = j + 1;
            const bool ownNext = cn < Ns && (cn % NW) == warp;
            auto update = [&](int c) {
                const zd u = A[j + (size_t)Ns * c];
#pragma unroll
                for (int r = 0; r < RPL; ++r) {
                    if (mine[r]) {
                        zd *ap = A + lane + 32 * r + (size_t)Ns * c;
                        zd v = *ap;
                        v.x -= f[r].x * u.x - f[r].y * u.y;
                        v.y -= f[r].x * u.y + f[r].y * u.x;
                        *ap = v;
                    }
                }
            };
            if (ownNext) {
                update(cn);
                __syncwarp();
                gj_cta_pivot<RPL>(A, Ns, cn, lane, sc);
            }
            int c0 = warp;
            if (!inv && c0 <= j) c0 += ((j + 1 - c0 + NW - 1) / NW) * NW;   // first column > j
            for (int c = c0; c < Ns; c += NW)
                if (c != j && c != cn) update(c);
            __syncthreads();
        }
        // log-determinant from the pivots, sign flip per interchange
        unsigned char *cb = (unsigned char *)col;
        double *redL = (double *)(cb + ((8 * Ns + 15) & ~15));
        zd *redP = (zd *)(cb + ((8 * Ns + 15) & ~15) + ((8 * NW + 15) & ~15));
        double ln = 0.0;
        zd ph = make_double2(1.0, 0.0);
        if (!sing && tid < Ns) {
            const double ad = zabs(myD);
            ln = log(ad);
            ph = make_double2(myD.x / ad, myD.y / ad);
            if (myPiv != tid) ph = zneg(ph);
        }
        for (int o = 16; o > 0; o >>= 1) {
            ln += __shfl_xor_sync(0xffffffffu, ln, o);
            zd q;
            q.x = __shfl_xor_sync(0xffffffffu, ph.x, o);
            q.y = __shfl_xor_sync(0xffffffffu, ph.y, o);
            ph = zmul(ph, q);
        }
        if (lane == 0) { redL[warp] = ln; redP[warp] = ph; }
        if (inv) {
            // column permutation that undoes the row interchanges, last first
            int *pv = (int *)col, *idx = pv + Ns;
            if (tid < Ns) pv[tid] = myPiv;
            __syncthreads();
            if (tid == 0) {
                for (int k = 0; k < Ns; ++k) idx[k] = k;
                for (int k = Ns - 1; k >= 0; --k) {
                    const int q = pv[k];
                    const int t = idx[k]; idx[k] = idx[q]; idx[q] = t;
                }
            }
            __syncthreads();
            for (int e = tid; e < Ns * Ns; e += NT) {
                const int i = e % Ns, k = e / Ns;
                Xg[e] = A[i + (size_t)Ns * idx[k]];
            }
        }
        __syncthreads();
        // a singular block adds lognorm -1e300 with phase 1
        // (lognormPhaseDeterminant, tensor_2d_common_fun.cpp:75-84)
        if (sing) {
            singular = true;
            if (tid == 0) logdetSum = zadd(logdetSum, make_double2(-1e300, 0.0));
        } else if (tid == 0) {
            double lnT = 0.0;
            zd phT = make_double2(1.0, 0.0);
            for (int k = 0; k < NW; ++k) { lnT += redL[k]; phT = zmul(phT, redP[k]); }
            const zd ld = zadd(make_double2(lnT, 0.0), zlog(phT));
            logdetSum = zadd(logdetSum, ld);
        }
    }
    if (tid == 0) {
        const zd lwR = zadd(logwAdd, logw[w]);
        if (bl.mult == 2) logdetSum = zadd(logdetSum, logdetSum);
        const zd lo = zadd(zadd(zconj(logwT), lwR), logdetSum);
        logov[w] = lo;
        if (singular && status) atomicOr(status + w, (int)ST_SINGULAR);
        if (!(isfinite(lo.x) && isfinite(lo.y)) && status && !singular) atomicOr(status + w, (int)ST_NONFINITE);
        if (mode == LU_PROJECT) {
            const double ph = lo.y;
            const double c = cos(ph);
            if (c <= 0.0) {
                alive[w] = 0; surv[w] = 0;
            } else {
                logwOut[w] = zadd(logw[w], make_double2(log(c), -ph));
                surv[w] = 1;
            }
        } else if (mode == LU_POPWEIGHT) {
            const zd e = zexp(lo);
            if (e.x <= 0.0) {
                weight[w] = 0.0;
            } else {
                weight[w] = e.x;
                logwOut[w] = zsub(logw[w], lo);
            }
            alive[w] = 1;
        }
    }
}

// ---------------------------------------------------------------------------
// Same contract as lu_kernel for blocks of at most 32 columns, one warp per
// walker: Gauss-Jordan elimination with the zgetf2 pivot choice (first row
// of maximal |re|+|im| in the current column), in place in a padded shared
// tile (lane i owns row i), then the column unscrambling of the recorded row
// interchanges.  The pivots are the U diagonal of the LU factorisation, so
// the log-determinant follows logDeterminant (tensor_2d_common_fun.cpp:75-105).
// ---------------------------------------------------------------------------
constexpr int GJ_WARPS = 4;
constexpr int GJ_LD = 33;

__global__ void __launch_bounds__(GJ_WARPS * 32)
gj_warp_kernel(int W, Blocks bl, const zd *S, zd *Sinv, const int *active, const zd *logw,
               zd logwAdd, zd logwT, zd *logov, int *alive, int *surv, zd *logwOut, double *weight,
               int *status, int mode, int wantInverse)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int w = blockIdx.x * GJ_WARPS + warp;
    if (w >= W) return;
    zd *A = (zd *)smem_raw + (size_t)warp * 32 * GJ_LD;
    const bool act = (active == nullptr) || active[w] != 0;
    if (!act) {
        if (lane == 0) {
            if (mode == LU_PROJECT) surv[w] = 0;
            if (mode == LU_POPWEIGHT) { weight[w] = 0.0; alive[w] = 1; }
        }
        return;
    }
    bool singular = false;
    zd logdetSum = make_double2(0.0, 0.0);
    const bool inv = wantInverse && Sinv;
    for (int b = 0; b < bl.nblk; ++b) {
        const int Ns = bl.Ns[b];
        if (Ns == 0) continue;
        const zd *Sg = S + (size_t)w * bl.sStride + bl.sOff[b];
        for (int e = lane; e < Ns * Ns; e += 32) A[(e % Ns) * GJ_LD + e / Ns] = Sg[e];
        __syncwarp();
        double lognorm = 0.0;
        zd phase = make_double2(1.0, 0.0);
        int myPartner = lane;  // lane k keeps the row interchanged at step k
        bool sing = false;
        for (int k = 0; k < Ns; ++k) {
            double v = (lane >= k && lane < Ns) ? zcabs1(A[lane * GJ_LD + k]) : -1.0;
            if (!(v == v)) v = INFINITY;   // a NaN row wins: the comparisons below stay a total order
            int idx = lane;
            for (int o = 16; o > 0; o >>= 1) {
                double ov = __shfl_xor_sync(0xffffffffu, v, o);
                int oi = __shfl_xor_sync(0xffffffffu, idx, o);
                if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
            }
            // the pivot row steers the warp-wide branches below (each with a
            // full-mask __syncwarp): every lane takes lane 0's choice
            const int p = __shfl_sync(0xffffffffu, idx, 0);
            if (lane == k) myPartner = p;
            if (p != k) {
                for (int j = lane; j < Ns; j += 32) {
                    zd t = A[k * GJ_LD + j];
                    A[k * GJ_LD + j] = A[p * GJ_LD + j];
                    A[p * GJ_LD + j] = t;
                }
                __syncwarp();
            }
            const zd piv = A[k * GJ_LD + k];
            if (zeq0(piv)) {
                sing = true;
                __syncwarp();
                continue;
            }
            const double a = zabs(piv);
            lognorm += log(a);
            const zd f = (p != k) ? zneg(piv) : piv;
            phase = zmul(phase, make_double2(f.x / a, f.y / a));
            const zd pinv = zdiv(make_double2(1.0, 0.0), piv);
            __syncwarp();
            // normalise the pivot row; its column-k entry becomes 1/piv
            for (int j = lane; j < Ns; j += 32)
                A[k * GJ_LD + j] = (j == k) ? pinv : zmul(A[k * GJ_LD + j], pinv);
            __syncwarp();
            // eliminate column k from every other row (lane i owns row i);
            // without the inverse only the trailing block below and right of
            // the pivot (the LU elimination) is needed
            // (columns in chunks of 8: the chunk's loads are issued before its
            // stores, which the compiler cannot reorder across the shared tile)
            const bool elim = inv ? (lane < Ns && lane != k) : (lane > k && lane < Ns);
            if (elim) {
                zd *row = A + lane * GJ_LD;
                const zd *prow = A + k * GJ_LD;
                const zd dum = row[k];
                if (inv) row[k] = make_double2(0.0, 0.0);
                const int j1 = inv ? 0 : k + 1;
                for (int j0 = j1; j0 < Ns; j0 += 8) {
                    zd pv[8], r[8];
#pragma unroll
                    for (int t = 0; t < 8; ++t)
                        if (j0 + t < Ns) { pv[t] = prow[j0 + t]; r[t] = row[j0 + t]; }
#pragma unroll
                    for (int t = 0; t < 8; ++t)
                        if (j0 + t < Ns) {
                            r[t].x -= pv[t].x * dum.x - pv[t].y * dum.y;
                            r[t].y -= pv[t].x * dum.y + pv[t].y * dum.x;
                            row[j0 + t] = r[t];
                        }
                }
            }
            __syncwarp();
        }
        // undo the row interchanges as column swaps, last first
        for (int k = Ns - 1; k >= 0 && inv; --k) {
            const int p = __shfl_sync(0xffffffffu, myPartner, k);
            if (p != k && lane < Ns) {
                zd t = A[lane * GJ_LD + k];
                A[lane * GJ_LD + k] = A[lane * GJ_LD + p];
                A[lane * GJ_LD + p] = t;
            }
        }
        __syncwarp();
        // a singular block adds lognorm -1e300 with phase 1
        // (lognormPhaseDeterminant, tensor_2d_common_fun.cpp:75-84)
        if (sing) {
            singular = true;
            logdetSum = zadd(logdetSum, make_double2(-1e300, 0.0));
        } else {
            zd ld = zadd(make_double2(lognorm, 0.0), zlog(phase));
            logdetSum = zadd(logdetSum, ld);
        }
        if (wantInverse && Sinv) {
            zd *Xg = Sinv + (size_t)w * bl.sStride + bl.sOff[b];
            for (int e = lane; e < Ns * Ns; e += 32) Xg[e] = A[(e % Ns) * GJ_LD + e / Ns];
        }
        __syncwarp();
    }
    if (lane == 0) {
        zd lwR = zadd(logwAdd, logw[w]);
        if (bl.mult == 2) logdetSum = zadd(logdetSum, logdetSum);
        zd lo = zadd(zadd(zconj(logwT), lwR), logdetSum);
        logov[w] = lo;
        if (singular && status) atomicOr(status + w, (int)ST_SINGULAR);
        if (!(isfinite(lo.x) && isfinite(lo.y)) && status && !singular) atomicOr(status + w, (int)ST_NONFINITE);
        if (mode == LU_PROJECT) {
            double ph = lo.y;
            double c = cos(ph);
            if (c <= 0.0) {
                alive[w] = 0; surv[w] = 0;
            } else {
                logwOut[w] = zadd(logw[w], make_double2(log(c), -ph));
                surv[w] = 1;
            }
        } else if (mode == LU_POPWEIGHT) {
            zd e = zexp(lo);
            if (e.x <= 0.0) {
                weight[w] = 0.0;
            } else {
                weight[w] = e.x;
                logwOut[w] = zsub(logw[w], lo);
            }
            alive[w] = 1;
        }
    }
}

// ---------------------------------------------------------------------------
// Gauss-Jordan with the matrix in registers (gj_regw_kernel below), same
// contract as gj_warp_kernel for one or two blocks of 17..64 columns: each
// row lives in registers (padded with zeros to the window; only Ns steps
// run, after which the last Ns window slots hold the inverse columns).  The
// column loop is not unrolled; instead every row rotates by one slot per
// step, so the current column is always register slot 0 and every register
// index is static.
//   - pivot: zgetf2's choice, first position >= k of maximal |re|+|im| in the
//     column; rows are not moved, each lane keeps the position its row has in
//     the interchanged matrix (ties go to the lower position, as in izamax);
//   - the chosen row is published in shared memory (a broadcast source);
//     every other row i takes a_ij -= (a_ik / piv) a_pj and
//     a_ik = -a_ik / piv (in-place Gauss-Jordan, which leaves the inverse of the
//     interchanged matrix); the pivot row is not rescaled but keeps a row scale
//     1/piv, applied once at the end.
// The pivots are the U diagonal of the LU factorisation: log|det| is the sum of
// their logs and the phase their product with one sign flip per interchange
// (logDeterminant, tensor_2d_common_fun.cpp:75-105).
// ---------------------------------------------------------------------------
// 1 / b by Smith's scaling (one ratio, one reciprocal)
__device__ __forceinline__ zd zrcp(zd b)
{
    if (fabs(b.y) <= fabs(b.x)) {
        const double r = b.y / b.x, d = 1.0 / (b.x + b.y * r);
        return make_double2(d, -r * d);
    }
    const double r = b.x / b.y, d = 1.0 / (b.y + b.x * r);
    return make_double2(r * d, -d);
}

// A rank that orders candidates like the pivot search: for values >= +0 the
// IEEE bits are monotonic; NaN ranks as infinity; ineligible rows rank 0.
__device__ __forceinline__ unsigned long long gr_rank(zd a0, bool eligible)
{
    double v = zcabs1(a0);
    if (!(v == v)) v = INFINITY;
    return eligible ? (unsigned long long)__double_as_longlong(v) + 1ull : 0ull;
}

// 1 / b without a division, so that it schedules between other arithmetic:
// b is scaled by a power of two (exact) so that max(|re|, |im|) lies in
// [1, 2), the real reciprocal y of d = |b|^2 in [1, 8) starts from the
// single-precision approximation and takes two Newton-Raphson steps
// y <- y + y (1 - d y), each of which doubles the correct bits (about 21 ->
// 42 -> full precision), and 1/b = s conj(b s) y.  Within a few ulp of the
// rounded quotient; a NaN or infinite b gives NaN (callers test zero first).
__device__ __forceinline__ zd zrcp_nr(zd b)
{
    const double m = fmax(fabs(b.x), fabs(b.y));
    const long long e = (__double_as_longlong(m) >> 52) & 0x7ff;
    const double s = __longlong_as_double((2046 - e) << 52);   // 2^(1023 - e)
    const double xs = b.x * s, ys = b.y * s;
    const double d = fma(xs, xs, ys * ys);
    double y = (double)__fdividef(1.0f, (float)d);
    y = fma(y, fma(-d, y, 1.0), y);
    y = fma(y, fma(-d, y, 1.0), y);
    const double t = y * s;
    return make_double2(xs * t, -ys * t);
}

// Position of the warp's best candidate: largest rank, then lowest position.
__device__ __forceinline__ int gr_warp_best(unsigned long long u, int pos)
{
    const unsigned hi = (unsigned)(u >> 32), lo = (unsigned)u;
    const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
    const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
    const unsigned key = (hi == mhi && lo == mlo) ? (unsigned)pos : 0xffffffffu;
    return (int)__reduce_min_sync(0xffffffffu, key);
}

// Per-walker finish of the block log-determinants: the overlap's log and,
// by mode, the constraint or the population weight.  ldB/sgB hold the
// walker's nb block log-determinants and singular flags.
__device__ void lu_walker_finish(int w, bool act, int nb, int mult, const zd *ldB, const int *sgB,
                                 const zd *logw, zd logwAdd, zd logwT, zd *logov, int *alive, int *surv,
                                 zd *logwOut, double *weight, int *status, int mode)
{
    if (!act) {
        if (mode == LU_PROJECT) surv[w] = 0;
        if (mode == LU_POPWEIGHT) { weight[w] = 0.0; alive[w] = 1; }
        return;
    }
    bool singular = false;
    zd logdetSum = make_double2(0.0, 0.0);
    // a singular block adds lognorm -1e300 with phase 1
    // (lognormPhaseDeterminant, tensor_2d_common_fun.cpp:75-84)
    for (int t = 0; t < nb; ++t) {
        const bool sb = sgB[t] != 0;
        singular = singular || sb;
        logdetSum = zadd(logdetSum, sb ? make_double2(-1e300, 0.0) : ldB[t]);
    }
    const zd lwR = zadd(logwAdd, logw[w]);
    if (mult == 2) logdetSum = zadd(logdetSum, logdetSum);
    const zd lo = zadd(zadd(zconj(logwT), lwR), logdetSum);
    logov[w] = lo;
    if (singular && status) atomicOr(status + w, (int)ST_SINGULAR);
    if (!(isfinite(lo.x) && isfinite(lo.y)) && status && !singular) atomicOr(status + w, (int)ST_NONFINITE);
    if (mode == LU_PROJECT) {
        const double ph = lo.y;
        const double c = cos(ph);
        if (c <= 0.0) {
            alive[w] = 0; surv[w] = 0;
        } else {
            logwOut[w] = zadd(logw[w], make_double2(log(c), -ph));
            surv[w] = 1;
        }
    } else if (mode == LU_POPWEIGHT) {
        const zd e = zexp(lo);
        if (e.x <= 0.0) {
            weight[w] = 0.0;
        } else {
            weight[w] = e.x;
            logwOut[w] = zsub(logw[w], lo);
        }
        alive[w] = 1;
    }
}

// ---------------------------------------------------------------------------
// The same rotated Gauss-Jordan with the window split between two column
// halves, one CTA per matrix: RH row halves x 2 column halves of SL slots
// (RH = 2, SL = 32 for blocks of 33-64 columns, four warps; RH = 1, SL = 16
// for 17-32 columns, two warps).  Warp (rh, ch) holds rows rh*32+lane and
// half ch of a 2 SL-column window that moves by one column per step.  The half-0 warps hold
// the current column in slot 0; while they update step k they already search
// the pivot of step k+1 in their new slot 0 (max |re|+|im|, ties to the lower
// position, NaN first), and each warp's winning lane publishes its row, its
// position and the reciprocal of its pivot.  After one CTA barrier per step:
//   - half 0 updates from the published half-0 row of the winner; the last
//     slot of every row (and of the pivot row) is the updated slot 0 of half
//     1 from the step before, passed through shared memory;
//   - half 1 takes its factor f = a_k * (1/piv) from the published column k,
//     the pivot row's lane writes its half-1 row, a barrier of the half-1
//     warps, then half 1 updates and takes the new inverse column in its last
//     slot.
// Shared buffers alternate between even and odd steps, so the only CTA-wide
// barrier per step is the one that publishes step k+1's inputs.
// Only Ns steps run and the padding is zero: padding rows stay zero in every
// real column and are never chosen, and after step Ns the window holds the
// inverse columns 0..Ns-1 in its last Ns slots.  Row r's final position is
// the image of r under the interchanges applied first to last, so column j
// of the interchanged inverse is column r of the inverse for the row r whose
// final position is j.  The two blocks of a two-block walker run as a
// cluster of two CTAs; rank 0 combines them through distributed shared
// memory.
// ---------------------------------------------------------------------------
struct GR64Cand {
    unsigned long long u;   // rank of the candidate: bits of |re|+|im| plus one, 0 if not eligible
    int key;                // its position
    int row;                // its row (rh*32+lane)
    zd a0;                  // its value in the current column
    zd q;                   // 1 / a0, zero when a0 is zero
};

// named barrier 1 of the column groups other than 0
__device__ __forceinline__ void upper_groups_bar(int threads)
{
    asm volatile("bar.sync 1, %0;" ::"r"(threads) : "memory");
}

template <int NB, int SL, int RH, int NQ>
__global__ void __launch_bounds__(32 * RH * NQ, SL == 16 ? 65536 / (32 * RH * NQ * 128) : 2)
gj_regw_kernel(int W, Blocks bl, const zd *S, zd *Sinv, float *Sinv32, long long s32, const int *active,
                const zd *logw, zd logwAdd, zd logwT, zd *logov, int *alive, int *surv, zd *logwOut,
                double *weight, int *status, int mode, int wantInverse)
{
    constexpr int NR = 32 * RH;                      // rows of the window
    __shared__ __align__(16) zd prowC[2][RH][SL];   // [step parity][rh]: half 0 of each warp's candidate
    __shared__ __align__(16) zd prowQ[NQ][SL];      // [cq >= 1]: column group cq of the pivot row
    __shared__ __align__(16) zd colS[2][NR];        // [step parity][row]: the current column
    __shared__ __align__(16) zd xS[NQ][2][NR];      // [cq >= 1][step parity][row]: group cq's updated slot 0
    __shared__ __align__(16) GR64Cand cand[2][RH];  // [step parity][rh]
    __shared__ __align__(16) zd pivS[NR];
    __shared__ __align__(16) zd phS[RH];
    __shared__ double lnS[RH];
    __shared__ int pvS[NR];
    __shared__ int jxS[NR];
    __shared__ zd ldS;
    __shared__ int sgS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rh = warp / NQ, ch = warp % NQ;   // ch: the column group
    const int r = rh * 32 + lane;
    const int w = NB == 1 ? (int)blockIdx.x : (int)(blockIdx.x >> 1);
    const int b = NB == 1 ? 0 : (int)(blockIdx.x & 1);
    const bool act = (active == nullptr) || active[w] != 0;
    const int Ns = b == 0 ? bl.Ns[0] : bl.Ns[1];
    const long long sOff = b == 0 ? bl.sOff[0] : bl.sOff[1];
    const bool inv = wantInverse && (Sinv || Sinv32);
    bool sing = false;
    zd ld = make_double2(0.0, 0.0);
    if (act && Ns > 0) {   // uniform over the CTA
        const zd *Sg = S + (size_t)w * bl.sStride + sOff;
        zd a[SL];
#pragma unroll
        for (int s = 0; s < SL; ++s) {
            const int c = ch * SL + s;
            a[s] = (r < Ns && c < Ns) ? Sg[r + (size_t)Ns * c] : make_double2(0.0, 0.0);
        }
        int pos = r;
        // step 0's inputs, as if a step -1 had produced them: each group's
        // last slot as the next group's "updated slot 0"
        if (ch < NQ - 1) xS[ch + 1][1][r] = a[SL - 1];
        if (ch == 0) {
            colS[0][r] = a[0];
            const unsigned long long u = gr_rank(a[0], true);
            if (pos == gr_warp_best(u, pos)) {
                GR64Cand c;
                c.u = u; c.key = pos; c.row = r; c.a0 = a[0];
                c.q = zeq0(a[0]) ? make_double2(0.0, 0.0) : zrcp_nr(a[0]);
                cand[0][rh] = c;
#pragma unroll
                for (int s = 0; s < SL - 1; ++s) prowC[0][rh][s] = a[s];
            }
        }
#pragma unroll 1
        for (int k = 0; k < Ns; ++k) {
            __syncthreads();   // step k's candidates, column, half-0 rows and half 1's last slots
            const int cb = k & 1, pb = cb ^ 1;
            int second = 0;
            if constexpr (RH == 2) {
                const unsigned long long u0 = cand[cb][0].u, u1 = cand[cb][1].u;
                const int k0 = cand[cb][0].key, k1 = cand[cb][1].key;
                second = (u1 > u0 || (u1 == u0 && k1 < k0)) ? 1 : 0;
            }
            const int p = cand[cb][second].key;
            const zd q = cand[cb][second].q;
            if (threadIdx.x == 0) {
                const zd piv = cand[cb][second].a0;
                pvS[k] = p;
                pivS[k] = piv;
                sing = sing || zeq0(piv);
            }
            const bool isP = (pos == p);
            if (pos == k) pos = p;
            if (isP) pos = k;
            if (ch == 0) {
                a[SL - 1] = xS[1][pb][r];
                const zd *pr = prowC[cb][second];
                const zd pLast = xS[1][pb][cand[cb][second].row];
                const zd f = isP ? make_double2(0.0, 0.0) : zmul(a[0], q);
                {
                    const zd pv = pr[1];
                    a[0].x = fma(-f.x, pv.x, fma(f.y, pv.y, a[1].x));
                    a[0].y = fma(-f.x, pv.y, fma(-f.y, pv.x, a[1].y));
                }
                // the pivot search of step k+1 on the new slot 0 (also after
                // the last step, where nothing reads it, so the step stays
                // one straight-line block the compiler can interleave)
                colS[pb][r] = a[0];
                const unsigned long long u = gr_rank(a[0], pos > k);
                const bool win = (pos == gr_warp_best(u, pos));
                const zd qr = zrcp_nr(a[0]);
                const zd qn = zeq0(a[0]) ? make_double2(0.0, 0.0) : qr;
#pragma unroll
                for (int s = 2; s < SL; ++s) {
                    const zd pv = s < SL - 1 ? pr[s] : pLast;
                    a[s - 1].x = fma(-f.x, pv.x, fma(f.y, pv.y, a[s].x));
                    a[s - 1].y = fma(-f.x, pv.y, fma(-f.y, pv.x, a[s].y));
                }
                if (win) {
                    GR64Cand c;
                    c.u = u; c.key = pos; c.row = r; c.a0 = a[0];
                    c.q = qn;
                    cand[pb][rh] = c;
#pragma unroll
                    for (int s = 0; s < SL - 1; ++s) prowC[pb][rh][s] = a[s];
                }
            } else {
                // a middle group's last slot: its right neighbour's slot 0 of step k-1
                if (ch < NQ - 1) a[SL - 1] = xS[ch + 1][pb][r];
                const zd f = isP ? make_double2(0.0, 0.0) : zmul(colS[cb][r], q);
                zd *pq = prowQ[ch];
                if (isP) {
#pragma unroll
                    for (int s = 0; s < SL; ++s) pq[s] = a[s];
                }
                if constexpr (RH * (NQ - 1) > 1) upper_groups_bar(32 * RH * (NQ - 1));
                else __syncwarp();
                zd x;
                x.x = fma(-f.x, pq[0].x, fma(f.y, pq[0].y, a[0].x));
                x.y = fma(-f.x, pq[0].y, fma(-f.y, pq[0].x, a[0].y));
                xS[ch][cb][r] = x;
#pragma unroll
                for (int s = 1; s < SL; ++s) {
                    const zd pv = pq[s];
                    a[s - 1].x = fma(-f.x, pv.x, fma(f.y, pv.y, a[s].x));
                    a[s - 1].y = fma(-f.x, pv.y, fma(-f.y, pv.x, a[s].y));
                }
                // the last group takes the new inverse column; the others
                // take their neighbour's slot 0 at the next step
                if (ch == NQ - 1) a[SL - 1] = isP ? make_double2(1.0, 0.0) : zneg(f);
            }
        }
        if (threadIdx.x == 0) sgS = sing ? 1 : 0;
        __syncthreads();   // last slots of step Ns-1, all pivots
        sing = sgS != 0;
        if (ch < NQ - 1) a[SL - 1] = xS[ch + 1][(Ns - 1) & 1][r];
        const bool real = r < Ns;   // padding rows keep positions >= Ns
        const zd myD = real ? pivS[pos] : make_double2(1.0, 0.0);
        if (ch == 0) {
            // log-determinant: every real row supplied exactly one pivot
            double ln = 0.0;
            zd ph = make_double2(1.0, 0.0);
            if (real && !sing) {
                const double ad = zabs(myD);
                ln = log(ad);
                ph = make_double2(myD.x / ad, myD.y / ad);
                if (pvS[pos] != pos) ph = zneg(ph);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                ln += __shfl_xor_sync(0xffffffffu, ln, o);
                zd t;
                t.x = __shfl_xor_sync(0xffffffffu, ph.x, o);
                t.y = __shfl_xor_sync(0xffffffffu, ph.y, o);
                ph = zmul(ph, t);
            }
            if (lane == 0) { lnS[rh] = ln; phS[rh] = ph; }
            if (real) jxS[pos] = r;
        }
        __syncthreads();
        if (threadIdx.x == 0 && !sing) {
            if constexpr (RH == 2) ld = zadd(make_double2(lnS[0] + lnS[1], 0.0), zlog(zmul(phS[0], phS[1])));
            else ld = zadd(make_double2(lnS[0], 0.0), zlog(phS[0]));
        }
        if (inv && real) {
            // window slot t = SL ch + s holds interchanged column j = t - (NQ SL - Ns)
            const zd sc = sing ? make_double2(0.0, 0.0) : zrcp(myD);
            const int j0 = ch * SL - (NQ * SL - Ns);
            if (Sinv32) {
                // fp32 planes [re | im], each Ns x Ns column-major
                float *Xr = Sinv32 + (size_t)w * s32 + 2 * sOff, *Xi = Xr + (size_t)Ns * Ns;
#pragma unroll
                for (int s = 0; s < SL; ++s) {
                    const int j = j0 + s;
                    if (j >= 0) {
                        const int c = jxS[j];
                        const zd v = zmul(sc, a[s]);
                        Xr[pos + (size_t)Ns * c] = (float)v.x;
                        Xi[pos + (size_t)Ns * c] = (float)v.y;
                    }
                }
            } else {
                zd *Xg = Sinv + (size_t)w * bl.sStride + sOff;
#pragma unroll
                for (int s = 0; s < SL; ++s) {
                    const int j = j0 + s;
                    if (j >= 0) Xg[pos + (size_t)Ns * jxS[j]] = zmul(sc, a[s]);
                }
            }
        }
    }
    if (threadIdx.x == 0) { ldS = ld; sgS = sing ? 1 : 0; }
    if constexpr (NB == 2) {
        cg::cluster_group cl = cg::this_cluster();
        cl.sync();
        if (threadIdx.x == 0 && b == 0) {
            const zd ldB[2] = {ldS, *cl.map_shared_rank(&ldS, 1)};
            const int sgB[2] = {sgS, *cl.map_shared_rank(&sgS, 1)};
            lu_walker_finish(w, act, 2, bl.mult, ldB, sgB, logw, logwAdd, logwT, logov, alive, surv, logwOut,
                             weight, status, mode);
        }
        cl.sync();   // rank 1's shared memory stays until rank 0 has read it
    } else {
        if (threadIdx.x == 0) {
            const int sg = sing ? 1 : 0;
            lu_walker_finish(w, act, 1, bl.mult, &ld, &sg, logw, logwAdd, logwT, logov, alive, surv, logwOut,
                             weight, status, mode);
        }
    }
}

// ---------------------------------------------------------------------------
// Exclusive scan of survivors x draws -> per-walker offset into the random
// stream; reproduces the reference's sequential walker-major draw order
// (afqmcPhaselessProjection.cpp:80-101, NiupNidn.cpp:66-84).
// ---------------------------------------------------------------------------
__global__ void rng_scan_kernel(int W, const int *surv, int draws, unsigned long long *counter,
                                unsigned long long *offs)
{
    __shared__ unsigned long long warpSums[32];
    __shared__ unsigned long long carry;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (tid == 0) carry = *counter;
    __syncthreads();
    for (int base = 0; base < W; base += blockDim.x) {
        int w = base + tid;
        unsigned long long v = (w < W && surv[w]) ? (unsigned long long)draws : 0ULL;
        unsigned long long x = v;
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warpSums[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int nw = blockDim.x >> 5;
            unsigned long long s = lane < nw ? warpSums[lane] : 0ULL;
            for (int o = 1; o < 32; o <<= 1) {
                unsigned long long y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            if (lane < nw) warpSums[lane] = s;  // inclusive prefix of warp totals
        }
        __syncthreads();
        unsigned long long prefix = carry + (wid > 0 ? warpSums[wid - 1] : 0ULL) + x - v;
        if (w < W) offs[w] = prefix;
        __syncthreads();
        if (tid == blockDim.x - 1) carry = prefix + v;
        __syncthreads();
    }
    if (tid == 0) *counter = carry;
}

// ---------------------------------------------------------------------------
// Hubbard force: HubbardSOCMeasureFixedSDSD::getForce (:73-116) with the
// Green's function diagonal / off-diagonal of SDSDOperation (:91-141).
// ---------------------------------------------------------------------------
__global__ void cp_force_kernel(int W, HubbardDev h, const zd *thetaT, long long tStride,
                                const int *surv, double *force)
{
    const int w = blockIdx.x;
    if (!surv[w]) return;
    const int L = h.L, N = h.N, n = h.n;
    const zd *th = thetaT + (size_t)w * tStride;
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
        double f;
        if (h.constForce) {
            f = h.constForce[i];
        } else {
            zd a = make_double2(0.0, 0.0), b = make_double2(0.0, 0.0);
            if (h.decomp <= 1) {
                for (int j = 0; j < N; ++j) {
                    zfma(a, zconj(h.phiT[i + (size_t)n * j]), th[j + (size_t)N * i]);
                    zfma(b, zconj(h.phiT[i + L + (size_t)n * j]), th[j + (size_t)N * (i + L)]);
                }
            } else {
                for (int j = 0; j < N; ++j) {
                    zfma(a, zconj(h.phiT[i + (size_t)n * j]), th[j + (size_t)N * (i + L)]);
                    zfma(b, zconj(h.phiT[i + L + (size_t)n * j]), th[j + (size_t)N * i]);
                }
            }
            zd bgv;
            if (h.decomp == 0) bgv = make_double2(a.x + b.x - 1.0, a.y + b.y);
            else if (h.decomp == 1) bgv = zsub(a, b);
            else if (h.decomp == 2) bgv = zadd(a, b);
            else bgv = zsub(a, b);
            f = zmul(h.gamma[i], bgv).x;
            if (f > h.forceCap) f = h.forceCap;
            if (f < -h.forceCap) f = -h.forceCap;
        }
        force[(size_t)w * L + i] = f;
    }
}

__device__ __forceinline__ zd zcosh(zd z)
{
    zd e = zexp(z), ei = zexp(zneg(z));
    return zscale(zadd(e, ei), 0.5);
}
__device__ __forceinline__ zd zsinh(zd z)
{
    zd e = zexp(z), ei = zexp(zneg(z));
    return zscale(zsub(e, ei), 0.5);
}
__device__ __forceinline__ zd zcos(zd z)
{
    double s, c;
    sincos(z.x, &s, &c);
    return make_double2(c * cosh(z.y), -s * sinh(z.y));
}
__device__ __forceinline__ zd zsin(zd z)
{
    double s, c;
    sincos(z.x, &s, &c);
    return make_double2(s * cosh(z.y), c * sinh(z.y));
}

// The 2x2 block of site i of a NiupNidn two-body sample with auxiliary
// field x (setTwoBodySampleMatrix, NiupNidn.cpp:252-322): the field part
// exp(gamma_i x) (or its cosh/sinh, cos/sin form for the hopping
// decompositions) times the constant one-site factor constDiag.
__device__ __forceinline__ void cp_site_matrix(const HubbardDev &h, int i, int x, zd &a00, zd &a01, zd &a10,
                                               zd &a11)
{
    const zd ga = zscale(h.gamma[i], (double)x);
    if (h.decomp == 0) {
        const zd e = zexp(ga);
        a00 = zmul(e, h.cd00[i]); a10 = zmul(e, h.cd10[i]); a01 = zmul(e, h.cd01[i]); a11 = zmul(e, h.cd11[i]);
    } else if (h.decomp == 1) {
        const zd e = zexp(ga), ei = zdiv(make_double2(1.0, 0.0), e);
        a00 = zmul(e, h.cd00[i]); a10 = zmul(ei, h.cd10[i]); a01 = zmul(e, h.cd01[i]); a11 = zmul(ei, h.cd11[i]);
    } else if (h.decomp == 2) {
        const zd c = zcosh(ga), s = zsinh(ga);
        a00 = zadd(zmul(c, h.cd00[i]), zmul(s, h.cd10[i]));
        a10 = zadd(zmul(s, h.cd00[i]), zmul(c, h.cd10[i]));
        a01 = zadd(zmul(c, h.cd01[i]), zmul(s, h.cd11[i]));
        a11 = zadd(zmul(s, h.cd01[i]), zmul(c, h.cd11[i]));
    } else {
        const zd c = zcos(ga), s = zsin(ga);
        a00 = zadd(zmul(c, h.cd00[i]), zmul(s, h.cd10[i]));
        a10 = zadd(zmul(zneg(s), h.cd00[i]), zmul(c, h.cd10[i]));
        a01 = zadd(zmul(c, h.cd01[i]), zmul(s, h.cd11[i]));
        a11 = zadd(zmul(zneg(s), h.cd01[i]), zmul(c, h.cd11[i]));
    }
}

// The force-independent log-weight of a sample (getTwoBodySampleFromAux,
// NiupNidn.cpp:100-130): L log(1/2), plus for densityCharge dt U_sum / 2 and
// minus the Kahan sum of aux_i gamma_i (erroranalysisHao/include/kahan.h).
__device__ __forceinline__ zd cp_sample_logw(const HubbardDev &h, const int *aux)
{
    const int L = h.L;
    if (h.decomp != 0) return make_double2(log(0.5) * L, 0.0);
    zd sum = make_double2(0.0, 0.0), comp = make_double2(0.0, 0.0);
    for (int i = 0; i < L; ++i) {
        const zd y = zsub(zscale(h.gamma[i], (double)aux[i]), comp);
        const zd t = zadd(sum, y);
        comp = zsub(zsub(t, sum), y);
        sum = t;
    }
    return zsub(make_double2(log(0.5) * L + h.dtUSum * 0.5, 0.0), sum);
}

// ---------------------------------------------------------------------------
// Hubbard aux-field sampling + two-body sample + its application:
// NiupNidn::sampleAuxFromForce (NiupNidn.cpp:66-84),
// getTwoBodySampleFromAuxForce (:100-142, setTwoBodySampleMatrix :252-322),
// NiupNidnSampleSDOperation::applyToRight (NiupNidnSDOperation.cpp:15-41),
// and the walker log-weight bookkeeping of the driver step
// (afqmcConstraintPathProjection.cpp:63-72).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
cp_sample_apply_kernel(int W, HubbardDev h, const double *force, const int *surv,
                       const unsigned long long *offs, uint64_t seed, const zd *wf, zd *wfTmp,
                       zd *logw, double dtET, zd hopLogw, int *auxOut)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int w = blockIdx.x;
    if (!surv[w]) return;
    const int L = h.L, N = h.N, n = h.n;
    zd *d00 = (zd *)smem_raw, *d01 = d00 + L, *d10 = d00 + 2 * L, *d11 = d00 + 3 * L;
    int *aux = (int *)(d00 + 4 * L);
    double *fs = (double *)(aux + L + (L & 1));
    const double *fw = h.constForce ? h.constForce : force + (size_t)w * L;
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
        double f = fw[i];
        double em = exp(-f), ep = exp(f);
        double prob = em / (em + ep);
        int x = (rng_uniform(seed, offs[w] + (unsigned long long)i) < prob) ? -1 : 1;
        aux[i] = x;
        if (auxOut) auxOut[(size_t)w * L + i] = x;
        fs[i] = x * f - log(ep + em);   // the site's term of the force's log-probability
        cp_site_matrix(h, i, x, d00[i], d01[i], d10[i], d11[i]);
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        // the site terms summed by warp 0 in a fixed order (lane-strided
        // partial sums, then a shuffle tree); the sample's own log-weight keeps
        // the reference's in-order compensated sum
        const int lane = threadIdx.x;
        double lp = 0.0;
        for (int i = lane; i < L; i += 32) lp += fs[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) lp += __shfl_xor_sync(0xffffffffu, lp, o);
        if (lane == 0) {
            zd lw = cp_sample_logw(h, aux);
            lw.x -= lp;
            zd t = zadd(lw, logw[w]);
            t.x += dtET;
            logw[w] = zadd(hopLogw, t);
        }
    }
    const zd *src = wf + (size_t)w * n * N;
    zd *dst = wfTmp + (size_t)w * n * N;
    for (int e = threadIdx.x; e < L * N; e += blockDim.x) {
        int i = e % L, j = e / L;
        zd a = src[i + (size_t)n * j], b = src[i + L + (size_t)n * j];
        zd r0 = zmul(d00[i], a), r1 = zmul(d10[i], a);
        zfma(r0, d01[i], b);
        zfma(r1, d11[i], b);
        dst[i + (size_t)n * j] = r0;
        dst[i + L + (size_t)n * j] = r1;
    }
}

// ---------------------------------------------------------------------------
// Back-propagation pieces (afqmcConstraintPathBP: afqmcConstraintPathMeasure.cpp
// addMeasurement, afqmcConstraintPathBackPropagation.cpp).
//
// A recorded field sample applied to every walker whose record is valid
// (getTwoBodySampleFromAux, NiupNidn.cpp:100-130): to the right
// (NiupNidnSampleSDOperation::applyToRight, NiupNidnSDOperation.cpp:15-41,
// logw += sample logw) or to the left (applyToLeft, :43-68: the 2x2 blocks
// conjugated and their off-diagonals exchanged, logw += conj(sample logw)),
// plus extraLogw (the log-weight of a one-body factor applied after it).
// One block per walker; aux holds L fields per walker.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
cp_aux_apply_kernel(int W, HubbardDev h, const int *aux, const int *valid, const zd *wf, zd *wfOut, zd *logw,
                    int left, zd extraLogw)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int w = blockIdx.x;
    if (!valid[w]) return;
    const int L = h.L, N = h.N, n = h.n;
    zd *d00 = (zd *)smem_raw, *d01 = d00 + L, *d10 = d00 + 2 * L, *d11 = d00 + 3 * L;
    const int *x = aux + (size_t)w * L;
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
        zd a00, a01, a10, a11;
        cp_site_matrix(h, i, x[i], a00, a01, a10, a11);
        if (left) {
            d00[i] = zconj(a00); d01[i] = zconj(a10); d10[i] = zconj(a01); d11[i] = zconj(a11);
        } else {
            d00[i] = a00; d01[i] = a01; d10[i] = a10; d11[i] = a11;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const zd lw = cp_sample_logw(h, x);
        logw[w] = zadd(extraLogw, zadd(left ? zconj(lw) : lw, logw[w]));
    }
    const zd *src = wf + (size_t)w * n * N;
    zd *dst = wfOut + (size_t)w * n * N;
    for (int e = threadIdx.x; e < L * N; e += blockDim.x) {
        const int i = e % L, j = e / L;
        const zd a = src[i + (size_t)n * j], b = src[i + L + (size_t)n * j];
        zd r0 = zmul(d00[i], a), r1 = zmul(d10[i], a);
        zfma(r0, d01[i], b);
        zfma(r1, d11[i], b);
        dst[i + (size_t)n * j] = r0;
        dst[i + L + (size_t)n * j] = r1;
    }
}

// The population-control table applied to recorded rows: for steps
// s < nsteps, row (s, w) takes row (s, table[w]) when table[w] != w
// (AfqmcBackPropagationPop::operator=, the first BPNumber field records of
// the parent).  Parents keep their own slot, so the copies are independent.
__global__ void bp_gather_rows_kernel(int W, int rowlen, int nsteps, const int *table, int *data)
{
    const int w = blockIdx.x, st = blockIdx.y;
    if (w >= W || st >= nsteps) return;
    const int p = table[w];
    if (p == w || p < 0 || p >= W) return;
    const int *src = data + ((size_t)st * W + p) * rowlen;
    int *dst = data + ((size_t)st * W + w) * rowlen;
    for (int i = threadIdx.x; i < rowlen; i += blockDim.x) dst[i] = src[i];
}

// The commute estimator's energies from a walker's full Green's matrix
// (HubbardSOCMeasureCommuteSDSD::addEnergy, :143-188): K = sum K(j,i) G(j,i),
// V = sum_i U_i (G_ii G_{i+L,i+L} - G_{i,i+L} G_{i+L,i}), and the chemical
// potential and field terms; den = exp(logov), as the mixed estimator's.
// One block per walker, fixed-order block reductions.
__global__ void __launch_bounds__(256)
cp_commute_energy_kernel(int W, int L, const zd *G, const zd *K, const double *U, const double *mu,
                         const double *hx, const double *hy, const double *hz, const int *alive,
                         const zd *logov, zd *eloc, zd *den, zd *parts)
{
    __shared__ double red[32];
    const int w = blockIdx.x;
    if (w >= W || !alive[w]) return;
    const int n = 2 * L;
    const zd *g = G + (size_t)w * n * n;
    zd kE = make_double2(0, 0), vE = make_double2(0, 0), rE = make_double2(0, 0);
    for (long long e = threadIdx.x; e < (long long)n * n; e += blockDim.x) kE = zadd(kE, zmul(K[e], g[e]));
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
        auto at = [&](int r, int c) { return g[r + (size_t)n * c]; };
        vE = zadd(vE, zscale(zsub(zmul(at(i, i), at(i + L, i + L)), zmul(at(i, i + L), at(i + L, i))), U[i]));
        rE = zadd(rE, zscale(at(i, i), -mu[i] + hz[i] * 0.5));
        rE = zadd(rE, zscale(at(i + L, i + L), -mu[i] - hz[i] * 0.5));
        rE = zadd(rE, zmul(make_double2(hx[i] * 0.5, -hy[i] * 0.5), at(i, i + L)));
        rE = zadd(rE, zmul(make_double2(hx[i] * 0.5, hy[i] * 0.5), at(i + L, i)));
    }
    kE = block_zsum(kE, red);
    vE = block_zsum(vE, red);
    rE = block_zsum(rE, red);
    if (threadIdx.x == 0) {
        eloc[w] = zadd(zadd(kE, vE), rE);
        den[w] = zexp(logov[w]);
        parts[3 * (size_t)w + 0] = kE;
        parts[3 * (size_t)w + 1] = vE;
        parts[3 * (size_t)w + 2] = rE;
    }
}

__global__ void zconj_kernel(long long count, const zd *src, zd *dst)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
         e += (long long)gridDim.x * blockDim.x)
        dst[e] = zconj(src[e]);
}

// ---------------------------------------------------------------------------
// Phaseless force + aux sampling + sample log-weight + second cos projection:
// RealMaterialMoleculeMeasureFixedSD2sSD2is::getForce (:93-116),
// CholeskyReal::sampleAuxFromForce (choleskyReal.cpp:57-65),
// getTwoBodySampleFromAuxForce (:104-124) and
// afqmcPhaselessProjection.cpp:89-118.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
pl_sample_kernel(int W, CholDev c, const zd *xbar, int *surv, int *alive,
                 const unsigned long long *offs, uint64_t seed, zd *aux, zd *force, zd *logw,
                 double dtET, zd hopLogw)
{
    __shared__ double red[32];
    const int w = blockIdx.x;
    if (!surv[w]) return;
    const int G = c.G;
    zd f2 = make_double2(0, 0), xf = make_double2(0, 0), xb = make_double2(0, 0);
    for (int g = threadIdx.x; g < G; g += blockDim.x) {
        zd f;
        if (c.constForce) {
            f = c.constForce[g];
        } else {
            zd x = xbar[g + (size_t)G * w];
            double a = x.x - c.bg[g], b = x.y;
            f = make_double2(-b * c.sqrtMinusDtIm, a * c.sqrtMinusDtIm);
            double af = zabs(f);
            if (af > c.forceCap) f = make_double2(f.x * c.forceCap / af, f.y * c.forceCap / af);
        }
        double gs = rng_gaussian(seed, offs[w] + 2ULL * g);
        zd x = make_double2(gs + f.x, f.y);
        aux[g + (size_t)G * w] = x;
        force[g + (size_t)G * w] = f;
        zfma(f2, f, f);
        zfma(xf, x, f);
        zfma(xb, x, make_double2(c.bg[g], 0.0));
    }
    f2 = block_zsum(f2, red);
    xf = block_zsum(xf, red);
    xb = block_zsum(xb, red);
    if (threadIdx.x == 0) {
        double phase = xf.y;
        double cs = cos(phase);
        if (cs <= 0.0) {
            alive[w] = 0; surv[w] = 0;
        } else {
            zd lw = logw[w];
            lw.x += log(cs);
            // sample logw = 0.5 f.f - x.f - sqrt(-dt) x.bg, sqrt(-dt) = i sqrtMinusDtIm
            zd smp = zsub(zscale(f2, 0.5), xf);
            smp = zsub(smp, make_double2(-c.sqrtMinusDtIm * xb.y, c.sqrtMinusDtIm * xb.x));
            zd t = zadd(smp, lw);
            t.x += dtET;
            logw[w] = zadd(hopLogw, t);
        }
    }
}

// ---------------------------------------------------------------------------
// Taylor series step of LogHop2isSD2isOperation (logHop2isSD2isOperation.cpp:
// 159-195): walkerNew += term_k, then the dynamicOrder convergence test
// max|term_k| <= accuracy from order checkFrom on.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
taylor_accum_kernel(int W, long long wsize, const zd *term, zd *wfNew, const int *surv, int *done,
                    int *order, int k, int checkFrom, double acc, int isLast, int *status)
{
    __shared__ double red[32];
    const int w = blockIdx.x;
    if (!surv[w] || done[w]) return;
    const zd *t = term + (size_t)w * wsize;
    zd *o = wfNew + (size_t)w * wsize;
    double mx = 0.0;
    for (long long e = threadIdx.x; e < wsize; e += blockDim.x) {
        zd v = t[e];
        zd a = o[e];
        o[e] = zadd(a, v);
        mx = fmax(mx, zabs(v));
    }
    if (k >= checkFrom) {
        mx = block_max(mx, red);
        if (threadIdx.x == 0) {
            if (mx <= acc) { done[w] = 1; order[w] = k; }
            else if (isLast) { done[w] = 1; order[w] = k; atomicOr(status + w, (int)ST_TAYLOR_CAP); }
        }
    }
}

// ---------------------------------------------------------------------------
// Modified Gram-Schmidt orthonormalisation of a walker, replacing the
// Householder QR of SD::stabilize / SD2is::stabilize (SD.cpp:42-56,
// SD2is.cpp:48-76, QRMatrix_cpu tensor_2d_bl_cpu.cpp:263-315).  R's diagonal
// is positive, so logw += sum log R_jj (+ the first Nmin again for SD2is);
// the determinant-invariant quantities (overlaps, G, E_L) equal the
// reference's, whose Q differs by a +-1 column gauge.
// ---------------------------------------------------------------------------
template <bool SMEM>
__global__ void __launch_bounds__(256)
mgs_kernel(int W, int n, int ncol, int nup, int ndn, int isSD2is, zd *wf, zd *logw,
           const int *alive, int *status)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[32];
    const int w = blockIdx.x;
    if (alive && !alive[w]) return;
    zd *g = wf + (size_t)w * n * ncol;
    zd *A = SMEM ? (zd *)smem_raw : g;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
    if (SMEM) {
        for (int e = tid; e < n * ncol; e += nt) A[e] = g[e];
        __syncthreads();
    }
    const int nmin = nup < ndn ? nup : ndn;
    double logR = 0.0, logRmin = 0.0;
    int bad = 0;
    for (int j = 0; j < ncol; ++j) {
        double s = 0.0;
        for (int i = tid; i < n; i += nt) { zd v = A[i + (size_t)n * j]; s += v.x * v.x + v.y * v.y; }
        s = block_sum(s, red);
        double r = sqrt(s);
        if (r == 0.0) bad = 1;
        double inv = r > 0.0 ? 1.0 / r : 0.0;
        for (int i = tid; i < n; i += nt) A[i + (size_t)n * j] = zscale(A[i + (size_t)n * j], inv);
        if (tid == 0) {
            double lr = log(r);
            logR += lr;
            if (j < nmin) logRmin += lr;
        }
        __syncthreads();
        for (int c = j + 1 + wid; c < ncol; c += nw) {
            zd d = make_double2(0.0, 0.0);
            for (int i = lane; i < n; i += 32) zfma(d, zconj(A[i + (size_t)n * j]), A[i + (size_t)n * c]);
            d.x = warp_sum(d.x);
            d.y = warp_sum(d.y);
            for (int i = lane; i < n; i += 32) {
                zd q = A[i + (size_t)n * j];
                zd v = A[i + (size_t)n * c];
                v.x -= d.x * q.x - d.y * q.y;
                v.y -= d.x * q.y + d.y * q.x;
                A[i + (size_t)n * c] = v;
            }
        }
        __syncthreads();
    }
    if (SMEM)
        for (int e = tid; e < n * ncol; e += nt) g[e] = A[e];
    if (tid == 0) {
        zd lw = logw[w];
        if (!isSD2is) lw.x += logR;
        else if (nup == ndn) lw.x += 2.0 * logR;
        else lw.x += logR + logRmin;
        logw[w] = lw;
        if (bad && status) atomicOr(status + w, (int)ST_ZERO_NORM);
    }
}

// ---------------------------------------------------------------------------
// The same Gram-Schmidt with each column in registers: column c belongs to
// TPC adjacent lanes, lane k of the group holding rows k + TPC r (r < 16), so
// a column's reductions are log2(TPC) shuffles inside the group and its
// loads are coalesced.  Step j: the owners of column j form its norm,
// normalise it and publish it as q_j in shared memory (alternate buffers for
// odd and even j); one CTA barrier; every later column c takes
// d = q_j^H a_c and a_c -= d q_j.  Columns and the log R_jj sum keep the
// order of mgs_kernel.  One CTA of ncol * TPC threads per walker.  F32: the
// walkers of the mixed form, fp32 planes [re n x ncol | im n x ncol]; the
// columns stay FP64 in registers through the sweep and are rounded to fp32
// once at the end.
// ---------------------------------------------------------------------------
constexpr int MGSC_RB = 16;   // rows per lane

template <int TPC, bool F32>
__global__ void __launch_bounds__(512, 1)
mgs_col_kernel(int W, int n, int ncol, int nup, int ndn, int isSD2is, void *wfv, zd *logw, const int *alive,
               int *status)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    zd *q = (zd *)smem_raw;                          // [2][n]
    double *logr = (double *)(q + 2 * (size_t)n);    // [ncol]
    __shared__ int badS;
    const int w = blockIdx.x;
    if (alive && !alive[w]) return;   // uniform over the CTA
    const int tid = threadIdx.x, c = tid / TPC, k = tid % TPC;
    const bool col = c < ncol;
    // the shuffles run inside branches taken by whole lane groups only
    const unsigned gmask = (TPC == 32 ? 0xffffffffu : ((1u << TPC) - 1u)) << ((tid & 31) & ~(TPC - 1));
    const size_t ws = (size_t)n * ncol;
    zd *g = F32 ? nullptr : (zd *)wfv + (size_t)w * ws;
    float *g32 = F32 ? (float *)wfv + (size_t)w * 2 * ws : nullptr;
    zd a[MGSC_RB];
#pragma unroll
    for (int r = 0; r < MGSC_RB; ++r) {
        const int i = k + TPC * r;
        const size_t e = i + (size_t)n * c;
        if (!(col && i < n)) a[r] = make_double2(0.0, 0.0);
        else if (F32) a[r] = make_double2(g32[e], g32[ws + e]);
        else a[r] = g[e];
    }
    if (tid == 0) badS = 0;
    for (int j = 0; j < ncol; ++j) {
        zd *qj = q + (size_t)(j & 1) * n;
        if (c == j) {
            double s0 = 0.0, s1 = 0.0;
#pragma unroll
            for (int r = 0; r < MGSC_RB; r += 2) {
                s0 = fma(a[r].x, a[r].x, fma(a[r].y, a[r].y, s0));
                s1 = fma(a[r + 1].x, a[r + 1].x, fma(a[r + 1].y, a[r + 1].y, s1));
            }
            double s = s0 + s1;
#pragma unroll
            for (int o = 1; o < TPC; o <<= 1) s += __shfl_xor_sync(gmask, s, o, TPC);
            const double rj = sqrt(s);
            const double inv = rj > 0.0 ? 1.0 / rj : 0.0;
#pragma unroll
            for (int r = 0; r < MGSC_RB; ++r) {
                a[r] = zscale(a[r], inv);
                const int i = k + TPC * r;
                if (i < n) qj[i] = a[r];
            }
            if (k == 0) {
                logr[j] = log(rj);
                if (rj == 0.0) badS = 1;
            }
        }
        __syncthreads();   // q_j published
        if (col && c > j) {
            zd d0 = make_double2(0.0, 0.0), d1 = make_double2(0.0, 0.0);
#pragma unroll
            for (int r = 0; r < MGSC_RB; r += 2) {
                const int i0 = k + TPC * r, i1 = i0 + TPC;
                if (i0 < n) zfma(d0, zconj(qj[i0]), a[r]);
                if (i1 < n) zfma(d1, zconj(qj[i1]), a[r + 1]);
            }
            zd d = zadd(d0, d1);
#pragma unroll
            for (int o = 1; o < TPC; o <<= 1) {
                d.x += __shfl_xor_sync(gmask, d.x, o, TPC);
                d.y += __shfl_xor_sync(gmask, d.y, o, TPC);
            }
#pragma unroll
            for (int r = 0; r < MGSC_RB; ++r) {
                const int i = k + TPC * r;
                if (i < n) {
                    const zd qv = qj[i];
                    a[r].x -= d.x * qv.x - d.y * qv.y;
                    a[r].y -= d.x * qv.y + d.y * qv.x;
                }
            }
        }
    }
    if (col) {
#pragma unroll
        for (int r = 0; r < MGSC_RB; ++r) {
            const int i = k + TPC * r;
            const size_t e = i + (size_t)n * c;
            if (i < n) {
                if (F32) {
                    g32[e] = (float)a[r].x;
                    g32[ws + e] = (float)a[r].y;
                } else {
                    g[e] = a[r];
                }
            }
        }
    }
    __syncthreads();
    if (tid == 0) {
        const int nmin = nup < ndn ? nup : ndn;
        double logR = 0.0, logRmin = 0.0;
        for (int jj = 0; jj < ncol; ++jj) {
            logR += logr[jj];
            if (jj < nmin) logRmin += logr[jj];
        }
        zd lw = logw[w];
        if (!isSD2is) lw.x += logR;
        else if (nup == ndn) lw.x += 2.0 * logR;
        else lw.x += logR + logRmin;
        logw[w] = lw;
        if (badS && status) atomicOr(status + w, (int)ST_ZERO_NORM);
    }
}

// ---------------------------------------------------------------------------
// popConfiguration (populationControlConfiguration.cpp:24-101) for one
// process: W uniforms from the stream, the comb over the normalised weights
// accumulated in the reference's serial order (bit-exact tables), then the
// slot filling.  The `number[zero_i]` read is bounds-checked first.
// ---------------------------------------------------------------------------
__global__ void pop_comb_kernel(int W, const double *weight, const double *uniforms, uint64_t seed,
                                unsigned long long *counter, int *number, int *table, int *status,
                                int useSmem)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x;
    const unsigned long long c0 = counter ? *counter : 0ULL;
    // stage weights, uniforms and counts in shared memory (parallel), then the
    // comb and the slot filling run serially in the reference's order
    double *sw = useSmem ? (double *)smem_raw : nullptr;
    double *su = useSmem ? sw + W : nullptr;
    int *sn = useSmem ? (int *)(su + W) : number;
    if (useSmem) {
        for (int i = tid; i < W; i += blockDim.x) {
            sw[i] = weight[i];
            su[i] = uniforms ? uniforms[i] : rng_uniform(seed, c0 + (unsigned long long)i);
            sn[i] = 0;
        }
    } else {
        for (int i = tid; i < W; i += blockDim.x) sn[i] = 0;
    }
    __syncthreads();
    if (tid != 0) return;
    const double *wt = useSmem ? sw : weight;
    double sum = 0.0;
    for (int i = 0; i < W; ++i) sum += wt[i];
    int index_old = 0;
    double prob_sum_old = wt[0] / sum;
    for (int i = 0; i < W; ++i) {
        double u = useSmem ? su[i] : (uniforms ? uniforms[i] : rng_uniform(seed, c0 + (unsigned long long)i));
        double prob_sum_new = (i + u) / (W * 1.0);
        while (prob_sum_new > prob_sum_old && index_old < W - 1) {
            index_old++;
            prob_sum_old += wt[index_old] / sum;
        }
        sn[index_old]++;
    }
    if (counter) *counter = c0 + (unsigned long long)W;
    for (int i = 0; i < W; ++i) table[i] = (sn[i] != 0) ? i : -1;
    int zero_i = 0, one_i = 0, max_i = W;
    while (zero_i < max_i && sn[zero_i] != 0) zero_i++;
    while (one_i < max_i && sn[one_i] <= 1) one_i++;
    while (zero_i < max_i && one_i < max_i) {
        table[zero_i] = one_i;
        sn[zero_i]++;
        sn[one_i]--;
        while (zero_i < max_i && sn[zero_i] != 0) zero_i++;
        while (one_i < max_i && sn[one_i] <= 1) one_i++;
    }
    int bad = 0;
    for (int i = 0; i < W; ++i) if (sn[i] != 1) bad = 1;
    if (bad && status) status[0] |= 16;
}

// Same table as pop_comb_kernel, with the serial parts reduced to the two
// FP64 summation chains whose order the reference fixes (the weight sum and
// the running probability sum of popConfiguration,
// populationControlConfiguration.cpp:24-101); everything else is parallel:
//  - sample i lands on the first parent k whose running sum P_k >= (i+u_i)/W
//    (capped at W-1): a binary search, since (i+u_i)/W increases with i and
//    the serial pointer only moves forward;
//  - the k-th empty slot (in index order) receives the k-th surplus copy,
//    parents enumerated in index order, each giving number-1 copies: ranks
//    from block scans and a binary search over the surplus prefix.
// One CTA of 1024 threads; weights, uniforms, sums and counts in shared memory.
constexpr int POP_PAR_THREADS = 1024;

__device__ int block_excl_scan_1024(int v, int *scratch)
{
    // scratch: 32 ints
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) scratch[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int t = scratch[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        scratch[lane] = t;
    }
    __syncthreads();
    const int base = warp > 0 ? scratch[warp - 1] : 0;
    const int r = base + x - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(POP_PAR_THREADS)
pop_comb_par_kernel(int W, const double *weight, const double *uniforms, uint64_t seed,
                    unsigned long long *counter, int *table, int *status)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *sw = (double *)smem_raw;     // weights, then running sums P
    double *su = sw + W;                 // uniforms, then two int arrays
    int *sn = (int *)(su + W);           // copies per parent
    __shared__ int scan[32];
    __shared__ double ssum;
    const int tid = threadIdx.x;
    const unsigned long long c0 = counter ? *counter : 0ULL;
    for (int i = tid; i < W; i += POP_PAR_THREADS) {
        sw[i] = weight[i];
        su[i] = uniforms ? uniforms[i] : rng_uniform(seed, c0 + (unsigned long long)i);
        sn[i] = 0;
    }
    __syncthreads();
    if (tid == 0) {
        double sum = 0.0;
        for (int i = 0; i < W; ++i) sum += sw[i];
        ssum = sum;
    }
    __syncthreads();
    const double sum = ssum;
    for (int i = tid; i < W; i += POP_PAR_THREADS) sw[i] = sw[i] / sum;
    __syncthreads();
    if (tid == 0) {
        double acc = sw[0];
        for (int i = 1; i < W; ++i) {
            acc += sw[i];
            sw[i] = acc;
        }
    }
    __syncthreads();
    for (int i = tid; i < W; i += POP_PAR_THREADS) {
        const double t = (i + su[i]) / (W * 1.0);
        int lo = 0, hi = W - 1;   // first k with P_k >= t, else W - 1
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (t > sw[mid]) lo = mid + 1;
            else hi = mid;
        }
        atomicAdd(&sn[lo], 1);
    }
    __syncthreads();
    if (tid == 0 && counter) *counter = c0 + (unsigned long long)W;
    // ranks of the empty slots and prefix of surplus copies (contiguous chunks per thread)
    int *rankE = (int *)su, *endX = rankE + W;
    const int chunk = (W + POP_PAR_THREADS - 1) / POP_PAR_THREADS;
    const int b0 = min(W, tid * chunk), b1 = min(W, b0 + chunk);
    int ce = 0, cx = 0;
    for (int i = b0; i < b1; ++i) {
        ce += sn[i] == 0 ? 1 : 0;
        cx += sn[i] > 1 ? sn[i] - 1 : 0;
    }
    int e0 = block_excl_scan_1024(ce, scan);
    int x0 = block_excl_scan_1024(cx, scan);
    for (int i = b0; i < b1; ++i) {
        rankE[i] = e0;
        e0 += sn[i] == 0 ? 1 : 0;
        x0 += sn[i] > 1 ? sn[i] - 1 : 0;
        endX[i] = x0;
    }
    __syncthreads();
    int bad = 0;
    for (int i = tid; i < W; i += POP_PAR_THREADS) {
        if (sn[i] != 0) {
            table[i] = i;
        } else {
            const int k = rankE[i];
            int lo = 0, hi = W - 1;   // first parent whose surplus prefix exceeds k
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (endX[mid] > k) hi = mid;
                else lo = mid + 1;
            }
            if (endX[lo] > k) table[i] = lo;
            else { table[i] = -1; bad = 1; }
        }
    }
    if (bad && status) atomicOr(status, 16);
}

// populationControl<T> serial branch (populationControl.h:110-117): parents
// keep their own slot, so the copies can run in parallel in place.
__global__ void pop_gather_kernel(int W, long long wsize, const int *table, zd *wf, zd *logw)
{
    const int i = blockIdx.x;
    const int j = table[i];
    if (j == i || j < 0) return;
    const zd *src = wf + (size_t)j * wsize;
    zd *dst = wf + (size_t)i * wsize;
    for (long long e = threadIdx.x; e < wsize; e += blockDim.x) dst[e] = src[e];
    if (threadIdx.x == 0) logw[i] = logw[j];
}

// Observables of HubbardSOCMeasureObserveSDSD::addMeasurement
// (HubbardSOCMeasureObserveSDSD.cpp:42-185), den-weighted and summed over the
// alive walkers: greenMatrixNum and densityDensityNum (n x n, n = 2L), and
// splusSminusNum, sminusSplusNum, spairSpairNum (L x L).  One thread per
// element (i, j); each sums over the walkers in order, so the sums are
// reproducible.  G holds each walker's full Green's matrix, column-major.
__global__ void __launch_bounds__(256)
cp_observe_kernel(int W, int L, const zd *G, const zd *den, const int *alive, zd *gNum, zd *ddNum,
                  zd *pmNum, zd *mpNum, zd *pairNum)
{
    const int n = 2 * L;
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= (long long)n * n) return;
    const int i = (int)(e % n), j = (int)(e / n);
    const bool small = i < L && j < L;
    zd sg = make_double2(0, 0), sd = make_double2(0, 0), spm = make_double2(0, 0), smp = make_double2(0, 0),
       spr = make_double2(0, 0);
    for (int w = 0; w < W; ++w) {
        if (!alive[w]) continue;
        const zd d = den[w];
        const zd *g = G + (size_t)w * n * n;
        auto at = [&](int r, int c) { return g[r + (size_t)n * c]; };
        const zd gij = at(i, j);
        sg = zadd(sg, zmul(gij, d));
        const zd dd = (i == j) ? at(i, i) : zsub(zmul(at(i, i), at(j, j)), zmul(gij, at(j, i)));
        sd = zadd(sd, zmul(dd, d));
        if (small) {
            zd pm, mp;
            if (i == j) {
                const zd both = zsub(zmul(at(i, i), at(i + L, i + L)), zmul(at(i, i + L), at(i + L, i)));
                pm = zsub(at(i, i), both);
                mp = zsub(at(i + L, i + L), both);
            } else {
                pm = zadd(zneg(zmul(gij, at(j + L, i + L))), zmul(at(i, i + L), at(j + L, j)));
                mp = zadd(zneg(zmul(at(i + L, j + L), at(j, i))), zmul(at(i + L, i), at(j, j + L)));
            }
            const zd pr = zsub(zmul(gij, at(i + L, j + L)), zmul(at(i, j + L), at(i + L, j)));
            spm = zadd(spm, zmul(pm, d));
            smp = zadd(smp, zmul(mp, d));
            spr = zadd(spr, zmul(pr, d));
        }
    }
    gNum[e] = zadd(gNum[e], sg);
    ddNum[e] = zadd(ddNum[e], sd);
    if (small) {
        const long long s = i + (long long)L * j;
        pmNum[s] = zadd(pmNum[s], spm);
        mpNum[s] = zadd(mpNum[s], smp);
        pairNum[s] = zadd(pairNum[s], spr);
    }
}

// Walkers idx[k] -> transfer record k of buf (the walker's matrix, then its
// logw), or back (unpack: record k -> slot idx[k]); one block per record.
__global__ void walker_xfer_kernel(int count, long long wsize, const int *idx, zd *wf, zd *logw, zd *buf,
                                   int unpack)
{
    const int k = blockIdx.x;
    if (k >= count) return;
    const int w = idx[k];
    zd *rec = buf + (size_t)k * (wsize + 1);
    zd *mat = wf + (size_t)w * wsize;
    if (unpack) {
        for (long long e = threadIdx.x; e < wsize; e += blockDim.x) mat[e] = rec[e];
        if (threadIdx.x == 0) logw[w] = rec[wsize];
    } else {
        for (long long e = threadIdx.x; e < wsize; e += blockDim.x) rec[e] = mat[e];
        if (threadIdx.x == 0) rec[wsize] = logw[w];
    }
}

__global__ void set_int_kernel(int *p, int v, int count)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) p[i] = v;
}

__global__ void copy_masked_kernel(int W, long long wsize, const zd *src, zd *dst, const int *mask)
{
    const int w = blockIdx.x;
    if (mask && !mask[w]) return;
    const zd *s = src + (size_t)w * wsize;
    zd *d = dst + (size_t)w * wsize;
    for (long long e = threadIdx.x; e < wsize; e += blockDim.x) d[e] = s[e];
}

// ---------------------------------------------------------------------------
// Hubbard local energy: HubbardSOCMeasureFixedSDSD::addEnergy (:178-218).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
cp_energy_kernel(int W, HubbardDev h, const zd *wfDaggerK, const zd *thetaT, long long tStride,
                 const double *U, const double *mu, const double *hx, const double *hy,
                 const double *hz, const int *alive, const zd *logov, zd *eloc, zd *den,
                 zd *parts, zd *sites)
{
    __shared__ double red[32];
    const int w = blockIdx.x;
    if (!alive[w]) return;
    const int L = h.L, N = h.N, n = h.n;
    const zd *th = thetaT + (size_t)w * tStride;
    // site terms of addNupNdn / addSplusSminus (HubbardSOCMeasureFixedSDSD.cpp:221-255)
    zd *st = sites + (size_t)w * 4 * L;
    zd K = make_double2(0, 0), V = make_double2(0, 0), R = make_double2(0, 0);
    for (int e = threadIdx.x; e < N * n; e += blockDim.x) zfma(K, wfDaggerK[e], th[e]);
    // P adjacent lanes per site, lane p taking j = p, p + P, ...: the loads of a
    // site come in runs of P entries and each sum is N / P long; the P
    // partial sums meet in a shuffle tree
    const int P = L >= 256 ? 1 : L >= 128 ? 2 : L >= 64 ? 4 : 8;
    const int part = threadIdx.x % P;
    const int sitesPerPass = blockDim.x / P;
    for (int i0 = 0; i0 < L; i0 += sitesPerPass) {
        const int i = i0 + threadIdx.x / P;
        const bool site = i < L;   // uniform over each lane group of P
        zd gi = make_double2(0, 0), gL = make_double2(0, 0), oi = make_double2(0, 0), oL = make_double2(0, 0);
        if (site) {
            for (int j = part; j < N; j += P) {
                zd pi = zconj(h.phiT[i + (size_t)n * j]), pL = zconj(h.phiT[i + L + (size_t)n * j]);
                zfma(gi, pi, th[j + (size_t)N * i]);
                zfma(gL, pL, th[j + (size_t)N * (i + L)]);
                zfma(oi, pi, th[j + (size_t)N * (i + L)]);
                zfma(oL, pL, th[j + (size_t)N * i]);
            }
        }
        for (int o = 1; o < P; o <<= 1) {
            gi.x += __shfl_xor_sync(0xffffffffu, gi.x, o); gi.y += __shfl_xor_sync(0xffffffffu, gi.y, o);
            gL.x += __shfl_xor_sync(0xffffffffu, gL.x, o); gL.y += __shfl_xor_sync(0xffffffffu, gL.y, o);
            oi.x += __shfl_xor_sync(0xffffffffu, oi.x, o); oi.y += __shfl_xor_sync(0xffffffffu, oi.y, o);
            oL.x += __shfl_xor_sync(0xffffffffu, oL.x, o); oL.y += __shfl_xor_sync(0xffffffffu, oL.y, o);
        }
        if (!site || part != 0) continue;
        st[i] = gi;
        st[i + L] = gL;
        st[i + 2 * L] = oi;
        st[i + 3 * L] = oL;
        zd t = zsub(zmul(gi, gL), zmul(oi, oL));
        V = zadd(V, zscale(t, U[i]));
        R = zadd(R, zscale(gi, -mu[i] + hz[i] * 0.5));
        R = zadd(R, zscale(gL, -mu[i] - hz[i] * 0.5));
        R = zadd(R, zmul(make_double2(hx[i] * 0.5, -hy[i] * 0.5), oi));
        R = zadd(R, zmul(make_double2(hx[i] * 0.5, hy[i] * 0.5), oL));
    }
    K = block_zsum(K, red);
    V = block_zsum(V, red);
    R = block_zsum(R, red);
    if (threadIdx.x == 0) {
        eloc[w] = zadd(zadd(K, V), R);
        den[w] = zexp(logov[w]);
        parts[3 * (size_t)w + 0] = K;
        parts[3 * (size_t)w + 1] = V;
        parts[3 * (size_t)w + 2] = R;
    }
}

// ---------------------------------------------------------------------------
// Exchange term ex_g = sum_sigma tr(D D), D = A_g,sigma theta_sigma
// (RealMaterialMoleculeMeasureFixedSD2sSD2is::calculateCholeskyEx :258-284);
// grid (walker, g-chunk), operand chunks of 32 orbitals staged in smem.
// ---------------------------------------------------------------------------
constexpr int EX_KC = 32;
constexpr int EX_GCH = 16;

// dynamic smem: As[Ns*EX_KC], Ts[Ns*EX_KC], Ds[Ns*Ns] for the largest block
__global__ void __launch_bounds__(256)
pl_exchange_kernel(int W, int n, int G, Blocks bl, const zd *Aall, long long Ktot,
                   const zd *thetaT, const int *alive, zd *ex, int maxNs, int thetaLayout)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    zd *As = (zd *)smem_raw;
    zd *Ts = As + maxNs * EX_KC;
    zd *Ds = Ts + maxNs * EX_KC;
    __shared__ double red[32];
    const int w = blockIdx.x;
    if (!alive[w]) return;
    const int g0 = blockIdx.y * EX_GCH;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int g = g0; g < G && g < g0 + EX_GCH; ++g) {
        zd exg = make_double2(0.0, 0.0);
        for (int b = 0; b < bl.nblk; ++b) {
            const int Ns = bl.Ns[b];
            if (Ns == 0) continue;
            const zd *A = Aall + (size_t)g * Ktot + bl.tOff[b];
            const zd *T = thetaT + (size_t)w * bl.tStride + bl.tOff[b];
            const int ne = Ns * Ns;
            zd acc[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) acc[q] = make_double2(0.0, 0.0);
            for (int i0 = 0; i0 < n; i0 += EX_KC) {
                int kc = min(EX_KC, n - i0);
                for (int e = tid; e < Ns * kc; e += nt) {
                    As[e] = A[(size_t)Ns * i0 + e];
                    // thetaLayout 0: thetaT (b + Ns i); 1: theta (i + n b)
                    Ts[e] = thetaLayout == 0 ? T[(size_t)Ns * i0 + e]
                                             : T[(size_t)(i0 + e / Ns) + (size_t)n * (e % Ns)];
                }
                __syncthreads();
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    int e = tid + q * nt;
                    if (e < ne) {
                        int a = e % Ns, bb = e / Ns;
                        zd s = acc[q];
                        for (int ii = 0; ii < kc; ++ii) zfma(s, As[a + Ns * ii], Ts[bb + Ns * ii]);
                        acc[q] = s;
                    }
                }
                __syncthreads();
            }
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                int e = tid + q * nt;
                if (e < ne) Ds[e] = acc[q];
            }
            __syncthreads();
            zd part = make_double2(0.0, 0.0);
            for (int e = tid; e < ne; e += nt) {
                int a = e % Ns, bb = e / Ns;
                zfma(part, Ds[a + Ns * bb], Ds[bb + Ns * a]);
            }
            part = block_zsum(part, red);
            exg = zadd(exg, part);
        }
        if (tid == 0) ex[g + (size_t)G * w] = exg;
    }
}

// ---------------------------------------------------------------------------
// Phaseless local energy: addEnergy (:197-220) with calculateTenergy
// (:222-235); T is an elementwise product in the stacked thetaT layout.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
pl_energy_kernel(int W, int G, long long Ktot, const zd *wfDaggerT, const zd *thetaT,
                 const zd *xbar, const zd *ex, const zd *exTot, const int *alive, const zd *logov,
                 zd *eloc, zd *den, zd *tloc, long long tLen, int tMult)
{
    __shared__ double red[32];
    const int w = blockIdx.x;
    if (!alive[w]) return;
    const zd *th = thetaT + (size_t)w * Ktot;
    zd T = make_double2(0, 0), H = make_double2(0, 0);
    for (long long e = threadIdx.x; e < tLen; e += blockDim.x) zfma(T, wfDaggerT[e], th[e]);
    for (int g = threadIdx.x; g < G; g += blockDim.x) {
        zd x = xbar[g + (size_t)G * w];
        zd t = zmul(x, x);
        H = zadd(H, exTot ? t : zsub(t, ex[g + (size_t)G * w]));
    }
    T = block_zsum(T, red);
    H = block_zsum(H, red);
    if (threadIdx.x == 0) {
        if (tMult == 2) T = zadd(T, T);
        if (exTot) H = zsub(H, exTot[w]);
        zd e = zadd(zscale(H, 0.5), T);
        eloc[w] = e;
        den[w] = zexp(logov[w]);
        if (tloc) tloc[w] = T;
    }
}

// Accumulate the estimator numerators/denominator over alive walkers
// (writeThreadSum / MPISum of the reference become plain sums).  Block 0
// reduces the scalars, block 1+g the per-vector sums of g; each block sums a
// fixed strided partition then a fixed tree, so the order is reproducible.
__device__ __forceinline__ zd block_zsum_fixed(zd v, double *scratch)
{
    return block_zsum(v, scratch);
}

__global__ void __launch_bounds__(256)
measure_reduce_kernel(int W, const int *alive, const zd *eloc, const zd *den, const zd *parts,
                      int nparts, zd *acc, int G, const zd *xbar, const zd *ex, zd *bgNum,
                      zd *exNum)
{
    __shared__ double red[32];
    const int tid = threadIdx.x, nt = blockDim.x;
    if (blockIdx.x == 0) {
        zd sd = make_double2(0, 0), sh = make_double2(0, 0);
        zd sp[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
        for (int w = tid; w < W; w += nt) {
            if (!alive[w]) continue;
            zd d = den[w];
            sd = zadd(sd, d);
            sh = zadd(sh, zmul(eloc[w], d));
            for (int k = 0; k < nparts; ++k) sp[k] = zadd(sp[k], zmul(parts[(size_t)nparts * w + k], d));
        }
        sd = block_zsum_fixed(sd, red);
        sh = block_zsum_fixed(sh, red);
        for (int k = 0; k < nparts; ++k) sp[k] = block_zsum_fixed(sp[k], red);
        if (tid == 0) {
            acc[0] = zadd(acc[0], sd);
            acc[1] = zadd(acc[1], sh);
            for (int k = 0; k < nparts; ++k) acc[2 + k] = zadd(acc[2 + k], sp[k]);
        }
        return;
    }
    const int g = blockIdx.x - 1;
    if (!xbar || g >= G) return;
    zd sb = make_double2(0, 0), se = make_double2(0, 0);
    for (int w = tid; w < W; w += nt) {
        if (!alive[w]) continue;
        zd d = den[w];
        sb = zadd(sb, zmul(xbar[g + (size_t)G * w], d));
        if (ex) se = zadd(se, zmul(ex[g + (size_t)G * w], d));
    }
    sb = block_zsum_fixed(sb, red);
    se = block_zsum_fixed(se, red);
    if (tid == 0) {
        bgNum[g] = zadd(bgNum[g], sb);
        if (ex) exNum[g] = zadd(exNum[g], se);
    }
}

// FP64 inverses -> fp32 planes [re | im] (each Ns x Ns column-major), for the
// LU kernels that write FP64 only
__global__ void sinv_to_f32_kernel(int W, Blocks bl, const zd *Sinv, float *Sinv32, long long s32)
{
    const int w = blockIdx.x;
    for (int b = 0; b < bl.nblk; ++b) {
        const int Ns = b == 0 ? bl.Ns[0] : bl.Ns[1];
        const long long sOff = b == 0 ? bl.sOff[0] : bl.sOff[1];
        const zd *X = Sinv + (size_t)w * bl.sStride + sOff;
        float *Xr = Sinv32 + (size_t)w * s32 + 2 * sOff, *Xi = Xr + (size_t)Ns * Ns;
        for (int e = threadIdx.x; e < Ns * Ns; e += blockDim.x) {
            const zd v = X[e];
            Xr[e] = (float)v.x;
            Xi[e] = (float)v.y;
        }
    }
}

}  // namespace

// ============================================================== launchers
static void launch_lu_fp64(int W, const Blocks &bl, zd *S, zd *Sinv, const int *active, const zd *logw,
                           zd logwAdd, zd logwT, zd *logov, int *alive, int *surv, zd *logwOut,
                           double *weight, int *status, int mode, bool wantInverse, cudaStream_t s);

void launch_lu_logdet_inverse(int W, const Blocks &bl, zd *S, zd *Sinv, const int *active,
                              const zd *logw, zd logwAdd, zd logwT, zd *logov, int *alive,
                              int *surv, zd *logwOut, double *weight, int *status, int mode,
                              bool wantInverse, cudaStream_t s)
{
    launch_lu_logdet_inverse32(W, bl, S, Sinv, nullptr, active, logw, logwAdd, logwT, logov, alive, surv,
                               logwOut, weight, status, mode, wantInverse, s);
}

// the split-window register LU: one CTA per block, the two blocks of a
// two-block walker as a cluster of two CTAs
template <int SL, int RH, int NQ>
static void launch_regw(int W, const Blocks &bl, zd *S, zd *X64, float *Sinv32, long long s32, const int *active,
                        const zd *logw, zd logwAdd, zd logwT, zd *logov, int *alive, int *surv, zd *logwOut,
                        double *weight, int *status, int mode, int inv, cudaStream_t s)
{
    constexpr int T = 32 * RH * NQ;
    if (bl.nblk == 1) {
        gj_regw_kernel<1, SL, RH, NQ><<<W, T, 0, s>>>(W, bl, S, X64, Sinv32, s32, active, logw, logwAdd, logwT,
                                                      logov, alive, surv, logwOut, weight, status, mode, inv);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(2 * W));
    cfg.blockDim = dim3(T);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, gj_regw_kernel<2, SL, RH, NQ>, W, bl, (const zd *)S, X64, Sinv32, s32, active, logw,
                       logwAdd, logwT, logov, alive, surv, logwOut, weight, status, mode, inv);
}

void launch_lu_logdet_inverse32(int W, const Blocks &bl, zd *S, zd *Sinv, float *Sinv32, const int *active,
                                const zd *logw, zd logwAdd, zd logwT, zd *logov, int *alive, int *surv,
                                zd *logwOut, double *weight, int *status, int mode, bool wantInverse,
                                cudaStream_t s)
{
    int maxNs = 0;
    for (int b = 0; b < bl.nblk; ++b) maxNs = bl.Ns[b] > maxNs ? bl.Ns[b] : maxNs;
    const long long s32 = sinv32_stride(bl);
    if (maxNs > 16 && maxNs <= 64 && (bl.nblk == 1 || bl.nblk == 2)) {
        g_launch_count++;
        if (maxNs <= 32)
            launch_regw<16, 1, 2>(W, bl, S, Sinv32 ? nullptr : Sinv, Sinv32, s32, active, logw, logwAdd, logwT, logov,
                               alive, surv, logwOut, weight, status, mode, wantInverse ? 1 : 0, s);
        else
            launch_regw<32, 2, 2>(W, bl, S, Sinv32 ? nullptr : Sinv, Sinv32, s32, active, logw, logwAdd, logwT, logov,
                               alive, surv, logwOut, weight, status, mode, wantInverse ? 1 : 0, s);
        return;
    }
    launch_lu_fp64(W, bl, S, Sinv, active, logw, logwAdd, logwT, logov, alive, surv, logwOut, weight, status,
                   mode, wantInverse, s);
    if (Sinv32 && wantInverse && Sinv) {
        g_launch_count++;
        sinv_to_f32_kernel<<<W, 256, 0, s>>>(W, bl, Sinv, Sinv32, s32);
    }
}

static void launch_lu_fp64(int W, const Blocks &bl, zd *S, zd *Sinv, const int *active, const zd *logw,
                           zd logwAdd, zd logwT, zd *logov, int *alive, int *surv, zd *logwOut,
                           double *weight, int *status, int mode, bool wantInverse, cudaStream_t s)
{
    g_launch_count++;
    int maxNs = 0;
    for (int b = 0; b < bl.nblk; ++b) maxNs = bl.Ns[b] > maxNs ? bl.Ns[b] : maxNs;
    if (maxNs <= 32) {
        const size_t smem = (size_t)GJ_WARPS * 32 * GJ_LD * sizeof(zd);
        static std::atomic<unsigned long long> gattr{0};
        if (first_on_device(gattr)) {
            cudaFuncSetAttribute(gj_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        }
        gj_warp_kernel<<<(W + GJ_WARPS - 1) / GJ_WARPS, GJ_WARPS * 32, smem, s>>>(
            W, bl, S, Sinv, active, logw, logwAdd, logwT, logov, alive, surv, logwOut, weight, status,
            mode, wantInverse ? 1 : 0);
        return;
    }
    if (maxNs <= GJ_CTA_MAX_NS) {
        const size_t smem = gj_cta_smem(maxNs);
        static std::atomic<unsigned long long> cattr{0};
        if (first_on_device(cattr)) {
            cudaFuncSetAttribute(gj_cta_kernel<256, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)gj_cta_smem(64));
            cudaFuncSetAttribute(gj_cta_kernel<512, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)gj_cta_smem(GJ_CTA_MAX_NS));
        }
        if (maxNs <= 64)
            gj_cta_kernel<256, 2><<<W, 256, smem, s>>>(W, bl, S, Sinv, active, logw, logwAdd, logwT, logov,
                                                        alive, surv, logwOut, weight, status, mode,
                                                        wantInverse ? 1 : 0, maxNs);
        else
            gj_cta_kernel<512, 4><<<W, 512, smem, s>>>(W, bl, S, Sinv, active, logw, logwAdd, logwT, logov,
                                                        alive, surv, logwOut, weight, status, mode,
                                                        wantInverse ? 1 : 0, maxNs);
        return;
    }
    if (maxNs <= LU_SMEM_MAX_NS) {
        size_t smem = (size_t)2 * maxNs * maxNs * sizeof(zd) + (size_t)(maxNs + 4) * sizeof(int);
        static std::atomic<unsigned long long> attr{0};
        if (first_on_device(attr)) {
            cudaFuncSetAttribute(lu_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
        }
        lu_kernel<true><<<W, 256, smem, s>>>(W, bl, S, Sinv, active, logw, logwAdd, logwT, logov,
                                              alive, surv, logwOut, weight, status, mode,
                                              wantInverse ? 1 : 0, maxNs);
    } else {
        size_t smem = (size_t)(maxNs + 4) * sizeof(int);
        lu_kernel<false><<<W, 256, smem, s>>>(W, bl, S, Sinv, active, logw, logwAdd, logwT, logov,
                                               alive, surv, logwOut, weight, status, mode,
                                               wantInverse ? 1 : 0, maxNs);
    }
}

void launch_rng_scan(int W, const int *surv, int draws, unsigned long long *counter,
                     unsigned long long *offs, cudaStream_t s)
{
    g_launch_count++;
    rng_scan_kernel<<<1, 1024, 0, s>>>(W, surv, draws, counter, offs);
}

void launch_cp_force(int W, const HubbardDev &h, const zd *thetaT, long long tStride,
                     const int *surv, double *force, cudaStream_t s)
{
    g_launch_count++;
    cp_force_kernel<<<W, 128, 0, s>>>(W, h, thetaT, tStride, surv, force);
}

void launch_cp_sample_apply(int W, const HubbardDev &h, const double *force, const int *surv,
                            const unsigned long long *offs, uint64_t seed, const zd *wf,
                            zd *wfTmp, zd *logw, double dtET, zd hopLogw, int *auxOut,
                            cudaStream_t s)
{
    g_launch_count++;
    size_t smem = (size_t)4 * h.L * sizeof(zd) + (size_t)(h.L + 1) * sizeof(int) + (size_t)h.L * sizeof(double) + 16;
    cp_sample_apply_kernel<<<W, 256, smem, s>>>(W, h, force, surv, offs, seed, wf, wfTmp, logw,
                                                 dtET, hopLogw, auxOut);
}

void launch_pl_sample(int W, const CholDev &c, const zd *xbar, const int *surv_in, int *surv,
                      int *alive, const unsigned long long *offs, uint64_t seed, zd *aux,
                      zd *force, zd *logw, double dtET, zd hopLogw, cudaStream_t s)
{
    g_launch_count++;
    (void)surv_in;
    pl_sample_kernel<<<W, 256, 0, s>>>(W, c, xbar, surv, alive, offs, seed, aux, force, logw, dtET,
                                        hopLogw);
}

void launch_taylor_accum(int W, long long wsize, const zd *term, zd *wfNew, const int *surv,
                         int *done, int *order, int k, int checkFrom, double acc, int isLast,
                         int *status, cudaStream_t s)
{
    g_launch_count++;
    taylor_accum_kernel<<<W, 256, 0, s>>>(W, wsize, term, wfNew, surv, done, order, k, checkFrom,
                                           acc, isLast, status);
}

// Gram-Schmidt with the columns in registers (mgs_col_kernel) where
// ncol * TPC lanes fit one CTA of 512; false where the shape does not fit.
bool launch_mgs_col(int W, int n, int ncol, int nup, int ndn, int isSD2is, void *wf, bool f32, zd *logw,
                    const int *alive, int *status, cudaStream_t s)
{
    int tpc = 1;
    while (tpc * MGSC_RB < n && tpc < 32) tpc <<= 1;
    if (!(tpc * MGSC_RB >= n && tpc <= 16 && ncol * tpc <= 512 && ncol > 0)) return false;
    const int threads = (ncol * tpc + 31) / 32 * 32;
    const size_t smem = (size_t)2 * n * sizeof(zd) + (size_t)ncol * sizeof(double);
#define MGSC_LAUNCH(T)                                                                                     \
    (f32 ? mgs_col_kernel<T, true><<<W, threads, smem, s>>>(W, n, ncol, nup, ndn, isSD2is, wf, logw, alive, \
                                                             status)                                        \
         : mgs_col_kernel<T, false><<<W, threads, smem, s>>>(W, n, ncol, nup, ndn, isSD2is, wf, logw, alive, \
                                                              status))
    switch (tpc) {
    case 1: MGSC_LAUNCH(1); break;
    case 2: MGSC_LAUNCH(2); break;
    case 4: MGSC_LAUNCH(4); break;
    case 8: MGSC_LAUNCH(8); break;
    default: MGSC_LAUNCH(16); break;
    }
#undef MGSC_LAUNCH
    return true;
}

void launch_mgs(int W, int n, int ncol, int nup, int ndn, int isSD2is, zd *wf, zd *logw,
                const int *alive, int *status, cudaStream_t s)
{
    g_launch_count++;
    if (launch_mgs_col(W, n, ncol, nup, ndn, isSD2is, wf, false, logw, alive, status, s)) return;
    size_t bytes = (size_t)n * ncol * sizeof(zd);
    if (bytes <= 160 * 1024) {
        static std::atomic<unsigned long long> attr{0};
        if (first_on_device(attr)) {
            cudaFuncSetAttribute(mgs_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
        }
        mgs_kernel<true><<<W, 256, bytes, s>>>(W, n, ncol, nup, ndn, isSD2is, wf, logw, alive, status);
    } else {
        mgs_kernel<false><<<W, 256, 0, s>>>(W, n, ncol, nup, ndn, isSD2is, wf, logw, alive, status);
    }
}

void launch_pop_comb(int W, const double *weight, const double *uniforms, uint64_t seed,
                     unsigned long long *counter, int *number, int *table, int *status,
                     cudaStream_t s)
{
    g_launch_count++;
    const size_t smem = (size_t)W * (2 * sizeof(double) + sizeof(int));
    if (smem <= 200 * 1024) {
        static std::atomic<unsigned long long> pattr{0};
        if (first_on_device(pattr)) {
            cudaFuncSetAttribute(pop_comb_par_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        }
        pop_comb_par_kernel<<<1, POP_PAR_THREADS, smem, s>>>(W, weight, uniforms, seed, counter, table, status);
        return;
    }
    const int useSmem = smem <= 160 * 1024 ? 1 : 0;
    static std::atomic<unsigned long long> attr{0};
    if (first_on_device(attr)) {
        cudaFuncSetAttribute(pop_comb_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    }
    pop_comb_kernel<<<1, 256, useSmem ? smem : 0, s>>>(W, weight, uniforms, seed, counter, number, table,
                                                       status, useSmem);
}

void launch_pop_gather(int W, long long wsize, const int *table, zd *wf, zd *logw, cudaStream_t s)
{
    g_launch_count++;
    pop_gather_kernel<<<W, 256, 0, s>>>(W, wsize, table, wf, logw);
}

void launch_cp_observe(int W, int L, const zd *G, const zd *den, const int *alive, zd *obs, cudaStream_t s)
{
    g_launch_count++;
    const long long n2 = 4LL * L * L, l2 = (long long)L * L;
    cp_observe_kernel<<<(unsigned)((n2 + 255) / 256), 256, 0, s>>>(W, L, G, den, alive, obs, obs + n2, obs + 2 * n2,
                                                                  obs + 2 * n2 + l2, obs + 2 * n2 + 2 * l2);
}

void launch_cp_aux_apply(int W, const HubbardDev &h, const int *aux, const int *valid, const zd *wf, zd *wfOut,
                         zd *logw, bool left, zd extraLogw, cudaStream_t s)
{
    g_launch_count++;
    cp_aux_apply_kernel<<<W, 256, (size_t)4 * h.L * sizeof(zd), s>>>(W, h, aux, valid, wf, wfOut, logw, left ? 1 : 0,
                                                                      extraLogw);
}

void launch_bp_gather_rows(int W, int rowlen, int nsteps, const int *table, int *data, cudaStream_t s)
{
    if (nsteps <= 0) return;
    g_launch_count++;
    bp_gather_rows_kernel<<<dim3((unsigned)W, (unsigned)nsteps), 64, 0, s>>>(W, rowlen, nsteps, table, data);
}

void launch_cp_commute_energy(int W, int L, const zd *G, const zd *K, const double *U, const double *mu,
                              const double *hx, const double *hy, const double *hz, const int *alive,
                              const zd *logov, zd *eloc, zd *den, zd *parts, cudaStream_t s)
{
    g_launch_count++;
    cp_commute_energy_kernel<<<W, 256, 0, s>>>(W, L, G, K, U, mu, hx, hy, hz, alive, logov, eloc, den, parts);
}

void launch_zconj(long long count, const zd *src, zd *dst, cudaStream_t s)
{
    g_launch_count++;
    const long long blocks = std::min<long long>((count + 255) / 256, 4096);
    zconj_kernel<<<(unsigned)blocks, 256, 0, s>>>(count, src, dst);
}

void launch_walker_xfer(int count, long long wsize, const int *idx, zd *wf, zd *logw, zd *buf, bool unpack,
                        cudaStream_t s)
{
    g_launch_count++;
    walker_xfer_kernel<<<count, 256, 0, s>>>(count, wsize, idx, wf, logw, buf, unpack ? 1 : 0);
}

void launch_set_int(int *p, int v, int count, cudaStream_t s)
{
    g_launch_count++;
    set_int_kernel<<<(count + 255) / 256, 256, 0, s>>>(p, v, count);
}

void launch_copy_masked(int W, long long wsize, const zd *src, zd *dst, const int *mask,
                        cudaStream_t s)
{
    g_launch_count++;
    copy_masked_kernel<<<W, 256, 0, s>>>(W, wsize, src, dst, mask);
}

void launch_cp_energy(int W, const HubbardDev &h, const zd *wfDaggerK, const zd *thetaT,
                      long long tStride, const double *U, const double *mu, const double *hx,
                      const double *hy, const double *hz, const int *alive, const zd *logov,
                      zd *eloc, zd *den, zd *parts, zd *sites, cudaStream_t s)
{
    g_launch_count++;
    cp_energy_kernel<<<W, 256, 0, s>>>(W, h, wfDaggerK, thetaT, tStride, U, mu, hx, hy, hz, alive,
                                        logov, eloc, den, parts, sites);
}

int launch_pl_exchange(int W, int n, int G, const Blocks &bl, const zd *Aall, long long Ktot,
                       const zd *thetaT, const int *alive, zd *ex, cudaStream_t s, int thetaLayout)
{
    g_launch_count++;
    int maxNs = 0;
    for (int b = 0; b < bl.nblk; ++b) maxNs = bl.Ns[b] > maxNs ? bl.Ns[b] : maxNs;
    if (maxNs > 64) return -1;
    size_t smem = ((size_t)2 * maxNs * EX_KC + (size_t)maxNs * maxNs) * sizeof(zd);
    static std::atomic<unsigned long long> attr{0};
    if (first_on_device(attr)) {
        cudaFuncSetAttribute(pl_exchange_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    }
    dim3 grid(W, (G + EX_GCH - 1) / EX_GCH);
    pl_exchange_kernel<<<grid, 256, smem, s>>>(W, n, G, bl, Aall, Ktot, thetaT, alive, ex, maxNs,
                                                thetaLayout);
    return 0;
}

void launch_pl_energy(int W, int G, long long Ktot, const zd *wfDaggerT, const zd *thetaT,
                      const zd *xbar, const zd *ex, const int *alive, const zd *logov, zd *eloc,
                      zd *den, zd *tloc, cudaStream_t s, const zd *exTot, long long tLen, int tMult)
{
    g_launch_count++;
    pl_energy_kernel<<<W, 256, 0, s>>>(W, G, Ktot, wfDaggerT, thetaT, xbar, ex, exTot, alive, logov,
                                        eloc, den, tloc, tLen < 0 ? Ktot : tLen, tMult);
}

void launch_measure_reduce(int W, const int *alive, const zd *eloc, const zd *den, const zd *parts,
                           int nparts, zd *acc, int G, const zd *xbar, const zd *ex, zd *bgNum,
                           zd *exNum, cudaStream_t s)
{
    g_launch_count++;
    int blocks = 1 + (xbar ? G : 0);
    measure_reduce_kernel<<<blocks, 256, 0, s>>>(W, alive, eloc, den, parts, nparts, acc, G, xbar, ex,
                                                  bgNum, exNum);
}

namespace {
// LogHop2isSD2isOperation order statistics (logHop2isSD2isOperation.cpp:146-157):
// stats[0] calls, [1] total order, [2] min, [3] max.
__global__ void __launch_bounds__(256) taylor_stats_kernel(int W, const int *mask, const int *order, long long *stats)
{
    __shared__ double red[32];
    double calls = 0, total = 0, mn = 1e30, mx = 0;
    for (int w = threadIdx.x; w < W; w += blockDim.x) {
        if (!mask[w]) continue;
        double o = order[w];
        calls += 1; total += o;
        mn = fmin(mn, o); mx = fmax(mx, o);
    }
    calls = block_sum(calls, red);
    total = block_sum(total, red);
    mx = block_max(mx, red);
    mn = -block_max(-mn, red);
    if (threadIdx.x == 0) {
        stats[0] += (long long)calls;
        stats[1] += (long long)total;
        if (calls > 0) {
            if ((long long)mn < stats[2]) stats[2] = (long long)mn;
            if ((long long)mx > stats[3]) stats[3] = (long long)mx;
        }
    }
}
}  // namespace

void launch_taylor_stats(int W, const int *mask, const int *order, long long *stats, cudaStream_t s)
{
    g_launch_count++;
    taylor_stats_kernel<<<1, 256, 0, s>>>(W, mask, order, stats);
}

// popConfiguration with the count array in caller-provided global scratch
// (W ints), used by the allocation-free entry point.  The kernel clears the
// scratch before use.
void launch_pop_comb_scratch(int W, const double *weight, const double *uniforms, int *number,
                             int *table, cudaStream_t s)
{
    g_launch_count++;
    pop_comb_kernel<<<1, 256, 0, s>>>(W, weight, uniforms, 0, nullptr, number, table, nullptr, 0);
}
