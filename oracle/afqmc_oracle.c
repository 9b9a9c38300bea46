/*
 * afqmc_oracle.c -- CPU restatement of the AFQMCLAB walker step (FP64).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle for the
 * CUDA engine in afqmclab_b200/.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py load it; the product path
 * never does.
 *
 * Every routine restates one function of the reference (hshi/AFQMCLAB) in
 * plain C99, serial and in the reference's own summation order, and cites the
 * file:line it follows (paths relative to the AFQMCLAB project root).  The
 * reference's LAPACK calls are restated from the published unblocked
 * algorithms (zgetf2/zgetrs, zgeqr2/zung2r), and its SPRNG stream is replaced
 * by the counter-based SplitMix64 generator that the CUDA engine also uses
 * (uniform k of stream `seed` = top 53 bits of mix(mix(seed) + (k+1)*golden)).
 *
 * Pinning: the known-answer tests of the reference (SDTest.cpp:158-173,
 * SD2sTest.cpp:183-200, SD2isTest.cpp:164-178,
 * logHop2isSD2isOperationTest.cpp:25-94, HubbardSOCMeasureFixedSDSDTest.cpp,
 * populationControlTest.cpp:29-45 for the slot-filling part) are run against
 * this file by tests/test_oracle_pins.py.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#ifdef OR_BLAS
#include <dlfcn.h>
#include <stdio.h>
#endif

/* ------------------------------------------------------------------ */
/* Walker-parallel loops.  Walkers are independent within each pass of  */
/* the step and of the measurement; or_parallel_for runs body(ctx, i)   */
/* for i = 0..n-1 on up to `threads` threads (one when threads <= 1).   */
/* Every result that depends on the order of walkers (random-stream     */
/* offsets, the estimator sums) is computed serially outside it, so    */
/* the thread count does not change any output.                         */
/* ------------------------------------------------------------------ */
typedef void (*or_body_fn)(void *ctx, int i);
typedef struct { or_body_fn fn; void *ctx; int n; int next; } or_pfor;
static void *or_pfor_worker(void *p)
{
    or_pfor *f = (or_pfor *)p;
    for (;;) {
        int i = __atomic_fetch_add(&f->next, 1, __ATOMIC_RELAXED);
        if (i >= f->n) break;
        f->fn(f->ctx, i);
    }
    return NULL;
}
static void or_parallel_for(int n, int threads, or_body_fn fn, void *ctx)
{
    if (threads > n) threads = n;
    if (threads <= 1) { for (int i = 0; i < n; ++i) fn(ctx, i); return; }
    or_pfor f = {fn, ctx, n, 0};
    pthread_t *tid = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)(threads - 1));
    int started = 0;
    for (int t = 0; t < threads - 1; ++t)
        if (pthread_create(&tid[t], NULL, or_pfor_worker, &f) == 0) started++;
        else break;
    or_pfor_worker(&f);
    for (int t = 0; t < started; ++t) pthread_join(tid[t], NULL);
    free(tid);
}
static pthread_mutex_t or_stats_mu = PTHREAD_MUTEX_INITIALIZER;

typedef double complex zc;

#define OR_PI 3.14159265358979324

/* ------------------------------------------------------------------ */
/* RNG: counter-based SplitMix64 (replaces SPRNG, random_hao.cpp:73-85) */
/* ------------------------------------------------------------------ */
static uint64_t or_mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

uint64_t or_rng_bits(uint64_t seed, uint64_t k)
{
    return or_mix64(or_mix64(seed) + (k + 1ULL) * 0x9E3779B97F4A7C15ULL);
}

double or_rng_uniform_at(uint64_t seed, uint64_t k)
{
    return (double)(or_rng_bits(seed, k) >> 11) * 0x1.0p-53;
}

typedef struct { uint64_t seed, counter; } or_rng;

static double or_uniform(or_rng *r) { return or_rng_uniform_at(r->seed, r->counter++); }

/* gaussianHao(): random_hao.cpp:78-85, two uniforms per call, no caching. */
static double or_gaussian(or_rng *r)
{
    double tmp = or_uniform(r);
    if (tmp == 0) tmp += 1e-300;
    double u2 = or_uniform(r);
    return sqrt(-2.0 * log(tmp)) * cos(2.0 * OR_PI * u2);
}

void or_rng_fill_uniform(uint64_t seed, uint64_t counter, int n, double *out)
{
    for (int i = 0; i < n; ++i) out[i] = or_rng_uniform_at(seed, counter + (uint64_t)i);
}

/* ------------------------------------------------------------------ */
/* Dense helpers (column-major, like TensorHao, tensor_core.h:83-91)    */
/* ------------------------------------------------------------------ */
#define IDX(i, j, ld) ((size_t)(i) + (size_t)(j) * (size_t)(ld))

static zc opv(char t, const zc *A, int lda, int i, int j)
{
    if (t == 'N') return A[IDX(i, j, lda)];
    if (t == 'T') return A[IDX(j, i, lda)];
    return conj(A[IDX(j, i, lda)]);
}

/* C = alpha op(A) op(B) + beta C; restates gmm_cpu (tensor_2d_bl_cpu.cpp:61-75). */
#ifdef OR_BLAS
/* The timed CPU baseline build (liboracle_blas.so): the GEMM- and GEMV-shaped
 * work goes through an optimised BLAS, as the reference's BL_NAME(gmm) /
 * BL_NAME(gemv) calls do (common/tensorHao/source/tensor_2d_bl_cpu.cpp:61-75).
 * The library and its symbol prefix come from AFQMC_ORACLE_BLAS and
 * AFQMC_ORACLE_BLAS_PREFIX; without them the plain loops below run. */
typedef void (*or_zgemm_t)(const char *, const char *, const int *, const int *, const int *, const zc *,
                           const zc *, const int *, const zc *, const int *, const zc *, zc *, const int *);
typedef void (*or_zgemv_t)(const char *, const int *, const int *, const zc *, const zc *, const int *,
                           const zc *, const int *, const zc *, zc *, const int *);
typedef void (*or_dgemv_t)(const char *, const int *, const int *, const double *, const double *,
                           const int *, const double *, const int *, const double *, double *, const int *);
static or_zgemm_t p_zgemm;
static or_zgemv_t p_zgemv;
static or_dgemv_t p_dgemv;
static pthread_once_t or_blas_once = PTHREAD_ONCE_INIT;
static void or_blas_load(void)
{
    const char *path = getenv("AFQMC_ORACLE_BLAS");
    const char *pre = getenv("AFQMC_ORACLE_BLAS_PREFIX");
    if (!path) return;
    void *h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!h) return;
    char name[128];
    snprintf(name, sizeof name, "%szgemm_", pre ? pre : "");
    p_zgemm = (or_zgemm_t)dlsym(h, name);
    snprintf(name, sizeof name, "%szgemv_", pre ? pre : "");
    p_zgemv = (or_zgemv_t)dlsym(h, name);
    snprintf(name, sizeof name, "%sdgemv_", pre ? pre : "");
    p_dgemv = (or_dgemv_t)dlsym(h, name);
    if (!p_zgemm || !p_zgemv || !p_dgemv) p_zgemm = NULL, p_zgemv = NULL, p_dgemv = NULL;
}
static int or_blas(void)
{
    pthread_once(&or_blas_once, or_blas_load);
    return p_zgemm != NULL;
}
int or_blas_available(void) { return or_blas(); }
#else
static int or_blas(void) { return 0; }
int or_blas_available(void) { return 0; }
#endif

void or_zgemm(char ta, char tb, int m, int n, int k, zc alpha, const zc *A, int lda,
              const zc *B, int ldb, zc beta, zc *C, int ldc)
{
#ifdef OR_BLAS
    if (or_blas()) { p_zgemm(&ta, &tb, &m, &n, &k, &alpha, A, &lda, B, &ldb, &beta, C, &ldc); return; }
#endif
    if (ta == 'C' && tb == 'N') {
        /* contiguous dot products: C(i,j) = sum_l conj(A(l,i)) B(l,j) */
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < m; ++i) {
                const zc *a = A + IDX(0, i, lda), *b = B + IDX(0, j, ldb);
                zc s = 0;
                for (int l = 0; l < k; ++l) s += conj(a[l]) * b[l];
                C[IDX(i, j, ldc)] = (beta == 0 ? 0 : beta * C[IDX(i, j, ldc)]) + alpha * s;
            }
        return;
    }
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < m; ++i) {
            zc s = 0;
            for (int l = 0; l < k; ++l) s += opv(ta, A, lda, i, l) * opv(tb, B, ldb, l, j);
            C[IDX(i, j, ldc)] = (beta == 0 ? 0 : beta * C[IDX(i, j, ldc)]) + alpha * s;
        }
    }
}

/* Fast path for C = A(m x k, 'N') * B(k x n, 'N'), column-major, beta = 0. */
static void or_zgemm_nn(int m, int n, int k, zc alpha, const zc *A, int lda, const zc *B, int ldb,
                        zc *C, int ldc)
{
#ifdef OR_BLAS
    if (or_blas()) {
        const zc zero = 0;
        p_zgemm("N", "N", &m, &n, &k, &alpha, A, &lda, B, &ldb, &zero, C, &ldc);
        return;
    }
#endif
    for (int j = 0; j < n; ++j) {
        zc *c = C + IDX(0, j, ldc);
        for (int i = 0; i < m; ++i) c[i] = 0;
        for (int l = 0; l < k; ++l) {
            zc b = alpha * B[IDX(l, j, ldb)];
            const zc *a = A + IDX(0, l, lda);
            for (int i = 0; i < m; ++i) c[i] += a[i] * b;
        }
    }
}

static double cabs1(zc z) { return fabs(creal(z)) + fabs(cimag(z)); }

/* LU with partial pivoting, unblocked zgetf2 (what LUconstruct_cpu calls,
 * tensor_2d_bl_cpu.cpp:145-167).  ipiv is 1-based like LAPACK. Returns info. */
int or_zgetrf(int n, zc *A, int lda, int *ipiv)
{
    int info = 0;
    for (int j = 0; j < n; ++j) {
        int p = j; double best = cabs1(A[IDX(j, j, lda)]);
        for (int i = j + 1; i < n; ++i) {
            double v = cabs1(A[IDX(i, j, lda)]);
            if (v > best) { best = v; p = i; }
        }
        ipiv[j] = p + 1;
        if (A[IDX(p, j, lda)] != 0) {
            if (p != j)
                for (int c = 0; c < n; ++c) {
                    zc t = A[IDX(j, c, lda)]; A[IDX(j, c, lda)] = A[IDX(p, c, lda)]; A[IDX(p, c, lda)] = t;
                }
            zc inv = 1.0 / A[IDX(j, j, lda)];
            for (int i = j + 1; i < n; ++i) A[IDX(i, j, lda)] *= inv;
        } else if (info == 0) {
            info = j + 1;
        }
        for (int c = j + 1; c < n; ++c) {
            zc u = A[IDX(j, c, lda)];
            if (u == 0) continue;
            for (int i = j + 1; i < n; ++i) A[IDX(i, c, lda)] -= A[IDX(i, j, lda)] * u;
        }
    }
    return info;
}

/* zgetrs with TRANS='T': solve A^T X = B given A = P L U.
 * Restates solve_lineq_cpu(..., 'T') (tensor_2d_bl_cpu.cpp:218-258). */
void or_zgetrs_T(int n, int nrhs, const zc *LU, int lda, const int *ipiv, zc *B, int ldb)
{
    for (int r = 0; r < nrhs; ++r) {
        zc *b = B + IDX(0, r, ldb);
        /* U^T y = b (U^T lower triangular, non-unit) */
        for (int i = 0; i < n; ++i) {
            zc s = b[i];
            for (int k = 0; k < i; ++k) s -= LU[IDX(k, i, lda)] * b[k];
            b[i] = s / LU[IDX(i, i, lda)];
        }
        /* L^T z = y (unit upper) */
        for (int i = n - 1; i >= 0; --i) {
            zc s = b[i];
            for (int k = i + 1; k < n; ++k) s -= LU[IDX(k, i, lda)] * b[k];
            b[i] = s;
        }
        /* x = P z: undo interchanges in reverse order */
        for (int i = n - 1; i >= 0; --i) {
            int p = ipiv[i] - 1;
            if (p != i) { zc t = b[i]; b[i] = b[p]; b[p] = t; }
        }
    }
}

/* logDeterminant / lognormPhaseDeterminant, tensor_2d_common_fun.cpp:75-105 */
zc or_logdet(int n, const zc *LU, int lda, const int *ipiv, int info)
{
    if (info > 0) return -1e300;
    double lognorm = 0; zc phase = 1;
    for (int i = 0; i < n; ++i) {
        zc d = LU[IDX(i, i, lda)];
        double a = cabs(d);
        lognorm += log(a);
        if (ipiv[i] != i + 1) phase *= (-d / a); else phase *= (d / a);
    }
    return lognorm + clog(phase);
}

/* Householder QR of ph (L x N), ph <- Q; returns det(R) made positive, like
 * QRMatrix_cpu (tensor_2d_bl_cpu.cpp:263-315): zgeqrf (zgeqr2) then zungqr
 * (zung2r); R diagonal is real (zlarfg); if prod R_ii < 0, column 0 of Q and
 * detList(0) are negated.  detList may be NULL. */
double or_qr(int L, int N, zc *ph, double *detList)
{
    zc *tau = (zc *)calloc((size_t)N, sizeof(zc));
    double *rdiag = (double *)calloc((size_t)N, sizeof(double));
    for (int j = 0; j < N; ++j) {
        zc alpha = ph[IDX(j, j, L)];
        double xnorm2 = 0;
        for (int i = j + 1; i < L; ++i) { double a = cabs(ph[IDX(i, j, L)]); xnorm2 += a * a; }
        double xnorm = sqrt(xnorm2);
        zc t; double beta;
        if (xnorm == 0 && cimag(alpha) == 0) {
            t = 0; beta = creal(alpha);
        } else {
            double nrm = sqrt(creal(alpha) * creal(alpha) + cimag(alpha) * cimag(alpha) + xnorm * xnorm);
            beta = creal(alpha) >= 0 ? -nrm : nrm;
            t = (beta - alpha) / beta;
            zc scal = 1.0 / (alpha - beta);
            for (int i = j + 1; i < L; ++i) ph[IDX(i, j, L)] *= scal;
        }
        tau[j] = t; rdiag[j] = beta;
        ph[IDX(j, j, L)] = 1.0;
        /* apply H^H = I - conj(tau) v v^H to columns j+1..N-1 */
        for (int c = j + 1; c < N; ++c) {
            zc w = 0;
            for (int i = j; i < L; ++i) w += conj(ph[IDX(i, j, L)]) * ph[IDX(i, c, L)];
            w *= conj(t);
            for (int i = j; i < L; ++i) ph[IDX(i, c, L)] -= ph[IDX(i, j, L)] * w;
        }
        ph[IDX(j, j, L)] = beta;
    }
    double det_re; zc det = 1.0;
    for (int i = 0; i < N; ++i) { det *= rdiag[i]; if (detList) detList[i] = rdiag[i]; }
    /* zung2r: Q = H_0 H_1 ... H_{N-1} applied to the first N columns of I */
    zc *v = (zc *)calloc((size_t)L * N, sizeof(zc));
    for (int j = 0; j < N; ++j) {
        v[IDX(j, j, L)] = 1.0;
        for (int i = j + 1; i < L; ++i) v[IDX(i, j, L)] = ph[IDX(i, j, L)];
    }
    for (int i = 0; i < L * N; ++i) ph[i] = 0;
    for (int j = 0; j < N; ++j) ph[IDX(j, j, L)] = 1.0;
    for (int j = N - 1; j >= 0; --j) {
        for (int c = j; c < N; ++c) {
            zc w = 0;
            for (int i = j; i < L; ++i) w += conj(v[IDX(i, j, L)]) * ph[IDX(i, c, L)];
            w *= tau[j];
            for (int i = j; i < L; ++i) ph[IDX(i, c, L)] -= v[IDX(i, j, L)] * w;
        }
    }
    free(v);
    det_re = creal(det);
    if (det_re < 0) {
        det_re = -det_re;
        if (detList) detList[0] = -detList[0];
        for (int i = 0; i < L; ++i) ph[IDX(i, 0, L)] = -ph[IDX(i, 0, L)];
    }
    free(tau); free(rdiag);
    return det_re;
}

/* SD::stabilize (SD.cpp:42-56): logw += log(QR det). */
void or_sd_stabilize(int L, int N, zc *wf, zc *logw)
{
    *logw += clog(or_qr(L, N, wf, NULL));
}

/* SD::normalize(ratio) (SD.cpp:57-75) for the known-answer test. */
zc or_sd_normalize_ratio(int L, int N, zc *wf, double *ratio)
{
    double *d = (double *)malloc(sizeof(double) * N);
    zc lw = clog(or_qr(L, N, wf, d));
    double mn = 1e300, mx = 0;
    for (int i = 0; i < N; ++i) { double a = fabs(d[i]); if (a < mn) mn = a; if (a > mx) mx = a; }
    *ratio = mn / mx;
    free(d);
    return lw;
}

/* SD2is::stabilize (SD2is.cpp:48-76). */
void or_sd2is_stabilize(int L, int Nup, int Ndn, zc *wf, zc *logw)
{
    int Nmax = Nup > Ndn ? Nup : Ndn, Nmin = Nup < Ndn ? Nup : Ndn;
    if (Nup == Ndn) { *logw += 2.0 * clog(or_qr(L, Nmax, wf, NULL)); return; }
    double *d = (double *)malloc(sizeof(double) * Nmax);
    *logw += clog(or_qr(L, Nmax, wf, d));
    zc norm = 1.0;
    for (int i = 0; i < Nmin; ++i) norm *= d[i];
    *logw += clog(norm);
    free(d);
}

/* SD2is::normalize(ratio) for the known-answer test. */
zc or_sd2is_normalize_ratio(int L, int Nup, int Ndn, zc *wf, double *ratio)
{
    int Nmax = Nup > Ndn ? Nup : Ndn, Nmin = Nup < Ndn ? Nup : Ndn;
    double *d = (double *)malloc(sizeof(double) * Nmax);
    zc lw = clog(or_qr(L, Nmax, wf, d));
    zc norm = 1.0;
    for (int i = 0; i < Nmin; ++i) norm *= d[i];
    lw += clog(norm);
    double mn = 1e300, mx = 0;
    for (int i = 0; i < Nmax; ++i) { double a = fabs(d[i]); if (a < mn) mn = a; if (a > mx) mx = a; }
    *ratio = mn / mx;
    free(d);
    return lw;
}

/* SD2s::normalize(ratio) (SD2s.cpp:58-90): ratio = min(ratioUp, ratioDn). */
static double or_ratio(const double *d, int n)
{
    double mn = 1e300, mx = 0;
    for (int i = 0; i < n; ++i) { double a = fabs(d[i]); if (a < mn) mn = a; if (a > mx) mx = a; }
    return mn / mx;
}

zc or_sd2s_normalize_ratio(int L, int Nup, int Ndn, zc *wfUp, zc *wfDn, double *ratio)
{
    double *du = (double *)malloc(sizeof(double) * (Nup + Ndn));
    double *dd = du + Nup;
    zc lw = clog(or_qr(L, Nup, wfUp, du));
    lw += clog(or_qr(L, Ndn, wfDn, dd));
    double ru = or_ratio(du, Nup), rd = or_ratio(dd, Ndn);
    *ratio = ru < rd ? ru : rd;
    free(du);
    return lw;
}

/* ------------------------------------------------------------------ */
/* Walker x walker (SDSDOperation.cpp:52-186, SD2sSD2isOperation.cpp)   */
/* ------------------------------------------------------------------ */

/* SDSDOperation: logOverlap (:65-72), theta_T (:166-173), diag (:91-111),
 * off-diagonal (:113-141).  thetaT is N x n; outputs may be NULL.
 * Returns the LU info. */
int or_sdsd(int n, int N, const zc *phiT, zc logwT, const zc *phi, zc logw, zc *logOverlap,
            zc *thetaT, zc *greenDiag, zc *greenOffDiag)
{
    zc *S = (zc *)malloc(sizeof(zc) * N * N);
    int *ipiv = (int *)malloc(sizeof(int) * N);
    or_zgemm('C', 'N', N, N, n, 1.0, phiT, n, phi, n, 0.0, S, N);
    int info = or_zgetrf(N, S, N, ipiv);
    if (logOverlap) *logOverlap = conj(logwT) + logw + or_logdet(N, S, N, ipiv, info);
    if (thetaT || greenDiag || greenOffDiag) {
        zc *tt = thetaT ? thetaT : (zc *)malloc(sizeof(zc) * N * n);
        for (int a = 0; a < N; ++a)
            for (int i = 0; i < n; ++i) tt[IDX(a, i, N)] = phi[IDX(i, a, n)];
        or_zgetrs_T(N, n, S, N, ipiv, tt, N);
        if (greenDiag) {
            for (int i = 0; i < n; ++i) greenDiag[i] = 0;
            for (int j = 0; j < N; ++j)
                for (int i = 0; i < n; ++i) greenDiag[i] += conj(phiT[IDX(i, j, n)]) * tt[IDX(j, i, N)];
        }
        if (greenOffDiag) {
            int h = n / 2;
            for (int i = 0; i < n; ++i) greenOffDiag[i] = 0;
            for (int j = 0; j < N; ++j)
                for (int i = 0; i < h; ++i) {
                    greenOffDiag[i] += conj(phiT[IDX(i, j, n)]) * tt[IDX(j, i + h, N)];
                    greenOffDiag[i + h] += conj(phiT[IDX(i + h, j, n)]) * tt[IDX(j, i, N)];
                }
        }
        if (!thetaT) free(tt);
    }
    free(S); free(ipiv);
    return info;
}

/* SD2sSD2isOperation (SD2sSD2isOperation.cpp:28-230).  Right Up/Dn are the
 * first Nup/Ndn columns of the same wf (:40-43).  thetaUpT: Nup x n,
 * thetaDnT: Ndn x n (either may be NULL). */
int or_sd2s_sd2is(int n, int Nup, int Ndn, const zc *phiTUp, const zc *phiTDn, zc logwT,
                  const zc *phi, zc logw, zc *logOverlap, zc *thetaUpT, zc *thetaDnT)
{
    int Ns[2] = {Nup, Ndn};
    const zc *pT[2] = {phiTUp, phiTDn};
    zc *th[2] = {thetaUpT, thetaDnT};
    zc ld = 0; int infoAll = 0;
    for (int s = 0; s < 2; ++s) {
        int N = Ns[s];
        zc *S = (zc *)malloc(sizeof(zc) * N * N);
        int *ipiv = (int *)malloc(sizeof(int) * (N > 0 ? N : 1));
        or_zgemm('C', 'N', N, N, n, 1.0, pT[s], n, phi, n, 0.0, S, N);
        int info = or_zgetrf(N, S, N, ipiv);
        if (info) infoAll = info;
        ld += or_logdet(N, S, N, ipiv, info);
        if (th[s]) {
            for (int a = 0; a < N; ++a)
                for (int i = 0; i < n; ++i) th[s][IDX(a, i, N)] = phi[IDX(i, a, n)];
            or_zgetrs_T(N, n, S, N, ipiv, th[s], N);
        }
        free(S); free(ipiv);
    }
    if (logOverlap) *logOverlap = conj(logwT) + logw + ld;
    return infoAll;
}

/* ------------------------------------------------------------------ */
/* mathHao helpers (simple_fun.cpp:7-91)                               */
/* ------------------------------------------------------------------ */
zc or_solve_cosh_eq_exp(double y)
{
    zc ey = exp(y);
    zc g = clog(ey - csqrt(ey * ey - 1.0));
    if (fabs(creal(g)) < fabs(cimag(g))) g = I * cimag(g); else g = creal(g);
    return g;
}

zc or_solve_cos_eq_exp(double y)
{
    zc ey = exp(y);
    zc g = cacos(ey);
    if (fabs(creal(g)) < fabs(cimag(g))) g = I * cimag(g); else g = creal(g);
    return g;
}

void or_exp2by2(double *a, double *b, zc *c)
{
    if (cabs(*c) < 1e-60) { *a = exp(*a); *b = exp(*b); *c = 0; return; }
    double abs_c = cabs(*c), arg_c = carg(*c);
    double d0, d1; zc v00, v01, v10, v11;
    if (fabs(*a - *b) < 1e-60) {
        double norm = 1.0 / sqrt(2.0);
        d0 = exp(-abs_c + *a); d1 = exp(abs_c + *b);
        v00 = -norm; v10 = norm * cexp(I * arg_c); v01 = norm; v11 = norm * cexp(I * arg_c);
    } else {
        double xi = 0.5 * atan(2.0 * abs_c / (*a - *b));
        d0 = exp(0.5 * cos(2.0 * xi) * (*a - *b) + sin(2.0 * xi) * abs_c + (*a + *b) * 0.5);
        d1 = exp(-0.5 * cos(2.0 * xi) * (*a - *b) - sin(2.0 * xi) * abs_c + (*a + *b) * 0.5);
        v00 = cexp(-I * arg_c * 0.5) * cos(xi);
        v10 = cexp(I * arg_c * 0.5) * sin(xi);
        v01 = -cexp(-I * arg_c * 0.5) * sin(xi);
        v11 = cexp(I * arg_c * 0.5) * cos(xi);
    }
    double na = creal(d0 * v00 * conj(v00) + d1 * v01 * conj(v01));
    double nb = creal(d0 * v10 * conj(v10) + d1 * v11 * conj(v11));
    *c = d0 * v10 * conj(v00) + d1 * v11 * conj(v01);
    *a = na; *b = nb;
}

/* ------------------------------------------------------------------ */
/* NiupNidn (NiupNidn.cpp:12-322)                                      */
/* decomp: 0 densityCharge, 1 densitySpin, 2 hopCharge, 3 hopSpin       */
/* ------------------------------------------------------------------ */
void or_niupnidn_consts(int L, double dt, int decomp, const double *U, const double *mu,
                        const double *hx, const double *hy, const double *hz, zc *gamma, zc *cd00,
                        zc *cd01, zc *cd10, zc *cd11, double *dtUSum)
{
    double s = 0;
    for (int i = 0; i < L; ++i) s += U[i];
    *dtUSum = dt * s;
    for (int i = 0; i < L; ++i) {
        double dtU = dt * U[i];
        if (decomp == 0) gamma[i] = or_solve_cosh_eq_exp(-dtU * 0.5);
        else if (decomp == 3) gamma[i] = or_solve_cos_eq_exp(dtU * 0.5);
        else gamma[i] = or_solve_cosh_eq_exp(dtU * 0.5);
        double a = -dt * (U[i] * 0.5 - mu[i] + hz[i] * 0.5);
        double b = -dt * (U[i] * 0.5 - mu[i] - hz[i] * 0.5);
        zc c = -dt * 0.5 * (hx[i] + I * hy[i]);
        or_exp2by2(&a, &b, &c);
        cd00[i] = a; cd01[i] = conj(c); cd10[i] = c; cd11[i] = b;
    }
}

/* ------------------------------------------------------------------ */
/* LogHop2isSD2isOperation Taylor series (logHop2isSD2isOperation.cpp)  */
/* flag 0 = fixedOrder, 1 = dynamicOrder.  trans 'N' (applyToRight) or  */
/* 'C' (applyToLeft).  Returns the order reached.                       */
/* ------------------------------------------------------------------ */
int or_loghop_apply(int flag, int taylorOrder, double accuracy, int baseOrder, char trans, int n,
                    int ncol, const zc *M, const zc *wf, zc *wfNew)
{
    zc *old = (zc *)malloc(sizeof(zc) * n * ncol);
    zc *nw = (zc *)malloc(sizeof(zc) * n * ncol);
    memcpy(wfNew, wf, sizeof(zc) * n * ncol);
    memcpy(old, wf, sizeof(zc) * n * ncol);
    int order = 0;
    int fixedMax = (flag == 0 && taylorOrder > 0) ? taylorOrder : baseOrder;
    while (order < fixedMax) {
        if (trans == 'N') or_zgemm_nn(n, ncol, n, 1.0 / (order + 1.0), M, n, old, n, nw, n);
        else or_zgemm(trans, 'N', n, ncol, n, 1.0 / (order + 1.0), M, n, old, n, 0.0, nw, n);
        for (int i = 0; i < n * ncol; ++i) wfNew[i] += nw[i];
        zc *t = old; old = nw; nw = t;
        order++;
    }
    if (!(flag == 0 && taylorOrder > 0)) {
        int conv;
        do {
            if (trans == 'N') or_zgemm_nn(n, ncol, n, 1.0 / (order + 1.0), M, n, old, n, nw, n);
            else or_zgemm(trans, 'N', n, ncol, n, 1.0 / (order + 1.0), M, n, old, n, 0.0, nw, n);
            for (int i = 0; i < n * ncol; ++i) wfNew[i] += nw[i];
            zc *t = old; old = nw; nw = t;
            order++;
            conv = 1;
            for (int i = 0; i < n * ncol; ++i)
                if (cabs(old[i]) > accuracy) { conv = 0; break; }
        } while (!conv);
    }
    free(old); free(nw);
    return order;
}

/* ------------------------------------------------------------------ */
/* Population control (populationControlConfiguration.cpp:9-101)       */
/* uniforms: the L draws popConfiguration takes, in order.              */
/* The `number[zero_i]` read is bounds-checked before dereference.      */
/* ------------------------------------------------------------------ */
void or_pop_check(int L, const double *w, double *minW, double *maxW, double *avgW)
{
    double sum = 0; for (int i = 0; i < L; ++i) sum += w[i];
    double mx = 0, mn = 1e20;
    for (int i = 0; i < L; ++i) { if (mx < w[i]) mx = w[i]; if (mn > w[i]) mn = w[i]; }
    *minW = mn; *maxW = mx; *avgW = sum / (L * 1.0);
}

static void or_fill_slots(int L, int size, int *number, int *table)
{
    int L_chunk = L / size;
    for (int c = 0; c < size; ++c) {
        int zero_i = L_chunk * c, one_i = L_chunk * c, max_i = L_chunk * (c + 1);
        while (zero_i < max_i && number[zero_i] != 0) zero_i++;
        while (one_i < max_i && number[one_i] <= 1) one_i++;
        while (zero_i < max_i && one_i < max_i) {
            table[zero_i] = one_i; number[zero_i]++; number[one_i]--;
            while (zero_i < max_i && number[zero_i] != 0) zero_i++;
            while (one_i < max_i && number[one_i] <= 1) one_i++;
        }
    }
    if (size > 1) {
        int zero_i = 0, one_i = 0, max_i = L;
        while (zero_i < max_i && number[zero_i] != 0) zero_i++;
        while (one_i < max_i && number[one_i] <= 1) one_i++;
        while (zero_i < max_i && one_i < max_i) {
            table[zero_i] = one_i; number[zero_i]++; number[one_i]--;
            while (zero_i < max_i && number[zero_i] != 0) zero_i++;
            while (one_i < max_i && number[one_i] <= 1) one_i++;
        }
    }
}

/* Returns 0 on success, 1 if some slot does not end with exactly one walker. */
int or_pop_configuration(int L, int size, const double *weight, const double *uniforms, int *table)
{
    double sum = 0; for (int i = 0; i < L; ++i) sum += weight[i];
    double *prob = (double *)malloc(sizeof(double) * L);
    for (int i = 0; i < L; ++i) prob[i] = weight[i] / sum;
    int *number = (int *)calloc((size_t)L, sizeof(int));
    int index_old = 0; double prob_sum_old = prob[0];
    for (int i = 0; i < L; ++i) {
        double prob_sum_new = (i + uniforms[i]) / (L * 1.0);
        while (prob_sum_new > prob_sum_old && index_old < L - 1) {
            index_old++;
            prob_sum_old += prob[index_old];
        }
        number[index_old]++;
    }
    for (int i = 0; i < L; ++i) if (number[i] != 0) table[i] = i;
    or_fill_slots(L, size, number, table);
    int bad = 0;
    for (int i = 0; i < L; ++i) if (number[i] != 1) bad = 1;
    free(prob); free(number);
    return bad;
}

/* The slot-filling half of popConfiguration from given copy counts. */
int or_pop_fill_from_counts(int L, int size, const int *counts, int *table)
{
    int *number = (int *)malloc(sizeof(int) * L);
    memcpy(number, counts, sizeof(int) * L);
    for (int i = 0; i < L; ++i) table[i] = (number[i] != 0) ? i : -1;
    or_fill_slots(L, size, number, table);
    int bad = 0;
    for (int i = 0; i < L; ++i) if (number[i] != 1) bad = 1;
    free(number);
    return bad;
}

/* ================================================================== */
/* Population engines: the two driver steps over a whole population.   */
/* ================================================================== */

enum { OR_CP = 0, OR_PL = 1 };

typedef struct {
    int kind;              /* OR_CP or OR_PL */
    int n, N, Nup, Ndn, W; /* n rows; N columns of a walker */
    int L;                 /* CP: sites; PL: unused */
    int G;                 /* PL: Cholesky vectors */
    int decomp, forceType;
    double dt, ET, forceCap;
    int mgsStep, popStep, mgsIndex, popIndex;
    or_rng rng;
    /* walkers */
    zc *wf, *logw; int *alive;
    /* trial */
    zc *phiT, *phiTDn; zc logwT;
    /* one-body: dense exp (Hop/Hop2is) or Taylor (LogHop2is) */
    zc *expMinusDtK, *expHalfDtK, *expMinusHalfDtK; zc logwExpMinusDtK, logwExpHalfDtK, logwExpMinusHalfDtK;
    zc *logExpMinusDtK; zc logwLogExpMinusDtK; int useLogOneBody;
    /* CP two-body */
    zc *gamma, *cd00, *cd01, *cd10, *cd11; double dtUSum; double *constForceCP;
    double *U, *mu, *hx, *hy, *hz; zc *wfDaggerK;
    /* PL two-body */
    double *chol;      /* n x n x G real */
    double *bg;        /* G */
    zc *A;             /* (Nup+Ndn) x n x G: [Aup (Nup,n,G); Adn (Ndn,n,G)] stored per spin */
    zc *Aup, *Adn;
    zc *wfDaggerTUp, *wfDaggerTDn;
    zc sqrtMinusDt;
    zc *constForcePL;
    /* measurement accumulators */
    zc den, HNum, KNum, VNum, RNum, TNum;
    zc *bgNum, *exNum;
    zc *siteNum;       /* CP: NupNum, NdnNum, SplusNum, SminusNum (4 x L) */
    int observe;       /* CP observe estimator on */
    zc *obsNum;        /* greenMatrixNum, densityDensityNum (n x n), S+S-, S-S+, pair (L x L) */
    /* taylor statistics */
    long taylorCalls, taylorTotal; int taylorMin, taylorMax;
    int nthreads;
} or_engine;

static size_t or_wsize(const or_engine *e) { return (size_t)e->n * e->N; }

void or_destroy(or_engine *e)
{
    if (!e) return;
    void *ptrs[] = {e->wf, e->logw, e->alive, e->phiT, e->phiTDn, e->expMinusDtK, e->expHalfDtK,
                    e->expMinusHalfDtK, e->logExpMinusDtK, e->gamma, e->cd00, e->cd01, e->cd10,
                    e->cd11, e->constForceCP, e->U, e->mu, e->hx, e->hy, e->hz, e->wfDaggerK,
                    e->chol, e->bg, e->Aup, e->Adn, e->wfDaggerTUp, e->wfDaggerTDn,
                    e->constForcePL, e->bgNum, e->exNum, e->siteNum, e->obsNum};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); ++i) free(ptrs[i]);
    free(e);
}

static zc *zdup(const double *src, size_t count)
{
    if (!src) return NULL;
    zc *p = (zc *)malloc(sizeof(zc) * count);
    memcpy(p, src, sizeof(zc) * count);
    return p;
}
static double *ddup(const double *src, size_t count)
{
    if (!src) return NULL;
    double *p = (double *)malloc(sizeof(double) * count);
    memcpy(p, src, sizeof(double) * count);
    return p;
}

/* CP engine: tutorials/afqmcConstraintPath (afqmcConstraintPath.cpp:20-34).
 * K is 2L x 2L complex (HubbardSOC::K), exp matrices are the Hop operators
 * built by HubbardSOC::returnExpMinusAlphaK (HubbardSOC.cpp:109-118). */
or_engine *or_cp_create(int L, int N, int W, int decomp, int forceType, double dt, double ET,
                        double forceCap, int mgsStep, int popStep, const double *K,
                        const double *expMinusDtK, const double *expHalfDtK,
                        const double *expMinusHalfDtK, const double *U, const double *mu,
                        const double *hx, const double *hy, const double *hz,
                        const double *constForce, const double *phiT, double logwT_re,
                        double logwT_im, uint64_t seed)
{
    or_engine *e = (or_engine *)calloc(1, sizeof(or_engine));
    e->kind = OR_CP; e->L = L; e->n = 2 * L; e->N = N; e->Nup = N; e->Ndn = 0; e->W = W;
    e->decomp = decomp; e->forceType = forceType; e->dt = dt; e->ET = ET; e->forceCap = forceCap;
    e->mgsStep = mgsStep; e->popStep = popStep;
    e->rng.seed = seed; e->rng.counter = 0;
    int n = e->n;
    e->wf = (zc *)calloc((size_t)W * n * N, sizeof(zc));
    e->logw = (zc *)calloc((size_t)W, sizeof(zc));
    e->alive = (int *)calloc((size_t)W, sizeof(int));
    e->phiT = zdup(phiT, (size_t)n * N);
    e->logwT = logwT_re + I * logwT_im;
    e->expMinusDtK = zdup(expMinusDtK, (size_t)n * n);
    e->expHalfDtK = zdup(expHalfDtK, (size_t)n * n);
    e->expMinusHalfDtK = zdup(expMinusHalfDtK, (size_t)n * n);
    e->U = ddup(U, L); e->mu = ddup(mu, L); e->hx = ddup(hx, L); e->hy = ddup(hy, L); e->hz = ddup(hz, L);
    e->constForceCP = (double *)calloc((size_t)L, sizeof(double));
    e->siteNum = (zc *)calloc((size_t)4 * L, sizeof(zc));
    if (constForce) memcpy(e->constForceCP, constForce, sizeof(double) * L);
    e->gamma = (zc *)malloc(sizeof(zc) * L);
    e->cd00 = (zc *)malloc(sizeof(zc) * L); e->cd01 = (zc *)malloc(sizeof(zc) * L);
    e->cd10 = (zc *)malloc(sizeof(zc) * L); e->cd11 = (zc *)malloc(sizeof(zc) * L);
    or_niupnidn_consts(L, dt, decomp, U, mu, hx, hy, hz, e->gamma, e->cd00, e->cd01, e->cd10, e->cd11,
                       &e->dtUSum);
    /* HubbardSOCMeasureFixedSDSD::initWfDaggerK (:160-167): N x 2L */
    e->wfDaggerK = (zc *)malloc(sizeof(zc) * N * n);
    or_zgemm('C', 'N', N, n, n, 1.0, e->phiT, n, (const zc *)K, n, 0.0, e->wfDaggerK, N);
    return e;
}

/* Phaseless engine: tutorials/afqmcPhaseless (afqmcPhaseless.cpp:32-68).
 * chol is n x n x G (RealMaterialMolecule::choleskyVecs), t the one-body
 * matrix used by the T energy (initWfDaggerT), bg the Cholesky background.
 * One-body: either the dense Hop2is matrices (expMinusDtK etc, complex)
 * or the LogHop2is matrix logExpMinusDtK = -dt*Kp used through the Taylor
 * series (useLogOneBody = 1). */
or_engine *or_pl_create(int n, int Nup, int Ndn, int G, int W, int forceType, double dt, double ET,
                        double forceCap, int mgsStep, int popStep, const double *chol,
                        const double *bg, const double *t, const double *expMinusDtK,
                        double logwExpMinusDtK, const double *expHalfDtK, double logwExpHalfDtK,
                        const double *expMinusHalfDtK, double logwExpMinusHalfDtK,
                        const double *logExpMinusDtK, double logwLogExpMinusDtK,
                        const double *constForce, const double *phiTUp, const double *phiTDn,
                        double logwT_re, double logwT_im, uint64_t seed)
{
    or_engine *e = (or_engine *)calloc(1, sizeof(or_engine));
    e->kind = OR_PL; e->n = n; e->Nup = Nup; e->Ndn = Ndn; e->N = Nup > Ndn ? Nup : Ndn; e->W = W;
    e->G = G; e->forceType = forceType; e->dt = dt; e->ET = ET; e->forceCap = forceCap;
    e->mgsStep = mgsStep; e->popStep = popStep;
    e->rng.seed = seed; e->rng.counter = 0;
    int N = e->N;
    e->wf = (zc *)calloc((size_t)W * n * N, sizeof(zc));
    e->logw = (zc *)calloc((size_t)W, sizeof(zc));
    e->alive = (int *)calloc((size_t)W, sizeof(int));
    e->phiT = zdup(phiTUp, (size_t)n * Nup);
    e->phiTDn = zdup(phiTDn, (size_t)n * Ndn);
    e->logwT = logwT_re + I * logwT_im;
    e->expMinusDtK = zdup(expMinusDtK, (size_t)n * n); e->logwExpMinusDtK = logwExpMinusDtK;
    e->expHalfDtK = zdup(expHalfDtK, (size_t)n * n); e->logwExpHalfDtK = logwExpHalfDtK;
    e->expMinusHalfDtK = zdup(expMinusHalfDtK, (size_t)n * n); e->logwExpMinusHalfDtK = logwExpMinusHalfDtK;
    e->logExpMinusDtK = zdup(logExpMinusDtK, (size_t)n * n); e->logwLogExpMinusDtK = logwLogExpMinusDtK;
    e->useLogOneBody = (expMinusDtK == NULL);
    e->chol = ddup(chol, (size_t)n * n * G);
    e->bg = ddup(bg, G);
    /* sqrt(-dt * complex(1, 0)) as choleskyReal.cpp:17 evaluates it: the
     * product's imaginary part is -0.0, so the principal root is -i sqrt(dt) */
    e->sqrtMinusDt = -sqrt(dt) * I;
    e->constForcePL = (zc *)calloc((size_t)G, sizeof(zc));
    if (constForce) memcpy(e->constForcePL, constForce, sizeof(zc) * G);
    /* initWfDaggerT (:148-163) and initWfDaggerCholeskyVecs (:165-186) */
    zc *tc = (zc *)malloc(sizeof(zc) * n * n);
    for (int i = 0; i < n * n; ++i) tc[i] = t[i];
    e->wfDaggerTUp = (zc *)malloc(sizeof(zc) * Nup * n);
    e->wfDaggerTDn = (zc *)malloc(sizeof(zc) * (Ndn > 0 ? Ndn : 1) * n);
    or_zgemm('C', 'N', Nup, n, n, 1.0, e->phiT, n, tc, n, 0.0, e->wfDaggerTUp, Nup);
    or_zgemm('C', 'N', Ndn, n, n, 1.0, e->phiTDn, n, tc, n, 0.0, e->wfDaggerTDn, Ndn);
    e->Aup = (zc *)malloc(sizeof(zc) * (size_t)Nup * n * G);
    e->Adn = (zc *)malloc(sizeof(zc) * (size_t)(Ndn > 0 ? Ndn : 1) * n * G);
    for (int g = 0; g < G; ++g) {
        for (int i = 0; i < n * n; ++i) tc[i] = chol[(size_t)g * n * n + i];
        or_zgemm('C', 'N', Nup, n, n, 1.0, e->phiT, n, tc, n, 0.0, e->Aup + (size_t)g * Nup * n, Nup);
        or_zgemm('C', 'N', Ndn, n, n, 1.0, e->phiTDn, n, tc, n, 0.0, e->Adn + (size_t)g * Ndn * n, Ndn);
    }
    free(tc);
    e->bgNum = (zc *)calloc((size_t)G, sizeof(zc));
    e->exNum = (zc *)calloc((size_t)G, sizeof(zc));
    e->taylorMin = 1 << 30;
    return e;
}

void or_set_walkers(or_engine *e, const double *wf, const double *logw, const int *alive)
{
    memcpy(e->wf, wf, sizeof(zc) * or_wsize(e) * e->W);
    memcpy(e->logw, logw, sizeof(zc) * e->W);
    memcpy(e->alive, alive, sizeof(int) * e->W);
}
void or_get_walkers(const or_engine *e, double *wf, double *logw, int *alive)
{
    if (wf) memcpy(wf, e->wf, sizeof(zc) * or_wsize(e) * e->W);
    if (logw) memcpy(logw, e->logw, sizeof(zc) * e->W);
    if (alive) memcpy(alive, e->alive, sizeof(int) * e->W);
}
void or_set_rng(or_engine *e, uint64_t seed, uint64_t counter) { e->rng.seed = seed; e->rng.counter = counter; }
uint64_t or_get_rng_counter(const or_engine *e) { return e->rng.counter; }
void or_set_ET(or_engine *e, double ET) { e->ET = ET; }
void or_set_threads(or_engine *e, int nthreads) { e->nthreads = nthreads; }

static zc or_walker_logoverlap(or_engine *e, const zc *wf, zc logw, zc *thUp, zc *thDn, int *info)
{
    zc lo;
    if (e->kind == OR_CP) *info = or_sdsd(e->n, e->N, e->phiT, e->logwT, wf, logw, &lo, thUp, NULL, NULL);
    else *info = or_sd2s_sd2is(e->n, e->Nup, e->Ndn, e->phiT, e->phiTDn, e->logwT, wf, logw, &lo, thUp, thDn);
    return lo;
}

/* log overlaps of every walker with the trial (alive or not) */
void or_log_overlaps(or_engine *e, double *out)
{
    zc *o = (zc *)out; int info;
    for (int w = 0; w < e->W; ++w) o[w] = or_walker_logoverlap(e, e->wf + or_wsize(e) * w, e->logw[w], NULL, NULL, &info);
}

/* Green's function G = conj(phiT) thetaT (n x n) of walker w (CP), or of spin s (PL). */
void or_green_matrix(or_engine *e, int w, int spin, double *out)
{
    int n = e->n; zc *G = (zc *)out; int info;
    const zc *wf = e->wf + or_wsize(e) * w;
    if (e->kind == OR_CP) {
        zc *th = (zc *)malloc(sizeof(zc) * e->N * n);
        or_sdsd(n, e->N, e->phiT, e->logwT, wf, e->logw[w], NULL, th, NULL, NULL);
        /* gmm(conj(phiT), thetaT) (SDSDOperation.cpp:74-89) */
        zc *cl = (zc *)malloc(sizeof(zc) * n * e->N);
        for (int i = 0; i < n * e->N; ++i) cl[i] = conj(e->phiT[i]);
        or_zgemm('N', 'N', n, n, e->N, 1.0, cl, n, th, e->N, 0.0, G, n);
        free(cl); free(th);
    } else {
        int Ns = spin == 0 ? e->Nup : e->Ndn;
        zc *thu = (zc *)malloc(sizeof(zc) * e->Nup * n);
        zc *thd = (zc *)malloc(sizeof(zc) * (e->Ndn > 0 ? e->Ndn : 1) * n);
        (void)or_walker_logoverlap(e, wf, e->logw[w], thu, thd, &info);
        const zc *pt = spin == 0 ? e->phiT : e->phiTDn;
        zc *cl = (zc *)malloc(sizeof(zc) * n * Ns);
        for (int i = 0; i < n * Ns; ++i) cl[i] = conj(pt[i]);
        or_zgemm('N', 'N', n, n, Ns, 1.0, cl, n, spin == 0 ? thu : thd, Ns, 0.0, G, n);
        free(cl); free(thu); free(thd);
    }
}

/* ---------------- CP step pieces ---------------- */

/* HubbardSOCMeasureFixedSDSD::getForce (:73-116) */
static void or_cp_force(const or_engine *e, const zc *gd, const zc *god, double *force)
{
    int L = e->L;
    for (int i = 0; i < L; ++i) {
        zc bgv;
        if (e->decomp == 0) bgv = gd[i] + gd[i + L] - 1.0;
        else if (e->decomp == 1) bgv = gd[i] - gd[i + L];
        else if (e->decomp == 2) bgv = god[i] + god[i + L];
        else bgv = god[i] - god[i + L];
        double f = creal(e->gamma[i] * bgv);
        if (f > e->forceCap) f = e->forceCap;
        if (f < -e->forceCap) f = -e->forceCap;
        force[i] = f;
    }
}

/* NiupNidn::getTwoBodySampleFromAuxForce + NiupNidnSampleSDOperation::applyToRight */
static zc or_cp_sample_apply(const or_engine *e, const int *aux, const double *force, const zc *wf,
                             zc *wfNew)
{
    int L = e->L, N = e->N, n = e->n;
    zc *d00 = (zc *)malloc(sizeof(zc) * 4 * L), *d01 = d00 + L, *d10 = d00 + 2 * L, *d11 = d00 + 3 * L;
    zc logw;
    /* setTwoBodySampleMatrix (NiupNidn.cpp:252-322) */
    for (int i = 0; i < L; ++i) {
        zc ga = aux[i] * 1.0 * e->gamma[i];
        if (e->decomp == 0) {
            zc x = cexp(ga);
            d00[i] = x * e->cd00[i]; d10[i] = x * e->cd10[i]; d01[i] = x * e->cd01[i]; d11[i] = x * e->cd11[i];
        } else if (e->decomp == 1) {
            zc x = cexp(ga), y = 1.0 / x;
            d00[i] = x * e->cd00[i]; d10[i] = y * e->cd10[i]; d01[i] = x * e->cd01[i]; d11[i] = y * e->cd11[i];
        } else if (e->decomp == 2) {
            zc c = ccosh(ga), s = csinh(ga);
            d00[i] = c * e->cd00[i] + s * e->cd10[i]; d10[i] = s * e->cd00[i] + c * e->cd10[i];
            d01[i] = c * e->cd01[i] + s * e->cd11[i]; d11[i] = s * e->cd01[i] + c * e->cd11[i];
        } else {
            zc c = ccos(ga), s = csin(ga);
            d00[i] = c * e->cd00[i] + s * e->cd10[i]; d10[i] = -s * e->cd00[i] + c * e->cd10[i];
            d01[i] = c * e->cd01[i] + s * e->cd11[i]; d11[i] = -s * e->cd01[i] + c * e->cd11[i];
        }
    }
    /* getTwoBodySampleFromAux (:100-133): logw */
    if (e->decomp == 0) {
        /* KahanData sum of aux*gamma (kahan.h) */
        zc sum = 0, comp = 0;
        for (int i = 0; i < L; ++i) {
            zc y = aux[i] * 1.0 * e->gamma[i] - comp;
            zc t = sum + y;
            comp = (t - sum) - y;
            sum = t;
        }
        logw = log(0.5) * L + e->dtUSum * 0.5 - sum;
    } else {
        logw = log(0.5) * L;
    }
    /* logProbOfAuxFromForce (:86-98) */
    double lp = 0;
    for (int i = 0; i < L; ++i) lp += aux[i] * force[i] - log(exp(force[i]) + exp(-force[i]));
    logw = logw - lp;
    /* NiupNidnSDOperation.cpp:15-41 */
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < L; ++i) {
            zc a = wf[IDX(i, j, n)], b = wf[IDX(i + L, j, n)];
            wfNew[IDX(i, j, n)] = d00[i] * a + d01[i] * b;
            wfNew[IDX(i + L, j, n)] = d10[i] * a + d11[i] * b;
        }
    free(d00);
    return logw;
}

/* ---------------- PL step pieces ---------------- */

/* RealMaterialMoleculeMeasureFixedSD2sSD2is::calculateCholeskyBg (:237-256) */
static void or_pl_cholesky_bg(const or_engine *e, const zc *thUp, const zc *thDn, zc *xbar)
{
    int n = e->n, G = e->G, Nu = e->Nup, Nd = e->Ndn;
#ifdef OR_BLAS
    if (or_blas()) {
        /* xbar = A_up^T theta_up + A_dn^T theta_dn (two zgemv, calculateCholeskyBg) */
        const zc one = 1, zero = 0;
        const int inc = 1, ku = Nu * n, kd = Nd * n;
        p_zgemv("T", &ku, &G, &one, e->Aup, &ku, thUp, &inc, &zero, xbar, &inc);
        if (kd > 0) p_zgemv("T", &kd, &G, &one, e->Adn, &kd, thDn, &inc, &one, xbar, &inc);
        return;
    }
#endif
    for (int g = 0; g < G; ++g) {
        zc s = 0;
        const zc *au = e->Aup + (size_t)g * Nu * n;
        for (int k = 0; k < Nu * n; ++k) s += au[k] * thUp[k];
        const zc *ad = e->Adn + (size_t)g * Nd * n;
        zc s2 = 0;
        for (int k = 0; k < Nd * n; ++k) s2 += ad[k] * thDn[k];
        xbar[g] = s + s2;
    }
}

/* ...::getForce (:93-116) */
static void or_pl_force(const or_engine *e, const zc *xbar, zc *force)
{
    for (int g = 0; g < e->G; ++g) {
        zc f = (xbar[g] - e->bg[g]) * e->sqrtMinusDt;
        double a = cabs(f);
        force[g] = a > e->forceCap ? f * e->forceCap / a : f;
    }
}

/* M = sum_g aux_g sqrt(-dt) L_g  (choleskyReal.cpp:160-169, one zgemv) */
static void or_pl_build_M(const or_engine *e, const zc *aux, zc *M)
{
    int n2 = e->n * e->n;
#ifdef OR_BLAS
    if (or_blas()) {
        /* real L: M = L c with c = sqrt(-dt) aux, as two dgemv (real, imaginary part) */
        int G = e->G, inc = 1;
        double *cr = (double *)malloc(sizeof(double) * G), *ci = (double *)malloc(sizeof(double) * G);
        double *mr = (double *)malloc(sizeof(double) * n2), *mi = (double *)malloc(sizeof(double) * n2);
        for (int g = 0; g < G; ++g) { zc c = aux[g] * e->sqrtMinusDt; cr[g] = creal(c); ci[g] = cimag(c); }
        const double one = 1.0, zero = 0.0;
        p_dgemv("N", &n2, &G, &one, e->chol, &n2, cr, &inc, &zero, mr, &inc);
        p_dgemv("N", &n2, &G, &one, e->chol, &n2, ci, &inc, &zero, mi, &inc);
        for (int i = 0; i < n2; ++i) M[i] = mr[i] + I * mi[i];
        free(cr); free(ci); free(mr); free(mi);
        return;
    }
#endif
    for (int i = 0; i < n2; ++i) M[i] = 0;
    for (int g = 0; g < e->G; ++g) {
        zc c = aux[g] * e->sqrtMinusDt;
        const double *Lg = e->chol + (size_t)g * n2;
        for (int i = 0; i < n2; ++i) M[i] += Lg[i] * c;
    }
}

/* logw of CholeskyReal::getTwoBodySampleFromAuxForce (choleskyReal.cpp:104-124):
 * 1/2 sum f^2 - sum x f - sqrt(-dt) sum x bg */
static zc or_pl_sample_logw(const or_engine *e, const zc *aux, const zc *force)
{
    zc f2 = 0, xf = 0, xb = 0;
    for (int g = 0; g < e->G; ++g) { f2 += force[g] * force[g]; xf += aux[g] * force[g]; xb += aux[g] * e->bg[g]; }
    return 0.5 * f2 - xf - e->sqrtMinusDt * xb;
}

/* Stand-alone two-body sample of the engine's Cholesky vectors and
 * background: M (n x n) and its logw for given aux and force (G each). */
void or_pl_two_body_sample(const or_engine *e, const double *aux, const double *force, double *M,
                           double *logw)
{
    or_pl_build_M(e, (const zc *)aux, (zc *)M);
    *(zc *)logw = or_pl_sample_logw(e, (const zc *)aux, (const zc *)force);
}

static void or_taylor_stats(or_engine *e, int order)
{
    e->taylorCalls++; e->taylorTotal += order;
    if (order < e->taylorMin) e->taylorMin = order;
    if (order > e->taylorMax) e->taylorMax = order;
}

void or_taylor_stats_get(const or_engine *e, long *calls, long *total, int *mn, int *mx)
{
    *calls = e->taylorCalls; *total = e->taylorTotal; *mn = e->taylorMin; *mx = e->taylorMax;
}

/* apply the step's one-body operator (expMinusDtK) to one walker */
static void or_apply_one_body(or_engine *e, const zc *mat, zc matLogw, int useLog, const zc *wf,
                              zc logw, zc *wfNew, zc *logwNew)
{
    int n = e->n, N = e->N;
    if (!useLog) {
        or_zgemm_nn(n, N, n, 1.0, mat, n, wf, n, wfNew, n);
    } else {
        int ord = or_loghop_apply(1, 0, 1e-10, 3, 'N', n, N, mat, wf, wfNew);
        or_taylor_stats(e, ord);
    }
    *logwNew = matLogw + logw;
}

typedef struct { or_engine *e; size_t ws; zc *lo; int *surv; } or_pass1_ctx;
static void or_pass1_body(void *c_, int w)
{
    or_pass1_ctx *c = (or_pass1_ctx *)c_;
    or_engine *e = c->e; size_t ws = c->ws; zc *lo = c->lo; int *surv = c->surv;
        if (!e->alive[w]) return;
        int info;
        lo[w] = or_walker_logoverlap(e, e->wf + ws * w, e->logw[w], NULL, NULL, &info);
        double phase = cimag(lo[w]);
        if (cos(phase) <= 0.0) { e->alive[w] = 0; return; }
        e->logw[w] += log(cos(phase)) - I * phase;
        surv[w] = 1;
    }

typedef struct { or_engine *e; size_t ws; int n, N; const int *surv; const uint64_t *offs; } or_pass2_ctx;
static void or_pass2_body(void *c_, int w)
{
    or_pass2_ctx *c = (or_pass2_ctx *)c_;
    or_engine *e = c->e; size_t ws = c->ws; int n = c->n, N = c->N;
    const int *surv = c->surv; const uint64_t *offs = c->offs;
        if (!surv[w]) return;
        or_rng r = {e->rng.seed, offs[w]};
        zc *wf = e->wf + ws * w;
        zc *tmp = (zc *)malloc(sizeof(zc) * ws);
        zc logwTmp;
        if (e->kind == OR_CP) {
            int L = e->L;
            double *force = (double *)malloc(sizeof(double) * L);
            int *aux = (int *)malloc(sizeof(int) * L);
            if (e->forceType == 1) memcpy(force, e->constForceCP, sizeof(double) * L);
            else {
                zc *gd = (zc *)malloc(sizeof(zc) * n), *god = (zc *)malloc(sizeof(zc) * n);
                zc dummy;
                or_sdsd(n, N, e->phiT, e->logwT, wf, e->logw[w], &dummy, NULL, gd, god);
                or_cp_force(e, gd, god, force);
                free(gd); free(god);
            }
            /* NiupNidn::sampleAuxFromForce (NiupNidn.cpp:66-84) */
            for (int i = 0; i < L; ++i) {
                double em = exp(-force[i]), ep = exp(force[i]);
                double prob = em / (em + ep);
                aux[i] = (or_uniform(&r) < prob) ? -1 : 1;
            }
            zc sl = or_cp_sample_apply(e, aux, force, wf, tmp);
            logwTmp = sl + e->logw[w];
            free(force); free(aux);
        } else {
            int G = e->G;
            zc *force = (zc *)malloc(sizeof(zc) * G), *aux = (zc *)malloc(sizeof(zc) * G);
            if (e->forceType == 1) memcpy(force, e->constForcePL, sizeof(zc) * G);
            else {
                zc *thu = (zc *)malloc(sizeof(zc) * e->Nup * n);
                zc *thd = (zc *)malloc(sizeof(zc) * (e->Ndn > 0 ? e->Ndn : 1) * n);
                zc *xb = (zc *)malloc(sizeof(zc) * G);
                int info;
                (void)or_walker_logoverlap(e, wf, e->logw[w], thu, thd, &info);
                or_pl_cholesky_bg(e, thu, thd, xb);
                or_pl_force(e, xb, force);
                free(thu); free(thd); free(xb);
            }
            /* CholeskyReal::sampleAuxFromForce (choleskyReal.cpp:57-65) */
            for (int g = 0; g < G; ++g) aux[g] = or_gaussian(&r) + force[g];
            /* getTwoBodySampleFromAuxForce (:104-124) */
            zc sampleLogw = or_pl_sample_logw(e, aux, force);
            /* second cos projection (afqmcPhaselessProjection.cpp:105-111) */
            zc auxForce = 0;
            for (int g = 0; g < G; ++g) auxForce += aux[g] * force[g];
            double phase = cimag(auxForce);
            if (cos(phase) <= 0.0) {
                e->alive[w] = 0;
                free(force); free(aux); free(tmp);
                return;
            }
            e->logw[w] += log(cos(phase));
            zc *M = (zc *)malloc(sizeof(zc) * n * n);
            or_pl_build_M(e, aux, M);
            int ord;
            ord = or_loghop_apply(1, 0, 1e-10, 3, 'N', n, N, M, wf, tmp);
pthread_mutex_lock(&or_stats_mu);
            or_taylor_stats(e, ord);
            pthread_mutex_unlock(&or_stats_mu);
            logwTmp = sampleLogw + e->logw[w];
            free(M); free(force); free(aux);
        }
        logwTmp += e->dt * e->ET;
        if (e->kind == OR_CP) {
            or_zgemm_nn(n, N, n, 1.0, e->expMinusDtK, n, tmp, n, wf, n);
            e->logw[w] = 0.0 + logwTmp; /* Hop::logw is 0 (hop.cpp:10-12) */
        } else if (!e->useLogOneBody) {
            or_zgemm_nn(n, N, n, 1.0, e->expMinusDtK, n, tmp, n, wf, n);
            e->logw[w] = e->logwExpMinusDtK + logwTmp;
        } else {
            int ord = or_loghop_apply(1, 0, 1e-10, 3, 'N', n, N, e->logExpMinusDtK, tmp, wf);
            (void)ord;
            e->logw[w] = e->logwLogExpMinusDtK + logwTmp;
        }
        free(tmp);
    }

/* One projection step for every alive walker:
 *   CP: AfqmcConstraintPath::projectExpMinusDtKExpMinusDtV
 *       (afqmcConstraintPathProjection.cpp:37-74)
 *   PL: AfqmcPhaseless::projectExpMinusDtKExpMinusDtV
 *       (afqmcPhaselessProjection.cpp:75-121)
 * The walker loop is split at the first cos projection: survivors' stream
 * offsets follow the reference's walker-major draw order exactly. */
static void or_project_dtk_dtv(or_engine *e)
{
    int W = e->W, n = e->n, N = e->N;
    size_t ws = or_wsize(e);
    int draws = (e->kind == OR_CP) ? e->L : 2 * e->G;
    uint64_t base = e->rng.counter;
    int *surv = (int *)calloc((size_t)W, sizeof(int));
    uint64_t *offs = (uint64_t *)calloc((size_t)W, sizeof(uint64_t));
    zc *lo = (zc *)calloc((size_t)W, sizeof(zc));
    /* pass 1: overlap and first cos projection (independent per walker) */
{
        or_pass1_ctx c1 = {e, ws, lo, surv};
        or_parallel_for(W, e->nthreads, or_pass1_body, &c1);
    }

    uint64_t acc = 0;
    for (int w = 0; w < W; ++w) { offs[w] = base + acc; acc += surv[w] ? (uint64_t)draws : 0; }
    e->rng.counter = base + acc;
    /* pass 2: force, sampling, two-body and one-body propagation */
{
        or_pass2_ctx c2 = {e, ws, n, N, surv, offs};
        or_parallel_for(W, e->nthreads, or_pass2_body, &c2);
    }

    free(surv); free(offs); free(lo);
}

typedef struct { or_engine *e; size_t ws; } or_gm_ctx;
static void or_gm_body(void *c_, int w)
{
    or_gm_ctx *c = (or_gm_ctx *)c_;
    or_engine *e = c->e; size_t ws = c->ws;
        if (!e->alive[w]) return;
        if (e->kind == OR_CP) or_sd_stabilize(e->n, e->N, e->wf + ws * w, &e->logw[w]);
        else or_sd2is_stabilize(e->n, e->Nup, e->Ndn, e->wf + ws * w, &e->logw[w]);
    }

/* modifyGM (afqmcConstraintPathProjection.cpp:95-101; afqmcPhaselessProjection.cpp:142-148) */
void or_modify_gm(or_engine *e)
{
    size_t ws = or_wsize(e);
or_gm_ctx c = {e, ws};
    or_parallel_for(e->W, e->nthreads, or_gm_body, &c);

}

/* popControl (afqmcConstraintPathProjection.cpp:103-156) in the serial
 * build: weights, popConfiguration(1, weight), in-place copies.
 * table/weights outputs may be NULL. */
/* The weights half of popControl (afqmcConstraintPathProjection.cpp:106-122):
 * weight = Re exp(logOverlap), logw -= logOverlap, every walker revived. */
void or_pop_weights(or_engine *e, double *weight)
{
    int W = e->W; size_t ws = or_wsize(e);
    for (int w = 0; w < W; ++w) {
        if (e->alive[w]) {
            int info;
            zc lo = or_walker_logoverlap(e, e->wf + ws * w, e->logw[w], NULL, NULL, &info);
            double ov = creal(cexp(lo));
            if (ov <= 0.0) { weight[w] = 0.0; e->alive[w] = 0; }
            else { weight[w] = ov; e->logw[w] -= lo; }
        } else {
            weight[w] = 0.0;
        }
    }
    for (int w = 0; w < W; ++w) e->alive[w] = 1; /* checkAndResetWalkerIsAlive */
}

void or_pop_control(or_engine *e, int *tableOut, double *weightOut)
{
    int W = e->W; size_t ws = or_wsize(e);
    double *weight = (double *)calloc((size_t)W, sizeof(double));
    or_pop_weights(e, weight);
    double *u = (double *)malloc(sizeof(double) * W);
    for (int i = 0; i < W; ++i) u[i] = or_uniform(&e->rng);
    int *table = (int *)malloc(sizeof(int) * W);
    or_pop_configuration(W, 1, weight, u, table);
    for (int i = 0; i < W; ++i) {
        int j = table[i];
        if (i != j) { memcpy(e->wf + ws * i, e->wf + ws * j, sizeof(zc) * ws); e->logw[i] = e->logw[j]; }
    }
    if (tableOut) memcpy(tableOut, table, sizeof(int) * W);
    if (weightOut) memcpy(weightOut, weight, sizeof(double) * W);
    free(weight); free(u); free(table);
}

/* projectOneStep (afqmcConstraintPathProjection.cpp:76-93) with cadence. */
void or_project_one_step(or_engine *e, int nsteps)
{
    for (int s = 0; s < nsteps; ++s) {
        or_project_dtk_dtv(e);
        e->mgsIndex++;
        if (e->mgsIndex == e->mgsStep) { or_modify_gm(e); e->mgsIndex = 0; }
        e->popIndex++;
        if (e->popIndex == e->popStep) { or_pop_control(e, NULL, NULL); e->popIndex = 0; }
    }
}

void or_set_cadence(or_engine *e, int mgsIndex, int popIndex) { e->mgsIndex = mgsIndex; e->popIndex = popIndex; }

/* RealMaterialMolecule::updateBackGround (realMaterialMolecule.cpp:103-115):
 * the new background reaches the force, the two-body sample weight and the
 * measurement at once.  With expMinusDtK non-null the one-body operators are
 * replaced as well, by the dense propagators the driver rebuilds from the new
 * background (afqmcPhaseless.cpp:145-170), which ends the Taylor form. */
void or_pl_update_background(or_engine *e, const double *bg, const double *expMinusDtK,
                             double logwExpMinusDtK, const double *expHalfDtK,
                             double logwExpHalfDtK, const double *expMinusHalfDtK,
                             double logwExpMinusHalfDtK)
{
    memcpy(e->bg, bg, sizeof(double) * e->G);
    if (!expMinusDtK) return;
    size_t n2 = (size_t)e->n * e->n;
    free(e->expMinusDtK); free(e->expHalfDtK); free(e->expMinusHalfDtK);
    e->expMinusDtK = zdup(expMinusDtK, n2); e->logwExpMinusDtK = logwExpMinusDtK;
    e->expHalfDtK = zdup(expHalfDtK, n2); e->logwExpHalfDtK = logwExpHalfDtK;
    e->expMinusHalfDtK = zdup(expMinusHalfDtK, n2); e->logwExpMinusHalfDtK = logwExpMinusHalfDtK;
    e->useLogOneBody = 0;
}

/* projectExpMinusHalfDtK / projectExpHalfDtK: which = -1 (exp(-dt/2 K)) or +1 (exp(+dt/2 K)) */
void or_project_half(or_engine *e, int which)
{
    size_t ws = or_wsize(e);
    const zc *mat = which < 0 ? e->expMinusHalfDtK : e->expHalfDtK;
    zc mlw = which < 0 ? e->logwExpMinusHalfDtK : e->logwExpHalfDtK;
    zc *tmp = (zc *)malloc(sizeof(zc) * ws);
    for (int w = 0; w < e->W; ++w) {
        if (!e->alive[w]) continue;
        if (e->kind == OR_PL && e->useLogOneBody)
            (void)or_loghop_apply(1, 0, 1e-10, 3, 'N', e->n, e->N, mat, e->wf + ws * w, tmp);
        else
            or_zgemm_nn(e->n, e->N, e->n, 1.0, mat, e->n, e->wf + ws * w, e->n, tmp, e->n);
        memcpy(e->wf + ws * w, tmp, sizeof(zc) * ws);
        e->logw[w] = mlw + e->logw[w];
    }
    free(tmp);
}

void or_reset_measurement(or_engine *e)
{
    e->den = e->HNum = e->KNum = e->VNum = e->RNum = e->TNum = 0;
    if (e->bgNum) for (int g = 0; g < e->G; ++g) e->bgNum[g] = e->exNum[g] = 0;
    if (e->siteNum) for (int k = 0; k < 4 * e->L; ++k) e->siteNum[k] = 0;
    if (e->obsNum) for (int k = 0; k < 11 * e->L * e->L; ++k) e->obsNum[k] = 0;
}

/* observe estimator switch and sums (greenMatrixNum, densityDensityNum,
 * splusSminusNum, sminusSplusNum, spairSpairNum, back to back) */
void or_cp_set_observables(or_engine *e, int on)
{
    if (on && !e->obsNum) e->obsNum = (zc *)calloc((size_t)11 * e->L * e->L, sizeof(zc));
    e->observe = on;
}
void or_get_observables(const or_engine *e, double *out)
{
    memcpy(out, e->obsNum, sizeof(zc) * 11 * e->L * e->L);
}

/* per-walker local energy of a propagated walker, accumulated with weight den */
/* HubbardSOCMeasureObserveSDSD::addGreenMatrix .. addSpairSpair
 * (HubbardSOCMeasureObserveSDSD.cpp:75-177) for one walker's full G */
static void or_cp_observables(int L, const zc *G, zc *out)
{
    int n = 2 * L;
    zc *gm = out, *dd = out + (size_t)n * n, *pm = dd + (size_t)n * n, *mp = pm + (size_t)L * L,
       *pr = mp + (size_t)L * L;
#define GG(r, c) G[(r) + (size_t)n * (c)]
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            gm[i + (size_t)n * j] = GG(i, j);
            dd[i + (size_t)n * j] = (i == j) ? GG(i, i) : GG(i, i) * GG(j, j) - GG(i, j) * GG(j, i);
        }
    for (int j = 0; j < L; ++j)
        for (int i = 0; i < L; ++i) {
            zc a, b;
            if (i == j) {
                zc both = GG(i, i) * GG(i + L, i + L) - GG(i, i + L) * GG(i + L, i);
                a = GG(i, i) - both;
                b = GG(i + L, i + L) - both;
            } else {
                a = -GG(i, j) * GG(j + L, i + L) + GG(i, i + L) * GG(j + L, j);
                b = -GG(i + L, j + L) * GG(j, i) + GG(i + L, i) * GG(j, j + L);
            }
            pm[i + (size_t)L * j] = a;
            mp[i + (size_t)L * j] = b;
            pr[i + (size_t)L * j] = GG(i, j) * GG(i + L, j + L) - GG(i, j + L) * GG(i + L, j);
        }
#undef GG
}

static void or_cp_walker_energy(or_engine *e, const zc *wf, zc logw, zc *elocOut, zc *denOut,
                                zc *KVR, zc *sites, zc *obs)
{
    int n = e->n, N = e->N, L = e->L;
    zc *th = (zc *)malloc(sizeof(zc) * N * n), *gd = (zc *)malloc(sizeof(zc) * n),
       *god = (zc *)malloc(sizeof(zc) * n);
    zc lo;
    or_sdsd(n, N, e->phiT, e->logwT, wf, logw, &lo, th, gd, god);
    zc den = cexp(lo);
    /* HubbardSOCMeasureFixedSDSD::addEnergy (:178-218) */
    zc K = 0, V = 0, R = 0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < N; ++j) K += e->wfDaggerK[IDX(j, i, N)] * th[IDX(j, i, N)];
    for (int i = 0; i < L; ++i) V += e->U[i] * (gd[i] * gd[i + L] - god[i] * god[i + L]);
    for (int i = 0; i < L; ++i) {
        R += (-e->mu[i] + e->hz[i] * 0.5) * gd[i];
        R += (-e->mu[i] - e->hz[i] * 0.5) * gd[i + L];
        R += (e->hx[i] * 0.5 - I * e->hy[i] * 0.5) * god[i];
        R += (e->hx[i] * 0.5 + I * e->hy[i] * 0.5) * god[i + L];
    }
    KVR[0] = K; KVR[1] = V; KVR[2] = R;
    if (obs) {
        /* G = conj(phiT) thetaT (SDSDOperation.cpp:74-89) */
        zc *G = (zc *)malloc(sizeof(zc) * n * n);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                zc g = 0;
                for (int a = 0; a < N; ++a) g += conj(e->phiT[IDX(i, a, n)]) * th[IDX(a, j, N)];
                G[IDX(i, j, n)] = g;
            }
        or_cp_observables(L, G, obs);
        free(G);
    }
    /* addNupNdn / addSplusSminus (HubbardSOCMeasureFixedSDSD.cpp:221-255) */
    for (int i = 0; i < L; ++i) {
        sites[i] = gd[i];
        sites[i + L] = gd[i + L];
        sites[i + 2 * L] = god[i];
        sites[i + 3 * L] = god[i + L];
    }
    *elocOut = K + V + R;
    *denOut = den;
    free(th); free(gd); free(god);
}

/* RealMaterialMoleculeMeasureFixedSD2sSD2is::addEnergy (:197-220).  The
 * walker's terms are written to xbOut/exOut (G each) and *Tout, *denOut,
 * *elocOut; or_add_mixed_measurement adds them to the sums in walker order. */
static void or_pl_walker_energy(or_engine *e, const zc *wf, zc logw, zc *elocOut, zc *denOut,
                                zc *Tout, zc *xbOut, zc *exOut)
{
    int n = e->n, G = e->G, Nu = e->Nup, Nd = e->Ndn;
    zc *thu = (zc *)malloc(sizeof(zc) * Nu * n), *thd = (zc *)malloc(sizeof(zc) * (Nd > 0 ? Nd : 1) * n);
    int info;
    zc lo = or_walker_logoverlap(e, wf, logw, thu, thd, &info);
    zc den = cexp(lo);
    /* calculateTenergy (:222-235) */
    zc T = 0;
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < Nu; ++j) T += e->wfDaggerTUp[IDX(j, i, Nu)] * thu[IDX(j, i, Nu)];
        for (int j = 0; j < Nd; ++j) T += e->wfDaggerTDn[IDX(j, i, Nd)] * thd[IDX(j, i, Nd)];
    }
    zc *xb = (zc *)malloc(sizeof(zc) * G), *ex = (zc *)malloc(sizeof(zc) * G);
    or_pl_cholesky_bg(e, thu, thd, xb);
    /* calculateCholeskyEx (:258-284): D = A_g theta (N x N), ex = tr(D D) */
    int Nm = Nu > Nd ? Nu : Nd;
    zc *D = (zc *)malloc(sizeof(zc) * Nm * Nm);
    for (int g = 0; g < G; ++g) {
        zc s = 0;
        for (int sp = 0; sp < 2; ++sp) {
            int Ns = sp == 0 ? Nu : Nd;
            const zc *A = (sp == 0 ? e->Aup : e->Adn) + (size_t)g * Ns * n;
            const zc *th = sp == 0 ? thu : thd;
            /* D(a,b) = sum_i A(a,i) theta(i,b), theta(i,b) = thetaT(b,i) */
            if (or_blas() && Ns > 0) {
                or_zgemm('N', 'T', Ns, Ns, n, 1.0, A, Ns, th, Ns, 0.0, D, Ns);
            } else {
                for (int b = 0; b < Ns; ++b)
                    for (int a = 0; a < Ns; ++a) {
                        zc d = 0;
                        for (int i = 0; i < n; ++i) d += A[IDX(a, i, Ns)] * th[IDX(b, i, Ns)];
                        D[IDX(a, b, Ns)] = d;
                    }
            }
            for (int i = 0; i < Ns; ++i)
                for (int j = 0; j < Ns; ++j) s += D[IDX(j, i, Ns)] * D[IDX(i, j, Ns)];
        }
        ex[g] = s;
    }
    zc H = 0;
    for (int g = 0; g < G; ++g) H += (xb[g] * xb[g] - ex[g]);
    H *= 0.5;
    H += T;
    *elocOut = H;
    *denOut = den;
    *Tout = T;
    memcpy(xbOut, xb, sizeof(zc) * G);
    memcpy(exOut, ex, sizeof(zc) * G);
    free(thu); free(thd); free(xb); free(ex); free(D);
}

typedef struct { or_engine *e; size_t ws; int G; zc *el, *dn, *terms, *xb, *ex, *sites, *obs; size_t nobs; } or_meas_ctx;
static void or_meas_body(void *c_, int w)
{
    or_meas_ctx *c = (or_meas_ctx *)c_;
    or_engine *e = c->e; size_t ws = c->ws; int G = c->G;
    zc *el = c->el, *dn = c->dn, *terms = c->terms, *xb = c->xb, *ex = c->ex, *sites = c->sites;
    zc *obs = c->obs ? c->obs + (size_t)w * c->nobs : NULL;
        if (!e->alive[w]) return;
        zc *tmp = (zc *)malloc(sizeof(zc) * ws);
        zc lwTmp;
        if (e->kind == OR_PL && e->useLogOneBody) {
            /* expHalfDtK only exists as a Taylor operator in this case */
            int ord = or_loghop_apply(1, 0, 1e-10, 3, 'N', e->n, e->N, e->expHalfDtK, e->wf + ws * w, tmp);
            (void)ord;
            lwTmp = e->logwExpHalfDtK + e->logw[w];
        } else {
            or_zgemm_nn(e->n, e->N, e->n, 1.0, e->expHalfDtK, e->n, e->wf + ws * w, e->n, tmp, e->n);
            lwTmp = e->logwExpHalfDtK + e->logw[w];
        }
        if (e->kind == OR_CP) or_cp_walker_energy(e, tmp, lwTmp, el + w, dn + w, terms + 3 * w,
                                                  sites + (size_t)w * 4 * e->L, obs);
        else or_pl_walker_energy(e, tmp, lwTmp, el + w, dn + w, terms + 3 * w, xb + (size_t)w * G,
                                 ex + (size_t)w * G);
        free(tmp);
    }

/* addMixedMeasurement (afqmcConstraintPathMeasure.cpp:9-23,
 * afqmcPhaselessMeasure.cpp:9-28).  eloc/den per walker may be NULL.
 * Walkers are evaluated independently (in parallel when built with OpenMP)
 * and added to the sums serially in walker order, as the reference's loop
 * does, so the sums do not depend on the thread count. */
void or_add_mixed_measurement(or_engine *e, double *elocOut, double *denOut)
{
    size_t ws = or_wsize(e);
    int W = e->W, G = e->kind == OR_PL ? e->G : 0;
    zc *el = (zc *)calloc((size_t)W, sizeof(zc)), *dn = (zc *)calloc((size_t)W, sizeof(zc));
    zc *terms = (zc *)calloc((size_t)W * 3, sizeof(zc));
    zc *xb = G ? (zc *)calloc((size_t)W * G, sizeof(zc)) : NULL;
    zc *ex = G ? (zc *)calloc((size_t)W * G, sizeof(zc)) : NULL;
    zc *sites = e->kind == OR_CP ? (zc *)calloc((size_t)W * 4 * e->L, sizeof(zc)) : NULL;
    size_t nobs = (size_t)11 * e->L * e->L;
    zc *obs = (e->kind == OR_CP && e->observe) ? (zc *)calloc((size_t)W * nobs, sizeof(zc)) : NULL;
    or_meas_ctx c = {e, ws, G, el, dn, terms, xb, ex, sites, obs, nobs};
    or_parallel_for(W, e->nthreads, or_meas_body, &c);

    for (int w = 0; w < W; ++w) {
        if (!e->alive[w]) continue;
        zc den = dn[w];
        e->den += den;
        if (e->kind == OR_CP) {
            e->KNum += terms[3 * w] * den; e->VNum += terms[3 * w + 1] * den; e->RNum += terms[3 * w + 2] * den;
            for (int k = 0; k < 4 * e->L; ++k) e->siteNum[k] += sites[(size_t)w * 4 * e->L + k] * den;
            if (obs)
                for (size_t k = 0; k < nobs; ++k) e->obsNum[k] += obs[(size_t)w * nobs + k] * den;
        } else {
            e->TNum += terms[3 * w] * den;
            for (int g = 0; g < G; ++g) {
                e->bgNum[g] += xb[(size_t)w * G + g] * den;
                e->exNum[g] += ex[(size_t)w * G + g] * den;
            }
        }
        e->HNum += el[w] * den;
    }
    if (elocOut) memcpy(elocOut, el, sizeof(zc) * W);
    if (denOut) memcpy(denOut, dn, sizeof(zc) * W);
    free(el); free(dn); free(terms); free(xb); free(ex); free(sites); free(obs);
}

/* measurement sums: out[0..]= den, HNum, (CP) KNum, VNum, RNum | (PL) TNum */
void or_get_measurement(const or_engine *e, double *out)
{
    zc *o = (zc *)out;
    o[0] = e->den; o[1] = e->HNum;
    if (e->kind == OR_CP) { o[2] = e->KNum; o[3] = e->VNum; o[4] = e->RNum; }
    else { o[2] = e->TNum; o[3] = 0; o[4] = 0; }
}
/* NupNum, NdnNum, SplusNum, SminusNum, L complex each (CP) */
void or_get_site_nums(const or_engine *e, double *out)
{
    memcpy(out, e->siteNum, sizeof(zc) * 4 * e->L);
}
void or_get_cholesky_nums(const or_engine *e, double *bgNum, double *exNum)
{
    memcpy(bgNum, e->bgNum, sizeof(zc) * e->G);
    memcpy(exNum, e->exNum, sizeof(zc) * e->G);
}

/* Stand-alone pieces for unit parity. */
void or_pl_force_single(or_engine *e, int w, double *xbarOut, double *forceOut)
{
    int n = e->n, info;
    zc *thu = (zc *)malloc(sizeof(zc) * e->Nup * n), *thd = (zc *)malloc(sizeof(zc) * (e->Ndn > 0 ? e->Ndn : 1) * n);
    (void)or_walker_logoverlap(e, e->wf + or_wsize(e) * w, e->logw[w], thu, thd, &info);
    or_pl_cholesky_bg(e, thu, thd, (zc *)xbarOut);
    or_pl_force(e, (zc *)xbarOut, (zc *)forceOut);
    free(thu); free(thd);
}

void or_cp_force_single(or_engine *e, int w, double *forceOut)
{
    int n = e->n;
    zc *gd = (zc *)malloc(sizeof(zc) * n), *god = (zc *)malloc(sizeof(zc) * n), lo;
    or_sdsd(n, e->N, e->phiT, e->logwT, e->wf + or_wsize(e) * w, e->logw[w], &lo, NULL, gd, god);
    or_cp_force(e, gd, god, forceOut);
    free(gd); free(god);
}
