// Kernels of the AFQMC walker step that are not plain GEMMs.
#pragma once
#include "common.cuh"

// Overlap blocks of one walker: CP (SD) has one block of N columns; the
// phaseless SD2is walker has an up block (Nup) and a down block (Ndn), both
// starting at column 0 of the same matrix (SD2sSD2isOperation.cpp:40-43).
struct Blocks {
    int nblk;
    int Ns[2];
    long long sOff[2];   // offset of block b inside a walker's S/Sinv slot
    long long tOff[2];   // offset of block b inside a walker's thetaT slot
    long long sStride;   // per-walker S slot size (elements)
    long long tStride;   // per-walker thetaT slot size (elements)
    // log-det multiplicity of the listed blocks: 2 when one listed block
    // stands for two identical spin blocks (same trial, same walker columns)
    int mult = 1;
};

enum { LU_PLAIN = 0, LU_PROJECT = 1, LU_POPWEIGHT = 2 };

void launch_lu_logdet_inverse(int W, const Blocks &bl, zd *S, zd *Sinv, const int *active,
                              const zd *logw, zd logwAdd, zd logwT, zd *logov, int *alive,
                              int *surv, zd *logwOut, double *weight, int *status, int mode,
                              bool wantInverse, cudaStream_t s);
// Floats per walker of the fp32 inverse slots: 2 sStride rounded up to a
// multiple of 4, so every walker's slot starts on a 16-byte boundary.
inline long long sinv32_stride(const Blocks &bl) { return (2 * bl.sStride + 3) & ~3LL; }
// Same as launch_lu_logdet_inverse, with the inverses (when wanted) written as
// fp32 planes [re | im] (each Ns x Ns column-major) at
// Sinv32 + w * sinv32_stride(bl) + 2 sOff[b]; Sinv is FP64 scratch for the
// kernels that produce FP64 first.
void launch_lu_logdet_inverse32(int W, const Blocks &bl, zd *S, zd *Sinv, float *Sinv32, const int *active,
                                const zd *logw, zd logwAdd, zd logwT, zd *logov, int *alive, int *surv,
                                zd *logwOut, double *weight, int *status, int mode, bool wantInverse,
                                cudaStream_t s);

void launch_rng_scan(int W, const int *surv, int draws, unsigned long long *counter,
                     unsigned long long *offs, cudaStream_t s);

// Hubbard (NiupNidn) pieces
struct HubbardDev {
    int L, N, n, decomp;
    const zd *gamma, *cd00, *cd01, *cd10, *cd11;
    double dtUSum, forceCap;
    const double *constForce;  // non-null for constForce
    const zd *phiT;
};
void launch_cp_force(int W, const HubbardDev &h, const zd *thetaT, long long tStride,
                     const int *surv, double *force, cudaStream_t s);
void launch_cp_sample_apply(int W, const HubbardDev &h, const double *force, const int *surv,
                            const unsigned long long *offs, uint64_t seed, const zd *wf,
                            zd *wfTmp, zd *logw, double dtET, zd hopLogw, int *auxOut,
                            cudaStream_t s);

// Phaseless (CholeskyReal) pieces
struct CholDev {
    int n, G;
    const double *bg;
    // sqrt(-dt) = i * sqrtMinusDtIm.  The reference evaluates it as
    // sqrt(-dt * complex(1, 0)) (choleskyReal.cpp:17), whose argument has
    // imaginary part -0.0, so the principal root is -i sqrt(dt):
    // sqrtMinusDtIm = -sqrt(dt).
    double forceCap, sqrtMinusDtIm;
    const zd *constForce;      // non-null for constForce
};
void launch_pl_sample(int W, const CholDev &c, const zd *xbar, const int *surv_in, int *surv,
                      int *alive, const unsigned long long *offs, uint64_t seed, zd *aux,
                      zd *force, zd *logw, double dtET, zd hopLogw, cudaStream_t s);

// Taylor series bookkeeping: wfNew += term; convergence per walker
void launch_taylor_accum(int W, long long wsize, const zd *term, zd *wfNew, const int *surv,
                         int *done, int *order, int k, int checkFrom, double acc, int isLast,
                         int *status, cudaStream_t s);

// Modified Gram-Schmidt stabilisation (replaces SD::stabilize / SD2is::stabilize)
// Gram-Schmidt with the columns in registers; wf is zd (f32 false) or the
// mixed form's fp32 planes (f32 true).  Returns false (nothing launched)
// where the shape does not fit one CTA of 512 lanes.
bool launch_mgs_col(int W, int n, int ncol, int nup, int ndn, int isSD2is, void *wf, bool f32, zd *logw,
                    const int *alive, int *status, cudaStream_t s);
void launch_mgs(int W, int n, int ncol, int nup, int ndn, int isSD2is, zd *wf, zd *logw,
                const int *alive, int *status, cudaStream_t s);

// Population control
// uniforms == NULL: draw W uniforms from the stream at *counter (then advance it)
void launch_pop_comb(int W, const double *weight, const double *uniforms, uint64_t seed,
                     unsigned long long *counter, int *number, int *table, int *status,
                     cudaStream_t s);
// Observe-estimator sums (greenMatrixNum, densityDensityNum: n x n each;
// splusSminusNum, sminusSplusNum, spairSpairNum: L x L each, in that order in obs).
void launch_cp_observe(int W, int L, const zd *G, const zd *den, const int *alive, zd *obs, cudaStream_t s);
// back-propagation: a recorded field sample applied to the right or the
// left of the walkers whose record is valid; recorded rows gathered by a
// population-control table; the commute estimator's energies from full G;
// an elementwise conjugate copy
void launch_cp_aux_apply(int W, const HubbardDev &h, const int *aux, const int *valid, const zd *wf, zd *wfOut,
                         zd *logw, bool left, zd extraLogw, cudaStream_t s);
void launch_bp_gather_rows(int W, int rowlen, int nsteps, const int *table, int *data, cudaStream_t s);
void launch_cp_commute_energy(int W, int L, const zd *G, const zd *K, const double *U, const double *mu,
                              const double *hx, const double *hy, const double *hz, const int *alive,
                              const zd *logov, zd *eloc, zd *den, zd *parts, cudaStream_t s);
void launch_zconj(long long count, const zd *src, zd *dst, cudaStream_t s);
// Batched walker transfer records (matrix + logw each), walker idx[k] <-> record k.
void launch_walker_xfer(int count, long long wsize, const int *idx, zd *wf, zd *logw, zd *buf, bool unpack,
                        cudaStream_t s);
void launch_pop_gather(int W, long long wsize, const int *table, zd *wf, zd *logw,
                       cudaStream_t s);
void launch_set_int(int *p, int v, int count, cudaStream_t s);
void launch_copy_masked(int W, long long wsize, const zd *src, zd *dst, const int *mask,
                        cudaStream_t s);

// Measurement
void launch_cp_energy(int W, const HubbardDev &h, const zd *wfDaggerK, const zd *thetaT,
                      long long tStride, const double *U, const double *mu, const double *hx,
                      const double *hy, const double *hz, const int *alive, const zd *logov,
                      zd *eloc, zd *den, zd *parts, zd *sites, cudaStream_t s);
// Aall: column g = [A_g,up (Nup x n); A_g,dn (Ndn x n)] flattened (Ktot rows);
// returns -1 when a block is wider than 64 columns.
int launch_pl_exchange(int W, int n, int G, const Blocks &bl, const zd *Aall, long long Ktot,
                       const zd *thetaT, const int *alive, zd *ex, cudaStream_t s,
                       int thetaLayout = 0);
void launch_pl_energy(int W, int G, long long Ktot, const zd *wfDaggerT, const zd *thetaT,
                      const zd *xbar, const zd *ex, const int *alive, const zd *logov, zd *eloc,
                      zd *den, zd *tloc, cudaStream_t s, const zd *exTot = nullptr, long long tLen = -1,
                      int tMult = 1);
// (exTot: the per-walker sum over g of ex, used instead of ex when given;
// the kinetic sum runs over the first tLen entries of a walker's thetaT
// slot, default all Ktot, counted tMult times)
// Sums over alive walkers into device accumulators:
// acc[0] += sum den, acc[1] += sum eloc*den, acc[2+k] += sum parts[w*nparts+k]*den;
// with xbar/ex (phaseless): bgNum[g] += sum xbar*den, exNum[g] += sum ex*den
// (exNum untouched when ex is null).
void launch_measure_reduce(int W, const int *alive, const zd *eloc, const zd *den, const zd *parts,
                           int nparts, zd *acc, int G, const zd *xbar, const zd *ex, zd *bgNum,
                           zd *exNum, cudaStream_t s);
void launch_taylor_stats(int W, const int *mask, const int *order, long long *stats, cudaStream_t s);
void launch_pop_comb_scratch(int W, const double *weight, const double *uniforms, int *number,
                             int *table, cudaStream_t s);
