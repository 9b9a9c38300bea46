/*
 * afqmc_b200.h -- C ABI of the B200 AFQMC walker-step engine.
 *
 * The engine keeps a whole walker population resident in GPU memory as one
 * strided batch and advances it with hand-written sm_100a kernels.  Each
 * entry point below replaces one member (or loop) of the reference's
 * compile-time plugin API for this path (hshi/AFQMCLAB); the reference
 * interface is cited beside every declaration (file:line, relative to the
 * AFQMCLAB project root).
 *
 * Conventions
 *  - Every function returns an int status: 0 = OK, otherwise an AFQMC_ERR_*
 *    code; afqmc_last_error() gives a message.  Nothing here calls exit().
 *  - Host buffers use the reference's storage: complex<double> interleaved
 *    (re, im), column-major (TensorHao, tensor_core.h:83-91); a population is
 *    W walker matrices stacked one after the other (walker w at w*n*ncol).
 *  - "complex" scalars are passed as two doubles (re, im).
 *  - All device work is issued on the engine's stream (afqmc_set_stream); the
 *    get_* calls synchronise that stream before returning host data.
 */
#ifndef AFQMC_B200_H
#define AFQMC_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define AFQMC_OK 0
#define AFQMC_ERR_ARG 1
#define AFQMC_ERR_CUDA 2
#define AFQMC_ERR_STATE 3
#define AFQMC_ERR_UNSUPPORTED 4

/* precision forms */
#define AFQMC_FP64 0   /* plain form: every contraction in FP64 */
#define AFQMC_MIXED 1  /* tensor-core contractions, FP64 LU/log-det/weights/QR */

/* NiupNidn decompositions (NiupNidn.h:16) */
#define AFQMC_DENSITY_CHARGE 0
#define AFQMC_DENSITY_SPIN 1
#define AFQMC_HOP_CHARGE 2
#define AFQMC_HOP_SPIN 3

/* force types (afqmcConstraintPathMethod.h / afqmcPhaselessMethod.h forceType) */
#define AFQMC_DYNAMIC_FORCE 0
#define AFQMC_CONST_FORCE 1

typedef struct afqmc_engine afqmc_engine;

/* Last error message of the calling thread (empty when none). */
const char *afqmc_last_error(void);

/* Library version string. */
const char *afqmc_version(void);

/* ---------------------------------------------------------------------------
 * Constrained-path Hubbard engine: SD walkers (2L x N), HubbardSOC model,
 * NiupNidn two-body, HubbardSOCMeasureFixedSDSD mixed estimator.
 * Replaces AfqmcConstraintPath::initialParameters/initialMeasure
 * (tutorials/afqmcConstraintPath/source/afqmcConstraintPath.cpp:20-38):
 *   K                 2L x 2L complex   HubbardSOC::K (HubbardSOC.cpp:39-59)
 *   expMinusDtK, expHalfDtK, expMinusHalfDtK
 *                     2L x 2L complex   Hop matrices from returnExpMinusAlphaK
 *                                       (HubbardSOC.cpp:109-118); Hop::logw = 0
 *   U, mu, hx, hy, hz L doubles each    (NiupNidn ctor, NiupNidn.cpp:12-26)
 *   const_force       L doubles or NULL (readForce, NiupNidn.cpp:58-64)
 *   phiT              2L x N complex    trial SD (phiT.dat)
 * ------------------------------------------------------------------------- */
int afqmc_cp_create(int L, int N, int W, int decomp, int force_type, double dt, double ET,
                    double force_cap, int mgs_step, int pop_control_step, int precision,
                    const double *K, const double *expMinusDtK, const double *expHalfDtK,
                    const double *expMinusHalfDtK, const double *U, const double *mu,
                    const double *hx, const double *hy, const double *hz,
                    const double *const_force, const double *phiT, double logwT_re,
                    double logwT_im, unsigned long long seed, afqmc_engine **out);

/* ---------------------------------------------------------------------------
 * Phaseless real-material engine: SD2is right walkers (n x max(Nup,Ndn)),
 * SD2s trial, RealMaterialMolecule + CholeskyReal, mixed estimator
 * RealMaterialMoleculeMeasureFixedSD2sSD2is.
 * Replaces AfqmcPhaseless::initialParameters/initialMeasure
 * (tutorials/afqmcPhaseless/source/afqmcPhaseless.cpp:32-72):
 *   chol   n x n x G real   RealMaterialMolecule::choleskyVecs (realMaterialMolecule.cpp:41-60)
 *   bg     G real           choleskyBg
 *   t      n x n real       one-body matrix of the T energy (initWfDaggerT, :148-163)
 *   expMinusDtK/expHalfDtK/expMinusHalfDtK (n x n complex) with their logw:
 *          Hop2is operators of returnExpMinusAlphaK (realMaterialMolecule.cpp:117-132);
 *          pass NULL for all three to use the Taylor (LogHop2is) form instead:
 *   logExpMinusDtK (n x n complex) + logw: returnLogExpMinusAlphaK (:134-146);
 *          in that case expHalfDtK/expMinusHalfDtK slots hold the LogHop2is
 *          matrices of +-dt/2 (as in the oracle).
 *   const_force  G complex or NULL
 *   phiTUp (n x Nup), phiTDn (n x Ndn) complex: SD2s trial
 * ------------------------------------------------------------------------- */
int afqmc_pl_create(int n, int Nup, int Ndn, int G, int W, int force_type, double dt, double ET,
                    double force_cap, int mgs_step, int pop_control_step, int precision,
                    const double *chol, const double *bg, const double *t,
                    const double *expMinusDtK, double logwExpMinusDtK, const double *expHalfDtK,
                    double logwExpHalfDtK, const double *expMinusHalfDtK,
                    double logwExpMinusHalfDtK, const double *logExpMinusDtK,
                    double logwLogExpMinusDtK, const double *const_force, const double *phiTUp,
                    const double *phiTDn, double logwT_re, double logwT_im,
                    unsigned long long seed, afqmc_engine **out);

int afqmc_destroy(afqmc_engine *e);

/* Work stream (a cudaStream_t); NULL restores the engine's own stream. */
int afqmc_set_stream(afqmc_engine *e, void *cuda_stream);
int afqmc_synchronize(afqmc_engine *e);

/* Population upload/download in the reference layout.
 * Walker data: SD::wfRef/logwRef (SD.h:17-62), SD2is (SD2is.h:17-64);
 * alive: the driver's walkerIsAlive vector. */
int afqmc_set_walkers(afqmc_engine *e, const double *wf, const double *logw, const int *alive);
int afqmc_get_walkers(afqmc_engine *e, double *wf, double *logw, int *alive);
/* Pipelined form of afqmc_set_walkers (same layout; no counterpart in the
 * reference, whose walkers stay in host memory): the host-to-device copy runs
 * on an internal copy stream while earlier work on the engine's stream is still
 * running, and the population is installed on the engine's stream after all
 * work enqueued before the call; returns without waiting.  Host buffers should
 * be pinned and must stay unchanged until the copy has finished
 * (afqmc_upload_wait, or any call that synchronizes the engine's stream after
 * the install).  The first call allocates two device staging slots. */
int afqmc_set_walkers_async(afqmc_engine *e, const double *wf, const double *logw, const int *alive);
/* The same asynchronous upload for the phaseless mixed form with the walkers
 * already in its fp32 layout: per walker 2 n Ncol floats, the real parts
 * (n x Ncol, column-major) then the imaginary parts; the form keeps its
 * walkers in that layout, so this moves half the bytes of the FP64 upload.
 * Other engines return AFQMC_ERR_UNSUPPORTED.  The first call allocates two
 * fp32 staging slots.  (SD2is::read/write carry complex doubles; the
 * difference is only the upload format.) */
int afqmc_set_walkers_f32_async(afqmc_engine *e, const float *wf32, const double *logw, const int *alive);
int afqmc_upload_wait(afqmc_engine *e);

/* Counter-based random stream: replaces randomHaoInit/randomHaoSave/Read
 * (common/randomHao/source/random_hao.cpp:10-71).  The stream is the
 * SplitMix64 sequence of `seed`; `counter` is the next draw's position. */
int afqmc_set_rng(afqmc_engine *e, unsigned long long seed, unsigned long long counter);
int afqmc_get_rng(afqmc_engine *e, unsigned long long *seed, unsigned long long *counter);

/* method.ET (afqmcConstraintPathMethod.h ET) */
int afqmc_set_ET(afqmc_engine *e, double ET);
/* mgsIndex / popControlIndex of projectOneStep */
int afqmc_set_cadence(afqmc_engine *e, int mgs_index, int pop_control_index);

/* projectOneStep x nsteps (afqmcConstraintPathProjection.cpp:76-93,
 * afqmcPhaselessProjection.cpp:123-140): projectExpMinusDtKExpMinusDtV, then
 * modifyGM every mgs_step and popControl every pop_control_step. */
int afqmc_project_one_step(afqmc_engine *e, int nsteps);

/* With enable != 0, afqmc_project_one_step and afqmc_add_mixed_measurement
 * replay CUDA graphs of their kernel sequences (one per cadence variant),
 * captured on first use after one direct step; changing E_T, the seed, the
 * stream or the one-body operators re-captures.  No counterpart in the
 * reference (it launches nothing). */
int afqmc_set_graphs(afqmc_engine *e, int enable);

/* projectExpMinusHalfDtK (which = -1) / projectExpHalfDtK (which = +1)
 * (afqmcConstraintPathProjection.cpp:11-29, afqmcPhaselessProjection.cpp:11-73) */
int afqmc_project_half(afqmc_engine *e, int which);

/* modifyGM: stabilize() every alive walker (SD.cpp:42-56, SD2is.cpp:48-76) */
int afqmc_modify_gm(afqmc_engine *e);

/* popControl (afqmcConstraintPathProjection.cpp:103-156): weights, comb
 * (popConfiguration, populationControlConfiguration.cpp:24-101) and copies
 * (populationControl<T>, populationControl.h:110-117).  table_out (W ints)
 * and weight_out (W doubles) are optional host outputs. */
int afqmc_pop_control(afqmc_engine *e, int *table_out, double *weight_out);

/* Mixed estimator: addMixedMeasurement (afqmcConstraintPathMeasure.cpp:9-23,
 * afqmcPhaselessMeasure.cpp:9-28), reSet, and the accumulated sums.
 * afqmc_get_measurement writes 5 complex numbers:
 *   CP: den, HNum, KNum, VNum, RNum   PL: den, HNum, TNum, 0, 0 */
int afqmc_reset_measurement(afqmc_engine *e);
int afqmc_add_mixed_measurement(afqmc_engine *e);
int afqmc_get_measurement(afqmc_engine *e, double *out);
/* Site sums of the constrained-path mixed estimator, L complex each (NULL
 * skips one): NupNum, NdnNum (den-weighted G diagonals of the up and down
 * sites) and SplusNum, SminusNum (the two spin-flip off-diagonals), as
 * HubbardSOCMeasureFixedSDSD::addNupNdn / addSplusSminus accumulate them
 * (HubbardSOCMeasureFixedSDSD.cpp:221-255); the *TotNum totals are their sums.
 * CP only. */
int afqmc_get_site_nums(afqmc_engine *e, double *NupNum, double *NdnNum, double *SplusNum,
                        double *SminusNum);
/* Observe estimator of the constrained path (HubbardSOCMeasureObserveSDSD,
 * HubbardSOCMeasureObserveSDSD.cpp:42-185): with on != 0 every
 * afqmc_add_mixed_measurement also builds each walker's full Green's matrix
 * and adds den-weighted greenMatrixNum and densityDensityNum (2L x 2L each)
 * and splusSminusNum, sminusSplusNum, spairSpairNum (L x L each);
 * afqmc_reset_measurement clears them.  Off by default (W x 4L^2 complex of
 * device memory when on).  CP only. */
int afqmc_cp_set_observables(afqmc_engine *e, int on);
/* The observe sums, complex column-major (NULL skips one). */
int afqmc_get_observables(afqmc_engine *e, double *greenNum, double *densityDensityNum,
                          double *splusSminusNum, double *sminusSplusNum, double *spairSpairNum);
/* Back-propagated estimator of the constrained path (tutorials/
 * afqmcConstraintPathBP: prepareBackPropagation,
 * afqmcConstraintPathBackPropagation.cpp:11-20; addMeasurement,
 * afqmcConstraintPathMeasure.cpp:47-78).  afqmc_cp_bp_begin starts a window of
 * `steps` steps from the current walkers (measure_skip: the driver's
 * measureSkipStep); every step then records its auxiliary fields and any
 * population-control table.  Once `steps` steps are recorded,
 * afqmc_cp_bp_measure resamples the window-start walkers by the recorded
 * tables, propagates the trial leftwards through each walker's recorded
 * fields, and adds the observe estimator (den, HNum/KNum/VNum/RNum from the
 * full Green's matrix, greenMatrixNum, ...) for the pair, weighted by the
 * current walker's overlap; with steps >= measure_skip the window then slides
 * by measure_skip steps, otherwise back-propagation stops until the next
 * afqmc_cp_bp_begin.  FP64 form, observe estimator on
 * (afqmc_cp_set_observables); a step past a full window is an error.
 * afqmc_cp_bp_state reports whether a window is open and its BPIndex. */
int afqmc_cp_bp_begin(afqmc_engine *e, int steps, int measure_skip);
int afqmc_cp_bp_measure(afqmc_engine *e);
int afqmc_cp_bp_state(afqmc_engine *e, int *active, int *index);
/* choleskyBgNum / choleskyExNum (G complex each), PL only */
int afqmc_get_cholesky_nums(afqmc_engine *e, double *bgNum, double *exNum);

/* Background update + propagator replacement: RealMaterialMolecule::
 * updateBackGround (realMaterialMolecule.cpp:103-115) and the rebuild in
 * afqmcPhaseless.cpp:151-177.  Matrices as in afqmc_pl_create (NULL keeps). */
int afqmc_pl_update_background(afqmc_engine *e, const double *bg, const double *expMinusDtK,
                               double logwExpMinusDtK, const double *expHalfDtK,
                               double logwExpHalfDtK, const double *expMinusHalfDtK,
                               double logwExpMinusHalfDtK);

/* Propagator rebuild on the GPU from the engine's current background:
 * RealMaterialMolecule::setKp (Kp = K + sum_g bg_g L_g,
 * realMaterialMolecule.cpp:155-166) and the three returnExpMinusAlphaK
 * calls of afqmcPhaseless.cpp:151-177 (alpha = dt, -dt/2, dt/2 into
 * expMinusDtK, expHalfDtK, expMinusHalfDtK; logw = alpha * 0.5 * sum bg^2,
 * realMaterialMolecule.cpp:117-131).  K: the model's one-body K, n x n
 * column-major.  exp(-alpha Kp) is a scaled Taylor series evaluated with
 * FP64 GEMMs (the reference diagonalises Kp; same matrix function).  The
 * engine leaves the Taylor one-body form, as after a dense update. */
int afqmc_pl_rebuild_propagators(afqmc_engine *e, const double *K);

/* Adjoint of the mixed local energy E = sum_w den_w E_w / sum_w den_w and of
 * the mean log-overlap at the current walkers (no one-body half step), with
 * respect to the one-body matrix t (RealMaterialMolecule::t), the Cholesky
 * vectors (choleskyVecs) and the trial orbitals of the SD2s trial (E depends
 * on conj(phiT) only; the orbital outputs are d/dconj(phiT)).  dE_dt is the
 * mixed one-body density matrix (sum_s G_s of SD2sSD2isOperation::
 * returnGreenMatrixUp/Dn, SD2sSD2isOperation.cpp:74-104, den-weighted).
 * Outputs (host, complex, column-major, any may be NULL): energy (1),
 * mean_logov (1), dE_dt (n x n), dE_dchol (n x n x G), dE_dconj_phiT_up
 * (n x Nup), dE_dconj_phiT_dn (n x Ndn), dLogov_dconj_phiT_up/dn.
 * dE_dchol may instead be device memory of the engine's GPU (found by
 * cudaPointerGetAttributes): the gradient is then written there directly,
 * with no copy to the host (device memory of another GPU: AFQMC_ERR_ARG).
 * FP64; determinants and D_g are recomputed per walker, nothing is stored. */
int afqmc_pl_adjoint(afqmc_engine *e, double *energy, double *mean_logov, double *dE_dt,
                     double *dE_dchol, double *dE_dconj_phiT_up, double *dE_dconj_phiT_dn,
                     double *dLogov_dconj_phiT_up, double *dLogov_dconj_phiT_dn);

/* Diagnostics (gauge-invariant quantities for parity checks) */
/* log <phiT|phi_w> of every walker: SDSDOperation::returnLogOverlap (SDSDOperation.cpp:65-72) */
int afqmc_log_overlaps(afqmc_engine *e, double *out);
/* G = conj(phiT) thetaT of one walker (SDSDOperation.cpp:74-89; spin for SD2is) */
int afqmc_green_matrix(afqmc_engine *e, int walker, int spin, double *out);
/* dynamicOrder statistics of LogHop2isSD2isOperation::print (logHop2isSD2isOperation.cpp:56-88) */
int afqmc_taylor_stats(afqmc_engine *e, long long *calls, long long *total, int *min_order,
                       int *max_order);
/* OR of the per-walker status bits since creation (1 singular overlap,
 * 2 non-finite value, 4 Taylor order cap, 8 zero column norm, 16 comb) */
int afqmc_status(afqmc_engine *e, int *status_or);

/* Self-check of the bounded waits of the tensor-core kernels: one CTA that
 * holds a TMEM allocation waits, with the same wait helpers those kernels
 * use, on two mbarriers that nothing arrives at, gives up after limit_cycles
 * SM cycles (clamped to [1000, about one second]), completes the phases
 * itself, frees its TMEM and returns.  *error_word receives the bits of the
 * waits that gave up (1: spinning wait, 2: suspending wait): 3 when the
 * bounds work.  Nothing is in flight while it waits, and the context stays
 * usable.  Synchronises `stream` (a cudaStream_t).  No counterpart in the
 * reference (it has no device code). */
int afqmc_bounded_wait_check(long long limit_cycles, int *error_word, void *stream);

/* Phase profiler: CUDA events around each phase of the step on the engine's
 * stream (replaces the reference's 1-second TimerHao, common/timeHao/include/
 * time_hao.h:16-41).  Enabling resets the totals; afqmc_profile_get writes
 * AFQMC_NPHASES milliseconds totals and launch counts. */
#define AFQMC_NPHASES 12
#define AFQMC_PH_OVERLAP 0     /* S = phiT^H phi */
#define AFQMC_PH_LU 1          /* LU, log-det, inverse, first cos projection */
#define AFQMC_PH_THETA 2       /* thetaT = S^-T phi^T */
#define AFQMC_PH_FORCE 3       /* force (Hubbard G diagonal / Cholesky xbar) */
#define AFQMC_PH_SAMPLE 4      /* aux-field sampling (+ Hubbard 2x2 apply) */
#define AFQMC_PH_MBUILD 5      /* M = sqrt(-dt) sum_g x_g L_g */
#define AFQMC_PH_TAYLOR 6      /* exp(M) phi */
#define AFQMC_PH_ONEBODY 7     /* exp(-dt K) phi */
#define AFQMC_PH_STABILIZE 8   /* modifyGM */
#define AFQMC_PH_POPCONTROL 9  /* popControl */
#define AFQMC_PH_EXCHANGE 10   /* exchange term of the measurement */
#define AFQMC_PH_MEASURE 11    /* rest of the measurement */
int afqmc_profile_enable(afqmc_engine *e, int on);
/* Number of kernels this library has launched since it was loaded. */
long long afqmc_launch_count(void);
int afqmc_profile_get(afqmc_engine *e, double *ms, long long *counts);

/* ---------------------------------------------------------------------------
 * Stand-alone batched operations on device pointers (same layouts).
 * ------------------------------------------------------------------------- */
/* popConfiguration for one process (populationControlConfiguration.cpp:24-101)
 * with explicit uniforms: weights, uniforms (W doubles each), table (W ints).
 * stream is a cudaStream_t (may be NULL). */
int afqmc_pop_configuration_dev(int W, const double *weights, const double *uniforms, int *table,
                                void *stream);

/* ---- uneven batches ----
 * Engines of different lattice size and filling advanced together: each
 * afqmc_batch_step is one CUDA-graph launch holding one branch per engine
 * (each on its engine's stream).  The engines must share mgs_step,
 * pop_control_step and their current cadence indices.  The first step runs
 * directly (one-time setup, autotuning); the graphs are captured after it.
 * No counterpart in the reference, which runs one lattice per process. */
typedef struct afqmc_batch afqmc_batch;
int afqmc_batch_create(afqmc_engine **engines, int count, afqmc_batch **out);
int afqmc_batch_step(afqmc_batch *b, int nsteps);
int afqmc_batch_synchronize(afqmc_batch *b);
/* Launch the batch's graphs on a caller-owned cudaStream_t (NULL is refused:
 * the legacy default stream cannot be captured). */
int afqmc_batch_set_stream(afqmc_batch *b, void *cuda_stream);
int afqmc_batch_destroy(afqmc_batch *b);
/* Process-wide switch of the GEMM autotuner: with enable != 0 every new
 * FP64 GEMM shape is timed once over the candidate tile shapes (outside
 * stream capture) and the fastest is kept for that shape. */
int afqmc_set_autotune(int enable);

/* ---- population control across processes (one population per GPU) ----
 * The reference gathers the weights on rank 0, builds the table there and
 * moves walkers with MPI (populationControl<T>, populationControl.h:20-109;
 * popConfiguration(size, weight), populationControlConfiguration.cpp:24-101).
 * Here every rank computes the same table from the gathered weights and a
 * shared uniform stream, then walkers move point to point (NCCL / gloo),
 * see afqmclab_b200/parallel.py. */
/* popConfiguration(size, weight) on the host, with explicit uniforms
 * (L = size * walkers per rank); table[i] is the global parent of slot i. */
int afqmc_pop_configuration_host(int L, int size, const double *weight, const double *uniforms,
                                 int *table);
/* First half of popControl on this rank: weights Re<phiT|phi>, logw -= logOverlap,
 * walkers revived (afqmcConstraintPathProjection.cpp:106-122). */
int afqmc_pop_weights(afqmc_engine *e, double *weight_out);
/* Bytes of one walker in the transfer format: its n x ncol complex128
 * matrix followed by its complex128 logw. */
long long afqmc_walker_bytes(afqmc_engine *e);
/* Copy walker w to / from a device buffer of afqmc_walker_bytes bytes. */
int afqmc_copy_walker_out(afqmc_engine *e, int w, void *dst_dev);
int afqmc_copy_walker_in(afqmc_engine *e, int w, const void *src_dev);
/* Batched transfer records for the walkers that change rank: pack writes
 * walkers idx[0..count) back to back (afqmc_walker_bytes each) to dst_dev;
 * unpack fills slots[0..count) (distinct) from src_dev.  One kernel each, so
 * a whole population control's moves to one peer travel as one message
 * (the reference sends one walker per MPI message, populationControl.h:55-100).
 * idx / slots are host arrays. */
int afqmc_pack_walkers(afqmc_engine *e, int count, const int *idx, void *dst_dev);
int afqmc_unpack_walkers(afqmc_engine *e, int count, const int *slots, const void *src_dev);
/* In-place copies walker[i] = walker[table[i]] within this rank (table in
 * local indices; parents keep their own slot). */
int afqmc_apply_table(afqmc_engine *e, const int *table);

/* Allocation-free variant of afqmc_pop_configuration_dev, for callers that
 * cannot allocate device memory where they need a population-control table
 * (a host framework that owns the GPU memory through its own pool, a fixed
 * start-up memory budget, or a loop that cannot afford an allocation's
 * implicit synchronisation).  It has no counterpart in the reference.
 * Same inputs, outputs and table as afqmc_pop_configuration_dev; its only
 * scratch, the per-walker copy counts, is a file-scope device array of
 * AFQMC_NOALLOC_MAX_WALKERS ints that every GPU loading the library holds
 * until the process exits.  W above that limit is rejected with
 * AFQMC_ERR_ARG.  The first call on a device looks up that array's device
 * address (cudaGetSymbolAddress) with the device current; make that first
 * call before any stream capture.  The kernel clears the counts itself, but
 * all calls share the one array: calls that overlap on the GPU (different
 * streams, no ordering) race on it. */
#define AFQMC_NOALLOC_MAX_WALKERS 65536
int afqmc_pop_configuration_noalloc_dev(int W, const double *weights, const double *uniforms,
                                        int *table, void *stream);

/* Tensor-core (tcgen05) bf16 GEMM used by the mixed-precision form, the
 * batched counterpart of gmm_cpu (tensor_2d_bl_cpu.cpp:61-75):
 * C[m + n*ldc] = alpha * sum_k A[m*lda + k] * B[n*ldb + k]  (A, B bf16
 * K-major; C fp32, or bf16 with out_bf16 != 0).  With splits > 1, K is cut
 * into `splits` equal parts (multiples of 64) and part s is written at
 * C + s*split_stride.  Synchronises `stream` before returning. */
int afqmc_gemm_bf16_dev(int M, int N, int K, const void *A, long long lda, const void *B,
                        long long ldb, void *C, long long ldc, int out_bf16, int splits,
                        long long split_stride, float alpha, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* AFQMC_B200_H */
