/*
 * afqmclab_b200.hpp -- C++ face of the B200 AFQMC walker-step engine.
 *
 * Header-only classes over the C ABI (afqmc_b200.h) that carry the names and
 * member signatures the reference's drivers bind through their typedefs
 * (tutorials/afqmcPhaseless/include/afqmcPhaselessDefine.h:10-26,
 *  tutorials/afqmcConstraintPath/include/afqmcConstraintPathDefine.h:10-24).
 *
 * The reference keeps `std::vector<WalkerRight> walker` in host memory and
 * calls one operation per walker; here the population lives on the GPU and
 * every call acts on all walkers at once.  Per-walker accessors of the
 * reference (returnLogOverlap, returnGreenMatrix*, walker[i].getLogw(), ...)
 * map onto slices of those batch results.
 *
 * Data layout is the reference's: std::complex<double>, column-major
 * (TensorHao, common/tensorHao/include/tensor_core.h:83-91).  Errors throw
 * afqmclab_b200::Error carrying the C-ABI status and message; the reference
 * prints and exit(1)s instead (e.g. SDSDOperation.cpp:34-38).
 *
 * Link with -lafqmc_b200 (and -lcudart where the linker asks for it).
 * Nothing here includes a CUDA header: streams are passed as void *.
 */
#ifndef AFQMCLAB_B200_HPP
#define AFQMCLAB_B200_HPP

#include <complex>
#include <cstddef>
#include <fstream>
#include <iomanip>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "afqmc_b200.h"

namespace afqmclab_b200 {

typedef std::complex<double> Complex;

// ------------------------------------------------------------------ errors
class Error : public std::runtime_error {
public:
    Error(int code, const std::string &msg) : std::runtime_error(msg), code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

inline void check(int rc, const char *what)
{
    if (rc != AFQMC_OK) throw Error(rc, std::string(what) + ": " + afqmc_last_error());
}

// ------------------------------------------------------------- containers
// Column-major complex matrix, the TensorHao<complex<double>,2> layout.
class Matrix {
public:
    Matrix() = default;
    Matrix(int rows, int cols) : rows_(rows), cols_(cols), data_((size_t)rows * cols) {}
    void resize(int rows, int cols)
    {
        rows_ = rows;
        cols_ = cols;
        data_.assign((size_t)rows * cols, Complex(0.0, 0.0));
    }
    int rank(int d) const { return d == 0 ? rows_ : cols_; }
    Complex &operator()(int i, int j) { return data_[i + (size_t)rows_ * j]; }
    const Complex &operator()(int i, int j) const { return data_[i + (size_t)rows_ * j]; }
    Complex *data() { return data_.data(); }
    const Complex *data() const { return data_.data(); }
    size_t size() const { return data_.size(); }

private:
    int rows_ = 0, cols_ = 0;
    std::vector<Complex> data_;
};

namespace detail {
// The reference's text forms (common/readWriteHao/include/readWriteFstream.h,
// TensorHao::write/read in common/tensorHao/include/tensor_core.h:278-301):
// a scalar per line, a complex number as two fields of width 26, a matrix as
// its rank, its shape, then one entry per line column by column.
inline void write_complex(std::ofstream &f, const Complex &z)
{
    f << std::setprecision(16) << std::scientific << std::setw(26) << z.real() << std::setw(26) << z.imag()
      << "\n";
}
inline void write_matrix(std::ofstream &f, const Matrix &m)
{
    f << 2 << "\n" << m.rank(0) << " " << m.rank(1) << " \n";
    for (size_t k = 0; k < m.size(); ++k) write_complex(f, m.data()[k]);
}
inline Complex read_complex(std::ifstream &f)
{
    double re = 0, im = 0;
    f >> re >> im;
    return Complex(re, im);
}
inline void read_matrix(std::ifstream &f, Matrix &m)
{
    int rank = 0, r = 0, c = 0;
    f >> rank >> r >> c;
    if (!f || rank != 2 || r < 0 || c < 0) throw Error(AFQMC_ERR_ARG, "walker file: bad matrix header");
    m.resize(r, c);
    for (size_t k = 0; k < m.size(); ++k) m.data()[k] = read_complex(f);
    if (!f) throw Error(AFQMC_ERR_ARG, "walker file: truncated matrix");
}
}  // namespace detail

// ---------------------------------------------------------------- walkers
// SD (afqmc/blocks/walker/SD/include/SD.h:17-62): logw and an L x N matrix.
// File format of SD::write / SD::read (SD.cpp:85-103): logw, then the matrix.
class SD {
public:
    SD() = default;
    SD(int L, int N) : wf_(L, N) {}
    void resize(int L, int N) { wf_.resize(L, N); }
    int getL() const { return wf_.rank(0); }
    int getN() const { return wf_.rank(1); }
    const Complex &getLogw() const { return logw_; }
    Complex &logwRef() { return logw_; }
    const Matrix &getWf() const { return wf_; }
    Matrix &wfRef() { return wf_; }
    void addLogw(Complex x) { logw_ += x; }
    void write(const std::string &filename) const
    {
        std::ofstream f(filename, std::ios::out | std::ios::trunc);
        if (!f) throw Error(AFQMC_ERR_ARG, "cannot write " + filename);
        detail::write_complex(f, logw_);
        detail::write_matrix(f, wf_);
    }
    void read(const std::string &filename)
    {
        std::ifstream f(filename);
        if (!f) throw Error(AFQMC_ERR_ARG, "cannot read " + filename);
        logw_ = detail::read_complex(f);
        detail::read_matrix(f, wf_);
    }
    double getMemory() const { return 16.0 * (double)wf_.size() + 16.0; }

private:
    Complex logw_ = Complex(0.0, 0.0);
    Matrix wf_;
};

// SD2is (SD2is.h:17-64): restricted walker, one L x max(Nup, Ndn) matrix
// whose first Nup / Ndn columns are the two spin blocks.  File format of
// SD2is::write / SD2is::read (SD2is.cpp:105-127): logw, Nup, Ndn, the matrix.
class SD2is {
public:
    SD2is() = default;
    SD2is(int L, int Nup, int Ndn) : nup_(Nup), ndn_(Ndn), wf_(L, Nup > Ndn ? Nup : Ndn) {}
    void resize(int L, int Nup, int Ndn)
    {
        nup_ = Nup;
        ndn_ = Ndn;
        wf_.resize(L, Nup > Ndn ? Nup : Ndn);
    }
    int getL() const { return wf_.rank(0); }
    int getNup() const { return nup_; }
    int getNdn() const { return ndn_; }
    const Complex &getLogw() const { return logw_; }
    Complex &logwRef() { return logw_; }
    const Matrix &getWf() const { return wf_; }
    Matrix &wfRef() { return wf_; }
    void addLogw(Complex x) { logw_ += x; }
    void write(const std::string &filename) const
    {
        std::ofstream f(filename, std::ios::out | std::ios::trunc);
        if (!f) throw Error(AFQMC_ERR_ARG, "cannot write " + filename);
        detail::write_complex(f, logw_);
        f << std::setw(26) << nup_ << "\n" << std::setw(26) << ndn_ << "\n";
        detail::write_matrix(f, wf_);
    }
    void read(const std::string &filename)
    {
        std::ifstream f(filename);
        if (!f) throw Error(AFQMC_ERR_ARG, "cannot read " + filename);
        logw_ = detail::read_complex(f);
        f >> nup_ >> ndn_;
        detail::read_matrix(f, wf_);
    }
    double getMemory() const { return 16.0 * (double)wf_.size() + 16.0 + 8.0; }

private:
    int nup_ = 0, ndn_ = 0;
    Complex logw_ = Complex(0.0, 0.0);
    Matrix wf_;
};

// SD2s (SD2s.h:17-65): the trial, separate up and down matrices.
struct SD2s {
    Complex logw = Complex(0.0, 0.0);
    Matrix wfUp, wfDn;
    int getL() const { return wfUp.rank(0); }
    int getNup() const { return wfUp.rank(1); }
    int getNdn() const { return wfDn.rank(1); }
};

// ---------------------------------------------------------- models, methods
// One-body operators exp(-alpha K) with their log weight (Hop, Hop2is).
struct Hop {
    Matrix matrix;
    Complex logw = Complex(0.0, 0.0);
};

// HubbardSOC (afqmc/model/HubbardRealSpaceSOC/include/HubbardSOC.h): L sites,
// N electrons, 2L x 2L hopping K and the site fields.
struct HubbardSOC {
    int L = 0, N = 0;
    Matrix K;
    std::vector<double> mu, hx, hy, hz, U;
};

// RealMaterialMolecule (afqmc/model/realMaterialMolecule/include/
// realMaterialMolecule.h:28-35): one-body t (n x n, real), Cholesky vectors
// (n x n x G, real, column-major per vector), background (G).
struct RealMaterialMolecule {
    int L = 0, Nup = 0, Ndn = 0, choleskyNumber = 0;
    std::vector<double> t, choleskyVecs, choleskyBg;
    int getL() const { return L; }
    int getNup() const { return Nup; }
    int getNdn() const { return Ndn; }
    int getCholeskyNumber() const { return choleskyNumber; }
};

// The parameters of AfqmcConstraintPathMethod / AfqmcPhaselessMethod that the
// walker step reads.
struct Method {
    double dt = 0.01, ET = 0.0, forceCap = 1.5;
    int mgsStep = 10, popControlStep = 10;
    int walkerSize = 1;
    int forceType = AFQMC_DYNAMIC_FORCE;          // "dynamicForce" / "constForce"
    int decompType = AFQMC_DENSITY_SPIN;          // constrained path only
    int precision = AFQMC_FP64;                   // AFQMC_FP64 or AFQMC_MIXED
    unsigned long long seed = 1;
};

// ------------------------------------------------------------- population
// The whole walker population of one driver, resident on the GPU: replaces
// `std::vector<WalkerRight> walker` + `walkerIsAlive` and the per-walker loops
// of projectOneStep / modifyGM / popControl
// (afqmcConstraintPathProjection.cpp:37-179, afqmcPhaselessProjection.cpp:75-225).
class Population {
public:
    Population(const Population &) = delete;
    Population &operator=(const Population &) = delete;
    Population(Population &&o) noexcept { swap(o); }
    Population &operator=(Population &&o) noexcept
    {
        swap(o);
        return *this;
    }
    ~Population()
    {
        if (e_) afqmc_destroy(e_);
    }

    // Constrained path: SD walkers, HubbardSOC, NiupNidn
    // (AfqmcConstraintPath::initialParameters, afqmcConstraintPath.cpp:20-38).
    static Population constraintPath(const HubbardSOC &model, const Hop &expMinusDtK, const Hop &expHalfDtK,
                                     const Hop &expMinusHalfDtK, const SD &phiT, const Method &m,
                                     const std::vector<double> *constForce = nullptr)
    {
        Population p;
        const int L = model.L;
        if ((int)model.mu.size() != L || (int)model.hx.size() != L || (int)model.hy.size() != L ||
            (int)model.hz.size() != L || (int)model.U.size() != L)
            throw Error(AFQMC_ERR_ARG, "HubbardSOC: field arrays must have L entries");
        check(afqmc_cp_create(L, model.N, m.walkerSize, m.decompType, m.forceType, m.dt, m.ET, m.forceCap,
                              m.mgsStep, m.popControlStep, m.precision, dbl(model.K), dbl(expMinusDtK.matrix),
                              dbl(expHalfDtK.matrix), dbl(expMinusHalfDtK.matrix), model.U.data(),
                              model.mu.data(), model.hx.data(), model.hy.data(), model.hz.data(),
                              constForce ? constForce->data() : nullptr, dbl(phiT.getWf()),
                              phiT.getLogw().real(), phiT.getLogw().imag(), m.seed, &p.e_),
              "afqmc_cp_create");
        p.kind_ = 0;
        p.n_ = 2 * L;
        p.nup_ = model.N;
        p.ndn_ = 0;
        p.ncol_ = model.N;
        p.W_ = m.walkerSize;
        return p;
    }

    // Phaseless: SD2is walkers, SD2s trial, RealMaterialMolecule, CholeskyReal
    // (AfqmcPhaseless::initialParameters, afqmcPhaseless.cpp:32-72).  Dense
    // one-body operators (Hop2is); see phaselessTaylor for the LogHop2is form.
    static Population phaseless(const RealMaterialMolecule &model, const Hop &expMinusDtK,
                                const Hop &expHalfDtK, const Hop &expMinusHalfDtK, const SD2s &phiT,
                                const Method &m, const std::vector<Complex> *constForce = nullptr)
    {
        return makePhaseless(model, &expMinusDtK, expHalfDtK, expMinusHalfDtK, nullptr, phiT, m, constForce);
    }
    // Taylor-series one-body form (LogHop2is of returnLogExpMinusAlphaK,
    // realMaterialMolecule.cpp:134-146): logExpMinusDtK is -dt Kp, and the
    // half-step slots take the LogHop2is matrices of +-dt/2.
    static Population phaselessTaylor(const RealMaterialMolecule &model, const Hop &logExpMinusDtK,
                                      const Hop &logExpHalfDtK, const Hop &logExpMinusHalfDtK,
                                      const SD2s &phiT, const Method &m)
    {
        return makePhaseless(model, nullptr, logExpHalfDtK, logExpMinusHalfDtK, &logExpMinusDtK, phiT, m,
                             nullptr);
    }

    int size() const { return W_; }
    int getL() const { return n_; }
    afqmc_engine *handle() const { return e_; }

    // CUDA stream (a cudaStream_t) for all of this population's work.
    void setStream(void *cudaStream) { check(afqmc_set_stream(e_, cudaStream), "afqmc_set_stream"); }
    void synchronize() { check(afqmc_synchronize(e_), "afqmc_synchronize"); }
    void setCudaGraphs(bool on) { check(afqmc_set_graphs(e_, on ? 1 : 0), "afqmc_set_graphs"); }

    // walkers and walkerIsAlive (initialWalker / readAllWalkers / writeAllWalkers)
    void setWalkers(const std::vector<SD> &w, const std::vector<int> &alive)
    {
        requireKind(0);
        upload(w, alive);
    }
    void setWalkers(const std::vector<SD2is> &w, const std::vector<int> &alive)
    {
        requireKind(1);
        upload(w, alive);
    }
    void getWalkers(std::vector<SD> &w, std::vector<int> &alive)
    {
        requireKind(0);
        download(w, alive);
    }
    void getWalkers(std::vector<SD2is> &w, std::vector<int> &alive)
    {
        requireKind(1);
        download(w, alive);
    }

    // randomHaoInit / randomHaoSave / randomHaoRead (random_hao.cpp:10-71):
    // a counter-based stream, reproducible from (seed, counter).
    void setRandom(unsigned long long seed, unsigned long long counter = 0)
    {
        check(afqmc_set_rng(e_, seed, counter), "afqmc_set_rng");
    }
    std::pair<unsigned long long, unsigned long long> randomState() const
    {
        unsigned long long s = 0, c = 0;
        check(afqmc_get_rng(e_, &s, &c), "afqmc_get_rng");
        return {s, c};
    }
    void setET(double ET) { check(afqmc_set_ET(e_, ET), "afqmc_set_ET"); }
    void setCadence(int mgsIndex, int popControlIndex)
    {
        check(afqmc_set_cadence(e_, mgsIndex, popControlIndex), "afqmc_set_cadence");
    }

    // projectOneStep (x nsteps), projectExpMinusHalfDtK / projectExpHalfDtK,
    // modifyGM, popControl
    void projectOneStep(int nsteps = 1) { check(afqmc_project_one_step(e_, nsteps), "afqmc_project_one_step"); }
    void projectExpMinusHalfDtK() { check(afqmc_project_half(e_, -1), "afqmc_project_half"); }
    void projectExpHalfDtK() { check(afqmc_project_half(e_, +1), "afqmc_project_half"); }
    void modifyGM() { check(afqmc_modify_gm(e_), "afqmc_modify_gm"); }
    // popControl; returns the table (walker i <- walker table[i]) and the weights
    std::vector<int> popControl(std::vector<double> *weights = nullptr)
    {
        std::vector<int> table(W_);
        std::vector<double> w(W_);
        check(afqmc_pop_control(e_, table.data(), w.data()), "afqmc_pop_control");
        if (weights) *weights = std::move(w);
        return table;
    }

    // Background update and propagator replacement
    // (RealMaterialMolecule::updateBackGround, realMaterialMolecule.cpp:103-115)
    void updateBackGround(const std::vector<double> &bg, const Hop &expMinusDtK, const Hop &expHalfDtK,
                          const Hop &expMinusHalfDtK)
    {
        requireKind(1);
        check(afqmc_pl_update_background(e_, bg.data(), dbl(expMinusDtK.matrix), expMinusDtK.logw.real(),
                                         dbl(expHalfDtK.matrix), expHalfDtK.logw.real(),
                                         dbl(expMinusHalfDtK.matrix), expMinusHalfDtK.logw.real()),
              "afqmc_pl_update_background");
    }
    // New background only (updateBackGround); the propagators stay
    void updateBackGround(const std::vector<double> &bg)
    {
        requireKind(1);
        check(afqmc_pl_update_background(e_, bg.data(), nullptr, 0.0, nullptr, 0.0, nullptr, 0.0),
              "afqmc_pl_update_background");
    }
    // expMinusDtK, expMinusHalfDtK, expHalfDtK = model.returnExpMinusAlphaK(dt, dt/2, -dt/2)
    // (afqmcPhaseless.cpp:151-177), built on the GPU from the current
    // background and the model's K (n x n, column-major)
    void rebuildPropagators(const std::vector<double> &K)
    {
        requireKind(1);
        check(afqmc_pl_rebuild_propagators(e_, K.data()), "afqmc_pl_rebuild_propagators");
    }

    // Back-propagation of the constrained path (tutorials/afqmcConstraintPathBP):
    // prepareBackPropagation, the full-window test of the driver loop
    // (BPIndex == backPropagationStep) and addMeasurement.  FP64 form with the
    // observe estimator on (setObservables).
    void setObservables(bool on)
    {
        requireKind(0);
        check(afqmc_cp_set_observables(e_, on ? 1 : 0), "afqmc_cp_set_observables");
    }
    void prepareBackPropagation(int backPropagationStep, int measureSkipStep)
    {
        requireKind(0);
        check(afqmc_cp_bp_begin(e_, backPropagationStep, measureSkipStep), "afqmc_cp_bp_begin");
    }
    bool backPropagationReady(int backPropagationStep) const
    {
        int active = 0, index = 0;
        check(afqmc_cp_bp_state(e_, &active, &index), "afqmc_cp_bp_state");
        return active != 0 && index == backPropagationStep;
    }
    void addBackPropagationMeasurement() { check(afqmc_cp_bp_measure(e_), "afqmc_cp_bp_measure"); }

    // OR of the per-walker status bits (1 singular overlap, 2 non-finite,
    // 4 Taylor order cap, 8 zero column norm, 16 comb, 32 tensor-core wait)
    int status() const
    {
        int s = 0;
        check(afqmc_status(e_, &s), "afqmc_status");
        return s;
    }
    // dynamicOrder statistics (LogHop2isSD2isOperation::print,
    // logHop2isSD2isOperation.cpp:56-88): calls, total order, min, max
    void taylorStatistics(long long &calls, long long &total, int &minOrder, int &maxOrder) const
    {
        check(afqmc_taylor_stats(e_, &calls, &total, &minOrder, &maxOrder), "afqmc_taylor_stats");
    }

    int nup() const { return nup_; }
    int ndn() const { return ndn_; }
    int kind() const { return kind_; }
    int choleskyNumber() const { return G_; }

private:
    Population() = default;
    void swap(Population &o)
    {
        std::swap(e_, o.e_);
        std::swap(kind_, o.kind_);
        std::swap(n_, o.n_);
        std::swap(nup_, o.nup_);
        std::swap(ndn_, o.ndn_);
        std::swap(ncol_, o.ncol_);
        std::swap(W_, o.W_);
        std::swap(G_, o.G_);
    }
    static const double *dbl(const Matrix &m) { return m.size() ? (const double *)m.data() : nullptr; }
    static const double *cdbl(const std::vector<Complex> *v)
    {
        return v ? (const double *)v->data() : nullptr;
    }
    void requireKind(int k) const
    {
        if (kind_ != k)
            throw Error(AFQMC_ERR_ARG, k == 0 ? "SD walkers belong to a constrained-path population"
                                              : "SD2is walkers belong to a phaseless population");
    }
    static Population makePhaseless(const RealMaterialMolecule &model, const Hop *expMinusDtK,
                                    const Hop &half, const Hop &minusHalf, const Hop *logExpMinusDtK,
                                    const SD2s &phiT, const Method &m, const std::vector<Complex> *constForce)
    {
        Population p;
        const size_t n = (size_t)model.L, G = (size_t)model.choleskyNumber;
        if (model.t.size() != n * n || model.choleskyVecs.size() != n * n * G || model.choleskyBg.size() != G)
            throw Error(AFQMC_ERR_ARG, "RealMaterialMolecule: t, choleskyVecs or choleskyBg has the wrong size");
        check(afqmc_pl_create(model.L, model.Nup, model.Ndn, model.choleskyNumber, m.walkerSize, m.forceType,
                              m.dt, m.ET, m.forceCap, m.mgsStep, m.popControlStep, m.precision,
                              model.choleskyVecs.data(), model.choleskyBg.data(), model.t.data(),
                              expMinusDtK ? dbl(expMinusDtK->matrix) : nullptr,
                              expMinusDtK ? expMinusDtK->logw.real() : 0.0, dbl(half.matrix), half.logw.real(),
                              dbl(minusHalf.matrix), minusHalf.logw.real(),
                              logExpMinusDtK ? dbl(logExpMinusDtK->matrix) : nullptr,
                              logExpMinusDtK ? logExpMinusDtK->logw.real() : 0.0, cdbl(constForce),
                              dbl(phiT.wfUp), dbl(phiT.wfDn), phiT.logw.real(), phiT.logw.imag(), m.seed, &p.e_),
              "afqmc_pl_create");
        p.kind_ = 1;
        p.n_ = model.L;
        p.nup_ = model.Nup;
        p.ndn_ = model.Ndn;
        p.ncol_ = model.Nup > model.Ndn ? model.Nup : model.Ndn;
        p.W_ = m.walkerSize;
        p.G_ = model.choleskyNumber;
        return p;
    }
    template <class Walker>
    void upload(const std::vector<Walker> &w, const std::vector<int> &alive)
    {
        if ((int)w.size() != W_ || (int)alive.size() != W_)
            throw Error(AFQMC_ERR_ARG, "setWalkers: need one walker and one alive flag per slot");
        const size_t ws = (size_t)n_ * ncol_;
        std::vector<Complex> wf(ws * W_), logw(W_);
        for (int i = 0; i < W_; ++i) {
            const Matrix &m = w[i].getWf();
            if (m.rank(0) != n_ || m.rank(1) != ncol_) throw Error(AFQMC_ERR_ARG, "setWalkers: walker shape");
            std::copy(m.data(), m.data() + ws, wf.begin() + ws * i);
            logw[i] = w[i].getLogw();
        }
        check(afqmc_set_walkers(e_, (const double *)wf.data(), (const double *)logw.data(), alive.data()),
              "afqmc_set_walkers");
    }
    void shapeWalker(SD &w) const { w.resize(n_, ncol_); }
    void shapeWalker(SD2is &w) const { w.resize(n_, nup_, ndn_); }
    template <class Walker>
    void download(std::vector<Walker> &w, std::vector<int> &alive)
    {
        const size_t ws = (size_t)n_ * ncol_;
        std::vector<Complex> wf(ws * W_), logw(W_);
        alive.assign(W_, 0);
        check(afqmc_get_walkers(e_, (double *)wf.data(), (double *)logw.data(), alive.data()),
              "afqmc_get_walkers");
        w.resize(W_);
        for (int i = 0; i < W_; ++i) {
            shapeWalker(w[i]);
            std::copy(wf.begin() + ws * i, wf.begin() + ws * (i + 1), w[i].wfRef().data());
            w[i].logwRef() = logw[i];
        }
    }

    afqmc_engine *e_ = nullptr;
    int kind_ = -1, n_ = 0, nup_ = 0, ndn_ = 0, ncol_ = 0, W_ = 0, G_ = 0;
};

// ------------------------------------------------------- walker-walker ops
// SDSDOperation / SD2sSD2isOperation (SDSDOperation.h:17-58,
// SD2sSD2isOperation.h:18-64) between the trial and every walker.  The
// reference builds one operation per walker and asks it for returnLogOverlap
// and returnGreenMatrix*; here one call evaluates the whole population.
class WalkerWalkerOperation {
public:
    explicit WalkerWalkerOperation(Population &p) : p_(&p) {}
    // logOverlap of every walker (SDSDOperation.cpp:65-72)
    std::vector<Complex> returnLogOverlaps()
    {
        std::vector<Complex> out(p_->size());
        check(afqmc_log_overlaps(p_->handle(), (double *)out.data()), "afqmc_log_overlaps");
        return out;
    }
    Complex returnLogOverlap(int walker) { return returnLogOverlaps().at(walker); }
    // G = conj(phiT) thetaT of one walker (SDSDOperation.cpp:74-89): the
    // constrained-path G, or the spin-up block of the phaseless walker
    Matrix returnGreenMatrix(int walker) { return green(walker, 0); }
    Matrix returnGreenMatrixUp(int walker) { return green(walker, 0); }
    Matrix returnGreenMatrixDn(int walker) { return green(walker, 1); }

private:
    Matrix green(int walker, int spin)
    {
        Matrix g(p_->getL(), p_->getL());
        check(afqmc_green_matrix(p_->handle(), walker, spin, (double *)g.data()), "afqmc_green_matrix");
        return g;
    }
    Population *p_;
};

// -------------------------------------------------------- mixed estimator
// HubbardSOCMeasureFixedSDSD / RealMaterialMoleculeMeasureFixedSD2sSD2is:
// reSet, addMeasurement over the population (addMixedMeasurement,
// afqmcConstraintPathMeasure.cpp:9-23, afqmcPhaselessMeasure.cpp:9-28),
// returnEnergy = sum HNum / sum den (:58-66), returnCholeskyBg (:68-82).
class ModelMeasureMixed {
public:
    explicit ModelMeasureMixed(Population &p) : p_(&p) {}
    void reSet() { check(afqmc_reset_measurement(p_->handle()), "afqmc_reset_measurement"); }
    void addMixedMeasurement() { check(afqmc_add_mixed_measurement(p_->handle()), "afqmc_add_mixed_measurement"); }
    // den, HNum and (CP) KNum, VNum, RNum | (PL) TNum, 0, 0
    std::vector<Complex> sums() const
    {
        std::vector<Complex> out(5);
        check(afqmc_get_measurement(p_->handle(), (double *)out.data()), "afqmc_get_measurement");
        return out;
    }
    Complex returnEnergy() const
    {
        std::vector<Complex> s = sums();
        return s[1] / s[0];
    }
    Complex returnDenominator() const { return sums()[0]; }
    // choleskyBgNum / den (phaseless): the next background
    std::vector<double> returnCholeskyBg() const
    {
        std::vector<Complex> bg, ex;
        choleskyNums(bg, ex);
        const Complex den = returnDenominator();
        std::vector<double> out(bg.size());
        for (size_t g = 0; g < bg.size(); ++g) out[g] = (bg[g] / den).real();
        return out;
    }
    void choleskyNums(std::vector<Complex> &bgNum, std::vector<Complex> &exNum) const
    {
        if (p_->kind() != 1) throw Error(AFQMC_ERR_ARG, "choleskyNums: phaseless population only");
        bgNum.assign(p_->choleskyNumber(), Complex(0.0, 0.0));
        exNum.assign(p_->choleskyNumber(), Complex(0.0, 0.0));
        check(afqmc_get_cholesky_nums(p_->handle(), (double *)bgNum.data(), (double *)exNum.data()),
              "afqmc_get_cholesky_nums");
    }

private:
    Population *p_;
};

// ------------------------------------------------------ population control
// popConfiguration(size, weight) with explicit uniforms
// (populationControlConfiguration.cpp:24-101): table[i] is the parent of slot
// i; `size` is the number of processes the walkers are spread over.
inline std::vector<int> popConfiguration(int size, const std::vector<double> &weight,
                                         const std::vector<double> &uniforms)
{
    if (weight.size() != uniforms.size()) throw Error(AFQMC_ERR_ARG, "popConfiguration: one uniform per walker");
    std::vector<int> table(weight.size());
    check(afqmc_pop_configuration_host((int)weight.size(), size, weight.data(), uniforms.data(), table.data()),
          "afqmc_pop_configuration_host");
    return table;
}

// popCheck (populationControlConfiguration.cpp:9-22): (min, max, average)
// weight, with the reference's starting values (max from 0, min from 1e20).
inline std::tuple<double, double, double> popCheck(const std::vector<double> &weight)
{
    if (weight.empty()) throw Error(AFQMC_ERR_ARG, "popCheck: no weights");
    double sum = 0.0, maxW = 0.0, minW = 1e20;
    for (double w : weight) sum += w;
    for (double w : weight) {
        if (maxW < w) maxW = w;
        if (minW > w) minW = w;
    }
    return std::make_tuple(minW, maxW, sum / (double)weight.size());
}

}  // namespace afqmclab_b200

#endif  // AFQMCLAB_B200_HPP
