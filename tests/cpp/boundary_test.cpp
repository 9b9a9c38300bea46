// C++ caller of the engine through include/afqmclab_b200.hpp, the way a
// reference driver binds it (compiled with g++ and run by
// tests/test_cpp_boundary.py).
//
//   boundary_test cpu <dir>     argument errors, walker files, popCheck and
//                               popConfiguration against <dir>/pop_*.bin
//   boundary_test pl <dir>      phaseless population from <dir>: upload, steps,
//                               measurement; results written to <dir>/out_*.bin
//   boundary_test cp <dir>      the same for a constrained-path population
//
// Inputs are raw little-endian arrays (double; complex as (re, im) pairs) and
// a params.txt of whitespace-separated numbers.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "afqmclab_b200.hpp"

using namespace afqmclab_b200;

namespace {

int failures = 0;
#define EXPECT(cond)                                                              \
    do {                                                                          \
        if (!(cond)) {                                                            \
            std::cerr << __FILE__ << ":" << __LINE__ << ": failed: " #cond "\n"; \
            ++failures;                                                           \
        }                                                                         \
    } while (0)

template <class T>
std::vector<T> load(const std::string &path)
{
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) throw std::runtime_error("cannot open " + path);
    const std::streamsize bytes = f.tellg();
    f.seekg(0);
    std::vector<T> v((size_t)bytes / sizeof(T));
    f.read((char *)v.data(), bytes);
    return v;
}

template <class T>
void save(const std::string &path, const std::vector<T> &v)
{
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    f.write((const char *)v.data(), (std::streamsize)(v.size() * sizeof(T)));
}

Matrix matrix(const std::vector<Complex> &v, int r, int c)
{
    if (v.size() != (size_t)r * c) throw std::runtime_error("matrix size");
    Matrix m(r, c);
    std::copy(v.begin(), v.end(), m.data());
    return m;
}

std::vector<double> params(const std::string &dir)
{
    std::ifstream f(dir + "/params.txt");
    std::vector<double> p;
    double x;
    while (f >> x) p.push_back(x);
    return p;
}

template <class F>
int expect_error(F &&f)
{
    try {
        f();
    } catch (const Error &e) {
        return e.code();
    }
    return 0;
}

// ------------------------------------------------------------------ cpu
int run_cpu(const std::string &dir)
{
    // argument errors are reported as such, with or without a GPU
    HubbardSOC hub;
    hub.L = 4;
    hub.N = 3;
    hub.K.resize(8, 8);
    hub.mu = hub.hx = hub.hy = hub.hz = hub.U = std::vector<double>(4, 0.0);
    Hop h;
    h.matrix.resize(8, 8);
    SD trial(8, 3);
    Method m;
    m.walkerSize = 0;
    EXPECT(expect_error([&] { Population::constraintPath(hub, h, h, h, trial, m); }) == AFQMC_ERR_ARG);
    m.walkerSize = 4;
    m.mgsStep = 0;
    EXPECT(expect_error([&] { Population::constraintPath(hub, h, h, h, trial, m); }) == AFQMC_ERR_ARG);
    m.mgsStep = 10;
    m.precision = 7;
    EXPECT(expect_error([&] { Population::constraintPath(hub, h, h, h, trial, m); }) == AFQMC_ERR_ARG);
    m.precision = AFQMC_FP64;
    hub.U.resize(3);
    EXPECT(expect_error([&] { Population::constraintPath(hub, h, h, h, trial, m); }) == AFQMC_ERR_ARG);
    hub.U.resize(4);
    hub.N = 9;   // more electrons than spin orbitals
    EXPECT(expect_error([&] { Population::constraintPath(hub, h, h, h, trial, m); }) == AFQMC_ERR_ARG);
    hub.N = 3;
    RealMaterialMolecule mol;
    mol.L = 6;
    mol.Nup = 2;
    mol.Ndn = 2;
    mol.choleskyNumber = 3;
    mol.t.assign(36, 0.0);
    mol.choleskyVecs.assign(10, 0.0);   // wrong size
    mol.choleskyBg.assign(3, 0.0);
    SD2s t2;
    t2.wfUp.resize(6, 2);
    t2.wfDn.resize(6, 2);
    Hop h6;
    h6.matrix.resize(6, 6);
    EXPECT(expect_error([&] { Population::phaseless(mol, h6, h6, h6, t2, m); }) == AFQMC_ERR_ARG);
    // a valid population: created on a GPU machine, AFQMC_ERR_CUDA without one
    const int rc = expect_error([&] { Population p = Population::constraintPath(hub, h, h, h, trial, m); });
    EXPECT(rc == 0 || rc == AFQMC_ERR_CUDA);

    // walker files in the reference's formats round-trip exactly
    SD w(5, 2);
    SD2is w2(5, 3, 2);
    for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 5; ++i) w.wfRef()(i, j) = Complex(0.1 * i - 0.3 * j, 1.0 / (1 + i + j));
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 5; ++i) w2.wfRef()(i, j) = Complex(std::sin(i + 7 * j), std::cos(3 * i - j));
    w.logwRef() = Complex(-1.25, 0.5);
    w2.logwRef() = Complex(3.0e-7, -2.5);
    w.write(dir + "/sd.dat");
    w2.write(dir + "/sd2is.dat");
    SD r;
    SD2is r2;
    r.read(dir + "/sd.dat");
    r2.read(dir + "/sd2is.dat");
    EXPECT(r.getL() == 5 && r.getN() == 2 && r.getLogw() == w.getLogw());
    EXPECT(r2.getL() == 5 && r2.getNup() == 3 && r2.getNdn() == 2 && r2.getLogw() == w2.getLogw());
    for (size_t k = 0; k < w.getWf().size(); ++k) EXPECT(r.getWf().data()[k] == w.getWf().data()[k]);
    for (size_t k = 0; k < w2.getWf().size(); ++k) EXPECT(r2.getWf().data()[k] == w2.getWf().data()[k]);

    // popCheck and popConfiguration
    const std::vector<double> wts = load<double>(dir + "/pop_weights.bin");
    const std::vector<double> uni = load<double>(dir + "/pop_uniforms.bin");
    const std::vector<int> expect = load<int>(dir + "/pop_table.bin");
    const std::vector<int> expect2 = load<int>(dir + "/pop_table_size2.bin");
    double mn, mx, avg;
    std::tie(mn, mx, avg) = popCheck(wts);
    double s = 0;
    for (double x : wts) s += x;
    EXPECT(mx >= mn && std::fabs(avg - s / wts.size()) < 1e-15);
    EXPECT(popConfiguration(1, wts, uni) == expect);
    EXPECT(popConfiguration(2, wts, uni) == expect2);
    EXPECT(expect_error([&] { popConfiguration(3, wts, uni); }) == AFQMC_ERR_ARG);   // size must divide W
    std::cout << (failures ? "FAILED" : "cpu ok") << "\n";
    return failures ? 1 : 0;
}

// --------------------------------------------------------------- phaseless
int run_pl(const std::string &dir)
{
    const std::vector<double> p = params(dir);
    const int n = (int)p[0], nup = (int)p[1], ndn = (int)p[2], G = (int)p[3], W = (int)p[4];
    Method m;
    m.dt = p[5];
    m.ET = p[6];
    m.forceCap = p[7];
    m.mgsStep = (int)p[8];
    m.popControlStep = (int)p[9];
    m.seed = (unsigned long long)p[10];
    const int nsteps = (int)p[11];
    m.walkerSize = W;
    m.precision = (int)p[14];
    RealMaterialMolecule mol;
    mol.L = n;
    mol.Nup = nup;
    mol.Ndn = ndn;
    mol.choleskyNumber = G;
    mol.t = load<double>(dir + "/t.bin");
    mol.choleskyVecs = load<double>(dir + "/chol.bin");
    mol.choleskyBg = load<double>(dir + "/bg.bin");
    Hop eK, eH, eMH;
    eK.matrix = matrix(load<Complex>(dir + "/expMinusDtK.bin"), n, n);
    eK.logw = p[12];
    eH.matrix = matrix(load<Complex>(dir + "/expHalfDtK.bin"), n, n);
    eH.logw = -p[13];
    eMH.matrix = matrix(load<Complex>(dir + "/expMinusHalfDtK.bin"), n, n);
    eMH.logw = p[13];
    SD2s trial;
    trial.wfUp = matrix(load<Complex>(dir + "/phiTUp.bin"), n, nup);
    trial.wfDn = matrix(load<Complex>(dir + "/phiTDn.bin"), n, ndn);
    Population pop = Population::phaseless(mol, eK, eH, eMH, trial, m);

    // walkers: SD2is objects, as the driver's std::vector<WalkerRight>
    const std::vector<Complex> wf = load<Complex>(dir + "/wf.bin");
    const std::vector<Complex> lw = load<Complex>(dir + "/logw.bin");
    const int ncol = nup > ndn ? nup : ndn;
    std::vector<SD2is> walkers(W);
    std::vector<int> alive(W, 1);
    for (int i = 0; i < W; ++i) {
        walkers[i].resize(n, nup, ndn);
        std::copy(wf.begin() + (size_t)n * ncol * i, wf.begin() + (size_t)n * ncol * (i + 1),
                  walkers[i].wfRef().data());
        walkers[i].logwRef() = lw[i];
    }
    pop.setWalkers(walkers, alive);
    // a walker written and read back in the reference's file format
    walkers[0].write(dir + "/phi_0.dat");
    SD2is back;
    back.read(dir + "/phi_0.dat");
    EXPECT(back.getNup() == nup && back.getNdn() == ndn && back.getWf().data()[3] == walkers[0].getWf().data()[3]);

    ModelMeasureMixed meas(pop);
    WalkerWalkerOperation op(pop);
    pop.modifyGM();
    pop.projectOneStep(nsteps);
    meas.reSet();
    meas.addMixedMeasurement();
    const std::vector<Complex> sums = meas.sums();
    std::vector<Complex> bgNum, exNum;
    meas.choleskyNums(bgNum, exNum);
    const std::vector<Complex> lo = op.returnLogOverlaps();
    EXPECT(lo[1] == op.returnLogOverlap(1));
    const Matrix g0 = op.returnGreenMatrixDn(0);
    std::vector<int> table = pop.popControl();
    std::vector<SD2is> after;
    pop.getWalkers(after, alive);
    EXPECT((int)after.size() == W && after[0].getNup() == nup);
    long long calls = 0, total = 0;
    int mno = 0, mxo = 0;
    pop.taylorStatistics(calls, total, mno, mxo);
    EXPECT(calls > 0 && mno >= 3 && mxo >= mno);
    EXPECT(pop.status() == 0);
    save(dir + "/out_sums.bin", sums);
    save(dir + "/out_bgnum.bin", bgNum);
    save(dir + "/out_logov.bin", lo);
    save(dir + "/out_green.bin", std::vector<Complex>(g0.data(), g0.data() + g0.size()));
    save(dir + "/out_table.bin", table);
    std::vector<Complex> wfo;
    for (const SD2is &w : after) wfo.insert(wfo.end(), w.getWf().data(), w.getWf().data() + w.getWf().size());
    save(dir + "/out_wf.bin", wfo);
    std::cout << (failures ? "FAILED" : "pl ok") << " E=" << meas.returnEnergy() << "\n";
    return failures ? 1 : 0;
}

// ---------------------------------------------------------- constrained path
int run_cp(const std::string &dir)
{
    const std::vector<double> p = params(dir);
    const int L = (int)p[0], N = (int)p[1], W = (int)p[2];
    Method m;
    m.dt = p[3];
    m.ET = p[4];
    m.forceCap = p[5];
    m.mgsStep = (int)p[6];
    m.popControlStep = (int)p[7];
    m.seed = (unsigned long long)p[8];
    const int nsteps = (int)p[9];
    m.decompType = (int)p[10];
    m.walkerSize = W;
    HubbardSOC hub;
    hub.L = L;
    hub.N = N;
    hub.K = matrix(load<Complex>(dir + "/K.bin"), 2 * L, 2 * L);
    hub.U = load<double>(dir + "/U.bin");
    hub.mu = load<double>(dir + "/mu.bin");
    hub.hx = load<double>(dir + "/hx.bin");
    hub.hy = load<double>(dir + "/hy.bin");
    hub.hz = load<double>(dir + "/hz.bin");
    Hop eK, eH, eMH;
    eK.matrix = matrix(load<Complex>(dir + "/expMinusDtK.bin"), 2 * L, 2 * L);
    eH.matrix = matrix(load<Complex>(dir + "/expHalfDtK.bin"), 2 * L, 2 * L);
    eMH.matrix = matrix(load<Complex>(dir + "/expMinusHalfDtK.bin"), 2 * L, 2 * L);
    SD trial;
    trial.wfRef() = matrix(load<Complex>(dir + "/phiT.bin"), 2 * L, N);
    Population pop = Population::constraintPath(hub, eK, eH, eMH, trial, m);
    const std::vector<Complex> wf = load<Complex>(dir + "/wf.bin");
    std::vector<SD> walkers(W);
    std::vector<int> alive(W, 1);
    for (int i = 0; i < W; ++i) {
        walkers[i].resize(2 * L, N);
        std::copy(wf.begin() + (size_t)2 * L * N * i, wf.begin() + (size_t)2 * L * N * (i + 1),
                  walkers[i].wfRef().data());
    }
    pop.setWalkers(walkers, alive);
    EXPECT(expect_error([&] {
               std::vector<SD2is> wrong(W);
               pop.setWalkers(wrong, alive);
           }) == AFQMC_ERR_ARG);
    ModelMeasureMixed meas(pop);
    WalkerWalkerOperation op(pop);
    pop.projectOneStep(nsteps);
    meas.reSet();
    meas.addMixedMeasurement();
    const std::vector<Complex> sums = meas.sums();
    const std::vector<Complex> lo = op.returnLogOverlaps();
    const Matrix g0 = op.returnGreenMatrix(0);
    EXPECT(pop.status() == 0);
    save(dir + "/out_sums.bin", sums);
    save(dir + "/out_logov.bin", lo);
    save(dir + "/out_green.bin", std::vector<Complex>(g0.data(), g0.data() + g0.size()));
    std::cout << (failures ? "FAILED" : "cp ok") << " E=" << meas.returnEnergy() << "\n";
    return failures ? 1 : 0;
}

}  // namespace

int main(int argc, char **argv)
{
    if (argc < 3) {
        std::cerr << "usage: boundary_test cpu|pl|cp <dir>\n";
        return 2;
    }
    const std::string mode = argv[1], dir = argv[2];
    try {
        if (mode == "cpu") return run_cpu(dir);
        if (mode == "pl") return run_pl(dir);
        if (mode == "cp") return run_cp(dir);
    } catch (const std::exception &e) {
        std::cerr << "exception: " << e.what() << "\n";
        return 3;
    }
    std::cerr << "unknown mode " << mode << "\n";
    return 2;
}
