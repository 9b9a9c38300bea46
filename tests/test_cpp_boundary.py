"""The C++ face of the boundary (include/afqmclab_b200.hpp): tests/cpp/
boundary_test.cpp is compiled with g++ against libafqmc_b200.so and run.

  - CPU (no GPU needed): argument errors are reported as AFQMC_ERR_ARG before
    any device work, a valid population is created or refused with
    AFQMC_ERR_CUDA, SD / SD2is walker files round-trip in the reference's
    text format, and popCheck / popConfiguration agree with the oracle's comb
    (populationControlConfiguration.cpp:9-101) for one and two processes.
  - GPU: a phaseless and a constrained-path population created, filled,
    stepped and measured through the C++ classes give the same log-overlaps,
    Green's function, estimator sums, population-control table and walkers
    as the same calls through the ctypes binding (same library, same inputs:
    agreement to 1e-12).
"""
import os
import subprocess

import numpy as np
import pytest

from afqmclab_b200 import build, capi, inputs
from oracle import oracle as O
from tests.helpers import rel_err

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "boundary_test.cpp")
INC = os.path.join(ROOT, "include")


def compile_test(tmp):
    build.build()
    libdir = os.path.dirname(build.LIB)
    exe = os.path.join(tmp, "boundary_test")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", INC, SRC, "-o", exe,
           "-L", libdir, "-lafqmc_b200", "-Wl,-rpath," + libdir, "-Wl,--allow-shlib-undefined"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def run(exe, mode, d):
    r = subprocess.run([exe, mode, str(d)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def save(d, name, a):
    np.ascontiguousarray(a).tofile(os.path.join(d, name))


def load(d, name, dtype):
    return np.fromfile(os.path.join(d, name), dtype=dtype)


def test_cpp_layer_cpu(tmp_path):
    exe = compile_test(str(tmp_path))
    rng = np.random.default_rng(11)
    W = 40
    w = rng.uniform(0, 2, W)
    w[rng.uniform(size=W) < 0.2] = 0.0
    u = rng.uniform(size=W)
    save(tmp_path, "pop_weights.bin", w)
    save(tmp_path, "pop_uniforms.bin", u)
    save(tmp_path, "pop_table.bin", O.pop_configuration(w, u, size=1)[0].astype(np.int32))
    save(tmp_path, "pop_table_size2.bin", O.pop_configuration(w, u, size=2)[0].astype(np.int32))
    assert "cpu ok" in run(exe, "cpu", tmp_path)
    # the walker files the C++ layer writes are the ones the Python side reads
    wf, lw = inputs.read_sd(os.path.join(tmp_path, "sd.dat"))
    assert wf.shape == (5, 2) and lw == complex(-1.25, 0.5)


@pytest.mark.gpu
def test_cpp_layer_phaseless_matches_ctypes(tmp_path):
    exe = compile_test(str(tmp_path))
    m = inputs.molecule_inputs(32, 8, 6, 48, dt=0.01, decay=6.0)
    m.ET = -3.0
    W, seed, nsteps = 16, 123, 3
    wf, lw, al = inputs.initial_walkers(m.phiTUp, W, seed=5, noise=0.05)
    d = str(tmp_path)
    save(d, "t.bin", np.asfortranarray(m.t).ravel(order="F"))
    save(d, "chol.bin", np.asfortranarray(m.chol).ravel(order="F"))
    save(d, "bg.bin", m.bg)
    for k in ("expMinusDtK", "expHalfDtK", "expMinusHalfDtK", "phiTUp", "phiTDn"):
        save(d, k + ".bin", np.asarray(getattr(m, k), np.complex128).ravel(order="F"))
    save(d, "wf.bin", wf.ravel(order="F"))
    save(d, "logw.bin", lw)
    with open(os.path.join(d, "params.txt"), "w") as f:
        f.write(" ".join(repr(float(x)) for x in (m.n, m.nup, m.ndn, m.G, W, m.dt, m.ET, m.force_cap,
                                                   10, 10, seed, nsteps, m.logwDt, m.logwHalf,
                                                   capi.AFQMC_FP64)))
    assert "pl ok" in run(exe, "pl", d)
    g = capi.pl_engine(m, W, seed, 10, 10)
    g.set_walkers(wf, lw, al)
    g.modify_gm()
    g.step(nsteps)
    g.reset_measurement()
    g.add_mixed_measurement()
    assert rel_err(load(d, "out_sums.bin", np.complex128)[:3], g.measurement()[:3]) < 1e-12
    assert rel_err(load(d, "out_bgnum.bin", np.complex128), g.cholesky_nums()[0]) < 1e-12
    assert rel_err(load(d, "out_logov.bin", np.complex128), g.log_overlaps()) < 1e-12
    gr = load(d, "out_green.bin", np.complex128).reshape((m.n, m.n), order="F")
    assert rel_err(gr, g.green(0, 1)) < 1e-12
    table, _ = g.pop_control()
    assert np.array_equal(load(d, "out_table.bin", np.int32), table)
    wg, _, _ = g.get_walkers()
    wc = load(d, "out_wf.bin", np.complex128).reshape(wg.shape, order="F")
    assert rel_err(wc, wg) < 1e-12


@pytest.mark.gpu
def test_cpp_layer_constrained_path_matches_ctypes(tmp_path):
    exe = compile_test(str(tmp_path))
    m = inputs.hubbard_inputs(4, 4, 7, 7)
    m.ET = -12.0
    W, seed, nsteps = 12, 321, 4
    wf, lw, al = inputs.initial_walkers(m.phiT, W, seed=6, noise=0.05)
    d = str(tmp_path)
    for k in ("K", "expMinusDtK", "expHalfDtK", "expMinusHalfDtK", "phiT"):
        save(d, k + ".bin", np.asarray(getattr(m, k), np.complex128).ravel(order="F"))
    for k in ("U", "mu", "hx", "hy", "hz"):
        save(d, k + ".bin", np.asarray(getattr(m, k), np.float64))
    save(d, "wf.bin", wf.ravel(order="F"))
    with open(os.path.join(d, "params.txt"), "w") as f:
        f.write(" ".join(repr(float(x)) for x in (m.L, m.N, W, m.dt, m.ET, m.force_cap, 10, 40, seed,
                                                   nsteps, capi.DECOMP[m.decomp])))
    assert "cp ok" in run(exe, "cp", d)
    g = capi.cp_engine(m, W, seed, 10, 40)
    g.set_walkers(wf, lw, al)
    g.step(nsteps)
    g.reset_measurement()
    g.add_mixed_measurement()
    assert rel_err(load(d, "out_sums.bin", np.complex128), g.measurement()) < 1e-12
    assert rel_err(load(d, "out_logov.bin", np.complex128), g.log_overlaps()) < 1e-12
    gr = load(d, "out_green.bin", np.complex128).reshape((m.n, m.n), order="F")
    assert rel_err(gr, g.green(0)) < 1e-12
