"""The phaseless step at the headline shape against the oracle: n=128
orbitals, 32+32 electrons, G=640 Cholesky vectors, dt=0.005, the seeded
synthetic molecule (eigenvalues of h1 spaced on [-5, 5] Ha, Cholesky
spectrum exp(-g/60), RHF trial from the lowest 32 h1 orbitals).

Plain FP64 form, per step from identical walkers and random stream, 1e-10
relative: log-overlaps, Green's functions of both spins, the population-
control weights (bit-exact table), the mixed-estimator sums den, HNum, TNum
and the per-vector sums choleskyBgNum / choleskyExNum
(afqmcPhaselessProjection.cpp:75-121,
realMaterialMoleculeMeasureFixedSD2sSD2is.cpp:197-284).

Mixed-precision form (bf16/tf32 tensor-core contractions, FP64 LU /
log-det / weights / Gram-Schmidt) against the same oracle:
  - after one step from identical walkers, log-overlaps within 2e-2
    (real part) and phases within 2e-2;
  - the mixed-estimator energy, paired measurement by measurement over a
    short trajectory (same walkers, same random stream), within 0.5 mHa of
    the oracle's.
"""
import numpy as np
import pytest

from afqmclab_b200 import capi, inputs
from oracle import oracle as O
from tests.helpers import logov_close, rel_err
from tests.parity_common import ORACLE_THREADS, STEP_TOL, compare_state

pytestmark = pytest.mark.gpu

ENERGY_CRITERION_HA = 0.5e-3


@pytest.fixture(scope="module")
def headline():
    m = inputs.molecule_inputs(128, 32, 32, 640, dt=0.005)
    return m


def pair(m, W, seed, mgs, pop, precision, noise):
    g = capi.pl_engine(m, W, seed, mgs, pop, precision=precision)
    o = O.pl_engine(m, W, seed, mgs, pop)
    o.set_threads(ORACLE_THREADS)
    wf, lw, al = inputs.initial_walkers(m.phiTUp, W, seed=seed + 1, noise=noise)
    g.set_walkers(wf, lw, al)
    o.set_walkers(wf, lw, al)
    return g, o


def test_fp64_form_step_measure_and_pop_control(headline):
    m = headline
    W = 6
    seed = 4101
    g, o = pair(m, W, seed, 1000, 1000, capi.AFQMC_FP64, noise=0.05)
    assert logov_close(g.log_overlaps(), o.log_overlaps(), STEP_TOL) < STEP_TOL
    for w in (0, W - 1):
        for spin in (0, 1):
            assert rel_err(g.green(w, spin), o.green(w, spin)) < STEP_TOL
    for _ in range(2):
        wf, lw, al = o.get_walkers()
        g.set_walkers(wf, lw, al)
        g.set_rng(seed, o.rng_counter())
        g.step(1)
        o.step(1)
        compare_state(g, o, STEP_TOL)
    wf, lw, al = o.get_walkers()
    g.set_walkers(wf, lw, al)
    for e in (g, o):
        e.reset_measurement()
        e.add_mixed_measurement()
    mg, mo = g.measurement(), o.measurement()
    assert rel_err(mg[:3], mo[:3]) < STEP_TOL
    bg, eg = g.cholesky_nums()
    bo, eo = o.cholesky_nums()
    assert rel_err(bg, bo) < STEP_TOL
    assert rel_err(eg, eo) < STEP_TOL
    g.set_rng(seed, o.rng_counter())
    tg, wg = g.pop_control()
    to, wo = o.pop_control()
    assert rel_err(wg, wo) < STEP_TOL
    assert (tg == to).all()
    compare_state(g, o, STEP_TOL)


def test_fp64_form_stabilize(headline):
    m = headline
    W = 4
    g, o = pair(m, W, 4102, 1000, 1000, capi.AFQMC_FP64, noise=0.2)
    g.modify_gm()
    o.modify_gm()
    compare_state(g, o, STEP_TOL)
    for spin in (0, 1):
        assert rel_err(g.green(1, spin), o.green(1, spin)) < STEP_TOL


def test_mixed_form_one_step(headline):
    m = headline
    W = 32
    g, o = pair(m, W, 4103, 1000, 1000, capi.AFQMC_MIXED, noise=0.02)
    assert logov_close(g.log_overlaps(), o.log_overlaps(), 1e-5) < 1e-5
    g.step(1)
    o.step(1)
    _, _, ag = g.get_walkers()
    _, _, ao = o.get_walkers()
    assert (ag == ao).all()
    assert g.rng_counter() == o.rng_counter()
    lg, lo = g.log_overlaps(), o.log_overlaps()
    a = ao.astype(bool)
    assert np.abs(lg[a].real - lo[a].real).max() < 2e-2
    assert np.abs(np.exp(1j * lg[a].imag) - np.exp(1j * lo[a].imag)).max() < 2e-2
    assert g.status() == 0


def test_mixed_form_energy_within_half_mha_of_oracle(headline):
    """Paired mixed-estimator energies: both sides start from the same
    walkers and random stream; modifyGM every 5 steps; one measurement
    (afqmcPhaselessMeasure.cpp:9-28) every 5 steps over 15 steps."""
    m = headline
    W = 48
    g, o = pair(m, W, 4104, 5, 1000, capi.AFQMC_MIXED, noise=0.0)
    eg, eo = [], []
    for step in range(16):
        if step % 5 == 0:
            for e, acc in ((g, eg), (o, eo)):
                e.reset_measurement()
                e.add_mixed_measurement()
                mm = e.measurement()
                acc.append((mm[1] / mm[0]).real)
        if step < 15:
            g.step(1)
            o.step(1)
    d = np.abs(np.array(eg) - np.array(eo))
    assert d.max() <= ENERGY_CRITERION_HA, (eg, eo)
    assert g.status() == 0
