"""Background update and propagator rebuild of the phaseless engine
(RealMaterialMolecule::updateBackGround, realMaterialMolecule.cpp:103-115,
and the rebuild in afqmcPhaseless.cpp:151-177): after
afqmc_pl_update_background with a new background and the dense operators
built from it, the engine must step exactly like an oracle created from the
same new inputs (1e-10 per step from identical walkers), whether it started
in the dense (Hop2is) or the Taylor (LogHop2is) one-body form.  The mixed
form must follow the FP64 form through the same update to mixed-precision
accuracy."""
import numpy as np
import pytest

from afqmclab_b200 import capi, inputs
from oracle import oracle as O
from tests.helpers import logov_close, rel_err
from tests.parity_common import ORACLE_THREADS, STEP_TOL, TRAJ_TOL, compare_state, molecule, pair_pl

pytestmark = pytest.mark.gpu


def new_background(m, scale):
    m2 = molecule(n=m.n, nup=m.nup, ndn=m.ndn, G=m.G)
    m2.set_background(scale * np.cos(np.arange(m2.G)))
    m2.ET = m.ET
    return m2


@pytest.mark.parametrize("log_one_body", [False, True])
def test_update_background_matches_fresh_oracle(log_one_body):
    m = molecule()
    W = 12
    seed = 71
    g, o = pair_pl(m, W, seed, 1000, 1000, log_one_body=log_one_body)
    g.step(2)
    o.step(2)
    compare_state(g, o, TRAJ_TOL)
    m2 = new_background(m, 0.02)
    g.update_background(m2)
    o2 = O.pl_engine(m2, W, seed, 1000, 1000)
    o2.set_threads(ORACLE_THREADS)
    wf, lw, al = o.get_walkers()
    o2.set_walkers(wf, lw, al)
    o2.set_rng(seed, o.rng_counter())
    for _ in range(2):
        wf, lw, al = o2.get_walkers()
        g.set_walkers(wf, lw, al)
        g.set_rng(seed, o2.rng_counter())
        g.step(1)
        o2.step(1)
        compare_state(g, o2, STEP_TOL)
    wf, lw, al = o2.get_walkers()
    g.set_walkers(wf, lw, al)
    for e in (g, o2):
        e.reset_measurement()
        e.add_mixed_measurement()
    assert rel_err(g.measurement()[:3], o2.measurement()[:3]) < STEP_TOL
    bg, eg = g.cholesky_nums()
    bo, eo = o2.cholesky_nums()
    assert rel_err(bg, bo) < STEP_TOL and rel_err(eg, eo) < STEP_TOL


def test_update_background_rejects_partial_switch_from_taylor_form():
    m = molecule()
    g = capi.pl_engine(m, 4, 3, log_one_body=True)
    m2 = new_background(m, 0.02)
    m2.expHalfDtK = None
    with pytest.raises(capi.AfqmcError):
        g.update_background(m2)


def test_mixed_form_follows_fp64_through_update():
    m = inputs.molecule_inputs(64, 16, 16, 128, dt=0.005, decay=30.0, seed=7)
    m.ET = -5.0
    W = 48
    f = capi.pl_engine(m, W, 81, 1000, 1000, precision=capi.AFQMC_FP64)
    x = capi.pl_engine(m, W, 81, 1000, 1000, precision=capi.AFQMC_MIXED)
    wf, lw, al = inputs.initial_walkers(m.phiTUp, W, seed=82, noise=0.02)
    f.set_walkers(wf, lw, al)
    x.set_walkers(wf, lw, al)
    f.step(1)
    x.step(1)
    m2 = inputs.molecule_inputs(64, 16, 16, 128, dt=0.005, decay=30.0, seed=7)
    m2.set_background(0.05 * np.cos(np.arange(m2.G)))
    m2.ET = m.ET
    f.update_background(m2)
    x.update_background(m2)
    wf, lw, al = f.get_walkers()
    f.set_walkers(wf, lw, al)
    x.set_walkers(wf, lw, al)
    f.step(1)
    x.step(1)
    _, _, af = f.get_walkers()
    _, _, ax = x.get_walkers()
    assert (af == ax).all()
    a = af.astype(bool)
    lf, lx = f.log_overlaps(), x.log_overlaps()
    assert np.abs(lf[a].real - lx[a].real).max() < 2e-2
    assert np.abs(np.exp(1j * lf[a].imag) - np.exp(1j * lx[a].imag)).max() < 2e-2
    for e in (f, x):
        e.reset_measurement()
        e.add_mixed_measurement()
    mf, mx = f.measurement(), x.measurement()
    assert abs(mf[1] / mf[0] - mx[1] / mx[0]) < 2e-3 * abs(mf[1] / mf[0])
    assert x.status() == 0


# ---------------------------------------------------------------------------
# The propagator rebuild on the GPU (afqmc_pl_rebuild_propagators) against
# the eigensystem route of the reference (returnExpMinusAlphaK,
# realMaterialMolecule.cpp:117-131, here host numpy eigh of Kp): the two
# engines hold the same background, one receives the operators built on the
# host, the other rebuilds them itself from K.  project_half(+1 / -1)
# applies expHalfDtK / expMinusHalfDtK with no random numbers; steps then
# exercise expMinusDtK and the log-weights.  dt = 0.4 makes ||dt Kp|| large
# enough that the series is scaled and squared.

def _rebuilt_pair(m, m2, W, seed, log_one_body, precision):
    host = capi.pl_engine(m, W, seed, 1000, 1000, log_one_body=log_one_body, precision=precision)
    dev = capi.pl_engine(m, W, seed, 1000, 1000, log_one_body=log_one_body, precision=precision)
    host.update_background(m2)
    dev.update_background_only(m2.bg)
    dev.rebuild_propagators(m2.K)
    return host, dev


def _same_walkers(a, b, tol):
    wa, la, aa = a.get_walkers()
    wb, lb, ab = b.get_walkers()
    assert (aa == ab).all()
    assert rel_err(wb, wa) < tol
    assert np.abs(lb - la).max() < tol * max(1.0, np.abs(la).max())


@pytest.mark.parametrize("log_one_body,dt", [(False, 0.01), (True, 0.01), (False, 0.4)])
def test_gpu_rebuild_matches_eigensystem_route(log_one_body, dt):
    m = molecule()
    m.dt = dt
    m.set_background(m.bg)
    m2 = molecule()
    m2.dt = dt
    m2.set_background(0.02 * np.cos(np.arange(m2.G)))
    m2.ET = m.ET
    W, seed = 10, 91
    host, dev = _rebuilt_pair(m, m2, W, seed, log_one_body, capi.AFQMC_FP64)
    wf, lw, al = inputs.initial_walkers(m.phiTUp, W, seed=seed + 1, noise=0.05)
    for which in (+1, -1):
        for e in (host, dev):
            e.set_walkers(wf, lw, al)
            e.project_half(which)
        _same_walkers(host, dev, 1e-12)
    if dt > 0.1:
        return
    for e in (host, dev):
        e.set_walkers(wf, lw, al)
        e.set_rng(seed, 0)
        e.step(3)
    assert host.rng_counter() == dev.rng_counter()
    _same_walkers(host, dev, 1e-10)
    for e in (host, dev):
        e.reset_measurement()
        e.add_mixed_measurement()
    assert rel_err(dev.measurement()[:3], host.measurement()[:3]) < STEP_TOL


def test_gpu_rebuild_mixed_form():
    m = inputs.molecule_inputs(64, 16, 16, 128, dt=0.005, decay=30.0, seed=7)
    m.ET = -5.0
    m2 = inputs.molecule_inputs(64, 16, 16, 128, dt=0.005, decay=30.0, seed=7)
    m2.set_background(0.05 * np.cos(np.arange(m2.G)))
    m2.ET = m.ET
    W, seed = 48, 83
    host, dev = _rebuilt_pair(m, m2, W, seed, False, capi.AFQMC_MIXED)
    wf, lw, al = inputs.initial_walkers(m.phiTUp, W, seed=seed + 1, noise=0.02)
    for e in (host, dev):
        e.set_walkers(wf, lw, al)
        e.set_rng(seed, 0)
        e.step(2)
    # the same tf32/bf16 operators up to the last bits of exp(-dt Kp)
    _same_walkers(host, dev, 1e-5)
    assert dev.status() == 0
