"""Observe estimator of the constrained path (HubbardSOCMeasureObserveSDSD,
HubbardSOCMeasureObserveSDSD.cpp:42-185) on the GPU against the oracle:
den-weighted greenMatrixNum and densityDensityNum (2L x 2L),
splusSminusNum, sminusSplusNum and spairSpairNum (L x L), accumulated over
two measurements of identical walkers, to 1e-10 of the largest entry; the
mixed-precision form (whose measurement runs on an FP64 copy) against the
FP64 form to fp32 accuracy."""
import numpy as np
import pytest

from afqmclab_b200 import capi, inputs
from tests.parity_common import hubbard, pair_cp

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _check(og, oo, tol):
    for k in oo:
        scale = max(1.0, np.abs(oo[k]).max())
        assert np.abs(og[k] - oo[k]).max() < tol * scale, k


@pytest.mark.parametrize("nx,ny,nup,ndn,fields", [(4, 4, 7, 7, True), (6, 6, 14, 13, False)])
def test_observables_match_oracle(nx, ny, nup, ndn, fields):
    m = hubbard("densitySpin", fields, nx=nx, ny=ny, nup=nup, ndn=ndn)
    W = 10
    g, o = pair_cp(m, W, 61, 1000, 1000, noise=0.05)
    g.step(2)
    o.step(2)
    wf, lw, al = o.get_walkers()
    g.set_walkers(wf, lw, al)
    for e in (g, o):
        e.set_observables(True)
        e.reset_measurement()
        e.add_mixed_measurement()
    g.step(1)
    o.step(1)
    wf, lw, al = o.get_walkers()
    g.set_walkers(wf, lw, al)
    for e in (g, o):
        e.add_mixed_measurement()
    og, oo = g.observables(), o.observables()
    _check(og, oo, TOL)
    den = g.measurement()[0]
    assert abs(np.trace(og["greenMatrixNum"]) / den - m.N) < 1e-9
    # diag(densityDensity) = diag(G): n_i^2 = n_i
    assert np.abs(np.diag(og["densityDensityNum"]) - np.diag(og["greenMatrixNum"])).max() < 1e-12 * abs(den)


def test_observables_mixed_form_follow_fp64():
    m = hubbard("densitySpin", False, nx=4, ny=4, nup=7, ndn=7)
    W = 16
    f = capi.cp_engine(m, W, 7, 1000, 1000, "constForce")
    x = capi.cp_engine(m, W, 7, 1000, 1000, "constForce", precision=capi.AFQMC_MIXED)
    wf, lw, al = inputs.initial_walkers(m.phiT, W, seed=8, noise=0.05)
    for e in (f, x):
        e.set_walkers(wf, lw, al)
        e.set_observables(True)
        e.step(2)
        e.reset_measurement()
        e.add_mixed_measurement()
    _check(x.observables(), f.observables(), 1e-4)
