"""Uneven batch: Hubbard lattices of different size and filling advanced as
one graph launch per step give the same populations as each engine stepped
alone; the GEMM autotuner changes tile shapes, not results."""
import numpy as np
import pytest

from afqmclab_b200 import capi, inputs

pytestmark = pytest.mark.gpu

LATTICES = [(4, 4, 7, 7, 4.0), (6, 6, 16, 16, 8.0), (8, 8, 28, 28, 4.0)]
W = 48


def _engines(precision=capi.AFQMC_FP64):
    out = []
    for k, (nx, ny, nu, nd, U) in enumerate(LATTICES):
        m = inputs.hubbard_inputs(nx, ny, nu, nd, t=1.0, tp=0.0, U=U, dt=0.01)
        e = capi.cp_engine(m, W, 100 + k, mgs_step=3, pop_step=5, precision=precision)
        e.set_walkers(*inputs.initial_walkers(m.phiT, W, seed=7 + k, noise=0.05))
        out.append(e)
    return out


def _state(e):
    wf, lw, al = e.get_walkers()
    return wf, lw, al, e.rng_counter()


@pytest.mark.parametrize("precision", [capi.AFQMC_FP64, capi.AFQMC_MIXED])
def test_batch_matches_separate_engines(precision):
    steps = 11
    solo = _engines(precision)
    for e in solo:
        e.step(steps)
    ref = [_state(e) for e in solo]
    for e in solo:
        e.close()

    engines = _engines(precision)
    b = capi.Batch(engines)
    b.step(steps)
    b.synchronize()
    for e, r in zip(engines, ref):
        s = _state(e)
        assert (s[2] == r[2]).all()
        assert s[3] == r[3]
        assert np.array_equal(s[1], r[1])
        assert np.array_equal(s[0], r[0])
    b.close()
    for e in engines:
        e.close()


def test_autotuned_tiles_keep_results():
    steps = 7
    base = _engines()
    for e in base:
        e.step(steps)
    ref = [_state(e) for e in base]
    for e in base:
        e.close()
    capi.set_autotune(True)
    try:
        engines = _engines()
        b = capi.Batch(engines)
        b.step(steps)
        b.synchronize()
        for e, r in zip(engines, ref):
            s = _state(e)
            assert (s[2] == r[2]).all()
            np.testing.assert_allclose(s[0], r[0], rtol=0, atol=1e-12)
            np.testing.assert_allclose(s[1], r[1], rtol=0, atol=1e-12)
        b.close()
        for e in engines:
            e.close()
    finally:
        capi.set_autotune(False)


def test_batch_rejects_mismatched_cadence():
    m = inputs.hubbard_inputs(4, 4, 7, 7)
    a = capi.cp_engine(m, 8, 1, mgs_step=3, pop_step=5)
    c = capi.cp_engine(m, 8, 2, mgs_step=4, pop_step=5)
    with pytest.raises(RuntimeError):
        capi.Batch([a, c])
    a.close()
    c.close()
