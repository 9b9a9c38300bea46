"""Constrained-path mixed-precision form (tcgen05 kind::tf32 contractions
with compensated hi/lo operands, also for the measurement's half step and
overlap; FP64 LU/log-det, weights, re-orthonormalisation, population control
and the rest of the measurement) against the plain FP64 form on the same
walkers and random stream.

Tolerances: with a constant force (identical aux fields) walkers and
log-weights agree to 2e-5 relative after several steps (fp32 walkers,
3-term tf32 products); with the dynamic force (tf32 Green's function entries)
at least 90% of walkers take the same aux fields in the first step; the mixed
estimator on identical walkers agrees to 2e-5 relative in the energy and to
1e-4 in the normalisation sum_w overlap_w (the half step and the overlap as
3-term tf32 products, about 1e-7 per entry, amplified in each walker's
overlap determinant; the ratio cancels most of it), and, along a run, to
2e-3 relative."""
import numpy as np
import pytest

from afqmclab_b200 import capi, inputs

pytestmark = pytest.mark.gpu

LATTICES = {
    "4x4": (4, 4, 7, 7, 4.0, 0.0),
    "6x6": (6, 6, 16, 16, 8.0, 0.0),
    "8x8": (8, 8, 28, 28, 4.0, -0.2),
    "10x10": (10, 10, 40, 40, 4.0, 0.0),
}


def hubbard(name, dt=0.01):
    nx, ny, nu, nd, U, tp = LATTICES[name]
    m = inputs.hubbard_inputs(nx, ny, nu, nd, t=1.0, tp=tp, U=U, dt=dt)
    return m


def pair(m, W, seed, mgs=1000, pop=1000, noise=0.05, const_force=None):
    ft = "constForce" if const_force is not None else "dynamicForce"
    f = capi.cp_engine(m, W, seed, mgs, pop, force_type=ft, precision=capi.AFQMC_FP64,
                       const_force=const_force)
    x = capi.cp_engine(m, W, seed, mgs, pop, force_type=ft, precision=capi.AFQMC_MIXED,
                       const_force=const_force)
    wf, lw, al = inputs.initial_walkers(m.phiT, W, seed=seed + 1, noise=noise)
    f.set_walkers(wf, lw, al)
    x.set_walkers(wf, lw, al)
    return f, x


def walker_err(a, b):
    return np.abs(a - b).max() / np.abs(a).max()


@pytest.mark.parametrize("name", list(LATTICES))
def test_const_force_steps_match_fp64(name):
    m = hubbard(name)
    W = 40
    rng = np.random.default_rng(3)
    cf = 0.2 * rng.standard_normal(m.L)
    f, x = pair(m, W, 11, const_force=cf)
    assert np.abs(f.log_overlaps() - x.log_overlaps()).max() < 1e-5
    f.step(4)
    x.step(4)
    wf, lf, af = f.get_walkers()
    wx, lx, ax = x.get_walkers()
    assert (af == ax).all()
    assert f.rng_counter() == x.rng_counter()
    a = af.astype(bool)
    print(name, "walker error", walker_err(wf[:, :, a], wx[:, :, a]), "logw", np.abs(lf[a] - lx[a]).max())
    assert walker_err(wf[:, :, a], wx[:, :, a]) < 2e-5
    assert np.abs(lf[a] - lx[a]).max() < 2e-5 * max(1.0, np.abs(lf[a]).max())
    of, ox = f.log_overlaps(), x.log_overlaps()
    assert np.abs(of[a].real - ox[a].real).max() < 1e-4
    assert x.status() == 0


@pytest.mark.parametrize("name", ["4x4", "8x8", "10x10"])
def test_dynamic_force_first_step(name):
    m = hubbard(name)
    W = 64
    f, x = pair(m, W, 13)
    f.step(1)
    x.step(1)
    wf, _, af = f.get_walkers()
    wx, _, ax = x.get_walkers()
    assert (af == ax).all()
    same = [walker_err(wf[:, :, w], wx[:, :, w]) < 1e-4 for w in range(W) if af[w]]
    assert np.mean(same) >= 0.9, np.mean(same)
    print(name, "walkers with the same aux fields:", np.mean(same))
    assert x.status() == 0


@pytest.mark.parametrize("name", ["4x4", "8x8"])
def test_measurement_on_same_walkers(name):
    m = hubbard(name)
    f, x = pair(m, 32, 17, noise=0.1)
    for e in (f, x):
        e.reset_measurement()
        e.add_mixed_measurement()
    mf, mx = f.measurement(), x.measurement()
    assert abs(mf[0] - mx[0]) < 1e-4 * abs(mf[0])
    assert abs(mf[1] / mf[0] - mx[1] / mx[0]) < 2e-5 * abs(mf[1] / mf[0])
    print(name, "den", abs(mf[0] - mx[0]) / abs(mf[0]), "E", abs(mf[1] / mf[0] - mx[1] / mx[0]) / abs(mf[1] / mf[0]))


def test_cadence_and_population_control():
    m = hubbard("6x6")
    W = 48
    cf = 0.1 * np.random.default_rng(5).standard_normal(m.L)
    f, x = pair(m, W, 23, mgs=2, pop=3, const_force=cf)
    f.step(7)
    x.step(7)
    wf, lf, af = f.get_walkers()
    wx, lx, ax = x.get_walkers()
    assert (af == ax).all()
    assert f.rng_counter() == x.rng_counter()
    assert walker_err(wf, wx) < 2e-5
    assert x.status() == 0


def test_energy_tracks_fp64():
    m = hubbard("8x8", dt=0.005)
    m.ET = -60.0
    W = 64
    f, x = pair(m, W, 29, mgs=5, pop=10)
    ef, ex = [], []
    for step in range(20):
        for e, acc in ((f, ef), (x, ex)):
            if step % 5 == 0:
                e.reset_measurement()
                e.add_mixed_measurement()
                mm = e.measurement()
                acc.append((mm[1] / mm[0]).real)
            e.step(1)
    ef, ex = np.array(ef), np.array(ex)
    assert np.all(np.abs(ef - ex) < 2e-3 * np.abs(ef)), (ef, ex)
    assert x.status() == 0


def test_rejects_odd_site_count():
    m = inputs.hubbard_inputs(3, 3, 4, 4)
    with pytest.raises(capi.AfqmcError):
        capi.cp_engine(m, 8, 1, precision=capi.AFQMC_MIXED)
