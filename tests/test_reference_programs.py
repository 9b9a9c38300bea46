"""The oracle against the reference itself: the reference's own tutorial
programs (afqmcConstraintPath, afqmcPhaseless), built from its sources into
oracle/_ref with stand-ins only for the absent libraries (googletest, HDF5,
SPRNG -> the SplitMix64 stream the oracle uses, BLAS/LAPACK -> OpenBLAS), run
on the same inputs, walkers and seed.

Both follow the same random stream in the same order, so whole trajectories
agree to rounding: the per-block estimator sums the programs write (den.dat,
HNum.dat, ...) and the walkers they write at the end (writeWalkers after the
closing half step), through E_T adjustment, modified Gram-Schmidt and
population control.  Parity tolerance: 1e-9 relative (FP64 throughout; the
observed agreement is ~1e-13).
"""
import os
import sys

import numpy as np
import pytest

from afqmclab_b200 import driver, inputs
from oracle import oracle as O

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                "oracle", "ref"))
import ref_run  # noqa: E402

TOL = 1e-9

needs_cp = pytest.mark.skipif(not ref_run.available("cp"),
                              reason="reference programs not built (reference sources absent)")
needs_pl = pytest.mark.skipif(not ref_run.available("pl"),
                              reason="reference programs not built (reference sources absent)")


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(1.0, np.abs(b).max()))


def compare_streams(sums, out, names):
    """sums: the driver's block sums (blocks x k, columns in `names` order)."""
    for j, name in enumerate(names):
        assert _rel(sums[:, j], out[name]) < TOL, name
    e_mine = sums[:, 1] / sums[:, 0]
    e_ref = out["HNum"] / out["den"]
    assert _rel(e_mine, e_ref) < TOL


def compare_walkers(eng, out, tol=TOL):
    wf_r, lw_r, al_r = out["walkers"]
    wf, lw, al = eng.get_walkers()
    assert np.array_equal(al.astype(bool), al_r.astype(bool))
    a = al_r.astype(bool)
    assert _rel(wf[:, :, a], wf_r[:, :, a]) < tol
    assert np.abs(lw[a].real - lw_r[a].real).max() < tol * max(1.0, np.abs(lw_r[a].real).max())
    assert np.abs(np.exp(1j * lw[a].imag) - np.exp(1j * lw_r[a].imag)).max() < tol


def run_cp_both(m, W, seed, meth, mgs, pop, force_type="dynamicForce", make_engine=None, noise=0.05):
    wf, lw, al = inputs.initial_walkers(m.phiT, W, seed=seed + 1, noise=noise)
    out, _ = ref_run.run_cp(m, meth, wf, lw, seed, mgs_step=mgs, pop_step=pop, force_type=force_type)
    make = make_engine or O.cp_engine
    eng = make(m, W, seed, mgs_step=mgs, pop_step=pop, force_type=force_type)
    eng.set_walkers(wf, lw, al)
    ref_run.start_like_program(eng, "cp", m, seed)
    sums = driver.run_constraint_path(eng, meth)
    return eng, sums, out


def run_pl_both(m, W, seed, meth, mgs, pop, force_type="dynamicForce", make_engine=None, noise=0.05,
                on_block=None):
    wf, lw, al = inputs.initial_walkers(m.phiTUp, W, seed=seed + 1, noise=noise)
    out, _ = ref_run.run_pl(m, meth, wf, lw, seed, mgs_step=mgs, pop_step=pop, force_type=force_type)
    make = make_engine or O.pl_engine
    eng = make(m, W, seed, mgs_step=mgs, pop_step=pop, force_type=force_type)
    eng.set_walkers(wf, lw, al)
    ref_run.start_like_program(eng, "pl", m, seed)
    sums = driver.run_phaseless(eng, m, meth, on_block=on_block)
    return eng, sums, out


CP_METHOD = dict(dt=0.01, thermalSize=20, writeNumber=5, measureNumberPerWrite=2, measureSkipStep=5,
                 ETAdjustStep=4, ETAdjustMaxSize=12)
PL_METHOD = dict(dt=0.01, thermalSize=20, writeNumber=5, measureNumberPerWrite=2, measureSkipStep=5,
                 ETAndBackGroundAdjustStep=2, ETAndBackGroundAdjustMaxSize=0,
                 ETAndBackGroundGrowthEstimateStep=2, ETAndBackGroundGrowthEstimateMaxSize=0)


@needs_cp
@pytest.mark.parametrize("decomp,force", [("densitySpin", "dynamicForce"),
                                          ("densityCharge", "dynamicForce"),
                                          ("hopSpin", "dynamicForce"),
                                          ("hopCharge", "constForce")])
def test_oracle_follows_constraint_path_program(decomp, force):
    m = inputs.hubbard_inputs(4, 4, 7, 7, U=4.0, dt=0.01, decomp=decomp)
    m.ET = inputs.hubbard_trial_energy(m)
    meth = driver.ConstraintPathMethod(**CP_METHOD)
    eng, sums, out = run_cp_both(m, 8, 1201, meth, mgs=3, pop=7, force_type=force)
    compare_streams(sums, out, ["den", "HNum", "KNum", "VNum", "RNum"])
    compare_walkers(eng, out)


@needs_cp
def test_oracle_follows_constraint_path_program_100_walkers():
    """The 4x4, 7+7, U=4 lattice with 100 walkers, 90 steps."""
    m = inputs.hubbard_inputs(4, 4, 7, 7, U=4.0, dt=0.01)
    m.ET = inputs.hubbard_trial_energy(m)
    meth = driver.ConstraintPathMethod(**CP_METHOD)
    eng, sums, out = run_cp_both(m, 100, 77, meth, mgs=10, pop=40)
    compare_streams(sums, out, ["den", "HNum", "KNum", "VNum", "RNum"])
    compare_walkers(eng, out)


@needs_pl
@pytest.mark.parametrize("nup,ndn,force", [(4, 3, "dynamicForce"), (4, 4, "dynamicForce"),
                                           (4, 3, "constForce"), (3, 0, "dynamicForce")])
def test_oracle_follows_phaseless_program(nup, ndn, force):
    m = inputs.molecule_inputs(n=16, nup=nup, ndn=ndn, G=24, dt=0.01, decay=6.0, seed=7)
    meth = driver.PhaselessMethod(**PL_METHOD)
    nums = []
    eng, sums, out = run_pl_both(m, 8, 4321, meth, mgs=3, pop=7, force_type=force,
                                 on_block=lambda i, e: nums.append(e.cholesky_nums()))
    compare_streams(sums, out, ["den", "HNum", "TNum"])
    # the per-block background and exchange sums (G each)
    assert _rel(np.array([b for b, _ in nums]), out["choleskyBgNum"]) < TOL
    assert _rel(np.array([x for _, x in nums]), out["choleskyExNum"]) < TOL
    compare_walkers(eng, out)


@needs_pl
def test_oracle_follows_phaseless_program_with_background():
    """A non-zero background (the mean-field shift the driver would have
    adjusted to) enters the propagators, the force and the sample weight."""
    m = inputs.molecule_inputs(n=16, nup=4, ndn=4, G=24, dt=0.01, decay=6.0, seed=8)
    rng = np.random.default_rng(5)
    m.set_background(0.2 * rng.standard_normal(m.G))
    meth = driver.PhaselessMethod(**PL_METHOD)
    eng, sums, out = run_pl_both(m, 8, 99, meth, mgs=3, pop=7)
    compare_streams(sums, out, ["den", "HNum", "TNum"])
    compare_walkers(eng, out)


@needs_pl
@pytest.mark.parametrize("adj_max,growth_max", [(6, 0), (6, 12)])
def test_oracle_follows_phaseless_program_adjusting_background(adj_max, growth_max):
    """isETAndBackGroundAdjustable: the run starts in the Taylor one-body form
    (LogHop2is, dynamicOrder), adjusts E_T and the background from the mixed
    estimator every ETAndBackGroundAdjustStep steps, optionally averages the
    growth estimate, then rebuilds the dense propagators from the final
    background (afqmcPhaseless.cpp:43-66, 125-170)."""
    m = inputs.molecule_inputs(n=16, nup=4, ndn=3, G=24, dt=0.01, decay=6.0, seed=9)
    meth = driver.PhaselessMethod(dt=0.01, thermalSize=16, writeNumber=3, measureNumberPerWrite=2,
                                  measureSkipStep=3, ETAndBackGroundAdjustStep=2,
                                  ETAndBackGroundAdjustMaxSize=adj_max,
                                  ETAndBackGroundGrowthEstimateStep=2,
                                  ETAndBackGroundGrowthEstimateMaxSize=growth_max)
    assert meth.adjustable()

    def make(m_, W, seed, **kw):
        return O.pl_engine(m_, W, seed, log_one_body=True, **kw)

    eng, sums, out = run_pl_both(m, 8, 555, meth, mgs=3, pop=5, make_engine=make)
    compare_streams(sums, out, ["den", "HNum", "TNum"])
    compare_walkers(eng, out)
