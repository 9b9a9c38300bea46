"""The CUDA engine against the reference itself: the same trajectories as
tests/test_reference_programs.py, with the engine's FP64 form (through the
C-ABI) in place of the oracle.  The reference's own tutorial programs
(oracle/_ref, built from the reference's sources) run on the host on the
same inputs, walkers and seed; the engine follows their random stream, so
the per-block estimator sums and the final walkers agree to rounding.

The engine's modified Gram-Schmidt gives R_jj > 0 where the reference's
Householder QR gives signs, so final walkers are compared through
gauge-invariant quantities: each spin block's projector
phi (phi^H phi)^-1 phi^H and the log-overlap with the trial (log-weight
included, phase mod 2 pi).

Tolerance: 1e-8 relative over the whole run (FP64; GPU reductions sum in a
different order than the reference's serial loops)."""
import numpy as np
import pytest

from afqmclab_b200 import capi, driver, inputs
from oracle import oracle as O
from tests import test_reference_programs as R
from tests.helpers import logov_close

pytestmark = pytest.mark.gpu

TOL = 1e-8


def _projector(a):
    return a @ np.linalg.solve(a.conj().T @ a, a.conj().T)


def _compare_walkers(eng, out, m, kind):
    wf_r, lw_r, al_r = out["walkers"]
    wf, lw, al = eng.get_walkers()
    assert np.array_equal(al.astype(bool), al_r.astype(bool))
    blocks = [m.N] if kind == "cp" else [b for b in (m.nup, m.ndn) if b > 0]
    lo_g, lo_r = [], []
    for w in np.flatnonzero(al_r):
        for nb in blocks:
            assert R._rel(_projector(wf[:, :nb, w]), _projector(wf_r[:, :nb, w])) < TOL
        if kind == "cp":
            lo_g.append(O.sdsd(m.phiT, m.logwT, wf[:, :, w], lw[w])[0])
            lo_r.append(O.sdsd(m.phiT, m.logwT, wf_r[:, :, w], lw_r[w])[0])
        else:
            lo_g.append(O.sd2s_sd2is(m.phiTUp, m.phiTDn, m.logwT, wf[:, :, w], lw[w], m.nup, m.ndn)[0])
            lo_r.append(O.sd2s_sd2is(m.phiTUp, m.phiTDn, m.logwT, wf_r[:, :, w], lw_r[w], m.nup,
                                     m.ndn)[0])
    assert logov_close(np.array(lo_g), np.array(lo_r), TOL) < TOL


def _streams(sums, out, names):
    for j, name in enumerate(names):
        assert R._rel(sums[:, j], out[name]) < TOL, name
    assert R._rel(sums[:, 1] / sums[:, 0], out["HNum"] / out["den"]) < TOL


@R.needs_cp
@pytest.mark.parametrize("decomp,force", [("densitySpin", "dynamicForce"),
                                          ("hopCharge", "constForce")])
def test_engine_follows_constraint_path_program(decomp, force):
    m = inputs.hubbard_inputs(4, 4, 7, 7, U=4.0, dt=0.01, decomp=decomp)
    m.ET = inputs.hubbard_trial_energy(m)
    meth = driver.ConstraintPathMethod(**R.CP_METHOD)
    eng, sums, out = R.run_cp_both(m, 8, 1201, meth, mgs=3, pop=7, force_type=force,
                                   make_engine=capi.cp_engine)
    _streams(sums, out, ["den", "HNum", "KNum", "VNum", "RNum"])
    _compare_walkers(eng, out, m, "cp")
    eng.close()


@R.needs_cp
def test_engine_follows_constraint_path_program_100_walkers():
    m = inputs.hubbard_inputs(4, 4, 7, 7, U=4.0, dt=0.01)
    m.ET = inputs.hubbard_trial_energy(m)
    meth = driver.ConstraintPathMethod(**R.CP_METHOD)
    eng, sums, out = R.run_cp_both(m, 100, 77, meth, mgs=10, pop=40, make_engine=capi.cp_engine)
    _streams(sums, out, ["den", "HNum", "KNum", "VNum", "RNum"])
    _compare_walkers(eng, out, m, "cp")
    eng.close()


@R.needs_pl
@pytest.mark.parametrize("nup,ndn", [(4, 3), (4, 4)])
def test_engine_follows_phaseless_program(nup, ndn):
    """(4, 4) with a real trial takes the engine's closed-shell single-block
    form; (4, 3) the two-block form."""
    m = inputs.molecule_inputs(n=16, nup=nup, ndn=ndn, G=24, dt=0.01, decay=6.0, seed=7)
    meth = driver.PhaselessMethod(**R.PL_METHOD)
    nums = []
    eng, sums, out = R.run_pl_both(m, 8, 4321, meth, mgs=3, pop=7, make_engine=capi.pl_engine,
                                   on_block=lambda i, e: nums.append(e.cholesky_nums()))
    _streams(sums, out, ["den", "HNum", "TNum"])
    assert R._rel(np.array([b for b, _ in nums]), out["choleskyBgNum"]) < TOL
    assert R._rel(np.array([x for _, x in nums]), out["choleskyExNum"]) < TOL
    _compare_walkers(eng, out, m, "pl")
    eng.close()


@R.needs_pl
def test_engine_follows_phaseless_program_adjusting_background():
    m = inputs.molecule_inputs(n=16, nup=4, ndn=3, G=24, dt=0.01, decay=6.0, seed=9)
    meth = driver.PhaselessMethod(dt=0.01, thermalSize=16, writeNumber=3, measureNumberPerWrite=2,
                                  measureSkipStep=3, ETAndBackGroundAdjustStep=2,
                                  ETAndBackGroundAdjustMaxSize=6,
                                  ETAndBackGroundGrowthEstimateStep=2,
                                  ETAndBackGroundGrowthEstimateMaxSize=12)

    def make(m_, W, seed, **kw):
        return capi.pl_engine(m_, W, seed, log_one_body=True, **kw)

    eng, sums, out = R.run_pl_both(m, 8, 555, meth, mgs=3, pop=5, make_engine=make)
    _streams(sums, out, ["den", "HNum", "TNum"])
    _compare_walkers(eng, out, m, "pl")
    eng.close()
