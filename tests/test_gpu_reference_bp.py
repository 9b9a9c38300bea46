"""The back-propagated estimator against the reference's own back-propagation
program (tutorials/afqmcConstraintPathBP, built from the reference's sources
into oracle/_ref with the same stand-ins as the other reference programs).

Engine (FP64 form, observe estimator on) and program start from the same
walkers and random stream and run the tutorial's loop: thermalisation with
E_T adjustment, a back-propagation window opened after it, and blocks of
measurements in which every full window is measured (the window-start
walkers resampled by the recorded population-control tables, the trial
propagated leftwards through each walker's recorded fields, the observe
estimator accumulated for the pair, weighted by the current walker's
overlap).  Per block, den, HNum, KNum, VNum, RNum and the five observe
matrices must agree to 1e-8 relative (FP64 on both sides; the GPU sums in a
different order).  Both window regimes are covered: backPropagationStep
at least measureSkipStep (the window slides) and below it (a new window per
measurement), with population control inside the windows.
"""
import os
import sys

import numpy as np
import pytest

from afqmclab_b200 import capi, driver, inputs

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "ref"))
import ref_run  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_run.available("bp"),
                                 reason="reference programs not built (reference sources absent)")]

TOL = 1e-8


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(1.0, np.abs(b).max()))


@pytest.mark.parametrize("bp_steps,decomp", [(8, "densitySpin"), (3, "densitySpin"), (8, "hopCharge")])
def test_back_propagation_follows_reference_program(bp_steps, decomp):
    m = inputs.hubbard_inputs(4, 4, 7, 7, U=4.0, dt=0.01, decomp=decomp)
    m.ET = inputs.hubbard_trial_energy(m)
    W, seed, mgs, pop = 8, 2203, 3, 7
    meth = driver.ConstraintPathBPMethod(dt=0.01, thermalSize=10, writeNumber=3, measureNumberPerWrite=2,
                                         measureSkipStep=5, ETAdjustStep=4, ETAdjustMaxSize=8,
                                         backPropagationStep=bp_steps)
    wf, lw, al = inputs.initial_walkers(m.phiT, W, seed=seed + 1, noise=0.05)
    out, _ = ref_run.run_cp_bp(m, meth, bp_steps, wf, lw, seed, mgs_step=mgs, pop_step=pop)

    eng = capi.cp_engine(m, W, seed, mgs, pop)
    eng.set_observables(True)
    eng.set_walkers(wf, lw, al)
    ref_run.start_like_program(eng, "bp", m, seed)
    obs = []
    sums = driver.run_constraint_path_bp(eng, meth, on_block=lambda i, e: obs.append(e.observables()))
    eng.close()

    for j, name in enumerate(["den", "HNum", "KNum", "VNum", "RNum"]):
        assert _rel(sums[:, j], out[name]) < TOL, name
    for name in ref_run.OBSERVE_STREAMS:
        mine = np.array([o[name].ravel(order="F") for o in obs])
        assert _rel(mine, out[name]) < TOL, name
