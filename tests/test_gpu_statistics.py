"""Statistical agreement over a full run of configuration 1: the 4x4
periodic Hubbard model, t=1, U=4, 7+7 electrons, free-electron trial,
densitySpin decomposition, dt=0.01, 100 walkers, modifyGM every 10 and
popControl every 40 steps, 2000 steps (200 thermalisation steps with E_T
adjustment, then 180 blocks of 2 measurements 5 steps apart), the
constrained-path driver loop of the reference
(afqmcConstraintPath.cpp:93-148).

The GPU engine (plain FP64 form) and the oracle each run it from their own
seed; their final mixed-estimator energies sum(HNum)/sum(den) must agree
within 3 combined standard errors, each error taken from the block analysis
of the reference's NumDenErrorAnalysis (the largest over block sizes that
leave at least 10 blocks)."""
import numpy as np
import pytest

from afqmclab_b200 import capi, driver, inputs
from oracle import oracle as O
from tests.helpers import num_den_block_analysis
from tests.parity_common import ORACLE_THREADS

pytestmark = pytest.mark.gpu

METHOD = driver.ConstraintPathMethod(dt=0.01, thermalSize=200, writeNumber=180, measureNumberPerWrite=2,
                                     measureSkipStep=5, ETAdjustStep=10, ETAdjustMaxSize=100)


def run(make, seed):
    m, c = inputs.make_config("hubbard4x4")
    eng = make(m, c["W"], seed, c["mgs"], c["pop"])
    wf, lw, al = inputs.initial_walkers(m.phiT, c["W"])     # setWalkerFromPhiT
    eng.set_walkers(wf, lw, al)
    eng.modify_gm()                                         # initialMgsAndPopControl
    eng.pop_control()
    sums = driver.run_constraint_path(eng, METHOD)
    return sums, eng


def test_config1_energy_agrees_with_oracle_within_statistical_error():
    def oracle_engine(*a):
        e = O.cp_engine(*a)
        e.set_threads(ORACLE_THREADS)
        return e

    sg, eg = run(capi.cp_engine, 20240601)
    so, _ = run(oracle_engine, 20240777)
    Eg, errg, _ = num_den_block_analysis(sg[:, 1], sg[:, 0])
    Eo, erro, _ = num_den_block_analysis(so[:, 1], so[:, 0])
    assert eg.status() == 0
    assert 0 < errg < 0.05 and 0 < erro < 0.05, (errg, erro)
    combined = np.sqrt(errg ** 2 + erro ** 2)
    assert abs(Eg.real - Eo.real) < 3 * combined, (Eg, errg, Eo, erro)
    # the constrained-path energy of the 4x4 U=4 7+7 model lies below the
    # free-electron trial energy and above -16 t
    m, _ = inputs.make_config("hubbard4x4")
    assert -16.0 < Eg.real < inputs.hubbard_trial_energy(m)
