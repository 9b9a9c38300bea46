"""GPU engine (C-ABI, plain FP64 form) against the CPU oracle on identical
inputs and identical random streams.

Tolerances (plain FP64 form): per-step log-overlaps, Green's functions and
local energies agree to 1e-10 relative when both sides start the step from the
same walkers; a multi-step trajectory stays within 1e-8; population-control
tables are bit-exact.
"""
import numpy as np
import pytest

from afqmclab_b200 import capi, inputs
from oracle import oracle as O
from tests.helpers import logov_close, rel_err
from tests.parity_common import (STEP_TOL, TRAJ_TOL, compare_state, hubbard, molecule,
                                  pair_cp, pair_pl)

pytestmark = pytest.mark.gpu


# ------------------------------------------------------------------ CP
def test_cp_overlap_and_green():
    m = hubbard("densitySpin", fields=True)
    g, o = pair_cp(m, 12, 7, 10, 40, noise=0.2)
    err = logov_close(g.log_overlaps(), o.log_overlaps(), STEP_TOL)
    assert err < STEP_TOL
    for w in (0, 5, 11):
        assert rel_err(g.green(w), o.green(w)) < STEP_TOL


@pytest.mark.parametrize("decomp,fields", [("densitySpin", False), ("densityCharge", True),
                                           ("hopSpin", True), ("hopCharge", True)])
def test_cp_single_step_parity(decomp, fields):
    m = hubbard(decomp, fields)
    W = 24
    g, o = pair_cp(m, W, 21, 1000, 1000)
    for step in range(4):
        wf, lw, al = o.get_walkers()
        g.set_walkers(wf, lw, al)
        g.set_rng(21, o.rng_counter())
        g.step(1)
        o.step(1)
        compare_state(g, o, STEP_TOL)
        _, _, al = o.get_walkers()
        for w in np.nonzero(al)[0][:3]:
            assert rel_err(g.green(w), o.green(w)) < STEP_TOL


def test_cp_trajectory_with_stabilize_and_pop_control():
    """Config-1 shapes (4x4, 7+7, densitySpin, dt=0.01): 24 steps with
    modifyGM every 4 and popControl every 6; the engine and the oracle run
    independently from the same start."""
    m = hubbard("densitySpin")
    W = 32
    g, o = pair_cp(m, W, 5, 4, 6)
    for step in range(24):
        g.step(1)
        o.step(1)
        compare_state(g, o, TRAJ_TOL)


def test_cp_pop_control_table_bit_exact():
    m = hubbard("densitySpin")
    W = 40
    g, o = pair_cp(m, W, 9, 1000, 1000, noise=0.3)
    g.step(3)
    o.step(3)
    wf, lw, al = o.get_walkers()
    g.set_walkers(wf, lw, al)
    g.set_rng(9, o.rng_counter())
    tg, wg = g.pop_control()
    to, wo = o.pop_control()
    assert rel_err(wg, wo) < STEP_TOL
    assert (tg == to).all()
    compare_state(g, o, STEP_TOL)


def test_cp_stabilize_is_gauge_invariant():
    m = hubbard("densityCharge", fields=True)
    g, o = pair_cp(m, 10, 3, 1000, 1000, noise=0.3)
    g.modify_gm()
    o.modify_gm()
    compare_state(g, o, STEP_TOL)
    for w in range(3):
        assert rel_err(g.green(w), o.green(w)) < STEP_TOL
    wf, _, _ = g.get_walkers()
    for w in range(3):
        q = wf[:, :, w]
        assert np.allclose(q.conj().T @ q, np.eye(q.shape[1]), atol=1e-12)


def test_cp_const_force_step():
    m = hubbard("densitySpin")
    W = 16
    g, o = pair_cp(m, W, 13, 1000, 1000, force="constForce")
    g.step(2)
    o.step(2)
    compare_state(g, o, TRAJ_TOL)


def test_cp_measurement_parity():
    m = hubbard("densitySpin", fields=True)
    W = 20
    g, o = pair_cp(m, W, 17, 1000, 1000, noise=0.2)
    g.step(2)
    o.step(2)
    wf, lw, al = o.get_walkers()
    g.set_walkers(wf, lw, al)
    g.reset_measurement()
    o.reset_measurement()
    g.add_mixed_measurement()
    o.add_mixed_measurement()
    mg, mo = g.measurement(), o.measurement()
    assert rel_err(mg[:2], mo[:2]) < STEP_TOL
    assert abs(mg[1] / mg[0] - mo[1] / mo[0]) < STEP_TOL * abs(mo[1] / mo[0])
    for k in (2, 3, 4):
        assert abs(mg[k] - mo[k]) <= STEP_TOL * max(1.0, abs(mo[1]))
    # NupNum, NdnNum, SplusNum, SminusNum (HubbardSOCMeasureFixedSDSD.cpp:221-255)
    sg, so = g.site_nums(), o.site_nums()
    for a, b in zip(sg, so):
        assert np.abs(a - b).max() <= STEP_TOL * abs(mo[0])
    assert abs((sg[0].sum() + sg[1].sum()) / mg[0] - m.N) < 1e-9


def test_cp_project_half_roundtrip():
    m = hubbard("densitySpin")
    g, o = pair_cp(m, 8, 1, 1000, 1000, noise=0.1)
    g.project_half(-1)
    o.project_half(-1)
    compare_state(g, o, STEP_TOL)
    g.project_half(+1)
    o.project_half(+1)
    compare_state(g, o, STEP_TOL)


# ------------------------------------------------------------------ PL
@pytest.mark.parametrize("nup,ndn", [(4, 3), (4, 4)])
def test_pl_overlap_and_green(nup, ndn):
    m = molecule(nup=nup, ndn=ndn)
    g, o = pair_pl(m, 8, 3, 10, 10, noise=0.2)
    assert logov_close(g.log_overlaps(), o.log_overlaps(), STEP_TOL) < STEP_TOL
    for w in (0, 7):
        for s in (0, 1):
            assert rel_err(g.green(w, s), o.green(w, s)) < STEP_TOL


@pytest.mark.parametrize("log_one_body", [False, True])
def test_pl_single_step_parity(log_one_body):
    m = molecule()
    W = 16
    g, o = pair_pl(m, W, 31, 1000, 1000, log_one_body=log_one_body)
    for step in range(3):
        wf, lw, al = o.get_walkers()
        g.set_walkers(wf, lw, al)
        g.set_rng(31, o.rng_counter())
        g.step(1)
        o.step(1)
        compare_state(g, o, STEP_TOL)
    assert g.taylor_stats()[0] > 0


def test_pl_trajectory_with_stabilize_and_pop_control():
    m = molecule()
    W = 24
    g, o = pair_pl(m, W, 41, 3, 5)
    for step in range(15):
        g.step(1)
        o.step(1)
        compare_state(g, o, TRAJ_TOL)
    assert g.taylor_stats() == o.taylor_stats()


def test_pl_measurement_parity():
    m = molecule()
    W = 12
    g, o = pair_pl(m, W, 43, 1000, 1000, noise=0.1)
    g.step(2)
    o.step(2)
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


def test_pl_const_force_and_background_update():
    m = molecule()
    W = 8
    g, o = pair_pl(m, W, 47, 1000, 1000, force="constForce")
    g.step(2)
    o.step(2)
    compare_state(g, o, TRAJ_TOL)
    # background update + propagator rebuild (realMaterialMolecule.cpp:103-178)
    m2 = molecule()
    m2.set_background(0.01 * np.arange(m2.G))
    g2, o2 = pair_pl(m2, W, 48, 1000, 1000)
    g2.step(2)
    o2.step(2)
    compare_state(g2, o2, TRAJ_TOL)


# ------------------------------------------------------------ pop control
def test_pop_configuration_dev_bit_exact():
    import torch
    rng = np.random.default_rng(77)
    for W in (1, 7, 1000, 4096):
        w = rng.uniform(0, 3, W)
        w[rng.uniform(size=W) < 0.1] = 0.0
        if w.sum() == 0:
            w[0] = 1.0
        u = rng.uniform(size=W)
        table_o, bad = O.pop_configuration(w, u)
        tw = torch.tensor(w, device="cuda", dtype=torch.float64)
        tu = torch.tensor(u, device="cuda", dtype=torch.float64)
        tt = torch.zeros(W, device="cuda", dtype=torch.int32)
        capi.pop_configuration_dev(tw.data_ptr(), tu.data_ptr(), tt.data_ptr(), W)
        torch.cuda.synchronize()
        assert (tt.cpu().numpy() == table_o).all()


# ------------------------------------------- wider overlap blocks (33..120)
@pytest.mark.parametrize("nx,ny,nup,ndn", [(6, 6, 20, 20), (8, 8, 28, 28), (10, 10, 40, 40)])
def test_cp_wide_blocks_step_and_pop_control(nx, ny, nup, ndn):
    """Blocks of 40, 56 and 80 columns take the shared-memory Gauss-Jordan
    path (inverse) and its LU-only variant (population-control weights)."""
    m = hubbard("densitySpin", True, nx=nx, ny=ny, nup=nup, ndn=ndn)
    W = 6
    g, o = pair_cp(m, W, 31, 1000, 2, noise=0.1)
    err = logov_close(g.log_overlaps(), o.log_overlaps(), STEP_TOL)
    assert err < STEP_TOL
    for w in (0, 3):
        assert rel_err(g.green(w), o.green(w)) < STEP_TOL
    for step in range(2):
        wf, lw, al = o.get_walkers()
        g.set_walkers(wf, lw, al)
        g.set_rng(31, o.rng_counter())
        g.set_cadence(0, step)
        o_before = o.rng_counter()
        g.step(1)
        o.step(1)
        compare_state(g, o, STEP_TOL)
    assert g.rng_counter() == o.rng_counter() and o.rng_counter() > o_before


def test_pl_wide_blocks_step():
    m = molecule(n=96, nup=40, ndn=36, G=48)
    W = 4
    g, o = pair_pl(m, W, 41, 1000, 1000)
    err = logov_close(g.log_overlaps(), o.log_overlaps(), STEP_TOL)
    assert err < STEP_TOL
    wf, lw, al = o.get_walkers()
    g.set_walkers(wf, lw, al)
    g.step(1)
    o.step(1)
    compare_state(g, o, STEP_TOL)
    for w in (0, 2):
        for spin in (0, 1):
            assert rel_err(g.green(w, spin), o.green(w, spin)) < STEP_TOL


def test_pl_fp64_closed_shell_matches_two_block_form():
    """With the same trial for both spins the FP64 form computes one spin
    block and counts it twice, and evaluates the exchange as FP64 GEMMs; a
    trial whose down block differs from the up block in one last bit takes
    the two-block path.  Both agree with each other and with the oracle."""
    m = molecule(n=32, nup=6, ndn=6, G=40)
    assert np.array_equal(m.phiTUp, m.phiTDn)
    m2 = molecule(n=32, nup=6, ndn=6, G=40)
    d = m2.phiTDn.copy()
    d[0, 0] = np.nextafter(d[0, 0].real, np.inf) + 1j * d[0, 0].imag
    m2.phiTDn = np.asfortranarray(d)
    W = 16
    out = []
    for mm in (m, m2):
        g, o = pair_pl(mm, W, 91, 3, 1000, noise=0.05)
        g.step(4)
        o.step(4)
        compare_state(g, o, TRAJ_TOL)
        for e in (g, o):
            e.reset_measurement()
            e.add_mixed_measurement()
        mg, mo = g.measurement(), o.measurement()
        assert rel_err(mg[:3], mo[:3]) < STEP_TOL
        bg, eg = g.cholesky_nums()
        bo, eo = o.cholesky_nums()
        assert rel_err(bg, bo) < STEP_TOL and rel_err(eg, eo) < STEP_TOL
        out.append((g.log_overlaps(), mg))
    assert logov_close(out[0][0], out[1][0], 1e-9) < 1e-9
    assert abs(out[0][1][1] / out[0][1][0] - out[1][1][1] / out[1][1][0]) < 1e-9
