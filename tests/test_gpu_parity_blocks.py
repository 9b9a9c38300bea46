"""Overlap blocks of 17 to 32 columns against the oracle (plain FP64 form).

Every LU, log-determinant and inverse of a block 17 to 32 columns wide runs
in the register-resident Gauss-Jordan kernel: one warp per matrix, lane i
holding row i, padded with the identity up to 32.  That covers the 32-column
spin blocks of the headline molecule, the 6x6 16+16 lattice, and open-shell
mixes such as 32+17 where the second block is padded.  The engine and the
oracle start from the same walkers and random stream; per step they must
agree on log-overlaps and Green's functions of both spins (the inverse feeds
theta, so G checks it), on the population-control weights (the LU-only
elimination) and tables (bit-exact), and on the mixed-estimator sums, all to
1e-10 (SDSDOperation.cpp:154-173, SD2sSD2isOperation.cpp:187-211,
tensor_2d_common_fun.cpp:75-105).
"""
import numpy as np
import pytest

from tests.helpers import logov_close, rel_err
from tests.parity_common import STEP_TOL, compare_state, hubbard, molecule, pair_cp, pair_pl

pytestmark = pytest.mark.gpu


def resync_step(g, o, seed, nsteps):
    """Load the oracle's state into the engine, then take one step on both."""
    for _ in range(nsteps):
        wf, lw, al = o.get_walkers()
        g.set_walkers(wf, lw, al)
        g.set_rng(seed, o.rng_counter())
        g.step(1)
        o.step(1)
        compare_state(g, o, STEP_TOL)


def check_pop_control(g, o, seed):
    wf, lw, al = o.get_walkers()
    g.set_walkers(wf, lw, al)
    g.set_rng(seed, o.rng_counter())
    tg, wg = g.pop_control()
    to, wo = o.pop_control()
    assert rel_err(wg, wo) < STEP_TOL
    assert (tg == to).all()
    assert len(set(to.tolist())) < len(to), "weights too even: the comb copied nothing"
    compare_state(g, o, STEP_TOL)


@pytest.mark.parametrize("n,nup,ndn", [(64, 17, 17), (64, 24, 20), (64, 32, 32), (64, 32, 17),
                                       (64, 32, 10), (48, 29, 23)])
def test_pl_register_lu_blocks(n, nup, ndn):
    m = molecule(n=n, nup=nup, ndn=ndn, G=48)
    W = 8
    seed = 100 + nup + ndn
    g, o = pair_pl(m, W, seed, 1000, 1000, noise=0.1)
    assert logov_close(g.log_overlaps(), o.log_overlaps(), STEP_TOL) < STEP_TOL
    for w in (0, W - 1):
        for spin in (0, 1):
            assert rel_err(g.green(w, spin), o.green(w, spin)) < STEP_TOL
    resync_step(g, o, seed, 2)
    for e in (g, o):
        e.reset_measurement()
    wf, lw, al = o.get_walkers()
    g.set_walkers(wf, lw, al)
    g.add_mixed_measurement()
    o.add_mixed_measurement()
    mg, mo = g.measurement(), o.measurement()
    assert rel_err(mg[:3], mo[:3]) < STEP_TOL
    bg, eg = g.cholesky_nums()
    bo, eo = o.cholesky_nums()
    assert rel_err(bg, bo) < STEP_TOL and rel_err(eg, eo) < STEP_TOL
    check_pop_control(g, o, seed)


@pytest.mark.parametrize("nx,ny,nup,ndn", [(4, 4, 9, 9), (6, 6, 12, 12), (6, 6, 16, 16),
                                           (6, 6, 14, 13)])
def test_cp_register_lu_blocks(nx, ny, nup, ndn):
    m = hubbard("densitySpin", True, nx=nx, ny=ny, nup=nup, ndn=ndn)
    W = 8
    seed = 200 + nup + ndn
    g, o = pair_cp(m, W, seed, 1000, 1000, noise=0.1)
    assert logov_close(g.log_overlaps(), o.log_overlaps(), STEP_TOL) < STEP_TOL
    for w in (0, W - 1):
        assert rel_err(g.green(w), o.green(w)) < STEP_TOL
    resync_step(g, o, seed, 2)
    wf, lw, al = o.get_walkers()
    g.set_walkers(wf, lw, al)
    for e in (g, o):
        e.reset_measurement()
        e.add_mixed_measurement()
    mg, mo = g.measurement(), o.measurement()
    assert rel_err(mg[:2], mo[:2]) < STEP_TOL
    for k in (2, 3, 4):
        assert abs(mg[k] - mo[k]) <= STEP_TOL * max(1.0, abs(mo[1]))
    check_pop_control(g, o, seed)


@pytest.mark.parametrize("n,nup,ndn", [(64, 32, 17), (64, 24, 20)])
def test_pl_register_lu_stabilize_then_step(n, nup, ndn):
    """modifyGM (SD2is::stabilize, SD2is.cpp:48-76) before the step: the
    Gram-Schmidt gauge differs from Householder's by column signs, so the
    comparison is on gauge-invariant quantities."""
    m = molecule(n=n, nup=nup, ndn=ndn, G=48)
    W = 6
    seed = 300 + nup
    g, o = pair_pl(m, W, seed, 1000, 1000, noise=0.1)
    g.modify_gm()
    o.modify_gm()
    compare_state(g, o, STEP_TOL)
    for w in (0, 3):
        for spin in (0, 1):
            assert rel_err(g.green(w, spin), o.green(w, spin)) < STEP_TOL
    g.step(1)
    o.step(1)
    compare_state(g, o, 1e-9)
