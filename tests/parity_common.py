"""Shared set-up of the GPU-engine / oracle parity tests: seeded models,
engine-oracle pairs on identical walkers and random streams, and the
comparison of gauge-invariant state (alive flags, random-stream counter,
log-overlaps with their phase mod 2 pi).

Tolerances of the plain FP64 form: 1e-10 per step from identical walkers,
1e-8 over a multi-step trajectory."""
import os

import numpy as np

from afqmclab_b200 import capi, inputs
from oracle import oracle as O
from tests.helpers import logov_close

STEP_TOL = 1e-10
TRAJ_TOL = 1e-8
ORACLE_THREADS = os.cpu_count() or 1


def hubbard(decomp="densitySpin", fields=False, nx=4, ny=4, nup=7, ndn=7, **kw):
    m = inputs.hubbard_inputs(nx, ny, nup, ndn, decomp=decomp, **kw)
    if fields:
        rng = np.random.default_rng(4)
        L = m.L
        m.mu = rng.uniform(-0.3, 0.3, L)
        m.hx = rng.uniform(-0.4, 0.4, L)
        m.hy = rng.uniform(-0.4, 0.4, L)
        m.hz = rng.uniform(-0.4, 0.4, L)
    m.ET = -12.0
    return m


def molecule(n=16, nup=4, ndn=3, G=24, **kw):
    m = inputs.molecule_inputs(n, nup, ndn, G, dt=0.01, decay=6.0, **kw)
    m.ET = -3.0
    return m


def pair_cp(m, W, seed, mgs, pop, force="dynamicForce", noise=0.05):
    g = capi.cp_engine(m, W, seed, mgs, pop, force)
    o = O.cp_engine(m, W, seed, mgs, pop, force)
    o.set_threads(ORACLE_THREADS)
    wf, lw, al = inputs.initial_walkers(m.phiT, W, seed=seed + 1, noise=noise)
    o.set_walkers(wf, lw, al)
    g.set_walkers(wf, lw, al)
    return g, o


def pair_pl(m, W, seed, mgs, pop, log_one_body=False, force="dynamicForce", noise=0.05):
    g = capi.pl_engine(m, W, seed, mgs, pop, force, log_one_body=log_one_body)
    o = O.pl_engine(m, W, seed, mgs, pop, force, log_one_body=log_one_body)
    o.set_threads(ORACLE_THREADS)
    wf, lw, al = inputs.initial_walkers(m.phiTUp, W, seed=seed + 1, noise=noise)
    o.set_walkers(wf, lw, al)
    g.set_walkers(wf, lw, al)
    return g, o


def compare_state(g, o, tol):
    _, _, ag = g.get_walkers()
    _, _, ao = o.get_walkers()
    assert (ag == ao).all(), "alive flags differ"
    assert g.rng_counter() == o.rng_counter()
    lg, lo = g.log_overlaps(), o.log_overlaps()
    alive = ao.astype(bool)
    err = logov_close(lg[alive], lo[alive], tol)
    assert err < tol, f"log-overlap mismatch {err}"
    return err
