"""CUDA-graph replay of the step and of the measurement gives the same
population as direct launches (same kernels, same order: identical bits)."""
import numpy as np
import pytest

from afqmclab_b200 import capi, inputs

pytestmark = pytest.mark.gpu


def _run(make, graphs, steps=13, measure_every=5):
    e = make()
    e.set_graphs(graphs)
    meas = []
    for i in range(steps):
        if i % measure_every == 0:
            e.reset_measurement()
            e.add_mixed_measurement()
            meas.append(e.measurement())
        e.step(1)
    wf, lw, al = e.get_walkers()
    out = (wf, lw, al, e.rng_counter(), np.array(meas), e.log_overlaps())
    e.close()
    return out


@pytest.mark.parametrize("kind", ["cp_fp64", "cp_mixed", "pl_fp64", "pl_mixed"])
def test_graph_replay_matches_direct_launches(kind):
    if kind.startswith("cp"):
        m = inputs.hubbard_inputs(4, 4, 7, 7)
        m.ET = -12.0
        prec = capi.AFQMC_MIXED if kind == "cp_mixed" else capi.AFQMC_FP64

        def make():
            g = capi.cp_engine(m, 32, 5, 3, 4, precision=prec)
            g.set_walkers(*inputs.initial_walkers(m.phiT, 32, seed=1, noise=0.05))
            return g
    else:
        m = inputs.molecule_inputs(64, 16, 16, 128, dt=0.005, decay=30.0, seed=7)
        prec = capi.AFQMC_MIXED if kind == "pl_mixed" else capi.AFQMC_FP64

        def make():
            g = capi.pl_engine(m, 32, 9, 3, 4, precision=prec)
            g.set_walkers(*inputs.initial_walkers(m.phiTUp, 32, seed=2, noise=0.02))
            return g
    a = _run(make, False)
    b = _run(make, True)
    assert (a[2] == b[2]).all()
    assert a[3] == b[3]
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[4], b[4])
