"""The engine side of the cross-rank population control on one GPU (a
world of one rank): pop weights, walker transfer buffers and local table
application reproduce the engine's own popControl exactly."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist

from afqmclab_b200 import capi, inputs, parallel

pytestmark = pytest.mark.gpu


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("precision", [capi.AFQMC_FP64, capi.AFQMC_MIXED])
def test_single_rank_global_pop_control_matches_engine(precision):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_port())
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        m = inputs.molecule_inputs(64, 16, 16, 128, dt=0.005, decay=30.0, seed=7)
        walkers = inputs.initial_walkers(m.phiTUp, 32, seed=3, noise=0.05)
        a = capi.pl_engine(m, 32, 21, 1000, 1000, precision=precision)
        b = capi.pl_engine(m, 32, 21, 1000, 1000, precision=precision)
        for e in (a, b):
            e.set_walkers(*walkers)
            e.step(3)
        counter = a.rng_counter()
        ta, _ = a.pop_control()
        tb, nxt = parallel.global_pop_control(parallel.EnginePopulation(b, "cuda"), seed=21,
                                              counter=counter)
        assert np.array_equal(ta, tb)
        assert nxt == a.rng_counter()
        wa, la, aa = a.get_walkers()
        wb, lb, ab = b.get_walkers()
        assert np.array_equal(aa, ab)
        assert np.allclose(wa, wb, rtol=0, atol=1e-7)
        assert np.allclose(la, lb, rtol=0, atol=1e-12)
        # a walker through the transfer buffer round-trips unchanged
        buf = torch.empty(b.walker_bytes() // 8, dtype=torch.float64, device="cuda")
        b.copy_walker_out(5, buf.data_ptr())
        b.copy_walker_in(7, buf.data_ptr())
        wb2, lb2, _ = b.get_walkers()
        assert np.array_equal(wb2[:, :, 7], wb2[:, :, 5]) and lb2[7] == lb2[5]
        a.close()
        b.close()
    finally:
        dist.destroy_process_group()
