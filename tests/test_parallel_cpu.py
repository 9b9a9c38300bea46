"""Population control across ranks (afqmclab_b200/parallel.py) on CPU:
the shared comb stream and the host popConfiguration against the oracle, and
a world-size-2 gloo run against the serial table on the concatenated
population (populationControl.h:20-109)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as tmp

from afqmclab_b200 import capi, parallel
from oracle import oracle as O


def test_stream_uniforms_match_oracle():
    u = parallel.stream_uniforms(985456376, 17, 500)
    assert np.array_equal(u, O.rng_uniform(985456376, 17, 500))


@pytest.mark.parametrize("size", [1, 2, 4])
def test_host_pop_configuration_matches_oracle(size):
    rng = np.random.default_rng(size)
    L = 400
    w = rng.uniform(0, 3, L)
    w[rng.uniform(size=L) < 0.2] = 0.0
    u = rng.uniform(size=L)
    t_o, bad = O.pop_configuration(w, u, size=size)
    assert bad == 0
    assert np.array_equal(capi.pop_configuration_host(w, u, size=size), t_o)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, W, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    rng = np.random.default_rng(1234)
    allw = rng.uniform(0, 2, W * world)
    allw[rng.uniform(size=W * world) < 0.25] = 0.0
    walkers = torch.arange(W * world * 3, dtype=torch.float64).reshape(W * world, 3)
    mine = walkers[rank * W:(rank + 1) * W].clone()
    pop = parallel.ArrayPopulation(mine, allw[rank * W:(rank + 1) * W])
    table, counter = parallel.global_pop_control(pop, seed=77, counter=100)
    np.save(os.path.join(out_dir, f"r{rank}.npy"), pop.walkers.numpy())
    np.save(os.path.join(out_dir, f"t{rank}.npy"), table)
    dist.barrier()
    dist.destroy_process_group()


def test_global_pop_control_two_ranks(tmp_path):
    W, world = 40, 2
    tmp.spawn(_worker, args=(world, _free_port(), W, str(tmp_path)), nprocs=world, join=True)
    rng = np.random.default_rng(1234)
    allw = rng.uniform(0, 2, W * world)
    allw[rng.uniform(size=W * world) < 0.25] = 0.0
    table = capi.pop_configuration_host(allw, parallel.stream_uniforms(77, 100, W * world), size=world)
    walkers = np.arange(W * world * 3, dtype=np.float64).reshape(W * world, 3)
    expect = walkers[table]
    got = np.concatenate([np.load(tmp_path / f"r{r}.npy") for r in range(world)])
    assert np.array_equal(np.load(tmp_path / "t0.npy"), table)
    assert np.array_equal(np.load(tmp_path / "t1.npy"), table)
    assert np.array_equal(got, expect)
    # popConfiguration(size) keeps most copies on their own rank
    cross = sum(1 for i, j in enumerate(table) if i // W != j // W)
    assert cross < W // 2
