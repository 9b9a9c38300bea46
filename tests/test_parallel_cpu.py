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


# ------------------------------------------------ engines as the populations
class OraclePopulation:
    """The oracle engine behind the same population interface as a GPU
    engine (parallel.EnginePopulation): weights, batched pack / unpack of
    transfer records (matrix + logw), local copies."""

    def __init__(self, eng):
        self.eng, self.W = eng, eng.W

    def weights(self):
        return self.eng.pop_weights()

    def pack_many(self, idx):
        wf, lw, _ = self.eng.get_walkers()
        recs = [np.concatenate([wf[:, :, j].ravel(order="F"), [lw[j]]]) for j in idx]
        return torch.from_numpy(np.concatenate(recs).view(np.float64).copy())

    def empty_many(self, count):
        return torch.empty(count * (self.eng.n * self.eng.ncol + 1) * 2, dtype=torch.float64)

    def unpack_many(self, slots, buf):
        wf, lw, al = self.eng.get_walkers()
        z = buf.numpy().view(np.complex128).reshape(len(slots), -1)
        for k, i in enumerate(slots):
            wf[:, :, i] = z[k, :-1].reshape(wf.shape[:2], order="F")
            lw[i] = z[k, -1]
        self.eng.set_walkers(wf, lw, al)

    def apply_local(self, table):
        wf, lw, al = self.eng.get_walkers()
        self.eng.set_walkers(wf[:, :, table], lw[table], al)


def _engine_worker(rank, world, port, W, out_dir):
    from afqmclab_b200 import inputs
    from tests.parity_common import molecule
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    m = molecule()
    e = O.pl_engine(m, W, 50 + rank, 1000, 1000)
    wf, lw, al = inputs.initial_walkers(m.phiTUp, W, seed=60 + rank, noise=0.1)
    e.set_walkers(wf, lw, al)
    e.step(3)
    wf0, lw0, al0 = e.get_walkers()
    np.save(os.path.join(out_dir, f"before{rank}.npy"), wf0)
    np.save(os.path.join(out_dir, f"lwbefore{rank}.npy"), lw0)
    np.save(os.path.join(out_dir, f"albefore{rank}.npy"), al0)
    pop = OraclePopulation(e)
    table, counter = parallel.global_pop_control(pop, seed=91, counter=7)
    wf1, lw1, al1 = e.get_walkers()
    np.save(os.path.join(out_dir, f"after{rank}.npy"), wf1)
    np.save(os.path.join(out_dir, f"lwafter{rank}.npy"), lw1)
    np.save(os.path.join(out_dir, f"table{rank}.npy"), table)
    e.reset_measurement()
    e.add_mixed_measurement()
    tot, bg, ex = parallel.global_measurement(e)
    np.save(os.path.join(out_dir, f"meas{rank}.npy"), e.measurement())
    np.save(os.path.join(out_dir, f"tot{rank}.npy"), tot)
    dist.barrier()
    dist.destroy_process_group()


def test_global_pop_control_of_engines_matches_one_population(tmp_path):
    """Two ranks of oracle engines: after the cross-rank population control
    the concatenated populations equal one population of 2W walkers to which
    the weights half of popControl and the popConfiguration(size=2) table
    were applied; the cross-rank estimator sums are the sums of both ranks."""
    from afqmclab_b200 import inputs
    from tests.parity_common import molecule
    W, world = 10, 2
    tmp.spawn(_engine_worker, args=(world, _free_port(), W, str(tmp_path)), nprocs=world, join=True)
    m = molecule()
    before = np.concatenate([np.load(tmp_path / f"before{r}.npy") for r in range(world)], axis=2)
    lwb = np.concatenate([np.load(tmp_path / f"lwbefore{r}.npy") for r in range(world)])
    alb = np.concatenate([np.load(tmp_path / f"albefore{r}.npy") for r in range(world)])
    one = O.pl_engine(m, W * world, 1, 1000, 1000)
    one.set_walkers(before, lwb, alb)
    weights = one.pop_weights()
    wf1, lw1, _ = one.get_walkers()
    table = capi.pop_configuration_host(weights, parallel.stream_uniforms(91, 7, W * world), size=world)
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / f"table{r}.npy"), table)
    after = np.concatenate([np.load(tmp_path / f"after{r}.npy") for r in range(world)], axis=2)
    lwa = np.concatenate([np.load(tmp_path / f"lwafter{r}.npy") for r in range(world)])
    assert np.array_equal(after, wf1[:, :, table])
    assert np.array_equal(lwa, lw1[table])
    assert any(i // W != int(j) // W for i, j in enumerate(table)), "no walker changed rank"
    meas = [np.load(tmp_path / f"meas{r}.npy") for r in range(world)]
    for r in range(world):
        assert np.allclose(np.load(tmp_path / f"tot{r}.npy"), meas[0] + meas[1], rtol=1e-15, atol=0)
