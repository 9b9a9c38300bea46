"""On-disk records (afqmclab_b200/records.py) on CPU, with the oracle engine
standing in for the GPU engine (it has the same population interface).

  - A run that writes its walker and random-stream checkpoints, is stopped and
    resumed from the files continues exactly like the uninterrupted run
    (the files carry 17 significant digits, so every double round-trips).
  - Dead walkers are not written and come back dead (readAllWalkers,
    afqmcConstraintPathSetWalker.cpp:79-88).
  - The estimator streams have writeThreadSum's semantics: with two gloo
    ranks the files hold the sum of both ranks' partial sums, written once.
"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as tmp

from afqmclab_b200 import inputs, records
from oracle import oracle as O
from tests.parity_common import hubbard, molecule


def make(kind, W, seed):
    if kind == "cp":
        m = hubbard("densitySpin", fields=True)
        e = O.cp_engine(m, W, seed, 4, 6)
        wf, lw, al = inputs.initial_walkers(m.phiT, W, seed=seed + 1, noise=0.05)
    else:
        m = molecule()
        e = O.pl_engine(m, W, seed, 4, 6)
        wf, lw, al = inputs.initial_walkers(m.phiTUp, W, seed=seed + 1, noise=0.05)
    e.set_walkers(wf, lw, al)
    return e


@pytest.mark.parametrize("kind", ["cp", "pl"])
def test_checkpoint_resume_matches_uninterrupted_run(kind, tmp_path):
    W, seed = 12, 17
    a = make(kind, W, seed)
    a.step(5)
    wf, lw, al = a.get_walkers()
    al[3] = 0                       # a dead walker is not written
    a.set_walkers(wf, lw, al)
    records.write_walkers(a, str(tmp_path))
    records.save_random(a, str(tmp_path))
    records.save_random(a, str(tmp_path))   # the earlier checkpoint moves to random.bk
    assert os.path.exists(tmp_path / "random.bk" / "checkpoint_0.dat")
    assert not os.path.exists(tmp_path / "walkers" / "phi_3.dat")
    a.set_cadence(5 % 4, 5 % 6)
    a.step(7)
    # a fresh engine (other seed) restores walkers and stream position, then resumes
    b2 = make(kind, W, 999)
    assert records.read_walkers(b2, str(tmp_path)) == W - 1
    s, c = records.read_random(b2, str(tmp_path))
    assert s == seed
    _, _, alive_b = b2.get_walkers()
    assert alive_b[3] == 0 and alive_b.sum() == W - 1
    b2.set_cadence(5 % 4, 5 % 6)
    b2.step(7)
    wa, la, aa = a.get_walkers()
    wb, lb, ab = b2.get_walkers()
    assert np.array_equal(aa, ab)
    assert np.array_equal(wa[:, :, aa.astype(bool)], wb[:, :, ab.astype(bool)])
    assert np.array_equal(la[aa.astype(bool)], lb[ab.astype(bool)])
    assert a.rng_counter() == b2.rng_counter()


@pytest.mark.parametrize("kind", ["cp", "pl"])
def test_estimator_streams_single_rank(kind, tmp_path):
    e = make(kind, 8, 5)
    e.step(2)
    sums = []
    for block in range(3):
        e.reset_measurement()
        e.add_mixed_measurement()
        sums.append(e.measurement())
        records.write_measurement(e, str(tmp_path))
        e.step(1)
    den = records.read_stream(str(tmp_path / "den.dat"))[:, 0]
    H = records.read_stream(str(tmp_path / "HNum.dat"))[:, 0]
    assert np.array_equal(den, np.array([s[0] for s in sums]))
    assert np.array_equal(H, np.array([s[1] for s in sums]))
    if kind == "cp":
        nup = records.read_stream(str(tmp_path / "NupNum.dat"), per_block=e.n // 2)
        tot = records.read_stream(str(tmp_path / "NupTotNum.dat"))[:, 0]
        assert nup.shape == (3, e.n // 2)
        assert np.allclose(nup.sum(axis=1), tot, rtol=1e-14, atol=0)
        assert np.allclose(((tot + records.read_stream(str(tmp_path / "NdnTotNum.dat"))[:, 0]) / den).real,
                           14.0, atol=1e-9)
    else:
        bg = records.read_stream(str(tmp_path / "choleskyBgNum.dat"), per_block=e.G)
        assert bg.shape == (3, e.G)
        assert np.array_equal(records.read_stream(str(tmp_path / "TNum.dat"))[:, 0],
                              np.array([s[2] for s in sums]))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _stream_worker(rank, world, port, out_dir, kind):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    e = make(kind, 6, 30 + rank)
    e.step(2)
    e.reset_measurement()
    e.add_mixed_measurement()
    np.save(os.path.join(out_dir, f"m{rank}.npy"), e.measurement())
    if kind == "pl":
        np.save(os.path.join(out_dir, f"b{rank}.npy"), e.cholesky_nums()[0])
    records.write_measurement(e, out_dir)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["cp", "pl"])
def test_estimator_streams_sum_over_two_ranks(kind, tmp_path):
    world = 2
    tmp.spawn(_stream_worker, args=(world, _free_port(), str(tmp_path), kind), nprocs=world, join=True)
    m = [np.load(tmp_path / f"m{r}.npy") for r in range(world)]
    den = records.read_stream(str(tmp_path / "den.dat"))
    H = records.read_stream(str(tmp_path / "HNum.dat"))
    assert den.shape == (1, 1)                      # written once, by rank 0
    assert abs(den[0, 0] - (m[0][0] + m[1][0])) <= 1e-15 * abs(den[0, 0])
    assert abs(H[0, 0] - (m[0][1] + m[1][1])) <= 1e-15 * abs(H[0, 0])
    if kind == "pl":
        b = [np.load(tmp_path / f"b{r}.npy") for r in range(world)]
        bg = records.read_stream(str(tmp_path / "choleskyBgNum.dat"), per_block=len(b[0]))
        assert np.allclose(bg[0], b[0] + b[1], rtol=1e-15, atol=1e-300)
