"""On-disk records of a run, in the reference's formats, so that a run can
stop and resume and the reference's analysis scripts read its output.

  - Walker checkpoint: walkers/phi_<i>.dat, one file per live walker, i the
    global walker index (AfqmcConstraintPath::writeWalkers and the
    "readAllWalkers" start, afqmcConstraintPathSetWalker.cpp:79-120; the
    phaseless driver's twins, afqmcPhaselessSetWalker.cpp:79-120), each in
    the SD / SD2is file format (SD.cpp:85-103, SD2is.cpp:105-127).
  - Random-stream checkpoint: random/checkpoint_<rank>.dat, an int byte count
    then the packed state (randomHaoSave / randomHaoRead,
    common/randomHao/source/random_hao.cpp:33-71).  The engine's stream is
    counter based, so the packed state is its (seed, counter) pair; the
    previous checkpoint is kept in random.bk as the reference does.
  - Estimator streams: den.dat, HNum.dat, ... appended once per block
    (HubbardSOCMeasureFixedSDSD::write, HubbardSOCMeasureFixedSDSD.cpp:118-136;
    RealMaterialMoleculeMeasureFixedSD2sSD2is::write, :118-125), with
    writeThreadSum's semantics (writeThreadSum.h:11-26): the partial sums of
    all ranks are added and rank 0 writes.

Multi-rank use goes through torch.distributed when a process group is
initialised (gloo or NCCL); with none, the caller is rank 0 of one.
"""
import os
import shutil
import struct

import numpy as np

from . import inputs

_SEED_COUNTER = struct.Struct("<QQ")


def rank_world():
    try:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            return dist.get_rank(), dist.get_world_size()
    except Exception:
        pass
    return 0, 1


def _barrier():
    rank, world = rank_world()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def sum_over_ranks(a):
    """writeThreadSum's MPISum: element-wise sum of a complex array over ranks."""
    rank, world = rank_world()
    a = np.ascontiguousarray(a, dtype=np.complex128)
    if world == 1:
        return a
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(a.view(np.float64).copy())
    if dist.get_backend() == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy().view(np.complex128)


# ------------------------------------------------------------------ walkers
def write_walkers(eng, directory=".", walkers_per_rank=None):
    """writeWalkers: rank 0 replaces `directory`/walkers, then every rank
    writes its live walkers as phi_<rank*walkers_per_rank + i>.dat."""
    rank, _ = rank_world()
    base_dir = os.path.join(directory, "walkers")
    if rank == 0:
        shutil.rmtree(base_dir, ignore_errors=True)
        os.makedirs(base_dir, exist_ok=True)
    _barrier()
    per = walkers_per_rank or eng.W
    wf, logw, alive = eng.get_walkers()
    for i in range(eng.W):
        if not alive[i]:
            continue
        path = os.path.join(base_dir, f"phi_{rank * per + i}.dat")
        if eng.kind == "pl":
            inputs.write_sd2is(wf[:, :, i], logw[i], eng.nup, eng.ndn, path)
        else:
            inputs.write_sd(wf[:, :, i], logw[i], path)
    _barrier()


def read_walkers(eng, directory=".", walkers_per_rank=None, seed=0):
    """The "readAllWalkers" start: slot i reads phi_<rank*walkers_per_rank + i>.dat
    and is alive; a slot without a file gets a seeded random normalised
    matrix and is dead (fillWalkerRandomly, walkerIsAlive = false), so the
    next population control refills it."""
    rank, _ = rank_world()
    per = walkers_per_rank or eng.W
    rng = np.random.default_rng(seed + rank)
    wf = np.zeros((eng.n, eng.ncol, eng.W), np.complex128, order="F")
    logw = np.zeros(eng.W, np.complex128)
    alive = np.zeros(eng.W, np.int32)
    for i in range(eng.W):
        path = os.path.join(directory, "walkers", f"phi_{rank * per + i}.dat")
        if os.path.exists(path):
            if eng.kind == "pl":
                m, lw, nup, ndn = inputs.read_sd2is(path)
                if (nup, ndn) != (eng.nup, eng.ndn):
                    raise ValueError(f"{path}: Nup/Ndn {nup}/{ndn}, engine has {eng.nup}/{eng.ndn}")
            else:
                m, lw = inputs.read_sd(path)
            if m.shape != (eng.n, eng.ncol):
                raise ValueError(f"{path}: walker shape {m.shape}, engine has {(eng.n, eng.ncol)}")
            wf[:, :, i] = m
            logw[i] = lw
            alive[i] = 1
        else:
            q, _ = np.linalg.qr(rng.standard_normal((eng.n, eng.ncol))
                                + 1j * rng.standard_normal((eng.n, eng.ncol)))
            wf[:, :, i] = q
    eng.set_walkers(wf, logw, alive)
    return int(alive.sum())


# ------------------------------------------------------------ random stream
def save_random(eng, directory="."):
    """randomHaoSave: rank 0 moves random/ to random.bk, then every rank
    writes random/checkpoint_<rank>.dat (int size, then the packed state)."""
    rank, _ = rank_world()
    rdir = os.path.join(directory, "random")
    bk = os.path.join(directory, "random.bk")
    if rank == 0:
        os.makedirs(rdir, exist_ok=True)
        shutil.rmtree(bk, ignore_errors=True)
        os.makedirs(bk, exist_ok=True)
        for f in os.listdir(rdir):
            shutil.move(os.path.join(rdir, f), os.path.join(bk, f))
    _barrier()
    seed, counter = eng.rng_state()
    packed = _SEED_COUNTER.pack(seed, counter)
    with open(os.path.join(rdir, f"checkpoint_{rank}.dat"), "wb") as f:
        f.write(struct.pack("<i", len(packed)) + packed)
    _barrier()


def read_random(eng, directory="."):
    """randomHaoRead: restore this rank's (seed, counter) from its checkpoint."""
    rank, _ = rank_world()
    with open(os.path.join(directory, "random", f"checkpoint_{rank}.dat"), "rb") as f:
        size = struct.unpack("<i", f.read(4))[0]
        packed = f.read(size)
    if size != _SEED_COUNTER.size or len(packed) != size:
        raise ValueError("random checkpoint: not a (seed, counter) record")
    seed, counter = _SEED_COUNTER.unpack(packed)
    eng.set_rng(seed, counter)
    return seed, counter


# --------------------------------------------------------- estimator streams
def _append_complex(path, values):
    with open(path, "a") as f:
        for z in np.atleast_1d(values):
            f.write(f"{z.real:26.16e}{z.imag:26.16e}\n")


def write_measurement(eng, directory="."):
    """ModelMeasureMixed::write: append this block's sums to the estimator
    files (summed over ranks, written by rank 0).  Constrained path: den,
    KNum, VNum, RNum, HNum, NupNum, NdnNum, SplusNum, SminusNum and their
    totals; phaseless: den, TNum, choleskyBgNum, choleskyExNum, HNum."""
    rank, _ = rank_world()
    m = eng.measurement()
    if eng.kind == "cp":
        site = eng.site_nums()
        parts = np.concatenate([m[:5], *site, [s.sum() for s in site]])
        tot = sum_over_ranks(parts)
        L = len(site[0])
        if rank == 0:
            den, H, K, V, R = tot[:5]
            for name, val in (("den", den), ("KNum", K), ("VNum", V), ("RNum", R), ("HNum", H)):
                _append_complex(os.path.join(directory, name + ".dat"), val)
            off = 5
            for name in ("NupNum", "NdnNum", "SplusNum", "SminusNum"):
                _append_complex(os.path.join(directory, name + ".dat"), tot[off:off + L])
                off += L
            for name in ("NupTotNum", "NdnTotNum", "SplusTotNum", "SminusTotNum"):
                _append_complex(os.path.join(directory, name + ".dat"), tot[off])
                off += 1
        if getattr(eng, "observe", False):
            # HubbardSOCMeasureObserveSDSD::write (HubbardSOCMeasureObserveSDSD.cpp:51-60)
            obs = eng.observables()
            names = ["greenMatrixNum", "densityDensityNum", "splusSminusNum", "sminusSplusNum",
                     "spairSpairNum"]
            tot = sum_over_ranks(np.concatenate([obs[k].ravel(order="F") for k in names]))
            off = 0
            for k in names:
                size = obs[k].size
                if rank == 0:
                    _append_complex(os.path.join(directory, k + ".dat"), tot[off:off + size])
                off += size
    else:
        bg, ex = eng.cholesky_nums()
        parts = np.concatenate([m[:3], bg, ex])
        tot = sum_over_ranks(parts)
        G = len(bg)
        if rank == 0:
            den, H, T = tot[:3]
            _append_complex(os.path.join(directory, "den.dat"), den)
            _append_complex(os.path.join(directory, "TNum.dat"), T)
            _append_complex(os.path.join(directory, "choleskyBgNum.dat"), tot[3:3 + G])
            _append_complex(os.path.join(directory, "choleskyExNum.dat"), tot[3 + G:3 + 2 * G])
            _append_complex(os.path.join(directory, "HNum.dat"), H)
    _barrier()


def read_stream(path, per_block=1):
    """An estimator file as a (blocks, per_block) complex array."""
    vals = np.loadtxt(path, ndmin=2)
    z = vals[:, 0] + 1j * vals[:, 1]
    return z.reshape(-1, per_block)
