"""Population control and estimators across processes, one walker population
per GPU.

The reference runs W/P walkers per MPI rank and, at every popControlStep,
gathers the weights on rank 0, builds the table there, scatters it and moves
walkers one MPI message each (populationControl<T>, populationControl.h:20-109;
popConfiguration(size, weight), populationControlConfiguration.cpp:24-101).
Its estimators are summed over ranks before they are used or written
(HubbardSOCMeasureFixedSDSD::returnEnergy, HubbardSOCMeasureFixedSDSD.cpp:52-61).

Here every rank all-gathers the weights, draws the comb's uniforms from one
shared counter-based stream and builds the same table itself (no scatter).
Only the walkers whose parent lives on another rank move: all moves from one
rank to another are packed into one contiguous buffer by one kernel and
travel as one point-to-point message (NCCL over NVLink between GPUs, gloo
between CPU processes), then one kernel unpacks them.  popConfiguration
fills empty slots inside each rank's chunk first, so most copies stay local.
"""
import numpy as np
import torch
import torch.distributed as dist

from . import capi

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def _mix(z):
    z = (z ^ (z >> np.uint64(30))) * _M1
    z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def stream_uniforms(seed, counter, count):
    """Uniforms counter..counter+count-1 of the engine's SplitMix64 stream."""
    with np.errstate(over="ignore"):
        k = np.arange(counter, counter + count, dtype=np.uint64) + np.uint64(1)
        b = _mix(_mix(np.uint64(seed)) + k * _GOLDEN)
    return (b >> np.uint64(11)).astype(np.float64) * 2.0**-53


class EnginePopulation:
    """Adapter for a GPU engine (capi.Engine)."""

    def __init__(self, eng, device):
        self.eng, self.device = eng, device
        self.W = eng.W
        self.words = eng.walker_bytes() // 8

    def weights(self):
        return self.eng.pop_weights()

    def pack_many(self, idx):
        buf = torch.empty(len(idx) * self.words, dtype=torch.float64, device=self.device)
        self.eng.pack_walkers(idx, buf.data_ptr())
        return buf

    def empty_many(self, count):
        return torch.empty(count * self.words, dtype=torch.float64, device=self.device)

    def unpack_many(self, slots, buf):
        self.eng.unpack_walkers(slots, buf.data_ptr())

    def apply_local(self, table):
        self.eng.apply_table(table)


class ArrayPopulation:
    """A population held as rows of a tensor (walker data + weight), for CPU runs."""

    def __init__(self, walkers, weights):
        self.walkers = walkers
        self.w = np.asarray(weights, dtype=np.float64)
        self.W = walkers.shape[0]

    def weights(self):
        return self.w

    def pack_many(self, idx):
        return self.walkers[list(idx)].clone().reshape(-1)

    def empty_many(self, count):
        return torch.empty((count,) + tuple(self.walkers.shape[1:]), dtype=self.walkers.dtype).reshape(-1)

    def unpack_many(self, slots, buf):
        self.walkers[list(slots)] = buf.reshape((len(slots),) + tuple(self.walkers.shape[1:]))

    def apply_local(self, table):
        for i, j in enumerate(table):
            if i != j:
                self.walkers[i] = self.walkers[j]


def transfer_plan(table, W, rank):
    """For this rank: {peer: parents to send (local indices, table order)} and
    {peer: slots to fill (local indices, same order)}, plus the local table."""
    sends, recvs = {}, {}
    local = np.arange(W, dtype=np.int32)
    for i, j in enumerate(table):
        j = int(j)
        ri, rj = i // W, j // W
        if ri == rj:
            if ri == rank:
                local[i - rank * W] = j - rank * W
            continue
        if rj == rank:
            sends.setdefault(ri, []).append(j - rank * W)
        elif ri == rank:
            recvs.setdefault(rj, []).append(i - rank * W)
    return sends, recvs, local


def global_pop_control(pop, seed, counter, group=None, device="cpu"):
    """One population control over all ranks.  Returns (global table, next counter)."""
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    W = pop.W
    w_local = torch.tensor(pop.weights(), dtype=torch.float64, device=device)
    gathered = [torch.empty_like(w_local) for _ in range(world)]
    dist.all_gather(gathered, w_local, group=group)
    weights = torch.cat(gathered).cpu().numpy()
    L = W * world
    table = capi.pop_configuration_host(weights, stream_uniforms(seed, counter, L), size=world)
    sends, recvs, local = transfer_plan(table, W, rank)
    ops, incoming = [], []
    for peer in sorted(sends):
        ops.append(dist.P2POp(dist.isend, pop.pack_many(sends[peer]), peer, group))
    for peer in sorted(recvs):
        buf = pop.empty_many(len(recvs[peer]))
        ops.append(dist.P2POp(dist.irecv, buf, peer, group))
        incoming.append((recvs[peer], buf))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    # local copies read only this rank's own parents, which the incoming
    # walkers never overwrite (a slot filled from another rank is not a
    # parent here), so the order of the two steps is free
    pop.apply_local(local)
    for slots, buf in incoming:
        pop.unpack_many(slots, buf)
    return table, counter + L


def global_measurement(eng, group=None, device="cpu"):
    """Mixed-estimator sums of all ranks (MPISum of den, HNum, ...):
    returns the summed 5-vector of afqmc_get_measurement and, for a
    phaseless engine, the summed choleskyBgNum / choleskyExNum."""
    m = eng.measurement()
    parts = [m]
    if eng.kind == "pl":
        parts.extend(eng.cholesky_nums())
    flat = np.concatenate(parts)
    t = torch.from_numpy(flat.view(np.float64).copy()).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    tot = t.cpu().numpy().view(np.complex128)
    if eng.kind == "pl":
        G = eng.G
        return tot[:5], tot[5:5 + G], tot[5 + G:5 + 2 * G]
    return tot[:5], None, None
