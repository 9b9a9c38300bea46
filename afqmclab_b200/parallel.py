"""Population control across processes, one walker population per GPU.

The reference runs W/P walkers per MPI rank and, at every popControlStep,
gathers the weights on rank 0, builds the table there, scatters it and moves
walkers with MPI_Isend/Recv (populationControl<T>, populationControl.h:20-109;
popConfiguration(size, weight), populationControlConfiguration.cpp:24-101).

Here every rank all-gathers the weights, draws the comb's uniforms from one
shared counter-based stream and builds the same table itself (no scatter);
only the walkers whose parent lives on another rank move, point to point
(NCCL over NVLink between GPUs, gloo between CPU processes).  popConfiguration
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

    def pack(self, j):
        buf = torch.empty(self.words, dtype=torch.float64, device=self.device)
        self.eng.copy_walker_out(j, buf.data_ptr())
        return buf

    def empty(self):
        return torch.empty(self.words, dtype=torch.float64, device=self.device)

    def unpack(self, i, buf):
        self.eng.copy_walker_in(i, buf.data_ptr())

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

    def pack(self, j):
        return self.walkers[j].clone()

    def empty(self):
        return torch.empty_like(self.walkers[0])

    def unpack(self, i, buf):
        self.walkers[i] = buf

    def apply_local(self, table):
        for i, j in enumerate(table):
            if i != j:
                self.walkers[i] = self.walkers[j]


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
    ops, recvd = [], []
    for i, j in enumerate(table):
        ri, rj = i // W, int(j) // W
        if ri == rj:
            continue
        if rj == rank:
            ops.append(dist.P2POp(dist.isend, pop.pack(int(j) - rank * W), ri, group))
        elif ri == rank:
            buf = pop.empty()
            ops.append(dist.P2POp(dist.irecv, buf, rj, group))
            recvd.append((i - rank * W, buf))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    for i, buf in recvd:
        pop.unpack(i, buf)
    local = np.arange(W, dtype=np.int32)
    for i in range(rank * W, (rank + 1) * W):
        j = int(table[i])
        if j // W == rank:
            local[i - rank * W] = j - rank * W
    pop.apply_local(local)
    return table, counter + L
