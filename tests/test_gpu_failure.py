"""Failure detection, tested without faulting the GPU.

  - Walkers with a zero column (singular overlap) or a NaN entry are injected
    through the C-ABI.  The singular one must get the reference's log-det,
    lognorm -1e300 for each singular spin block (lognormPhaseDeterminant,
    tensor_2d_common_fun.cpp:75-84, summed over the blocks as
    SD2sSD2isOperation.cpp:84-94 does), and set status bit 1 in the step; the
    NaN one sets status bit 2.  The healthy
    walkers must still match the oracle, and the engine must stay usable.
  - The bounded waits of the tensor-core kernels: a CTA waits, with the same
    wait helpers, on mbarriers that nothing arrives at and a short limit; both
    waits must give up and report, and the context must stay usable (a
    tensor-core GEMM runs correctly right after).
"""
import time

import numpy as np
import pytest

from afqmclab_b200 import capi
from tests.helpers import logov_close, rel_err
from tests.parity_common import STEP_TOL, hubbard, molecule, pair_cp, pair_pl

pytestmark = pytest.mark.gpu


def _inject(wf):
    wf = wf.copy(order="F")
    wf[:, 2, 1] = 0.0                 # walker 1: zero column -> singular overlap
    wf[3, 0, 3] = np.nan              # walker 3: non-finite entry
    return wf


def _check_injected(g, o, healthy, seed):
    lg = g.log_overlaps()
    lo = o.log_overlaps()
    # each singular spin block adds -1e300 (one block for SD, two for this
    # SD2is walker, whose zero column lies in both blocks)
    assert lg[1].real == lo[1].real and lo[1].real <= -1e300
    assert not np.isfinite(lg[3])
    assert logov_close(lg[healthy], lo[healthy], STEP_TOL) < STEP_TOL
    assert g.status() == 0               # diagnostics record no status
    g.step(1)
    o.step(1)
    st = g.status()
    assert st & 1, f"singular overlap not reported (status {st})"
    assert st & 2, f"non-finite walker not reported (status {st})"
    assert g.rng_counter() == o.rng_counter()
    lg, lo = g.log_overlaps(), o.log_overlaps()
    _, _, ao = o.get_walkers()
    h = [w for w in healthy if ao[w]]
    assert h and logov_close(lg[h], lo[h], STEP_TOL) < STEP_TOL
    # the engine stays usable: healthy walkers everywhere, one more step
    wf, lw, al = o.get_walkers()
    for bad in (1, 3):
        wf[:, :, bad] = wf[:, :, healthy[0]]
        lw[bad] = lw[healthy[0]]
        al[bad] = 1
    o.set_walkers(wf, lw, al)
    g.set_walkers(wf, lw, al)
    g.set_rng(seed, o.rng_counter())
    g.step(1)
    o.step(1)
    assert logov_close(g.log_overlaps(), o.log_overlaps(), STEP_TOL) < STEP_TOL


def test_cp_singular_and_nonfinite_walkers():
    m = hubbard("densitySpin", fields=True)
    W = 6
    g, o = pair_cp(m, W, 61, 1000, 1000, noise=0.05)
    wf, lw, al = o.get_walkers()
    wf = _inject(wf)
    g.set_walkers(wf, lw, al)
    o.set_walkers(wf, lw, al)
    _check_injected(g, o, [0, 2, 4, 5], 61)


def test_pl_singular_and_nonfinite_walkers():
    m = molecule(n=16, nup=4, ndn=3, G=24)
    W = 6
    g, o = pair_pl(m, W, 62, 1000, 1000, noise=0.05)
    wf, lw, al = o.get_walkers()
    wf = _inject(wf)
    g.set_walkers(wf, lw, al)
    o.set_walkers(wf, lw, al)
    _check_injected(g, o, [0, 2, 4, 5], 62)


def test_bounded_waits_give_up_and_report():
    import torch
    limit = 2_000_000                  # about 1 ms of SM cycles
    t0 = time.perf_counter()
    bits = capi.bounded_wait_check(limit)
    dt = time.perf_counter() - t0
    assert bits == 3, f"wait bits {bits}"
    assert dt < 5.0
    # the context is still usable: a tcgen05 GEMM right after
    M, N, K = 256, 128, 256
    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    C = torch.zeros(N, M, device="cuda", dtype=torch.float32)
    capi.gemm_bf16_dev(M, N, K, A.data_ptr(), K, B.data_ptr(), K, C.data_ptr(), M)
    ref = (B.float() @ A.float().T)
    assert rel_err(C.cpu().numpy(), ref.cpu().numpy()) < 2e-5
