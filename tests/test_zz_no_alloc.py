"""The allocation-free popConfiguration entry point.

Callers that cannot allocate device memory where they need a population-
control table (their GPU memory is owned by a host framework's pool, or fixed
at start-up, or the loop cannot take an allocation's synchronisation) use
afqmc_pop_configuration_noalloc_dev, whose scratch is a file-scope device
array.  Checked through the C ABI against the allocating entry point
afqmc_pop_configuration_dev on two calls in a row; the tables are integers,
so they must agree exactly.
"""
import numpy as np
import pytest
import torch

from afqmclab_b200 import capi

pytestmark = pytest.mark.gpu


def _dev(a, dtype):
    return torch.tensor(a, device="cuda", dtype=dtype)


def test_noalloc_pop_configuration_matches_allocating_entry_point():
    rng = np.random.default_rng(2024)
    # two calls in a row; the second is larger, so it also covers counts the
    # first call left behind in the shared scratch array
    for W in (3000, 4096):
        w = rng.uniform(0.0, 2.0, W)
        w[rng.uniform(size=W) < 0.15] = 0.0
        u = rng.uniform(size=W)
        tw, tu = _dev(w, torch.float64), _dev(u, torch.float64)
        t_ref = torch.full((W,), -7, device="cuda", dtype=torch.int32)
        t_new = torch.full((W,), -7, device="cuda", dtype=torch.int32)
        capi.pop_configuration_dev(tw.data_ptr(), tu.data_ptr(), t_ref.data_ptr(), W)
        capi.pop_configuration_noalloc_dev(tw.data_ptr(), tu.data_ptr(), t_new.data_ptr(), W)
        torch.cuda.synchronize()
        ref, new = t_ref.cpu().numpy(), t_new.cpu().numpy()
        assert (ref >= 0).all()
        assert np.array_equal(new, ref)


def test_noalloc_pop_configuration_at_and_below_its_limit():
    """W at the scratch limit, then sizes that run the serial comb kernel
    (above the parallel comb's shared-memory capacity) and the parallel one,
    in falling order, so that every call after the first finds larger counts
    from the previous call in the shared array and reuses the cached device
    address.  Checked against the allocating entry point and the oracle's
    comb (populationControlConfiguration.cpp:24-101)."""
    from oracle import oracle as O
    rng = np.random.default_rng(77)
    for W in (capi_max(), 20000, 4096):
        w = rng.uniform(0.0, 2.0, W)
        w[rng.uniform(size=W) < 0.2] = 0.0
        u = rng.uniform(size=W)
        tw, tu = _dev(w, torch.float64), _dev(u, torch.float64)
        t_ref = torch.full((W,), -7, device="cuda", dtype=torch.int32)
        t_new = torch.full((W,), -7, device="cuda", dtype=torch.int32)
        capi.pop_configuration_dev(tw.data_ptr(), tu.data_ptr(), t_ref.data_ptr(), W)
        capi.pop_configuration_noalloc_dev(tw.data_ptr(), tu.data_ptr(), t_new.data_ptr(), W)
        torch.cuda.synchronize()
        ref, new = t_ref.cpu().numpy(), t_new.cpu().numpy()
        table_o, _ = O.pop_configuration(w, u)
        assert np.array_equal(ref, table_o)
        assert np.array_equal(new, ref)


def capi_max():
    """AFQMC_NOALLOC_MAX_WALKERS as the header declares it."""
    import os
    import re
    hdr = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                       "afqmc_b200.h")
    return int(re.search(r"#define AFQMC_NOALLOC_MAX_WALKERS (\d+)", open(hdr).read()).group(1))


def test_noalloc_pop_configuration_rejects_sizes_above_its_scratch():
    W = capi_max() + 1
    t = torch.zeros(4, device="cuda", dtype=torch.float64)
    with pytest.raises(capi.AfqmcError, match="scratch limit"):
        capi.pop_configuration_noalloc_dev(t.data_ptr(), t.data_ptr(), t.data_ptr(), W)
