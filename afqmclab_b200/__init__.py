"""B200-native AFQMC walker-step engine (hshi/AFQMCLAB hot path).

The compute path is the C-ABI library libafqmc_b200.so (hand-written sm_100a
kernels, include/afqmc_b200.h); `capi` binds it, `inputs` builds seeded
synthetic Hamiltonians and trials in the reference's formats.
"""
from . import inputs  # noqa: F401

__all__ = ["capi", "inputs", "build"]
