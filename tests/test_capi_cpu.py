"""CPU-side checks of the engine library: it loads, exports every symbol the
header declares, its random stream equals the oracle's, and its argument
checks reject bad input (no GPU needed)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from afqmclab_b200 import build, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "afqmc_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(afqmc_\w+)\s*\(", src)))


def test_library_builds_and_loads():
    build.build()
    assert capi.lib().afqmc_version().startswith(b"afqmclab_b200")


def test_every_declared_symbol_is_exported():
    L = capi.lib()
    syms = declared_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(capi.SYMBOLS)


def test_create_rejects_bad_arguments():
    L = capi.lib()
    h = ctypes.c_void_p()
    r = L.afqmc_cp_create(4, 10, 0, 1, 0, 0.01, 0.0, 1.5, 10, 10, 0, *([None] * 11), 0.0, 0.0, 1,
                          ctypes.byref(h))
    assert r != 0 and h.value is None
    assert len(capi.lib().afqmc_last_error()) > 0


def test_device_rng_header_matches_oracle(tmp_path):
    """Compile the product's host/device RNG (csrc/common.cuh) for the host and
    compare its stream and Box-Muller draws with the oracle's."""
    from oracle import oracle as O
    src = tmp_path / "rng.cu"
    src.write_text('#include "common.cuh"\n#include <cstdio>\nint main(){\n'
                   '  unsigned long long ks[5]={0,1,2,1000,(1ULL<<40)+7};\n'
                   '  for(int i=0;i<5;++i) printf("%.17g %.17g\\n", rng_uniform(985456376ULL, ks[i]),'
                   ' rng_gaussian(985456376ULL, ks[i]));\n  return 0;}\n')
    exe = tmp_path / "rng"
    subprocess.check_call(["nvcc", "-O2", "-I", os.path.join(ROOT, "afqmclab_b200", "csrc"),
                           str(src), "-o", str(exe)])
    out = subprocess.check_output([str(exe)]).decode().split()
    vals = np.array(out, dtype=float).reshape(5, 2)
    for i, k in enumerate([0, 1, 2, 1000, 2**40 + 7]):
        u = O.rng_uniform(985456376, k, 2)
        assert vals[i, 0] == u[0]
        g = np.sqrt(-2 * np.log(u[0])) * np.cos(2 * 3.14159265358979324 * u[1])
        assert abs(vals[i, 1] - g) < 1e-14
