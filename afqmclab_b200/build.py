"""Builds the engine's shared library libafqmc_b200.so in-tree with nvcc for
sm_100a (B200).  Run `python -m afqmclab_b200.build`."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libafqmc_b200.so")
SOURCES = ["engine.cu", "zgemm.cu", "walker_kernels.cu", "mixed.cu", "tc_gemm.cu", "exchange_tc.cu", "noalloc.cu", "adjoint.cu", "cp_mixed.cu", "overlap_tc.cu", "theta_tc.cu", "exchange_gemm.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "afqmc_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not needs_build():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *ARCH, "-O3", "-std=c++17", "-lineinfo", "-shared", "-Xcompiler", "-fPIC",
           "--expt-relaxed-constexpr", "-o", LIB + ".tmp", *sources(), "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
