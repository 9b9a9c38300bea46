"""Builds the engine's shared library libafqmc_b200.so in-tree with nvcc for
sm_100a (B200).  Run `python -m afqmclab_b200.build`.

Each source is compiled to an object under _build/ (in parallel, and only
when the source or a header changed), then the objects are linked into the
shared library."""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libafqmc_b200.so")
SOURCES = ["engine.cu", "zgemm.cu", "walker_kernels.cu", "mixed.cu", "tc_gemm.cu", "exchange_tc.cu",
           "noalloc.cu", "adjoint.cu", "cp_mixed.cu", "overlap_tc.cu", "theta_tc.cu",
           "exchange_gemm.cu", "exchange_f64.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
HEADER = os.path.join(os.path.dirname(HERE), "include", "afqmc_b200.h")


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    return hs + [HEADER]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def needs_build():
    deps = sources() + _headers()
    return _stale(LIB, deps)


def build(force=False, verbose=False, jobs=None):
    if not force and not needs_build():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(OBJ, exist_ok=True)
    headers = _headers()
    objs = []
    todo = []
    for src in sources():
        obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            todo.append([nvcc, *ARCH, *FLAGS, "-c", "-o", obj + ".tmp", src])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd, cwd=CSRC)
        os.replace(cmd[cmd.index("-o") + 1], cmd[cmd.index("-o") + 1][:-4])

    with ThreadPoolExecutor(max_workers=jobs or min(len(todo) or 1, os.cpu_count() or 1)) as ex:
        list(ex.map(run, todo))
    link = [nvcc, *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lcudart"]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.check_call(link, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
