"""Runs the reference's own tutorial programs (oracle/_ref/afqmcConstraintPath
and oracle/_ref/afqmcPhaseless, built from the reference's sources by
oracle/ref/Makefile) on inputs written in the reference's file formats, and
reads back the estimator streams they write.

TEST INFRASTRUCTURE ONLY: used by tests/ to pin the oracle against the
reference itself, and by the CPU legs of bench.py; never by the product.

Inputs written per run, in a scratch directory the program runs in:
  - afqmc_param: key/value lines read by readBySearchString
    (AfqmcConstraintPathMethod::read, afqmcConstraintPathMethod.cpp:19-46;
    AfqmcPhaselessMethod::read, afqmcPhaselessMethod.cpp:19-46);
  - model_param: HubbardSOC's text format (HubbardSOC.cpp:39-60), or for the
    molecule the HDF5 stand-in container that RealMaterialMolecule::read
    (realMaterialMolecule.cpp:41-60) reads through the build's H5Cpp shim;
  - phiT.dat and walkers/phi_<i>.dat ("readFromFile" / "readAllWalkers",
    afqmcConstraintPathSetWalker.cpp:9-120, afqmcPhaselessSetWalker.cpp:9-120).

Random numbers: the build's SPRNG stand-in is the SplitMix64 stream that the
oracle and the engine use (uniform k of seed s = or_rng_uniform_at(s, k)),
consumed in the reference's own order.  Before the projection the programs
draw one auxiliary-field sample in estimateMemory
(afqmcConstraintPath.cpp:60-62, afqmcPhaseless.cpp:86-88): L uniforms for
the Hubbard model (NiupNidn::sampleAuxFromForce), 2G for the molecule (G
gaussianHao calls), so a trajectory of the oracle that starts at that
counter follows the program's.
"""
import os
import shutil
import struct
import subprocess
import sys
import tempfile
import time

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.normpath(os.path.join(_HERE, "..", "_ref"))
PROGRAMS = {"cp": "afqmcConstraintPath", "pl": "afqmcPhaseless", "bp": "afqmcConstraintPathBP"}

sys.path.insert(0, os.path.normpath(os.path.join(_HERE, "..", "..")))
from afqmclab_b200 import inputs  # noqa: E402


def program(kind):
    return os.path.join(REF_DIR, PROGRAMS[kind])


def available(kind="cp"):
    return os.access(program(kind), os.X_OK)


def build(reference="/root/reference"):
    """Compile the programs from the reference's sources (only where they are)."""
    if not os.path.isdir(reference):
        return False
    subprocess.check_call(["make", "-s", "-j8", "-C", _HERE, f"REF={reference}"])
    return True


def rng_offset(kind, m):
    """Uniforms the program draws in estimateMemory, before its first
    projection step."""
    return m.L if kind in ("cp", "bp") else 2 * m.G


def start_like_program(eng, kind, m, seed):
    """Bring an engine (the oracle's or the CUDA one) holding the walkers the
    program reads to the state the program starts projecting from:
    initialMgsAndPopControl (modifyGM, then popControl, at the start of the
    stream; afqmcConstraintPathSetWalker.cpp:120-124, afqmcPhaselessSetWalker.cpp:
    122-126), then the stream advanced past estimateMemory's draws."""
    eng.set_rng(seed, 0)
    eng.modify_gm()
    eng.pop_control()
    eng.set_rng(seed, eng.rng_counter() + rng_offset(kind, m))


# ----------------------------------------------------------------- writers
def write_container(path, entries):
    """The HDF5 stand-in container (shim/h5_shim.cpp): "AFQH5SH1", a count,
    then per dataset its name, rank, dims and bytes.  Scalars are rank-1
    datasets of one element, as writeFile(size_t/double) creates them."""
    with open(path, "wb") as f:
        f.write(b"AFQH5SH1")
        f.write(struct.pack("<Q", len(entries)))
        for name, arr in entries:
            raw = np.ascontiguousarray(arr).tobytes(order="C")
            key = name.encode()
            f.write(struct.pack("<Q", len(key)) + key)
            f.write(struct.pack("<QQ", 1, np.asarray(arr).size))
            f.write(struct.pack("<Q", len(raw)) + raw)


def write_molecule_model_param(m, path):
    """RealMaterialMolecule::write's datasets (realMaterialMolecule.cpp:62-76)."""
    u64 = np.uint64
    write_container(path, [
        ("L", np.array([m.n], u64)), ("Nup", np.array([m.nup], u64)),
        ("Ndn", np.array([m.ndn], u64)), ("choleskyNumber", np.array([m.G], u64)),
        ("t", np.asarray(m.t, np.float64).ravel(order="F")),
        ("K", np.asarray(m.K, np.float64).ravel(order="F")),
        ("choleskyVecs", np.asarray(m.chol, np.float64).ravel(order="F")),
        ("choleskyBg", np.asarray(m.bg, np.float64).ravel()),
    ])


def write_afqmc_param(path, params):
    with open(path, "w") as f:
        for k, v in params.items():
            f.write(f"{k} {v}\n")


def _sd2s_write(phiTUp, phiTDn, logw, path):
    """SD2s::write (SD2s.cpp:114-123): logw, then the two matrices."""
    with open(path, "w") as f:
        f.write(inputs._complex_line(logw))
        for wf in (phiTUp, phiTDn):
            f.write("".join(inputs._matrix_lines(np.asfortranarray(wf))))


# ------------------------------------------------------------------ runs
def _blas_env(threads):
    env = dict(os.environ)
    if "AFQMC_ORACLE_BLAS" not in env:
        import glob
        import scipy
        libs = glob.glob(os.path.join(os.path.dirname(scipy.__file__) + ".libs",
                                      "libscipy_openblas*.so"))
        if not libs:
            raise RuntimeError("no OpenBLAS for the reference programs")
        env["AFQMC_ORACLE_BLAS"] = libs[0]
        env["AFQMC_ORACLE_BLAS_PREFIX"] = "scipy_"
    env["OPENBLAS_NUM_THREADS"] = str(threads)
    return env


def _run(kind, workdir, threads, timeout):
    env = _blas_env(threads)
    r = subprocess.run([program(kind)], cwd=workdir, env=env, capture_output=True, text=True,
                       timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{PROGRAMS[kind]} exited {r.returncode}: {r.stdout[-2000:]}{r.stderr[-2000:]}")
    return r.stdout


def _streams(workdir, names):
    out = {}
    for name in names:
        p = os.path.join(workdir, name + ".dat")
        if os.path.exists(p):
            v = np.loadtxt(p, ndmin=2)
            out[name] = v[:, 0] + 1j * v[:, 1]
    return out


def _final_walkers(workdir, kind, shape):
    """The walkers prepareStop writes (writeWalkers after the closing half
    step): (wf, logw, alive), dead slots zero."""
    n, ncol, W = shape
    wf = np.zeros(shape, np.complex128, order="F")
    logw = np.zeros(W, np.complex128)
    alive = np.zeros(W, np.int32)
    for i in range(W):
        p = os.path.join(workdir, "walkers", f"phi_{i}.dat")
        if os.path.exists(p):
            if kind == "pl":
                m, lw, _, _ = inputs.read_sd2is(p)
            else:
                m, lw = inputs.read_sd(p)
            wf[:, :, i] = m
            logw[i] = lw
            alive[i] = 1
    return wf, logw, alive


def _common_params(method, W, seed, force_type, force_cap, mgs_step, pop_step, ET):
    return {
        "dt": repr(float(method.dt)), "thermalSize": method.thermalSize,
        "writeNumber": method.writeNumber, "measureNumberPerWrite": method.measureNumberPerWrite,
        "measureSkipStep": method.measureSkipStep, "walkerSizePerThread": W,
        "forceType": force_type, "forceCap": repr(float(force_cap)),
        "initialPhiTFlag": "readFromFile", "initialWalkerFlag": "readAllWalkers",
        "mgsStep": mgs_step, "popControlStep": pop_step, "ET": repr(float(ET)), "seed": seed,
    }


def stage_model(kind, m, directory):
    """Write model_param and phiT.dat once, for runs that link them."""
    os.makedirs(directory, exist_ok=True)
    if kind == "cp":
        inputs.write_hubbard_model_param(m, os.path.join(directory, "model_param"))
        inputs.write_sd(m.phiT, m.logwT, os.path.join(directory, "phiT.dat"))
    else:
        write_molecule_model_param(m, os.path.join(directory, "model_param"))
        _sd2s_write(m.phiTUp, m.phiTDn, m.logwT, os.path.join(directory, "phiT.dat"))


def prepare(kind, m, method, wf, logw, seed, mgs_step, pop_step, force_type, workdir,
            model_dir=None):
    """Write one run's inputs into `workdir`: afqmc_param, the walkers, and
    model_param / phiT.dat (linked from `model_dir` when given)."""
    W = wf.shape[2]
    p = _common_params(method, W, seed, force_type, m.force_cap, mgs_step, pop_step, m.ET)
    if kind == "cp":
        p.update({"decompType": m.decomp, "ETAdjustStep": method.ETAdjustStep,
                  "ETAdjustMaxSize": method.ETAdjustMaxSize})
    else:
        p.update({
            "ETAndBackGroundAdjustStep": method.ETAndBackGroundAdjustStep,
            "ETAndBackGroundAdjustMaxSize": method.ETAndBackGroundAdjustMaxSize,
            "ETAndBackGroundGrowthEstimateStep": method.ETAndBackGroundGrowthEstimateStep,
            "ETAndBackGroundGrowthEstimateMaxSize": method.ETAndBackGroundGrowthEstimateMaxSize})
    write_afqmc_param(os.path.join(workdir, "afqmc_param"), p)
    if model_dir is None:
        stage_model(kind, m, workdir)
    else:
        for f in ("model_param", "phiT.dat"):
            dst = os.path.join(workdir, f)
            if os.path.lexists(dst):
                os.remove(dst)
            os.symlink(os.path.join(os.path.abspath(model_dir), f), dst)
    wdir = os.path.join(workdir, "walkers")
    shutil.rmtree(wdir, ignore_errors=True)
    os.makedirs(wdir)
    for i in range(W):
        path = os.path.join(wdir, f"phi_{i}.dat")
        if kind == "pl":
            inputs.write_sd2is(wf[:, :, i], logw[i], m.nup, m.ndn, path)
        else:
            inputs.write_sd(wf[:, :, i], logw[i], path)


def run_cp(m, method, wf, logw, seed, mgs_step=10, pop_step=40, force_type="dynamicForce",
           threads=1, workdir=None, timeout=600):
    """One run of afqmcConstraintPath on the Hubbard inputs `m`, starting from
    walkers wf (n x N x W) with log-weights logw.  Returns the estimator
    streams (den, HNum, KNum, VNum, RNum, one row per block), the final
    walkers, and the program's stdout."""
    own = workdir is None
    workdir = workdir or tempfile.mkdtemp(prefix="afqmc_ref_cp_")
    try:
        prepare("cp", m, method, wf, logw, seed, mgs_step, pop_step, force_type, workdir)
        log = _run("cp", workdir, threads, timeout)
        out = _streams(workdir, ["den", "HNum", "KNum", "VNum", "RNum"])
        out["walkers"] = _final_walkers(workdir, "cp", wf.shape)
        return out, log
    finally:
        if own:
            shutil.rmtree(workdir, ignore_errors=True)


OBSERVE_STREAMS = ["greenMatrixNum", "densityDensityNum", "splusSminusNum", "sminusSplusNum",
                   "spairSpairNum"]


def run_cp_bp(m, method, bp_steps, wf, logw, seed, mgs_step=10, pop_step=40, force_type="dynamicForce",
              threads=1, workdir=None, timeout=600):
    """One run of afqmcConstraintPathBP (back-propagation, observe estimator)
    on the Hubbard inputs `m` with backPropagationStep = bp_steps.  Returns the
    streams den, HNum, KNum, VNum, RNum (one row per block) and the observe
    streams (one 2L x 2L or L x L matrix per block, column-major rows), the
    final walkers and the program's stdout."""
    own = workdir is None
    workdir = workdir or tempfile.mkdtemp(prefix="afqmc_ref_bp_")
    try:
        prepare("cp", m, method, wf, logw, seed, mgs_step, pop_step, force_type, workdir)
        with open(os.path.join(workdir, "afqmc_param"), "a") as f:
            f.write(f"backPropagationStep {bp_steps}\n")
        log = _run("bp", workdir, threads, timeout)
        out = _streams(workdir, ["den", "HNum", "KNum", "VNum", "RNum"])
        nb = len(out["den"])
        for name in OBSERVE_STREAMS:
            v = _streams(workdir, [name]).get(name)
            if v is not None:
                out[name] = v.reshape(nb, -1)
        out["walkers"] = _final_walkers(workdir, "cp", wf.shape)
        return out, log
    finally:
        if own:
            shutil.rmtree(workdir, ignore_errors=True)


def run_pl(m, method, wf, logw, seed, mgs_step=10, pop_step=10, force_type="dynamicForce",
           threads=1, workdir=None, timeout=600):
    """One run of afqmcPhaseless on the molecule inputs `m` (background and
    E_T as `m` holds them), starting from SD2is walkers wf (n x max(Nup,Ndn)
    x W).  Returns the estimator streams (den, HNum, TNum, one row per block;
    choleskyBgNum, choleskyExNum, G per block), the final walkers, and the
    program's stdout."""
    own = workdir is None
    workdir = workdir or tempfile.mkdtemp(prefix="afqmc_ref_pl_")
    try:
        prepare("pl", m, method, wf, logw, seed, mgs_step, pop_step, force_type, workdir)
        log = _run("pl", workdir, threads, timeout)
        out = _streams(workdir, ["den", "HNum", "TNum"])
        for name in ("choleskyBgNum", "choleskyExNum"):
            s = _streams(workdir, [name]).get(name)
            if s is not None:
                out[name] = s.reshape(-1, m.G)
        out["walkers"] = _final_walkers(workdir, "pl", wf.shape)
        return out, log
    finally:
        if own:
            shutil.rmtree(workdir, ignore_errors=True)


def timed_sample(kind, m, walkers_per_proc, steps, warmup, measure_skip, procs, mgs_step,
                 pop_step, seed=1000, timeout=1800):
    """Throughput of the reference programs on the host cores: `procs`
    single-threaded processes run at once (standing for the MPI ranks the
    reference's own build would run, walkerSizePerThread walkers each), each
    twice: `warmup` steps only, then `warmup + steps` steps with a mixed
    measurement every `measure_skip` steps.  A process's projection time is
    the difference of its two wall times, which removes start-up, input
    reading and the closing writes; the slowest process sets the rate.
    Returns (walker-steps per second, seconds of the slowest difference)."""
    from afqmclab_b200 import driver
    env = _blas_env(1)
    root = tempfile.mkdtemp(prefix=f"afqmc_ref_{kind}_bench_")
    try:
        stage_model(kind, m, os.path.join(root, "model"))
        phi = m.phiT if kind == "cp" else m.phiTUp
        blocks = max(1, steps // measure_skip)
        steps = blocks * measure_skip
        walls = {}
        for phase, (write_number, per_write) in (("short", (0, 1)), ("long", (1, blocks))):
            if kind == "cp":
                meth = driver.ConstraintPathMethod(dt=m.dt, thermalSize=warmup, writeNumber=write_number,
                                                   measureNumberPerWrite=per_write,
                                                   measureSkipStep=measure_skip, ETAdjustStep=1,
                                                   ETAdjustMaxSize=0)
            else:
                meth = driver.PhaselessMethod(dt=m.dt, thermalSize=warmup, writeNumber=write_number,
                                              measureNumberPerWrite=per_write,
                                              measureSkipStep=measure_skip,
                                              ETAndBackGroundAdjustStep=1,
                                              ETAndBackGroundAdjustMaxSize=0,
                                              ETAndBackGroundGrowthEstimateStep=1,
                                              ETAndBackGroundGrowthEstimateMaxSize=0)
            runs = []
            for p in range(procs):
                wd = os.path.join(root, f"{phase}_{p}")
                os.makedirs(wd)
                wf, lw, _ = inputs.initial_walkers(phi, walkers_per_proc, seed=seed + p, noise=0.01)
                prepare(kind, m, meth, wf, lw, seed + p, mgs_step, pop_step, "dynamicForce", wd,
                        model_dir=os.path.join(root, "model"))
                runs.append(wd)
            started = []
            for wd in runs:
                started.append((time.perf_counter(),
                                subprocess.Popen([program(kind)], cwd=wd, env=env,
                                                 stdout=subprocess.DEVNULL, stderr=subprocess.PIPE)))
            walls[phase] = []
            for t0, pr in started:
                _, err = pr.communicate(timeout=timeout)
                walls[phase].append(time.perf_counter() - t0)
                if pr.returncode != 0:
                    raise RuntimeError(f"{PROGRAMS[kind]} exited {pr.returncode}: {err[-1000:]}")
        diff = max(max(lg - sh for lg, sh in zip(walls["long"], walls["short"])), 1e-9)
        return procs * walkers_per_proc * steps / diff, diff, steps
    finally:
        shutil.rmtree(root, ignore_errors=True)
