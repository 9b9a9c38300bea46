#!/usr/bin/env python
"""Walker-step throughput of the B200 AFQMC engine (one JSON line on stdout).

A step is one projectOneStep of the whole population (force, sampling,
two-body Taylor propagation, one-body propagation, with modifyGM and
popControl at the drivers' cadence) plus the mixed measurement every
`measure_skip` steps (measureSkipStep = 5, the reference default).  The
default workload is the synthetic phaseless molecule n=128, 32+32 electrons,
G=640 Cholesky vectors, 2048 walkers, dt=0.005.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload molecule128|hubbard8x8|...] [--precision mixed|fp64]

Under torchrun (N > 1) the ranks hold the shards of one population, each
shard the size of the one-GPU workload (weak scaling): population control
runs across ranks at the reference's cadence (all-gathered weights, one
comb, walkers that change rank moved as one NCCL message per peer) and the
estimator sums are all-reduced at every measurement; the timed region is
bracketed by a barrier and the maximum over ranks is reported.
`--impl reference` times the reference's own tutorial program for the
workload (built from its sources into oracle/_ref) on the host cores, as
concurrent single-threaded processes (rank 0 only); where the programs were
not built it times the CPU oracle port of the same algorithm instead.  The
cpu_baseline object of the main line is the same measurement on a smaller
sample.
"""
import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "walker-steps/s on 1 B200: mixed-precision vs FP64 form at |ΔE|≤0.5 mHa"
UNIT = "walker-steps/s"


# ------------------------------------------------------------------ helpers
def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """SM clocks, power and throttle reasons of this process's GPU, sampled
    by a thread through NVML every ~2 ms during the timed region (nvidia-smi's
    50 ms period would miss a short region); nvidia-smi is the fallback."""

    REASONS = {"hw_slowdown": 8, "hw_thermal_slowdown": 64, "sw_thermal_slowdown": 32,
               "sw_power_cap": 4}
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, cuda_device):
        self.dev = cuda_device
        self.samples = []
        self.t0 = None
        self.stop_flag = threading.Event()
        self.thread = None
        self.proc = None
        self.nv = None
        self.handle = None
        self.smax = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.dev)
        uuid = getattr(props, "uuid", None)
        if uuid is not None:
            try:
                return pynvml, pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + str(uuid)).encode())
            except Exception:
                pass
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        idx = self.dev
        if vis:
            try:
                idx = int(vis.split(",")[self.dev])
            except ValueError:
                pass
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(idx)

    def _poll(self):
        nv, h = self.nv, self.handle
        while not self.stop_flag.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                self.samples.append((time.time(), float(sm), int(rs), pw))
            except Exception:
                pass
            time.sleep(0.002)

    def start(self):
        try:
            self.nv, self.handle = self._nvml_handle()
            self.smax = float(self.nv.nvmlDeviceGetMaxClockInfo(self.handle, self.nv.NVML_CLOCK_SM))
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nv = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read_smi, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read_smi(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                bits = sum(v for (nm, v), x in zip(self.REASONS.items(), f[5:9])
                           if x.lower().startswith("active"))
                self.smax = float(f[2])
                self.samples.append((time.time(), float(f[1]), bits, float(f[3])))
            except ValueError:
                continue

    def begin(self):
        """Mark the start of the timed region; earlier samples are dropped."""
        self.t0 = time.time()

    def stop(self):
        self.stop_flag.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)
        if self.nv is None and self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no NVML and no nvidia-smi"],
                    "samples": 0}
        sel = [x for x in self.samples if self.t0 is None or x[0] >= self.t0]
        reasons = sorted(nm for nm, bit in self.REASONS.items() if any(x[2] & bit for x in sel))
        sm = [x[1] for x in sel]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax,
                "sm_mhz_min": min(sm) if sm else None,
                "power_w_max": max(x[3] for x in sel) if sel else None,
                "reasons": reasons, "samples": len(sm),
                "source": "nvml" if self.nv is not None else "nvidia-smi"}


# ------------------------------------------------------- algorithmic counts
def phase_flops(c, m, taylor_avg):
    """Algorithmic real FLOPs of one launch of each timed phase (complex MAC = 8,
    real x complex MAC = 4), for the phaseless workload."""
    n, nup, ndn, G, W = m.n, m.nup, m.ndn, m.G, c["W"]
    K = (nup + ndn) * n
    # A_g = phiT^H L_g is real for a real trial (the Cholesky vectors are
    # real): the exchange product D = A_g theta is then real x complex
    real_a = not (np.any(np.asarray(m.phiTUp).imag) or np.any(np.asarray(m.phiTDn).imag))
    fa = 4.0 if real_a else 8.0
    f = {
        "mbuild": 4.0 * n * n * G * W,
        "force": fa * G * K * W,
        "taylor": 8.0 * n * n * max(nup, ndn) * W * taylor_avg,
        "exchange": fa * (nup * nup + ndn * ndn) * n * G * W + 8.0 * (nup * nup + ndn * ndn) * G * W,
        "overlap": 8.0 * (nup * nup + ndn * ndn) * n * W,
        "onebody": 8.0 * n * n * max(nup, ndn) * W,
    }
    # with real A the exchange runs as three GEMMs per spin block of
    # Kb = Ns n: Z = V U^T (2 Kb^2 2W), [M_re; M_im] = [Ar; Ai] Bt^T
    # (2 2Kb Kb 2W) and Y = Rt X^T (2 2Kb G Kb); the flops counted are those
    # executed, fewer than the blockwise tr(DD) count above
    if real_a and n % 32 == 0 and W % 4 == 0 and all((ns * n) % 256 == 0 for ns in (nup, ndn) if ns):
        f["exchange"] = sum((ns * n) ** 2 * (12.0 * W + 4.0 * G) for ns in (nup, ndn) if ns)
    return f


# DRAM bytes (read + write) per phase occurrence of the dominant kernel, from
# one ncu capture of the same workload (dram__bytes_read.sum +
# dram__bytes_write.sum, summed over the phase's launches).
NCU_TRAFFIC = {
    ("molecule128", "mixed", "taylor"): (201.41e6 + 35.22e6, "1 taylor_ts_kernel<32,128> launch"),
    ("molecule128", "mixed", "mbuild"): (27.56e6 + 80.28e6,
                                         "1 tc_gemm_t_kernel<1> launch (M-build; its writes partly still in L2 at the end)"),
}


def cp_phase_model(m, W, precision):
    """Algorithmic work of one launch of each timed phase of the constrained-path
    step: ("bytes", B) for the mixed form (HBM-bound: fp32 hi/lo walker planes
    read and written once per phase), ("flops", F) for the FP64 form."""
    n, N = 2 * m.L, m.N
    if precision == "mixed":
        walker = 16.0 * n * N            # hi + lo planes, re + im, fp32
        return {
            "overlap": ("bytes", W * (walker + 16.0 * N * N)),
            "force": ("bytes", W * (16.0 * N * N + 2 * 16.0 * N * N + walker / 2 + 8.0 * n)),
            "sample": ("bytes", W * 2 * walker),
            "onebody": ("bytes", W * 2 * walker),
        }
    return {
        "overlap": ("flops", 8.0 * N * N * n * W),
        "theta": ("flops", 8.0 * N * N * n * W),
        "onebody": ("flops", 8.0 * n * n * N * W),
    }


NO_LOCAL_POP = 1 << 30   # pop_control_step of an engine whose comb runs across ranks


def build_engine(capi, inputs, name, precision, seed, local_pop=True):
    """The workload's engine and population.  With local_pop False the engine
    never combs on its own (the cross-rank population control does)."""
    m, c = inputs.make_config(name)
    prec = capi.AFQMC_MIXED if precision == "mixed" else capi.AFQMC_FP64
    pop = c["pop"] if local_pop else NO_LOCAL_POP
    if c["kind"] == "pl":
        eng = capi.pl_engine(m, c["W"], seed, c["mgs"], pop, precision=prec)
        wf, lw, al = inputs.initial_walkers(m.phiTUp, c["W"])
    else:
        eng = capi.cp_engine(m, c["W"], seed, c["mgs"], pop, precision=prec)
        wf, lw, al = inputs.initial_walkers(m.phiT, c["W"])
    eng.set_walkers(wf, lw, al)
    # initialMgsAndPopControl (afqmcPhaselessSetWalker.cpp:140-144)
    eng.modify_gm()
    if local_pop:
        eng.pop_control()
    return eng, m, c, (wf, lw, al)


def run_steps(eng, k, start, measure_skip):
    for i in range(k):
        if (start + i) % measure_skip == 0:
            eng.add_mixed_measurement()
        eng.step(1)


class ShardedRunner:
    """Steps of one population sharded over the ranks (N > 1): the engine
    steps its own walkers; every pop_step steps the population control runs
    across ranks (all-gather of the weights, the same comb on every rank,
    walkers that change rank packed into one message per peer), and every
    measurement's sums are all-reduced (the reference's MPISum of HNum, den
    and the per-vector sums).  Every rank takes the same collective steps."""

    def __init__(self, eng, pop_step, measure_skip, device, seed=20240503):
        from afqmclab_b200 import parallel
        self.parallel = parallel
        self.eng, self.pop_step, self.measure_skip = eng, pop_step, measure_skip
        self.device = device
        self.pop = parallel.EnginePopulation(eng, device)
        self.seed, self.counter = seed, 0

    def control(self):
        _, self.counter = self.parallel.global_pop_control(self.pop, self.seed, self.counter,
                                                           device=self.device)

    def __call__(self, k, start):
        for i in range(k):
            s = start + i
            if s % self.measure_skip == 0:
                self.eng.add_mixed_measurement()
                self.parallel.global_measurement(self.eng, device=self.device)
            self.eng.step(1)
            if (s + 1) % self.pop_step == 0:
                self.control()


def energy_check(capi, inputs, name, steps, measure_skip, stream, seed):
    """Mixed vs FP64 form from identical walkers and random stream: mixed
    estimator E = HNum/den (one measurement = addMixedMeasurement over the
    population, afqmcPhaselessMeasure.cpp:9-28) every measure_skip steps."""
    out = {}
    for prec in ("fp64", "mixed"):
        eng, m, c, _ = build_engine(capi, inputs, name, prec, seed)
        eng.set_stream(stream.cuda_stream)
        es = []
        for i in range(steps):
            if i % measure_skip == 0:
                eng.reset_measurement()
                eng.add_mixed_measurement()
                mm = eng.measurement()
                es.append((mm[1] / mm[0]).real)
            eng.step(1)
        out[prec] = np.array(es)
        eng.close()
    d = (out["mixed"] - out["fp64"]) * 1e3
    return {"steps": steps, "measurements": len(d), "E_fp64_Ha": out["fp64"].tolist(),
            "E_mixed_Ha": out["mixed"].tolist(), "dE_mHa": d.tolist(),
            "max_abs_dE_mHa": float(np.abs(d).max()), "mean_dE_mHa": float(d.mean()),
            "criterion_mHa": 0.5, "pass": bool(np.abs(d).max() <= 0.5),
            "method": "paired: same walkers, same random stream, measurement by measurement"}


def bench_uneven(args, capi, inputs, torch, rank, world):
    """The uneven batch: four Hubbard lattices of different size and filling
    (1024 walkers each) advanced as one graph launch per step, in the chosen
    form, then the same batch in the plain FP64 form from the same walkers and
    random streams; per-lattice mixed estimators are compared measurement by
    measurement."""
    precision = "fp64" if args.precision == "fp64" else "mixed"
    stream = torch.cuda.Stream()

    def make(prec, seed0):
        engines, tot = [], 0
        for k, name in enumerate(inputs.UNEVEN_BATCH):
            e, m, c, _ = build_engine(capi, inputs, name, prec, seed0 + k)
            engines.append(e)
            tot += c["W"]
        b = capi.Batch(engines)
        b.set_stream(stream.cuda_stream)
        return b, engines, tot

    def run(b, engines, k, start, energies=None):
        for i in range(k):
            if (start + i) % args.measure_skip == 0:
                for j, e in enumerate(engines):
                    if energies is not None:
                        e.reset_measurement()
                    e.add_mixed_measurement()
                    if energies is not None:
                        mm = e.measurement()
                        energies[j].append((mm[1] / mm[0]).real)
            b.step(1)

    out = {}
    for prec in ([precision, "fp64"] if precision == "mixed" and not args.no_fp64_side else [precision]):
        b, engines, tot = make(prec, 77 + 10 * rank)
        run(b, engines, args.warmup, 0)
        b.synchronize()
        launches0 = capi.launch_count()
        clocks = ClockSampler(torch.cuda.current_device())
        torch.cuda.synchronize()
        clocks.start()
        clocks.begin()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run(b, engines, args.steps, args.warmup)
        e1.record(stream)
        while not e1.query():   # polling: the clock sampler runs meanwhile
            time.sleep(0.0005)
        b.synchronize()
        clk = clocks.stop()
        ms = e0.elapsed_time(e1)
        out[prec] = {"value": tot * args.steps / (ms / 1e3), "ms_per_step": ms / args.steps,
                     "gpu_launches": int(capi.launch_count() - launches0), "clocks": clk}
        b.close()
        for e in engines:
            e.close()
    # paired energies: same walkers and random streams in both forms
    energies = {}
    if precision == "mixed" and args.energy_steps > 0:
        for prec in ("fp64", "mixed"):
            b, engines, _ = make(prec, 4242)
            acc = [[] for _ in engines]
            run(b, engines, args.energy_steps, 0, acc)
            b.synchronize()
            energies[prec] = acc
            b.close()
            for e in engines:
                e.close()
        per = {}
        for j, name in enumerate(inputs.UNEVEN_BATCH):
            ef, ex = np.array(energies["fp64"][j]), np.array(energies["mixed"][j])
            per[name] = {"E_fp64": ef.tolist(), "E_mixed": ex.tolist(),
                         "max_abs_dE": float(np.abs(ex - ef).max()),
                         "max_rel_dE": float(np.abs((ex - ef) / ef).max())}
        energies = per
    main = out[precision]
    line = {"metric": METRIC, "value": main["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": main["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "tf32/f32 tensor + f64" if precision == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": "uneven", "lattices": inputs.UNEVEN_BATCH,
                       "walkers_per_lattice": 1024, "precision": precision,
                       "measure_skip": args.measure_skip, "cuda_graphs": "one graph launch per step"},
            "gpu_launches": main["gpu_launches"], "clocks": main["clocks"],
            "fp64_form": out.get("fp64") if precision == "mixed" else None,
            "speedup_mixed_over_fp64": (out["fp64"]["ms_per_step"] / main["ms_per_step"])
            if precision == "mixed" and "fp64" in out else None,
            "energy_check": energies or None}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def bench_adjoint(args, capi, inputs, torch, rank, world):
    """Adjoint throughput: afqmc_pl_adjoint (mixed local energy, mean
    log-overlap and their gradients with respect to t, the Cholesky vectors and
    the trial orbitals, FP64, per-walker recomputation) on the population of a
    phaseless workload after a few projection steps."""
    name = args.adjoint_workload
    m, c = inputs.make_config(name)
    W = c["W"]
    eng = capi.pl_engine(m, W, 77 + rank, c["mgs"], c["pop"], precision=capi.AFQMC_FP64)
    eng.set_walkers(*inputs.initial_walkers(m.phiTUp, W))
    eng.modify_gm()
    eng.pop_control()
    eng.step(3)
    eng.synchronize()
    reps = max(1, args.steps // 50)
    n, G, N = m.n, m.G, m.nup + m.ndn
    # dE/dL_g (n x n x G complex, 1.3 GB at n=256) stays in HBM as a torch
    # tensor; the other outputs are host arrays
    dchol = torch.empty(n * n * G, dtype=torch.complex128, device="cuda")
    eng.adjoint(chol_out=dchol)   # warm-up (allocations, first launches)
    eng.synchronize()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    clocks.begin()
    t0 = time.perf_counter()
    out = None
    for _ in range(reps):
        out = eng.adjoint(chol_out=dchol)
    eng.synchronize()
    dt = time.perf_counter() - t0
    clk = clocks.stop()
    line = {"metric": "walker adjoint evaluations/s (E, dE/dt, dE/dL_g, dE/dconj(phiT)), FP64",
            "value": W * reps / dt, "unit": "walker-evaluations/s", "n_gpus": world, "steps": reps,
            "warmup": 1, "ms_per_step": dt / reps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "adjoint", "model": name, "n_orbitals": n, "electrons": [m.nup, m.ndn],
                       "cholesky": G, "walkers": W, "timing": "host wall clock around synchronous calls",
                       "outputs": "dE/dL_g into a CUDA tensor, the rest to host arrays"},
            "energy": [float(out["E"].real), float(out["E"].imag)],
            "gradient_norms": {"dE_dt": float(np.abs(out["dE_dt"]).max()),
                               "dE_dchol": float(dchol.abs().max())},
            "clocks": clk}
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()
    return 0


def default_precision(args):
    if args.precision != "auto":
        return args.precision
    if args.workload in ("adjoint",):
        return "fp64"
    return "mixed" if os.environ.get("AFQMC_BENCH_FP64") is None else "fp64"


def workload_config(name, precision, measure_skip, world, graphs):
    """The `config` object of the bench line (both arms print the same one)."""
    from afqmclab_b200 import inputs
    c = inputs.CONFIGS[name]
    n = c["n"] if c["kind"] == "pl" else 2 * c["nx"] * c["ny"]
    return {"workload": name, "precision": precision, "n_orbitals": n,
            "electrons": [c.get("nup"), c.get("ndn")], "cholesky": c.get("G"),
            "walkers_per_gpu": c["W"], "dt": c["dt"], "mgs_step": c["mgs"],
            "pop_control_step": c["pop"], "measure_skip": measure_skip,
            "parallelism": f"walker-dp{world}", "l2": "inputs larger than L2 (no flush)",
            "cuda_graphs": graphs}


# ---------------------------------------------------------------- CPU arm
def _cpu_worker(args):
    name, nwalk, steps, seed, measure_skip, warmup = args
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    from afqmclab_b200 import inputs
    from oracle import oracle as O
    m, c = inputs.make_config(name)
    if c["kind"] == "pl":
        eng = O.pl_engine(m, nwalk, seed, c["mgs"], c["pop"])
        wf, lw, al = inputs.initial_walkers(m.phiTUp, nwalk)
    else:
        eng = O.cp_engine(m, nwalk, seed, c["mgs"], c["pop"])
        wf, lw, al = inputs.initial_walkers(m.phiT, nwalk)
    eng.set_walkers(wf, lw, al)
    for i in range(warmup):
        if i % measure_skip == 0:
            eng.add_mixed_measurement()
        eng.step(1)
    t0 = time.perf_counter()
    for i in range(steps):
        if (warmup + i) % measure_skip == 0:
            eng.add_mixed_measurement()
        eng.step(1)
    return nwalk * steps, time.perf_counter() - t0


def ref_measure(name, steps, measure_skip, warmup=2, max_procs=None, walkers_per_proc=None):
    """The reference's own program for the workload (afqmcPhaseless or
    afqmcConstraintPath, built from the reference's sources into oracle/_ref)
    on the host cores: P single-threaded processes at once, standing for the
    MPI ranks of the reference's own build (walkerSizePerThread walkers each;
    the cross-rank population exchange is not included).  Returns
    (walker-steps/s, P, sample) or None when the programs were not built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))
    import ref_run
    from afqmclab_b200 import inputs
    m, c = inputs.make_config(name)
    kind = c["kind"]
    if not ref_run.available(kind):
        return None
    P = min(os.cpu_count() or 1, max_procs or 64)
    if walkers_per_proc is None:
        walkers_per_proc = 4 if kind == "pl" else max(1, min(16, c["W"] // P))
    v, secs, st = ref_run.timed_sample(kind, m, walkers_per_proc, steps, warmup, measure_skip, P,
                                       c["mgs"], c["pop"])
    sample = (f"{P} concurrent single-threaded {ref_run.PROGRAMS[kind]} processes (the reference's "
              f"tutorial program built from its sources, BLAS/LAPACK through OpenBLAS, 1 thread) x "
              f"{walkers_per_proc} walkers x {st} steps of {name} (measurement every {measure_skip} "
              f"steps, after {warmup} steps); projection time = wall time of the run minus that of "
              f"the same run stopped after the warm-up steps, slowest process ({secs:.2f} s)")
    return v, P, sample


def cpu_measure(name, steps, measure_skip, max_procs=None, walkers_per_proc=None, warmup=0):
    """Oracle port on the host cores: P single-threaded processes, each with
    its own small population (the reference's MPI walker parallelism); each
    process takes `warmup` untimed steps, then `steps` timed ones."""
    from afqmclab_b200 import inputs
    c = inputs.CONFIGS[name]
    cores = os.cpu_count() or 1
    P = min(cores, max_procs or 64)
    if walkers_per_proc is None:
        walkers_per_proc = 2 if c["kind"] == "pl" else max(1, min(16, c["W"] // P))
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    # the oracle build whose GEMM/GEMV-shaped work runs through OpenBLAS, as the
    # reference's runs through its BLAS (the spawned workers inherit this)
    from oracle import oracle as O
    blas = O.scipy_blas()
    if blas:
        os.environ["AFQMC_ORACLE_BLAS"], os.environ["AFQMC_ORACLE_BLAS_PREFIX"] = blas
    ctx = mp.get_context("spawn")
    with ctx.Pool(P) as pool:
        res = pool.map(_cpu_worker, [(name, walkers_per_proc, steps, 1000 + i, measure_skip, warmup)
                                     for i in range(P)])
    total = sum(r[0] for r in res)
    wall = max(r[1] for r in res)
    sample = (f"{P} processes x {walkers_per_proc} walkers x {steps} steps of {name} "
              f"(measurement every {measure_skip} steps, {warmup} untimed warm-up steps), "
              f"slowest process timed; GEMM/GEMV work through "
              f"{'OpenBLAS (' + os.path.basename(blas[0]) + ', 1 thread)' if blas else 'plain loops'}")
    return total / wall, P, sample


# ------------------------------------------------------------------ main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="molecule128")
    ap.add_argument("--precision", default="auto", choices=["auto", "mixed", "fp64"])
    ap.add_argument("--measure-skip", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=20)
    ap.add_argument("--no-fp64-side", action="store_true")
    ap.add_argument("--no-graphs", action="store_true")
    ap.add_argument("--energy-steps", type=int, default=60)
    ap.add_argument("--adjoint-workload", default="molecule256")
    args = ap.parse_args()
    rank, world, local = dist_info()

    if args.impl == "reference":
        if rank != 0:
            return 0
        t0 = time.perf_counter()
        steps = min(args.steps, 200)
        r = ref_measure(args.workload, steps, args.measure_skip, warmup=args.warmup)
        if r is not None:
            (v, P, sample), kind = r, "reference"
            form = ("the reference's own tutorial program (FP64), built from its sources, "
                    "single-threaded processes")
        else:
            v, P, sample = cpu_measure(args.workload, steps, args.measure_skip, warmup=args.warmup)
            kind = "port"
            form = "CPU restatement of the reference's FP64 path (oracle/), single-threaded processes"
        line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": workload_config(args.workload, default_precision(args), args.measure_skip,
                                          args.gpus, not args.no_graphs),
                "reference_form": form,
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": P, "kind": kind,
                                 "sample": sample},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0},
                "wall_s": time.perf_counter() - t0}
        print(json.dumps(line), flush=True)
        return 0

    import torch
    from afqmclab_b200 import capi, inputs
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    if args.workload == "adjoint":
        r = bench_adjoint(args, capi, inputs, torch, rank, world)
        if world > 1:
            torch.distributed.destroy_process_group()
        return r

    if args.workload == "uneven":
        r = bench_uneven(args, capi, inputs, torch, rank, world)
        if world > 1:
            torch.distributed.destroy_process_group()
        return r

    precision = default_precision(args)
    local_pop = world == 1
    try:
        eng, m, c, init = build_engine(capi, inputs, args.workload, precision, 77 + rank, local_pop)
    except capi.AfqmcError:
        if args.precision != "auto":
            raise
        precision = "fp64"
        eng, m, c, init = build_engine(capi, inputs, args.workload, precision, 77 + rank, local_pop)
    W = c["W"]
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    if not args.no_graphs:
        eng.set_graphs(True)
    if world == 1:
        def runner(k, start):
            run_steps(eng, k, start, args.measure_skip)
    else:
        runner = ShardedRunner(eng, c["pop"], args.measure_skip, torch.device("cuda", local))
        runner.control()   # initialMgsAndPopControl's popControl, across ranks

    # warm-up
    runner(args.warmup, 0)
    eng.synchronize()

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # per-phase CUDA-event times (direct launches) over K steps, then the
    # timed region: K steps, inputs resident in HBM (population + model
    # tensors exceed the 126 MB L2 at this size), graphs replayed
    eng.profile(True)
    runner(args.steps, args.warmup)
    eng.synchronize()
    prof = eng.profile_get()
    eng.profile(False)
    runner(2, args.warmup + args.steps)
    eng.synchronize()
    launches0 = capi.launch_count()
    clocks = ClockSampler(dev)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    clocks.begin()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    runner(args.steps, args.warmup + 2 + args.steps)
    ev1.record(stream)
    # wait by polling, so the clock-sampling thread gets the interpreter
    # while the GPU runs (the event pair times the device, not this loop)
    while not ev1.query():
        time.sleep(0.0005)
    barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = capi.launch_count() - launches0
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    value = W * args.steps * world / (ms / 1e3)

    # e2e: the same steps through the C ABI with host buffers: each step
    # uploads the population from pinned host memory and reads back the
    # estimator sums.  The upload of step i+1 is enqueued (afqmc_set_walkers_async)
    # while step i runs, so the copy overlaps the compute of the previous step.
    # The phaseless mixed form keeps its walkers as fp32 planes, and a caller
    # of that form hands them over in that layout (afqmc_set_walkers_f32_async,
    # half the bytes of complex doubles); the other forms upload complex doubles.
    wf0, lw0, al0 = init
    f32 = precision == "mixed" and c["kind"] == "pl"
    if f32:
        n0, nc0, nw0 = wf0.shape
        planes = np.empty((nw0, 2, n0 * nc0), np.float32)
        for w in range(nw0):
            flat = wf0[:, :, w].reshape(-1, order="F")
            planes[w, 0] = flat.real
            planes[w, 1] = flat.imag
        h_wf = torch.from_numpy(planes.reshape(-1)).pin_memory()
        upload = eng.set_walkers_f32_async
        wf_bytes = h_wf.numel() * 4
        how = "fp32 walkers in the mixed form's planar layout (afqmc_set_walkers_f32_async), pipelined"
    else:
        h_wf = torch.from_numpy(np.ascontiguousarray(wf0.reshape(-1, order="F").view(np.float64))).pin_memory()
        upload = eng.set_walkers_async
        wf_bytes = h_wf.numel() * 8
        how = "complex128 walkers (afqmc_set_walkers_async), pipelined"
    h_lw = torch.from_numpy(np.ascontiguousarray(lw0.view(np.float64))).pin_memory()
    h_al = torch.from_numpy(np.ascontiguousarray(al0)).pin_memory()
    meas = np.zeros(5, np.complex128)
    lib = capi.lib()
    e2e_steps = args.steps
    # the first pipelined upload creates the copy stream and the two device
    # staging slots: do it, and one step, before the clock starts
    upload(h_wf.data_ptr(), h_lw.data_ptr(), h_al.data_ptr())
    eng.upload_wait()
    runner(1, 1)
    capi._check(lib.afqmc_get_measurement(eng.h, meas.ctypes.data))
    eng.synchronize()
    barrier()
    t0 = time.perf_counter()
    upload(h_wf.data_ptr(), h_lw.data_ptr(), h_al.data_ptr())
    for i in range(e2e_steps):
        runner(1, i)
        if i + 1 < e2e_steps:
            upload(h_wf.data_ptr(), h_lw.data_ptr(), h_al.data_ptr())
        capi._check(lib.afqmc_get_measurement(eng.h, meas.ctypes.data))
    e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": W * e2e_steps * world / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": int(wf_bytes + h_lw.numel() * 8 + h_al.numel() * 4),
           "d2h_bytes_per_step": int(meas.nbytes), "upload": how + " (next step's copy overlaps this step)"}

    # roofline of the dominant phase
    calls, total, mn, mx = eng.taylor_stats()
    status = eng.status()
    tavg = total / calls if calls else 0.0
    roof = None
    if c["kind"] == "pl":
        fl = phase_flops(c, m, tavg)
        cand = {k: v for k, v in prof.items() if k in fl and v[1] > 0}
        top = max(cand, key=lambda k: cand[k][0])
        t_launch = prof[top][0] / prof[top][1] / 1e3
        achieved = fl[top] / t_launch / 1e12
        peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
        if precision == "mixed":
            # the kernel runs for ~0.1 ms inside a timed region far shorter
            # than the seconds-long sustained measurement: the burst figure
            peak = json.load(open(peaks_path))["bf16_tflops"] if os.path.exists(peaks_path) else 1590.0
            bound = "tensor"
            psrc = "measured bf16 burst (of measured)" if os.path.exists(peaks_path) else "fallback"
        else:
            peak, bound, psrc = 37.2, "fp64", "nominal FP64 (148 SM x 64 DFMA x 1.965 GHz); not in MEASURED_PEAKS.json"
        roof = {"bound": bound, "kernel": top, "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                "flops_per_launch": fl[top], "launch_ms": t_launch * 1e3, "peak_source": psrc}
        tr = NCU_TRAFFIC.get((args.workload, precision, top))
        if tr:
            roof["traffic"] = tr[0]
            roof["traffic_note"] = "bytes per phase occurrence, " + tr[1] + ", from ncu"
    else:
        model = cp_phase_model(m, W, precision)
        cand = {k: v for k, v in prof.items() if k in model and v[1] > 0}
        top = max(cand, key=lambda k: cand[k][0])
        t_launch = prof[top][0] / prof[top][1] / 1e3
        kind, amount = model[top]
        peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
        have = os.path.exists(peaks_path)
        if kind == "bytes":
            peak = json.load(open(peaks_path))["hbm_gbs"] if have else 6650.0
            roof = {"bound": "hbm", "kernel": top, "achieved": amount / t_launch / 1e9, "peak": peak,
                    "unit": "GB/s", "traffic": None, "bytes_per_launch": amount,
                    "launch_ms": t_launch * 1e3,
                    "peak_source": "measured copy bandwidth" if have else "fallback"}
        else:
            peak = 37.2
            roof = {"bound": "fp64", "kernel": top, "achieved": amount / t_launch / 1e12, "peak": peak,
                    "unit": "TFLOP/s", "traffic": None, "flops_per_launch": amount,
                    "launch_ms": t_launch * 1e3,
                    "peak_source": "nominal FP64 (148 SM x 64 DFMA x 1.965 GHz); not in MEASURED_PEAKS.json"}
        roof["frac"] = roof["achieved"] / roof["peak"]

    # the plain FP64 form side by side, and the paired energy check: both
    # forms from the same walkers and random stream, mixed estimator every
    # measure_skip steps (energies compared measurement by measurement)
    side = None
    echeck = None
    if precision == "mixed" and not args.no_fp64_side:
        eng.close()
        f64, _, _, _ = build_engine(capi, inputs, args.workload, "fp64", 77 + rank)
        f64.set_stream(stream.cuda_stream)
        if not args.no_graphs:
            f64.set_graphs(True)
        run_steps(f64, 2, 0, args.measure_skip)
        f64.synchronize()
        k64 = max(5, min(args.steps, 10))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run_steps(f64, k64, 2, args.measure_skip)
        e1.record(stream)
        e1.synchronize()
        ms64 = e0.elapsed_time(e1)
        side = {"value": W * k64 * world / (ms64 / 1e3), "ms_per_step": ms64 / k64, "steps": k64,
                "speedup_mixed_over_fp64": (ms64 / k64) / (ms / args.steps),
                "algorithm": "same as the mixed form: closed-shell single spin block, exchange as "
                             "GEMMs (FP64 CUDA-core GEMMs)"}
        # per-phase times of the FP64 form (direct launches, after the timed steps)
        f64.profile(True)
        run_steps(f64, k64, 2 + k64, args.measure_skip)
        f64.synchronize()
        side["phases_ms"] = {k: round(v[0], 3) for k, v in f64.profile_get().items() if v[1] > 0}
        f64.profile(False)
        f64.close()
        if args.energy_steps > 0:
            echeck = energy_check(capi, inputs, args.workload, args.energy_steps, args.measure_skip,
                                  stream, 4242 + rank)
        eng = None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = ref_measure(args.workload, args.cpu_steps, args.measure_skip)
        if r is not None:
            v, P, sample = r
            cpu = {"value": v, "unit": UNIT, "cores": P, "kind": "reference", "sample": sample}
        else:
            v, P, sample = cpu_measure(args.workload, args.cpu_steps, args.measure_skip)
            cpu = {"value": v, "unit": UNIT, "cores": P, "kind": "port", "sample": sample}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16/f32 tensor + f64" if precision == "mixed" else "f64",
            "data": "synthetic",
            "config": workload_config(args.workload, precision, args.measure_skip, world,
                                      not args.no_graphs),
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clk,
            "phases_ms": {k: round(v[0], 3) for k, v in prof.items() if v[1] > 0},
            "taylor_order": {"avg": tavg, "min": mn, "max": mx},
            "status": status,
            "fp64_form": side,
            "energy_check": echeck,
        }
        print(json.dumps(line), flush=True)
    if eng is not None:
        eng.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
