"""ctypes binding of the engine's C ABI (include/afqmc_b200.h).

This is the host-side mirror used by the tests and bench.py: the same entry
points a C++ or cgo/JNI caller binds.  The library is the in-tree
libafqmc_b200.so built for sm_100a; importing this module on a machine
without it raises immediately (there is no fallback path).
"""
import ctypes
import os

import numpy as np

from . import build as _build

_lib = None

AFQMC_FP64, AFQMC_MIXED = 0, 1
DECOMP = {"densityCharge": 0, "densitySpin": 1, "hopCharge": 2, "hopSpin": 3}
FORCE = {"dynamicForce": 0, "constForce": 1}

SYMBOLS = [
    "afqmc_last_error", "afqmc_version", "afqmc_cp_create", "afqmc_pl_create", "afqmc_destroy",
    "afqmc_set_stream", "afqmc_synchronize", "afqmc_set_walkers", "afqmc_get_walkers",
    "afqmc_set_walkers_f32_async", "afqmc_set_walkers_async", "afqmc_upload_wait",
    "afqmc_set_rng", "afqmc_get_rng", "afqmc_set_ET", "afqmc_set_cadence",
    "afqmc_project_one_step", "afqmc_project_half", "afqmc_modify_gm", "afqmc_pop_control",
    "afqmc_reset_measurement", "afqmc_add_mixed_measurement", "afqmc_get_measurement",
    "afqmc_get_cholesky_nums", "afqmc_pl_update_background", "afqmc_pl_rebuild_propagators", "afqmc_log_overlaps",
    "afqmc_green_matrix", "afqmc_taylor_stats", "afqmc_status", "afqmc_pop_configuration_dev",
    "afqmc_profile_enable", "afqmc_profile_get", "afqmc_launch_count", "afqmc_gemm_bf16_dev",
    "afqmc_pop_configuration_noalloc_dev", "afqmc_set_graphs", "afqmc_pl_adjoint",
    "afqmc_pop_configuration_host", "afqmc_pop_weights", "afqmc_walker_bytes",
    "afqmc_copy_walker_out", "afqmc_copy_walker_in", "afqmc_apply_table",
    "afqmc_batch_create", "afqmc_batch_step", "afqmc_batch_synchronize", "afqmc_batch_destroy",
    "afqmc_batch_set_stream",
    "afqmc_set_autotune", "afqmc_bounded_wait_check", "afqmc_get_site_nums",
    "afqmc_pack_walkers", "afqmc_unpack_walkers", "afqmc_cp_set_observables",
    "afqmc_cp_bp_begin", "afqmc_cp_bp_measure", "afqmc_cp_bp_state",
    "afqmc_get_observables",
]

PHASES = ["overlap", "lu", "theta", "force", "sample", "mbuild", "taylor", "onebody", "stabilize",
          "popcontrol", "exchange", "measure"]


class AfqmcError(RuntimeError):
    pass


def lib_path():
    return _build.LIB


def lib():
    global _lib
    if _lib is None:
        path = lib_path()
        if not os.path.exists(path):
            raise AfqmcError(f"engine library {path} is missing: run python -m afqmclab_b200.build")
        _lib = ctypes.CDLL(path)
        _declare(_lib)
    return _lib


def _declare(L):
    P, I, D, U64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_ulonglong
    PP = ctypes.POINTER(ctypes.c_void_p)
    L.afqmc_last_error.restype = ctypes.c_char_p
    L.afqmc_version.restype = ctypes.c_char_p
    L.afqmc_cp_create.argtypes = [I, I, I, I, I, D, D, D, I, I, I, P, P, P, P, P, P, P, P, P, P,
                                  P, D, D, U64, PP]
    L.afqmc_pl_create.argtypes = [I, I, I, I, I, I, D, D, D, I, I, I, P, P, P, P, D, P, D, P, D,
                                  P, D, P, P, P, D, D, U64, PP]
    for name in ["afqmc_destroy", "afqmc_synchronize", "afqmc_modify_gm",
                 "afqmc_reset_measurement", "afqmc_add_mixed_measurement"]:
        getattr(L, name).argtypes = [P]
    L.afqmc_set_stream.argtypes = [P, P]
    L.afqmc_set_walkers.argtypes = [P, P, P, P]
    L.afqmc_get_walkers.argtypes = [P, P, P, P]
    L.afqmc_set_walkers_async.argtypes = [P, P, P, P]
    L.afqmc_set_walkers_f32_async.argtypes = [P, P, P, P]
    L.afqmc_upload_wait.argtypes = [P]
    L.afqmc_set_rng.argtypes = [P, U64, U64]
    L.afqmc_get_rng.argtypes = [P, ctypes.POINTER(U64), ctypes.POINTER(U64)]
    L.afqmc_set_ET.argtypes = [P, D]
    L.afqmc_set_cadence.argtypes = [P, I, I]
    L.afqmc_project_one_step.argtypes = [P, I]
    L.afqmc_project_half.argtypes = [P, I]
    L.afqmc_pop_control.argtypes = [P, P, P]
    L.afqmc_get_measurement.argtypes = [P, P]
    L.afqmc_get_cholesky_nums.argtypes = [P, P, P]
    L.afqmc_get_site_nums.argtypes = [P, P, P, P, P]
    L.afqmc_pl_update_background.argtypes = [P, P, P, D, P, D, P, D]
    L.afqmc_pl_rebuild_propagators.argtypes = [P, P]
    L.afqmc_log_overlaps.argtypes = [P, P]
    L.afqmc_green_matrix.argtypes = [P, I, I, P]
    L.afqmc_taylor_stats.argtypes = [P, ctypes.POINTER(ctypes.c_longlong),
                                     ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(I),
                                     ctypes.POINTER(I)]
    L.afqmc_status.argtypes = [P, ctypes.POINTER(I)]
    L.afqmc_pop_configuration_dev.argtypes = [I, P, P, P, P]
    L.afqmc_pop_configuration_noalloc_dev.argtypes = [I, P, P, P, P]
    L.afqmc_profile_enable.argtypes = [P, I]
    L.afqmc_profile_get.argtypes = [P, P, P]
    L.afqmc_launch_count.argtypes = []
    L.afqmc_set_graphs.argtypes = [P, I]
    L.afqmc_pl_adjoint.argtypes = [P, P, P, P, P, P, P, P, P]
    L.afqmc_pop_configuration_host.argtypes = [I, I, P, P, P]
    L.afqmc_pop_weights.argtypes = [P, P]
    L.afqmc_walker_bytes.argtypes = [P]
    L.afqmc_copy_walker_out.argtypes = [P, I, P]
    L.afqmc_copy_walker_in.argtypes = [P, I, P]
    L.afqmc_apply_table.argtypes = [P, P]
    L.afqmc_pack_walkers.argtypes = [P, I, P, P]
    L.afqmc_cp_set_observables.argtypes = [P, I]
    L.afqmc_cp_bp_begin.argtypes = [P, I, I]
    L.afqmc_cp_bp_measure.argtypes = [P]
    L.afqmc_cp_bp_state.argtypes = [P, ctypes.POINTER(I), ctypes.POINTER(I)]
    L.afqmc_get_observables.argtypes = [P, P, P, P, P, P]
    L.afqmc_unpack_walkers.argtypes = [P, I, P, P]
    L.afqmc_batch_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), I, PP]
    L.afqmc_batch_step.argtypes = [P, I]
    L.afqmc_batch_synchronize.argtypes = [P]
    L.afqmc_batch_destroy.argtypes = [P]
    L.afqmc_batch_set_stream.argtypes = [P, P]
    L.afqmc_set_autotune.argtypes = [I]
    L.afqmc_bounded_wait_check.argtypes = [ctypes.c_longlong, ctypes.POINTER(I), P]
    LL = ctypes.c_longlong
    L.afqmc_gemm_bf16_dev.argtypes = [I, I, I, P, LL, P, LL, P, LL, I, I, LL, ctypes.c_float, P]
    for name in SYMBOLS[2:]:
        getattr(L, name).restype = I
    L.afqmc_launch_count.restype = ctypes.c_longlong
    L.afqmc_walker_bytes.restype = ctypes.c_longlong


def _check(r):
    if r != 0:
        raise AfqmcError(f"afqmc error {r}: {lib().afqmc_last_error().decode()}")


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _z(a):
    return None if a is None else np.asfortranarray(a, dtype=np.complex128)


def _d(a):
    return None if a is None else np.asfortranarray(a, dtype=np.float64)


class Engine:
    """A walker population resident on the GPU (one engine handle)."""

    def __init__(self, handle, kind, n, ncol, W, G=0, nup=0, ndn=0, keep=()):
        self.h = handle
        self.kind, self.n, self.ncol, self.W, self.G = kind, n, ncol, W, G
        self.nup, self.ndn = nup, ndn
        self._keep = keep

    def close(self):
        if getattr(self, "h", None):
            lib().afqmc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # population
    def set_walkers(self, wf, logw, alive):
        wf = np.asfortranarray(wf, dtype=np.complex128)
        assert wf.shape == (self.n, self.ncol, self.W), wf.shape
        lw = np.ascontiguousarray(logw, dtype=np.complex128)
        al = np.ascontiguousarray(alive, dtype=np.int32)
        _check(lib().afqmc_set_walkers(self.h, _p(wf), _p(lw), _p(al)))

    def set_walkers_async(self, wf_ptr, logw_ptr, alive_ptr):
        """Pipelined upload from pinned host buffers given by address (they
        must stay unchanged until upload_wait() or a synchronizing call)."""
        _check(lib().afqmc_set_walkers_async(self.h, ctypes.c_void_p(wf_ptr), ctypes.c_void_p(logw_ptr),
                                             ctypes.c_void_p(alive_ptr)))

    def set_walkers_f32_async(self, wf32_ptr, logw_ptr, alive_ptr):
        """Asynchronous upload of fp32 walkers in the phaseless mixed form's
        layout (per walker: real plane then imaginary plane, n x ncol each,
        column-major) from host pointers (pinned)."""
        _check(lib().afqmc_set_walkers_f32_async(self.h, ctypes.c_void_p(wf32_ptr), ctypes.c_void_p(logw_ptr),
                                                 ctypes.c_void_p(alive_ptr)))

    def upload_wait(self):
        _check(lib().afqmc_upload_wait(self.h))

    def get_walkers(self):
        wf = np.zeros((self.n, self.ncol, self.W), np.complex128, order="F")
        lw = np.zeros(self.W, np.complex128)
        al = np.zeros(self.W, np.int32)
        _check(lib().afqmc_get_walkers(self.h, _p(wf), _p(lw), _p(al)))
        return wf, lw, al

    def set_rng(self, seed, counter=0):
        _check(lib().afqmc_set_rng(self.h, seed, counter))

    def rng_counter(self):
        return self.rng_state()[1]

    def rng_state(self):
        """(seed, counter) of the engine's random stream."""
        s, c = ctypes.c_ulonglong(), ctypes.c_ulonglong()
        _check(lib().afqmc_get_rng(self.h, ctypes.byref(s), ctypes.byref(c)))
        return s.value, c.value

    def set_ET(self, ET):
        _check(lib().afqmc_set_ET(self.h, ET))

    def set_cadence(self, mgs_index, pop_index):
        _check(lib().afqmc_set_cadence(self.h, mgs_index, pop_index))

    def set_stream(self, stream_ptr):
        _check(lib().afqmc_set_stream(self.h, stream_ptr))

    def set_graphs(self, enable=True):
        _check(lib().afqmc_set_graphs(self.h, 1 if enable else 0))

    def synchronize(self):
        _check(lib().afqmc_synchronize(self.h))

    # driver pieces
    def step(self, nsteps=1):
        _check(lib().afqmc_project_one_step(self.h, nsteps))

    def project_half(self, which):
        _check(lib().afqmc_project_half(self.h, which))

    def modify_gm(self):
        _check(lib().afqmc_modify_gm(self.h))

    def pop_control(self):
        table = np.zeros(self.W, np.int32)
        weight = np.zeros(self.W)
        _check(lib().afqmc_pop_control(self.h, _p(table), _p(weight)))
        return table, weight

    def reset_measurement(self):
        _check(lib().afqmc_reset_measurement(self.h))

    def add_mixed_measurement(self):
        _check(lib().afqmc_add_mixed_measurement(self.h))

    def measurement(self):
        out = np.zeros(5, np.complex128)
        _check(lib().afqmc_get_measurement(self.h, _p(out)))
        return out

    def cholesky_nums(self):
        b = np.zeros(self.G, np.complex128)
        e = np.zeros(self.G, np.complex128)
        _check(lib().afqmc_get_cholesky_nums(self.h, _p(b), _p(e)))
        return b, e

    def set_observables(self, on=True):
        _check(lib().afqmc_cp_set_observables(self.h, 1 if on else 0))
        self.observe = bool(on)

    # back-propagation (constrained path, FP64 form, observe estimator on)
    def bp_begin(self, steps, measure_skip):
        """prepareBackPropagation: open a window of `steps` recorded steps."""
        _check(lib().afqmc_cp_bp_begin(self.h, int(steps), int(measure_skip)))

    def bp_measure(self):
        """addMeasurement of the back-propagation driver (window full)."""
        _check(lib().afqmc_cp_bp_measure(self.h))

    def bp_state(self):
        """(window open, BPIndex)."""
        a, i = ctypes.c_int(), ctypes.c_int()
        _check(lib().afqmc_cp_bp_state(self.h, ctypes.byref(a), ctypes.byref(i)))
        return bool(a.value), i.value

    def observables(self):
        """greenMatrixNum, densityDensityNum (n x n), splusSminusNum,
        sminusSplusNum, spairSpairNum (L x L): the observe estimator's sums."""
        n, L = self.n, self.n // 2
        out = [np.zeros((n, n), np.complex128, order="F") for _ in range(2)]
        out += [np.zeros((L, L), np.complex128, order="F") for _ in range(3)]
        _check(lib().afqmc_get_observables(self.h, *[_p(a) for a in out]))
        return dict(zip(["greenMatrixNum", "densityDensityNum", "splusSminusNum", "sminusSplusNum",
                         "spairSpairNum"], out))

    def site_nums(self):
        """NupNum, NdnNum, SplusNum, SminusNum (L complex each), CP only."""
        L = self.n // 2
        out = [np.zeros(L, np.complex128) for _ in range(4)]
        _check(lib().afqmc_get_site_nums(self.h, *[_p(a) for a in out]))
        return out

    def update_background_only(self, bg):
        """New background for the two-body sampling; the one-body operators
        stay as they are (updateBackGround without a propagator rebuild)."""
        b = np.ascontiguousarray(bg, dtype=np.float64)
        _check(lib().afqmc_pl_update_background(self.h, _p(b), None, 0.0, None, 0.0, None, 0.0))

    def rebuild_propagators(self, K):
        """expMinusDtK, expHalfDtK and expMinusHalfDtK rebuilt on the GPU from
        the engine's current background and the model's one-body K
        (RealMaterialMolecule::returnExpMinusAlphaK)."""
        k = np.asfortranarray(K, dtype=np.float64)
        _check(lib().afqmc_pl_rebuild_propagators(self.h, _p(k)))

    def update_background(self, m):
        """m: MoleculeInputs after set_background()."""
        a = [_d(m.bg), _z(m.expMinusDtK), _z(m.expHalfDtK), _z(m.expMinusHalfDtK)]
        _check(lib().afqmc_pl_update_background(self.h, _p(a[0]), _p(a[1]), float(m.logwDt),
                                                _p(a[2]), -float(m.logwHalf), _p(a[3]),
                                                float(m.logwHalf)))

    # diagnostics
    def log_overlaps(self):
        out = np.zeros(self.W, np.complex128)
        _check(lib().afqmc_log_overlaps(self.h, _p(out)))
        return out

    def green(self, w, spin=0):
        out = np.zeros((self.n, self.n), np.complex128, order="F")
        _check(lib().afqmc_green_matrix(self.h, w, spin, _p(out)))
        return out

    def taylor_stats(self):
        c, t = ctypes.c_longlong(), ctypes.c_longlong()
        mn, mx = ctypes.c_int(), ctypes.c_int()
        _check(lib().afqmc_taylor_stats(self.h, ctypes.byref(c), ctypes.byref(t),
                                        ctypes.byref(mn), ctypes.byref(mx)))
        return c.value, t.value, mn.value, mx.value

    def profile(self, on=True):
        _check(lib().afqmc_profile_enable(self.h, 1 if on else 0))

    def profile_get(self):
        ms = np.zeros(len(PHASES))
        cnt = np.zeros(len(PHASES), np.int64)
        _check(lib().afqmc_profile_get(self.h, _p(ms), _p(cnt)))
        return {PHASES[i]: (float(ms[i]), int(cnt[i])) for i in range(len(PHASES))}

    def adjoint(self, want_chol=True, chol_out=None):
        """Mixed local energy, mean log-overlap and their gradients (afqmc_pl_adjoint).
        chol_out: optional complex128 torch tensor of n*n*G elements on the
        engine's GPU that receives dE/dL_g (column-major n x n x G) in place of
        a host array; the result's "dE_dchol" is then that tensor."""
        n, G, nu, nd = self.n, self.G, self.nup, self.ndn
        E = np.zeros(1, np.complex128)
        L = np.zeros(1, np.complex128)
        dt = np.zeros((n, n), np.complex128, order="F")
        if chol_out is not None:
            if not chol_out.is_cuda or chol_out.numel() != n * n * G or not chol_out.is_contiguous() \
                    or str(chol_out.dtype) != "torch.complex128":
                raise AfqmcError("chol_out must be a contiguous complex128 CUDA tensor of n*n*G elements")
            dc = chol_out
        else:
            dc = np.zeros((n, n, G), np.complex128, order="F") if want_chol else None
        du = np.zeros((n, nu), np.complex128, order="F")
        dd = np.zeros((n, max(nd, 1)), np.complex128, order="F")
        lu = np.zeros((n, nu), np.complex128, order="F")
        ld = np.zeros((n, max(nd, 1)), np.complex128, order="F")
        dcp = ctypes.c_void_p(dc.data_ptr()) if chol_out is not None else _p(dc)
        _check(lib().afqmc_pl_adjoint(self.h, _p(E), _p(L), _p(dt), dcp, _p(du),
                                      _p(dd) if nd else None, _p(lu), _p(ld) if nd else None))
        return {"E": E[0], "mean_logov": L[0], "dE_dt": dt, "dE_dchol": dc,
                "dE_dconj_phiT": (du, dd[:, :nd]), "dlogov_dconj_phiT": (lu, ld[:, :nd])}

    def pop_weights(self):
        w = np.zeros(self.W)
        _check(lib().afqmc_pop_weights(self.h, _p(w)))
        return w

    def walker_bytes(self):
        return int(lib().afqmc_walker_bytes(self.h))

    def copy_walker_out(self, w, dst_ptr):
        _check(lib().afqmc_copy_walker_out(self.h, w, dst_ptr))

    def copy_walker_in(self, w, src_ptr):
        _check(lib().afqmc_copy_walker_in(self.h, w, src_ptr))

    def pack_walkers(self, idx, dst_ptr):
        i = np.ascontiguousarray(idx, dtype=np.int32)
        _check(lib().afqmc_pack_walkers(self.h, len(i), _p(i), dst_ptr))

    def unpack_walkers(self, slots, src_ptr):
        i = np.ascontiguousarray(slots, dtype=np.int32)
        _check(lib().afqmc_unpack_walkers(self.h, len(i), _p(i), src_ptr))

    def apply_table(self, table):
        t = np.ascontiguousarray(table, dtype=np.int32)
        _check(lib().afqmc_apply_table(self.h, _p(t)))

    def status(self):
        s = ctypes.c_int()
        _check(lib().afqmc_status(self.h, ctypes.byref(s)))
        return s.value


def cp_engine(m, W, seed, mgs_step=10, pop_step=40, force_type="dynamicForce",
              precision=AFQMC_FP64, const_force=None):
    """Constrained-path Hubbard engine from a HubbardInputs bundle."""
    keep = [_z(m.K), _z(m.expMinusDtK), _z(m.expHalfDtK), _z(m.expMinusHalfDtK), _d(m.U),
            _d(m.mu), _d(m.hx), _d(m.hy), _d(m.hz), _d(const_force), _z(m.phiT)]
    h = ctypes.c_void_p()
    _check(lib().afqmc_cp_create(m.L, m.N, W, DECOMP[m.decomp], FORCE[force_type], m.dt, m.ET,
                                 m.force_cap, mgs_step, pop_step, precision,
                                 *[_p(a) for a in keep], float(np.real(m.logwT)),
                                 float(np.imag(m.logwT)), seed, ctypes.byref(h)))
    return Engine(h.value, "cp", 2 * m.L, m.N, W)


def pl_engine(m, W, seed, mgs_step=10, pop_step=10, force_type="dynamicForce",
              precision=AFQMC_FP64, log_one_body=False, const_force=None):
    """Phaseless engine from a MoleculeInputs bundle."""
    if log_one_body:
        mats = [None, 0.0, _z(m.logExpHalfDtK), -float(m.logwHalf), _z(m.logExpMinusHalfDtK),
                float(m.logwHalf), _z(m.logExpMinusDtK), float(m.logwDt)]
    else:
        mats = [_z(m.expMinusDtK), float(m.logwDt), _z(m.expHalfDtK), -float(m.logwHalf),
                _z(m.expMinusHalfDtK), float(m.logwHalf), None, 0.0]
    arrs = [_d(m.chol), _d(m.bg), _d(m.t)]
    cf = _z(const_force)
    tu, td = _z(m.phiTUp), _z(m.phiTDn)
    keep = arrs + [mats[0], mats[2], mats[4], mats[6], cf, tu, td]
    margs = [_p(mats[0]), mats[1], _p(mats[2]), mats[3], _p(mats[4]), mats[5], _p(mats[6]),
             mats[7]]
    h = ctypes.c_void_p()
    _check(lib().afqmc_pl_create(m.n, m.nup, m.ndn, m.G, W, FORCE[force_type], m.dt, m.ET,
                                 m.force_cap, mgs_step, pop_step, precision,
                                 *[_p(a) for a in arrs], *margs, _p(cf), _p(tu), _p(td),
                                 float(np.real(m.logwT)), float(np.imag(m.logwT)), seed,
                                 ctypes.byref(h)))
    return Engine(h.value, "pl", m.n, max(m.nup, m.ndn), W, G=m.G, nup=m.nup, ndn=m.ndn,
                  keep=keep)


def gemm_bf16_dev(M, N, K, A, lda, B, ldb, C, ldc, out_bf16=False, splits=1, split_stride=0,
                  alpha=1.0, stream=None):
    """Device-pointer tcgen05 GEMM (see afqmc_gemm_bf16_dev)."""
    _check(lib().afqmc_gemm_bf16_dev(M, N, K, A, lda, B, ldb, C, ldc, 1 if out_bf16 else 0, splits,
                                     split_stride, alpha, stream))


def pop_configuration_noalloc_dev(weights_dev_ptr, uniforms_dev_ptr, table_dev_ptr, W,
                                  stream=None):
    """popConfiguration that allocates nothing (see afqmc_pop_configuration_noalloc_dev)."""
    _check(lib().afqmc_pop_configuration_noalloc_dev(W, weights_dev_ptr, uniforms_dev_ptr,
                                                     table_dev_ptr, stream))


def pop_configuration_host(weights, uniforms, size=1):
    """popConfiguration(size, weight) with explicit uniforms (host)."""
    w = np.ascontiguousarray(weights, dtype=np.float64)
    u = np.ascontiguousarray(uniforms, dtype=np.float64)
    table = np.zeros(len(w), np.int32)
    _check(lib().afqmc_pop_configuration_host(len(w), size, _p(w), _p(u), _p(table)))
    return table


def bounded_wait_check(limit_cycles, stream=None):
    """Error bits of the bounded-wait self-check (see afqmc_bounded_wait_check)."""
    w = ctypes.c_int(-1)
    _check(lib().afqmc_bounded_wait_check(int(limit_cycles), ctypes.byref(w), stream))
    return w.value


def set_autotune(enable=True):
    _check(lib().afqmc_set_autotune(1 if enable else 0))


class Batch:
    """Engines advanced together, one graph launch per step (afqmc_batch_*)."""

    def __init__(self, engines):
        self.engines = list(engines)
        arr = (ctypes.c_void_p * len(self.engines))(*[e.h for e in self.engines])
        h = ctypes.c_void_p()
        _check(lib().afqmc_batch_create(arr, len(self.engines), ctypes.byref(h)))
        self.h = h.value

    def step(self, nsteps=1):
        _check(lib().afqmc_batch_step(self.h, nsteps))

    def synchronize(self):
        _check(lib().afqmc_batch_synchronize(self.h))

    def set_stream(self, stream_ptr):
        _check(lib().afqmc_batch_set_stream(self.h, stream_ptr))

    def close(self):
        if getattr(self, "h", None):
            lib().afqmc_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def launch_count():
    return int(lib().afqmc_launch_count())


def pop_configuration_dev(weights_dev_ptr, uniforms_dev_ptr, table_dev_ptr, W, stream=None):
    _check(lib().afqmc_pop_configuration_dev(W, weights_dev_ptr, uniforms_dev_ptr, table_dev_ptr,
                                             stream))
