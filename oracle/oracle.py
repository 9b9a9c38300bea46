"""ctypes binding of the CPU oracle (oracle/afqmc_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / --impl reference legs of bench.py, never by the product.

Arrays follow the reference's storage: complex128, column-major (Fortran
order), walkers stacked along the last axis.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# AFQMC_ORACLE_BLAS (a BLAS shared library) selects the build whose GEMM- and
# GEMV-shaped work runs through that BLAS: the timed CPU baseline.  The
# checker is the plain build.
_LIB = os.path.join(_HERE, "liboracle_blas.so" if os.environ.get("AFQMC_ORACLE_BLAS") else "liboracle.so")
_lib = None

c_int, c_double, c_u64, c_void_p, c_char = (ctypes.c_int, ctypes.c_double, ctypes.c_uint64,
                                           ctypes.c_void_p, ctypes.c_char)


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def scipy_blas():
    """(path, symbol prefix) of the OpenBLAS that scipy bundles, or None."""
    import glob
    import scipy
    libs = glob.glob(os.path.join(os.path.dirname(scipy.__file__) + ".libs", "libscipy_openblas*.so"))
    return (libs[0], "scipy_") if libs else None


def blas_available():
    return bool(lib().or_blas_available())


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(
                os.path.join(_HERE, "afqmc_oracle.c")):
            build()
        _lib = ctypes.CDLL(_LIB)
        _declare(_lib)
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(c_void_p)


def _z(a):
    if a is None:
        return None
    return np.asfortranarray(a, dtype=np.complex128)


def _d(a):
    if a is None:
        return None
    return np.ascontiguousarray(a, dtype=np.float64)


class C2(ctypes.Structure):
    """A C99 `double complex` passed or returned by value."""
    _fields_ = [("re", c_double), ("im", c_double)]


def _declare(L):
    P = c_void_p
    L.or_blas_available.restype = c_int
    L.or_rng_bits.restype = c_u64
    L.or_rng_bits.argtypes = [c_u64, c_u64]
    L.or_rng_uniform_at.restype = c_double
    L.or_rng_uniform_at.argtypes = [c_u64, c_u64]
    L.or_rng_fill_uniform.argtypes = [c_u64, c_u64, c_int, P]
    L.or_qr.restype = c_double
    L.or_qr.argtypes = [c_int, c_int, P, P]
    L.or_zgetrf.restype = c_int
    L.or_zgetrf.argtypes = [c_int, P, c_int, P]
    L.or_sd_normalize_ratio.restype = C2
    L.or_sd_normalize_ratio.argtypes = [c_int, c_int, P, P]
    L.or_sd2is_normalize_ratio.restype = C2
    L.or_sd2is_normalize_ratio.argtypes = [c_int, c_int, c_int, P, P]
    L.or_sd2s_normalize_ratio.restype = C2
    L.or_sd2s_normalize_ratio.argtypes = [c_int, c_int, c_int, P, P, P]
    L.or_sdsd.restype = c_int
    L.or_sdsd.argtypes = [c_int, c_int, P, C2, P, C2, P, P, P, P]
    L.or_sd2s_sd2is.restype = c_int
    L.or_sd2s_sd2is.argtypes = [c_int, c_int, c_int, P, P, C2, P,
                                C2, P, P, P]
    L.or_loghop_apply.restype = c_int
    L.or_loghop_apply.argtypes = [c_int, c_int, c_double, c_int, c_char, c_int, c_int, P, P, P]
    L.or_pop_configuration.restype = c_int
    L.or_pop_configuration.argtypes = [c_int, c_int, P, P, P]
    L.or_pop_fill_from_counts.restype = c_int
    L.or_pop_fill_from_counts.argtypes = [c_int, c_int, P, P]
    L.or_pop_check.argtypes = [c_int, P, P, P, P]
    L.or_niupnidn_consts.argtypes = [c_int, c_double, c_int, P, P, P, P, P, P, P, P, P, P, P]
    L.or_exp2by2.argtypes = [P, P, P]
    L.or_cp_create.restype = P
    L.or_cp_create.argtypes = [c_int, c_int, c_int, c_int, c_int, c_double, c_double, c_double,
                               c_int, c_int, P, P, P, P, P, P, P, P, P, P, P, c_double, c_double,
                               c_u64]
    L.or_pl_create.restype = P
    L.or_pl_create.argtypes = [c_int, c_int, c_int, c_int, c_int, c_int, c_double, c_double,
                               c_double, c_int, c_int, P, P, P, P, c_double, P, c_double, P,
                               c_double, P, c_double, P, P, P, c_double, c_double, c_u64]
    L.or_destroy.argtypes = [P]
    L.or_set_walkers.argtypes = [P, P, P, P]
    L.or_get_walkers.argtypes = [P, P, P, P]
    L.or_set_rng.argtypes = [P, c_u64, c_u64]
    L.or_get_rng_counter.restype = c_u64
    L.or_get_rng_counter.argtypes = [P]
    L.or_set_ET.argtypes = [P, c_double]
    L.or_pl_update_background.argtypes = [P, P, P, c_double, P, c_double, P, c_double]
    L.or_set_threads.argtypes = [P, c_int]
    L.or_log_overlaps.argtypes = [P, P]
    L.or_green_matrix.argtypes = [P, c_int, c_int, P]
    L.or_modify_gm.argtypes = [P]
    L.or_pop_control.argtypes = [P, P, P]
    L.or_pop_weights.argtypes = [P, P]
    L.or_cp_set_observables.argtypes = [P, c_int]
    L.or_get_observables.argtypes = [P, P]
    L.or_pl_two_body_sample.argtypes = [P, P, P, P, P]
    L.or_project_one_step.argtypes = [P, c_int]
    L.or_set_cadence.argtypes = [P, c_int, c_int]
    L.or_project_half.argtypes = [P, c_int]
    L.or_reset_measurement.argtypes = [P]
    L.or_add_mixed_measurement.argtypes = [P, P, P]
    L.or_get_measurement.argtypes = [P, P]
    L.or_get_cholesky_nums.argtypes = [P, P, P]
    L.or_get_site_nums.argtypes = [P, P]
    L.or_pl_force_single.argtypes = [P, c_int, P, P]
    L.or_cp_force_single.argtypes = [P, c_int, P]
    L.or_taylor_stats_get.argtypes = [P, P, P, P, P]


def _c2(z):
    return C2(float(np.real(z)), float(np.imag(z)))


def _cz(r):
    return complex(r.re, r.im)


# ---------------------------------------------------------------- pieces
def rng_uniform(seed, start, count):
    out = np.empty(count)
    lib().or_rng_fill_uniform(seed, start, count, _p(out))
    return out


def qr(ph):
    ph = _z(ph).copy(order="F")
    L, N = ph.shape
    det_list = np.zeros(N)
    det = lib().or_qr(L, N, _p(ph), _p(det_list))
    return ph, det, det_list


def sd_normalize(wf):
    wf = _z(wf).copy(order="F")
    ratio = c_double()
    r = lib().or_sd_normalize_ratio(wf.shape[0], wf.shape[1], _p(wf), ctypes.byref(ratio))
    return wf, _cz(r), ratio.value


def sd2is_normalize(wf, nup, ndn):
    wf = _z(wf).copy(order="F")
    ratio = c_double()
    r = lib().or_sd2is_normalize_ratio(wf.shape[0], nup, ndn, _p(wf), ctypes.byref(ratio))
    return wf, _cz(r), ratio.value


def sd2s_normalize(wf_up, wf_dn):
    wu = _z(wf_up).copy(order="F")
    wd = _z(wf_dn).copy(order="F")
    ratio = c_double()
    r = lib().or_sd2s_normalize_ratio(wu.shape[0], wu.shape[1], wd.shape[1], _p(wu), _p(wd),
                                      ctypes.byref(ratio))
    return wu, wd, _cz(r), ratio.value


def sdsd(phiT, logwT, phi, logw):
    """SDSDOperation: (logOverlap, thetaT (N x n), greenDiag, greenOffDiag, info)."""
    phiT = _z(phiT)
    phi = _z(phi)
    n, N = phi.shape
    lo = np.zeros(1, np.complex128)
    th = np.zeros((N, n), np.complex128, order="F")
    gd = np.zeros(n, np.complex128)
    god = np.zeros(n, np.complex128)
    info = lib().or_sdsd(n, N, _p(phiT), _c2(logwT), _p(phi), _c2(logw), _p(lo), _p(th), _p(gd),
                         _p(god) if n % 2 == 0 else None)
    return lo[0], th, gd, god, info


def sd2s_sd2is(phiTUp, phiTDn, logwT, phi, logw, nup, ndn):
    phiTUp, phiTDn, phi = _z(phiTUp), _z(phiTDn), _z(phi)
    n = phi.shape[0]
    lo = np.zeros(1, np.complex128)
    tu = np.zeros((nup, n), np.complex128, order="F")
    td = np.zeros((max(ndn, 1), n), np.complex128, order="F")
    info = lib().or_sd2s_sd2is(n, nup, ndn, _p(phiTUp), _p(phiTDn), _c2(logwT), _p(phi),
                               _c2(logw), _p(lo), _p(tu), _p(td))
    return lo[0], tu, td[:ndn], info


def loghop_apply(M, wf, flag="dynamicOrder", order=0, accuracy=1e-10, base=3, trans="N"):
    M, wf = _z(M), _z(wf)
    out = np.zeros_like(wf, order="F")
    fl = 0 if flag == "fixedOrder" else 1
    k = lib().or_loghop_apply(fl, order, accuracy, base, trans.encode(), wf.shape[0], wf.shape[1],
                              _p(M), _p(wf), _p(out))
    return out, k


def pop_configuration(weights, uniforms, size=1):
    w = _d(weights)
    u = _d(uniforms)
    table = np.zeros(len(w), np.int32)
    bad = lib().or_pop_configuration(len(w), size, _p(w), _p(u), _p(table))
    return table, bad


def pop_fill_from_counts(counts, size=1):
    c = np.ascontiguousarray(counts, dtype=np.int32)
    table = np.zeros(len(c), np.int32)
    bad = lib().or_pop_fill_from_counts(len(c), size, _p(c), _p(table))
    return table, bad


def pop_check(weights):
    w = _d(weights)
    a, b, c = c_double(), c_double(), c_double()
    lib().or_pop_check(len(w), _p(w), ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
    return a.value, b.value, c.value


DECOMP = {"densityCharge": 0, "densitySpin": 1, "hopCharge": 2, "hopSpin": 3}


def niupnidn_consts(dt, decomp, U, mu, hx, hy, hz):
    L = len(U)
    out = [np.zeros(L, np.complex128) for _ in range(5)]
    s = c_double()
    lib().or_niupnidn_consts(L, dt, DECOMP[decomp], _p(_d(U)), _p(_d(mu)), _p(_d(hx)), _p(_d(hy)),
                             _p(_d(hz)), *[_p(o) for o in out], ctypes.byref(s))
    return out + [s.value]


# ---------------------------------------------------------------- engines
class Engine:
    """One driver population (CP or phaseless) on the CPU oracle."""

    def __init__(self, handle, kind, n, ncol, W, G=0, nup=0, ndn=0):
        self.h = handle
        self.kind, self.n, self.ncol, self.W, self.G = kind, n, ncol, W, G
        self.nup, self.ndn = nup, ndn

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_destroy(self.h)
            self.h = None

    def set_walkers(self, wf, logw, alive):
        wf = np.asfortranarray(wf, dtype=np.complex128)
        assert wf.shape == (self.n, self.ncol, self.W)
        lw = np.ascontiguousarray(logw, dtype=np.complex128)
        al = np.ascontiguousarray(alive, dtype=np.int32)
        lib().or_set_walkers(self.h, _p(wf), _p(lw), _p(al))

    def get_walkers(self):
        wf = np.zeros((self.n, self.ncol, self.W), np.complex128, order="F")
        lw = np.zeros(self.W, np.complex128)
        al = np.zeros(self.W, np.int32)
        lib().or_get_walkers(self.h, _p(wf), _p(lw), _p(al))
        return wf, lw, al

    def set_rng(self, seed, counter=0):
        self.seed = seed
        lib().or_set_rng(self.h, seed, counter)

    def rng_state(self):
        return self.seed, self.rng_counter()

    def rng_counter(self):
        return lib().or_get_rng_counter(self.h)

    def set_ET(self, ET):
        lib().or_set_ET(self.h, ET)

    def set_cadence(self, mgs_index, pop_index):
        lib().or_set_cadence(self.h, mgs_index, pop_index)

    def update_background_only(self, bg):
        """updateBackGround: new background, one-body operators unchanged."""
        b = np.ascontiguousarray(bg, dtype=np.float64)
        lib().or_pl_update_background(self.h, _p(b), None, 0.0, None, 0.0, None, 0.0)
        self.bg = b.copy()

    def update_background(self, m):
        """New background and the dense propagators rebuilt from it (m: a
        MoleculeInputs after set_background)."""
        a = [np.ascontiguousarray(m.bg, dtype=np.float64), _z(m.expMinusDtK), _z(m.expHalfDtK),
             _z(m.expMinusHalfDtK)]
        lib().or_pl_update_background(self.h, _p(a[0]), _p(a[1]), float(m.logwDt), _p(a[2]),
                                      -float(m.logwHalf), _p(a[3]), float(m.logwHalf))
        self.bg = a[0].copy()

    def rebuild_propagators(self, K):
        """expMinusDtK, expMinusHalfDtK, expHalfDtK = returnExpMinusAlphaK(dt,
        dt/2, -dt/2) from the current background, by the reference's route
        (realMaterialMolecule.cpp:117-131, 155-178): Kp = K + sum_g bg_g L_g,
        its eigensystem, V exp(-alpha lambda) V^T, logw = alpha/2 sum bg^2."""
        n, G = self.n, self.G
        Kp = np.asarray(K, dtype=np.float64) + (self.chol.reshape(n * n, G, order="F") @ self.bg).reshape(
            n, n, order="F")
        lam, V = np.linalg.eigh(Kp)
        bg2 = float(sum(b * b for b in self.bg))

        def ex(alpha):
            return _z((V * np.exp(-alpha * lam)) @ V.T)

        a = [ex(self.dt), ex(-0.5 * self.dt), ex(0.5 * self.dt)]
        b = np.ascontiguousarray(self.bg, dtype=np.float64)
        lib().or_pl_update_background(self.h, _p(b), _p(a[0]), self.dt * 0.5 * bg2, _p(a[1]),
                                      -0.5 * self.dt * 0.5 * bg2, _p(a[2]), 0.5 * self.dt * 0.5 * bg2)

    def log_overlaps(self):
        out = np.zeros(self.W, np.complex128)
        lib().or_log_overlaps(self.h, _p(out))
        return out

    def green(self, w, spin=0):
        out = np.zeros((self.n, self.n), np.complex128, order="F")
        lib().or_green_matrix(self.h, w, spin, _p(out))
        return out

    def step(self, nsteps=1):
        lib().or_project_one_step(self.h, nsteps)

    def set_threads(self, nthreads):
        """Walker-parallel host threads for the step, modifyGM and the
        measurement; results do not depend on the count."""
        lib().or_set_threads(self.h, int(nthreads))

    def modify_gm(self):
        lib().or_modify_gm(self.h)

    def pop_control(self):
        table = np.zeros(self.W, np.int32)
        weight = np.zeros(self.W)
        lib().or_pop_control(self.h, _p(table), _p(weight))
        return table, weight

    def two_body_sample(self, aux, force):
        """(M, logw) of getTwoBodySampleFromAuxForce for explicit aux and force."""
        a = np.ascontiguousarray(aux, dtype=np.complex128)
        f = np.ascontiguousarray(force, dtype=np.complex128)
        M = np.zeros((self.n, self.n), np.complex128, order="F")
        lw = np.zeros(1, np.complex128)
        lib().or_pl_two_body_sample(self.h, _p(a), _p(f), _p(M), _p(lw))
        return M, lw[0]

    def pop_weights(self):
        w = np.zeros(self.W)
        lib().or_pop_weights(self.h, _p(w))
        return w

    def project_half(self, which):
        lib().or_project_half(self.h, which)

    def reset_measurement(self):
        lib().or_reset_measurement(self.h)

    def add_mixed_measurement(self):
        el = np.zeros(self.W, np.complex128)
        dn = np.zeros(self.W, np.complex128)
        lib().or_add_mixed_measurement(self.h, _p(el), _p(dn))
        return el, dn

    def measurement(self):
        out = np.zeros(5, np.complex128)
        lib().or_get_measurement(self.h, _p(out))
        return out

    def set_observables(self, on=True):
        lib().or_cp_set_observables(self.h, 1 if on else 0)
        self.observe = bool(on)

    def observables(self):
        n, L = self.n, self.n // 2
        out = np.zeros(11 * L * L, np.complex128)
        lib().or_get_observables(self.h, _p(out))
        names = ["greenMatrixNum", "densityDensityNum", "splusSminusNum", "sminusSplusNum",
                 "spairSpairNum"]
        sizes = [(n, n), (n, n), (L, L), (L, L), (L, L)]
        res, off = {}, 0
        for nm, sh in zip(names, sizes):
            k = sh[0] * sh[1]
            res[nm] = out[off:off + k].reshape(sh, order="F")
            off += k
        return res

    def site_nums(self):
        """NupNum, NdnNum, SplusNum, SminusNum (L complex each), CP only."""
        L = self.n // 2
        out = np.zeros(4 * L, np.complex128)
        lib().or_get_site_nums(self.h, _p(out))
        return [out[k * L:(k + 1) * L] for k in range(4)]

    def cholesky_nums(self):
        b = np.zeros(self.G, np.complex128)
        e = np.zeros(self.G, np.complex128)
        lib().or_get_cholesky_nums(self.h, _p(b), _p(e))
        return b, e

    def cp_force(self, w):
        out = np.zeros(self.n // 2)
        lib().or_cp_force_single(self.h, w, _p(out))
        return out

    def pl_force(self, w):
        xb = np.zeros(self.G, np.complex128)
        f = np.zeros(self.G, np.complex128)
        lib().or_pl_force_single(self.h, w, _p(xb), _p(f))
        return xb, f

    def taylor_stats(self):
        c, t = ctypes.c_long(), ctypes.c_long()
        mn, mx = c_int(), c_int()
        lib().or_taylor_stats_get(self.h, ctypes.byref(c), ctypes.byref(t), ctypes.byref(mn),
                                  ctypes.byref(mx))
        return c.value, t.value, mn.value, mx.value


def cp_engine(m, W, seed, mgs_step=10, pop_step=40, force_type="dynamicForce"):
    """m: a HubbardInputs (afqmclab_b200.inputs) bundle."""
    keep = []

    def z(a):
        a = _z(a)
        keep.append(a)
        return _p(a)

    def d(a):
        a = _d(a)
        keep.append(a)
        return _p(a)

    h = lib().or_cp_create(m.L, m.N, W, DECOMP[m.decomp], 0 if force_type == "dynamicForce" else 1,
                           m.dt, m.ET, m.force_cap, mgs_step, pop_step, z(m.K), z(m.expMinusDtK),
                           z(m.expHalfDtK), z(m.expMinusHalfDtK), d(m.U), d(m.mu), d(m.hx),
                           d(m.hy), d(m.hz), None, z(m.phiT), float(np.real(m.logwT)),
                           float(np.imag(m.logwT)), seed)
    eng = Engine(h, "cp", 2 * m.L, m.N, W)
    eng.seed = seed
    return eng


def pl_engine(m, W, seed, mgs_step=10, pop_step=10, force_type="dynamicForce", log_one_body=False):
    """m: a MoleculeInputs bundle."""
    keep = []

    def z(a):
        if a is None:
            return None
        a = _z(a)
        keep.append(a)
        return _p(a)

    def d(a):
        a = np.asfortranarray(a, dtype=np.float64)
        keep.append(a)
        return _p(a)

    if log_one_body:
        args = [None, 0.0, z(m.logExpHalfDtK), -float(m.logwHalf), z(m.logExpMinusHalfDtK),
                float(m.logwHalf), z(m.logExpMinusDtK), float(m.logwDt)]
    else:
        args = [z(m.expMinusDtK), float(m.logwDt), z(m.expHalfDtK), -float(m.logwHalf),
                z(m.expMinusHalfDtK), float(m.logwHalf), None, 0.0]
    h = lib().or_pl_create(m.n, m.nup, m.ndn, m.G, W, 0 if force_type == "dynamicForce" else 1,
                           m.dt, m.ET, m.force_cap, mgs_step, pop_step, d(m.chol), d(m.bg), d(m.t),
                           *args, None, z(m.phiTUp), z(m.phiTDn), float(np.real(m.logwT)),
                           float(np.imag(m.logwT)), seed)
    eng = Engine(h, "pl", m.n, max(m.nup, m.ndn), W, G=m.G, nup=m.nup, ndn=m.ndn)
    eng.seed = seed
    # the model arrays the propagator rebuild reads
    eng.chol = np.asfortranarray(m.chol, dtype=np.float64)
    eng.bg = np.array(m.bg, dtype=np.float64)
    eng.dt = float(m.dt)
    return eng
