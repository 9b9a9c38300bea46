"""Seeded synthetic inputs for the AFQMC walker step.

These play the role of the reference's input scripts
(scripts/supercubic/setHoping.py, scripts/pyscf/molecule.py,
tutorials/afqmcConstraintPath/scripts/generateInputFile.py): they build the
Hamiltonian, the trial determinant and the one-body propagators that the
reference's models return (HubbardSOC::returnExpMinusAlphaK,
HubbardSOC.cpp:109-118; RealMaterialMolecule::returnExpMinusAlphaK /
returnLogExpMinusAlphaK, realMaterialMolecule.cpp:117-146), and can write
them in the reference's file formats (HubbardSOC::write, HubbardSOC.cpp:61-75;
SD::write, SD.cpp:85-103; afqmc_param key/value files).

No dataset is involved: every matrix is generated from a fixed seed.
"""
from dataclasses import dataclass, field

import numpy as np


# ----------------------------------------------------------------- Hubbard
@dataclass
class HubbardInputs:
    nx: int
    ny: int
    L: int                 # sites; walker rows n = 2L (spin-orbit basis)
    N: int                 # electrons = determinant columns
    nup: int
    ndn: int
    U_val: float
    dt: float
    decomp: str
    K: np.ndarray          # 2L x 2L complex (HubbardSOC::K)
    U: np.ndarray
    mu: np.ndarray
    hx: np.ndarray
    hy: np.ndarray
    hz: np.ndarray
    phiT: np.ndarray       # 2L x N complex trial
    logwT: complex
    expMinusDtK: np.ndarray
    expHalfDtK: np.ndarray
    expMinusHalfDtK: np.ndarray
    ET: float = -10.0
    force_cap: float = 1.5

    @property
    def n(self):
        return 2 * self.L


def square_lattice_hopping(nx, ny, t=1.0, tp=0.0):
    """Nearest (t) and next-nearest (tp) neighbour hopping on a periodic
    nx x ny lattice, -t c_i^+ c_j convention (scripts/supercubic/setHoping.py:4-62)."""
    L = nx * ny
    H = np.zeros((L, L))

    def idx(x, y):
        return (x % nx) + nx * (y % ny)

    for y in range(ny):
        for x in range(nx):
            i = idx(x, y)
            for dx, dy, amp in ((1, 0, t), (0, 1, t), (1, 1, tp), (1, -1, tp)):
                if amp == 0.0:
                    continue
                j = idx(x + dx, y + dy)
                if i == j:
                    continue
                H[i, j] += -amp
                H[j, i] += -amp
    return H


def exp_minus_alpha(Kmat, alpha):
    """V exp(-alpha lambda) V^dagger from the Hermitian eigensystem of K."""
    lam, V = np.linalg.eigh(Kmat)
    return (V * np.exp(-alpha * lam)) @ V.conj().T


def _plane_wave_trial(nx, ny, nocc):
    """nocc lowest free-electron orbitals on the torus.  In an open shell the
    degenerate level is filled by a fixed choice: real cos/sin combinations
    of the plane waves in lexicographic (kx, ky) order."""
    L = nx * ny
    ks = []
    for a in range(nx):
        for b in range(ny):
            kx = 2 * np.pi * a / nx
            ky = 2 * np.pi * b / ny
            ks.append((round(-2 * (np.cos(kx) + np.cos(ky)), 12), a, b))
    ks.sort()
    xs = np.array([i % nx for i in range(L)])
    ys = np.array([i // nx for i in range(L)])
    cols = []
    used = set()
    for e, a, b in ks:
        if len(cols) == nocc:
            break
        if (a, b) in used:
            continue
        kx, ky = 2 * np.pi * a / nx, 2 * np.pi * b / ny
        phase = kx * xs + ky * ys
        partner = ((-a) % nx, (-b) % ny)
        used.add((a, b))
        if partner == (a, b):
            cols.append(np.cos(phase))
        else:
            used.add(partner)
            cols.append(np.cos(phase))
            if len(cols) < nocc:
                cols.append(np.sin(phase))
    M = np.array(cols).T
    q, _ = np.linalg.qr(M)
    return q[:, :nocc]


def _uhf_trial(Hk, nup, ndn, U, seed, iters=60):
    """Seeded unrestricted mean-field solve: start from a random staggered
    density, iterate H_sigma = K + U n_{-sigma} with linear mixing."""
    rng = np.random.default_rng(seed)
    L = Hk.shape[0]
    nu = np.clip(nup / L + 0.2 * rng.standard_normal(L), 0, 1)
    nd = np.clip(ndn / L + 0.2 * rng.standard_normal(L), 0, 1)
    for _ in range(iters):
        _, vu = np.linalg.eigh(Hk + np.diag(U * nd))
        _, vd = np.linalg.eigh(Hk + np.diag(U * nu))
        cu, cd = vu[:, :nup], vd[:, :ndn]
        nu = 0.5 * nu + 0.5 * np.sum(cu * cu, axis=1)
        nd = 0.5 * nd + 0.5 * np.sum(cd * cd, axis=1)
    return cu, cd


def hubbard_inputs(nx=4, ny=4, nup=7, ndn=7, t=1.0, tp=0.0, U=4.0, dt=0.01,
                   decomp="densitySpin", trial="free", seed=20240501):
    """Hubbard model in the reference's spin-orbit form: walker rows are the
    2L spin-orbitals (up sites then down sites), K is 2L x 2L."""
    L = nx * ny
    Hk = square_lattice_hopping(nx, ny, t, tp)
    K = np.zeros((2 * L, 2 * L), np.complex128)
    K[:L, :L] = Hk
    K[L:, L:] = Hk
    N = nup + ndn
    if trial == "free":
        cu = _plane_wave_trial(nx, ny, nup) if nup else np.zeros((L, 0))
        cd = _plane_wave_trial(nx, ny, ndn) if ndn else np.zeros((L, 0))
    else:
        cu, cd = _uhf_trial(Hk, nup, ndn, U, seed)
    phiT = np.zeros((2 * L, N), np.complex128)
    phiT[:L, :nup] = cu
    phiT[L:, nup:] = cd
    zeros = np.zeros(L)
    return HubbardInputs(
        nx=nx, ny=ny, L=L, N=N, nup=nup, ndn=ndn, U_val=U, dt=dt, decomp=decomp, K=K,
        U=np.full(L, float(U)), mu=zeros.copy(), hx=zeros.copy(), hy=zeros.copy(),
        hz=zeros.copy(), phiT=np.asfortranarray(phiT), logwT=0j,
        expMinusDtK=np.asfortranarray(exp_minus_alpha(K, dt)),
        expHalfDtK=np.asfortranarray(exp_minus_alpha(K, -0.5 * dt)),
        expMinusHalfDtK=np.asfortranarray(exp_minus_alpha(K, 0.5 * dt)))


def hubbard_trial_energy(m):
    """<phiT|H|phiT> / <phiT|phiT> of the Hubbard model (hopping, on-site U,
    spin-orbit basis); used as the energy shift E_T of the weights."""
    T = m.phiT
    G = T @ np.linalg.solve(T.conj().T @ T, T.conj().T)   # G[p, q] = <c_q^+ c_p>
    L = m.L
    e = np.trace(m.K @ G)
    d = np.diag(G)
    e += np.sum(m.U * (d[:L] * d[L:] - np.diag(G[L:, :L]) * np.diag(G[:L, L:])))
    return float(e.real)


# ---------------------------------------------------------------- molecule
@dataclass
class MoleculeInputs:
    n: int
    nup: int
    ndn: int
    G: int
    dt: float
    t: np.ndarray          # n x n real one-body (RealMaterialMolecule::t)
    K: np.ndarray          # t - 1/2 sum_g L_g L_g
    chol: np.ndarray       # n x n x G real, Fortran order
    bg: np.ndarray         # G
    phiTUp: np.ndarray
    phiTDn: np.ndarray
    logwT: complex
    Kp: np.ndarray = None
    expMinusDtK: np.ndarray = None
    expHalfDtK: np.ndarray = None
    expMinusHalfDtK: np.ndarray = None
    logExpMinusDtK: np.ndarray = None
    logExpHalfDtK: np.ndarray = None
    logExpMinusHalfDtK: np.ndarray = None
    logwDt: float = 0.0
    logwHalf: float = 0.0
    ET: float = 0.0
    force_cap: float = 1.5
    extra: dict = field(default_factory=dict)

    def set_background(self, bg):
        """RealMaterialMolecule::updateBackGround + propagator rebuild
        (realMaterialMolecule.cpp:103-178)."""
        self.bg = np.array(bg, dtype=np.float64)
        n = self.n
        Lmat = self.chol.reshape(n * n, self.G, order="F")
        self.Kp = self.K + (Lmat @ self.bg).reshape(n, n, order="F")
        bg2 = float(self.bg @ self.bg)
        lam, V = np.linalg.eigh(self.Kp)

        def ex(alpha):
            return np.asfortranarray(((V * np.exp(-alpha * lam)) @ V.T).astype(np.complex128))

        self.expMinusDtK = ex(self.dt)
        self.expMinusHalfDtK = ex(0.5 * self.dt)
        self.expHalfDtK = ex(-0.5 * self.dt)
        self.logwDt = self.dt * 0.5 * bg2
        self.logwHalf = 0.5 * self.dt * 0.5 * bg2
        self.logExpMinusDtK = np.asfortranarray((-self.dt * self.Kp).astype(np.complex128))
        self.logExpMinusHalfDtK = np.asfortranarray((-0.5 * self.dt * self.Kp).astype(np.complex128))
        self.logExpHalfDtK = np.asfortranarray((0.5 * self.dt * self.Kp).astype(np.complex128))


def symmetric_basis(n, G, seed):
    """First G members of a seeded orthonormal basis of real symmetric n x n
    matrices (Frobenius inner product), returned as an n x n x G array."""
    rng = np.random.default_rng(seed)
    iu = np.triu_indices(n)
    dim = len(iu[0])
    X = rng.standard_normal((dim, G))
    Q, _ = np.linalg.qr(X)
    # map the orthonormal coordinate vectors to symmetric matrices: off-diagonal
    # coordinates carry weight 1/sqrt(2) on both mirror entries
    out = np.zeros((n, n, G))
    w = np.where(iu[0] == iu[1], 1.0, 1.0 / np.sqrt(2.0))
    for g in range(G):
        M = np.zeros((n, n))
        M[iu] = Q[:, g] * w
        M = M + np.triu(M, 1).T
        out[:, :, g] = M
    return out


def molecule_inputs(n=128, nup=32, ndn=32, G=640, dt=0.005, decay=60.0, seed=20240502,
                    complex_h1=False):
    """Synthetic molecule-like Hamiltonian: L_g = sqrt(lambda_g) U_g with
    lambda_g = exp(-g/decay) and U_g orthonormal symmetric matrices (a PSD
    4-index tensor with that spectrum), h1 with eigenvalues spaced on
    [-5, 5] Ha, K = h1 - 1/2 sum_g L_g L_g (scripts/pyscf/molecule.py:128-132),
    RHF-like trial from the lowest h1 orbitals."""
    rng = np.random.default_rng(seed + 1)
    Ug = symmetric_basis(n, G, seed)
    lam = np.exp(-np.arange(G) / decay)
    chol = np.asfortranarray(Ug * np.sqrt(lam)[None, None, :])
    Qh, _ = np.linalg.qr(rng.standard_normal((n, n)))
    h1 = (Qh * np.linspace(-5.0, 5.0, n)) @ Qh.T
    h1 = 0.5 * (h1 + h1.T)
    K = h1 - 0.5 * np.einsum("ikg,kjg->ij", chol, chol)
    K = 0.5 * (K + K.T)
    _, V = np.linalg.eigh(h1)
    phiTUp = np.asfortranarray(V[:, :nup].astype(np.complex128))
    phiTDn = np.asfortranarray(V[:, :ndn].astype(np.complex128))
    m = MoleculeInputs(n=n, nup=nup, ndn=ndn, G=G, dt=dt, t=np.asfortranarray(h1),
                       K=np.asfortranarray(K), chol=chol, bg=np.zeros(G), phiTUp=phiTUp,
                       phiTDn=phiTDn, logwT=0j)
    m.set_background(np.zeros(G))
    m.ET = variational_energy(m)
    return m


def variational_energy(m):
    """<phiT|H|phiT>/<phiT|phiT> of the real RHF/UHF trial for
    H = sum t c^+c + 1/2 sum_g (sum L_g c^+c)^2 - 1/2 sum_g L_g L_g c^+c
    (the reference's T + 1/2 sum_g (xbar_g^2 - ex_g) at the trial itself)."""
    Pu = (m.phiTUp @ m.phiTUp.conj().T).real
    Pd = (m.phiTDn @ m.phiTDn.conj().T).real
    e = np.sum(m.t * (Pu + Pd))
    for g in range(m.G):
        Lg = m.chol[:, :, g]
        a = np.sum(Lg * Pu) + np.sum(Lg * Pd)
        ex = np.sum((Lg @ Pu) * (Lg @ Pu).T) + np.sum((Lg @ Pd) * (Lg @ Pd).T)
        e += 0.5 * (a * a - ex)
    return float(e)


# ------------------------------------------------------------------ walkers
def initial_walkers(phiT, W, seed=None, noise=0.0, nup=None, ndn=None):
    """W copies of the trial (setWalkerFromPhiT, SDSDOperation.cpp:188-198);
    with noise > 0 each copy gets a seeded complex perturbation, so parity
    tests exercise walkers that differ from each other.  For SD2is walkers
    pass the spin-up trial (SD2sSD2isOperation.cpp:216-230 picks the larger
    spin block)."""
    n, N = phiT.shape
    wf = np.repeat(np.asarray(phiT)[:, :, None], W, axis=2).astype(np.complex128)
    if noise > 0.0:
        rng = np.random.default_rng(seed)
        wf = wf + noise * (rng.standard_normal(wf.shape) + 1j * rng.standard_normal(wf.shape))
    return np.asfortranarray(wf), np.zeros(W, np.complex128), np.ones(W, np.int32)


# ------------------------------------------------------------------- files
def write_hubbard_model_param(m: HubbardInputs, path):
    """HubbardSOC::write text format (HubbardSOC.cpp:61-75)."""
    with open(path, "w") as f:
        f.write(f"{m.L:26d} \n{m.N:26d} \n")
        for z in np.asarray(m.K).ravel(order="F"):
            f.write(f"{z.real:26.18e} {z.imag:26.18e} \n")
        for arr in (m.mu, m.hx, m.hy, m.hz, m.U):
            for v in arr:
                f.write(f"{v:26.18e} \n")


def _complex_line(z):
    # writeFile(complex, ofstream) (common/readWriteHao/include/readWriteFstream.h):
    # setprecision(16), scientific, two fields of width 26
    return f"{z.real:26.16e}{z.imag:26.16e}\n"


def _matrix_lines(wf):
    # TensorHao::write (tensor_core.h:296-301): rank, shape, then the entries
    # column by column, one per line
    wf = np.asarray(wf)
    out = [f"2\n{wf.shape[0]} {wf.shape[1]} \n"]
    out.extend(_complex_line(z) for z in wf.ravel(order="F"))
    return "".join(out)


def _read_matrix(vals, k):
    rank, r, c = int(vals[k]), int(vals[k + 1]), int(vals[k + 2])
    if rank != 2:
        raise ValueError(f"walker file: matrix rank {rank}, expected 2")
    data = np.array(vals[k + 3:k + 3 + 2 * r * c], dtype=np.float64)
    if data.size != 2 * r * c:
        raise ValueError("walker file: truncated matrix")
    return (data[0::2] + 1j * data[1::2]).reshape((r, c), order="F")


def write_sd(wf, logw, path):
    """SD::write file format (SD.cpp:85-103): logw, then the matrix."""
    with open(path, "w") as f:
        f.write(_complex_line(complex(logw)) + _matrix_lines(wf))


def read_sd(path):
    """SD::read (SD.cpp:85-93): returns (wf, logw)."""
    vals = open(path).read().split()
    logw = complex(float(vals[0]), float(vals[1]))
    return _read_matrix(vals, 2), logw


def write_sd2is(wf, logw, nup, ndn, path):
    """SD2is::write file format (SD2is.cpp:105-127): logw, Nup, Ndn, the matrix."""
    with open(path, "w") as f:
        f.write(_complex_line(complex(logw)) + f"{nup:26d}\n{ndn:26d}\n" + _matrix_lines(wf))


def read_sd2is(path):
    """SD2is::read: returns (wf, logw, nup, ndn)."""
    vals = open(path).read().split()
    logw = complex(float(vals[0]), float(vals[1]))
    nup, ndn = int(vals[2]), int(vals[3])
    return _read_matrix(vals, 4), logw, nup, ndn


CONFIGS = {
    "hubbard4x4": dict(kind="cp", nx=4, ny=4, nup=7, ndn=7, t=1.0, tp=0.0, U=4.0, dt=0.01,
                       W=100, decomp="densitySpin", trial="free", mgs=10, pop=40),
    "hubbard8x8": dict(kind="cp", nx=8, ny=8, nup=28, ndn=28, t=1.0, tp=-0.2, U=4.0, dt=0.005,
                       W=1024, decomp="densitySpin", trial="uhf", mgs=10, pop=40),
    "molecule128": dict(kind="pl", n=128, nup=32, ndn=32, G=640, dt=0.005, W=2048, mgs=10,
                        pop=10),
    "molecule64": dict(kind="pl", n=64, nup=16, ndn=16, G=320, dt=0.005, W=512, mgs=10, pop=10),
    "molecule256": dict(kind="pl", n=256, nup=64, ndn=64, G=1280, dt=0.005, W=512, mgs=10,
                        pop=10),
    # the uneven batch: four lattices of different size and filling, U = 4 and 8
    "hubbard6x6": dict(kind="cp", nx=6, ny=6, nup=16, ndn=16, t=1.0, tp=0.0, U=4.0, dt=0.01,
                       W=1024, decomp="densitySpin", trial="free", mgs=10, pop=40),
    "hubbard8x8u8": dict(kind="cp", nx=8, ny=8, nup=28, ndn=28, t=1.0, tp=0.0, U=8.0, dt=0.01,
                         W=1024, decomp="densitySpin", trial="free", mgs=10, pop=40),
    "hubbard10x10": dict(kind="cp", nx=10, ny=10, nup=40, ndn=40, t=1.0, tp=0.0, U=4.0, dt=0.01,
                         W=1024, decomp="densitySpin", trial="free", mgs=10, pop=40),
    "hubbard12x12u8": dict(kind="cp", nx=12, ny=12, nup=60, ndn=60, t=1.0, tp=0.0, U=8.0,
                           dt=0.01, W=1024, decomp="densitySpin", trial="free", mgs=10, pop=40),
}

# Lattices advanced together as one batch (one graph launch per step).
UNEVEN_BATCH = ["hubbard6x6", "hubbard8x8u8", "hubbard10x10", "hubbard12x12u8"]


def make_config(name, **over):
    c = dict(CONFIGS[name])
    c.update(over)
    if c["kind"] == "cp":
        m = hubbard_inputs(c["nx"], c["ny"], c["nup"], c["ndn"], c["t"], c["tp"], c["U"], c["dt"],
                           c["decomp"], c["trial"])
        m.ET = hubbard_trial_energy(m)
    else:
        m = molecule_inputs(c["n"], c["nup"], c["ndn"], c["G"], c["dt"])
    return m, c
