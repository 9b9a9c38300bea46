"""The oracle and the host-side propagator builders against the explicit
formulas of the reference's own tests (CPU only).  The reference fills its
inputs with SPRNG, which is absent here; the same formulas are checked on
seeded inputs of the same shapes, to the reference tests' tolerance (1e-12).

  - realMaterialMoleculeFixedSD2sSD2isTest.cpp:78-168: the local energy
    T + 1/2 sum (x_g^2) - exchange against explicit 4-index contractions of
    the Green's functions, and the capped force bias.
  - choleskyRealTest.cpp:91-126: the two-body sample matrix and its weight.
  - SDSDOperationTest.cpp:68-97: log-overlap, Green's matrix, its diagonal and
    the two spin-flip off-diagonals.
  - realMaterialMoleculeTest.cpp:137-217: the one-body propagators after a
    background update (returnLogExpMinusAlphaK, returnExpMinusAlphaK).
  - HubbardSOCTest.cpp:78-108: repeated exp(-K) with re-orthonormalisation
    converges to the lowest eigenvectors of K.
"""
import numpy as np
import scipy.linalg as sl

from afqmclab_b200 import inputs
from oracle import oracle as O
from tests.helpers import logov_close

TOL = 1e-12


def SQRT_MINUS(dt):
    """sqrt(-dt * complex(1, 0)) as the reference writes it (choleskyReal.cpp:17,
    choleskyRealTest.cpp:106): the argument's imaginary part is -0.0, so the
    principal root is -i sqrt(dt)."""
    z = np.sqrt(complex(-dt, -0.0))
    assert z.imag < 0
    return z


def _sym(rng, n):
    a = rng.uniform(-1, 1, (n, n))
    return a + a.T


def _cplx(rng, shape):
    return rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)


def _small_molecule(rng, L, nup, ndn, G, dt, cap):
    t = _sym(rng, L)
    chol = np.zeros((L, L, G))
    for g in range(G):
        chol[:, :, g] = _sym(rng, L)
    bg = rng.uniform(-1, 1, G)
    K = t - 0.5 * np.einsum("kjg,kig->ji", chol, chol)
    eye = np.asfortranarray(np.eye(L, dtype=np.complex128))
    phiTUp = np.asfortranarray(_cplx(rng, (L, nup)))
    phiTDn = np.asfortranarray(_cplx(rng, (L, ndn)))
    m = inputs.MoleculeInputs(n=L, nup=nup, ndn=ndn, G=G, dt=dt, t=np.asfortranarray(t),
                              K=np.asfortranarray(K), chol=np.asfortranarray(chol), bg=bg,
                              phiTUp=phiTUp, phiTDn=phiTDn, logwT=0j, force_cap=cap)
    # identity one-body operators: the measurement's half step is then the
    # identity, and the energy is that of the walker as given
    m.expMinusDtK = m.expHalfDtK = m.expMinusHalfDtK = eye
    m.logwDt = m.logwHalf = 0.0
    return m


def _green(phiT, phi):
    """G = conj(phiT) thetaT with thetaT = (phiT^H phi)^-T phi^T (SDSDOperation.cpp:74-89)."""
    S = phiT.conj().T @ phi
    return (phi @ np.linalg.inv(S) @ phiT.conj().T).T


def test_molecule_energy_and_force_match_explicit_contractions():
    rng = np.random.default_rng(5)
    L, nup, ndn, G, dt, cap = 5, 3, 2, 6, 0.01, 0.21
    m = _small_molecule(rng, L, nup, ndn, G, dt, cap)
    o = O.pl_engine(m, 1, 1, 1000, 1000)
    phi = np.asfortranarray(_cplx(rng, (L, nup)))
    o.set_walkers(phi[:, :, None], np.zeros(1, np.complex128), np.ones(1, np.int32))
    Gu = _green(m.phiTUp, phi[:, :nup])
    Gd = _green(m.phiTDn, phi[:, :ndn])
    chol, t = m.chol, m.t
    T = np.sum(t * (Gu + Gd))
    xg = np.einsum("jig,ji->g", chol, Gu + Gd)
    bgE = 0.5 * np.sum(xg * xg)
    exE = 0.5 * np.einsum("lig,kjg,ik,jl->", chol, chol, Gu, Gu) \
        + 0.5 * np.einsum("lig,kjg,ik,jl->", chol, chol, Gd, Gd)
    H = T + bgE - exE
    o.reset_measurement()
    el, dn = o.add_mixed_measurement()
    assert abs(el[0] - H) < TOL * max(1.0, abs(H))
    # force: sqrt(-dt) (xbar - bg), capped in modulus (getForce, :93-116)
    xbar, force = o.pl_force(0)
    assert np.abs(xbar - xg).max() < TOL * max(1.0, np.abs(xg).max())
    f = (xg - m.bg) * SQRT_MINUS(dt)
    f = np.where(np.abs(f) > cap, f / np.abs(f) * cap, f)
    assert np.abs(force - f).max() < TOL


def test_cholesky_two_body_sample_matches_formula():
    rng = np.random.default_rng(6)
    L, G, dt = 10, 5, 0.01
    m = _small_molecule(rng, L, 2, 2, G, dt, 1.0)
    m.chol = np.asfortranarray(rng.uniform(-1, 1, (L, L, G)))
    o = O.pl_engine(m, 1, 1, 1000, 1000)
    force = _cplx(rng, G)
    aux = rng.standard_normal(G) + force
    M, logw = o.two_body_sample(aux, force)
    sq = SQRT_MINUS(dt)
    w = np.prod(np.exp(0.5 * force * force - aux * force - aux * sq * m.bg))
    assert abs(np.exp(logw) - w) < TOL * max(1.0, abs(w))
    Mx = sq * np.einsum("g,kjg->kj", aux, m.chol)
    assert np.abs(M - Mx).max() < TOL


def test_sdsd_log_overlap_and_green_match_formula():
    rng = np.random.default_rng(7)
    L, N = 10, 4
    left = _cplx(rng, (L, N))
    right = _cplx(rng, (L, N))
    lwL, lwR = 1.0 - 0.5j, 2.0 + 1.5j      # conj(lwL) + lwR = 3 + 2i
    lo, thetaT, gd, god, info = O.sdsd(left, lwL, right, lwR)
    assert info == 0
    S = left.conj().T @ right
    sign, logabs = np.linalg.slogdet(S)
    expect = logabs + np.log(sign) + np.conj(lwL) + lwR
    assert logov_close(np.array([lo]), np.array([expect]), TOL) < TOL
    Gm = _green(left, right)
    assert np.abs(thetaT - np.linalg.inv(S).T @ right.T).max() < TOL
    assert np.abs(gd - np.diag(Gm)).max() < TOL
    h = L // 2
    off = np.concatenate([[Gm[i, i + h] for i in range(h)], [Gm[i + h, i] for i in range(h)]])
    assert np.abs(god - off).max() < TOL


def test_molecule_propagators_after_background_update():
    m = inputs.molecule_inputs(12, 3, 3, 8, dt=0.05, decay=4.0)
    rng = np.random.default_rng(8)
    bg = rng.uniform(-1, 1, m.G)
    m.set_background(bg)
    dt = m.dt
    Kp = m.K + np.einsum("g,jig->ji", bg, m.chol)
    logw = 0.5 * dt * np.sum(bg * bg)
    assert abs(m.logwDt - logw) < TOL
    assert np.abs(m.logExpMinusDtK - (-dt * Kp)).max() < TOL
    assert np.abs(m.expMinusDtK - sl.expm(-dt * Kp)).max() < TOL
    assert np.abs(m.expMinusHalfDtK - sl.expm(-0.5 * dt * Kp)).max() < TOL
    assert np.abs(m.expHalfDtK - sl.expm(0.5 * dt * Kp)).max() < TOL
    assert abs(m.logwHalf - 0.5 * logw) < TOL


def test_hubbard_exp_minus_k_projects_onto_lowest_eigenvectors():
    rng = np.random.default_rng(9)
    L, N = 10, 5
    K = _cplx(rng, (2 * L, 2 * L))
    K = K + K.conj().T
    eK = inputs.exp_minus_alpha(K, 1.0)
    w = _cplx(rng, (2 * L, N))
    for _ in range(400):
        w, _, _ = O.qr(eK @ w)
    lam, V = np.linalg.eigh(K)
    assert np.abs(np.abs(w) - np.abs(V[:, :N])).max() < 1e-10
