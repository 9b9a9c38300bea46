"""Adjoint of the mixed local energy and of the mean log-overlap
(afqmc_pl_adjoint) on the phaseless shapes of the adjoint configuration
(n=64, 16+16 electrons): the energy and the one-body derivative against the
oracle (the den-weighted mixed Green's function of the reference's
SD2sSD2isOperation), every derivative against central finite differences
(step 1e-6, FP64) along random directions; a small population after 3 steps,
and the configuration's own size (L=320 Cholesky vectors, 512 walkers after
200 steps).

Tolerances: 1e-10 relative against the oracle; 1e-6 relative against the
finite differences."""
import numpy as np
import pytest
import torch

from afqmclab_b200 import adjoint, capi, inputs
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FD_STEP = 1e-6
FD_TOL = 1e-6


@pytest.fixture(scope="module")
def setup():
    m = inputs.molecule_inputs(64, 16, 16, 64, dt=0.005, decay=20.0, seed=11)
    m.ET = -20.0
    W = 48
    eng = capi.pl_engine(m, W, 3, 1000, 1000)
    eng.set_walkers(*inputs.initial_walkers(m.phiTUp, W, seed=5, noise=0.03))
    eng.step(3)
    walkers = eng.get_walkers()
    eng.close()
    return m, walkers, adjoint.AdjointContext(m, walkers)


def test_energy_and_density_matrix_match_oracle(setup):
    m, walkers, actx = setup
    out = actx.evaluate(m.t, m.chol, m.phiTUp, m.phiTDn)
    # oracle: mixed estimator with an identity half step = local energy at the walkers
    ident = np.eye(m.n, dtype=np.complex128)
    mo = inputs.MoleculeInputs(**{k: getattr(m, k) for k in ("n", "nup", "ndn", "G", "dt", "t", "K",
                                                             "chol", "bg", "phiTUp", "phiTDn",
                                                             "logwT")})
    mo.set_background(m.bg)
    mo.expHalfDtK = np.asfortranarray(ident)
    mo.logwHalf = 0.0
    o = O.pl_engine(mo, walkers[0].shape[2], 1)
    o.set_walkers(*walkers)
    el, den = o.add_mixed_measurement()
    meas = o.measurement()
    E_o = meas[1] / meas[0]
    assert abs(out["E"] - E_o) < 1e-10 * abs(E_o)
    # d E / d t = den-weighted mixed one-body density matrix sum_s G_s
    rdm = np.zeros((m.n, m.n), np.complex128)
    al = walkers[2].astype(bool)
    for w in np.nonzero(al)[0]:
        rdm += den[w] * (o.green(int(w), 0) + o.green(int(w), 1))
    rdm /= den[al].sum()
    assert np.abs(out["dE_dt"] - rdm).max() < 1e-10 * np.abs(rdm).max()


def _fd(actx, base, which, direction):
    args = [a.copy() for a in base]
    plus = [a.copy() for a in base]
    minus = [a.copy() for a in base]
    plus[which] = plus[which] + FD_STEP * direction
    minus[which] = minus[which] - FD_STEP * direction
    ep = actx.evaluate(*plus, want_chol=False)
    em = actx.evaluate(*minus, want_chol=False)
    del args
    return (ep["E"] - em["E"]) / (2 * FD_STEP), (ep["mean_logov"] - em["mean_logov"]) / (2 * FD_STEP)


def test_adjoint_matches_central_differences(setup):
    m, walkers, actx = setup
    base = [m.t.copy(), m.chol.copy(), m.phiTUp.copy(), m.phiTDn.copy()]
    out = actx.evaluate(*base)
    rng = np.random.default_rng(99)
    # one-body matrix t
    d = rng.standard_normal(m.t.shape)
    fd, _ = _fd(actx, base, 0, d)
    an = np.sum(out["dE_dt"] * d)
    assert abs(fd - an) <= FD_TOL * abs(an)
    # Cholesky vectors
    d = rng.standard_normal(m.chol.shape)
    fd, _ = _fd(actx, base, 1, d)
    an = np.sum(out["dE_dchol"] * d)
    assert abs(fd - an) <= FD_TOL * abs(an)
    # trial orbitals (E and log-overlap depend on conj(phiT): dE = sum dE/dconj * conj(delta))
    for s in (0, 1):
        d = rng.standard_normal(base[2 + s].shape) + 1j * rng.standard_normal(base[2 + s].shape)
        fdE, fdL = _fd(actx, base, 2 + s, d)
        anE = np.sum(out["dE_dconj_phiT"][s] * np.conj(d))
        anL = np.sum(out["dlogov_dconj_phiT"][s] * np.conj(d))
        assert abs(fdE - anE) <= FD_TOL * abs(anE)
        assert abs(fdL - anL) <= FD_TOL * abs(anL)


def test_autograd_wrapper_backward(setup):
    m, walkers, actx = setup
    t = torch.tensor(m.t, requires_grad=True)
    c = torch.tensor(m.chol, requires_grad=True)
    pu = torch.tensor(m.phiTUp, requires_grad=True)
    pd = torch.tensor(m.phiTDn, requires_grad=True)
    E = adjoint.MixedEnergy.apply(t, c, pu, pd, actx)
    E.backward()
    rng = np.random.default_rng(5)
    d = rng.standard_normal(m.t.shape)
    fd, _ = _fd(actx, [m.t, m.chol, m.phiTUp, m.phiTDn], 0, d)
    assert abs(np.real(fd) - float((t.grad.numpy() * d).sum())) <= FD_TOL * abs(np.real(fd))
    dz = rng.standard_normal(m.phiTUp.shape)  # real direction: d Re E = Re(<grad, dz>)
    fdz, _ = _fd(actx, [m.t, m.chol, m.phiTUp, m.phiTDn], 2, dz)
    got = float(np.real(np.sum(np.conj(pu.grad.numpy()) * dz)))
    assert abs(np.real(fdz) - got) <= FD_TOL * abs(np.real(fdz))



def _compare_forms(actx_real, actx_phase, m, phase):
    """The GEMM form (real trial) against the per-walker form (the same trial
    times a global phase c, which makes the half-rotated vectors complex): E,
    dE/dt and dE/dL_g are invariant under the phase and the orbital gradient
    rotates by c (dE/dconj(c phiT) = c dE/dconj(phiT))."""
    base = [m.t.copy(), m.chol.copy(), m.phiTUp.copy(), m.phiTDn.copy()]
    a = actx_real.evaluate(*base)
    b = actx_phase.evaluate(base[0], base[1], phase * base[2], phase * base[3])
    assert abs(a["E"] - b["E"]) < 1e-10 * abs(a["E"])
    for key in ("dE_dt", "dE_dchol"):
        assert np.abs(a[key] - b[key]).max() < 1e-9 * np.abs(a[key]).max(), key
    for s in (0, 1):
        ga, gb = phase * a["dE_dconj_phiT"][s], b["dE_dconj_phiT"][s]
        assert np.abs(ga - gb).max() < 1e-9 * np.abs(ga).max(), s
        la, lb = phase * a["dlogov_dconj_phiT"][s], b["dlogov_dconj_phiT"][s]
        assert np.abs(la - lb).max() < 1e-9 * np.abs(la).max(), s


def test_gemm_and_per_walker_forms_agree(setup):
    """Every evaluation form on the same walkers: a restricted trial (block 0
    counted twice) and an unrestricted real trial (each block its own
    operands), each against the per-walker form."""
    m, walkers, actx = setup
    phase = np.exp(0.3j)
    _compare_forms(actx, actx, m, phase)
    rng = np.random.default_rng(7)
    m3 = inputs.molecule_inputs(64, 16, 16, 64, dt=0.005, decay=20.0, seed=11)
    m3.ET = -20.0
    q, _ = np.linalg.qr(m3.phiTDn.real + 0.1 * rng.standard_normal(m3.phiTDn.shape))
    m3.phiTDn = np.asfortranarray(q.astype(np.complex128))
    assert not np.allclose(m3.phiTDn, m3.phiTUp)
    actx3 = adjoint.AdjointContext(m3, walkers)
    _compare_forms(actx3, actx3, m3, phase)


def test_chol_gradient_into_device_memory(setup):
    """dE/dL_g written straight into a CUDA tensor equals the host copy."""
    m, walkers, actx = setup
    eng = capi.pl_engine(m, walkers[0].shape[2], 1, precision=capi.AFQMC_FP64)
    try:
        eng.set_walkers(*walkers)
        host = eng.adjoint()
        dev = torch.zeros(m.n * m.n * m.G, dtype=torch.complex128, device="cuda")
        out = eng.adjoint(chol_out=dev)
        got = dev.cpu().numpy().reshape((m.n, m.n, m.G), order="F")
        assert np.array_equal(got, host["dE_dchol"])
        assert out["E"] == host["E"]
        with pytest.raises(capi.AfqmcError):
            eng.adjoint(chol_out=torch.zeros(3, dtype=torch.complex128, device="cuda"))
    finally:
        eng.close()


def _fd_richardson(actx, base, which, direction, h=1e-4):
    """Central differences at h and h/2 combined as (4 D(h/2) - D(h)) / 3:
    truncation O(h^4), rounding about eps |f| / h."""
    def central(step):
        plus = [a.copy() for a in base]
        minus = [a.copy() for a in base]
        plus[which] = plus[which] + step * direction
        minus[which] = minus[which] - step * direction
        ep = actx.evaluate(*plus, want_chol=False)
        em = actx.evaluate(*minus, want_chol=False)
        return np.array([(ep["E"] - em["E"]) / (2 * step), (ep["mean_logov"] - em["mean_logov"]) / (2 * step)])

    d1, d2 = central(h), central(h / 2)
    return (4 * d2 - d1) / 3


def test_adjoint_at_the_configuration_size():
    """The adjoint configuration as stated: n=64, 16+16 electrons, 320
    Cholesky vectors, 512 walkers after 200 steps (Gram-Schmidt and
    population control every 10): energy and density matrix against the
    oracle (1e-10), every derivative class against Richardson-extrapolated
    central differences (1e-6).  After 200 steps the weights have spread and
    the estimator's curvature along a random direction makes a plain central
    difference at step 1e-6 err by about 1e-6 relative; the extrapolation
    removes that truncation error."""
    m = inputs.molecule_inputs(64, 16, 16, 320, dt=0.005, decay=60.0, seed=13)
    m.ET = -20.0
    W = 512
    eng = capi.pl_engine(m, W, 17, 10, 10)
    eng.set_walkers(*inputs.initial_walkers(m.phiTUp, W, seed=19, noise=0.03))
    eng.step(200)
    assert eng.status() == 0
    walkers = eng.get_walkers()
    eng.close()
    actx = adjoint.AdjointContext(m, walkers)
    test_energy_and_density_matrix_match_oracle((m, walkers, actx))

    base = [m.t.copy(), m.chol.copy(), m.phiTUp.copy(), m.phiTDn.copy()]
    out = actx.evaluate(*base)
    rng = np.random.default_rng(101)
    d = rng.standard_normal(m.t.shape)
    fdE, _ = _fd_richardson(actx, base, 0, d)
    an = np.sum(out["dE_dt"] * d)
    assert abs(fdE - an) <= FD_TOL * abs(an)
    d = rng.standard_normal(m.chol.shape)
    fdE, _ = _fd_richardson(actx, base, 1, d)
    an = np.sum(out["dE_dchol"] * d)
    assert abs(fdE - an) <= FD_TOL * abs(an)
    for s in (0, 1):
        d = rng.standard_normal(base[2 + s].shape) + 1j * rng.standard_normal(base[2 + s].shape)
        fdE, fdL = _fd_richardson(actx, base, 2 + s, d)
        anE = np.sum(out["dE_dconj_phiT"][s] * np.conj(d))
        anL = np.sum(out["dlogov_dconj_phiT"][s] * np.conj(d))
        assert abs(fdE - anE) <= FD_TOL * abs(anE), (s, fdE, anE)
        assert abs(fdL - anL) <= FD_TOL * abs(anL), (s, fdL, anL)
