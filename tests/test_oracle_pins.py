"""The CPU oracle against the reference's own known-answer tests (CPU only)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import cm, golden

K = golden()


def test_sd_normalize_kat():
    g = K["sd_normalize"]
    _, lw, ratio = O.sd_normalize(cm(g["wf"], g["shape"]))
    assert abs(lw - g["logw"]) < 1e-12
    assert ratio == pytest.approx(g["ratio"], rel=1e-13)


def test_sd2is_normalize_kat():
    g = K["sd2is_normalize"]
    _, lw, ratio = O.sd2is_normalize(cm(g["wf"], g["shape"]), g["nup"], g["ndn"])
    assert abs(lw - g["logw"]) < 1e-12
    assert ratio == pytest.approx(g["ratio"], rel=1e-13)


def test_sd2s_normalize_kat():
    g = K["sd2s_normalize"]
    _, _, lw, ratio = O.sd2s_normalize(cm(g["wf_up"], g["shape_up"]), cm(g["wf_dn"], g["shape_dn"]))
    assert abs(lw - g["logw"]) < 1e-12
    assert ratio == pytest.approx(g["ratio"], rel=1e-13)


def test_qr_is_orthonormal_and_reconstructs():
    rng = np.random.default_rng(3)
    A = rng.standard_normal((12, 5)) + 1j * rng.standard_normal((12, 5))
    Q, det, dl = O.qr(A)
    assert np.allclose(Q.conj().T @ Q, np.eye(5), atol=1e-13)
    assert det > 0 and abs(np.prod(dl) - det) < 1e-10 * det
    R = Q.conj().T @ A
    assert np.allclose(np.tril(R, -1), 0, atol=1e-12)
    assert np.allclose(np.abs(np.diag(R)), np.abs(dl), rtol=1e-12)


@pytest.mark.parametrize("trans,key", [("N", "right"), ("C", "left")])
def test_loghop_fixed_order_kat(trans, key):
    g = K["loghop_taylor"]
    M = g["M_scale"] * cm(g["M"], (3, 3))
    wf = cm(g["wf"], (3, 2))
    out, k = O.loghop_apply(M, wf, "fixedOrder", g["fixed_order"], 1e-8, trans=trans)
    assert k == g["fixed_order"]
    assert np.abs(out - cm(g[key], (3, 2))).max() < g["fixed_tol"]


@pytest.mark.parametrize("trans,key", [("N", "right"), ("C", "left")])
def test_loghop_dynamic_order_kat(trans, key):
    g = K["loghop_taylor"]
    M = g["M_scale"] * cm(g["M"], (3, 3))
    wf = cm(g["wf"], (3, 2))
    out, k = O.loghop_apply(M, wf, "dynamicOrder", 0, g["auto_accuracy"], trans=trans)
    assert k == g["auto_order"]
    assert np.abs(out - cm(g[key], (3, 2))).max() < g["auto_tol"]


def test_loghop_matches_expm():
    from scipy.linalg import expm
    rng = np.random.default_rng(5)
    M = 0.05 * (rng.standard_normal((10, 10)) + 1j * rng.standard_normal((10, 10)))
    wf = rng.standard_normal((10, 3)) + 1j * rng.standard_normal((10, 3))
    out, k = O.loghop_apply(M, wf)
    assert k >= 4
    assert np.abs(out - expm(M) @ wf).max() < 1e-9


def test_pop_fill_pin_from_golden_table():
    """populationControlTest.cpp:29-45: the copy counts implied by the golden
    table, refilled by the slot-filling algorithm, give back that table."""
    g = K["pop_configuration"]
    table = np.array(g["table_one_based"]) - 1
    counts = np.bincount(table, minlength=g["L"])
    t, bad = O.pop_fill_from_counts(counts, size=g["size"])
    assert bad == 0
    assert (t == table).all()


def test_pop_comb_counts_are_stratified():
    rng = np.random.default_rng(9)
    w = rng.uniform(0, 5, 200)
    w[::17] = 0.0
    u = rng.uniform(size=200)
    table, bad = O.pop_configuration(w, u)
    assert bad == 0
    counts = np.bincount(table, minlength=200)
    assert (counts[w == 0] == 0).all()
    expect = w / w.sum() * 200
    assert np.all(np.abs(np.cumsum(counts) - np.cumsum(expect)) <= 1.0 + 1e-9)


@pytest.mark.parametrize("case", range(2))
def test_pop_check_kat(case):
    g = K["pop_check"][case]
    mn, mx, avg = O.pop_check(g["weights"])
    assert (mn, mx) == (g["min"], g["max"])
    assert avg == pytest.approx(g["avg"], rel=1e-15)


def test_rng_uniform_restatement():
    """The oracle's stream equals a pure-Python SplitMix64 restatement."""
    M = (1 << 64) - 1

    def mix(z):
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        return z ^ (z >> 31)

    seed = 985456376
    for k in [0, 1, 2, 1000, 2**40 + 7]:
        b = mix((mix(seed) + (k + 1) * 0x9E3779B97F4A7C15) & M)
        assert O.rng_uniform(seed, k, 1)[0] == (b >> 11) * 2.0**-53


def test_niupnidn_consts_match_closed_form():
    """gamma solves cosh(gamma)=exp(dtU/2) (densitySpin); constDiag = exp of the
    2x2 one-body block (exp2by2Matrix) -- checked with scipy's expm."""
    from scipy.linalg import expm
    rng = np.random.default_rng(1)
    L, dt = 6, 0.01
    U, mu, hx, hy, hz = (rng.uniform(1, 4, L), rng.uniform(-1, 1, L), rng.uniform(-1, 1, L),
                         rng.uniform(-1, 1, L), rng.uniform(-1, 1, L))
    gam, c00, c01, c10, c11, s = O.niupnidn_consts(dt, "densitySpin", U, mu, hx, hy, hz)
    assert np.allclose(np.cosh(gam), np.exp(dt * U / 2), rtol=1e-12)
    assert s == pytest.approx(dt * U.sum())
    for i in range(L):
        a = -dt * (U[i] / 2 - mu[i] + hz[i] / 2)
        b = -dt * (U[i] / 2 - mu[i] - hz[i] / 2)
        c = -dt * 0.5 * (hx[i] + 1j * hy[i])
        E = expm(np.array([[a, np.conj(c)], [c, b]]))
        assert np.allclose([[c00[i], c01[i]], [c10[i], c11[i]]], E, atol=1e-14)


def test_hubbard_u0_energy_kat():
    """HubbardSOCMeasureFixedSDSDTest.cpp:11-63: with U=0 and the trial equal to
    the lowest N eigenvectors of K, the mixed energy is the sum of the lowest N
    eigenvalues."""
    from afqmclab_b200 import inputs
    m = inputs.hubbard_inputs(3, 2, 2, 1, U=0.0, trial="free")
    lam, V = np.linalg.eigh(m.K)
    m.phiT = np.asfortranarray(V[:, :m.N].astype(np.complex128))
    W = 3
    e = O.cp_engine(m, W, seed=1)
    wf, lw, al = inputs.initial_walkers(m.phiT, W)
    e.set_walkers(wf, lw, al)
    e.add_mixed_measurement()
    meas = e.measurement()
    assert abs(meas[1] / meas[0] - lam[:m.N].sum()) < 1e-12


def test_oracle_cp_step_runs_and_counts_draws():
    from afqmclab_b200 import inputs
    m = inputs.hubbard_inputs(4, 4, 7, 7, trial="free")
    W = 8
    e = O.cp_engine(m, W, seed=11, mgs_step=2, pop_step=3)
    wf, lw, al = inputs.initial_walkers(m.phiT, W, seed=2, noise=0.05)
    e.set_walkers(wf, lw, al)
    e.step(1)
    _, _, alive = e.get_walkers()
    assert e.rng_counter() == alive.sum() * m.L
    e.step(2)
    lo = e.log_overlaps()
    assert np.isfinite(lo).all()
