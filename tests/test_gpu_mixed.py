"""Mixed-precision form (tcgen05 bf16 contractions, FP64 LU / log-det /
weights / re-orthonormalisation) against the plain FP64 form of the engine on
the same walkers and random stream.

Tolerances: after one step from identical walkers the log-overlaps agree to
2e-2 (bf16 operands, fp32 accumulation); the mixed estimator's energy agrees
to 2e-3 relative; population-control bookkeeping (alive flags, random-stream
counter) is identical."""
import numpy as np
import pytest

from afqmclab_b200 import capi, inputs

pytestmark = pytest.mark.gpu


def molecule(n=64, nup=16, ndn=16, G=128):
    m = inputs.molecule_inputs(n, nup, ndn, G, dt=0.005, decay=30.0, seed=7)
    m.ET = -5.0
    return m


def pair(m, W, seed, mgs=1000, pop=1000, noise=0.02):
    f = capi.pl_engine(m, W, seed, mgs, pop, precision=capi.AFQMC_FP64)
    x = capi.pl_engine(m, W, seed, mgs, pop, precision=capi.AFQMC_MIXED)
    wf, lw, al = inputs.initial_walkers(m.phiTUp, W, seed=seed + 1, noise=noise)
    f.set_walkers(wf, lw, al)
    x.set_walkers(wf, lw, al)
    return f, x


@pytest.mark.parametrize("n,nup,ndn,G", [(64, 16, 16, 128), (128, 32, 32, 256), (64, 16, 8, 64)])
def test_mixed_single_step_matches_fp64(n, nup, ndn, G):
    m = molecule(n, nup, ndn, G)
    W = 48
    f, x = pair(m, W, 11)
    assert np.abs(f.log_overlaps() - x.log_overlaps()).max() < 1e-5
    f.step(1)
    x.step(1)
    _, _, af = f.get_walkers()
    _, _, ax = x.get_walkers()
    assert (af == ax).all()
    assert f.rng_counter() == x.rng_counter()
    lf, lx = f.log_overlaps(), x.log_overlaps()
    a = af.astype(bool)
    assert np.abs(lf[a].real - lx[a].real).max() < 2e-2
    assert np.abs(np.exp(1j * lf[a].imag) - np.exp(1j * lx[a].imag)).max() < 2e-2
    assert x.status() == 0


def test_mixed_energy_tracks_fp64():
    m = molecule()
    W = 64
    f, x = pair(m, W, 21, mgs=5, pop=10)
    for e in (f, x):
        e.modify_gm()
        e.pop_control()
    ef, ex = [], []
    for step in range(20):
        for e, acc in ((f, ef), (x, ex)):
            if step % 5 == 0:
                e.reset_measurement()
                e.add_mixed_measurement()
                mm = e.measurement()
                acc.append((mm[1] / mm[0]).real)
            e.step(1)
    ef, ex = np.array(ef), np.array(ex)
    assert np.all(np.abs(ef - ex) < 2e-3 * np.abs(ef)), (ef, ex)
    # the mixed series stops at the FP64 rule's tolerance or where a term
    # falls below fp32 resolution of the walker, whichever comes first: never
    # later than the FP64 form, never before the minimum order 4
    cf, cx = f.taylor_stats(), x.taylor_stats()
    assert cx[1] / cx[0] <= cf[1] / cf[0] + 0.5
    assert cx[2] >= 4
    assert x.status() == 0


@pytest.mark.parametrize("n,nup,ndn,G", [(64, 16, 16, 128), (128, 32, 32, 128), (64, 16, 8, 64)])
def test_mixed_measurement_matches_fp64_on_same_walkers(n, nup, ndn, G):
    m = molecule(n, nup, ndn, G)
    W = 32
    f, x = pair(m, W, 31, noise=0.05)
    for e in (f, x):
        e.reset_measurement()
        e.add_mixed_measurement()
    mf, mx = f.measurement(), x.measurement()
    assert abs(mf[0] - mx[0]) < 1e-4 * abs(mf[0])
    assert abs(mf[1] / mf[0] - mx[1] / mx[0]) < 2e-3 * abs(mf[1] / mf[0])
    bf, exf = f.cholesky_nums()
    bx, exx = x.cholesky_nums()
    assert np.abs(bf - bx).max() < 2e-2 * np.abs(bf).max()
    assert np.abs(exf - exx).max() < 2e-2 * np.abs(exf).max()


def test_mixed_rejects_unsupported_shapes():
    m = inputs.molecule_inputs(16, 4, 3, 24, dt=0.01, decay=6.0)
    with pytest.raises(capi.AfqmcError):
        capi.pl_engine(m, 8, 1, precision=capi.AFQMC_MIXED)


@pytest.mark.parametrize("n,nup,ndn,G", [(64, 16, 16, 64), (128, 32, 32, 64), (64, 16, 8, 64)])
def test_mixed_stabilisation_matches_fp64(n, nup, ndn, G):
    """The mixed form's FP64 Cholesky QR of the fp32 walkers gives the same
    orthonormal columns (R with positive real diagonal, so the same gauge)
    and log-weight shift as the FP64 form's Gram-Schmidt, to fp32 accuracy."""
    m = molecule(n, nup, ndn, G)
    W = 40
    f, x = pair(m, W, 31, noise=0.2)
    f.modify_gm()
    x.modify_gm()
    wf_f, lw_f, _ = f.get_walkers()
    wf_x, lw_x, _ = x.get_walkers()
    assert np.abs(lw_x - lw_f).max() < 1e-5
    assert np.abs(wf_x - wf_f).max() < 1e-5
    q = wf_x[:, :, 0]
    assert np.abs(q.conj().T @ q - np.eye(q.shape[1])).max() < 1e-5
    assert x.status() == 0


def test_mixed_restricted_matches_two_block_form():
    """With the same trial for both spins (nup = ndn) the mixed form computes
    one spin block and doubles it; a trial whose down block differs from the
    up block in one last bit takes the two-block path.  Both agree on the
    log-overlaps, the energy and the per-vector sums to mixed-precision
    accuracy after a few steps with a measurement."""
    m = molecule(128, 32, 32, 128)
    assert np.array_equal(m.phiTUp, m.phiTDn)
    m2 = molecule(128, 32, 32, 128)
    d = m2.phiTDn.copy()
    d[0, 0] = np.nextafter(d[0, 0].real, np.inf) + 1j * d[0, 0].imag
    m2.phiTDn = np.asfortranarray(d)
    W = 64
    out = []
    for mm in (m, m2):
        x = capi.pl_engine(mm, W, 41, 1000, 1000, precision=capi.AFQMC_MIXED)
        wf, lw, al = inputs.initial_walkers(mm.phiTUp, W, seed=42, noise=0.05)
        x.set_walkers(wf, lw, al)
        x.step(3)
        x.reset_measurement()
        x.add_mixed_measurement()
        mm_ = x.measurement()
        out.append((x.log_overlaps(), mm_[1] / mm_[0], x.cholesky_nums(), x.status()))
    (l1, e1, (b1, x1), s1), (l2, e2, (b2, x2), s2) = out
    assert s1 == 0 and s2 == 0
    assert np.abs(l1 - l2).max() < 1e-4
    assert abs(e1 - e2) < 2e-6 * abs(e1)
    assert np.abs(b1 - b2).max() < 1e-4 * np.abs(b1).max()
    assert np.abs(x1 - x2).max() < 1e-4 * np.abs(x1).max()
