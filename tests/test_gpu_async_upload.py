"""Pipelined population upload: afqmc_set_walkers_async installs the same
population as afqmc_set_walkers, and uploading step i+1's walkers while step
i is still running on the engine's stream gives the results of the serial
sequence, bit for bit (FP64 and mixed-precision forms)."""
import numpy as np
import pytest
import torch

from afqmclab_b200 import capi, inputs

pytestmark = pytest.mark.gpu

W = 64


def _engine(precision):
    m = inputs.molecule_inputs(n=64, nup=16, ndn=16, G=128, dt=0.005)
    e = capi.pl_engine(m, W, 11, mgs_step=3, pop_step=4, precision=precision)
    return e, m


def _pinned_population(m, seed):
    wf, lw, al = inputs.initial_walkers(m.phiTUp, W, seed=seed, noise=0.03)
    h_wf = torch.from_numpy(np.ascontiguousarray(wf.reshape(-1, order="F").view(np.float64))).pin_memory()
    h_lw = torch.from_numpy(np.ascontiguousarray(lw.view(np.float64))).pin_memory()
    h_al = torch.from_numpy(np.ascontiguousarray(al)).pin_memory()
    return (wf, lw, al), (h_wf, h_lw, h_al)


@pytest.mark.parametrize("precision", [capi.AFQMC_FP64, capi.AFQMC_MIXED])
def test_async_upload_matches_serial(precision):
    pops = [_pinned_population(_engine(capi.AFQMC_FP64)[1], seed) for seed in (3, 4, 5)]

    # serial: set, step, measure, read back
    ref = []
    e, _ = _engine(precision)
    for (wf, lw, al), _h in pops:
        e.set_walkers(wf, lw, al)
        e.reset_measurement()
        e.add_mixed_measurement()
        e.step(2)
        ref.append((e.measurement(), e.get_walkers()))
    e.close()

    # pipelined: upload k+1 is enqueued while step k runs
    got = []
    e, _ = _engine(precision)
    h = pops[0][1]
    e.set_walkers_async(h[0].data_ptr(), h[1].data_ptr(), h[2].data_ptr())
    for k in range(len(pops)):
        e.reset_measurement()
        e.add_mixed_measurement()
        e.step(2)
        meas = e.measurement()
        walkers = e.get_walkers()
        got.append((meas, walkers))
        if k + 1 < len(pops):
            h = pops[k + 1][1]
            e.set_walkers_async(h[0].data_ptr(), h[1].data_ptr(), h[2].data_ptr())
    e.upload_wait()
    e.close()

    for (m_ref, w_ref), (m_got, w_got) in zip(ref, got):
        assert np.array_equal(m_ref, m_got)
        for a, b in zip(w_ref, w_got):
            assert np.array_equal(a, b)


def test_async_upload_overlaps_running_step():
    """The copy is enqueued behind a running step and installed after it."""
    e, m = _engine(capi.AFQMC_MIXED)
    (wf, lw, al), h = _pinned_population(m, 9)
    e.set_walkers(wf, lw, al)
    e.step(3)                      # enqueued, not waited for
    e.set_walkers_async(h[0].data_ptr(), h[1].data_ptr(), h[2].data_ptr())
    got = e.get_walkers()
    e.close()
    assert np.array_equal(got[1], lw)
    assert np.array_equal(got[2], al)
    # the mixed form keeps fp32 walkers: the round trip is exact to fp32
    np.testing.assert_allclose(got[0], wf, rtol=0, atol=1e-6)


def _fp32_planes(wf):
    """The phaseless mixed form's walker layout: per walker the real parts of
    the n x ncol matrix (column-major), then the imaginary parts, as fp32."""
    n, ncol, nw = wf.shape
    out = np.empty((nw, 2, n * ncol), np.float32)
    for w in range(nw):
        flat = wf[:, :, w].reshape(-1, order="F")
        out[w, 0] = flat.real.astype(np.float32)
        out[w, 1] = flat.imag.astype(np.float32)
    return out.reshape(-1)


def test_fp32_upload_installs_the_same_population():
    """afqmc_set_walkers_f32_async with the walkers in the mixed form's fp32
    layout installs bit for bit what afqmc_set_walkers installs from complex
    doubles (the same fp32 rounding), and the steps that follow agree exactly;
    the FP64 form rejects it."""
    pops = [_pinned_population(_engine(capi.AFQMC_FP64)[1], seed) for seed in (6, 7)]
    ref = []
    e, _ = _engine(capi.AFQMC_MIXED)
    for (wf, lw, al), _h in pops:
        e.set_walkers(wf, lw, al)
        e.step(2)
        ref.append((e.get_walkers(), e.log_overlaps()))
    e.close()

    got = []
    e, _ = _engine(capi.AFQMC_MIXED)
    for (wf, lw, al), h in pops:
        h32 = torch.from_numpy(_fp32_planes(wf)).pin_memory()
        e.set_walkers_f32_async(h32.data_ptr(), h[1].data_ptr(), h[2].data_ptr())
        e.step(2)
        got.append((e.get_walkers(), e.log_overlaps()))
        e.upload_wait()
    e.close()
    for (w_ref, lo_ref), (w_got, lo_got) in zip(ref, got):
        for a, b in zip(w_ref, w_got):
            assert np.array_equal(a, b)
        assert np.array_equal(lo_ref, lo_got)

    f, m = _engine(capi.AFQMC_FP64)
    (wf, lw, al), h = pops[0]
    h32 = torch.from_numpy(_fp32_planes(wf)).pin_memory()
    with pytest.raises(capi.AfqmcError):
        f.set_walkers_f32_async(h32.data_ptr(), h[1].data_ptr(), h[2].data_ptr())
    f.close()
