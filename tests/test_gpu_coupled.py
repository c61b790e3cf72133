"""coupled2d on the GPU (equations/coupled2d/*) against the CPU oracle.

The device-prepared medium (squares, Gaussian smoothing, centered gradients
and Laplacians) and the FP32 run (seismograms and snapshots of P and S) equal
the FP32 oracle bit for bit; the FP64 oracle bounds the error (1e-5 relative L2).
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _model(nx=70, nz=54, seed=4):
    from fomo_b200.synthetic import layered_elastic

    vp, vs, _ = layered_elastic(nx, nz, n_layers=4, seed=seed)
    return vp, vs


@pytest.mark.parametrize("fd_order,sigma", [(2, 3.0), (4, 0.0), (6, 1.5), (8, 3.0), (10, 2.2)])
def test_coupled_medium_bitwise(fomo, oracle, fd_order, sigma):
    vp, vs = _model(41, 33)
    nbc = 7
    got = fomo.debug_coupled_medium(vp, vs, 10.0, nbc, fd_order, sigma)
    o = oracle.coupled2d(vp, vs, 10.0, 1e-3, 1, sx=[5], sz=[5], rx=[5], rz=[5],
                         wavelet=np.zeros((1, 1), np.float32), nbc=nbc, fd_order=fd_order,
                         smooth_sigma=sigma, medium=True)
    want = o["medium"]
    for k in range(8):
        assert np.array_equal(got[:, :, k], want[:, :, k]), k


@pytest.mark.parametrize("fd_order", [2, 4, 6, 8, 10])
def test_coupled2d_bitwise_vs_oracle(fomo, oracle, fd_order):
    vp, vs = _model()
    nt, nbc = 300, 12
    rx = np.arange(1, 71, 3)
    rz = np.full(rx.size, 9)
    w = fomo.ricker_wavelet(15.0, 1e-3, nt)
    kw = dict(sx=[35], sz=[20], rx=rx, rz=rz, nbc=nbc, fd_order=fd_order, snap_interval=75)
    r = fomo.coupled2d(vp, vs, 10.0, 1e-3, nt, 15.0, **kw)
    o = oracle.coupled2d(vp, vs, 10.0, 1e-3, nt, wavelet=w[None], **kw)
    assert np.array_equal(r.seis_P, o["seis_P"])
    assert np.array_equal(r.seis_S, o["seis_S"])
    assert len(r.snaps_P) == len(r.snaps_S) == 4
    for k in range(4):
        assert np.array_equal(r.snaps_P[k], o["snaps_P"][:, :, k])
        assert np.array_equal(r.snaps_S[k], o["snaps_S"][:, :, k])
    o64 = oracle.coupled2d(vp, vs, 10.0, 1e-3, nt, wavelet=w[None], prec=64, **kw)
    assert rel_l2(r.seis_P, o64["seis_P"]) < 1e-5
    assert rel_l2(r.seis_S, o64["seis_S"]) < 1e-5
    assert np.abs(r.seis_S).max() > 0
    # two 150-step replayed chunks: 2 launches a step, 2 snapshot kernels per
    # frame and the step-index advance
    assert fomo.api.last_stats.gpu_launches == 2 * (2 * 150 + 2 * 2 + 1)


def test_coupled2d_keywords(fomo, oracle):
    """v_ref_p, v_ref_s, smooth_sigma and a custom wavelet reach the kernels."""
    vp, vs = _model(50, 40, seed=9)
    nt = 200
    w = (fomo.ricker_wavelet(12.0, 1e-3, nt) * 2.0).astype(np.float32)
    # two coincident sources (added in source order) and receivers on a source cell
    rx = np.concatenate([np.arange(1, 51, 2), [25, 25]])
    rz = np.concatenate([np.full(25, 6), [10, 10]])
    kw = dict(sx=[25, 30, 25], sz=[10, 12, 10], rx=rx, rz=rz, nbc=10, fd_order=6)
    r = fomo.coupled2d(vp, vs, 10.0, 1e-3, nt, 12.0, v_ref_p=2000.0, v_ref_s=900.0,
                       smooth_sigma=1.0, wavelet=w, **kw)
    o = oracle.coupled2d(vp, vs, 10.0, 1e-3, nt, wavelet=np.repeat(w[None], 3, axis=0),
                         v_ref_p=2000.0, v_ref_s=900.0, smooth_sigma=1.0, **kw)
    assert np.array_equal(r.seis_P, o["seis_P"])
    assert np.array_equal(r.seis_S, o["seis_S"])


def test_homogeneous_s_stays_zero(fomo):
    n = 60
    vp = np.full((n, n), 2500.0, np.float32)
    vs = np.full((n, n), 1500.0, np.float32)
    r = fomo.coupled2d(vp, vs, 10.0, 1e-3, 150, 15.0, sx=[30], sz=[30], rx=[10, 20, 40],
                       rz=[30, 30, 30], nbc=10, fd_order=8)
    assert np.abs(r.seis_P).max() > 0
    assert not np.any(r.seis_S)


def test_coupled2d_chunks_equal_step_launches(fomo, monkeypatch):
    """Snapshots every 40 steps, 290 steps: three replayed 80-step chunks and a
    50-step remainder launched step by step (FOMO_F_STEP_LAUNCH: all steps)."""
    from fomo_b200 import _lib as L

    vp, vs = _model(60, 44, seed=2)
    kw = dict(sx=[30], sz=[12], rx=np.arange(1, 61, 3), rz=np.full(20, 8), nbc=10, fd_order=8,
              snap_interval=40)
    a = fomo.coupled2d(vp, vs, 10.0, 1e-3, 290, 15.0, **kw)
    orig = fomo.api._opts

    def opts(*oa, **okw):
        o = orig(*oa, **okw)
        o.flags |= L.FOMO_F_STEP_LAUNCH
        return o

    monkeypatch.setattr(fomo.api, "_opts", opts)
    b = fomo.coupled2d(vp, vs, 10.0, 1e-3, 290, 15.0, **kw)
    assert fomo.api.last_stats.gpu_launches == 2 * 290
    assert np.array_equal(a.seis_P, b.seis_P)
    assert np.array_equal(a.seis_S, b.seis_S)
    assert len(a.snaps_P) == 7
    for x, y in zip(a.snaps_P + a.snaps_S, b.snaps_P + b.snaps_S):
        assert np.array_equal(x, y)
