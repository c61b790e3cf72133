"""Uneven-size batch: every shot of fomo_acoustic2d_uneven equals the oracle's
single-shot acoustic2d (and libfomo_b200's own acoustic2d) bit for bit, for
every tile shape and strip width the autotuner can pick, in both kernel forms
(the fused single sweep and the velocity / pressure kernels)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TILES = ["32,8", "64,4", "128,2", "16,16", "32,4"]


def _shots(seed=0):
    from fomo_b200.synthetic import grf2d

    sizes = [(37, 29), (61, 44), (23, 52), (90, 31), (48, 48)]
    vps, rhos, sx, sz, rx, rz = [], [], [], [], [], []
    for s, (nx, nz) in enumerate(sizes):
        vp = grf2d(nx, nz, 10.0, 3000.0, 500.0, 60.0, seed + s, 2000.0, 4000.0)
        rho = np.full((nx, nz), 2000.0 + 50 * s, np.float32, order="F")
        if s == 1:  # vacuum free surface on one shot
            vp[:, 0] = 0.0
            rho[:, 0] = 0.0
        vps.append(vp)
        rhos.append(rho)
        sx.append([nx // 2, 3] if s == 2 else nx // 2)
        sz.append([5, nz - 2] if s == 2 else 5)
        r = np.arange(1, nx + 1, 3)
        rx.append(r)
        rz.append(np.full(r.size, 4))
    return vps, rhos, sx, sz, rx, rz


@pytest.mark.parametrize("tile", TILES)
def test_uneven_equals_single_shots(fomo, oracle, monkeypatch, tile):
    monkeypatch.setenv("FOMO_UNEVEN_TILE", tile)
    vps, rhos, sx, sz, rx, rz = _shots()
    nt, nbc, dt = 120, 7, 1e-3
    r = fomo.acoustic2d_uneven(vps, rhos, 10.0, dt, nt, 20.0, sx=sx, sz=sz, rx=rx, rz=rz,
                               nbc=nbc, fd_order=8)
    assert r.stats.tile == tuple(int(v) for v in tile.split(","))
    w = fomo.ricker_wavelet(20.0, dt, nt)
    for s in range(len(vps)):
        sxs, szs = np.atleast_1d(sx[s]), np.atleast_1d(sz[s])
        o = oracle.acoustic2d(vps[s], rhos[s], 10.0, dt, nt, sx=sxs, sz=szs, rx=rx[s], rz=rz[s],
                              wavelet=np.repeat(w[None, :], sxs.size, axis=0), nbc=nbc,
                              fd_order=8)
        for k, name in enumerate(("seis_p", "seis_vx", "seis_vz")):
            assert np.array_equal(r.shots[s][k], o[name][:, :, 0]), (s, name)
        assert np.abs(r.shots[s][0]).max() > 0


@pytest.mark.parametrize("fd_order", [2, 10])
def test_uneven_orders_and_autotune(fomo, oracle, monkeypatch, fd_order):
    monkeypatch.delenv("FOMO_UNEVEN_TILE", raising=False)
    vps, rhos, sx, sz, rx, rz = _shots(seed=9)
    nt = 90
    r = fomo.acoustic2d_uneven(vps, rhos, 10.0, 1e-3, nt, 20.0, sx=sx, sz=sz, rx=rx, rz=rz,
                               nbc=5, fd_order=fd_order)
    assert r.stats.kernel_time_s > 0 and r.stats.n_shots == 5
    for s in (0, 2, 4):
        single = fomo.acoustic2d(vps[s], rhos[s], 10.0, 1e-3, nt, 20.0,
                                 sx=np.atleast_1d(sx[s]), sz=np.atleast_1d(sz[s]), rx=rx[s],
                                 rz=rz[s], nbc=5, fd_order=fd_order)
        assert np.array_equal(r.shots[s][0], single.seis_p)
        assert np.array_equal(r.shots[s][1], single.seis_vx)
        assert np.array_equal(r.shots[s][2], single.seis_vz)


def test_uneven_rerun_deterministic(fomo):
    vps, rhos, sx, sz, rx, rz = _shots(seed=4)
    a = fomo.acoustic2d_uneven(vps, rhos, 10.0, 1e-3, 60, 20.0, sx=sx, sz=sz, rx=rx, rz=rz, nbc=6)
    b = fomo.acoustic2d_uneven(vps, rhos, 10.0, 1e-3, 60, 20.0, sx=sx, sz=sz, rx=rx, rz=rz, nbc=6)
    for x, y in zip(a.shots, b.shots):
        for u, v in zip(x, y):
            assert np.array_equal(u, v)


def test_uneven_on_legacy_default_stream(fomo):
    """The run is captured into a graph; a context borrowing the legacy default
    stream (what torch's default stream maps to) must still work."""
    import torch

    from fomo_b200 import _lib as L

    ctx = L.context(0)
    ctx.use_torch_stream(torch.cuda.current_stream())
    vps, rhos, sx, sz, rx, rz = _shots(seed=2)
    a = fomo.acoustic2d_uneven(vps, rhos, 10.0, 1e-3, 40, 20.0, sx=sx, sz=sz, rx=rx, rz=rz, nbc=6)
    ctx.set_stream(None)
    b = fomo.acoustic2d_uneven(vps, rhos, 10.0, 1e-3, 40, 20.0, sx=sx, sz=sz, rx=rx, rz=rz, nbc=6)
    for x, y in zip(a.shots, b.shots):
        assert np.array_equal(x[0], y[0])


def _wide_shots(seed=0):
    """Shots wider than one strip of either width (several strips per shot,
    ragged last strips), a vacuum top on one, two sources on another."""
    from fomo_b200.synthetic import grf2d

    sizes = [(260, 30), (37, 29), (150, 44), (23, 71), (301, 25)]
    vps, rhos, sx, sz, rx, rz = [], [], [], [], [], []
    for s, (nx, nz) in enumerate(sizes):
        vp = grf2d(nx, nz, 10.0, 3000.0, 500.0, 60.0, seed + s, 2000.0, 4000.0)
        rho = np.full((nx, nz), 2000.0 + 50 * s, np.float32, order="F")
        if s == 2:
            vp[:, 0] = 0.0
            rho[:, 0] = 0.0
        vps.append(vp)
        rhos.append(rho)
        sx.append([nx // 2, 3] if s == 3 else nx // 3)
        sz.append([5, nz - 2] if s == 3 else 5)
        r = np.arange(1, nx + 1, 3)
        rx.append(r)
        rz.append(np.full(r.size, 4))
    return vps, rhos, sx, sz, rx, rz


@pytest.mark.parametrize("width", ["128", "224"])
@pytest.mark.parametrize("fd_order", [4, 8, 10])
def test_uneven_fused_sweep_equals_two_kernels(fomo, oracle, monkeypatch, width, fd_order):
    """The fused single sweep (one launch per step for all shots) equals the
    velocity / pressure kernels bit for bit on every shot, and the oracle on
    two of them."""
    monkeypatch.delenv("FOMO_UNEVEN_TILE", raising=False)
    monkeypatch.setenv("FOMO_UNEVEN_SWEEP", width)
    vps, rhos, sx, sz, rx, rz = _wide_shots(seed=fd_order)
    nt, nbc, dt = 110, 6, 1e-3
    kw = dict(sx=sx, sz=sz, rx=rx, rz=rz, nbc=nbc, fd_order=fd_order)
    a = fomo.acoustic2d_uneven(vps, rhos, 10.0, dt, nt, 20.0, **kw)
    assert fomo.api.last_stats.kernel == 2
    assert a.stats.tile == (int(width), 0)
    b = fomo.acoustic2d_uneven(vps, rhos, 10.0, dt, nt, 20.0, kernel=1, **kw)
    assert fomo.api.last_stats.kernel == 1
    for s in range(len(vps)):
        for k in range(3):
            assert np.array_equal(a.shots[s][k], b.shots[s][k]), (s, k)
        assert np.abs(a.shots[s][0]).max() > 0
    w = fomo.ricker_wavelet(20.0, dt, nt)
    for s in (0, 3):
        sxs, szs = np.atleast_1d(sx[s]), np.atleast_1d(sz[s])
        o = oracle.acoustic2d(vps[s], rhos[s], 10.0, dt, nt, sx=sxs, sz=szs, rx=rx[s], rz=rz[s],
                              wavelet=np.repeat(w[None, :], sxs.size, axis=0), nbc=nbc,
                              fd_order=fd_order)
        for k, name in enumerate(("seis_p", "seis_vx", "seis_vz")):
            assert np.array_equal(a.shots[s][k], o[name][:, :, 0]), (s, name)
