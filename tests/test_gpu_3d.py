"""GPU parity of acoustic3d / elastic3d against the 3D CPU oracle.

FP32 results are compared bit-exactly (seismograms vx/vy/vz, plane snapshots,
final padded wavefields); the FP64 oracle of the same scheme bounds the error
at 1e-5 relative L2.  The HABC on both sides is the reference's 3D Higdon
formula in two-pass form (the reference's single-pass kernel races).
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _model3d(nx, ny, nz, seed, vacuum_top=True, fluid_pocket=False):
    from fomo_b200.synthetic import gardner_rho, grf3d

    vp = grf3d(nx, ny, nz, 10.0, 3000.0, 400.0, 40.0, seed, 2000.0, 4000.0)
    vs = np.asfortranarray((vp / np.float32(1.8)).astype(np.float32))
    rho = np.asfortranarray(gardner_rho(vp))
    if fluid_pocket:
        vs[3:7, 2:5, 6:9] = 0.0
    if vacuum_top:
        for a in (vp, vs, rho):
            a[:, :, 0] = 0.0
    return vp, vs, rho


def _acq(nx, ny, nz):
    sx, sy, sz = [nx // 2, 3], [ny // 2, ny - 2], [4, nz - 3]
    gx, gy = np.meshgrid(np.arange(1, nx + 1, 3), np.arange(2, ny + 1, 4), indexing="ij")
    rx, ry = gx.ravel(order="F"), gy.ravel(order="F")
    rz = np.full(rx.size, 3)
    return sx, sy, sz, rx, ry, rz


def _final_shape(nx, ny, nz, nbc, fd_order, nf):
    p = nbc + fd_order // 2
    return (nx + 2 * p, ny + 2 * p, nz + 2 * p, nf)


@pytest.mark.parametrize("fd_order", [2, 4, 8, 10])
@pytest.mark.parametrize("plane", ["xz", "xy", "yz"])
def test_acoustic3d_bitwise(fomo, oracle, fd_order, plane):
    nx, ny, nz, nt, nbc = 21, 17, 15, 70, 5
    vp, _, rho = _model3d(nx, ny, nz, seed=fd_order)
    sx, sy, sz, rx, ry, rz = _acq(nx, ny, nz)
    dt = 1e-3
    w = fomo.ricker_wavelet(25.0, dt, nt)
    fin = np.zeros(_final_shape(nx, ny, nz, nbc, fd_order, 4), np.float32, order="F")
    sv = fomo.acoustic3d(vp, rho, 10.0, dt, nt, 25.0, sx=sx, sy=sy, sz=sz, rx=rx, ry=ry, rz=rz,
                         nbc=nbc, fd_order=fd_order, snap_interval=20, snap_plane=plane,
                         final_state=fin)
    o = oracle.acoustic3d(vp, rho, 10.0, dt, nt, sx=sx, sy=sy, sz=sz, rx=rx, ry=ry, rz=rz,
                          wavelet=np.repeat(w[None, :], 2, axis=0), nbc=nbc, fd_order=fd_order,
                          snap_interval=20, snap_plane=plane, final=True)
    for k, name in enumerate(("seis_vx", "seis_vy", "seis_vz")):
        assert np.array_equal(sv[k], o[name]), name
    assert len(sv[3]) == 3
    for k in range(3):
        assert np.array_equal(sv[3][k], o["snaps"][:, :, k])
    assert np.array_equal(fin, o["final"])
    assert np.abs(sv[2]).max() > 0


@pytest.mark.parametrize("fd_order", [2, 6, 8])
def test_elastic3d_bitwise(fomo, oracle, fd_order):
    nx, ny, nz, nt, nbc = 19, 16, 14, 60, 4
    vp, vs, rho = _model3d(nx, ny, nz, seed=10 + fd_order, fluid_pocket=True)
    sx, sy, sz, rx, ry, rz = _acq(nx, ny, nz)
    dt = 8e-4
    w = fomo.ricker_wavelet(25.0, dt, nt)
    fin = np.zeros(_final_shape(nx, ny, nz, nbc, fd_order, 9), np.float32, order="F")
    sv = fomo.elastic3d(vp, vs, rho, 10.0, dt, nt, 25.0, sx=sx, sy=sy, sz=sz, rx=rx, ry=ry, rz=rz,
                        nbc=nbc, fd_order=fd_order, snap_interval=15, snap_plane="xz",
                        snap_index=5, final_state=fin)
    o = oracle.elastic3d(vp, vs, rho, 10.0, dt, nt, sx=sx, sy=sy, sz=sz, rx=rx, ry=ry, rz=rz,
                         wavelet=np.repeat(w[None, :], 2, axis=0), nbc=nbc, fd_order=fd_order,
                         snap_interval=15, snap_plane="xz", snap_index=5, final=True)
    for k, name in enumerate(("seis_vx", "seis_vy", "seis_vz")):
        assert np.array_equal(sv[k], o[name]), name
    assert len(sv[3]) == 4
    for k in range(4):
        assert np.array_equal(sv[3][k], o["snaps"][:, :, k])
    assert np.array_equal(fin, o["final"])


@pytest.mark.parametrize("fd_order", [2, 8, 10])
def test_elastic3d_zmarch_equals_per_cell(fomo, fd_order):
    """The z-marching updates (several 32x8 tiles and z-chunks, ragged edges)
    and the fused TMA half steps (kernel 2, the default: several 30x14 tiles,
    CTA ranges that cut tiles between z planes) equal the per-cell kernels bit
    for bit, wavefields included."""
    nx, ny, nz, nt, nbc = 61, 23, 45, 40, 5
    vp, vs, rho = _model3d(nx, ny, nz, seed=40 + fd_order, fluid_pocket=True)
    sx, sy, sz, rx, ry, rz = _acq(nx, ny, nz)
    kw = dict(sx=sx, sy=sy, sz=sz, rx=rx, ry=ry, rz=rz, nbc=nbc, fd_order=fd_order)
    shape = _final_shape(nx, ny, nz, nbc, fd_order, 9)
    f_pc = np.zeros(shape, np.float32, order="F")
    b = fomo.elastic3d(vp, vs, rho, 10.0, 8e-4, nt, 25.0, final_state=f_pc, kernel=1, **kw)
    assert fomo.api.last_stats.kernel == 1
    assert np.abs(f_pc).max() > 0
    for kernel, used in ((3, 3), (2, 2), (0, 2)):
        f_zm = np.zeros(shape, np.float32, order="F")
        a = fomo.elastic3d(vp, vs, rho, 10.0, 8e-4, nt, 25.0, final_state=f_zm, kernel=kernel,
                           **kw)
        assert fomo.api.last_stats.kernel == used
        for k in range(3):
            assert np.array_equal(a[k], b[k])
        assert np.array_equal(f_zm, f_pc)


@pytest.mark.parametrize("fd_order", [2, 8, 10])
def test_acoustic3d_fused_equals_per_cell(fomo, fd_order):
    """The fused TMA half steps of acoustic3d (the default, kernel 2) equal the
    per-cell updates with two-pass Higdon kernels (kernel 1) bit for bit,
    wavefields included, on a ragged grid of several tiles and segments."""
    nx, ny, nz, nt, nbc = 61, 23, 45, 40, 5
    vp, _, rho = _model3d(nx, ny, nz, seed=60 + fd_order)
    sx, sy, sz, rx, ry, rz = _acq(nx, ny, nz)
    kw = dict(sx=sx, sy=sy, sz=sz, rx=rx, ry=ry, rz=rz, nbc=nbc, fd_order=fd_order)
    shape = _final_shape(nx, ny, nz, nbc, fd_order, 4)
    f_pc = np.zeros(shape, np.float32, order="F")
    b = fomo.acoustic3d(vp, rho, 10.0, 1e-3, nt, 25.0, final_state=f_pc, kernel=1, **kw)
    assert fomo.api.last_stats.kernel == 1
    assert np.abs(f_pc).max() > 0
    for kernel in (2, 0):
        f_fu = np.zeros(shape, np.float32, order="F")
        a = fomo.acoustic3d(vp, rho, 10.0, 1e-3, nt, 25.0, final_state=f_fu, kernel=kernel, **kw)
        assert fomo.api.last_stats.kernel == 2
        for k in range(3):
            assert np.array_equal(a[k], b[k])
        assert np.array_equal(f_fu, f_pc)


@pytest.mark.parametrize("kind", ["acoustic", "elastic"])
def test_3d_error_vs_fp64(fomo, oracle, kind):
    nx, ny, nz, nt, nbc = 24, 22, 20, 120, 8
    vp, vs, rho = _model3d(nx, ny, nz, seed=7)
    sx, sy, sz, rx, ry, rz = _acq(nx, ny, nz)
    dt = 8e-4
    w = np.repeat(fomo.ricker_wavelet(20.0, dt, nt)[None, :], 2, axis=0)
    kw = dict(sx=sx, sy=sy, sz=sz, rx=rx, ry=ry, rz=rz, nbc=nbc, fd_order=8)
    if kind == "acoustic":
        sv = fomo.acoustic3d(vp, rho, 10.0, dt, nt, 20.0, **kw)
        o = oracle.acoustic3d(vp, rho, 10.0, dt, nt, wavelet=w, prec=64, **kw)
    else:
        sv = fomo.elastic3d(vp, vs, rho, 10.0, dt, nt, 20.0, **kw)
        o = oracle.elastic3d(vp, vs, rho, 10.0, dt, nt, wavelet=w, prec=64, **kw)
    for k, name in enumerate(("seis_vx", "seis_vy", "seis_vz")):
        assert rel_l2(sv[k], o[name]) <= 1e-5, name


def test_3d_rerun_deterministic(fomo):
    nx, ny, nz = 18, 15, 13
    vp, vs, rho = _model3d(nx, ny, nz, seed=2)
    sx, sy, sz, rx, ry, rz = _acq(nx, ny, nz)
    kw = dict(sx=sx, sy=sy, sz=sz, rx=rx, ry=ry, rz=rz, nbc=4, fd_order=8, snap_interval=10)
    a = fomo.elastic3d(vp, vs, rho, 10.0, 8e-4, 50, 25.0, **kw)
    b = fomo.elastic3d(vp, vs, rho, 10.0, 8e-4, 50, 25.0, **kw)
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(x, y)
    for x, y in zip(a[3], b[3]):
        assert np.array_equal(x, y)


def test_3d_argument_errors(fomo):
    vp = np.full((10, 9, 8), 2000.0, np.float32)
    rho = np.full_like(vp, 2000.0)
    kw = dict(sx=[5], sy=[5], sz=[4], rx=[2], ry=[2], rz=[2], nbc=3, fd_order=4)
    with pytest.raises(fomo.ArgumentError):
        fomo.acoustic3d(vp, rho, 10.0, 1e-3, 10, 20.0, snap_plane="zz", **kw)
    with pytest.raises(fomo.ArgumentError):
        fomo.acoustic3d(vp, rho, 10.0, 1e-3, 10, 20.0, **dict(kw, sy=[10]))
    with pytest.raises(ValueError):
        fomo.acoustic3d(vp, rho, 10.0, 1e-3, 10, 20.0, **dict(kw, fd_order=3))
