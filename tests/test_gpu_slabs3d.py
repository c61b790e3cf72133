"""GPU parity of the z-slab decomposition (fomo_slab3d_*) against the single-device run.

Several slabs share one device here and exchange halos by device copies (the
multi-GPU form sends the same plane blocks by NCCL; its schedule is covered on
CPU by tests/test_slabs3d_host.py).  Every receiver's seismogram and every
owned plane of every field after the last step must equal elastic3d /
acoustic3d (fused half steps) bit for bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _model(nx, ny, nz, seed):
    from fomo_b200.synthetic import gardner_rho, grf3d

    vp = grf3d(nx, ny, nz, 10.0, 3000.0, 400.0, 40.0, seed, 2000.0, 4000.0)
    vs = np.asfortranarray((vp / np.float32(1.8)).astype(np.float32))
    rho = np.asfortranarray(gardner_rho(vp))
    for a in (vp, vs, rho):
        a[:, :, 0] = 0.0  # vacuum top
    return vp, vs, rho


def _acq(nx, ny, nz, src_z):
    sx, sy, sz = [nx // 2, 5], [ny // 2, ny - 4], list(src_z)
    gx, gy = np.meshgrid(np.arange(1, nx + 1, 5), np.arange(2, ny + 1, 6), indexing="ij")
    rx, ry = gx.ravel(order="F"), gy.ravel(order="F")
    # receivers at depths that fall in every slab
    depths = (3, nz // 3, nz // 2, nz - 4)
    rz = np.array([depths[k % len(depths)] for k in range(rx.size)], dtype=np.int32)
    return dict(sx=sx, sy=sy, sz=sz, rx=rx, ry=ry, rz=rz)


def _check(fomo, slabs3d, elastic, fd_order, nbc, shape, nt, n_slabs=None, cuts=None,
           src_z=(4, 20)):
    nx, ny, nz = shape
    vp, vs, rho = _model(nx, ny, nz, 7)
    kw = dict(nbc=nbc, fd_order=fd_order, **_acq(nx, ny, nz, src_z))
    p = nbc + fd_order // 2
    nf = 9 if elastic else 4
    fin = np.zeros((nx + 2 * p, ny + 2 * p, nz + 2 * p, nf), dtype=np.float32, order="F")
    dt = 8e-4 if elastic else 1e-3
    if elastic:
        ref = fomo.elastic3d(vp, vs, rho, 10.0, dt, nt, 25.0, final_state=fin, kernel=2, **kw)
    else:
        ref = fomo.acoustic3d(vp, rho, 10.0, dt, nt, 25.0, final_state=fin, kernel=2, **kw)
    parts = []
    extra = dict(n_slabs=n_slabs or 2, cuts=cuts, final_state=parts)
    if elastic:
        got = slabs3d.elastic3d_slabs(vp, vs, rho, 10.0, dt, nt, 25.0, **kw, **extra)
    else:
        got = slabs3d.acoustic3d_slabs(vp, rho, 10.0, dt, nt, 25.0, **kw, **extra)
    assert np.abs(ref[2]).max() > 0  # the wave reached the receivers
    for k in range(3):
        np.testing.assert_array_equal(got[k], ref[k])
    covered = 0
    for z_lo, z_hi, fields in parts:
        for f in range(nf):
            want = np.transpose(fin[:, :, z_lo:z_hi, f], (2, 1, 0))
            np.testing.assert_array_equal(fields[f], want, err_msg=f"field {f} [{z_lo}, {z_hi})")
        covered += z_hi - z_lo
    assert covered == nz + 2 * p
    return parts


@pytest.fixture(scope="module")
def slabs3d(fomo):
    from fomo_b200 import slabs3d as m

    return m


@pytest.mark.parametrize("n_slabs", [2, 3])
def test_elastic3d_slabs_bitwise(fomo, slabs3d, n_slabs):
    parts = _check(fomo, slabs3d, True, 8, 8, (40, 34, 64), 70, n_slabs=n_slabs)
    assert len(parts) == n_slabs


def test_elastic3d_slabs_uneven_cuts_source_at_cut(fomo, slabs3d):
    # order 10, cuts at the edges of the allowed range; a source one plane
    # above and one below a cut (its injection reaches the neighbour's halo)
    nbc, fd_order, nz = 6, 10, 60
    pad = nbc + fd_order // 2
    nzp = nz + 2 * pad
    cuts = [(0, pad + 1), (pad + 1, 40), (40, nzp - pad - 1), (nzp - pad - 1, nzp)]
    src_z = (40 - pad, 41 - pad)  # 1-based interior z of padded planes 39 and 40
    _check(fomo, slabs3d, True, fd_order, nbc, (36, 30, nz), 50, cuts=cuts, src_z=src_z)


@pytest.mark.parametrize("fd_order", [4, 8])
def test_acoustic3d_slabs_bitwise(fomo, slabs3d, fd_order):
    _check(fomo, slabs3d, False, fd_order, 8, (44, 38, 60), 80, n_slabs=3)


def test_slab_refuses_cut_in_higdon_band(fomo, slabs3d):
    from fomo_b200._lib import FomoError

    nx, ny, nz = 30, 28, 40
    vp, vs, rho = _model(nx, ny, nz, 3)
    kw = dict(nbc=8, fd_order=8, **_acq(nx, ny, nz, (4, 10)))
    pad = 12
    for c in (pad, nz + pad):  # one plane past each end of the allowed range
        with pytest.raises(FomoError, match="Higdon z bands"):
            slabs3d.elastic3d_slabs(vp, vs, rho, 10.0, 8e-4, 10, 25.0,
                                    cuts=[(0, c), (c, nz + 2 * pad)], **kw)


def test_elastic3d_slabs_order2_one_plane_slab(fomo, slabs3d):
    # halo 1: a slab owning a single plane takes both halos from two neighbours
    nbc, fd_order, nz = 4, 2, 20
    pad = nbc + fd_order // 2          # 5: cuts in [6, 24] of 30 planes
    nzp = nz + 2 * pad
    cuts = [(0, 6), (6, 7), (7, 24), (24, nzp)]
    _check(fomo, slabs3d, True, fd_order, nbc, (26, 22, nz), 40, cuts=cuts, src_z=(2, 3))


def test_acoustic3d_slabs_source_on_cut(fomo, slabs3d):
    # order 6; the second source sits on the first plane of the second slab
    nbc, fd_order, nz = 6, 6, 48
    pad = nbc + fd_order // 2          # 9: 66 planes
    cuts = [(0, 30), (30, 66)]
    _check(fomo, slabs3d, False, fd_order, nbc, (34, 30, nz), 60, cuts=cuts,
           src_z=(4, 30 - pad + 1))
