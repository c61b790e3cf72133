"""Host-side behaviour of the Fomo API mirror: validation before any launch (no GPU)."""
import warnings

import numpy as np
import pytest


def _acoustic_inputs(nx=40, nz=30):
    vp = np.full((nx, nz), 3000.0, np.float32)
    rho = np.full((nx, nz), 2200.0, np.float32)
    return vp, rho


def test_geometry_errors(fomo):
    vp, rho = _acoustic_inputs()
    kw = dict(rx=[5, 10], rz=[3, 3])
    with pytest.raises(fomo.ArgumentError):
        fomo.acoustic2d(vp, rho, 10.0, 1e-3, 50, 15.0, sx=[45], sz=[3], **kw)
    with pytest.raises(fomo.ArgumentError):
        fomo.acoustic2d(vp, rho, 10.0, 1e-3, 50, 15.0, sx=[5], sz=[0], **kw)
    with pytest.raises(fomo.ArgumentError):
        fomo.elastic2d(vp, vp / 1.7, rho, 10.0, 1e-3, 50, 15.0, sx=[5], sz=[3], rx=[41], rz=[3])
    with pytest.raises(fomo.ArgumentError):
        fomo.elastic2d_batch(vp, vp / 1.7, rho, 10.0, 1e-3, 50, 15.0, sx=[5, 50], sz=[3, 3],
                             rx=[4], rz=[3])


def test_cfl_error(fomo):
    vp, rho = _acoustic_inputs()
    with pytest.raises(fomo.ArgumentError):  # verify_patch.jl:106-110
        fomo.acoustic2d(vp, rho, 10.0, 9e-3, 50, 15.0, sx=[5], sz=[3], rx=[4], rz=[3])
    with pytest.raises(fomo.ArgumentError):
        fomo.scalar2d(vp, 10.0, 9e-3, 50, 15.0, sx=[5], sz=[3], rx=[4], rz=[3])


def test_wavelet_length_and_keywords(fomo):
    vp, rho = _acoustic_inputs()
    kw = dict(sx=[5], sz=[3], rx=[4], rz=[3])
    with pytest.raises(fomo.ArgumentError):
        fomo.acoustic2d(vp, rho, 10.0, 1e-3, 50, 15.0, wavelet=np.zeros(49), **kw)
    with pytest.raises(fomo.ArgumentError):
        fomo.acoustic2d(vp, rho, 10.0, 1e-3, 50, 15.0, boundary="pml", **kw)
    with pytest.raises(fomo.ArgumentError):
        fomo.scalar2d(vp, 10.0, 1e-3, 50, 15.0, source_scale=":foo", **kw)
    with pytest.raises(fomo.ArgumentError):
        fomo.acoustic2d_batch(vp, rho, 10.0, 1e-3, 50, 15.0, sx=[[5, 6]], sz=[[3]], rx=[4], rz=[3])


def test_sponge_boundary_options(fomo):
    """boundary=:sponge sets FOMO_F_SPONGE and the Cerjan factor in fomo_opts."""
    from fomo_b200 import _lib as L
    from fomo_b200.api import _check_boundary, _opts

    assert _check_boundary(":sponge") and _check_boundary("sponge")
    assert not _check_boundary(":habc")
    o = _opts(sponge_factor=0.02)
    assert o.flags & L.FOMO_F_SPONGE and o.sponge_factor == np.float32(0.02)
    o = _opts()
    assert not o.flags & L.FOMO_F_SPONGE


def test_dispersion_warning(fomo):
    from fomo_b200.api import _check_numerics

    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        _check_numerics(3000.0, 500.0, 10.0, 1e-3, 30.0, 8)
    assert any("dispersion" in str(x.message) for x in w)


def test_ricker_matches_oracle(fomo, oracle):
    assert np.array_equal(fomo.ricker_wavelet(15.0, 1e-3, 700), oracle.ricker(15.0, 1e-3, 700))
    w = fomo.ricker_wavelet(10.0, 1e-3, 1000)
    assert abs(float(w.max()) - 1.0) < 1e-6 and np.argmax(w) == 150  # peak at 1.5/f0


@pytest.mark.parametrize("f0,dt,nt", [(15.0, 1e-3, 700), (20.0, 5e-4, 3000), (25.0, 5e-4, 2000),
                                      (12.0, 8e-4, 2500)])
def test_ricker_is_float32_arithmetic_within_float64_bound(fomo, f0, dt, nt):
    """utils/ricker_wavelet.jl:6-12 computes in Float32 (t0 = 1f0/f0, 1.5f0*t0,
    Float32 exp).  The mirror follows those steps: it sits within the rounding
    bound of a float64 evaluation of the same formula (absolute 2e-6 on a unit
    peak: tau cancels near the peak, where t ~ 1.5/f0 is resolved to a Float32
    ulp), and is not the float64 result rounded once."""
    w = fomo.ricker_wavelet(f0, dt, nt)
    assert w.dtype == np.float32 and w.shape == (nt,)
    f, d = float(np.float32(f0)), float(np.float32(dt))
    t = np.arange(nt, dtype=np.float64) * d
    x = np.pi * f * (t - 1.5 / f)
    w64 = (1.0 - 2.0 * x * x) * np.exp(-x * x)
    assert float(np.abs(w.astype(np.float64) - w64).max()) < 2e-6
    # the first samples are 1 - 2x^2 times exp(-x^2) with x ~ -1.5 pi: Float32 steps
    f32 = np.float32
    t1 = f32(f32(1.0) * np.float32(dt))
    x1 = f32(f32(np.float32(np.pi) * np.float32(f0)) *
             f32(t1 - f32(f32(1.5) * f32(f32(1.0) / np.float32(f0)))))
    a1 = f32(x1 * x1)
    assert w[1] == f32(f32(f32(1.0) - f32(2.0) * a1) * np.exp(-a1))


def test_scalar_source_scaling(fomo):
    from fomo_b200.api import scalar_wavelet_matrix

    vp = np.full((10, 8), 2000.0, np.float32)
    vp[3, 2] = 2500.0
    w = np.linspace(-1, 1, 7).astype(np.float32)
    m = scalar_wavelet_matrix(w, vp, 1e-3, [4, 1], [3, 1], "v2dt2")
    s0 = np.float32(np.float32(2500.0) * np.float32(2500.0) * (np.float32(1e-3) * np.float32(1e-3)))
    assert np.array_equal(m[0], (w * s0).astype(np.float32))
    assert np.array_equal(scalar_wavelet_matrix(w, vp, 1e-3, [4], [3], "none")[0], w)
    assert np.array_equal(scalar_wavelet_matrix(w, vp, 1e-3, [4], [3], "dt")[0],
                          (w * np.float32(1e-3)).astype(np.float32))


def test_fd_coefficients(fomo):
    a = fomo.get_fd_coefficients(8)
    assert a.dtype == np.float32 and a.size == 4
    assert np.float32(a[0]) == np.float32(1.1962890625)
    c0, d2 = fomo.get_centered_d2(4)
    assert c0 == np.float32(-2.5) and d2[0] == np.float32(4 / 3)
    with pytest.raises(ValueError):
        fomo.get_fd_coefficients(12)


def test_synthetic_layered_config(fomo):
    from fomo_b200.synthetic import elastic_batch_config

    c = elastic_batch_config()
    assert c["vp"].shape == (1000, 500) and c["sx"].size == 32 and c["rx"].size == 500
    assert 1500 <= c["vp"].min() and c["vp"].max() <= 4500
    assert np.allclose(c["vs"], c["vp"] / 1.73, rtol=1e-6)
    assert len(np.unique(c["vp"][0])) == 12


def test_uneven_batch_validation(fomo):
    vp1, rho1 = _acoustic_inputs(40, 30)
    vp2, rho2 = _acoustic_inputs(25, 35)
    kw = dict(sx=[20, 12], sz=[3, 3], rx=[[4, 8], [5]], rz=[[3, 3], [4]])
    with pytest.raises(fomo.ArgumentError):  # one entry per shot
        fomo.acoustic2d_uneven([vp1, vp2], [rho1], 10.0, 1e-3, 50, 15.0, **kw)
    with pytest.raises(fomo.ArgumentError):  # receiver outside shot 2's grid
        fomo.acoustic2d_uneven([vp1, vp2], [rho1, rho2], 10.0, 1e-3, 50, 15.0,
                               **dict(kw, rx=[[4], [30]], rz=[[3], [3]]))
    with pytest.raises(fomo.ArgumentError):  # CFL over the fastest shot
        fomo.acoustic2d_uneven([vp1, vp2 * 3], [rho1, rho2], 10.0, 1e-3, 50, 15.0, **kw)
    with pytest.raises(ValueError):
        fomo.acoustic2d_uneven([vp1, vp2], [rho1, rho2], 10.0, 1e-3, 50, 15.0, fd_order=7, **kw)


def test_coupled2d_validation(fomo):
    """coupled2d.jl:71-77: geometry and the centered CFL bound are checked on the
    host; the shapes of vp and vs must agree."""
    vp = np.full((40, 30), 3000.0, np.float32)
    vs = np.full((40, 30), 1700.0, np.float32)
    kw = dict(sx=[5], sz=[3], rx=[4], rz=[3])
    with pytest.raises(fomo.ArgumentError):
        fomo.coupled2d(vp, vs[:, :20], 10.0, 1e-3, 50, 15.0, **kw)
    with pytest.raises(fomo.ArgumentError):
        fomo.coupled2d(vp, vs, 10.0, 9e-3, 50, 15.0, **kw)
    with pytest.raises(fomo.ArgumentError):
        fomo.coupled2d(vp, vs, 10.0, 1e-3, 50, 15.0, sx=[41], sz=[3], rx=[4], rz=[3])
