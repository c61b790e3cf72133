"""coupled2d oracle (equations/coupled2d/*).

The reference ships no coupled2d test or reference output, so parity of this
restatement is unpinned to the reference's numbers; these checks pin it to the
mathematics instead:
  * the centered d1 / d2 tables (utils/FD_centered.jl:15-41) have the moments of
    their order of accuracy;
  * in a homogeneous medium every medium derivative vanishes and the split
    update is the scalar leapfrog: P equals scalar2d driven by the differenced
    wavelet (FP64), and S stays exactly 0;
  * mirror symmetry on a symmetric model: P even, S odd (as verify_patch.jl:59-73
    checks for the other solvers);
  * FP32 against FP64 within 1e-5.
"""
import numpy as np
import pytest

from conftest import rel_l2


@pytest.mark.parametrize("order", [2, 4, 6, 8, 10])
def test_centered_coefficient_moments(oracle, order):
    from fomo_b200.api import get_centered_d2

    N = order // 2

    c0, d2 = get_centered_d2(order)
    d1 = np.array({2: [1 / 2], 4: [2 / 3, -1 / 12], 6: [3 / 4, -3 / 20, 1 / 60],
                   8: [4 / 5, -1 / 5, 4 / 105, -1 / 280],
                   10: [5 / 6, -5 / 21, 5 / 84, -5 / 504, 1 / 1260]}[order], np.float32)
    l = np.arange(1, N + 1, dtype=np.float64)
    d1 = d1.astype(np.float64)
    assert abs(np.sum(2 * l * d1) - 1) < 1e-6
    for k in range(1, N):  # float32 rounding of the table, relative to the moment's size
        assert abs(np.sum(d1 * l ** (2 * k + 1))) < 1e-6 * np.sum(np.abs(d1) * l ** (2 * k + 1))
    d2 = np.asarray(d2, np.float64)
    assert abs(float(c0) + 2 * np.sum(d2)) < 1e-6
    assert abs(np.sum(d2 * l ** 2) - 1) < 1e-6
    for k in range(2, N + 1):
        assert abs(np.sum(d2 * l ** (2 * k))) < 1e-6 * np.sum(np.abs(d2) * l ** (2 * k))


def _exact_wavelet(oracle, nt):
    """A Ricker-shaped wavelet whose first differences are exact in float32."""
    r = oracle.ricker(15.0, 1e-3, nt).astype(np.float64)
    q = np.round(np.diff(np.concatenate([[0.0], r])) * 2 ** 20) / 2 ** 20
    return np.cumsum(q).astype(np.float32), q.astype(np.float32)


def test_homogeneous_coupled_p_is_the_scalar_leapfrog(oracle):
    n, nt = 161, 400
    vp = np.full((n, n), 2500.0, np.float32)
    vs = np.full((n, n), 1500.0, np.float32)
    w, dw = _exact_wavelet(oracle, nt)
    rx = np.arange(50, 113, 2)
    kw = dict(sx=[81], sz=[81], rx=rx, rz=np.full(rx.size, 81), nbc=20, fd_order=8)
    c = oracle.coupled2d(vp, vs, 10.0, 1e-3, nt, wavelet=w[None], prec=64, **kw)
    s = oracle.scalar2d(vp, 10.0, 1e-3, nt, wavelet=dw[None], prec=64, **kw)
    su = s["seis_u"] if s["seis_u"].ndim == 2 else s["seis_u"][:, :, 0]
    # the scalar oracle holds (v dt / dh)^2 as a float32 constant: a 1e-6 phase drift
    assert rel_l2(c["seis_P"], su) < 2e-6
    assert np.abs(c["seis_P"]).max() > 0.1
    assert not np.any(c["seis_S"])


def test_mirror_symmetry_p_even_s_odd(oracle):
    from fomo_b200.synthetic import symmetric_model

    vp, vs, _ = symmetric_model(201, 121)
    nt = 600
    rx = np.arange(40, 163)  # r <-> 202 - r
    c = oracle.coupled2d(vp, vs, 10.0, 1e-3, nt, sx=[101], sz=[41], rx=rx,
                         rz=np.full(rx.size, 41), wavelet=oracle.ricker(10.0, 1e-3, nt)[None],
                         nbc=20, fd_order=4)
    P, S = c["seis_P"], c["seis_S"]
    assert np.linalg.norm(P - P[::-1]) / np.linalg.norm(P) < 1e-5
    assert np.linalg.norm(S + S[::-1]) / np.linalg.norm(S) < 1e-5
    assert np.abs(S).max() > 1e-3 * np.abs(P).max()  # the coupling terms are active


def test_fp32_within_1e5_of_fp64(oracle):
    from fomo_b200.synthetic import layered_elastic

    vp, vs, _ = layered_elastic(80, 60, n_layers=4, seed=3)
    nt = 400
    kw = dict(sx=[40], sz=[20], rx=np.arange(1, 81, 2), rz=np.full(40, 10), nbc=15, fd_order=8,
              wavelet=oracle.ricker(15.0, 1e-3, nt)[None], snap_interval=100)
    a = oracle.coupled2d(vp, vs, 10.0, 1e-3, nt, prec=32, **kw)
    b = oracle.coupled2d(vp, vs, 10.0, 1e-3, nt, prec=64, **kw)
    assert rel_l2(a["seis_P"], b["seis_P"]) < 1e-5
    assert rel_l2(a["seis_S"], b["seis_S"]) < 1e-5
    assert rel_l2(a["snaps_P"], b["snaps_P"]) < 1e-5
