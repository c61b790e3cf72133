"""boundary=:sponge (boundary/sponge.jl, the legacy loops acoustic2d.jl:197-244 and
elastic2d.jl:168-212) on the GPU against the CPU oracle.

FP32 results are compared bit for bit; the FP64 oracle bounds the error
(tolerance 1e-5 relative L2).  The shielded mirror-symmetry check restates the
reference's own GPU test of the sponge path (test/verify_patch.jl:59-73).
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

FACTOR = 0.015


def _vacuum_top(*arrs):
    out = []
    for a in arrs:
        a = a.copy(order="F")
        a[:, 0] = 0.0
        out.append(a)
    return out


@pytest.fixture
def with_flags(monkeypatch, fomo):
    """Calls made through this fixture's function get extra fomo_opts settings."""
    orig = fomo.api._opts

    def run(fn, *a, flags=0, sponge_factor=None, **kw):
        def opts(*oa, **okw):
            if sponge_factor is not None:
                okw["sponge_factor"] = sponge_factor
            o = orig(*oa, **okw)
            o.flags |= flags
            return o

        monkeypatch.setattr(fomo.api, "_opts", opts)
        try:
            return fn(*a, **kw)
        finally:
            monkeypatch.setattr(fomo.api, "_opts", orig)

    return run


@pytest.mark.parametrize("fd_order", [2, 4, 8, 10])
def test_acoustic2d_sponge_bitwise_vs_oracle(fomo, oracle, fd_order):
    from fomo_b200.synthetic import two_layer

    vp, rho = _vacuum_top(*two_layer(63, 47))
    nt, nbc = 200, 12
    rx = np.arange(1, 64, 3)
    rz = np.full(rx.size, 9)
    w = fomo.ricker_wavelet(15.0, 1e-3, nt)
    M = fd_order // 2
    fin = np.zeros((63 + 2 * (nbc + M), 47 + 2 * (nbc + M), 3), np.float32, order="F")
    kw = dict(sx=[31], sz=[10], rx=rx, rz=rz, nbc=nbc, fd_order=fd_order, snap_interval=40)
    r = fomo.acoustic2d(vp, rho, 10.0, 1e-3, nt, 15.0, boundary=":sponge", sponge_factor=FACTOR,
                        final_state=fin, **kw)
    o = oracle.acoustic2d(vp, rho, 10.0, 1e-3, nt, wavelet=w.reshape(1, -1), final=True,
                          sponge_factor=FACTOR, **kw)
    for got, want in ((r.seis_p, o["seis_p"]), (r.seis_vx, o["seis_vx"]),
                      (r.seis_vz, o["seis_vz"])):
        assert np.array_equal(got, want[:, :, 0])
    assert len(r.snaps) == 5
    for k, s in enumerate(r.snaps):
        assert np.array_equal(s, o["snaps"][:, :, k, 0])
    assert np.array_equal(fin, o["final"][:, :, :, 0])
    o64 = oracle.acoustic2d(vp, rho, 10.0, 1e-3, nt, wavelet=w.reshape(1, -1), prec=64,
                            sponge_factor=FACTOR, **kw)
    assert rel_l2(r.seis_p, o64["seis_p"][:, :, 0]) < 1e-5
    # the sponge differs from HABC: the boundary really switched
    h = fomo.acoustic2d(vp, rho, 10.0, 1e-3, nt, 15.0, **kw)
    assert not np.array_equal(h.seis_p, r.seis_p)


@pytest.mark.parametrize("fd_order", [4, 8])
def test_elastic2d_sponge_bitwise_vs_oracle(fomo, oracle, fd_order):
    from fomo_b200.synthetic import layered_elastic

    vp, vs, rho = _vacuum_top(*layered_elastic(58, 44, n_layers=4, seed=11))
    nt, nbc = 180, 10
    rx = np.arange(1, 59, 3)
    rz = np.full(rx.size, 6)
    w = fomo.ricker_wavelet(20.0, 5e-4, nt)
    M = fd_order // 2
    fin = np.zeros((58 + 2 * (nbc + M), 44 + 2 * (nbc + M), 5), np.float32, order="F")
    kw = dict(sx=[29], sz=[8], rx=rx, rz=rz, nbc=nbc, fd_order=fd_order, snap_interval=45)
    r = fomo.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, 20.0, boundary="sponge", sponge_factor=FACTOR,
                       final_state=fin, **kw)
    o = oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, wavelet=w.reshape(1, -1), final=True,
                         sponge_factor=FACTOR, **kw)
    assert np.array_equal(r.seis_vx, o["seis_vx"][:, :, 0])
    assert np.array_equal(r.seis_vz, o["seis_vz"][:, :, 0])
    assert len(r.snaps) == 4
    for k, s in enumerate(r.snaps):
        assert np.array_equal(s, o["snaps"][:, :, k, 0])
    assert np.array_equal(fin, o["final"][:, :, :, 0])
    o64 = oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, wavelet=w.reshape(1, -1), prec=64,
                           sponge_factor=FACTOR, **kw)
    assert rel_l2(r.seis_vz, o64["seis_vz"][:, :, 0]) < 1e-5
    assert fomo.api.last_stats.kernel == 1  # the sponge runs the two-phase kernels


def test_sponge_chunks_equal_step_launches(fomo, with_flags):
    """Replayed CUDA-graph chunks and per-step launches give the same bits."""
    from fomo_b200 import _lib as L
    from fomo_b200.synthetic import two_layer

    vp, rho = _vacuum_top(*two_layer(70, 50))
    rx = np.arange(1, 71, 3)
    kw = dict(sx=[35], sz=[10], rx=rx, rz=np.full(rx.size, 8), nbc=10, fd_order=8,
              boundary="sponge", sponge_factor=0.02)
    a = fomo.acoustic2d(vp, rho, 10.0, 1e-3, 230, 15.0, **kw)
    b = with_flags(fomo.acoustic2d, vp, rho, 10.0, 1e-3, 230, 15.0, flags=L.FOMO_F_STEP_LAUNCH,
                   **kw)
    assert np.array_equal(a.seis_p, b.seis_p)
    assert np.array_equal(a.seis_vx, b.seis_vx)


def test_batch_sponge_bitwise_vs_oracle(fomo, oracle, with_flags):
    """The batch entry points accept FOMO_F_SPONGE too (one grid z-slice per shot)."""
    from fomo_b200.synthetic import layered_elastic

    vp, vs, rho = _vacuum_top(*layered_elastic(50, 40, n_layers=3, seed=2))
    nt = 150
    rx = np.arange(1, 51, 4)
    rz = np.full(rx.size, 5)
    w = fomo.ricker_wavelet(20.0, 5e-4, nt)
    kw = dict(sx=[12, 38], sz=[7, 20], rx=rx, rz=rz, nbc=8, fd_order=8)
    r = with_flags(fomo.elastic2d_batch, vp, vs, rho, 5.0, 5e-4, nt, 20.0, sponge_factor=FACTOR,
                   **kw)
    o = oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, wavelet=w.reshape(1, -1),
                         sponge_factor=FACTOR, n_shots=2, **kw)
    assert np.array_equal(r.seis_vz, o["seis_vz"])
    assert np.array_equal(r.seis_vx, o["seis_vx"])
    ra = with_flags(fomo.acoustic2d_batch, vp, rho, 5.0, 5e-4, nt, 20.0, sponge_factor=FACTOR,
                    **kw)
    oa = oracle.acoustic2d(vp, rho, 5.0, 5e-4, nt, wavelet=w.reshape(1, -1),
                           sponge_factor=FACTOR, n_shots=2, **kw)
    assert np.array_equal(ra.seis_p, oa["seis_p"])


def test_sponge_mirror_symmetry_under_causal_shielding(fomo):
    """verify_patch.jl:59-73 with boundary=:sponge: symmetric model, centred
    source, receivers shielded from the boundary: mirror residual < 1e-5."""
    from fomo_b200.synthetic import symmetric_model

    vp, vs, rho = symmetric_model(601, 201)
    rx = np.arange(150, 453)
    kw = dict(sx=[301], sz=[41], rx=rx, rz=np.full(rx.size, 41), nbc=30, fd_order=4,
              boundary=":sponge")

    def rel_sym(d):
        return float(np.linalg.norm(d - d[::-1]) / np.linalg.norm(d))

    def rel_asym_vx(d):
        e = d[1:]
        return float(np.linalg.norm(e + e[::-1]) / np.linalg.norm(e))

    a = fomo.acoustic2d(vp, rho, 10.0, 1e-3, 1200, 10.0, **kw)
    assert rel_sym(a.seis_p) < 1e-5 and rel_sym(a.seis_vz) < 1e-5
    assert rel_asym_vx(a.seis_vx) < 1e-5
    e = fomo.elastic2d(vp, vs, rho, 10.0, 1e-3, 1200, 10.0, **kw)
    assert rel_sym(e.seis_vz) < 1e-5 and rel_asym_vx(e.seis_vx) < 1e-5


def test_sponge_unsupported_combinations(fomo):
    from fomo_b200 import _lib as L
    from fomo_b200.synthetic import layered_elastic

    vp, vs, rho = layered_elastic(40, 30, n_layers=2, seed=1)
    kw = dict(sx=[20], sz=[5], rx=[10, 20], rz=[5, 5], nbc=8, fd_order=8, boundary="sponge")
    with pytest.raises(L.FomoError) as e:
        fomo.elastic2d(vp, vs, rho, 5.0, 5e-4, 20, 20.0, precision="fp16", **kw)
    assert e.value.code == L.FOMO_EUNSUPPORTED
    with pytest.raises(L.FomoError) as e:
        fomo.elastic2d(vp, vs, rho, 5.0, 5e-4, 20, 20.0, kernel=2, **kw)
    assert e.value.code == L.FOMO_EUNSUPPORTED
    with pytest.raises(L.FomoError) as e:
        fomo.elastic2d(vp, vs, rho, 5.0, 5e-4, 20, 20.0, sponge_factor=-1.0, **kw)
    assert e.value.code == L.FOMO_EARG


def test_sponge_with_no_layers_is_the_plain_update(fomo, oracle):
    """nbc = 0: no damped cells (reference: d < nbc never holds), so the sponge
    run is the bare update with a fixed outer ring; bit-exact to the oracle."""
    from fomo_b200.synthetic import two_layer

    vp, rho = _vacuum_top(*two_layer(50, 40))
    nt = 120
    w = fomo.ricker_wavelet(15.0, 1e-3, nt)
    kw = dict(sx=[25], sz=[10], rx=np.arange(1, 51, 4), rz=np.full(13, 6), nbc=0, fd_order=8)
    r = fomo.acoustic2d(vp, rho, 10.0, 1e-3, nt, 15.0, boundary="sponge", **kw)
    o = oracle.acoustic2d(vp, rho, 10.0, 1e-3, nt, wavelet=w[None], sponge_factor=FACTOR, **kw)
    assert np.array_equal(r.seis_p, o["seis_p"][:, :, 0])
    assert np.abs(r.seis_p).max() > 0
