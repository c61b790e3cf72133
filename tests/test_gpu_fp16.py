"""elastic2d with binary16 wavefield storage against the oracle's storage
emulation (bit for bit) and against the FP64 oracle (error bound)."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

SV, ST, BAND = 2.0 ** 22, 1.0, 32  # the library's storage scales and FP32 band


def _case():
    from fomo_b200.synthetic import layered_elastic

    vp, vs, rho = layered_elastic(120, 70, n_layers=5, seed=8)
    return vp, vs, rho


# nbc 30: the Higdon zone lies inside the FP32 band; nbc 60: it reaches past it.
# kernel 1: two-phase binary16 kernels; 2: the single sweep's binary16 form.
@pytest.mark.parametrize("kernel", [1, 2])
@pytest.mark.parametrize("fd_order,nbc", [(4, 30), (10, 30), (8, 60)])
def test_fp16_batch_bitwise_vs_emulation(fomo, oracle, fd_order, nbc, kernel):
    vp, vs, rho = _case()
    nt = 400
    rx = np.arange(1, 121, 4)
    rz = np.full(rx.size, 5)
    sx = np.array([[30], [90]])
    sz = np.array([[5], [40]])
    M = fd_order // 2
    nxp, nzp = 120 + 2 * (nbc + M), 70 + 2 * (nbc + M)
    fin = np.zeros((nxp, nzp, 5, 2), np.float32, order="F")
    r = fomo.elastic2d_batch(vp, vs, rho, 5.0, 5e-4, nt, 20.0, sx=sx, sz=sz, rx=rx, rz=rz,
                             nbc=nbc, fd_order=fd_order, precision="fp16", final_state=fin,
                             kernel=kernel)
    assert fomo.api.last_stats.kernel == kernel
    w = fomo.ricker_wavelet(20.0, 5e-4, nt).reshape(1, -1)
    kw = dict(sx=sx.T, sz=sz.T, rx=rx, rz=rz, wavelet=w, nbc=nbc, fd_order=fd_order, n_shots=2)
    o = oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, final=True, store="fp16", sv=SV, st=ST,
                         fp32_band=BAND, **kw)
    assert np.array_equal(r.seis_vx, o["seis_vx"])
    assert np.array_equal(r.seis_vz, o["seis_vz"])
    assert np.array_equal(fin, o["final"])
    ref = oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, prec=64, **kw)
    for k, name in ((r.seis_vx, "seis_vx"), (r.seis_vz, "seis_vz")):
        e = rel_l2(k, ref[name])
        assert 1e-6 < e < 2e-2, (name, e)


# variant,TX,CTAs per SM of the sweep's binary16 form: several strips (first and
# last touch the FP32 columns), segment boundaries inside the z band
@pytest.mark.parametrize("cfg", ["17,112,3", "18,56,2", "17,8,1", "18,40,1"])
def test_fp16_sweep_configs_bitwise(fomo, oracle, monkeypatch, cfg):
    from fomo_b200.synthetic import layered_elastic

    monkeypatch.setenv("FOMO_SWEEP_CONFIG", cfg)
    vp, vs, rho = layered_elastic(260, 90, n_layers=6, seed=21)
    nt, nbc, fd_order = 150, 40, 10
    rx = np.arange(1, 261, 6)
    rz = np.full(rx.size, 4)
    sx = np.array([[20], [240]])
    sz = np.array([[4], [80]])
    M = fd_order // 2
    fin = np.zeros((260 + 2 * (nbc + M), 90 + 2 * (nbc + M), 5, 2), np.float32, order="F")
    r = fomo.elastic2d_batch(vp, vs, rho, 5.0, 5e-4, nt, 20.0, sx=sx, sz=sz, rx=rx, rz=rz,
                             nbc=nbc, fd_order=fd_order, precision="fp16", final_state=fin,
                             kernel=2)
    w = fomo.ricker_wavelet(20.0, 5e-4, nt).reshape(1, -1)
    o = oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, sx=sx.T, sz=sz.T, rx=rx, rz=rz, wavelet=w,
                         nbc=nbc, fd_order=fd_order, n_shots=2, final=True, store="fp16", sv=SV,
                         st=ST, fp32_band=BAND)
    assert np.array_equal(r.seis_vx, o["seis_vx"])
    assert np.array_equal(r.seis_vz, o["seis_vz"])
    assert np.array_equal(fin, o["final"])


def test_fp16_single_equals_batch_and_snapshots(fomo, oracle):
    vp, vs, rho = _case()
    nt = 200
    rx = np.arange(1, 121, 5)
    rz = np.full(rx.size, 4)
    single = fomo.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, 20.0, sx=[60], sz=[10], rx=rx, rz=rz,
                            nbc=20, fd_order=8, snap_interval=50, precision="fp16")
    batch = fomo.elastic2d_batch(vp, vs, rho, 5.0, 5e-4, nt, 20.0, sx=[60], sz=[10], rx=rx, rz=rz,
                                 nbc=20, fd_order=8, precision="fp16")
    assert np.array_equal(single.seis_vx, batch.seis_vx[:, :, 0])
    assert np.array_equal(single.seis_vz, batch.seis_vz[:, :, 0])
    w = fomo.ricker_wavelet(20.0, 5e-4, nt).reshape(1, -1)
    o = oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, sx=[[60]], sz=[[10]], rx=rx, rz=rz,
                         wavelet=w, nbc=20, fd_order=8, snap_interval=50, store="fp16", sv=SV,
                         st=ST, fp32_band=BAND)
    assert len(single.snaps) == 4
    for k in range(4):
        assert np.array_equal(single.snaps[k], o["snaps"][:, :, k, 0])


def test_bf16_storage_is_refused(fomo):
    vp, vs, rho = _case()
    with pytest.raises(fomo.FomoError):
        fomo.elastic2d_batch(vp, vs, rho, 5.0, 5e-4, 20, 20.0, sx=[60], sz=[10], rx=[5], rz=[5],
                             nbc=20, precision="bf16")
