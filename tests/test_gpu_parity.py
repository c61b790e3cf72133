"""GPU parity: libfomo_b200 (through the C ABI) against the CPU oracle.

The kernels spell out the oracle's rounding sequence, so FP32 results are
compared BIT-EXACTLY (seismograms, snapshots, final wavefields, device-prepared
materials).  The FP64 oracle of the same scheme gives the reported error
(tolerance 1e-5 relative L2).
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

KERNELS = [1, 2]  # two-phase, single-sweep


SWEEP_CONFIGS = ["0,112,3", "1,144,1", "2,80,2", "2,20,4", "3,112,2", "0,64,1",
                 "4,224,1", "5,100,1", "6,40,1", "5,8,1",
                 "7,224,2", "8,196,2", "8,40,2", "7,8,1",
                 "9,224,2", "10,176,2", "11,112,4", "12,100,4", "11,8,1", "9,40,1",
                 "12,60,3", "13,224,2", "14,112,4", "15,100,3", "16,112,3", "14,8,1",
                 "13,40,1", "16,20,2",
                 "19,112,2", "19,100,1", "20,80,2", "21,40,4", "19,8,1", "21,20,2",
                 "20,10,3", "22,48,3", "22,8,2", "23,112,1",
                 "23,60,1"]  # variant,TX,CTAs per SM (19-23: shot-pair sweeps)


@pytest.fixture
def sweep_config(monkeypatch):
    def pin(cfg):
        if cfg:
            monkeypatch.setenv("FOMO_SWEEP_CONFIG", cfg)
        else:
            monkeypatch.delenv("FOMO_SWEEP_CONFIG", raising=False)
    return pin


def _vacuum_top(vp, *others):
    vp = vp.copy(order="F")
    vp[:, 0] = 0.0
    out = [vp]
    for o in others:
        o = o.copy(order="F")
        o[:, 0] = 0.0
        out.append(o)
    return out


# ---------------------------------------------------------------------------
def test_medium_preparation_bitwise(fomo, oracle):
    from fomo_b200.synthetic import layered_elastic

    vp, vs, rho = layered_elastic(37, 29, n_layers=5, seed=3)
    vp, vs, rho = _vacuum_top(vp, vs, rho)
    vs[5:9, 10:12] = 0.0  # fluid pocket: mu = 0 rules of elastic2d/medium.jl:64-66
    pad = 9
    got = fomo.debug_medium2d("elastic", vp, vs, rho, pad)
    want = oracle.medium2d("elastic", vp, vs, rho, pad)
    assert np.array_equal(got, want)
    got = fomo.debug_medium2d("acoustic", vp, None, rho, pad)
    want = oracle.medium2d("acoustic", vp, None, rho, pad)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("fd_order", [2, 4, 6, 8, 10])
@pytest.mark.parametrize("kernel", KERNELS)
def test_acoustic2d_bitwise_vs_oracle(fomo, oracle, fd_order, kernel):
    from fomo_b200.synthetic import two_layer

    vp, rho = two_layer(63, 47)
    vp, rho = _vacuum_top(vp, rho)
    nt, nbc = 160, 11
    rx = np.arange(1, 64, 3)
    rz = np.full(rx.size, 9)
    w = fomo.ricker_wavelet(15.0, 1e-3, nt)
    M = fd_order // 2
    fin = np.zeros((63 + 2 * (nbc + M), 47 + 2 * (nbc + M), 3), np.float32, order="F")
    r = fomo.acoustic2d(vp, rho, 10.0, 1e-3, nt, 15.0, sx=[31], sz=[10], rx=rx, rz=rz, nbc=nbc,
                        fd_order=fd_order, snap_interval=40, kernel=kernel, final_state=fin)
    o = oracle.acoustic2d(vp, rho, 10.0, 1e-3, nt, sx=[31], sz=[10], rx=rx, rz=rz,
                          wavelet=w.reshape(1, -1), nbc=nbc, fd_order=fd_order, snap_interval=40,
                          final=True)
    assert np.array_equal(r.seis_p, o["seis_p"][:, :, 0])
    assert np.array_equal(r.seis_vx, o["seis_vx"][:, :, 0])
    assert np.array_equal(r.seis_vz, o["seis_vz"][:, :, 0])
    assert len(r.snaps) == 4
    for k in range(4):
        assert np.array_equal(r.snaps[k], o["snaps"][:, :, k, 0])
    assert np.array_equal(fin, o["final"][:, :, :, 0])
    o64 = oracle.acoustic2d(vp, rho, 10.0, 1e-3, nt, sx=[31], sz=[10], rx=rx, rz=rz,
                            wavelet=w.reshape(1, -1), nbc=nbc, fd_order=fd_order, prec=64)
    assert rel_l2(r.seis_p, o64["seis_p"][:, :, 0]) < 1e-5


@pytest.mark.parametrize("fd_order", [4, 8, 10])
@pytest.mark.parametrize("kernel", KERNELS)
def test_elastic2d_bitwise_vs_oracle(fomo, oracle, fd_order, kernel):
    from fomo_b200.synthetic import layered_elastic

    vp, vs, rho = layered_elastic(71, 53, n_layers=4, seed=9)
    vp, vs, rho = _vacuum_top(vp, vs, rho)
    nt, nbc = 200, 10
    rx = np.arange(2, 71, 2)
    rz = np.full(rx.size, 6)
    w = fomo.ricker_wavelet(20.0, 5e-4, nt)
    M = fd_order // 2
    fin = np.zeros((71 + 2 * (nbc + M), 53 + 2 * (nbc + M), 5), np.float32, order="F")
    r = fomo.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, 20.0, sx=[35, 36], sz=[8, 8], rx=rx, rz=rz,
                       nbc=nbc, fd_order=fd_order, snap_interval=50, kernel=kernel,
                       final_state=fin)
    o = oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, sx=[[35], [36]], sz=[[8], [8]], rx=rx, rz=rz,
                         wavelet=np.repeat(w.reshape(1, -1), 2, axis=0), nbc=nbc,
                         fd_order=fd_order, snap_interval=50, final=True)
    assert np.array_equal(r.seis_vx, o["seis_vx"][:, :, 0])
    assert np.array_equal(r.seis_vz, o["seis_vz"][:, :, 0])
    for k in range(len(r.snaps)):
        assert np.array_equal(r.snaps[k], o["snaps"][:, :, k, 0])
    assert np.array_equal(fin, o["final"][:, :, :, 0])
    o64 = oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, sx=[[35], [36]], sz=[[8], [8]], rx=rx,
                           rz=rz, wavelet=np.repeat(w.reshape(1, -1), 2, axis=0), nbc=nbc,
                           fd_order=fd_order, prec=64)
    assert rel_l2(r.seis_vz, o64["seis_vz"][:, :, 0]) < 1e-5


@pytest.mark.parametrize("cfg", SWEEP_CONFIGS)
@pytest.mark.parametrize("fd_order", [2, 6, 10])
def test_elastic_single_sweep_configs_bitwise(fomo, oracle, sweep_config, cfg, fd_order):
    """Every strip width / z-segmentation of the single-sweep kernel, including
    segment boundaries inside the HABC bands, equals the oracle bit for bit."""
    from fomo_b200.synthetic import layered_elastic

    sweep_config(cfg)
    vp, vs, rho = layered_elastic(150, 131, n_layers=6, seed=12)
    vp, vs, rho = _vacuum_top(vp, vs, rho)
    nt, nbc = 140, 9
    rx = np.arange(1, 151, 7)
    rz = np.full(rx.size, 3)
    M = fd_order // 2
    fin = np.zeros((150 + 2 * (nbc + M), 131 + 2 * (nbc + M), 5, 2), np.float32, order="F")
    sx = np.array([[20], [131]])
    sz = np.array([[4], [120]])
    r = fomo.elastic2d_batch(vp, vs, rho, 5.0, 5e-4, nt, 20.0, sx=sx, sz=sz, rx=rx, rz=rz,
                             nbc=nbc, fd_order=fd_order, kernel=2, final_state=fin)
    w = fomo.ricker_wavelet(20.0, 5e-4, nt)
    o = oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, sx=sx.T, sz=sz.T, rx=rx, rz=rz,
                         wavelet=w.reshape(1, -1), nbc=nbc, fd_order=fd_order, n_shots=2,
                         final=True)
    assert np.array_equal(r.seis_vx, o["seis_vx"])
    assert np.array_equal(r.seis_vz, o["seis_vz"])
    assert np.array_equal(fin, o["final"])


@pytest.mark.parametrize("cfg", ["19,112,2", "21,40,2", "22,48,3", "20,8,1"])
def test_shot_pair_sweep_odd_batch_bitwise(fomo, oracle, sweep_config, cfg):
    """The shot-pair sweep on an odd batch (the last pair carries an all-zero
    shot) with coincident sources and a receiver on a source cell equals the
    oracle bit for bit, final wavefields included."""
    from fomo_b200.synthetic import layered_elastic

    sweep_config(cfg)
    vp, vs, rho = layered_elastic(97, 64, n_layers=5, seed=21)
    vp, vs, rho = _vacuum_top(vp, vs, rho)
    nt, nbc, fd_order = 150, 10, 8
    rx = np.array([1, 30, 48, 48, 97])
    rz = np.array([1, 7, 7, 64, 64])
    sx = np.array([[48, 48], [10, 11], [90, 30]])  # (n_shots, n_src)
    sz = np.array([[7, 7], [3, 60], [5, 5]])
    M = fd_order // 2
    fin = np.zeros((97 + 2 * (nbc + M), 64 + 2 * (nbc + M), 5, 3), np.float32, order="F")
    r = fomo.elastic2d_batch(vp, vs, rho, 5.0, 5e-4, nt, 20.0, sx=sx, sz=sz, rx=rx, rz=rz,
                             nbc=nbc, fd_order=fd_order, kernel=2, final_state=fin)
    w = fomo.ricker_wavelet(20.0, 5e-4, nt)
    o = oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, sx=sx.T, sz=sz.T, rx=rx, rz=rz,
                         wavelet=np.repeat(w.reshape(1, -1), 2, axis=0), nbc=nbc,
                         fd_order=fd_order, n_shots=3, final=True)
    assert np.array_equal(r.seis_vx, o["seis_vx"])
    assert np.array_equal(r.seis_vz, o["seis_vz"])
    assert np.array_equal(fin, o["final"])


@pytest.mark.parametrize("kernel", KERNELS)
def test_elastic2d_batch_bitwise_and_equals_single(fomo, oracle, kernel):
    from fomo_b200.synthetic import layered_elastic

    vp, vs, rho = layered_elastic(80, 50, n_layers=5, seed=4)
    nt = 180
    rx = np.arange(1, 81, 4)
    rz = np.full(rx.size, 5)
    sx = np.array([[10, 12], [40, 42], [70, 72]])  # (n_shots, n_src)
    sz = np.array([[5, 5], [6, 6], [7, 7]])
    r = fomo.elastic2d_batch(vp, vs, rho, 5.0, 5e-4, nt, 20.0, sx=sx, sz=sz, rx=rx, rz=rz,
                             nbc=9, fd_order=10, kernel=kernel)
    assert r.seis_vx.shape == (rx.size, nt, 3) and r.stats.n_shots == 3
    w = fomo.ricker_wavelet(20.0, 5e-4, nt)
    o = oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, sx=sx.T, sz=sz.T, rx=rx, rz=rz,
                         wavelet=np.repeat(w.reshape(1, -1), 2, axis=0), nbc=9, fd_order=10,
                         n_shots=3)
    assert np.array_equal(r.seis_vx, o["seis_vx"])
    assert np.array_equal(r.seis_vz, o["seis_vz"])
    for s in range(3):  # verify_batch.jl:116-151: batch == single, exactly
        one = fomo.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, 20.0, sx=list(sx[s]), sz=list(sz[s]),
                             rx=rx, rz=rz, nbc=9, fd_order=10, kernel=kernel)
        assert np.array_equal(one.seis_vx, r.seis_vx[:, :, s])
        assert np.array_equal(one.seis_vz, r.seis_vz[:, :, s])


@pytest.mark.parametrize("kernel", KERNELS)
def test_acoustic2d_batch_bitwise_and_equals_single(fomo, oracle, kernel):
    from fomo_b200.synthetic import two_layer

    vp, rho = two_layer(70, 44)
    nt = 150
    rx = np.arange(3, 70, 5)
    rz = np.full(rx.size, 4)
    sx = [15, 35, 55, 69]  # a vector = one source per shot (batch.jl:194)
    sz = [6, 6, 6, 44]
    r = fomo.acoustic2d_batch(vp, rho, 10.0, 1e-3, nt, 15.0, sx=sx, sz=sz, rx=rx, rz=rz,
                              nbc=8, fd_order=8, kernel=kernel)
    w = fomo.ricker_wavelet(15.0, 1e-3, nt)
    o = oracle.acoustic2d(vp, rho, 10.0, 1e-3, nt, sx=np.array([sx]), sz=np.array([sz]), rx=rx,
                          rz=rz, wavelet=w.reshape(1, -1), nbc=8, fd_order=8, n_shots=4)
    assert np.array_equal(r.seis_p, o["seis_p"])
    assert np.array_equal(r.seis_vx, o["seis_vx"])
    assert np.array_equal(r.seis_vz, o["seis_vz"])
    for s in range(4):
        one = fomo.acoustic2d(vp, rho, 10.0, 1e-3, nt, 15.0, sx=[sx[s]], sz=[sz[s]], rx=rx, rz=rz,
                              nbc=8, fd_order=8, kernel=kernel)
        assert np.array_equal(one.seis_p, r.seis_p[:, :, s])


@pytest.mark.parametrize("fd_order", [2, 6, 8, 10])
@pytest.mark.parametrize("source_scale", ["v2dt2", "dt", "none"])
def test_scalar2d_bitwise_vs_oracle(fomo, oracle, fd_order, source_scale):
    from fomo_b200.api import scalar_wavelet_matrix

    nx, nz, nt = 58, 41, 150
    vp = np.full((nx, nz), 3000.0, np.float32)
    vp[:, nz // 2 - 1:] = 3600.0
    rx = list(range(5, nx - 4, 6))
    rz = [4] * len(rx)
    fin = np.zeros((nx + 2 * (12 + fd_order // 2), nz + 2 * (12 + fd_order // 2), 2), np.float32,
                   order="F")
    r = fomo.scalar2d(vp, 10.0, 1e-3, nt, 15.0, sx=[29], sz=[8], rx=rx, rz=rz, nbc=12,
                      fd_order=fd_order, source_scale=source_scale, final_state=fin)
    wm = scalar_wavelet_matrix(fomo.ricker_wavelet(15.0, 1e-3, nt), vp, 1e-3, [29], [8],
                               source_scale)
    o = oracle.scalar2d(vp, 10.0, 1e-3, nt, sx=[29], sz=[8], rx=rx, rz=rz, wavelet=wm, nbc=12,
                        fd_order=fd_order, final=True)
    assert np.array_equal(r.seis_u, o["seis_u"])
    assert np.array_equal(fin, o["final"])


def test_rerun_is_bit_identical(fomo):
    """verify_det_graph.jl:152-185: the production loop run twice is bit-identical."""
    from fomo_b200.synthetic import layered_elastic

    vp, vs, rho = layered_elastic(90, 60, seed=8)
    kw = dict(sx=[[20], [60]], sz=[[5], [5]], rx=np.arange(1, 91, 2), rz=np.full(45, 5), nbc=10,
              fd_order=8)
    a = fomo.elastic2d_batch(vp, vs, rho, 5.0, 5e-4, 300, 20.0, **kw)
    b = fomo.elastic2d_batch(vp, vs, rho, 5.0, 5e-4, 300, 20.0, **kw)
    assert np.array_equal(a.seis_vx, b.seis_vx) and np.array_equal(a.seis_vz, b.seis_vz)


def test_custom_wavelet_equals_default_ricker(fomo):
    """verify_patch.jl:112-117: wavelet=ricker_wavelet(...) is bit-identical to the default."""
    from fomo_b200.synthetic import two_layer

    vp, rho = two_layer(50, 40)
    kw = dict(sx=[25], sz=[5], rx=np.arange(1, 51, 2), rz=np.full(25, 4), nbc=8, fd_order=4)
    r0 = fomo.acoustic2d(vp, rho, 10.0, 1e-3, 200, 10.0, **kw)
    r1 = fomo.acoustic2d(vp, rho, 10.0, 1e-3, 200, 10.0,
                         wavelet=fomo.ricker_wavelet(10.0, 1e-3, 200), **kw)
    assert np.array_equal(r0.seis_p, r1.seis_p)


def test_edge_geometry_coincident_sources_and_minimal_pad(fomo, oracle):
    """Receivers on the outermost interior cells, two sources on one cell
    (summed in source order), no absorbing layers beyond the stencil (nbc=0)."""
    from fomo_b200.synthetic import two_layer

    vp, rho = two_layer(30, 22)
    nt = 90
    rx = [1, 30, 1, 30, 15]
    rz = [1, 1, 22, 22, 11]
    w = fomo.ricker_wavelet(20.0, 1e-3, nt)
    for nbc, fd in [(0, 4), (1, 2), (3, 10)]:
        r = fomo.acoustic2d(vp, rho, 10.0, 1e-3, nt, 20.0, sx=[15, 15], sz=[11, 11], rx=rx, rz=rz,
                            nbc=nbc, fd_order=fd)
        o = oracle.acoustic2d(vp, rho, 10.0, 1e-3, nt, sx=[[15], [15]], sz=[[11], [11]], rx=rx,
                              rz=rz, wavelet=np.repeat(w.reshape(1, -1), 2, axis=0), nbc=nbc,
                              fd_order=fd)
        assert np.array_equal(r.seis_p, o["seis_p"][:, :, 0]), (nbc, fd)
        assert np.array_equal(r.seis_vz, o["seis_vz"][:, :, 0]), (nbc, fd)


def test_empty_receiver_spread(fomo):
    from fomo_b200.synthetic import two_layer

    vp, rho = two_layer(30, 20)
    r = fomo.acoustic2d(vp, rho, 10.0, 1e-3, 40, 15.0, sx=[10], sz=[5], rx=[], rz=[], nbc=5,
                        fd_order=4)
    assert r.seis_p.shape == (0, 40)


def test_kernel_time_reported(fomo):
    from fomo_b200.synthetic import two_layer

    vp, rho = two_layer(64, 48)
    r = fomo.acoustic2d(vp, rho, 10.0, 1e-3, 100, 15.0, sx=[30], sz=[5], rx=[10], rz=[5], nbc=8)
    assert r.stats.kernel_time_s > 0.0
