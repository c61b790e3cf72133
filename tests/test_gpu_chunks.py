"""Acoustic runs replay captured chunks of time steps (CUDA graphs with a device
step index); the results must equal step-by-step launches bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture
def step_launch(monkeypatch, fomo):
    """Calls made through this fixture's function launch every step from the host."""
    from fomo_b200 import _lib as L

    orig = fomo.api._opts

    def run(fn, *a, **kw):
        def opts(*oa, **okw):
            o = orig(*oa, **okw)
            o.flags |= L.FOMO_F_STEP_LAUNCH
            return o

        monkeypatch.setattr(fomo.api, "_opts", opts)
        try:
            return fn(*a, **kw)
        finally:
            monkeypatch.setattr(fomo.api, "_opts", orig)

    return run


def _model():
    from fomo_b200.synthetic import two_layer

    vp, rho = two_layer(90, 60)
    vp = vp.copy(order="F")
    vp[:, 0] = 0.0
    rho = rho.copy(order="F")
    rho[:, 0] = 0.0
    return vp, rho


def test_acoustic2d_chunks_equal_step_launches(fomo, step_launch):
    """Snapshots every 50 steps, 230 steps: four replayed 50-step chunks and a
    30-step remainder launched step by step."""
    vp, rho = _model()
    nt, nbc, order = 230, 12, 8
    rx = np.arange(1, 91, 3)
    rz = np.full(rx.size, 8)
    kw = dict(sx=[45], sz=[10], rx=rx, rz=rz, nbc=nbc, fd_order=order, snap_interval=50)
    shape = (90 + 2 * (nbc + 4), 60 + 2 * (nbc + 4), 3)
    fa = np.zeros(shape, np.float32, order="F")
    fb = np.zeros(shape, np.float32, order="F")
    a = fomo.acoustic2d(vp, rho, 10.0, 1e-3, nt, 15.0, final_state=fa, **kw)
    la = fomo.api.last_stats.gpu_launches
    b = step_launch(fomo.acoustic2d, vp, rho, 10.0, 1e-3, nt, 15.0, final_state=fb, **kw)
    lb = fomo.api.last_stats.gpu_launches
    for x, y in ((a.seis_p, b.seis_p), (a.seis_vx, b.seis_vx), (a.seis_vz, b.seis_vz)):
        assert np.array_equal(x, y)
    assert len(a.snaps) == len(b.snaps) == 4
    for x, y in zip(a.snaps, b.snaps):
        assert np.array_equal(x, y)
    assert np.array_equal(fa, fb)
    assert np.abs(a.seis_p).max() > 0
    # per chunk the replay adds a snapshot kernel and the step-index node (the
    # step-by-step path copies snapshots with cudaMemcpy2DAsync)
    assert la == lb + 8


def test_acoustic2d_streamed_snapshots_with_remainder(fomo, step_launch):
    """Snapshots every 40 steps, 290 steps: three replayed 80-step chunks whose six
    frames are copied out while later chunks run, and a 50-step remainder holding
    the seventh frame."""
    vp, rho = _model()
    kw = dict(sx=[45], sz=[10], rx=np.arange(1, 91, 4), rz=np.full(23, 8), nbc=10, fd_order=8,
              snap_interval=40)
    a = fomo.acoustic2d(vp, rho, 10.0, 1e-3, 290, 15.0, **kw)
    b = step_launch(fomo.acoustic2d, vp, rho, 10.0, 1e-3, 290, 15.0, **kw)
    assert len(a.snaps) == len(b.snaps) == 7
    for x, y in zip(a.snaps, b.snaps):
        assert np.array_equal(x, y)
    assert np.array_equal(a.seis_p, b.seis_p)
    assert all(np.abs(x).max() > 0 for x in a.snaps)


def test_acoustic2d_batch_chunks_equal_step_launches(fomo, step_launch):
    """Two shots, no snapshots, 200 steps: three 64-step chunks and 8 single steps."""
    vp, rho = _model()
    nt = 200
    rx = np.arange(1, 91, 4)
    rz = np.full(rx.size, 6)
    kw = dict(sx=[[20], [70]], sz=[[10], [30]], rx=rx, rz=rz, nbc=10, fd_order=6)
    a = fomo.acoustic2d_batch(vp, rho, 10.0, 1e-3, nt, 15.0, **kw)
    b = step_launch(fomo.acoustic2d_batch, vp, rho, 10.0, 1e-3, nt, 15.0, **kw)
    for x, y in ((a.seis_p, b.seis_p), (a.seis_vx, b.seis_vx), (a.seis_vz, b.seis_vz)):
        assert np.array_equal(x, y)
    assert not np.array_equal(a.seis_p[:, :, 0], a.seis_p[:, :, 1])


def test_acoustic2d_chunks_on_legacy_default_stream(fomo):
    """The chunk is captured on the context's own stream, so a context that
    borrows the legacy default stream (torch's default) still replays it."""
    import torch

    from fomo_b200 import _lib as L

    vp, rho = _model()
    kw = dict(sx=[45], sz=[10], rx=np.arange(1, 91, 5), rz=np.full(18, 8), nbc=10, fd_order=8)
    ctx = L.context(0)
    ctx.use_torch_stream(torch.cuda.current_stream())
    try:
        a = fomo.acoustic2d(vp, rho, 10.0, 1e-3, 150, 15.0, **kw)
    finally:
        ctx.set_stream(None)
    b = fomo.acoustic2d(vp, rho, 10.0, 1e-3, 150, 15.0, **kw)
    assert np.array_equal(a.seis_p, b.seis_p)
    assert np.array_equal(a.seis_vz, b.seis_vz)


def test_scalar2d_chunks_equal_step_launches(fomo, step_launch):
    """scalar2d rotates three buffers: 200 steps are three 63-step chunks and
    11 single steps."""
    from fomo_b200.synthetic import two_layer

    vp, _ = two_layer(80, 50)
    rx = np.arange(1, 81, 3)
    kw = dict(sx=[40], sz=[12], rx=rx, rz=np.full(rx.size, 6), nbc=10, fd_order=8)
    a = fomo.scalar2d(vp, 10.0, 1e-3, 200, 15.0, **kw)
    b = step_launch(fomo.scalar2d, vp, 10.0, 1e-3, 200, 15.0, **kw)
    assert np.array_equal(a.seis_u, b.seis_u)
    assert np.abs(a.seis_u).max() > 0


def test_elastic2d_two_phase_chunks_equal_step_launches(fomo, step_launch):
    """Two-phase elastic2d with vz snapshots every 40 steps, 190 steps: two
    80-step chunks and 30 single steps."""
    from fomo_b200.synthetic import layered_elastic

    vp, vs, rho = layered_elastic(70, 50, n_layers=4, seed=5)
    rx = np.arange(1, 71, 3)
    kw = dict(sx=[35], sz=[6], rx=rx, rz=np.full(rx.size, 5), nbc=10, fd_order=8,
              snap_interval=40, kernel=1)
    a = fomo.elastic2d(vp, vs, rho, 5.0, 5e-4, 190, 20.0, **kw)
    b = step_launch(fomo.elastic2d, vp, vs, rho, 5.0, 5e-4, 190, 20.0, **kw)
    assert np.array_equal(a.seis_vx, b.seis_vx)
    assert np.array_equal(a.seis_vz, b.seis_vz)
    assert len(a.snaps) == 4
    for x, y in zip(a.snaps, b.snaps):
        assert np.array_equal(x, y)
    assert np.abs(a.seis_vz).max() > 0


@pytest.mark.parametrize("launch", ["chunks", "steps"])
def test_single_shot_tagged_cells_vs_oracle(fomo, oracle, step_launch, launch):
    """Single-shot two-phase runs inject and record inside the last update
    kernel of a step: coincident sources add in source order and receivers on
    source cells see the injected value, as in the oracle."""
    from fomo_b200.synthetic import layered_elastic

    run = (lambda f, *a, **k: f(*a, **k)) if launch == "chunks" else step_launch
    vp, rho = _model()
    rx = np.concatenate([np.arange(1, 91, 7), [20, 20, 60]])
    rz = np.concatenate([np.full(13, 8), [10, 10, 25]])
    kw = dict(sx=[20, 60, 20], sz=[10, 25, 10], rx=rx, rz=rz, nbc=10, fd_order=8,
              snap_interval=40)
    nt = 170
    w = fomo.ricker_wavelet(15.0, 1e-3, nt)
    a = run(fomo.acoustic2d, vp, rho, 10.0, 1e-3, nt, 15.0, **kw)
    o = oracle.acoustic2d(vp, rho, 10.0, 1e-3, nt, wavelet=np.repeat(w[None], 3, axis=0), **kw)
    for x, y in ((a.seis_p, o["seis_p"]), (a.seis_vx, o["seis_vx"]), (a.seis_vz, o["seis_vz"])):
        assert np.array_equal(x, y[:, :, 0])
    for k, s in enumerate(a.snaps):
        assert np.array_equal(s, o["snaps"][:, :, k, 0])
    vp, vs, rho = layered_elastic(90, 60, n_layers=3, seed=8)
    we = fomo.ricker_wavelet(20.0, 5e-4, nt)
    e = run(fomo.elastic2d, vp, vs, rho, 5.0, 5e-4, nt, 20.0, kernel=1, **kw)
    oe = oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, wavelet=np.repeat(we[None], 3, axis=0), **kw)
    assert np.array_equal(e.seis_vx, oe["seis_vx"][:, :, 0])
    assert np.array_equal(e.seis_vz, oe["seis_vz"][:, :, 0])
    kws = {k: v for k, v in kw.items() if k != "snap_interval"}
    u = run(fomo.scalar2d, vp, 5.0, 5e-4, nt, 20.0, source_scale="none", **kws)
    ou = oracle.scalar2d(vp, 5.0, 5e-4, nt, wavelet=np.repeat(we[None], 3, axis=0), **kws)
    su = ou["seis_u"] if ou["seis_u"].ndim == 2 else ou["seis_u"][:, :, 0]
    assert np.array_equal(u.seis_u, su)
    assert np.abs(u.seis_u).max() > 0


@pytest.mark.parametrize("kernel", [1, 2])
def test_streamed_seismograms_vs_oracle(fomo, oracle, kernel):
    """Step-by-step runs copy the seismograms in 128-step blocks while the loop
    runs (two shots: one strided copy per block and component); 400 steps give
    three streamed blocks and a 16-step remainder."""
    from fomo_b200.synthetic import layered_elastic

    vp, vs, rho = layered_elastic(60, 40, n_layers=3, seed=12)
    nt = 400
    rx = np.arange(1, 61, 4)
    rz = np.full(rx.size, 5)
    kw = dict(sx=[15, 45], sz=[5, 8], rx=rx, rz=rz, nbc=8, fd_order=8)
    r = fomo.elastic2d_batch(vp, vs, rho, 5.0, 5e-4, nt, 20.0, kernel=kernel, **kw)
    w = fomo.ricker_wavelet(20.0, 5e-4, nt)
    o = oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, wavelet=w[None], n_shots=2, **kw)
    assert np.array_equal(r.seis_vx, o["seis_vx"])
    assert np.array_equal(r.seis_vz, o["seis_vz"])
    assert np.abs(r.seis_vz[:, -1, :]).max() > 0


@pytest.mark.parametrize("launch", ["chunks", "steps"])
def test_batch_tagged_cells_vs_oracle(fomo, oracle, step_launch, launch):
    """Batches inject and record on one shared tag plane: shot 0 has two
    coincident sources, shot 1 a source on the same cell, and a receiver sits
    there; each shot applies only its own sources."""
    from fomo_b200.synthetic import layered_elastic

    run = (lambda f, *a, **k: f(*a, **k)) if launch == "chunks" else step_launch
    vp, rho = _model()
    nt = 160
    rx = np.concatenate([np.arange(1, 91, 9), [20]])
    rz = np.concatenate([np.full(10, 8), [10]])
    kw = dict(sx=[[20, 20], [20, 60]], sz=[[10, 10], [10, 25]], rx=rx, rz=rz, nbc=10,
              fd_order=8)
    w = fomo.ricker_wavelet(15.0, 1e-3, nt)
    a = run(fomo.acoustic2d_batch, vp, rho, 10.0, 1e-3, nt, 15.0, **kw)
    okw = dict(kw, sx=np.array(kw["sx"]).T, sz=np.array(kw["sz"]).T)
    o = oracle.acoustic2d(vp, rho, 10.0, 1e-3, nt, wavelet=np.repeat(w[None], 2, axis=0),
                          n_shots=2, **okw)
    for x, y in ((a.seis_p, o["seis_p"]), (a.seis_vx, o["seis_vx"]), (a.seis_vz, o["seis_vz"])):
        assert np.array_equal(x, y)
    assert not np.array_equal(a.seis_p[:, :, 0], a.seis_p[:, :, 1])
    vp, vs, rho = layered_elastic(90, 60, n_layers=3, seed=8)
    we = fomo.ricker_wavelet(20.0, 5e-4, nt)
    e = run(fomo.elastic2d_batch, vp, vs, rho, 5.0, 5e-4, nt, 20.0, kernel=1, **kw)
    oe = oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, wavelet=np.repeat(we[None], 2, axis=0),
                          n_shots=2, **okw)
    assert np.array_equal(e.seis_vx, oe["seis_vx"])
    assert np.array_equal(e.seis_vz, oe["seis_vz"])
