"""GPU parity on the headline workload's own geometry.

elastic2d_batch at the benchmark's full grid and settings -- 1000x500
(padded 1170x670), dh 5 m, dt 0.5 ms, fd_order 10, nbc 80, the 12 seeded
Gardner layers, receivers every 2nd x at z=5, 20 Hz Ricker -- for two of its
32 shots (the first and the middle source) over the first 300 of its 3000
time steps, on the production single-sweep kernels.  Seismogram sample k of
a run depends only on steps 1..k, so these samples are the first 300 of the
full run's.

Bar: bit-identical to the FP32 oracle, and within 1e-5 relative L2 of the
FP64 oracle (the error every result states).
"""
import warnings

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

NT = 300
SHOTS = [0, 16]  # first and middle source of the 32-shot layout


@pytest.fixture(scope="module")
def headline(oracle):
    from fomo_b200 import ricker_wavelet
    from fomo_b200.synthetic import elastic_batch_config

    cfg = elastic_batch_config(32)
    sx = cfg["sx"][SHOTS].reshape(-1, 1)
    sz = cfg["sz"][SHOTS].reshape(-1, 1)
    w = ricker_wavelet(cfg["f0"], cfg["dt"], NT).reshape(1, -1)
    kw = dict(sx=sx.T, sz=sz.T, rx=cfg["rx"], rz=cfg["rz"], wavelet=w, nbc=cfg["nbc"],
              fd_order=cfg["fd_order"], n_shots=len(SHOTS))
    o32 = oracle.elastic2d(cfg["vp"], cfg["vs"], cfg["rho"], cfg["dh"], cfg["dt"], NT, **kw)
    o64 = oracle.elastic2d(cfg["vp"], cfg["vs"], cfg["rho"], cfg["dh"], cfg["dt"], NT, prec=64,
                           **kw)
    return cfg, sx, sz, o32, o64


# None: the autotuner's pick; then the shot-pair sweep and the one-shot
# warp-specialized sweep pinned (variant, strip width, CTAs per SM); "replica":
# the CUDA C++ replica of the reference's CUDA.jl step (FOMO_KERNEL_REPLICA)
@pytest.mark.parametrize("cfg_pin", [None, "19,112,2", "14,112,4", "replica"])
def test_headline_geometry_bitwise_and_fp64_error(fomo, headline, monkeypatch, cfg_pin):
    cfg, sx, sz, o32, o64 = headline
    if cfg_pin and cfg_pin != "replica":
        monkeypatch.setenv("FOMO_SWEEP_CONFIG", cfg_pin)
    else:
        monkeypatch.delenv("FOMO_SWEEP_CONFIG", raising=False)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")  # the layout is below 4 points per wavelength by design
        r = fomo.elastic2d_batch(cfg["vp"], cfg["vs"], cfg["rho"], cfg["dh"], cfg["dt"], NT,
                                 cfg["f0"], sx=sx, sz=sz, rx=cfg["rx"], rz=cfg["rz"],
                                 nbc=cfg["nbc"], fd_order=cfg["fd_order"],
                                 kernel=4 if cfg_pin == "replica" else 2)
    assert np.isfinite(r.seis_vz).all() and np.abs(r.seis_vz).max() > 0.0
    assert np.array_equal(r.seis_vx, o32["seis_vx"])
    assert np.array_equal(r.seis_vz, o32["seis_vz"])
    for comp in ("seis_vx", "seis_vz"):
        for s in range(len(SHOTS)):
            err = rel_l2(getattr(r, comp)[:, :, s], o64[comp][:, :, s])
            assert err <= 1e-5, (comp, s, err)
