"""Seeded synthetic models and acquisition layouts for the benchmark configurations.

No public dataset is involved: every model is generated here from a seed, with
the shapes, sizes and value distributions the benchmark configurations state.
"""
from __future__ import annotations

import numpy as np


def gardner_rho(vp: np.ndarray) -> np.ndarray:
    """rho = 310 * vp^0.25 (test/verify_patch.jl:27-28), evaluated in float64."""
    return (310.0 * np.asarray(vp, dtype=np.float64) ** 0.25).astype(np.float32)


def layered_elastic(nx=1000, nz=500, n_layers=12, seed=2, vmin=1500.0, vmax=4500.0,
                    vp_vs=1.73):
    """Flat layers with boundaries at round(k*nz/n_layers); vp ~ U(vmin, vmax) per layer."""
    rng = np.random.default_rng(seed)
    v = rng.uniform(vmin, vmax, n_layers).astype(np.float32)
    vp = np.empty((nx, nz), dtype=np.float32, order="F")
    edges = [int(round(k * nz / n_layers)) for k in range(n_layers + 1)]
    for k in range(n_layers):
        vp[:, edges[k]:edges[k + 1]] = v[k]
    vs = np.asfortranarray((vp / np.float32(vp_vs)).astype(np.float32))
    return vp, vs, np.asfortranarray(gardner_rho(vp))


def elastic_batch_config(n_shots=32, nx=1000, nz=500):
    """Elastic batch workload: 32 shots, 1000x500, dh 5 m, dt 0.5 ms, nt 3000,
    order 10, nbc 80, sources evenly along z=5, 500 receivers at z=5, 20 Hz."""
    vp, vs, rho = layered_elastic(nx, nz)
    sx = np.array([int(round((s + 0.5) * nx / n_shots)) for s in range(n_shots)])
    sx = np.clip(sx, 1, nx)
    sz = np.full(n_shots, 5)
    rx = np.arange(1, nx, 2)
    rz = np.full(rx.size, 5)
    return dict(vp=vp, vs=vs, rho=rho, dh=5.0, dt=5e-4, nt=3000, f0=20.0, fd_order=10, nbc=80,
                sx=sx, sz=sz, rx=rx, rz=rz)


def acoustic_single_config():
    """Acoustic single-shot workload: 400x300, dh 10, dt 1 ms, nt 2000, nbc 100,
    order 8, vp 2500, rho 2000, vacuum top row, source (200,10), receivers every
    2nd x on z=10, 15 Hz, snapshots every 50 steps."""
    nx, nz = 400, 300
    vp = np.full((nx, nz), 2500.0, dtype=np.float32, order="F")
    rho = np.full((nx, nz), 2000.0, dtype=np.float32, order="F")
    vp[:, 0] = 0.0
    rho[:, 0] = 0.0
    rx = np.arange(1, nx + 1, 2)
    return dict(vp=vp, rho=rho, dh=10.0, dt=1e-3, nt=2000, f0=15.0, fd_order=8, nbc=100,
                sx=[200], sz=[10], rx=rx, rz=np.full(rx.size, 10), snap_interval=50)


def symmetric_model(nx: int, nz: int):
    """Curved interface plus a Gaussian anomaly, mirror-symmetric in x
    (test/verify_patch.jl:17-30)."""
    xc = (nx + 1) / 2
    vp = np.full((nx, nz), 2000.0, dtype=np.float32)
    for i in range(1, nx + 1):
        zint = 100 + int(np.round(20 * np.cos(2 * np.pi * (i - xc) / nx)))
        vp[i - 1, zint - 1:] = 3000.0
    xg = (np.arange(1, nx + 1) - xc) / 30
    zg = (np.arange(1, nz + 1) - 60) / 15
    g = np.exp(-(xg[:, None] ** 2 + zg[None, :] ** 2)).astype(np.float32)
    vp = (vp + np.float32(400.0) * g).astype(np.float32)
    vs = (vp / np.float32(1.73)).astype(np.float32)
    return np.asfortranarray(vp), np.asfortranarray(vs), np.asfortranarray(gardner_rho(vp))


def edge_extend(m: np.ndarray, L: int) -> np.ndarray:
    """Clamp-extend a model by L cells on every side (test/verify_patch.jl:33-37)."""
    ix = np.clip(np.arange(1, m.shape[0] + 2 * L + 1) - L, 1, m.shape[0]) - 1
    iz = np.clip(np.arange(1, m.shape[1] + 2 * L + 1) - L, 1, m.shape[1]) - 1
    return np.asfortranarray(m[np.ix_(ix, iz)])


def two_layer(nx: int, nz: int, v1=3000.0, v2=3800.0, rho=2200.0):
    """Two-layer acoustic model of test/verify_det_graph.jl:35-56."""
    vp = np.full((nx, nz), v1, dtype=np.float32, order="F")
    vp[:, nz // 2 - 1:] = v2
    return vp, np.full((nx, nz), rho, dtype=np.float32, order="F")


def grf2d(nx: int, nz: int, dh: float, mean: float, std: float, corr: float, seed: int,
          vmin: float, vmax: float) -> np.ndarray:
    """Gaussian random field: white noise -> FFT -> sqrt(Gaussian spectrum with
    correlation length corr) -> IFFT -> standardise -> mean + std*field -> clip."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((nx, nz))
    kx = np.fft.fftfreq(nx, d=dh) * 2 * np.pi
    kz = np.fft.fftfreq(nz, d=dh) * 2 * np.pi
    k2 = kx[:, None] ** 2 + kz[None, :] ** 2
    spec = np.exp(-k2 * corr * corr / 4.0)
    f = np.real(np.fft.ifft2(np.fft.fft2(w) * np.sqrt(spec)))
    f = (f - f.mean()) / (f.std() + 1e-30)
    return np.asfortranarray(np.clip(mean + std * f, vmin, vmax).astype(np.float32))


def grf3d(nx: int, ny: int, nz: int, dh: float, mean: float, std: float, corr: float, seed: int,
          vmin: float, vmax: float) -> np.ndarray:
    """3D Gaussian random field (the 2D recipe of grf2d over three axes)."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((nx, ny, nz)).astype(np.float32)
    k2 = None
    for ax, n in enumerate((nx, ny, nz)):
        k = (np.fft.fftfreq(n, d=dh) * 2 * np.pi).astype(np.float32)
        shape = [1, 1, 1]
        shape[ax] = n
        k = k.reshape(shape) ** 2
        k2 = k if k2 is None else k2 + k
    spec = np.sqrt(np.exp(-k2 * np.float32(corr * corr / 4.0)))
    f = np.real(np.fft.ifftn(np.fft.fftn(w) * spec)).astype(np.float32)
    f = (f - f.mean()) / (f.std() + 1e-30)
    return np.asfortranarray(np.clip(mean + std * f, vmin, vmax).astype(np.float32))


def elastic3d_config(nx=400, ny=400, nz=300, seed=4, vmax=5000.0):
    """Single-shot elastic 3D workload: 400x400x300, dh 10 m, dt 0.8 ms,
    nt 2500, order 8, nbc 40; vp a 3D Gaussian random field (mean 3200, std
    500, correlation 250 m) clipped to 1500..vmax so dt meets the 3D CFL bound,
    vs = vp/1.8, Gardner rho, vacuum top plane; 12 Hz source at the centre at
    z=10; 200x200 receiver grid (every 2nd x and y) at z=10."""
    vp = grf3d(nx, ny, nz, 10.0, 3200.0, 500.0, 250.0, seed, 1500.0, vmax)
    vs = np.asfortranarray((vp / np.float32(1.8)).astype(np.float32))
    rho = np.asfortranarray(gardner_rho(vp))
    for a in (vp, vs, rho):
        a[:, :, 0] = 0.0
    gx, gy = np.meshgrid(np.arange(1, nx + 1, 2), np.arange(1, ny + 1, 2), indexing="ij")
    rx, ry = gx.ravel(order="F"), gy.ravel(order="F")
    return dict(vp=vp, vs=vs, rho=rho, dh=10.0, dt=8e-4, nt=2500, f0=12.0, fd_order=8, nbc=40,
                sx=[nx // 2], sy=[ny // 2], sz=[10], rx=rx, ry=ry, rz=np.full(rx.size, 10))


def uneven_batch_config(n_shots=64, seed=3, nt=2000):
    """Uneven acoustic batch: n_shots grids with nx ~ logU(200, 2000), nz ~
    logU(200, 800) (seed), dh 10 m, order 8, nt 2000, dt 1 ms, nbc 50; per shot
    vp a Gaussian random field (mean 3000, std 600, correlation 300 m, clipped
    to 1500..5000, seed+s), rho 2000; source (nx//2, 10), receivers every 2nd x
    on z=10, 15 Hz."""
    rng = np.random.default_rng(seed)
    nxs = np.rint(np.exp(rng.uniform(np.log(200), np.log(2000), n_shots))).astype(int)
    nzs = np.rint(np.exp(rng.uniform(np.log(200), np.log(800), n_shots))).astype(int)
    vps, rhos, sx, sz, rx, rz = [], [], [], [], [], []
    for s in range(n_shots):
        nx, nz = int(nxs[s]), int(nzs[s])
        vps.append(grf2d(nx, nz, 10.0, 3000.0, 600.0, 300.0, seed + s, 1500.0, 5000.0))
        rhos.append(np.full((nx, nz), 2000.0, dtype=np.float32, order="F"))
        sx.append(nx // 2)
        sz.append(10)
        r = np.arange(1, nx + 1, 2)
        rx.append(r)
        rz.append(np.full(r.size, 10))
    return dict(vps=vps, rhos=rhos, dh=10.0, dt=1e-3, nt=nt, f0=15.0, fd_order=8, nbc=50,
                sx=sx, sz=sz, rx=rx, rz=rz)
