"""Fomo.jl's public solvers over libfomo_b200 (same names, keywords, errors, results).

Each function validates its inputs exactly where the Julia reference does
(utils/checks.jl), builds the wavelet matrix as the reference's L5 code does,
then calls one C-ABI entry point; all stepping happens in the CUDA library.
Arrays follow the reference: models are ``(nx, nz)`` with x first, indices
1-based, seismograms ``(n_rec, nt[, n_shots])``.
"""
from __future__ import annotations

import ctypes as C
import warnings
from typing import NamedTuple, Optional, Sequence

import numpy as np

from . import _lib as L

__all__ = [
    "ArgumentError", "acoustic2d", "acoustic2d_batch", "elastic2d", "elastic2d_batch",
    "scalar2d", "acoustic3d", "elastic3d", "acoustic2d_uneven", "ricker_wavelet",
    "get_fd_coefficients",
    "get_centered_d2",
]


class ArgumentError(ValueError):
    """Invalid input, raised before any launch (Julia's ArgumentError)."""


# The library's fomo_stats of the most recent solver call in this process
# (kernel time, cell updates, algorithmic bytes, launches): diagnostics beyond
# the reference's result fields.
last_stats = None


def _remember(st):
    global last_stats
    last_stats = st
    return st


# utils/FD_utils.jl:5-11 (Float32 values of the reference's literals)
_FD = {
    2: [1.0],
    4: [1.125, -0.041666667],
    6: [1.171875, -0.065104167, 0.0046875],
    8: [1.1962890625, -0.079752604167, 0.0095703125, -0.000697544643],
    10: [1.2115478515625, -0.089721679687, 0.0138427734375, -0.00176565987723, 0.0001186795166],
}
# utils/FD_centered.jl:27-41
_D2C0 = {2: -2.0, 4: -5 / 2, 6: -49 / 18, 8: -205 / 72, 10: -5269 / 1800}
_D2 = {
    2: [1.0], 4: [4 / 3, -1 / 12], 6: [3 / 2, -3 / 20, 1 / 90],
    8: [8 / 5, -1 / 5, 8 / 315, -1 / 560], 10: [5 / 3, -5 / 21, 5 / 126, -5 / 1008, 1 / 3150],
}


def get_fd_coefficients(order: int) -> np.ndarray:
    if order not in _FD:
        raise ValueError(f"Unsupported FD order: {order}")
    return np.asarray(_FD[order], dtype=np.float64).astype(np.float32)


def get_centered_d2(order: int):
    if order not in _D2:
        raise ValueError(f"Unsupported FD order: {order} (centered d2)")
    return np.float32(_D2C0[order]), np.asarray(_D2[order], dtype=np.float64).astype(np.float32)


def ricker_wavelet(f0, dt, nt) -> np.ndarray:
    """Ricker wavelet (utils/ricker_wavelet.jl:6-12) in the reference's Float32 arithmetic.

    With f0 and dt Float32, as the public functions pass them, the reference
    evaluates: t = (0:nt-1) .* dt (a Float32 range: each element is the exact
    product rounded once), t0 = 1f0/f0, tau = t - 1.5f0*t0, x = Float32(pi)*f0*tau
    and (1 - 2x^2) * exp(-x^2), every operation rounded to Float32.  The
    exponential is the platform's single-precision exp (numpy's), which may
    differ from Julia's Float32 exp by an ulp on some samples.
    """
    f0 = np.float32(f0)
    dt = np.float32(dt)
    t = (np.arange(int(nt), dtype=np.float64) * np.float64(dt)).astype(np.float32)
    t0 = np.float32(1.0) / f0
    tau = t - np.float32(1.5) * t0
    x = (np.float32(np.pi) * f0) * tau
    a = x * x
    with np.errstate(under="ignore"):
        return ((np.float32(1.0) - np.float32(2.0) * a) * np.exp(-a)).astype(np.float32)


class Stats(NamedTuple):
    kernel_time_s: float


class BatchStats(NamedTuple):
    kernel_time_s: float
    n_shots: int


class Acoustic2DResult(NamedTuple):
    seis_p: np.ndarray
    seis_vx: np.ndarray
    seis_vz: np.ndarray
    snaps: list
    stats: Stats


class Elastic2DResult(NamedTuple):
    seis_vx: np.ndarray
    seis_vz: np.ndarray
    snaps: list
    stats: Stats


class Acoustic2DBatchResult(NamedTuple):
    seis_p: np.ndarray
    seis_vx: np.ndarray
    seis_vz: np.ndarray
    stats: BatchStats


class Elastic2DBatchResult(NamedTuple):
    seis_vx: np.ndarray
    seis_vz: np.ndarray
    stats: BatchStats


class Coupled2DResult(NamedTuple):
    """coupled2d's NamedTuple (coupled2d.jl:165-170)."""
    seis_P: np.ndarray
    seis_S: np.ndarray
    snaps_P: list
    snaps_S: list
    stats: Stats


class Scalar2DResult(NamedTuple):
    seis_u: np.ndarray
    stats: Stats


# ---------------------------------------------------------------------------
# checks (utils/checks.jl)
# ---------------------------------------------------------------------------
def _check_geometry(nx, nz, sx, sz, rx, rz):
    sx, sz, rx, rz = (np.asarray(a).ravel() for a in (sx, sz, rx, rz))
    if not (np.all((1 <= sx) & (sx <= nx)) and np.all((1 <= sz) & (sz <= nz))):
        raise ArgumentError(f"source index out of range: need 1 <= sx <= {nx}, 1 <= sz <= {nz}")
    if not (np.all((1 <= rx) & (rx <= nx)) and np.all((1 <= rz) & (rz <= nz))):
        raise ArgumentError(f"receiver index out of range: need 1 <= rx <= {nx}, 1 <= rz <= {nz}")


def _warn_dispersion(vmin_disp, f0, dh, ppw_min=4.0):
    fmax = np.float32(2.5) * np.float32(f0)
    ppw = float(vmin_disp) / float(fmax) / float(dh)
    if ppw < ppw_min:
        warnings.warn(f"dispersion risk: shortest wavelength has only {ppw:.1f} grid points "
                      f"(vmin={vmin_disp}, fmax~{float(fmax):.1f} Hz); reduce dh or f0",
                      stacklevel=3)


def _check_numerics(vmax, vmin_disp, dh, dt, f0, fd_order, centered=False):
    if fd_order not in _FD:
        raise ValueError(f"Unsupported FD order: {fd_order}")
    dmax = C.c_float()
    rc = L.lib().fomo_check_numerics(float(vmax), float(dh), float(dt), int(fd_order),
                                     1 if centered else 0, C.byref(dmax))
    if rc != L.FOMO_OK:
        kind = "CFL unstable (centered)" if centered else "CFL unstable"
        raise ArgumentError(f"{kind}: dt={dt} > dt_max={dmax.value:.4g} "
                            f"(vmax={vmax}, dh={dh}, fd_order={fd_order})")
    _warn_dispersion(vmin_disp, f0, dh)


def _min_pos(a) -> np.float32:
    """minimum(vp[vp .> 0]): scanned in memory order, in chunks (a boolean index
    of a column-major volume would walk it in row-major order)."""
    flat = np.asarray(a, dtype=np.float32).ravel(order="K")
    best = np.float32(np.inf)
    step = 1 << 22
    for i in range(0, flat.size, step):
        c = flat[i:i + step]
        c = c[c > 0]
        if c.size:
            best = min(best, np.float32(c.min()))
    if not np.isfinite(best):
        raise ArgumentError("model has no positive velocity")
    return np.float32(best)


def _f32F(a) -> np.ndarray:
    return np.asfortranarray(np.asarray(a, dtype=np.float32))


def _i32F(a) -> np.ndarray:
    return np.asfortranarray(np.asarray(a, dtype=np.int32))


def _ptr(a) -> Optional[int]:
    return None if a is None else a.ctypes.data


def _wavelet_row(wavelet, f0, dt, nt) -> np.ndarray:
    w = ricker_wavelet(f0, dt, nt) if wavelet is None else np.asarray(wavelet, dtype=np.float32).ravel()
    if w.size != nt:
        raise ArgumentError(f"wavelet length {w.size} != nt={nt}")
    return w


def _precision(p) -> int:
    key = str(p).lower().lstrip(":")
    table = {"fp32": L.FOMO_FP32, "float32": L.FOMO_FP32, "fp16": L.FOMO_FP16,
             "float16": L.FOMO_FP16, "bf16": L.FOMO_BF16, "bfloat16": L.FOMO_BF16}
    if key not in table:
        raise ArgumentError(f"precision must be fp32, fp16 or bf16, got {p}")
    return table[key]


def _opts(kernel: int = 0, final_state: Optional[np.ndarray] = None, precision: int = 0,
          sponge_factor=None):
    """``sponge_factor`` not None selects boundary=:sponge with that Cerjan factor."""
    o = L.Opts()
    o.flags = 0
    o.precision = precision
    o.kernel = kernel
    o.check_every = 0
    o.final_state = _ptr(final_state)
    o.sponge_factor = 0.0
    if sponge_factor is not None:
        o.flags |= L.FOMO_F_SPONGE
        o.sponge_factor = float(np.float32(sponge_factor))
    return o


def _grid(nx, nz, dh, dt, nt, nbc, fd_order, v_ref) -> L.Grid2D:
    return L.Grid2D(int(nx), int(nz), float(dh), float(dt), int(nt), int(nbc), int(fd_order),
                    float(v_ref))


def _acq(sxm: np.ndarray, szm: np.ndarray, wm: np.ndarray, rx: np.ndarray, rz: np.ndarray):
    n_src, ns = sxm.shape
    return L.Acq(ns, n_src, _ptr(sxm), _ptr(szm), _ptr(wm), rx.size, _ptr(rx), _ptr(rz))


def _check_boundary(boundary) -> bool:
    """acoustic2d.jl:65-66 / elastic2d.jl:63-64; True for the Cerjan sponge."""
    b = str(boundary).lstrip(":")
    if b not in ("habc", "sponge"):
        raise ArgumentError(f"boundary must be :habc or :sponge, got {boundary}")
    return b == "sponge"


def _snap_list(snaps: Optional[np.ndarray]) -> list:
    if snaps is None:
        return []
    return [np.asfortranarray(snaps[:, :, k]) for k in range(snaps.shape[2])]


# ---------------------------------------------------------------------------
# acoustic2d / elastic2d (single shot, n_src sources firing together)
# ---------------------------------------------------------------------------
def acoustic2d(vp, rho, dh, dt, nt, f0, *, sx: Sequence[int], sz: Sequence[int], rx, rz,
               nbc: int = 50, fd_order: int = 8, snap_interval: int = 0, boundary="habc",
               v_ref=None, sponge_factor=0.015, wavelet=None, scale_source_by_dt: bool = False,
               use_cuda_graph: bool = True, verbose: bool = True, device: int = 0,
               kernel: int = 0, final_state: Optional[np.ndarray] = None) -> Acoustic2DResult:
    """2D acoustic velocity-pressure simulation (equations/acoustic2d/acoustic2d.jl:47-192).

    ``boundary="sponge"`` runs the Cerjan layer of the user's ``nbc`` cells with
    ``sponge_factor`` (boundary/sponge.jl); ``v_ref`` is then ignored."""
    sponge = _check_boundary(boundary)
    vp, rho = _f32F(vp), _f32F(rho)
    nx, nz = vp.shape
    dh, dt, f0 = np.float32(dh), np.float32(dt), np.float32(f0)
    _check_geometry(nx, nz, sx, sz, rx, rz)
    _check_numerics(vp.max(), _min_pos(vp), dh, dt, f0, fd_order)
    v_ref = _min_pos(vp) if v_ref is None else np.float32(v_ref)
    w = _wavelet_row(wavelet, f0, dt, nt)
    sxv, szv = _i32F(sx).ravel(), _i32F(sz).ravel()
    if sxv.size != szv.size:
        raise ArgumentError("sx and sz lengths differ")
    wm = np.asfortranarray(np.repeat(w[None, :], sxv.size, axis=0))
    if scale_source_by_dt:
        wm = np.asfortranarray((wm * dt).astype(np.float32))
    rxv, rzv = _i32F(rx).ravel(), _i32F(rz).ravel()
    nrec = rxv.size
    seis = [np.zeros((nrec, nt), dtype=np.float32, order="F") for _ in range(3)]
    nsnap = nt // snap_interval if snap_interval > 0 else 0
    snaps = np.zeros((nx, nz, nsnap), dtype=np.float32, order="F") if nsnap else None
    st = L.Stats()
    ctx = L.context(device)
    g = _grid(nx, nz, dh, dt, nt, nbc, fd_order, v_ref)
    acq = _acq(sxv.reshape(-1, 1, order="F"), szv.reshape(-1, 1, order="F"), wm, rxv, rzv)
    o = _opts(kernel, final_state, sponge_factor=sponge_factor if sponge else None)
    ctx.check(L.lib().fomo_acoustic2d(ctx.handle, C.byref(g), _ptr(vp), _ptr(rho), C.byref(acq),
                                      int(snap_interval), _ptr(seis[0]), _ptr(seis[1]),
                                      _ptr(seis[2]), _ptr(snaps), C.byref(o), C.byref(st)))
    _remember(st)
    return Acoustic2DResult(seis[0], seis[1], seis[2], _snap_list(snaps), Stats(st.kernel_time_s))


def elastic2d(vp, vs, rho, dh, dt, nt, f0, *, sx: Sequence[int], sz: Sequence[int], rx, rz,
              nbc: int = 50, fd_order: int = 8, snap_interval: int = 0, boundary="habc",
              v_ref=None, sponge_factor=0.015, wavelet=None, scale_source_by_dt: bool = False,
              use_cuda_graph: bool = True, verbose: bool = True, device: int = 0,
              kernel: int = 0, final_state: Optional[np.ndarray] = None,
              precision="fp32") -> Elastic2DResult:
    """2D elastic velocity-stress simulation (equations/elastic2d/elastic2d.jl:45-163).

    ``boundary="sponge"`` as in :func:`acoustic2d` (FP32 storage only)."""
    sponge = _check_boundary(boundary)
    vp, vs, rho = _f32F(vp), _f32F(vs), _f32F(rho)
    nx, nz = vp.shape
    dh, dt, f0 = np.float32(dh), np.float32(dt), np.float32(f0)
    _check_geometry(nx, nz, sx, sz, rx, rz)
    vmin_disp = _min_pos(vs) if np.any(vs > 0) else _min_pos(vp)  # elastic2d.jl:69-71
    _check_numerics(vp.max(), vmin_disp, dh, dt, f0, fd_order)
    v_ref = _min_pos(vp) if v_ref is None else np.float32(v_ref)
    w = _wavelet_row(wavelet, f0, dt, nt)
    sxv, szv = _i32F(sx).ravel(), _i32F(sz).ravel()
    if sxv.size != szv.size:
        raise ArgumentError("sx and sz lengths differ")
    wm = np.asfortranarray(np.repeat(w[None, :], sxv.size, axis=0))
    if scale_source_by_dt:
        wm = np.asfortranarray((wm * dt).astype(np.float32))
    rxv, rzv = _i32F(rx).ravel(), _i32F(rz).ravel()
    nrec = rxv.size
    seis = [np.zeros((nrec, nt), dtype=np.float32, order="F") for _ in range(2)]
    nsnap = nt // snap_interval if snap_interval > 0 else 0
    snaps = np.zeros((nx, nz, nsnap), dtype=np.float32, order="F") if nsnap else None
    st = L.Stats()
    ctx = L.context(device)
    g = _grid(nx, nz, dh, dt, nt, nbc, fd_order, v_ref)
    acq = _acq(sxv.reshape(-1, 1, order="F"), szv.reshape(-1, 1, order="F"), wm, rxv, rzv)
    o = _opts(kernel, final_state, _precision(precision),
              sponge_factor=sponge_factor if sponge else None)
    ctx.check(L.lib().fomo_elastic2d(ctx.handle, C.byref(g), _ptr(vp), _ptr(vs), _ptr(rho),
                                     C.byref(acq), int(snap_interval), _ptr(seis[0]),
                                     _ptr(seis[1]), _ptr(snaps), C.byref(o), C.byref(st)))
    _remember(st)
    return Elastic2DResult(seis[0], seis[1], _snap_list(snaps), Stats(st.kernel_time_s))


# ---------------------------------------------------------------------------
# batch variants: sx/sz are (n_shots x n_src) (a vector = one source per shot)
# ---------------------------------------------------------------------------
def _shot_matrix(sx, sz):
    sxm = np.asarray(sx, dtype=np.int64)
    szm = np.asarray(sz, dtype=np.int64)
    if sxm.ndim == 1:
        sxm = sxm.reshape(-1, 1)
    if szm.ndim == 1:
        szm = szm.reshape(-1, 1)
    if sxm.shape != szm.shape:
        raise ArgumentError(f"sx and sz shapes differ: {sxm.shape} vs {szm.shape}")
    if sxm.shape[0] < 1:
        raise ArgumentError("at least 1 shot is required")
    return sxm, szm


def _batch_common(vp, dh, dt, nt, f0, sx, sz, rx, rz, fd_order, v_ref, wavelet,
                  scale_source_by_dt):
    nx, nz = vp.shape
    sxm, szm = _shot_matrix(sx, sz)
    ns, n_src = sxm.shape
    for s in range(ns):  # batch.jl:201-206
        _check_geometry(nx, nz, sxm[s], szm[s], rx, rz)
    _check_numerics(vp.max(), _min_pos(vp), dh, dt, f0, fd_order)
    v_ref = _min_pos(vp) if v_ref is None else np.float32(v_ref)
    w = _wavelet_row(wavelet, f0, dt, nt)
    wm = np.asfortranarray(np.repeat(w[None, :], n_src, axis=0))
    if scale_source_by_dt:
        wm = np.asfortranarray((wm * dt).astype(np.float32))
    # device layout (n_src, n_shots) (batch.jl:219-220)
    sxd, szd = _i32F(sxm.T), _i32F(szm.T)
    rxv, rzv = _i32F(rx).ravel(), _i32F(rz).ravel()
    return v_ref, wm, sxd, szd, rxv, rzv, ns


def acoustic2d_batch(vp, rho, dh, dt, nt, f0, *, sx, sz, rx, rz, nbc: int = 50,
                     fd_order: int = 8, v_ref=None, wavelet=None,
                     scale_source_by_dt: bool = False, verbose: bool = True, device: int = 0,
                     kernel: int = 0, final_state=None) -> Acoustic2DBatchResult:
    """Multi-shot acoustic run on one shared model (equations/acoustic2d/batch.jl:180-261)."""
    vp, rho = _f32F(vp), _f32F(rho)
    nx, nz = vp.shape
    dh, dt, f0 = np.float32(dh), np.float32(dt), np.float32(f0)
    v_ref, wm, sxd, szd, rxv, rzv, ns = _batch_common(vp, dh, dt, nt, f0, sx, sz, rx, rz,
                                                      fd_order, v_ref, wavelet, scale_source_by_dt)
    nrec = rxv.size
    seis = [np.zeros((nrec, nt, ns), dtype=np.float32, order="F") for _ in range(3)]
    st = L.Stats()
    ctx = L.context(device)
    g = _grid(nx, nz, dh, dt, nt, nbc, fd_order, v_ref)
    acq = _acq(sxd, szd, wm, rxv, rzv)
    o = _opts(kernel, final_state)
    ctx.check(L.lib().fomo_acoustic2d_batch(ctx.handle, C.byref(g), _ptr(vp), _ptr(rho),
                                            C.byref(acq), _ptr(seis[0]), _ptr(seis[1]),
                                            _ptr(seis[2]), C.byref(o), C.byref(st)))
    _remember(st)
    return Acoustic2DBatchResult(seis[0], seis[1], seis[2], BatchStats(st.kernel_time_s, ns))


def elastic2d_batch(vp, vs, rho, dh, dt, nt, f0, *, sx, sz, rx, rz, nbc: int = 50,
                    fd_order: int = 8, v_ref=None, wavelet=None,
                    scale_source_by_dt: bool = False, verbose: bool = True, device: int = 0,
                    kernel: int = 0, final_state=None, precision="fp32") -> Elastic2DBatchResult:
    """Multi-shot elastic run on one shared model (equations/elastic2d/batch.jl:197-261).

    ``precision="fp16"`` stores the wavefields in binary16 (FP32 arithmetic,
    FP32 storage in a 32-cell band at the grid edges); no reference
    counterpart."""
    vp, vs, rho = _f32F(vp), _f32F(vs), _f32F(rho)
    nx, nz = vp.shape
    dh, dt, f0 = np.float32(dh), np.float32(dt), np.float32(f0)
    v_ref, wm, sxd, szd, rxv, rzv, ns = _batch_common(vp, dh, dt, nt, f0, sx, sz, rx, rz,
                                                      fd_order, v_ref, wavelet, scale_source_by_dt)
    nrec = rxv.size
    seis = [np.zeros((nrec, nt, ns), dtype=np.float32, order="F") for _ in range(2)]
    st = L.Stats()
    ctx = L.context(device)
    g = _grid(nx, nz, dh, dt, nt, nbc, fd_order, v_ref)
    acq = _acq(sxd, szd, wm, rxv, rzv)
    o = _opts(kernel, final_state, _precision(precision))
    ctx.check(L.lib().fomo_elastic2d_batch(ctx.handle, C.byref(g), _ptr(vp), _ptr(vs), _ptr(rho),
                                           C.byref(acq), _ptr(seis[0]), _ptr(seis[1]),
                                           C.byref(o), C.byref(st)))
    _remember(st)
    return Elastic2DBatchResult(seis[0], seis[1], BatchStats(st.kernel_time_s, ns))


# ---------------------------------------------------------------------------
# scalar2d (equations/scalar2d/scalar2d.jl:104-189)
# ---------------------------------------------------------------------------
def scalar_wavelet_matrix(w, vp, dt, sx, sz, source_scale):
    """Rows of the wavelet scaled per source as scalar2d.jl:141-147 does."""
    n_src = len(sx)
    wm = np.repeat(np.asarray(w, dtype=np.float32)[None, :], n_src, axis=0)
    dt = np.float32(dt)
    if source_scale == "v2dt2":
        for q in range(n_src):
            v = np.float32(vp[sx[q] - 1, sz[q] - 1])
            wm[q, :] = (wm[q, :] * np.float32((v * v) * (dt * dt))).astype(np.float32)
    elif source_scale == "dt":
        wm = (wm * dt).astype(np.float32)
    return np.asfortranarray(wm)


def scalar2d(vp, dh, dt, nt, f0, *, sx, sz, rx, rz, nbc: int = 50, fd_order: int = 8,
             v_ref=None, wavelet=None, source_scale="v2dt2", verbose: bool = True,
             device: int = 0, kernel: int = 0, final_state=None) -> Scalar2DResult:
    """Second-order constant-density scalar wave (equations/scalar2d/scalar2d.jl:104-189)."""
    source_scale = str(source_scale).lstrip(":")
    if source_scale not in ("v2dt2", "dt", "none"):
        raise ArgumentError(f"source_scale must be :v2dt2 / :dt / :none, got {source_scale}")
    vp = _f32F(vp)
    nx, nz = vp.shape
    dh, dt, f0 = np.float32(dh), np.float32(dt), np.float32(f0)
    _check_geometry(nx, nz, sx, sz, rx, rz)
    _check_numerics(vp.max(), _min_pos(vp), dh, dt, f0, fd_order, centered=True)
    v_ref = _min_pos(vp) if v_ref is None else np.float32(v_ref)
    w = _wavelet_row(wavelet, f0, dt, nt)
    sxv, szv = _i32F(sx).ravel(), _i32F(sz).ravel()
    wm = scalar_wavelet_matrix(w, vp, dt, sxv, szv, source_scale)
    rxv, rzv = _i32F(rx).ravel(), _i32F(rz).ravel()
    seis = np.zeros((rxv.size, nt), dtype=np.float32, order="F")
    st = L.Stats()
    ctx = L.context(device)
    g = _grid(nx, nz, dh, dt, nt, nbc, fd_order, v_ref)
    acq = _acq(sxv.reshape(-1, 1, order="F"), szv.reshape(-1, 1, order="F"), wm, rxv, rzv)
    o = _opts(kernel, final_state)
    ctx.check(L.lib().fomo_scalar2d(ctx.handle, C.byref(g), _ptr(vp), C.byref(acq), _ptr(seis),
                                    C.byref(o), C.byref(st)))
    _remember(st)
    return Scalar2DResult(seis, Stats(st.kernel_time_s))


# ---------------------------------------------------------------------------
# uneven-size batch (no reference counterpart; each shot equals acoustic2d)
# ---------------------------------------------------------------------------
class UnevenStats(NamedTuple):
    kernel_time_s: float
    n_shots: int
    cell_updates: float
    tile: tuple


class Acoustic2DUnevenResult(NamedTuple):
    shots: list  # per shot (seis_p, seis_vx, seis_vz), each (n_rec, nt)
    stats: UnevenStats


def acoustic2d_uneven(vps, rhos, dh, dt, nt, f0, *, sx, sz, rx, rz, nbc: int = 50,
                      fd_order: int = 8, v_ref=None, wavelet=None,
                      scale_source_by_dt: bool = False, device: int = 0,
                      kernel: int = 0) -> Acoustic2DUnevenResult:
    """Many acoustic2d shots whose models differ in size, stepped together.

    ``vps``/``rhos``: one (nx_s, nz_s) model per shot; ``sx``/``sz``: per shot
    an index or a list of sources firing together; ``rx``/``rz``: per shot the
    receiver indices; ``v_ref``: None (each shot's min positive vp), a number,
    or one value per shot.  Each shot's seismograms equal ``acoustic2d`` on
    that shot (equations/acoustic2d/acoustic2d.jl:47-192) bit for bit.
    ``kernel``: 0 = the fused single sweep from order 4 (one launch per step
    for all shots), 1 = velocity and pressure kernels per step.  ``stats.tile``
    is (threads per strip, 0) for the sweep, the (x, z) block for two kernels.
    """
    ns = len(vps)
    if ns == 0 or len(rhos) != ns or len(sx) != ns or len(sz) != ns or len(rx) != ns \
            or len(rz) != ns:
        raise ArgumentError("vps, rhos, sx, sz, rx, rz need one entry per shot")
    if fd_order not in _FD:
        raise ValueError(f"Unsupported FD order: {fd_order}")
    dh, dt, f0 = np.float32(dh), np.float32(dt), np.float32(f0)
    models = [(_f32F(v), _f32F(r)) for v, r in zip(vps, rhos)]
    vmax = max(float(v.max()) for v, _ in models)
    vmin = min(float(_min_pos(v)) for v, _ in models)
    _check_numerics(vmax, vmin, dh, dt, f0, fd_order)
    w = _wavelet_row(wavelet, f0, dt, nt)
    if scale_source_by_dt:
        w = (w * dt).astype(np.float32)
    keep = []  # arrays referenced by the descriptors must outlive the call
    descs = (L.Shot2D * ns)()
    results = []
    for s, (vp, rho) in enumerate(models):
        if vp.shape != rho.shape or vp.ndim != 2:
            raise ArgumentError(f"shot {s + 1}: vp and rho must be matching 2D arrays")
        nx, nz = vp.shape
        sxv, szv = _i32F(np.atleast_1d(sx[s])).ravel(), _i32F(np.atleast_1d(sz[s])).ravel()
        rxv, rzv = _i32F(rx[s]).ravel(), _i32F(rz[s]).ravel()
        if sxv.size != szv.size or rxv.size != rzv.size:
            raise ArgumentError(f"shot {s + 1}: coordinate lengths differ")
        _check_geometry(nx, nz, sxv, szv, rxv, rzv)
        wm = np.asfortranarray(np.repeat(w[None, :], sxv.size, axis=0))
        seis = [np.zeros((rxv.size, nt), dtype=np.float32, order="F") for _ in range(3)]
        vr = v_ref[s] if isinstance(v_ref, (list, tuple, np.ndarray)) else v_ref
        vr = 0.0 if vr is None else float(np.float32(vr))
        d = descs[s]
        d.nx, d.nz, d.vp, d.rho = nx, nz, _ptr(vp), _ptr(rho)
        d.n_src, d.sx, d.sz, d.wavelet = sxv.size, _ptr(sxv), _ptr(szv), _ptr(wm)
        d.n_rec, d.rx, d.rz, d.v_ref = rxv.size, _ptr(rxv), _ptr(rzv), vr
        d.seis_p, d.seis_vx, d.seis_vz = _ptr(seis[0]), _ptr(seis[1]), _ptr(seis[2])
        keep += [vp, rho, sxv, szv, rxv, rzv, wm]
        results.append(tuple(seis))
    st = L.Stats()
    ctx = L.context(device)
    o = _opts(kernel)
    ctx.check(L.lib().fomo_acoustic2d_uneven(ctx.handle, float(dh), float(dt), int(nt), int(nbc),
                                             int(fd_order), ns, descs, C.byref(o), C.byref(st)))
    _remember(st)
    del keep
    tile = (st.sweep_config // 1000, st.sweep_config % 1000)
    return Acoustic2DUnevenResult(results, UnevenStats(st.kernel_time_s, ns, st.cell_updates, tile))


# ---------------------------------------------------------------------------
# 3D solvers: return (seis_vx, seis_vy, seis_vz, snaps) as the reference does
# ---------------------------------------------------------------------------
_PLANES = {"xz": 0, "xy": 1, "yz": 2}


class _Prep3(NamedTuple):
    vp: np.ndarray
    vs: Optional[np.ndarray]
    rho: np.ndarray
    grid: object      # L.Grid3D
    acq: object       # L.Acq3D (points into the arrays below)
    keep: tuple       # the acquisition arrays acq points into
    n_rec: int


def _prep3d(elastic, vp, vs, rho, dh, dt, nt, f0, sx, sy, sz, rx, ry, rz, nbc, fd_order, v_ref,
            wavelet) -> _Prep3:
    """Checked float32 / int32 arrays and the C structs of a 3D run."""
    vp, rho = _f32F(vp), _f32F(rho)
    vs = _f32F(vs) if elastic else None
    if vp.ndim != 3:
        raise ArgumentError("3D models are (nx, ny, nz) arrays")
    nx, ny, nz = vp.shape
    if fd_order not in _FD:
        raise ValueError(f"Unsupported FD order: {fd_order}")
    sxv, syv, szv = (_i32F(a).ravel() for a in (sx, sy, sz))
    rxv, ryv, rzv = (_i32F(a).ravel() for a in (rx, ry, rz))
    if not (sxv.size == syv.size == szv.size) or not (rxv.size == ryv.size == rzv.size):
        raise ArgumentError("coordinate vectors differ in length")
    for name, v, n in (("sx", sxv, nx), ("sy", syv, ny), ("sz", szv, nz), ("rx", rxv, nx),
                       ("ry", ryv, ny), ("rz", rzv, nz)):
        if not np.all((1 <= v) & (v <= n)):
            raise ArgumentError(f"{name} out of range 1..{n}")
    dh, dt, f0 = np.float32(dh), np.float32(dt), np.float32(f0)
    v_ref = _min_pos(vp) if v_ref is None else np.float32(v_ref)
    w = _wavelet_row(wavelet, f0, dt, nt)
    # every source fires the one Ricker row (acoustic3d.jl:64-66)
    wm = np.asfortranarray(np.repeat(w[None, :], sxv.size, axis=0))
    g = L.Grid3D(nx, ny, nz, float(dh), float(dt), int(nt), int(nbc), int(fd_order), float(v_ref))
    acq = L.Acq3D(sxv.size, _ptr(sxv), _ptr(syv), _ptr(szv), _ptr(wm), rxv.size, _ptr(rxv),
                  _ptr(ryv), _ptr(rzv))
    return _Prep3(vp, vs, rho, g, acq, (sxv, syv, szv, rxv, ryv, rzv, wm), int(rxv.size))


def _run3d(elastic, vp, vs, rho, dh, dt, nt, f0, sx, sy, sz, rx, ry, rz, nbc, fd_order,
           snap_interval, snap_plane, snap_index, v_ref, wavelet, device, final_state, kernel=0):
    plane = _PLANES.get(str(snap_plane).lstrip(":"))
    if plane is None:
        raise ArgumentError(f"snap_plane must be :xz, :xy or :yz, got {snap_plane}")
    pr = _prep3d(elastic, vp, vs, rho, dh, dt, nt, f0, sx, sy, sz, rx, ry, rz, nbc, fd_order,
                 v_ref, wavelet)
    vp, vs, rho, g, acq = pr.vp, pr.vs, pr.rho, pr.grid, pr.acq
    nx, ny, nz = vp.shape
    if snap_index == 0:
        snap_index = ny // 2  # acoustic3d.jl:50-52 (ny÷2 for every plane)
    seis = [np.zeros((pr.n_rec, nt), dtype=np.float32, order="F") for _ in range(3)]
    nsnap = nt // snap_interval if snap_interval > 0 else 0
    shape = {0: (nx, nz), 1: (nx, ny), 2: (ny, nz)}[plane]
    snaps = np.zeros(shape + (nsnap,), dtype=np.float32, order="F") if nsnap else None
    st = L.Stats()
    ctx = L.context(device)
    o = _opts(kernel, final_state)
    if elastic:
        rc = L.lib().fomo_elastic3d(ctx.handle, C.byref(g), _ptr(vp), _ptr(vs), _ptr(rho),
                                    C.byref(acq), int(snap_interval), plane, int(snap_index),
                                    _ptr(seis[0]), _ptr(seis[1]), _ptr(seis[2]), _ptr(snaps),
                                    C.byref(o), C.byref(st))
    else:
        rc = L.lib().fomo_acoustic3d(ctx.handle, C.byref(g), _ptr(vp), _ptr(rho), C.byref(acq),
                                     int(snap_interval), plane, int(snap_index), _ptr(seis[0]),
                                     _ptr(seis[1]), _ptr(seis[2]), _ptr(snaps), C.byref(o),
                                     C.byref(st))
    ctx.check(rc)
    _remember(st)
    return seis[0], seis[1], seis[2], _snap_list(snaps)


def acoustic3d(vp, rho, dh, dt, nt, f0, *, sx, sy, sz, rx, ry, rz, nbc: int = 50,
               fd_order: int = 8, snap_interval: int = 0, snap_plane="xz", snap_index: int = 0,
               v_ref=None, wavelet=None, device: int = 0,
               final_state: Optional[np.ndarray] = None, kernel: int = 0):
    """3D acoustic simulation (equations/acoustic3d/acoustic3d.jl:37-185).

    Returns ``(seis_vx, seis_vy, seis_vz, snaps)``; snapshots hold p on the
    chosen plane.  The HABC is the reference's 3D Higdon formula with
    read-only inputs (deterministic; the reference updates in place).
    ``kernel``: 0 or 2 = fused TMA half steps (update and Higdon boundary in
    one pass each), 1 = per-cell updates and two Higdon passes (identical
    results).
    """
    return _run3d(False, vp, None, rho, dh, dt, nt, f0, sx, sy, sz, rx, ry, rz, nbc, fd_order,
                  snap_interval, snap_plane, snap_index, v_ref, wavelet, device, final_state,
                  kernel)


def elastic3d(vp, vs, rho, dh, dt, nt, f0, *, sx, sy, sz, rx, ry, rz, nbc: int = 50,
              fd_order: int = 8, snap_interval: int = 0, snap_plane="xz", snap_index: int = 0,
              v_ref=None, wavelet=None, device: int = 0,
              final_state: Optional[np.ndarray] = None, kernel: int = 0):
    """3D elastic simulation (equations/elastic3d/elastic3d.jl:37-162).

    Returns ``(seis_vx, seis_vy, seis_vz, snaps)``; sources inject into txx,
    tyy and tzz; snapshots hold vz.  ``kernel``: 0 or 2 = fused TMA half steps
    (update and Higdon boundary in one pass each), 3 = z-marching updates with
    separate Higdon passes, 1 = per-cell updates (identical results).
    """
    return _run3d(True, vp, vs, rho, dh, dt, nt, f0, sx, sy, sz, rx, ry, rz, nbc, fd_order,
                  snap_interval, snap_plane, snap_index, v_ref, wavelet, device, final_state,
                  kernel)


def debug_medium2d(kind: str, vp, vs, rho, pad: int, dt=1.0, dh=1.0, device: int = 0):
    """Device-prepared padded materials (diagnostics): elastic/acoustic/scalar."""
    k = {"elastic": 0, "acoustic": 1, "scalar": 2}[kind]
    vp = _f32F(vp)
    vs = _f32F(vs) if vs is not None else None
    rho = _f32F(rho) if rho is not None else None
    nx, nz = vp.shape
    nf = {0: 5, 1: 3, 2: 1}[k]
    out = np.zeros((nx + 2 * pad, nz + 2 * pad, nf), dtype=np.float32, order="F")
    ctx = L.context(device)
    ctx.check(L.lib().fomo_debug_medium2d(ctx.handle, k, nx, nz, pad, float(np.float32(dt)),
                                          float(np.float32(dh)), _ptr(vp), _ptr(vs), _ptr(rho),
                                          _ptr(out)))
    return out


# ---------------------------------------------------------------------------
# coupled2d: coupled P-S potentials (equations/coupled2d/coupled2d.jl:53-171)
# ---------------------------------------------------------------------------
def coupled2d(vp, vs, dh, dt, nt, f0, *, sx: Sequence[int], sz: Sequence[int], rx, rz,
              nbc: int = 50, fd_order: int = 8, snap_interval: int = 0, v_ref_p=None,
              v_ref_s=None, smooth_sigma: float = 3.0, wavelet=None, verbose: bool = True,
              device: int = 0) -> Coupled2DResult:
    """2D coupled P-S potential simulation (constant density).  ``smooth_sigma``
    smooths alpha = vp^2, beta = vs^2 (grid points) before their derivatives."""
    vp, vs = _f32F(vp), _f32F(vs)
    nx, nz = vp.shape
    if vs.shape != vp.shape:
        raise ArgumentError("vp and vs sizes differ")
    dh, dt, f0 = np.float32(dh), np.float32(dt), np.float32(f0)
    _check_geometry(nx, nz, sx, sz, rx, rz)
    vmin_disp = _min_pos(vs) if np.any(vs > 0) else _min_pos(vp)  # coupled2d.jl:75-76
    _check_numerics(vp.max(), vmin_disp, dh, dt, f0, fd_order, centered=True)
    v_ref_p = _min_pos(vp) if v_ref_p is None else np.float32(v_ref_p)
    v_ref_s = _min_pos(vs) if v_ref_s is None else np.float32(v_ref_s)
    w = _wavelet_row(wavelet, f0, dt, nt)
    sxv, szv = _i32F(sx).ravel(), _i32F(sz).ravel()
    if sxv.size != szv.size:
        raise ArgumentError("sx and sz lengths differ")
    wm = np.asfortranarray(np.repeat(w[None, :], sxv.size, axis=0))
    rxv, rzv = _i32F(rx).ravel(), _i32F(rz).ravel()
    nrec = rxv.size
    seis = [np.zeros((nrec, nt), dtype=np.float32, order="F") for _ in range(2)]
    nsnap = nt // snap_interval if snap_interval > 0 else 0
    snaps = [np.zeros((nx, nz, nsnap), dtype=np.float32, order="F") if nsnap else None
             for _ in range(2)]
    st = L.Stats()
    ctx = L.context(device)
    g = _grid(nx, nz, dh, dt, nt, nbc, fd_order, v_ref_p)
    acq = _acq(sxv.reshape(-1, 1, order="F"), szv.reshape(-1, 1, order="F"), wm, rxv, rzv)
    o = _opts()
    ctx.check(L.lib().fomo_coupled2d(ctx.handle, C.byref(g), _ptr(vp), _ptr(vs), float(v_ref_s),
                                     float(smooth_sigma), C.byref(acq), int(snap_interval),
                                     _ptr(seis[0]), _ptr(seis[1]), _ptr(snaps[0]),
                                     _ptr(snaps[1]), C.byref(o), C.byref(st)))
    _remember(st)
    return Coupled2DResult(seis[0], seis[1], _snap_list(snaps[0]), _snap_list(snaps[1]),
                           Stats(st.kernel_time_s))


def debug_coupled_medium(vp, vs, dh, nbc, fd_order, smooth_sigma=3.0, device: int = 0):
    """coupled2d's device-prepared medium, (nx + 2 pad, nz + 2 pad, 8)."""
    vp, vs = _f32F(vp), _f32F(vs)
    nx, nz = vp.shape
    pad = nbc + fd_order // 2
    out = np.zeros((nx + 2 * pad, nz + 2 * pad, 8), np.float32, order="F")
    ctx = L.context(device)
    ctx.check(L.lib().fomo_debug_coupled_medium(ctx.handle, nx, nz, int(nbc), int(fd_order),
                                                float(dh), float(smooth_sigma), _ptr(vp),
                                                _ptr(vs), _ptr(out)))
    return out
