"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The oracle (``fomo_oracle.cpp``) restates Fomo.jl's time stepping on the CPU in
FP32 and FP64.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` may import this module; the product library never does.

Array conventions mirror the Julia reference: grids are ``(nx, nz)`` with x the
fastest (Fortran order), indices are 1-based and unpadded, source index
matrices are ``(n_src, n_shots)``, the wavelet matrix is ``(n_src, nt)`` and
seismograms are ``(n_rec, nt[, n_shots])``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "lib" / "libfomo_oracle.so"
_lib = None

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="F_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="F_CONTIGUOUS")


def build(force: bool = False) -> Path:
    """Compile the oracle with its Makefile (no-op when up to date)."""
    if force or not _LIB_PATH.exists() or (
        _LIB_PATH.stat().st_mtime < (_HERE / "fomo_oracle.cpp").stat().st_mtime
    ):
        subprocess.run(["make", "-C", str(_HERE)], check=True, capture_output=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(_LIB_PATH))
        vp = C.c_void_p
        L.oracle_elastic2d.restype = C.c_int
        L.oracle_elastic2d.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _f32p, _f32p, _f32p,
                                       C.c_float, C.c_float, C.c_int, C.c_int, C.c_int, C.c_float,
                                       C.c_int, _i32p, _i32p, _f32p, C.c_int, _i32p, _i32p,
                                       vp, vp, C.c_int, vp, vp]
        L.oracle_elastic2d_store.restype = C.c_int
        L.oracle_elastic2d_store.argtypes = [C.c_int, C.c_float, C.c_float, C.c_int] + \
            L.oracle_elastic2d.argtypes[1:]
        L.oracle_round_store.restype = None
        L.oracle_round_store.argtypes = [C.c_int, vp, vp, C.c_longlong]
        L.oracle_acoustic2d.restype = C.c_int
        L.oracle_acoustic2d.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _f32p, _f32p,
                                        C.c_float, C.c_float, C.c_int, C.c_int, C.c_int, C.c_float,
                                        C.c_int, _i32p, _i32p, _f32p, C.c_int, _i32p, _i32p,
                                        vp, vp, vp, C.c_int, vp, vp, C.c_int]
        L.oracle_acoustic2d_sponge.restype = C.c_int
        L.oracle_acoustic2d_sponge.argtypes = [C.c_int, C.c_float, C.c_int, C.c_int, C.c_int,
                                               _f32p, _f32p, C.c_float, C.c_float, C.c_int,
                                               C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f32p,
                                               C.c_int, _i32p, _i32p, vp, vp, vp, C.c_int, vp, vp]
        L.oracle_elastic2d_sponge.restype = C.c_int
        L.oracle_elastic2d_sponge.argtypes = [C.c_int, C.c_float, C.c_int, C.c_int, C.c_int,
                                              _f32p, _f32p, _f32p, C.c_float, C.c_float, C.c_int,
                                              C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f32p,
                                              C.c_int, _i32p, _i32p, vp, vp, C.c_int, vp, vp]
        L.oracle_sponge_table.restype = C.c_int
        L.oracle_sponge_table.argtypes = [C.c_int, C.c_float, vp]
        L.oracle_coupled2d.restype = C.c_int
        L.oracle_coupled2d.argtypes = [C.c_int, C.c_int, C.c_int, _f32p, _f32p, C.c_float,
                                       C.c_float, C.c_int, C.c_int, C.c_int, C.c_float,
                                       C.c_float, C.c_double, C.c_int, _i32p, _i32p, _f32p,
                                       C.c_int, _i32p, _i32p, vp, vp, C.c_int, vp, vp, vp]
        L.oracle_scalar2d.restype = C.c_int
        L.oracle_scalar2d.argtypes = [C.c_int, C.c_int, C.c_int, _f32p, C.c_float, C.c_float,
                                      C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, _i32p, _i32p,
                                      _f32p, C.c_int, _i32p, _i32p, vp, vp]
        L.oracle_medium2d_f32.restype = C.c_int
        L.oracle_medium2d_f32.argtypes = [C.c_int, C.c_int, C.c_int, _f32p, _f32p, _f32p, C.c_int, vp]
        L.oracle_habc_f32.restype = C.c_int
        L.oracle_habc_f32.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float, vp, vp]
        L.oracle_habc_apply_f32.restype = C.c_int
        L.oracle_habc_apply_f32.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                            C.c_float, C.c_int, vp, vp]
        a3 = [C.c_int, C.c_int, C.c_int, C.c_int]
        L.oracle_acoustic3d.restype = C.c_int
        L.oracle_acoustic3d.argtypes = a3 + [_f32p, _f32p, C.c_float, C.c_float, C.c_int, C.c_int,
                                             C.c_int, C.c_float, C.c_int, _i32p, _i32p, _i32p,
                                             _f32p, C.c_int, _i32p, _i32p, _i32p, vp, vp, vp,
                                             C.c_int, C.c_int, C.c_int, vp, vp]
        L.oracle_elastic3d.restype = C.c_int
        L.oracle_elastic3d.argtypes = a3 + [_f32p, _f32p, _f32p, C.c_float, C.c_float, C.c_int,
                                            C.c_int, C.c_int, C.c_float, C.c_int, _i32p, _i32p,
                                            _i32p, _f32p, C.c_int, _i32p, _i32p, _i32p, vp, vp, vp,
                                            C.c_int, C.c_int, C.c_int, vp, vp]
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_max_threads.restype = C.c_int
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def _f32(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float32))


def _i32(a):
    return np.asfortranarray(np.asarray(a, dtype=np.int32))


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _dt(prec):
    return {32: np.float32, 64: np.float64}[prec]


def default_v_ref(vp) -> float:
    vp = np.asarray(vp, dtype=np.float32)
    return float(vp[vp > 0].min())


def _src_matrix(sx, ns):
    a = _i32(sx)
    if a.ndim == 1:
        a = a.reshape(-1, 1, order="F") if ns == 1 else a.reshape(1, -1, order="F")
    return np.asfortranarray(a)


STORE = {"fp32": 0, "fp16": 1, "bf16": 2}


def round_store(x, store: str) -> np.ndarray:
    """Round float32 values to the storage format (RNE) and back to float32."""
    x = np.asfortranarray(np.asarray(x, dtype=np.float32))
    y = np.empty_like(x, order="F")
    lib().oracle_round_store(STORE[store], _ptr(x), _ptr(y), x.size)
    return y


def elastic2d(vp, vs, rho, dh, dt, nt, *, sx, sz, rx, rz, wavelet, nbc=50, fd_order=8,
              v_ref=None, snap_interval=0, prec=32, n_shots=1, final=False, store=None,
              sv=1.0, st=1.0, fp32_band=0, sponge_factor=None):
    """Elastic velocity-stress run.  ``sx``/``sz``: (n_src, n_shots).  ``wavelet``: (n_src, nt).

    ``store`` ("fp16"/"bf16") emulates FP32 arithmetic on wavefields stored
    in that format under power-of-two scales ``sv`` (velocity) and ``st``
    (stress); cells closer than ``fp32_band`` to an edge keep FP32 storage;
    results are returned unscaled.  ``sponge_factor`` (not None) selects
    boundary=:sponge, the Cerjan layer of boundary/sponge.jl, instead of HABC.
    """
    vp, vs, rho = _f32(vp), _f32(vs), _f32(rho)
    nx, nz = vp.shape
    sxm, szm = _src_matrix(sx, n_shots), _src_matrix(sz, n_shots)
    n_src, ns = sxm.shape
    w = _f32(wavelet).reshape(n_src, nt, order="F")
    rx, rz = _i32(rx), _i32(rz)
    nrec = rx.size
    T = _dt(prec)
    svx = np.zeros((nrec, nt, ns), dtype=T, order="F")
    svz = np.zeros_like(svx)
    nsnap = nt // snap_interval if snap_interval > 0 else 0
    snaps = np.zeros((nx, nz, nsnap, ns), dtype=T, order="F") if nsnap else None
    M = fd_order // 2
    nxp, nzp = nx + 2 * (nbc + M), nz + 2 * (nbc + M)
    fin = np.zeros((nxp, nzp, 5, ns), dtype=T, order="F") if final else None
    vr = default_v_ref(vp) if v_ref is None else float(v_ref)
    if sponge_factor is not None:
        if store is not None:
            raise ValueError("the sponge boundary runs FP32 storage only")
        rc = lib().oracle_elastic2d_sponge(prec, float(sponge_factor), nx, nz, ns, vp, vs, rho, dh,
                                           dt, nt, nbc, fd_order, n_src, sxm, szm, w, nrec, rx,
                                           rz, _ptr(svx), _ptr(svz), snap_interval, _ptr(snaps),
                                           _ptr(fin))
    elif store is not None:
        if prec != 32:
            raise ValueError("storage emulation runs FP32 arithmetic")
        rc = lib().oracle_elastic2d_store(STORE[store], sv, st, int(fp32_band), nx, nz, ns, vp, vs, rho, dh, dt,
                                          nt, nbc, fd_order, vr, n_src, sxm, szm, w, nrec, rx,
                                          rz, _ptr(svx), _ptr(svz), snap_interval, _ptr(snaps),
                                          _ptr(fin))
    else:
        rc = lib().oracle_elastic2d(prec, nx, nz, ns, vp, vs, rho, dh, dt, nt, nbc, fd_order, vr,
                                    n_src, sxm, szm, w, nrec, rx, rz, _ptr(svx), _ptr(svz),
                                    snap_interval, _ptr(snaps), _ptr(fin))
    if rc != 0:
        raise RuntimeError(f"oracle_elastic2d failed: {rc}")
    return dict(seis_vx=svx, seis_vz=svz, snaps=snaps, final=fin)


def acoustic2d(vp, rho, dh, dt, nt, *, sx, sz, rx, rz, wavelet, nbc=50, fd_order=8, v_ref=None,
               snap_interval=0, prec=32, n_shots=1, final=False, zone_nbc=0, sponge_factor=None):
    """Acoustic velocity-pressure run; ``sponge_factor`` (not None) selects the
    Cerjan sponge boundary (boundary/sponge.jl) instead of HABC."""
    vp, rho = _f32(vp), _f32(rho)
    nx, nz = vp.shape
    sxm, szm = _src_matrix(sx, n_shots), _src_matrix(sz, n_shots)
    n_src, ns = sxm.shape
    w = _f32(wavelet).reshape(n_src, nt, order="F")
    rx, rz = _i32(rx), _i32(rz)
    nrec = rx.size
    T = _dt(prec)
    sp = np.zeros((nrec, nt, ns), dtype=T, order="F")
    svx, svz = np.zeros_like(sp), np.zeros_like(sp)
    nsnap = nt // snap_interval if snap_interval > 0 else 0
    snaps = np.zeros((nx, nz, nsnap, ns), dtype=T, order="F") if nsnap else None
    M = fd_order // 2
    nxp, nzp = nx + 2 * (nbc + M), nz + 2 * (nbc + M)
    fin = np.zeros((nxp, nzp, 3, ns), dtype=T, order="F") if final else None
    vr = default_v_ref(vp) if v_ref is None else float(v_ref)
    if sponge_factor is not None:
        rc = lib().oracle_acoustic2d_sponge(prec, float(sponge_factor), nx, nz, ns, vp, rho, dh,
                                            dt, nt, nbc, fd_order, n_src, sxm, szm, w, nrec, rx,
                                            rz, _ptr(sp), _ptr(svx), _ptr(svz), snap_interval,
                                            _ptr(snaps), _ptr(fin))
    else:
        rc = lib().oracle_acoustic2d(prec, nx, nz, ns, vp, rho, dh, dt, nt, nbc, fd_order, vr,
                                     n_src, sxm, szm, w, nrec, rx, rz, _ptr(sp), _ptr(svx),
                                     _ptr(svz), snap_interval, _ptr(snaps), _ptr(fin),
                                     int(zone_nbc))
    if rc != 0:
        raise RuntimeError(f"oracle_acoustic2d failed: {rc}")
    return dict(seis_p=sp, seis_vx=svx, seis_vz=svz, snaps=snaps, final=fin)


def scalar2d(vp, dh, dt, nt, *, sx, sz, rx, rz, wavelet, nbc=50, fd_order=8, v_ref=None,
             prec=32, final=False):
    """``wavelet``: (n_src, nt), already scaled as the caller's source_scale asks."""
    vp = _f32(vp)
    nx, nz = vp.shape
    sx, sz = _i32(sx).ravel(order="F"), _i32(sz).ravel(order="F")
    n_src = sx.size
    w = _f32(wavelet).reshape(n_src, nt, order="F")
    rx, rz = _i32(rx), _i32(rz)
    nrec = rx.size
    T = _dt(prec)
    su = np.zeros((nrec, nt), dtype=T, order="F")
    M = fd_order // 2
    nxp, nzp = nx + 2 * (nbc + M), nz + 2 * (nbc + M)
    fin = np.zeros((nxp, nzp, 2), dtype=T, order="F") if final else None
    vr = default_v_ref(vp) if v_ref is None else float(v_ref)
    rc = lib().oracle_scalar2d(prec, nx, nz, vp, dh, dt, nt, nbc, fd_order, vr, n_src,
                               np.asfortranarray(sx), np.asfortranarray(sz), w, nrec, rx, rz,
                               _ptr(su), _ptr(fin))
    if rc != 0:
        raise RuntimeError(f"oracle_scalar2d failed: {rc}")
    return dict(seis_u=su, final=fin)


_PLANES = {"xz": 0, "xy": 1, "yz": 2}


def _run3d(kind, vp, vs, rho, dh, dt, nt, sx, sy, sz, rx, ry, rz, wavelet, nbc, fd_order, v_ref,
           snap_interval, snap_plane, snap_index, prec, final):
    vp, rho = _f32(vp), _f32(rho)
    nx, ny, nz = vp.shape
    sx, sy, sz = (_i32(a).ravel(order="F") for a in (sx, sy, sz))
    rx, ry, rz = (_i32(a).ravel(order="F") for a in (rx, ry, rz))
    n_src, nrec = sx.size, rx.size
    w = _f32(wavelet).reshape(n_src, nt, order="F")
    T = _dt(prec)
    seis = [np.zeros((nrec, nt), dtype=T, order="F") for _ in range(3)]
    plane = _PLANES[str(snap_plane).lstrip(":")]
    si = snap_index if snap_index > 0 else ny // 2
    shp = {0: (nx, nz), 1: (nx, ny), 2: (ny, nz)}[plane]
    nsnap = nt // snap_interval if snap_interval > 0 else 0
    snaps = np.zeros(shp + (nsnap,), dtype=T, order="F") if nsnap else None
    M = fd_order // 2
    pad = nbc + M
    nf = 9 if kind == "elastic" else 4
    fin = (np.zeros((nx + 2 * pad, ny + 2 * pad, nz + 2 * pad, nf), dtype=T, order="F")
           if final else None)
    vr = default_v_ref(vp) if v_ref is None else float(v_ref)
    common = (dh, dt, nt, nbc, fd_order, vr, n_src, np.asfortranarray(sx), np.asfortranarray(sy),
              np.asfortranarray(sz), w, nrec, np.asfortranarray(rx), np.asfortranarray(ry),
              np.asfortranarray(rz), _ptr(seis[0]), _ptr(seis[1]), _ptr(seis[2]), snap_interval,
              plane, si, _ptr(snaps), _ptr(fin))
    if kind == "elastic":
        rc = lib().oracle_elastic3d(prec, nx, ny, nz, vp, _f32(vs), rho, *common)
    else:
        rc = lib().oracle_acoustic3d(prec, nx, ny, nz, vp, rho, *common)
    if rc != 0:
        raise RuntimeError(f"oracle_{kind}3d failed: {rc}")
    return dict(seis_vx=seis[0], seis_vy=seis[1], seis_vz=seis[2], snaps=snaps, final=fin)


def acoustic3d(vp, rho, dh, dt, nt, *, sx, sy, sz, rx, ry, rz, wavelet, nbc=50, fd_order=8,
               v_ref=None, snap_interval=0, snap_plane="xz", snap_index=0, prec=32, final=False):
    return _run3d("acoustic", vp, None, rho, dh, dt, nt, sx, sy, sz, rx, ry, rz, wavelet, nbc,
                  fd_order, v_ref, snap_interval, snap_plane, snap_index, prec, final)


def elastic3d(vp, vs, rho, dh, dt, nt, *, sx, sy, sz, rx, ry, rz, wavelet, nbc=50, fd_order=8,
              v_ref=None, snap_interval=0, snap_plane="xz", snap_index=0, prec=32, final=False):
    return _run3d("elastic", vp, vs, rho, dh, dt, nt, sx, sy, sz, rx, ry, rz, wavelet, nbc,
                  fd_order, v_ref, snap_interval, snap_plane, snap_index, prec, final)


def medium2d(kind, vp, vs, rho, pad):
    """Padded host preparation.  kind 'elastic' -> (bx,bz,lam,lam2mu,mu_txz); 'acoustic' -> (bx,bz,kappa)."""
    vp, rho = _f32(vp), _f32(rho)
    vs = _f32(vs) if vs is not None else vp
    nx, nz = vp.shape
    k = 0 if kind == "elastic" else 1
    nf = 5 if k == 0 else 3
    out = np.zeros((nx + 2 * pad, nz + 2 * pad, nf), dtype=np.float32, order="F")
    lib().oracle_medium2d_f32(k, nx, nz, vp, vs, rho, pad, _ptr(out))
    return out


def habc_coeffs(pad, v_ref, dt, dh):
    qs = np.zeros(3, dtype=np.float32)
    wt = np.zeros((pad + 2, 3), dtype=np.float32, order="F")
    nbc = lib().oracle_habc_f32(pad, v_ref, dt, dh, _ptr(qs), _ptr(wt))
    return nbc, qs, wt


def habc_apply(f, f_old, pad, v_ref, dt, dh, kind):
    """One deterministic two-pass Higdon application (returns the corrected copy)."""
    f = np.array(f, dtype=np.float32, order="F", copy=True)
    fo = _f32(f_old)
    nxp, nzp = f.shape
    lib().oracle_habc_apply_f32(nxp, nzp, pad, v_ref, dt, dh, kind, _ptr(f), _ptr(fo))
    return f


def coupled2d(vp, vs, dh, dt, nt, *, sx, sz, rx, rz, wavelet, nbc=50, fd_order=8,
              v_ref_p=None, v_ref_s=None, smooth_sigma=3.0, snap_interval=0, prec=32,
              medium=False):
    """Coupled P-S potential run (equations/coupled2d).  ``wavelet``: (n_src, nt).
    ``medium=True`` also returns the eight prepared medium planes (nxp, nzp, 8)."""
    vp, vs = _f32(vp), _f32(vs)
    nx, nz = vp.shape
    sxv, szv = _i32(np.ravel(sx)), _i32(np.ravel(sz))
    n_src = sxv.size
    w = _f32(wavelet).reshape(n_src, nt, order="F")
    rx, rz = _i32(rx), _i32(rz)
    nrec = rx.size
    T = _dt(prec)
    sP = np.zeros((nrec, nt), dtype=T, order="F")
    sS = np.zeros_like(sP)
    nsnap = nt // snap_interval if snap_interval > 0 else 0
    snP = np.zeros((nx, nz, nsnap), dtype=T, order="F") if nsnap else None
    snS = np.zeros_like(snP) if nsnap else None
    M = fd_order // 2
    nxp, nzp = nx + 2 * (nbc + M), nz + 2 * (nbc + M)
    med = np.zeros((nxp, nzp, 8), dtype=T, order="F") if medium else None
    vrp = default_v_ref(vp) if v_ref_p is None else float(v_ref_p)
    vrs = default_v_ref(vs) if v_ref_s is None else float(v_ref_s)
    rc = lib().oracle_coupled2d(prec, nx, nz, vp, vs, dh, dt, nt, nbc, fd_order, vrp, vrs,
                                float(smooth_sigma), n_src, sxv, szv, w, nrec, rx, rz, _ptr(sP),
                                _ptr(sS), snap_interval, _ptr(snP), _ptr(snS), _ptr(med))
    if rc != 0:
        raise RuntimeError(f"oracle_coupled2d failed: {rc}")
    return dict(seis_P=sP, seis_S=sS, snaps_P=snP, snaps_S=snS, medium=med)


def sponge_table(nbc, factor):
    """Cerjan damping factors damp[d], d = 0 .. nbc-1 cells from the padded edge."""
    out = np.zeros(max(int(nbc), 0), np.float32)
    lib().oracle_sponge_table(int(nbc), float(factor), _ptr(out))
    return out


def ricker(f0, dt, nt):
    """Ricker wavelet (utils/ricker_wavelet.jl:6-12) with Float32 f0, dt: the
    range t = (0:nt-1) .* dt rounds each exact product once; t0 = 1f0/f0,
    tau = t .- 1.5f0*t0, x = (pi*f0) .* tau with pi taken as Float32, and
    (1 - 2 x^2) * exp(-x^2) are Float32 operations (exp: the platform's)."""
    f32 = np.float32
    f0, dt = f32(f0), f32(dt)
    t = np.array([f32(k * float(dt)) for k in range(int(nt))], dtype=np.float32)
    t0 = f32(f32(1.0) / f0)
    tau = (t - f32(f32(1.5) * t0)).astype(np.float32)
    pf = f32(f32(np.pi) * f0)
    x = (pf * tau).astype(np.float32)
    sq = (x * x).astype(np.float32)
    with np.errstate(under="ignore"):
        e = np.exp(-sq).astype(np.float32)
    return ((f32(1.0) - f32(2.0) * sq) * e).astype(np.float32)


if __name__ == "__main__":  # pragma: no cover
    print(build(), max_threads(), os.cpu_count())
