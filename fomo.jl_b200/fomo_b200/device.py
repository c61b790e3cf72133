"""Device-resident entry: call the solvers on CUDA tensors that already live in HBM.

The arrays are passed as device pointers (FOMO_F_DEVICE_PTRS) and the library
runs on the caller's current torch stream, so torch events on that stream time
exactly the library's work.  Tensors must be contiguous; 2D models are stored
(nz, nx) in torch's row-major order, which is the reference's column-major
(nx, nz) layout.
"""
from __future__ import annotations

import ctypes as C

from . import _lib as L

PROFILE = 0x2  # library-internal per-kernel timing (fomo_stats.sweep_ms)


def _p(t):
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("device entry points need contiguous CUDA tensors")
    return t.data_ptr()


def elastic2d_batch(vp, vs, rho, *, dh, dt, nt, nbc, fd_order, v_ref, sx, sz, wavelet, rx, rz,
                    seis_vx, seis_vz, kernel: int = 0, precision: int = 0, device: int = 0,
                    flags: int = 0):
    """vp/vs/rho: (nz, nx) float32; sx/sz: (n_shots, n_src) int32 (1-based);
    wavelet: (nt, n_src) float32; rx/rz: (n_rec,) int32; seis_*: (n_shots, nt, n_rec)."""
    import torch

    nz, nx = vp.shape
    ns, n_src = sx.shape
    ctx = L.context(device)
    ctx.use_torch_stream(torch.cuda.current_stream(vp.device))
    g = L.Grid2D(nx, nz, float(dh), float(dt), int(nt), int(nbc), int(fd_order), float(v_ref))
    acq = L.Acq(ns, n_src, _p(sx), _p(sz), _p(wavelet), rx.numel(), _p(rx), _p(rz))
    o = L.Opts()
    o.flags = L.FOMO_F_DEVICE_PTRS | flags
    o.precision = precision
    o.kernel = kernel
    st = L.Stats()
    ctx.check(L.lib().fomo_elastic2d_batch(ctx.handle, C.byref(g), _p(vp), _p(vs), _p(rho),
                                           C.byref(acq), _p(seis_vx), _p(seis_vz), C.byref(o),
                                           C.byref(st)))
    return st
