"""ctypes binding of libfomo_b200.so (the C ABI declared in include/fomo_b200.h).

The library is the only compute path: if it is missing or no CUDA device is
present, every solver raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

PKG_ROOT = Path(__file__).resolve().parent.parent  # fomo.jl_b200/
LIB_PATH = Path(os.environ.get("FOMO_B200_LIB", PKG_ROOT / "lib" / "libfomo_b200.so"))

FOMO_OK = 0
FOMO_EARG = -1
FOMO_ECUDA = -2
FOMO_ENOMEM = -3
FOMO_ENONFINITE = -4
FOMO_EUNSUPPORTED = -5

FOMO_F_DEVICE_PTRS = 1
FOMO_F_PROFILE = 2
FOMO_F_STEP_LAUNCH = 4
FOMO_F_SPONGE = 8
FOMO_FP32, FOMO_FP16, FOMO_BF16 = 0, 1, 2
FOMO_KERNEL_AUTO, FOMO_KERNEL_TWO_PHASE, FOMO_KERNEL_SINGLE_SWEEP = 0, 1, 2

# Every symbol include/fomo_b200.h declares (checked by the ABI tests).
EXPORTS = (
    "fomo_version", "fomo_create", "fomo_destroy", "fomo_last_error", "fomo_set_stream",
    "fomo_trim", "fomo_check_numerics", "fomo_acoustic2d", "fomo_acoustic2d_batch",
    "fomo_elastic2d", "fomo_elastic2d_batch", "fomo_scalar2d", "fomo_debug_medium2d",
    "fomo_scalar2d_noalloc", "fomo_acoustic3d", "fomo_elastic3d", "fomo_acoustic2d_uneven",
    "fomo_corr_param_count", "fomo_corr_features", "fomo_corr_target", "fomo_corr_forward",
    "fomo_corr_gradients", "fomo_corr_adam", "fomo_scalar2d_snapshots", "fomo_scalar2d_corrected",
    "fomo_coupled2d", "fomo_debug_coupled_medium", "fomo_slab3d_layout_of", "fomo_slab3d_create",
    "fomo_slab3d_step", "fomo_slab3d_seismograms", "fomo_slab3d_destroy",
)


class Grid2D(C.Structure):
    _fields_ = [("nx", C.c_int32), ("nz", C.c_int32), ("dh", C.c_float), ("dt", C.c_float),
                ("nt", C.c_int32), ("nbc", C.c_int32), ("fd_order", C.c_int32),
                ("v_ref", C.c_float)]


class Acq(C.Structure):
    _fields_ = [("n_shots", C.c_int32), ("n_src", C.c_int32), ("sx", C.c_void_p),
                ("sz", C.c_void_p), ("wavelet", C.c_void_p), ("n_rec", C.c_int32),
                ("rx", C.c_void_p), ("rz", C.c_void_p)]


class Grid3D(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("dh", C.c_float),
                ("dt", C.c_float), ("nt", C.c_int32), ("nbc", C.c_int32),
                ("fd_order", C.c_int32), ("v_ref", C.c_float)]


class Acq3D(C.Structure):
    _fields_ = [("n_src", C.c_int32), ("sx", C.c_void_p), ("sy", C.c_void_p),
                ("sz", C.c_void_p), ("wavelet", C.c_void_p), ("n_rec", C.c_int32),
                ("rx", C.c_void_p), ("ry", C.c_void_p), ("rz", C.c_void_p)]


class Shot2D(C.Structure):
    _fields_ = [("nx", C.c_int32), ("nz", C.c_int32), ("vp", C.c_void_p), ("rho", C.c_void_p),
                ("n_src", C.c_int32), ("sx", C.c_void_p), ("sz", C.c_void_p),
                ("wavelet", C.c_void_p), ("n_rec", C.c_int32), ("rx", C.c_void_p),
                ("rz", C.c_void_p), ("v_ref", C.c_float), ("seis_p", C.c_void_p),
                ("seis_vx", C.c_void_p), ("seis_vz", C.c_void_p)]


class Opts(C.Structure):
    _fields_ = [("flags", C.c_uint32), ("precision", C.c_int32), ("kernel", C.c_int32),
                ("check_every", C.c_int32), ("final_state", C.c_void_p),
                ("sponge_factor", C.c_float)]


class Stats(C.Structure):
    _fields_ = [("kernel_time_s", C.c_double), ("cell_updates", C.c_double),
                ("alg_bytes", C.c_double), ("n_shots", C.c_int32), ("gpu_launches", C.c_int32),
                ("kernel", C.c_int32), ("status", C.c_int32), ("sweep_ms", C.c_double),
                ("sweep_launches", C.c_int32), ("sweep_config", C.c_int32)]


class FomoError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libfomo_b200 error {code}: {msg}")
        self.code = code


_lib = None
_lock = threading.Lock()


def lib() -> C.CDLL:
    """Load the library (raises OSError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise OSError(f"libfomo_b200.so not built at {LIB_PATH} (run `make -C fomo.jl_b200`)")
            L = C.CDLL(str(LIB_PATH))
            vp, i32, f32 = C.c_void_p, C.c_int32, C.c_float
            L.fomo_version.restype = C.c_int
            L.fomo_create.argtypes = [C.POINTER(C.c_void_p), C.c_int]
            L.fomo_create.restype = C.c_int
            L.fomo_destroy.argtypes = [vp]
            L.fomo_destroy.restype = None
            L.fomo_last_error.argtypes = [vp]
            L.fomo_last_error.restype = C.c_char_p
            L.fomo_set_stream.argtypes = [vp, vp]
            L.fomo_trim.argtypes = [vp]
            L.fomo_check_numerics.argtypes = [f32, f32, f32, i32, i32, C.POINTER(C.c_float)]
            L.fomo_check_numerics.restype = C.c_int
            g, a, o, s = C.POINTER(Grid2D), C.POINTER(Acq), C.POINTER(Opts), C.POINTER(Stats)
            L.fomo_acoustic2d.argtypes = [vp, g, vp, vp, a, i32, vp, vp, vp, vp, o, s]
            L.fomo_acoustic2d_batch.argtypes = [vp, g, vp, vp, a, vp, vp, vp, o, s]
            L.fomo_elastic2d.argtypes = [vp, g, vp, vp, vp, a, i32, vp, vp, vp, o, s]
            L.fomo_elastic2d_batch.argtypes = [vp, g, vp, vp, vp, a, vp, vp, o, s]
            L.fomo_scalar2d.argtypes = [vp, g, vp, a, vp, o, s]
            L.fomo_debug_medium2d.argtypes = [vp, i32, i32, i32, i32, f32, f32, vp, vp, vp, vp]
            L.fomo_coupled2d.argtypes = [vp, g, vp, vp, f32, C.c_double, a, i32, vp, vp, vp, vp,
                                         o, s]
            L.fomo_debug_coupled_medium.argtypes = [vp, i32, i32, i32, i32, f32, C.c_double, vp,
                                                    vp, vp]
            L.fomo_scalar2d_noalloc.argtypes = [g, vp, a, vp, vp, C.c_char_p, i32]
            L.fomo_scalar2d_noalloc.restype = C.c_int
            L.fomo_acoustic2d_uneven.argtypes = [vp, f32, f32, i32, i32, i32, i32,
                                                 C.POINTER(Shot2D), o, s]
            L.fomo_acoustic2d_uneven.restype = C.c_int
            i64 = C.c_int64
            L.fomo_corr_param_count.restype = C.c_int
            L.fomo_corr_param_count.argtypes = []
            L.fomo_corr_features.argtypes = [vp, i32, i32, i32, vp, vp, vp, i64, vp, i64, vp, i64,
                                             vp, i32, vp, vp, vp, vp]
            L.fomo_corr_target.argtypes = [vp, i32, i32, i32, i32, vp, vp, vp, vp, i64, vp, i64, vp,
                                           i64, vp, vp, vp, i32, vp, vp]
            L.fomo_corr_forward.argtypes = [vp, i32, i32, i32, vp, vp, vp]
            L.fomo_corr_gradients.argtypes = [vp, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp]
            L.fomo_corr_adam.argtypes = [vp, i32, vp, vp, vp, vp, f32, f32, f32, f32, i32]
            L.fomo_scalar2d_snapshots.argtypes = [vp, g, vp, a, i32, i32, i32, vp, vp, o, s]
            L.fomo_scalar2d_corrected.argtypes = [vp, g, vp, a, vp, vp, o, s]
            for name in ("fomo_corr_features", "fomo_corr_target", "fomo_corr_forward",
                         "fomo_corr_gradients", "fomo_corr_adam", "fomo_scalar2d_snapshots",
                         "fomo_scalar2d_corrected"):
                getattr(L, name).restype = C.c_int
            g3, a3 = C.POINTER(Grid3D), C.POINTER(Acq3D)
            L.fomo_acoustic3d.argtypes = [vp, g3, vp, vp, a3, i32, i32, i32, vp, vp, vp, vp, o, s]
            L.fomo_elastic3d.argtypes = [vp, g3, vp, vp, vp, a3, i32, i32, i32, vp, vp, vp, vp,
                                         o, s]
            for name in ("fomo_acoustic2d", "fomo_acoustic2d_batch", "fomo_elastic2d",
                         "fomo_elastic2d_batch", "fomo_scalar2d", "fomo_debug_medium2d",
                         "fomo_set_stream", "fomo_trim", "fomo_acoustic3d", "fomo_elastic3d"):
                getattr(L, name).restype = C.c_int
            _lib = L
    return _lib


class Context:
    """One libfomo_b200 context (a stream and a reusable device workspace)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        rc = lib().fomo_create(C.byref(h), int(device))
        if rc != FOMO_OK:
            raise FomoError(rc, f"fomo_create(device={device}) failed (no usable CUDA device?)")
        self.handle = h
        self.device = device

    def check(self, rc: int) -> None:
        if rc != FOMO_OK:
            msg = lib().fomo_last_error(self.handle)
            raise FomoError(rc, msg.decode() if msg else "")

    def set_stream(self, stream_ptr: int | None) -> None:
        self.check(lib().fomo_set_stream(self.handle, C.c_void_p(stream_ptr or 0)))

    def use_torch_stream(self, stream) -> None:
        """Run on a torch stream.  torch reports its legacy default stream as 0,
        which fomo_set_stream would read as "the context's own (non-blocking)
        stream"; pass CUDA's legacy-stream handle (1) for it instead."""
        ptr = int(stream.cuda_stream)
        self.check(lib().fomo_set_stream(self.handle, C.c_void_p(ptr if ptr else 1)))

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().fomo_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order varies
        try:
            self.close()
        except Exception:
            pass


_ctx: dict[int, Context] = {}


def context(device: int = 0) -> Context:
    c = _ctx.get(device)
    if c is None:
        c = _ctx[device] = Context(device)
    return c
