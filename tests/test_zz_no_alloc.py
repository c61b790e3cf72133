"""fomo_scalar2d_noalloc: the allocation-free scalar2d entry point.

Callers that cannot allocate device memory (a plugin inside a framework whose
allocator owns all device memory, a fixed-budget service) use this entry; it
keeps its working buffers in one static 32 MiB device array.  These checks call
it through the C ABI with caller-owned device buffers and compare its
seismograms with the regular fomo_scalar2d entry point, bit for bit (the
tolerance every FP32 parity test here uses), on two calls in a row so that the
second call also proves the shared array is cleared between calls.  The file is
named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(nx=72, nz=54, nt=140, fd_order=8):
    vp = np.full((nx, nz), 3000.0, np.float32, order="F")
    vp[:, nz // 2 - 1:] = 3600.0
    rx = np.arange(4, nx - 2, 5, dtype=np.int32)
    rz = np.full(rx.size, 5, dtype=np.int32)
    return dict(vp=vp, nt=nt, fd_order=fd_order, nbc=10, sx=[nx // 2], sz=[9], rx=rx, rz=rz)


def _expected(fomo, c):
    r = fomo.scalar2d(c["vp"], 10.0, 1e-3, c["nt"], 15.0, sx=c["sx"], sz=c["sz"], rx=c["rx"],
                      rz=c["rz"], nbc=c["nbc"], fd_order=c["fd_order"], v_ref=3000.0)
    return r.seis_u


def _noalloc(fomo, c, stream_ptr=0):
    import torch

    from fomo_b200 import _lib as L
    from fomo_b200.api import scalar_wavelet_matrix

    dev = torch.device("cuda", 0)
    vp = c["vp"]
    nx, nz = vp.shape
    wm = scalar_wavelet_matrix(fomo.ricker_wavelet(15.0, 1e-3, c["nt"]), vp, 1e-3,
                               np.asarray(c["sx"]), np.asarray(c["sz"]), "v2dt2")
    d_vp = torch.from_numpy(np.ascontiguousarray(vp.T)).to(dev)
    d_w = torch.from_numpy(np.ascontiguousarray(wm.T)).to(dev)  # (nt, n_src) == (n_src, nt) F
    d_sx = torch.tensor(c["sx"], dtype=torch.int32, device=dev)
    d_sz = torch.tensor(c["sz"], dtype=torch.int32, device=dev)
    d_rx = torch.from_numpy(c["rx"]).to(dev)
    d_rz = torch.from_numpy(c["rz"]).to(dev)
    d_out = torch.full((c["nt"], c["rx"].size), float("nan"), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    g = L.Grid2D(nx, nz, 10.0, 1e-3, c["nt"], c["nbc"], c["fd_order"], 3000.0)
    acq = L.Acq(1, len(c["sx"]), d_sx.data_ptr(), d_sz.data_ptr(), d_w.data_ptr(), c["rx"].size,
                d_rx.data_ptr(), d_rz.data_ptr())
    err = C.create_string_buffer(256)
    rc = L.lib().fomo_scalar2d_noalloc(C.byref(g), d_vp.data_ptr(), C.byref(acq),
                                       d_out.data_ptr(), C.c_void_p(stream_ptr), err, 256)
    assert rc == 0, err.value.decode()
    return d_out.cpu().numpy().T  # (n_rec, nt)


def test_noalloc_matches_regular_entry_on_two_calls_in_a_row(fomo):
    c = _case()
    want = _expected(fomo, c)
    first = _noalloc(fomo, c)
    second = _noalloc(fomo, c)
    assert np.array_equal(first, want)
    assert np.array_equal(second, want)
    assert np.abs(want).max() > 0


def test_noalloc_after_a_larger_problem_and_on_a_torch_stream(fomo):
    import torch

    big = _case(nx=300, nz=220, nt=60, fd_order=10)
    _noalloc(fomo, big)  # leaves larger wavefields in the shared array
    c = _case(nx=48, nz=40, nt=90, fd_order=4)
    want = _expected(fomo, c)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        got = _noalloc(fomo, c, stream_ptr=s.cuda_stream)
    assert np.array_equal(got, want)


def test_noalloc_rejects_problems_beyond_its_array(fomo):
    from fomo_b200 import _lib as L

    g = L.Grid2D(3000, 3000, 10.0, 1e-3, 10, 50, 8, 3000.0)
    acq = L.Acq(1, 0, None, None, None, 0, None, None)
    err = C.create_string_buffer(256)
    rc = L.lib().fomo_scalar2d_noalloc(C.byref(g), C.c_void_p(16), C.byref(acq), None, None,
                                       err, 256)
    assert rc == L.FOMO_EARG
    assert b"no-alloc limit" in err.value
