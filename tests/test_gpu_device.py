"""The device-pointer entry (FOMO_F_DEVICE_PTRS, fomo_b200.device) against the
host API and the oracle: a single shot (injection and recording on tagged cells
inside the stress kernel, seismograms written straight to the caller's tensors)
and a two-shot batch (the separate inject/record kernel)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ns,kernel", [(1, 1), (2, 1), (2, 2)])
def test_device_entry_equals_oracle(fomo, oracle, ns, kernel):
    import torch

    from fomo_b200 import device
    from fomo_b200.synthetic import layered_elastic

    vp, vs, rho = layered_elastic(56, 40, n_layers=3, seed=21)
    nt, nbc, order = 200, 8, 8
    sx = np.array([[14], [42]][:ns], np.int32)
    sz = np.array([[6], [9]][:ns], np.int32)
    rx = np.arange(1, 57, 3).astype(np.int32)
    rz = np.full(rx.size, 5, np.int32)
    w = fomo.ricker_wavelet(20.0, 5e-4, nt)
    dev = torch.device("cuda:0")

    def t(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    svx = torch.zeros((ns, nt, rx.size), dtype=torch.float32, device=dev)
    svz = torch.zeros_like(svx)
    device.elastic2d_batch(t(vp.T), t(vs.T), t(rho.T), dh=5.0, dt=5e-4, nt=nt, nbc=nbc,
                           fd_order=order, v_ref=float(vp[vp > 0].min()), sx=t(sx), sz=t(sz),
                           wavelet=t(w.reshape(nt, 1)), rx=t(rx), rz=t(rz), seis_vx=svx,
                           seis_vz=svz, kernel=kernel)
    torch.cuda.synchronize()
    o = oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, sx=sx.T, sz=sz.T, rx=rx, rz=rz,
                         wavelet=w[None], nbc=nbc, fd_order=order, n_shots=ns)
    got_vz = svz.cpu().numpy().transpose(2, 1, 0)  # (n_rec, nt, ns)
    got_vx = svx.cpu().numpy().transpose(2, 1, 0)
    assert np.array_equal(got_vz, o["seis_vz"])
    assert np.array_equal(got_vx, o["seis_vx"])
    assert np.abs(got_vz).max() > 0
