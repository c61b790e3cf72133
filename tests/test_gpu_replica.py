"""The CUDA C++ replica of Fomo.jl's CUDA.jl elastic2d_batch step
(FOMO_KERNEL_REPLICA: batch.jl:157-183's eight launches with strip backups,
full-grid weight planes and the two-pass frame scratch) against the oracle.

It is the same-hardware baseline the bench reports beside the library's own
kernels, so it must compute the same thing: bit-identical to the FP32 oracle
(it uses the library's canonical arithmetic) and within 1e-5 relative L2 of
the FP64 oracle.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fd_order,nbc", [(2, 4), (8, 10), (10, 12)])
def test_replica_bitwise_vs_oracle(fomo, oracle, fd_order, nbc):
    from fomo_b200.synthetic import layered_elastic

    vp, vs, rho = layered_elastic(83, 61, n_layers=5, seed=31)
    vp[:, 0] = vs[:, 0] = rho[:, 0] = 0.0  # vacuum top row
    nt = 160
    rx = np.arange(1, 84, 4)
    rz = np.full(rx.size, 6)
    sx = np.array([[20], [41], [70]])  # (n_shots, n_src): distinct cells (the
    sz = np.array([[5], [30], [55]])   # reference's per-source += races on coincident ones)
    M = fd_order // 2
    fin = np.zeros((83 + 2 * (nbc + M), 61 + 2 * (nbc + M), 5, 3), np.float32, order="F")
    r = fomo.elastic2d_batch(vp, vs, rho, 5.0, 5e-4, nt, 20.0, sx=sx, sz=sz, rx=rx, rz=rz,
                             nbc=nbc, fd_order=fd_order, kernel=4, final_state=fin)
    w = fomo.ricker_wavelet(20.0, 5e-4, nt).reshape(1, -1)
    o = oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, sx=sx.T, sz=sz.T, rx=rx, rz=rz, wavelet=w,
                         nbc=nbc, fd_order=fd_order, n_shots=3, final=True)
    assert np.array_equal(r.seis_vx, o["seis_vx"])
    assert np.array_equal(r.seis_vz, o["seis_vz"])
    assert np.array_equal(fin, o["final"])
    o64 = oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, sx=sx.T, sz=sz.T, rx=rx, rz=rz,
                           wavelet=w, nbc=nbc, fd_order=fd_order, n_shots=3, prec=64)
    assert rel_l2(r.seis_vz, o64["seis_vz"]) <= 1e-5


def test_replica_rejects_other_forms(fomo):
    from fomo_b200.synthetic import two_layer

    vp, rho = two_layer(40, 30)
    with pytest.raises(Exception):
        fomo.acoustic2d(vp, rho, 10.0, 1e-3, 20, 15.0, sx=[20], sz=[5], rx=[5], rz=[5], nbc=5,
                        fd_order=4, kernel=4)
