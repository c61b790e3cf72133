"""Generate tests/golden/oracle_small.npz: small seeded oracle runs (FP32 and FP64).

The reference (Julia + CUDA.jl) cannot run in this container and ships no
golden vectors; these fixtures are regression pins of the oracle, which is
itself pinned to the reference's calibration numbers
(reference_calibration.json) by tests/test_oracle_pins.py.

    python tests/golden/make_golden.py
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "fomo.jl_b200"))


def compute(O):
    from fomo_b200.synthetic import layered_elastic, two_layer

    out = {}
    vp, rho = two_layer(50, 40)
    w = O.ricker(15.0, 1e-3, 120).reshape(1, -1)
    rx = np.arange(5, 46, 5)
    for prec in (32, 64):
        a = O.acoustic2d(vp, rho, 10.0, 1e-3, 120, sx=[25], sz=[6], rx=rx, rz=np.full(rx.size, 4),
                         wavelet=w, nbc=10, fd_order=8, snap_interval=40, prec=prec)
        out[f"ac_p_{prec}"] = a["seis_p"]
        out[f"ac_vx_{prec}"] = a["seis_vx"]
        out[f"ac_snaps_{prec}"] = a["snaps"]
    vp, vs, rhoe = layered_elastic(48, 36, n_layers=3, seed=11)
    w = O.ricker(20.0, 5e-4, 150).reshape(1, -1)
    sx = np.array([[12, 36]], dtype=np.int32)
    sz = np.array([[5, 5]], dtype=np.int32)
    rx = np.arange(2, 48, 4)
    for prec in (32, 64):
        e = O.elastic2d(vp, vs, rhoe, 5.0, 5e-4, 150, sx=sx, sz=sz, rx=rx, rz=np.full(rx.size, 5),
                        wavelet=w, nbc=8, fd_order=10, prec=prec, n_shots=2)
        out[f"el_vx_{prec}"] = e["seis_vx"]
        out[f"el_vz_{prec}"] = e["seis_vz"]
    vp = np.full((40, 30), 2800.0, np.float32)
    w = O.ricker(18.0, 1e-3, 100).reshape(1, -1)
    for prec in (32, 64):
        s = O.scalar2d(vp, 10.0, 1e-3, 100, sx=[20], sz=[5], rx=np.arange(3, 38, 5),
                       rz=np.full(7, 4), wavelet=w, nbc=9, fd_order=6, prec=prec)
        out[f"sc_u_{prec}"] = s["seis_u"]
    return out


if __name__ == "__main__":
    from oracle import oracle as O

    O.build()
    np.savez_compressed(HERE / "oracle_small.npz", **compute(O))
    print("wrote", HERE / "oracle_small.npz")
