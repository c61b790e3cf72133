"""Reduced-precision storage emulation of the oracle (no reference counterpart).

The storage rounding restates IEEE binary16 / bfloat16 round-to-nearest-even;
it is pinned here against numpy's float16 conversion and the bfloat16 bit
rule, and the storage path with FP32 storage must equal the plain FP32 run.
"""
import numpy as np

from conftest import rel_l2


def test_fp16_rounding_matches_numpy(oracle):
    rng = np.random.default_rng(0)
    x = rng.standard_normal(200000) * 10.0 ** rng.uniform(-12, 6, 200000)
    edge = [65504, 65519.99, 65520, 65535, 1e5, -7e4, 2.0 ** -24, 2.0 ** -25, 3 * 2.0 ** -26,
            2.0 ** -14, 2.0 ** -14 * (1 - 2.0 ** -11), np.inf, -np.inf, 0.0, -0.0, 1.0 + 2.0 ** -11]
    x = np.concatenate([x, edge]).astype(np.float32)
    with np.errstate(over="ignore"):
        want = x.astype(np.float16).astype(np.float32)
    got = oracle.round_store(x, "fp16")
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_bf16_rounding_rule(oracle):
    rng = np.random.default_rng(1)
    x = (rng.standard_normal(100000) * 10.0 ** rng.uniform(-30, 30, 100000)).astype(np.float32)
    x = np.concatenate([x, np.array([1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 1e-40, -1e-40],
                                    np.float32)])
    u = x.view(np.uint32).astype(np.uint64)
    want = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    got = oracle.round_store(x, "bf16").view(np.uint32)
    assert np.array_equal(got, want)


def _case(oracle, **kw):
    from fomo_b200.synthetic import layered_elastic

    vp, vs, rho = layered_elastic(60, 40, n_layers=4, seed=3)
    nt = 150
    w = oracle.ricker(20.0, 5e-4, nt).reshape(1, -1)
    return oracle.elastic2d(vp, vs, rho, 5.0, 5e-4, nt, sx=[[30]], sz=[[5]], rx=np.arange(1, 61, 3),
                            rz=np.full(20, 5), wavelet=w, nbc=10, fd_order=8, final=True, **kw)


def test_fp32_storage_path_equals_plain(oracle):
    a = _case(oracle)
    b = _case(oracle, store="fp32")
    # power-of-two scales are exact except where a value crosses the subnormal
    # range (the tiny precursor ahead of the wavefront), so scaled runs agree
    # to rounding level only
    c = _case(oracle, store="fp32", sv=2.0 ** 20, st=2.0 ** -3)
    for k in ("seis_vx", "seis_vz", "final"):
        assert np.array_equal(a[k], b[k])
        assert rel_l2(c[k], a[k]) < 1e-6


def test_fp16_storage_error_small_case(oracle):
    ref = _case(oracle, prec=64)
    h = _case(oracle, store="fp16", sv=2.0 ** 22, st=1.0, fp32_band=16)
    for k in ("seis_vx", "seis_vz"):
        e = rel_l2(h[k], ref[k])
        assert 1e-6 < e < 1e-2, (k, e)
