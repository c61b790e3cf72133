"""Pin the 3D CPU oracle against an independent vectorised restatement.

The reference has no 3D test or golden vector, and its 3D Higdon kernel
(boundary/habc/kernels_3d.jl:117-193) updates in place and races, so there is
no output of it to pin against.  The oracle's C++ loops are therefore checked
here, in float64, against a second restatement written directly from the
reference's formulas with whole-array numpy slicing:
  * padding and staggered buoyancy (utils/pad_array_3d.jl:8-89),
  * Lame parameters and harmonic shear moduli (equations/elastic3d/medium.jl:73-123),
  * the staggered updates (acoustic3d/update_velocity.jl:16-53,
    update_pressure.jl:16-50; elastic3d/update_velocity.jl:17-84,
    update_stress.jl:21-94),
  * the 3D Higdon average over active directions (kernels_3d.jl:151-193)
    evaluated from read-only inputs, with the weight offsets of habc_3d.jl:40-43,
  * inject-then-record order and plane snapshots (acoustic3d.jl:134-185).
Agreement is to 1e-12 relative (the two differ only in fma contraction).
"""
import numpy as np
import pytest

from conftest import rel_l2

_FD = {
    2: [1.0],
    4: [1.125, -0.041666667],
    8: [1.1962890625, -0.079752604167, 0.0095703125, -0.000697544643],
}


def _harm2(a, b):
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where((a == 0) & (b == 0), 0.0,
                        np.where(a == 0, 2.0 / b, np.where(b == 0, 2.0 / a, 2.0 / (a + b))))


def _harm4(a, b, c, d):
    with np.errstate(divide="ignore", invalid="ignore"):
        z = (a == 0) | (b == 0) | (c == 0) | (d == 0)
        return np.where(z, 0.0, 4.0 / (1 / a + 1 / b + 1 / c + 1 / d))


def _medium(vp, vs, rho, pad):
    P = lambda a: np.pad(np.asarray(a, np.float64), pad, mode="edge")  # noqa: E731
    vp, rho = P(vp), P(rho)
    b = [np.zeros_like(rho) for _ in range(3)]
    b[0][1:] = _harm2(rho[:-1], rho[1:])
    b[0][0] = b[0][1]
    b[1][:, 1:] = _harm2(rho[:, :-1], rho[:, 1:])
    b[1][:, 0] = b[1][:, 1]
    b[2][:, :, :-1] = _harm2(rho[:, :, :-1], rho[:, :, 1:])
    b[2][:, :, -1] = b[2][:, :, -2]
    if vs is None:
        return b, rho * vp * vp
    vs = P(vs)
    mu = rho * vs * vs
    lam = rho * vp * vp - 2 * mu
    l2m = lam + 2 * mu

    def spread(m, axes):
        # fill row 1 from row 2 along axes listed as "lo", last from last-1 along "hi"
        for ax, side in axes:
            idx = [slice(None)] * 3
            src = [slice(None)] * 3
            idx[ax], src[ax] = (0, 1) if side == "lo" else (-1, -2)
            m[tuple(idx)] = m[tuple(src)]
        return m

    mxy = np.zeros_like(mu)
    mxy[1:, 1:] = _harm4(mu[:-1, :-1], mu[1:, :-1], mu[:-1, 1:], mu[1:, 1:])
    spread(mxy, [(0, "lo"), (1, "lo")])
    mxz = np.zeros_like(mu)
    mxz[1:, :, :-1] = _harm4(mu[:-1, :, :-1], mu[1:, :, :-1], mu[:-1, :, 1:], mu[1:, :, 1:])
    spread(mxz, [(0, "lo"), (2, "hi")])
    myz = np.zeros_like(mu)
    myz[:, 1:, :-1] = _harm4(mu[:, :-1, :-1], mu[:, 1:, :-1], mu[:, :-1, 1:], mu[:, 1:, 1:])
    spread(myz, [(1, "lo"), (2, "hi")])
    return b, (lam, l2m, mxy, mxz, myz)


class _Stencil:
    def __init__(self, shape, M, a):
        self.shape, self.M, self.a = shape, M, a
        self.I = tuple(slice(M, n - M) for n in shape)

    def at(self, f, ax, s):
        idx = list(self.I)
        n = self.shape[ax]
        idx[ax] = slice(self.M + s, n - self.M + s)
        return f[tuple(idx)]

    def dm(self, f, ax):  # sum a_l (f[p+l-1] - f[p-l])
        return sum(a * (self.at(f, ax, l - 1) - self.at(f, ax, -l)) for l, a in enumerate(self.a, 1))

    def dp(self, f, ax):  # sum a_l (f[p+l] - f[p-l+1])
        return sum(a * (self.at(f, ax, l) - self.at(f, ax, 1 - l)) for l, a in enumerate(self.a, 1))


class _Habc3:
    def __init__(self, shape, pad, v_ref, dt, dh):
        # habc.jl:17-44 evaluated in the oracle's working precision (float64
        # here) from the Float32 inputs and the Float32 literal 0.45f0
        r = float(np.float32(v_ref)) * float(np.float32(dt)) / float(np.float32(dh))
        b, beta = float(np.float32(0.45)), 1.0
        self.q = (b * (beta + r) - r) / ((beta + r) * (1.0 - b))
        self.qt = (b * (beta + r) - beta) / ((beta + r) * (1.0 - b))
        self.qxt = b / (b - 1.0)
        nbc = pad - 1
        grids = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
        inner = np.ones(shape, bool)
        self.sign = []
        for g, n in zip(grids, shape):
            inner &= (g >= 1) & (g <= n - 2)
            self.sign.append(np.where(g <= nbc, 1, np.where(g >= n - 1 - nbc, -1, 0)))
        self.frame = inner & ((self.sign[0] != 0) | (self.sign[1] != 0) | (self.sign[2] != 0))
        dist = np.minimum.reduce([np.minimum(g, n - 1 - g) for g, n in zip(grids, shape)])
        self.w = [np.clip((dist - off) / (pad - 1), 0.0, 1.0) for off in (0.0, 0.25, 0.5, 0.75)]

    def apply(self, f, fo, kind):
        total = np.zeros_like(f)
        nd = np.zeros(f.shape)
        for ax in range(3):
            s = self.sign[ax]
            for sgn in (1, -1):
                m = self.frame & (s == sgn)
                fnb = np.roll(f, -sgn, axis=ax)
                fonb = np.roll(fo, -sgn, axis=ax)
                side = -self.q * fnb - self.qt * fo - self.qxt * fonb
                total = np.where(m, total + side, total)
                nd += m
        w = self.w[kind]
        with np.errstate(divide="ignore", invalid="ignore"):
            val = w * f + (1 - w) * total / nd
        f[self.frame] = val[self.frame]


def _run(kind, vp, vs, rho, dh, dt, nt, src, rec, wav, nbc, fd_order, snap_every, si):
    M = fd_order // 2
    pad = nbc + M
    b, mat = _medium(vp, vs, rho, pad)
    shape = b[0].shape
    st = _Stencil(shape, M, [float(np.float32(a)) for a in _FD[fd_order]])
    vpos = np.asarray(vp, np.float64)
    h = _Habc3(shape, pad, vpos[vpos > 0].min(), dt, dh)
    dtdh = float(np.float32(dt)) / float(np.float32(dh))
    I = st.I
    nf = 9 if kind == "elastic" else 4
    F = [np.zeros(shape) for _ in range(nf)]
    seis = np.zeros((3, len(rec), nt))
    snaps = []
    for it in range(nt):
        O = [f.copy() for f in F]
        if kind == "acoustic":
            p = F[3]
            F[0][I] += b[0][I] * dtdh * st.dm(p, 0)
            F[1][I] += b[1][I] * dtdh * st.dm(p, 1)
            F[2][I] += b[2][I] * dtdh * st.dp(p, 2)
        else:
            txx, tyy, tzz, txy, txz, tyz = F[3:]
            F[0][I] += b[0][I] * dtdh * (st.dm(txx, 0) + st.dp(txy, 1) + st.dm(txz, 2))
            F[1][I] += b[1][I] * dtdh * (st.dp(txy, 0) + st.dm(tyy, 1) + st.dm(tyz, 2))
            F[2][I] += b[2][I] * dtdh * (st.dp(txz, 0) + st.dp(tyz, 1) + st.dp(tzz, 2))
        for k in range(3):
            h.apply(F[k], O[k], k)
        vx, vy, vz = F[:3]
        if kind == "acoustic":
            F[3][I] += mat[I] * dtdh * (st.dp(vx, 0) + st.dp(vy, 1) + st.dm(vz, 2))
            h.apply(F[3], O[3], 3)
            inj = [3]
        else:
            lam, l2m, mxy, mxz, myz = (m[I] for m in mat)
            dxx, dyy, dzz = st.dp(vx, 0), st.dp(vy, 1), st.dm(vz, 2)
            F[3][I] += (l2m * dxx + lam * dyy + lam * dzz) * dtdh
            F[4][I] += (lam * dxx + l2m * dyy + lam * dzz) * dtdh
            F[5][I] += (lam * dxx + lam * dyy + l2m * dzz) * dtdh
            F[6][I] += mxy * (st.dm(vx, 1) + st.dm(vy, 0)) * dtdh
            F[7][I] += mxz * (st.dp(vx, 2) + st.dm(vz, 0)) * dtdh
            F[8][I] += myz * (st.dp(vy, 2) + st.dm(vz, 1)) * dtdh
            for k in range(3, 9):
                h.apply(F[k], O[k], 3)
            inj = [3, 4, 5]
        for q, (x, y, z) in enumerate(src):
            for k in inj:
                F[k][x + pad - 1, y + pad - 1, z + pad - 1] += wav[q, it]
        for r, (x, y, z) in enumerate(rec):
            for k in range(3):
                seis[k, r, it] = F[k][x + pad - 1, y + pad - 1, z + pad - 1]
        if snap_every and (it + 1) % snap_every == 0:
            f = F[2] if kind == "elastic" else F[3]
            snaps.append(f[pad:-pad, si + pad - 1, pad:-pad].copy())
    return seis, snaps, F


@pytest.mark.parametrize("kind", ["acoustic", "elastic"])
@pytest.mark.parametrize("fd_order", [2, 4, 8])
def test_oracle3d_matches_vectorised_restatement(oracle, kind, fd_order):
    rng = np.random.default_rng(fd_order)
    nx, ny, nz, nt, nbc = 11, 9, 8, 36, 3
    vp = rng.uniform(2000, 3500, (nx, ny, nz)).astype(np.float32)
    vs = (vp / np.float32(1.8)).astype(np.float32)
    rho = rng.uniform(1800, 2600, (nx, ny, nz)).astype(np.float32)
    vp[:, :, 0] = vs[:, :, 0] = rho[:, :, 0] = 0.0  # vacuum top
    vs[2:4, 3:5, 4:6] = 0.0  # fluid pocket
    src = [(6, 5, 4), (2, 8, 7)]
    rec = [(3, 2, 2), (9, 5, 3), (6, 6, 6)]
    wav = rng.standard_normal((2, nt)).astype(np.float32)
    dh, dt = 10.0, 7e-4
    si = 4
    seis, snaps, F = _run(kind, vp, vs if kind == "elastic" else None, rho, dh, dt, nt, src, rec,
                          wav, nbc, fd_order, 12, si)
    fn = oracle.elastic3d if kind == "elastic" else oracle.acoustic3d
    args = (vp, vs, rho) if kind == "elastic" else (vp, rho)
    o = fn(*args, dh, dt, nt, sx=[s[0] for s in src], sy=[s[1] for s in src],
           sz=[s[2] for s in src], rx=[r[0] for r in rec], ry=[r[1] for r in rec],
           rz=[r[2] for r in rec], wavelet=wav, nbc=nbc, fd_order=fd_order, snap_interval=12,
           snap_index=si, prec=64, final=True)
    for k, name in enumerate(("seis_vx", "seis_vy", "seis_vz")):
        assert np.abs(o[name]).max() > 0
        assert rel_l2(o[name], seis[k]) < 1e-12, name
    for k, s in enumerate(snaps):
        assert rel_l2(o["snaps"][:, :, k], s) < 1e-12
    for k, f in enumerate(F):
        assert rel_l2(o["final"][..., k], f) < 1e-12


def test_oracle3d_fp32_close_to_fp64(oracle):
    rng = np.random.default_rng(3)
    nx, ny, nz, nt = 14, 12, 10, 80
    vp = rng.uniform(2500, 3000, (nx, ny, nz)).astype(np.float32)
    vs = (vp / np.float32(1.8)).astype(np.float32)
    rho = np.full_like(vp, 2200.0)
    w = oracle.ricker(25.0, 7e-4, nt).reshape(1, -1)
    kw = dict(sx=[7], sy=[6], sz=[5], rx=[2, 12], ry=[3, 3], rz=[2, 2], wavelet=w, nbc=4,
              fd_order=8)
    a = oracle.elastic3d(vp, vs, rho, 10.0, 7e-4, nt, prec=32, **kw)
    b = oracle.elastic3d(vp, vs, rho, 10.0, 7e-4, nt, prec=64, **kw)
    for name in ("seis_vx", "seis_vy", "seis_vz"):
        assert rel_l2(a[name], b[name]) < 1e-5
