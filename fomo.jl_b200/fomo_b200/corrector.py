"""Learned coarse-grid corrector for scalar2d (no reference counterpart).

A 3-layer 3x3 CNN (6 -> 16 -> 16 -> 1 channels, bias-free, ReLU) adds a
correction to u^{n+1} after every step of a scalar2d run on a 2x coarser grid
with a 2x larger dt.  Its inputs are u^n, u^{n-1}, c2 u^n, c2^2 u^n and, at
the source cells, the values injected in this and the previous step.  Its forward and backward passes, the training-pair
construction and the Adam update are libfomo_b200 kernels (BF16 tensor-core
implicit GEMMs with FP32 accumulation); PyTorch only holds device memory.

Training pairs come from the solver itself: a fine run (dh, dt) writes its
interior wavefield every 2 fine steps sampled on every 2nd node, i.e. on the
coarse grid and time axis (physical positions x = (i-1) dh match).  For a
coarse step n -> n+1 the target is the part of the fine u^{n+1} that the plain
coarse step (plus its injection) misses.  Fine and coarse runs model the same
physical point source: the coarse raw wavelet is the fine one times
(dh_fine / dh_coarse)^2, because a point source of strength w on a grid of
spacing dh injects w * dh^2 worth of source density.

The plain fine-grid method stays the fallback and the reference that the
error is measured against (``evaluate``).
"""
from __future__ import annotations

import ctypes as C
from typing import NamedTuple, Optional, Sequence

import numpy as np

from . import _lib as L
from .api import (ArgumentError, _check_geometry, _check_numerics, _f32F, _grid, _i32F,
                  _min_pos, _ptr, _wavelet_row, ricker_wavelet, scalar_wavelet_matrix)

PATCH = 64
# Cells within SRC_RADIUS of the source (the network's receptive field) are left
# out of the targets: there the coarse/fine difference is the point source's
# own representation on each grid, which feeds back unstably when learned.
SRC_RADIUS = 3


def _torch():
    import torch

    return torch


def param_count() -> int:
    return int(L.lib().fomo_corr_param_count())


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal W1, W2; zero W3, so an untrained corrector adds nothing."""
    rng = np.random.default_rng(seed)
    w1 = rng.standard_normal(9 * 6 * 16) * np.sqrt(2.0 / (9 * 6))
    w2 = rng.standard_normal(9 * 16 * 16) * np.sqrt(2.0 / (9 * 16))
    w3 = np.zeros(9 * 16)
    return np.concatenate([w1, w2, w3]).astype(np.float32)


def _dev_opts():
    o = L.Opts()
    o.flags = L.FOMO_F_DEVICE_PTRS
    o.precision = 0
    o.kernel = 0
    o.check_every = 0
    o.final_state = None
    return o


def _p(t) -> int:
    return int(t.data_ptr())


# ---------------------------------------------------------------------------
# device primitives
# ---------------------------------------------------------------------------
class Kernels:
    """Thin wrappers of the fomo_corr_* entry points on torch CUDA tensors."""

    def __init__(self, device: int = 0):
        torch = _torch()
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.ctx = L.context(device)
        self.np = param_count()

    def _sync_stream(self):
        self.ctx.use_torch_stream(self.torch.cuda.current_stream(self.dev))

    def features(self, u, u_prev, c2, ld, u_off, c2_off, scale, n, h, w, src=None,
                 inj_next=None, inj_prev=None, n_src=1):
        """src: (n, n_src, 2) int32 window source cells (flattened) or None;
        inj_next / inj_prev: (n, n_src) injected values."""
        feat = self.torch.empty((n, h, w, 16), dtype=self.torch.bfloat16, device=self.dev)
        opt = lambda t: _p(t) if t is not None else None  # noqa: E731
        self._sync_stream()
        self.ctx.check(L.lib().fomo_corr_features(
            self.ctx.handle, n, h, w, u, u_prev, c2, ld, _p(u_off), 0, _p(c2_off), 0, opt(scale),
            n_src if src is not None else 0, opt(src), opt(inj_next), opt(inj_prev), _p(feat)))
        return feat

    def target(self, fd_order, u, u_prev, u_next, c2, ld, u_off, c2_off, scale, src, inj, n, h, w,
               src_r=SRC_RADIUS):
        tgt = self.torch.empty((n, h, w), dtype=self.torch.float32, device=self.dev)
        mask = self.torch.empty_like(tgt)
        self._sync_stream()
        self.ctx.check(L.lib().fomo_corr_target(
            self.ctx.handle, n, h, w, fd_order, u, u_prev, u_next, c2, ld, _p(u_off), 0,
            _p(c2_off), 0, _p(scale), _p(src), _p(inj), int(src_r), _p(tgt), _p(mask)))
        return tgt, mask

    def forward(self, feat, params):
        n, h, w, _ = feat.shape
        y = self.torch.empty((n, h, w), dtype=self.torch.float32, device=self.dev)
        self._sync_stream()
        self.ctx.check(L.lib().fomo_corr_forward(self.ctx.handle, n, h, w, _p(feat), _p(params),
                                                 _p(y)))
        return y

    def gradients(self, feat, target, mask, params, y_out=None):
        n, h, w, _ = feat.shape
        grad = self.torch.empty(self.np, dtype=self.torch.float32, device=self.dev)
        loss = self.torch.empty(1, dtype=self.torch.float32, device=self.dev)
        self._sync_stream()
        self.ctx.check(L.lib().fomo_corr_gradients(
            self.ctx.handle, n, h, w, _p(feat), _p(target), _p(mask) if mask is not None else None,
            _p(params), _p(grad), _p(loss), _p(y_out) if y_out is not None else None))
        return loss, grad

    def adam(self, params, grad, m, v, lr, step, beta1=0.9, beta2=0.999, eps=1e-8):
        self._sync_stream()
        self.ctx.check(L.lib().fomo_corr_adam(self.ctx.handle, self.np, _p(params), _p(grad), _p(m),
                                              _p(v), lr, beta1, beta2, eps, step))


# ---------------------------------------------------------------------------
# solver entry points
# ---------------------------------------------------------------------------
def smooth_source(xc, zc, sigma, radius):
    """A spatially smooth source on one grid: the cells (1-based) of the square
    of half-width `radius` around (xc, zc) and their weights exp(-r^2 / (2 sigma^2)),
    r and sigma in cells of that grid.  sigma = 0 is the point source (xc, zc).

    The weights sample one physical source density, so two grids sampling the
    same physical square (the fine one with twice the cells per side and sigma,
    radius in its own cells) inject the same source: each cell adds
    v^2 dt^2 * weight * wavelet, the scalar update's discretisation of a
    distributed source term, with no area factor."""
    if sigma <= 0:
        return [int(xc)], [int(zc)], np.ones(1, np.float32)
    sx, sz, wt = [], [], []
    for dz in range(-radius, radius + 1):
        for dx in range(-radius, radius + 1):
            sx.append(int(xc + dx))
            sz.append(int(zc + dz))
            wt.append(np.exp(-(dx * dx + dz * dz) / (2.0 * sigma * sigma)))
    return sx, sz, np.asarray(wt, np.float32)


def _scalar_inputs(vp, dh, dt, nt, f0, sx, sz, rx, rz, fd_order, wavelet, source_scale,
                   wavelet_factor, weights=None):
    vp = _f32F(vp)
    nx, nz = vp.shape
    dh, dt, f0 = np.float32(dh), np.float32(dt), np.float32(f0)
    _check_geometry(nx, nz, sx, sz, rx, rz)
    _check_numerics(vp.max(), _min_pos(vp), dh, dt, f0, fd_order, centered=True)
    w = _wavelet_row(wavelet, f0, dt, nt)
    if wavelet_factor != 1.0:
        w = (w * np.float32(wavelet_factor)).astype(np.float32)
    sxv, szv = _i32F(sx).ravel(), _i32F(sz).ravel()
    wm = scalar_wavelet_matrix(w, vp, dt, sxv, szv, str(source_scale).lstrip(":"))
    if weights is not None:
        wm = np.asfortranarray((wm * np.asarray(weights, np.float32)[:, None]).astype(np.float32))
    return vp, dh, dt, sxv, szv, wm, _i32F(rx).ravel(), _i32F(rz).ravel()


def scalar2d_corrected(vp, dh, dt, nt, f0, *, params, sx, sz, rx, rz, nbc: int = 50,
                       fd_order: int = 8, v_ref=None, wavelet=None, source_scale="v2dt2",
                       wavelet_factor: float = 1.0, weights=None, device: int = 0):
    """scalar2d (equations/scalar2d/scalar2d.jl:104-189) with the learned
    correction after every step.  weights: per-source factors of the wavelet
    (a smooth source, ``smooth_source``).  Returns (seis_u, kernel_time_s)."""
    vp, dh, dt, sxv, szv, wm, rxv, rzv = _scalar_inputs(vp, dh, dt, nt, f0, sx, sz, rx, rz,
                                                        fd_order, wavelet, source_scale,
                                                        wavelet_factor, weights)
    p = np.ascontiguousarray(params, dtype=np.float32)
    if p.size != param_count():
        raise ArgumentError(f"corrector needs {param_count()} parameters, got {p.size}")
    v_ref = _min_pos(vp) if v_ref is None else np.float32(v_ref)
    seis = np.zeros((rxv.size, nt), dtype=np.float32, order="F")
    st = L.Stats()
    ctx = L.context(device)
    g = _grid(vp.shape[0], vp.shape[1], dh, dt, nt, nbc, fd_order, v_ref)
    acq = L.Acq(1, sxv.size, _ptr(sxv), _ptr(szv), _ptr(wm), rxv.size, _ptr(rxv), _ptr(rzv))
    o = L.Opts()
    ctx.check(L.lib().fomo_scalar2d_corrected(ctx.handle, C.byref(g), _ptr(vp), C.byref(acq),
                                              _ptr(p), _ptr(seis), C.byref(o), C.byref(st)))
    return seis, st.kernel_time_s


def scalar2d_sources(vp, dh, dt, nt, f0, *, sx, sz, weights, rx, rz, nbc=50, fd_order=8,
                     wavelet=None, device=0):
    """Plain scalar2d with a per-source factor on the wavelet (a smooth source);
    returns (seis_u, kernel_time_s)."""
    vp, dh, dt, sxv, szv, wm, rxv, rzv = _scalar_inputs(vp, dh, dt, nt, f0, sx, sz, rx, rz,
                                                        fd_order, wavelet, "v2dt2", 1.0, weights)
    seis = np.zeros((rxv.size, nt), dtype=np.float32, order="F")
    st = L.Stats()
    ctx = L.context(device)
    g = _grid(vp.shape[0], vp.shape[1], dh, dt, nt, nbc, fd_order, _min_pos(vp))
    acq = L.Acq(1, sxv.size, _ptr(sxv), _ptr(szv), _ptr(wm), rxv.size, _ptr(rxv), _ptr(rzv))
    o = L.Opts()
    ctx.check(L.lib().fomo_scalar2d(ctx.handle, C.byref(g), _ptr(vp), C.byref(acq), _ptr(seis),
                                    C.byref(o), C.byref(st)))
    return seis, st.kernel_time_s


def fine_snapshots(vp, dh, dt, nt, f0, *, sx, sz, nbc=50, fd_order=8, stride=2, device=0,
                   rx=None, rz=None, weights=None):
    """Fine scalar2d run whose interior wavefield is kept every `stride` steps
    on every `stride`-th node: a torch tensor (nt // stride, ceil(nz/stride),
    ceil(nx/stride)); entry k is the field after step (k+1)*stride."""
    torch = _torch()
    dev = torch.device("cuda", device)
    rx = [1] if rx is None else rx
    rz = [1] if rz is None else rz
    vp, dh, dt, sxv, szv, wm, rxv, rzv = _scalar_inputs(vp, dh, dt, nt, f0, sx, sz, rx, rz,
                                                        fd_order, None, "v2dt2", 1.0, weights)
    nx, nz = vp.shape
    mx, mz = -(-nx // stride), -(-nz // stride)
    count = (nt - stride) // stride + 1
    snaps = torch.zeros((count, mz, mx), dtype=torch.float32, device=dev)
    d = {k: torch.from_numpy(np.ascontiguousarray(v.ravel(order="F"))).to(dev)
         for k, v in dict(vp=vp, sx=sxv, sz=szv, w=wm, rx=rxv, rz=rzv).items()}
    seis = torch.zeros((rxv.size, nt), dtype=torch.float32, device=dev)
    ctx = L.context(device)
    ctx.use_torch_stream(torch.cuda.current_stream(dev))
    g = _grid(nx, nz, dh, dt, nt, nbc, fd_order, _min_pos(vp))
    acq = L.Acq(1, sxv.size, _p(d["sx"]), _p(d["sz"]), _p(d["w"]), rxv.size, _p(d["rx"]),
                _p(d["rz"]))
    o = _dev_opts()
    st = L.Stats()
    ctx.check(L.lib().fomo_scalar2d_snapshots(ctx.handle, C.byref(g), _p(d["vp"]), C.byref(acq),
                                              stride, stride, stride, _p(snaps), _p(seis),
                                              C.byref(o), C.byref(st)))
    return snaps


def coarse_c2(vp_c, dh, dt, nbc, fd_order, device=0) -> np.ndarray:
    """c2 = (vp dt / dh)^2 of the coarse interior, prepared by the solver's
    own device medium kernel (so training targets use the solver's values)."""
    from .api import debug_medium2d

    pad = nbc + fd_order // 2
    c2 = debug_medium2d("scalar", vp_c, None, None, pad, dt=dt, dh=dh, device=device)[..., 0]
    return np.ascontiguousarray(c2[pad:-pad, pad:-pad].T)  # (nz, nx), x fastest


class Pairs(NamedTuple):
    feat: object    # (n, P, P, 16) bf16
    target: object  # (n, P, P) f32
    mask: object    # (n, P, P) f32


def make_pairs(K: Kernels, snaps, c2, src_xz, w_coarse, n_pairs, fd_order, rng,
               patch=PATCH, src_r=SRC_RADIUS) -> Pairs:
    """n_pairs training windows from one fine run's coarse-sampled snapshots.
    src_xz: 0-based coarse source cells [(x, z), ...] (the first is the centre);
    w_coarse: the coarse run's injected values (n_src, nt) (already source-scaled);
    src_r: half-width of the square around the centre left out of the targets."""
    src_xz = [tuple(v) for v in np.atleast_2d(np.asarray(src_xz))]
    w_coarse = np.atleast_2d(np.asarray(w_coarse, np.float32))
    n_src = len(src_xz)
    torch = K.torch
    count, mz, mx = snaps.shape
    plane = mz * mx
    c2t = torch.from_numpy(np.ascontiguousarray(c2, dtype=np.float32)).to(K.dev)
    # steps it = c + 2 with c the index of u^n: needs u^{n-1} = c-1 >= 0 and u^{n+1} = c+1
    amp = snaps.abs().amax(dim=(1, 2))
    active = torch.nonzero(amp[1:-1] > 1e-3 * amp.max()).flatten() + 1
    if active.numel() == 0:
        raise ArgumentError("fine run has no wavefield to learn from")
    cs = active[torch.from_numpy(rng.integers(0, active.numel(), n_pairs)).to(K.dev)]
    u_off, c_off, scale, src, inj, injp = [], [], [], [], [], []
    cs_h = cs.cpu().numpy()
    for k in range(n_pairs):
        c = int(cs_h[k])
        field = snaps[c].abs()
        # window centred on a point drawn in proportion to the local amplitude
        prob = field.flatten() / field.sum()
        idx = int(torch.multinomial(prob, 1, generator=None).item())
        zc, xc = divmod(idx, mx)
        x0 = int(np.clip(xc - patch // 2, 0, mx - patch))
        z0 = int(np.clip(zc - patch // 2, 0, mz - patch))
        u_off.append(c * plane + z0 * mx + x0)
        c_off.append(z0 * mx + x0)
        win = snaps[c, z0:z0 + patch, x0:x0 + patch].abs().max().item()
        scale.append(1.0 / win if win > 0 else 0.0)
        src.append([(sx_ - x0, sz_ - z0) for sx_, sz_ in src_xz])
        inj.append(w_coarse[:, c + 1])  # injected during step it = c + 2 (index it - 1)
        injp.append(w_coarse[:, c])     # and during the previous step
    t = lambda a, dt: torch.tensor(np.asarray(a), dtype=dt, device=K.dev)  # noqa: E731
    u_off, c_off = t(u_off, torch.int64), t(c_off, torch.int64)
    scale, inj, injp = t(scale, torch.float32), t(inj, torch.float32), t(injp, torch.float32)
    src_all = np.asarray(src, dtype=np.int32)  # (n, n_src, 2)
    src = t(src_all.ravel(), torch.int32)
    centre = t(src_all[:, 0, :].ravel(), torch.int32)
    inj_c = inj[:, 0].contiguous()
    inj, injp = inj.ravel().contiguous(), injp.ravel().contiguous()
    base = _p(snaps)
    feat = K.features(base, base - 4 * plane, _p(c2t), mx, u_off, c_off, scale, n_pairs, patch,
                      patch, src=src, inj_next=inj, inj_prev=injp, n_src=n_src)
    tgt, mask = K.target(fd_order, base, base - 4 * plane, base + 4 * plane, _p(c2t), mx, u_off,
                         c_off, scale, centre, inj_c, n_pairs, patch, patch, src_r=src_r)
    torch.cuda.synchronize(K.dev)
    return Pairs(feat, tgt, mask)


def train(K: Kernels, pairs: Pairs, params: np.ndarray, *, epochs=20, batch=32, lr=1e-3, seed=0,
          log=None):
    """Adam on the masked mean-square target error; returns (params, losses).

    The per-step targets are tiny next to the wavefield (about 1e-5 of it), so
    training runs on targets scaled to unit RMS and the scale is folded back
    into the last layer afterwards (the output is linear in W3)."""
    torch = K.torch
    msum = float(pairs.mask.sum().item())
    rms = float(((pairs.target * pairs.mask) ** 2).sum().item() / max(msum, 1.0)) ** 0.5
    scale = 1.0 / rms if rms > 0 else 1.0
    p0 = np.asarray(params, dtype=np.float32).copy()
    n3 = 9 * 16
    p0[-n3:] *= np.float32(scale)
    p = torch.from_numpy(p0).to(K.dev)
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    n = pairs.feat.shape[0]
    rng = np.random.default_rng(seed)
    step, losses = 0, []
    for ep in range(epochs):
        perm = torch.from_numpy(rng.permutation(n)).to(K.dev)
        tot = 0.0
        for b0 in range(0, n - batch + 1, batch):
            idx = perm[b0:b0 + batch]
            f = pairs.feat.index_select(0, idx).contiguous()
            tg = (pairs.target.index_select(0, idx) * scale).contiguous()
            mk = pairs.mask.index_select(0, idx).contiguous()
            loss, grad = K.gradients(f, tg, mk, p)
            step += 1
            K.adam(p, grad, m, v, lr, step)
            tot += float(loss.item())
        nb = max(1, n // batch)
        losses.append(tot / nb)
        if log:
            log(f"epoch {ep + 1}: loss {losses[-1]:.4e} (unit-RMS targets)")
    out = p.cpu().numpy()
    out[-n3:] /= np.float32(scale)
    return out, losses


def one_step_error(K: Kernels, pairs: Pairs, params) -> float:
    """Masked RMS of (corrector output - target) over the pairs, relative to the
    masked RMS of the target: 1.0 for the plain coarse step (no correction)."""
    torch = K.torch
    p = torch.from_numpy(np.asarray(params, dtype=np.float32)).to(K.dev)
    num = den = 0.0
    for b0 in range(0, pairs.feat.shape[0], 64):
        f = pairs.feat[b0:b0 + 64].contiguous()
        y = K.forward(f, p)
        m = pairs.mask[b0:b0 + 64]
        t = pairs.target[b0:b0 + 64]
        num += float((((y - t) * m) ** 2).sum().item())
        den += float(((t * m) ** 2).sum().item())
    return (num / den) ** 0.5 if den > 0 else 0.0


class Workload(NamedTuple):
    vp_fine: list
    vp_coarse: list
    src: list        # coarse (sx, sz), 1-based: the source centre
    rx: np.ndarray   # coarse receivers, 1-based
    rz: np.ndarray
    src_sigma: float = 0.0  # Gaussian width in coarse cells (0: point source)
    src_radius: int = 0     # half-width of the source square in coarse cells


def workload(n_shots, nxc, nzc, seed, corr=(100.0, 400.0), vmin=1500.0, vmax=4500.0,
             dh_fine=5.0, src_sigma=0.0):
    """Learned-coarse workload: per shot a 2D Gaussian random field on the fine
    grid (2 nxc - 1) x (2 nzc - 1) (correlation length ~ U(corr), clipped to
    vmin..vmax), its coarse model on every 2nd node, a source at a random x
    at coarse depth 10 (or nzc // 4 on small grids), receivers every 2nd
    coarse x at depth 10 (or nzc // 4).  src_sigma > 0 (coarse cells) makes
    the source a smooth Gaussian patch of half-width ceil(2.5 src_sigma),
    sampled identically by both grids (``smooth_source``)."""
    from .synthetic import grf2d

    rng = np.random.default_rng(seed)
    nxf, nzf = 2 * nxc - 1, 2 * nzc - 1
    radius = int(np.ceil(2.5 * src_sigma)) if src_sigma > 0 else 0
    depth = min(10, max(4, nzc // 4))
    depth = max(depth, radius + 1)
    vf, vc, src = [], [], []
    for s in range(n_shots):
        cl = float(rng.uniform(*corr))
        v = grf2d(nxf, nzf, dh_fine, 0.5 * (vmin + vmax), (vmax - vmin) / 5.0, cl,
                  seed * 1000 + s, vmin, vmax)
        vf.append(v)
        vc.append(np.asfortranarray(v[::2, ::2]))
        src.append((int(rng.integers(max(nxc // 8, radius) + 1, nxc - max(nxc // 8, radius))),
                    depth))
    rx = np.arange(2, nxc, 2)
    return Workload(vf, vc, src, rx, np.full(rx.size, depth), float(src_sigma), radius)


def _sources(w: Workload, s: int, fine: bool):
    """Source cells (1-based) and weights of shot s on the coarse or fine grid."""
    xc, zc = w.src[s]
    if fine:
        return smooth_source(2 * xc - 1, 2 * zc - 1, 2.0 * w.src_sigma, 2 * w.src_radius)
    return smooth_source(xc, zc, w.src_sigma, w.src_radius)


def _wavelet_factor(w: Workload) -> float:
    """Coarse raw wavelet / fine raw wavelet for the same physical source: a
    point source is a one-cell density 1/dh^2, so its coarse value is
    (dh_f / dh_c)^2 = 1/4 of the fine one; a smooth source samples the same
    density on both grids (factor 1)."""
    return 1.0 if w.src_sigma > 0 else 0.25


def pairs_from_fine(K, w: Workload, shots, *, dh_c, dt_c, nt_c, f0, nbc_c, fd_order, n_pairs,
                    rng):
    """Training pairs from fine runs of the given shots (solver-generated)."""
    torch = K.torch
    parts = []
    per = max(1, n_pairs // len(shots))
    for s in shots:
        fsx, fsz, fwt = _sources(w, s, fine=True)
        csx, csz, cwt = _sources(w, s, fine=False)
        snaps = fine_snapshots(w.vp_fine[s], dh_c / 2, dt_c / 2, 2 * nt_c, f0, sx=fsx, sz=fsz,
                               nbc=2 * nbc_c, fd_order=fd_order, weights=fwt)
        c2 = coarse_c2(w.vp_coarse[s], dh_c, dt_c, nbc_c, fd_order)
        wc = ricker_wavelet(f0, dt_c, nt_c) * np.float32(_wavelet_factor(w))
        wm = scalar_wavelet_matrix(wc, w.vp_coarse[s], np.float32(dt_c), csx, csz, "v2dt2")
        wm = (wm * cwt[:, None]).astype(np.float32)
        cells = [(x - 1, z - 1) for x, z in zip(csx, csz)]
        parts.append(make_pairs(K, snaps, c2, cells, wm, per, fd_order, rng,
                                src_r=w.src_radius + SRC_RADIUS))
        del snaps
    return Pairs(torch.cat([p.feat for p in parts]), torch.cat([p.target for p in parts]),
                 torch.cat([p.mask for p in parts]))


def evaluate(w: Workload, shots, params, *, dh_c, dt_c, nt_c, f0, nbc_c, fd_order):
    """Seismogram relative L2 against the fine run at matching physical
    receivers, for the plain coarse run and the corrected one, per shot; plus
    the coarse kernel times.  Returns a list of dicts."""
    out = []
    wc = ricker_wavelet(f0, dt_c, nt_c) * np.float32(_wavelet_factor(w))
    for s in shots:
        fsx, fsz, fwt = _sources(w, s, fine=True)
        csx, csz, cwt = _sources(w, s, fine=False)
        fine, t_fine = scalar2d_sources(w.vp_fine[s], dh_c / 2, dt_c / 2, 2 * nt_c, f0, sx=fsx,
                                        sz=fsz, weights=fwt, rx=2 * w.rx - 1, rz=2 * w.rz - 1,
                                        nbc=2 * nbc_c, fd_order=fd_order)
        ref = fine[:, 1::2]
        plain, t_plain = scalar2d_sources(w.vp_coarse[s], dh_c, dt_c, nt_c, f0, sx=csx, sz=csz,
                                          weights=cwt, rx=w.rx, rz=w.rz, nbc=nbc_c,
                                          fd_order=fd_order, wavelet=wc)
        corr, t_corr = scalar2d_corrected(w.vp_coarse[s], dh_c, dt_c, nt_c, f0, params=params,
                                          sx=csx, sz=csz, rx=w.rx, rz=w.rz, nbc=nbc_c,
                                          fd_order=fd_order, wavelet=wc, weights=cwt)
        e = lambda a: float(np.linalg.norm(a - ref) / np.linalg.norm(ref))  # noqa: E731
        out.append(dict(shot=s, err_plain=e(plain), err_corrected=e(corr), t_fine=t_fine,
                        t_plain=t_plain, t_corrected=t_corr))
    return out
