"""One 3D model split into z-slabs, one per GPU (the ``fomo_slab3d_*`` entry points).

No reference counterpart: Fomo advances a 3D model on one device
(``equations/elastic3d/elastic3d.jl:37-162``, ``acoustic3d/acoustic3d.jl:37-185``).
Here the padded grid is cut into z-slabs; every slab advances its planes with
the fused half steps, and between half steps the slabs exchange halo planes.
Fields are stored x fastest, then y, then z, so each halo is one contiguous
block of whole planes: the exchange is a NCCL send/recv of plain tensor views
(``torch.distributed.batch_isend_irecv``), or a device copy between slabs that
share a device.  The seismograms of every receiver, and every owned plane of
every field, equal the single-device ``elastic3d`` / ``acoustic3d`` run bit
for bit.

Rules the library checks (``fomo_slab3d_layout_of``): cuts lie in
``[cut_min, cut_max]`` = ``[pad + 1, nzp - pad - 1]`` (pad = nbc + fd_order/2),
clear of the z bands of the Higdon boundary and of the plane each band's z
terms read; a slab with a neighbour owns at least ``fd_order // 2`` planes
(the halo depth).

Halo fields of set B = it % 2 after each half step of step ``it``:
velocity -> vx vy vz (elastic) / vz (acoustic); stress or pressure (after
injection and recording) -> txz tyz tzz (elastic) / p (acoustic).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib as L

# The last run's time loop in this process: {"loop_s": device seconds from the
# first half step to the last exchange (CUDA events on the launching stream),
# "slabs": slabs held here, "gpu_launches": library kernels launched}.
last_run: dict = {}

# fields of set B exchanged after half step `half` (0 velocity, 1 stress / pressure)
HALO_FIELDS = {
    (True, 0): (0, 1, 2),
    (True, 1): (7, 8, 5),
    (False, 0): (2,),
    (False, 1): (3,),
}


class Layout(C.Structure):
    """``fomo_slab3d_layout``."""

    _fields_ = [("nxp", C.c_int32), ("nyp", C.c_int32), ("nzp", C.c_int32), ("ld", C.c_int32),
                ("plane", C.c_int64), ("z_lo", C.c_int32), ("z_hi", C.c_int32),
                ("z_base", C.c_int32), ("nz_local", C.c_int32), ("halo", C.c_int32),
                ("nfield", C.c_int32), ("cut_min", C.c_int32), ("cut_max", C.c_int32),
                ("state_floats", C.c_int64)]


def _bind():
    lib = L.lib()
    if not getattr(lib, "_slab3d_bound", False):
        vp, i32 = C.c_void_p, C.c_int32
        g3, a3 = C.POINTER(L.Grid3D), C.POINTER(L.Acq3D)
        lib.fomo_slab3d_layout_of.argtypes = [vp, i32, g3, i32, i32, C.POINTER(Layout)]
        lib.fomo_slab3d_create.argtypes = [vp, i32, g3, vp, vp, vp, a3, i32, i32, vp,
                                           C.POINTER(vp)]
        lib.fomo_slab3d_step.argtypes = [vp, i32, i32]
        lib.fomo_slab3d_seismograms.argtypes = [vp, vp, vp, vp, vp]
        lib.fomo_slab3d_destroy.argtypes = [vp]
        lib.fomo_slab3d_destroy.restype = None
        for name in ("fomo_slab3d_layout_of", "fomo_slab3d_create", "fomo_slab3d_step",
                     "fomo_slab3d_seismograms"):
            getattr(lib, name).restype = C.c_int
        lib._slab3d_bound = True
    return lib


# ---------------------------------------------------------------------------
# host logic (no device): cuts, halo regions, the exchange schedule
# ---------------------------------------------------------------------------
def plan_cuts(nzp: int, cut_min: int, cut_max: int, halo: int, n: int) -> list[tuple[int, int]]:
    """Owned plane ranges of ``n`` slabs over ``nzp`` padded planes.

    The cuts start from the balanced ones (``round(k * nzp / n)``), are moved
    into ``[cut_min, cut_max]``, then pushed apart (forward, then backward) so
    that every slab owns at least ``halo`` planes.  Raises ``ValueError`` when
    the grid is too thin for ``n`` slabs.
    """
    if n < 1:
        raise ValueError("need at least one slab")
    if n == 1:
        return [(0, nzp)]
    gap = max(halo, 1)
    cuts = [min(max(int(round(k * nzp / n)), cut_min), cut_max) for k in range(1, n)]
    for k in range(1, n - 1):
        cuts[k] = max(cuts[k], cuts[k - 1] + gap)
    cuts[-1] = min(cuts[-1], cut_max, nzp - gap)
    for k in range(n - 3, -1, -1):
        cuts[k] = min(cuts[k], cuts[k + 1] - gap)
    bounds = [0] + cuts + [nzp]
    for a, b in zip(bounds, bounds[1:]):
        if b - a < gap or not (cut_min <= b <= cut_max or b == nzp):
            raise ValueError(f"{n} z-slabs do not fit: cuts must lie in [{cut_min}, {cut_max}] "
                             f"and each slab needs at least {max(halo, 1)} planes")
    return list(zip(bounds, bounds[1:]))


@dataclass(frozen=True)
class HaloRegion:
    """Local plane ranges of one exchange with one neighbour."""

    peer: int                   # index of the neighbouring slab
    send: tuple[int, int]       # local planes sent (owned)
    recv: tuple[int, int]       # local planes received (halo)


def halo_regions(k: int, n: int, z_lo: int, z_hi: int, z_base: int, halo: int) -> list[HaloRegion]:
    """Exchanges of slab ``k`` of ``n``: with slab k-1 (lower z) first, then k+1."""
    out = []
    lo, hi = z_lo - z_base, z_hi - z_base
    if k > 0:
        out.append(HaloRegion(k - 1, (lo, lo + halo), (lo - halo, lo)))
    if k < n - 1:
        out.append(HaloRegion(k + 1, (hi - halo, hi), (hi, hi + halo)))
    return out


def field_view(state, nfield: int, nz_local: int, plane: int, s: int, f: int):
    """Field f of set s of a slab's state tensor as (nz_local, plane)."""
    return state.view(2, nfield, nz_local, plane)[s, f]


def exchange_dist(state, nfield: int, nz_local: int, plane: int, regions: Sequence[HaloRegion],
                  ranks: Sequence[int], fields: Sequence[int], B: int, group=None) -> None:
    """Halo exchange of one slab with its neighbours over torch.distributed.

    ``ranks[k]`` is the rank holding slab k.  Every send and receive is one
    contiguous block of whole planes (no packing), posted together in one
    ``batch_isend_irecv``; the call returns when all have completed.
    """
    import torch.distributed as dist

    ops = []
    for f in fields:
        vol = field_view(state, nfield, nz_local, plane, B, f)
        for r in regions:
            ops.append(dist.P2POp(dist.isend, vol[r.send[0]:r.send[1]], ranks[r.peer], group))
            ops.append(dist.P2POp(dist.irecv, vol[r.recv[0]:r.recv[1]], ranks[r.peer], group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()


def exchange_local(slabs: Sequence["SlabLike"], fields: Sequence[int], B: int) -> None:
    """Halo exchange between slabs held by this process (device copies)."""
    n = len(slabs)
    for k, s in enumerate(slabs):
        for r in halo_regions(k, n, s.z_lo, s.z_hi, s.z_base, s.halo):
            src = slabs[r.peer]
            # the planes slab k receives are the peer's owned planes of the same global z
            p0 = r.recv[0] + s.z_base - src.z_base
            for f in fields:
                dst = field_view(s.state, s.nfield, s.nz_local, s.plane, B, f)
                sv = field_view(src.state, src.nfield, src.nz_local, src.plane, B, f)
                dst[r.recv[0]:r.recv[1]].copy_(sv[p0:p0 + (r.recv[1] - r.recv[0])])


class SlabLike:
    """What the drivers need of a slab (the library's, or a host stand-in)."""

    z_lo: int
    z_hi: int
    z_base: int
    nz_local: int
    halo: int
    nfield: int
    plane: int
    state: object  # torch tensor of 2 * nfield * nz_local * plane floats

    def step(self, it: int, half: int) -> None:  # pragma: no cover - interface
        raise NotImplementedError


def run_local(slabs: Sequence[SlabLike], elastic: bool, nt: int, it0: int = 1) -> None:
    """Steps it0..nt of slabs that share this process, exchanging halos in between."""
    for it in range(it0, nt + 1):
        for half in (0, 1):
            for s in slabs:
                s.step(it, half)
            exchange_local(slabs, HALO_FIELDS[(elastic, half)], it % 2)


def run_rank(slab: SlabLike, k: int, ranks: Sequence[int], elastic: bool, nt: int,
             group=None, it0: int = 1) -> None:
    """Steps it0..nt of slab k on this rank, exchanging halos with the neighbours."""
    n = len(ranks)
    regions = halo_regions(k, n, slab.z_lo, slab.z_hi, slab.z_base, slab.halo)
    for it in range(it0, nt + 1):
        for half in (0, 1):
            slab.step(it, half)
            exchange_dist(slab.state, slab.nfield, slab.nz_local, slab.plane, regions, ranks,
                          HALO_FIELDS[(elastic, half)], it % 2, group)


# ---------------------------------------------------------------------------
# the library's slabs
# ---------------------------------------------------------------------------
def layout(elastic: bool, grid, z_lo: int, z_hi: int, ctx: Optional[L.Context] = None) -> Layout:
    """``fomo_slab3d_layout_of`` (host only: no device work)."""
    lib = _bind()
    lay = Layout()
    rc = lib.fomo_slab3d_layout_of(ctx.handle if ctx else None, int(elastic), C.byref(grid),
                                   int(z_lo), int(z_hi), C.byref(lay))
    if rc != L.FOMO_OK:
        if ctx is not None:
            ctx.check(rc)
        raise ValueError(f"z-slab [{z_lo}, {z_hi}) refused (fomo_slab3d_layout_of {rc})")
    return lay


class Slab(SlabLike):
    """One ``fomo_slab3d``: owned planes [z_lo, z_hi) of the padded grid on one device.

    The state is a torch tensor (so NCCL can send its halo planes); the
    library's kernels run on ``ctx``'s stream, which should be torch's current
    stream on the slab's device.
    """

    def __init__(self, ctx: L.Context, elastic: bool, prep, z_lo: int, z_hi: int):
        import torch

        lib = _bind()
        lay = layout(elastic, prep.grid, z_lo, z_hi, ctx)
        self.ctx, self.elastic, self.handle = ctx, bool(elastic), None
        for name, _ in Layout._fields_:
            setattr(self, name, getattr(lay, name))
        self.n_rec, self.nt = prep.n_rec, int(prep.grid.nt)
        self.state = torch.empty(int(lay.state_floats), dtype=torch.float32,
                                 device=torch.device("cuda", ctx.device))
        h = C.c_void_p()
        vs = prep.vs if elastic else None
        ctx.check(lib.fomo_slab3d_create(
            ctx.handle, int(elastic), C.byref(prep.grid), prep.vp.ctypes.data,
            vs.ctypes.data if vs is not None else None, prep.rho.ctypes.data, C.byref(prep.acq),
            int(z_lo), int(z_hi), C.c_void_p(self.state.data_ptr()), C.byref(h)))
        self.handle = h

    def step(self, it: int, half: int) -> None:
        self.ctx.check(_bind().fomo_slab3d_step(self.handle, int(it), int(half)))

    def seismograms(self):
        """(seis_vx, seis_vy, seis_vz, owned): (n_rec, nt) arrays, other slabs' receivers 0."""
        seis = [np.zeros((self.n_rec, self.nt), dtype=np.float32, order="F") for _ in range(3)]
        owned = np.zeros(max(self.n_rec, 1), dtype=np.uint8)
        self.ctx.check(_bind().fomo_slab3d_seismograms(
            self.handle, seis[0].ctypes.data, seis[1].ctypes.data, seis[2].ctypes.data,
            owned.ctypes.data))
        return seis[0], seis[1], seis[2], owned[:self.n_rec].astype(bool)

    def owned_field(self, s: int, f: int):
        """Field f of set s over the owned planes, as a (planes, nyp, nxp) tensor."""
        v = field_view(self.state, self.nfield, self.nz_local, self.plane, s, f)
        lo, hi = self.z_lo - self.z_base, self.z_hi - self.z_base
        return v[lo:hi].view(hi - lo, self.nyp, self.ld)[:, :, :self.nxp]

    def close(self) -> None:
        if self.handle is not None:
            _bind().fomo_slab3d_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order varies
        try:
            self.close()
        except Exception:
            pass


def grid_planes(grid) -> tuple[int, int, int, int]:
    """(padded planes, lowest cut, highest cut, halo depth) of a 3D grid.

    The Higdon z bands are the first and last pad - 1 planes past the edge
    plane (pad = nbc + fd_order/2), and a band plane's z term reads the plane
    next to it on the interior side: cuts lie in [pad + 1, nzp - pad - 1]."""
    halo = int(grid.fd_order) // 2
    pad = int(grid.nbc) + halo
    nzp = int(grid.nz) + 2 * pad
    return nzp, pad + 1, nzp - pad - 1, halo


def gather_parts(part, k, n, ranks, group, dev):
    """The rank of slab 0 receives every slab's owned receivers and returns the
    assembled seismograms; the other ranks send theirs and return None.
    ``dev``: the device of the transfers (the process group's)."""
    import torch
    import torch.distributed as dist

    vx, vy, vz, owned = part
    n_rec, nt = vx.shape
    if n_rec == 0:  # nothing recorded anywhere: no transfers
        return _assemble([part]) if k == 0 else None
    if k != 0:
        mask = torch.from_numpy(owned.astype(np.uint8)).to(dev)
        dist.send(mask, ranks[0], group)
        rows = np.stack([a[owned] for a in (vx, vy, vz)])  # (3, count, nt)
        if rows.size:
            dist.send(torch.from_numpy(np.ascontiguousarray(rows)).to(dev), ranks[0], group)
        return None
    parts = [part]
    for j in range(1, n):
        mask = torch.empty(n_rec, dtype=torch.uint8, device=dev)
        dist.recv(mask, ranks[j], group)
        m = mask.cpu().numpy().astype(bool)
        cnt = int(m.sum())
        got = [np.zeros((n_rec, nt), dtype=np.float32, order="F") for _ in range(3)]
        if cnt:
            buf = torch.empty((3, cnt, nt), dtype=torch.float32, device=dev)
            dist.recv(buf, ranks[j], group)
            rows = buf.cpu().numpy()
            for q in range(3):
                got[q][m] = rows[q]
        parts.append((got[0], got[1], got[2], m))
    return _assemble(parts)


def _assemble(parts):
    """Seismograms from per-slab (vx, vy, vz, owned): each receiver from its owner."""
    out = [np.array(parts[0][k], order="F") for k in range(3)]
    for vx, vy, vz, owned in parts[1:]:
        for k, a in enumerate((vx, vy, vz)):
            out[k][owned] = a[owned]
    return tuple(out)


class _LoopTimer:
    """Device time of a slab time loop into ``last_run``."""

    def __init__(self, n_here, nt):
        import torch

        self.n_here, self.nt = n_here, nt
        self.ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def __enter__(self):
        self.ev[0].record()
        return self

    def __exit__(self, *exc):
        if exc[0] is None:
            self.ev[1].record()
            self.ev[1].synchronize()
            last_run.clear()
            last_run.update(loop_s=self.ev[0].elapsed_time(self.ev[1]) * 1e-3, slabs=self.n_here,
                            gpu_launches=3 * self.nt * self.n_here)


def _run_slabs(elastic, args, n_slabs, cuts, device, group, final_state):
    import torch
    import torch.distributed as dist

    from .api import _prep3d

    prep = _prep3d(elastic, *args)
    nt = int(prep.grid.nt)
    distributed = dist.is_available() and dist.is_initialized() and (
        dist.get_world_size(group) > 1)
    n = dist.get_world_size(group) if distributed else (
        len(cuts) if cuts is not None else int(n_slabs))
    nzp, cut_min, cut_max, halo = grid_planes(prep.grid)
    if cuts is None:
        cuts = plan_cuts(nzp, cut_min, cut_max, halo, n)
    cuts = [(int(a), int(b)) for a, b in cuts]
    if len(cuts) != n:
        raise ValueError(f"{len(cuts)} slab ranges for {n} slabs")
    if cuts[0][0] != 0 or cuts[-1][1] != nzp or any(
            cuts[k][1] != cuts[k + 1][0] for k in range(n - 1)):
        raise ValueError(f"slab ranges must tile the padded planes 0..{nzp} in order: {cuts}")
    ctx = L.Context(device)
    with torch.cuda.device(device):
        ctx.use_torch_stream(torch.cuda.current_stream(device))
        if distributed:
            k = dist.get_rank(group)
            ranks = [dist.get_global_rank(group, r) if group is not None else r for r in range(n)]
            slab = None
            try:
                slab = Slab(ctx, elastic, prep, *cuts[k])
                with _LoopTimer(1, nt):
                    run_rank(slab, k, ranks, elastic, nt, group)
                part = slab.seismograms()
                if final_state is not None:
                    final_state.append((slab.z_lo, slab.z_hi, [
                        slab.owned_field(nt % 2, f).cpu().numpy() for f in range(slab.nfield)]))
                return gather_parts(part, k, n, ranks, group, slab.state.device)
            finally:
                if slab is not None:
                    slab.close()
                ctx.close()
        slabs = []
        try:
            for lo, hi in cuts:
                slabs.append(Slab(ctx, elastic, prep, lo, hi))
            with _LoopTimer(len(slabs), nt):
                run_local(slabs, elastic, nt)
            parts = [s.seismograms() for s in slabs]
            if final_state is not None:
                for s in slabs:
                    final_state.append((s.z_lo, s.z_hi, [
                        s.owned_field(nt % 2, f).cpu().numpy() for f in range(s.nfield)]))
        finally:
            for s in slabs:
                s.close()
            ctx.close()
        return _assemble(parts)


def elastic3d_slabs(vp, vs, rho, dh, dt, nt, f0, *, sx, sy, sz, rx, ry, rz, nbc: int = 50,
                    fd_order: int = 8, v_ref=None, wavelet=None, n_slabs: int = 2,
                    cuts: Optional[Sequence[tuple[int, int]]] = None, device: int = 0,
                    group=None, final_state: Optional[list] = None):
    """``elastic3d`` (equations/elastic3d/elastic3d.jl:37-162) over z-slabs.

    Under an initialised ``torch.distributed`` group of more than one rank,
    rank k holds slab k on ``device`` and halos travel by NCCL send/recv;
    otherwise ``n_slabs`` slabs share ``device`` and exchange by device copies.
    ``cuts`` gives each slab's owned padded planes (default: balanced; given,
    it sets the number of slabs of the one-process form).
    Returns ``(seis_vx, seis_vy, seis_vz)`` equal to ``elastic3d``'s bit for
    bit (``None`` on the ranks other than slab 0's).  ``final_state``, a list,
    receives ``(z_lo, z_hi, fields)`` per slab held here: the owned planes of
    every field after the last step, each (planes, nyp, nxp).  No snapshots.
    """
    return _run_slabs(True, (vp, vs, rho, dh, dt, nt, f0, sx, sy, sz, rx, ry, rz, nbc, fd_order,
                             v_ref, wavelet), n_slabs, cuts, device, group, final_state)


def acoustic3d_slabs(vp, rho, dh, dt, nt, f0, *, sx, sy, sz, rx, ry, rz, nbc: int = 50,
                     fd_order: int = 8, v_ref=None, wavelet=None, n_slabs: int = 2,
                     cuts: Optional[Sequence[tuple[int, int]]] = None, device: int = 0,
                     group=None, final_state: Optional[list] = None):
    """``acoustic3d`` (equations/acoustic3d/acoustic3d.jl:37-185) over z-slabs;
    see ``elastic3d_slabs``."""
    return _run_slabs(False, (vp, None, rho, dh, dt, nt, f0, sx, sy, sz, rx, ry, rz, nbc,
                              fd_order, v_ref, wavelet), n_slabs, cuts, device, group,
                      final_state)
