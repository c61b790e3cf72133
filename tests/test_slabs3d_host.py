"""Host logic of the z-slab decomposition (fomo_b200.slabs3d), on CPU.

The cut planner, the halo regions, the library's layout rules, and the
exchange schedule: a host stand-in slab with the dependency pattern of the
fused half steps (z windows of the halo fields N planes deep, in-plane reads of
fields that are never exchanged, injection and recording on owned planes) runs
through the same drivers the library's slabs use -- run_rank / exchange_dist /
gather_parts over gloo with world size 2 and 3, and run_local -- and must equal
one slab holding the whole grid bit for bit.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "fomo.jl_b200"))
from fomo_b200 import slabs3d as S  # noqa: E402


# ---------------------------------------------------------------------------
# cuts and regions
# ---------------------------------------------------------------------------
def test_plan_cuts_balanced_and_clamped():
    assert S.plan_cuts(88, 13, 75, 4, 1) == [(0, 88)]
    assert S.plan_cuts(88, 13, 75, 4, 2) == [(0, 44), (44, 88)]
    assert S.plan_cuts(88, 13, 75, 4, 3) == [(0, 29), (29, 59), (59, 88)]
    # balanced cuts that fall in the Higdon bands move to the allowed range
    cuts = S.plan_cuts(40, 13, 27, 2, 8)
    assert all(13 <= b <= 27 for _, b in cuts[:-1])
    assert cuts[0][0] == 0 and cuts[-1][1] == 40


def test_plan_cuts_too_thin_raises():
    with pytest.raises(ValueError, match="do not fit"):
        S.plan_cuts(40, 13, 27, 4, 6)
    with pytest.raises(ValueError):
        S.plan_cuts(40, 13, 27, 4, 0)


def test_halo_regions():
    # slab 1 of 3 owning [29, 59), holding [25, 63)
    r = S.halo_regions(1, 3, 29, 59, 25, 4)
    assert r == [S.HaloRegion(0, (4, 8), (0, 4)), S.HaloRegion(2, (30, 34), (34, 38))]
    assert S.halo_regions(0, 1, 0, 88, 0, 4) == []
    # the top slab receives from below only, the bottom slab from above only
    assert [x.peer for x in S.halo_regions(0, 3, 0, 29, 0, 4)] == [1]
    assert [x.peer for x in S.halo_regions(2, 3, 59, 88, 55, 4)] == [1]


def test_library_layout_rules():
    from fomo_b200 import _lib as L

    g = L.Grid3D(40, 34, 64, 10.0, 8e-4, 10, 8, 8, 3000.0)  # pad 12, 88 planes
    assert S.grid_planes(g) == (88, 13, 75, 4)
    lay = S.layout(True, g, 29, 59)
    assert (lay.nxp, lay.nyp, lay.nzp, lay.ld) == (64, 58, 88, 64)
    assert (lay.z_base, lay.nz_local, lay.halo, lay.nfield) == (25, 38, 4, 9)
    assert (lay.cut_min, lay.cut_max) == (13, 75)
    assert lay.state_floats == 2 * 9 * 64 * 58 * 38
    top = S.layout(False, g, 0, 13)
    assert (top.z_base, top.nz_local, top.nfield) == (0, 17, 4)
    for lo, hi in ((0, 12), (76, 88), (13, 15), (-1, 20), (20, 20), (0, 89)):
        with pytest.raises(ValueError):
            S.layout(True, g, lo, hi)
    S.layout(True, g, 0, 88)  # one slab: no cut


# ---------------------------------------------------------------------------
# a host stand-in slab
# ---------------------------------------------------------------------------
PLANE, NT, H, NZP = 10, 12, 2, 40
COEF = (np.float32(0.6), np.float32(-0.05))
SRC = ((5, 3), (14, 7), (15, 1))          # (padded plane, cell)
REC = ((3, 2), (14, 4), (15, 6), (20, 0), (26, 9), (27, 5), (39, 8))


class FakeSlab(S.SlabLike):
    def __init__(self, z_lo, z_hi):
        self.z_lo, self.z_hi, self.halo, self.nfield, self.plane = z_lo, z_hi, H, 9, PLANE
        self.z_base = max(z_lo - H, 0)
        self.nz_local = min(z_hi + H, NZP) - self.z_base
        self.state = torch.zeros(2 * 9 * self.nz_local * PLANE, dtype=torch.float32)
        self.seis = np.zeros((3, len(REC), NT), dtype=np.float32)
        self.owned = np.array([z_lo <= z < z_hi for z, _ in REC])

    def _get(self, v, s, f, z):
        return v[s, f, z] if 0 <= z < self.nz_local else torch.zeros(PLANE)

    def step(self, it, half):
        v = self.state.view(2, 9, self.nz_local, PLANE)
        A, B = (it + 1) & 1, it & 1
        lo, hi = self.z_lo - self.z_base, self.z_hi - self.z_base
        if half == 0:  # velocity: z windows of txz tyz tzz, in-plane txx..
            for f, wf in zip((0, 1, 2), (7, 8, 5)):
                for z in range(lo, hi):
                    acc = torch.zeros(PLANE)
                    for l in (1, 2):
                        acc = acc + COEF[l - 1] * (self._get(v, A, wf, z + l - 1)
                                                   - self._get(v, A, wf, z - l))
                    v[B, f, z] = 0.5 * v[A, f, z] + 0.25 * torch.roll(v[A, 3 + f, z], 1) + acc
        else:  # stress: z windows of the new vx vy vz, then inject and record
            for f in range(3, 9):
                vf = (f - 3) % 3
                for z in range(lo, hi):
                    acc = torch.zeros(PLANE)
                    for l in (1, 2):
                        acc = acc + COEF[l - 1] * (self._get(v, B, vf, z + l)
                                                   - self._get(v, B, vf, z - l + 1))
                    v[B, f, z] = 0.5 * v[A, f, z] + 0.125 * torch.roll(v[A, f, z], 1) + acc
            for zs, cell in SRC:
                if self.z_lo <= zs < self.z_hi:
                    for f in (3, 4, 5):
                        v[B, f, zs - self.z_base, cell] += float(it)
            for r, (zr, cell) in enumerate(REC):
                if self.owned[r]:
                    for k in range(3):
                        self.seis[k, r, it - 1] = v[B, k, zr - self.z_base, cell]

    def seismograms(self):
        return (np.asfortranarray(self.seis[0]), np.asfortranarray(self.seis[1]),
                np.asfortranarray(self.seis[2]), self.owned.copy())

    def owned_planes(self, s, f):
        v = self.state.view(2, 9, self.nz_local, PLANE)
        return v[s, f, self.z_lo - self.z_base:self.z_hi - self.z_base].clone()


def _whole():
    w = FakeSlab(0, NZP)
    S.run_local([w], True, NT)
    return w


CUTS = {2: [(0, 15), (15, 40)], 3: [(0, 15), (15, 27), (27, 40)]}


@pytest.mark.parametrize("n", [2, 3])
def test_run_local_equals_whole(n):
    w = _whole()
    assert np.abs(w.seis).max() > 0
    slabs = [FakeSlab(lo, hi) for lo, hi in CUTS[n]]
    S.run_local(slabs, True, NT)
    got = S._assemble([s.seismograms() for s in slabs])
    for k in range(3):
        np.testing.assert_array_equal(got[k], w.seis[k])
    for s in slabs:
        for f in range(9):
            want = w.owned_planes(NT % 2, f)[s.z_lo:s.z_hi]
            assert torch.equal(s.owned_planes(NT % 2, f), want)


def test_missing_exchange_is_detected():
    # without the halo exchange the slabs drift from the whole grid: the test
    # stand-in really depends on the halos
    w = _whole()
    slabs = [FakeSlab(lo, hi) for lo, hi in CUTS[2]]
    for it in range(1, NT + 1):
        for half in (0, 1):
            for s in slabs:
                s.step(it, half)
    got = S._assemble([s.seismograms() for s in slabs])
    assert not all(np.array_equal(got[k], w.seis[k]) for k in range(3))


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        lo, hi = CUTS[world][rank]
        slab = FakeSlab(lo, hi)
        ranks = list(range(world))
        S.run_rank(slab, rank, ranks, True, NT)
        res = S.gather_parts(slab.seismograms(), rank, world, ranks, None, torch.device("cpu"))
        w = _whole()
        ok = all(torch.equal(slab.owned_planes(NT % 2, f), w.owned_planes(NT % 2, f)[lo:hi])
                 for f in range(9))
        if rank == 0:
            ok = ok and all(np.array_equal(res[k], w.seis[k]) for k in range(3))
        else:
            ok = ok and res is None
        with open(os.path.join(out_dir, f"rank{rank}"), "w") as fh:
            fh.write("ok" if ok else "mismatch")
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_run_rank_gloo_equals_whole(world, tmp_path):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert [p.exitcode for p in procs] == [0] * world
    assert [(tmp_path / f"rank{r}").read_text() for r in range(world)] == ["ok"] * world


def test_cuts_must_tile_the_grid():
    # refused on the host, before any device work
    nx, ny, nz = 12, 10, 40  # nbc 4, order 4: pad 6, 52 padded planes
    vp = np.full((nx, ny, nz), 3000.0, dtype=np.float32, order="F")
    kw = dict(sx=[6], sy=[5], sz=[3], rx=[2, 3], ry=[2, 2], rz=[3, 30], nbc=4, fd_order=4)
    for cuts in ([(0, 20), (21, 52)], [(0, 20), (20, 50)], [(1, 20), (20, 52)],
                 [(0, 30), (20, 52)]):
        with pytest.raises(ValueError, match="tile the padded planes"):
            S.acoustic3d_slabs(vp, vp, 10.0, 1e-3, 5, 15.0, cuts=cuts, **kw)
