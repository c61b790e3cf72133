#!/usr/bin/env python
"""Benchmark: plain-FP32 elastic2d_batch, 32 shots on a 1000x500 grid (padded
1170x670), dh 5 m, dt 0.5 ms, nt 3000, fd_order 10, nbc 80, 12 seeded layers.

One "step" is one full elastic2d_batch run of the 32-shot batch (3000 time
steps).  `value` is shots/s with model, acquisition and outputs resident in
HBM (device entry point); `e2e` is the same metric through the public API
with pinned host inputs, the H2D copies and the seismogram D2H inside the
timed region.  Multi-GPU (torchrun): the job is 32 x N shots and every rank
runs its own 32 (shots are independent, no data-path collective), time = max
over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Secondary workloads (one JSON line each, same keys; not the default line):
    --workload elastic-fp16   the same batch with binary16 wavefield storage
    --workload uneven         64 acoustic shots on grids of uneven size (graph run)
    --workload elastic3d      elastic3d 400x400x300, nbc 40, order 8 (nt from --nt;
                              --grid3d / --kernel3d: other sizes and kernel forms)
    --workload acoustic3d     acoustic3d on the same model and grid
    --slabs K                 (with elastic3d / acoustic3d) the same model split into z-slabs
                              through fomo_b200.slabs3d: K slabs sharing one GPU, or under
                              torchrun one slab per rank with NCCL halo exchange (strong
                              scaling; the multi-GPU form has not been run here)
    --workload readme         steps/s on the grids of Fomo's published throughput table
    --workload sponge         Fomo's HABC-vs-sponge benchmark (acoustic and elastic 401x401)
    --workload coupled        coupled2d on the grids of Fomo's two coupled2d demos
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
for _p in (ROOT, ROOT / "fomo.jl_b200"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

METRIC = "shots/s"
WORKLOAD = ("elastic2d_batch fp32: 32 shots, 1000x500 grid (padded 1170x670), dh 5 m, dt 0.5 ms, "
            "nt 3000, fd_order 10, nbc 80, 12 seeded layers, 500 receivers, 20 Hz Ricker")


def _traffic():
    """DRAM bytes per launch of the sweep kernel from the committed ncu summary."""
    p = ROOT / "profiles" / "traffic.txt"
    if p.exists():
        for line in p.read_text().splitlines():
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":")[1])
    return None


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.out.flush()
        rows = []
        try:
            for line in Path(self.out.name).read_text().splitlines():
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        finally:
            os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def rank_config(shots_per_rank, world, rank):
    """This rank's share of the job: the batch workload of shots_per_rank * world
    shots (sources evenly along the surface), of which rank r runs shots
    r * shots_per_rank .. (r + 1) * shots_per_rank - 1.  Shots are independent,
    so the ranks need no data-path collective (weak scaling)."""
    from fomo_b200.synthetic import elastic_batch_config

    cfg = elastic_batch_config(n_shots=shots_per_rank * world)
    lo = rank * shots_per_rank
    cfg["sx"] = cfg["sx"][lo:lo + shots_per_rank].copy()
    cfg["sz"] = cfg["sz"][lo:lo + shots_per_rank].copy()
    return cfg


def max_over_ranks(x, world, device):
    """The maximum of x over all ranks (the job's time is its slowest rank's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline(cfg, target_s=12.0, threads=None):
    """The FP32 CPU oracle (OpenMP, all host threads) on a bounded sample:
    all 32 shots for a reduced number of time steps, scaled linearly to nt."""
    from oracle import oracle as O

    O.build()
    if threads:
        O.set_threads(threads)
    cores = O.max_threads()
    ns = cfg["sx"].size
    w = np.asarray(__import__("fomo_b200").ricker_wavelet(cfg["f0"], cfg["dt"], cfg["nt"]))

    def run(nt_s):
        t0 = time.perf_counter()
        O.elastic2d(cfg["vp"], cfg["vs"], cfg["rho"], cfg["dh"], cfg["dt"], nt_s,
                    sx=cfg["sx"].reshape(1, -1), sz=cfg["sz"].reshape(1, -1), rx=cfg["rx"],
                    rz=cfg["rz"], wavelet=w[:nt_s].reshape(1, -1), nbc=cfg["nbc"],
                    fd_order=cfg["fd_order"], n_shots=ns)
        return time.perf_counter() - t0

    t = run(2)
    nt_s = int(max(2, min(cfg["nt"], round(2 * target_s / max(t, 1e-6)))))
    return nt_s, cores, run


def l2_vs_fp64(cfg, seis_vx, seis_vz, shot, nt_s, threads=None):
    """Error statement of the timed run: its seismograms of one shot (numpy
    (n_rec, nt) arrays) over the first nt_s steps against the FP64 oracle of
    the same scheme, plus whether they equal the FP32 oracle bit for bit.
    Sample k of a seismogram depends only on steps 1..k, so the first nt_s
    samples of the full run are those of an nt_s-step run."""
    from oracle import oracle as O

    O.build()
    if threads:
        O.set_threads(threads)
    w = np.asarray(__import__("fomo_b200").ricker_wavelet(cfg["f0"], cfg["dt"], nt_s))
    kw = dict(sx=[[int(cfg["sx"][shot])]], sz=[[int(cfg["sz"][shot])]], rx=cfg["rx"], rz=cfg["rz"],
              wavelet=w.reshape(1, -1), nbc=cfg["nbc"], fd_order=cfg["fd_order"])
    t0 = time.perf_counter()
    o64 = O.elastic2d(cfg["vp"], cfg["vs"], cfg["rho"], cfg["dh"], cfg["dt"], nt_s, prec=64, **kw)
    o32 = O.elastic2d(cfg["vp"], cfg["vs"], cfg["rho"], cfg["dh"], cfg["dt"], nt_s, **kw)
    t = time.perf_counter() - t0

    def rel(a, b):
        a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    gx, gz = seis_vx[:, :nt_s], seis_vz[:, :nt_s]
    return {"vx": rel(gx, o64["seis_vx"][:, :, 0]), "vz": rel(gz, o64["seis_vz"][:, :, 0]),
            "bitwise_vs_fp32_oracle": bool(np.array_equal(gx, o32["seis_vx"][:, :, 0]) and
                                           np.array_equal(gz, o32["seis_vz"][:, :, 0])),
            "shot": int(shot), "nt_sampled": int(nt_s), "tolerance": 1e-5,
            "oracle": f"C++ restatement of the scheme in FP64 and FP32 ({t:.1f} s on the host)"}


def reference_arm(args, cfg):
    world, rank, _ = _dist()
    if rank != 0:
        return
    nt_s, cores, run = cpu_baseline(cfg, target_s=6.0)
    ns = cfg["sx"].size
    for _ in range(args.warmup):
        run(nt_s)
    times = [run(nt_s) for _ in range(args.steps)]
    t = float(np.mean(times))
    value = ns / (t * cfg["nt"] / nt_s)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "shots/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * cfg["nt"] / nt_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_shots": int(ns), "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": "shots/s", "cores": cores, "kind": "port",
                         "sample": f"{ns} shots x {nt_s} of {cfg['nt']} time steps per step, "
                                   "scaled linearly; FP32 C++/OpenMP restatement of Fomo's kernels "
                                   "(Julia reference not runnable on this box)"},
        "e2e": {"value": value, "unit": "shots/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def ours(args, cfg):
    import torch

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import fomo_b200 as F
    from fomo_b200 import _lib as L
    from fomo_b200 import device as D
    from fomo_b200.api import _check_numerics, _min_pos

    ns = cfg["sx"].size
    nt = cfg["nt"]
    _check_numerics(cfg["vp"].max(), _min_pos(cfg["vp"]), np.float32(cfg["dh"]),
                    np.float32(cfg["dt"]), np.float32(cfg["f0"]), cfg["fd_order"])
    v_ref = float(_min_pos(cfg["vp"]))
    w = F.ricker_wavelet(cfg["f0"], cfg["dt"], nt)

    def dev_f32(a2d):  # (nx, nz) Fortran == (nz, nx) row-major
        return torch.from_numpy(np.ascontiguousarray(np.asarray(a2d, np.float32).T)).to(dev)

    d_vp, d_vs, d_rho = dev_f32(cfg["vp"]), dev_f32(cfg["vs"]), dev_f32(cfg["rho"])
    d_sx = torch.tensor(cfg["sx"].reshape(ns, 1), dtype=torch.int32, device=dev)
    d_sz = torch.tensor(cfg["sz"].reshape(ns, 1), dtype=torch.int32, device=dev)
    d_w = torch.from_numpy(w.reshape(nt, 1).copy()).to(dev)
    d_rx = torch.tensor(cfg["rx"], dtype=torch.int32, device=dev)
    d_rz = torch.tensor(cfg["rz"], dtype=torch.int32, device=dev)
    nrec = cfg["rx"].size
    d_svx = torch.empty((ns, nt, nrec), dtype=torch.float32, device=dev)
    d_svz = torch.empty_like(d_svx)
    kernel = int(os.environ.get("FOMO_BENCH_KERNEL", "0"))

    def step(flags=0):
        return D.elastic2d_batch(d_vp, d_vs, d_rho, dh=cfg["dh"], dt=cfg["dt"], nt=nt,
                                 nbc=cfg["nbc"], fd_order=cfg["fd_order"], v_ref=v_ref, sx=d_sx,
                                 sz=d_sz, wavelet=d_w, rx=d_rx, rz=d_rz, seis_vx=d_svx,
                                 seis_vz=d_svz, kernel=kernel, device=local, flags=flags)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    for _ in range(args.warmup):
        st = step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    sweep_ms = []
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            st = step(flags=D.PROFILE)
            launches += st.gpu_launches + 1  # + the medium-preparation kernel
            sweep_ms.append(st.sweep_ms)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, dev)
    clocks = clk.summary()
    value = ns * world / (ms * 1e-3)
    cells = st.cell_updates
    gcell = cells * world / (ms * 1e-3) / 1e9
    alg_step = st.alg_bytes / nt  # bytes per time step of the 32-shot batch
    sweep = float(np.mean(sweep_ms))
    peak, peak_kind = _peaks()
    achieved = alg_step / (sweep * 1e-3) / 1e9 if sweep > 0 else None
    finite = bool(torch.isfinite(d_svz).all().item())

    if os.environ.get("FOMO_BENCH_NO_E2E"):
        line = {"metric": METRIC, "value": value, "unit": "shots/s", "ms_per_step": ms,
                "gcell_updates_per_s": gcell, "sweep_ms_per_step": sweep,
                "roofline_frac": (achieved / peak) if achieved else None, "n_shots": int(ns),
                "nt": nt, "kernel_family": st.kernel, "clocks": clocks,
                "sweep_config": st.sweep_config}
        if rank == 0:
            print(json.dumps(line), flush=True)
        return

    # ---- e2e through the public API: pinned host inputs, D2H of the seismograms
    def pinned(a):
        t = torch.empty(a.shape[::-1], dtype=torch.float32, pin_memory=True)
        t.copy_(torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.float32).T)))
        return t.numpy().T  # Fortran-ordered (nx, nz) view of pinned memory

    h_vp, h_vs, h_rho = pinned(cfg["vp"]), pinned(cfg["vs"]), pinned(cfg["rho"])
    ctx = L.context(local)
    ctx.use_torch_stream(stream)
    kw = dict(sx=cfg["sx"], sz=cfg["sz"], rx=cfg["rx"], rz=cfg["rz"], nbc=cfg["nbc"],
              fd_order=cfg["fd_order"], device=local, kernel=kernel)
    import warnings

    with warnings.catch_warnings():
        warnings.simplefilter("ignore")  # the config is below 4 points per wavelength by design
        F.elastic2d_batch(h_vp, h_vs, h_rho, cfg["dh"], cfg["dt"], nt, cfg["f0"], **kw)
        torch.cuda.synchronize()
        barrier()
        e2 = torch.cuda.Event(enable_timing=True)
        e3 = torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        for _ in range(args.steps):
            r = F.elastic2d_batch(h_vp, h_vs, h_rho, cfg["dh"], cfg["dt"], nt, cfg["f0"], **kw)
        e3.record(stream)
        torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(e2.elapsed_time(e3) / args.steps, world, dev)
    h2d = 3 * cfg["vp"].size * 4 + nt * 4 + 4 * 2 * (ns + nrec)
    d2h = r.seis_vx.nbytes + r.seis_vz.nbytes

    line = {
        "metric": METRIC, "value": value, "unit": "shots/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_shots_per_gpu": int(ns), "global_shots": int(ns * world),
                   "padded_grid": [1170, 670], "nt": nt, "parallelism": f"shots sharded x{world}",
                   "l2": "inputs larger than L2 (1.0 GB wavefield state per GPU)",
                   "kernel_family": {1: "two-phase", 2: "single-sweep"}.get(st.kernel, str(st.kernel)),
                   "sweep_config": st.sweep_config},
        "gcell_updates_per_s": gcell,
        "e2e": {"value": ns * world / (e2e_ms * 1e-3), "unit": "shots/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "traffic": _traffic() if st.kernel == 2 else None,
                     "peak_kind": peak_kind,
                     "kernel": f"time-step sweep ({st.sweep_launches} kernel(s)/step)",
                     "alg_bytes_per_launch": alg_step / max(st.sweep_launches, 1),
                     "sweep_ms_per_step": sweep},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "finite": finite,
    }
    if rank == 0 and world == 1 and not os.environ.get("FOMO_BENCH_NO_REPLICA"):
        # the same batch through the CUDA C++ replica of Fomo's CUDA.jl step
        # (FOMO_KERNEL_REPLICA), timed on a bounded number of steps and scaled
        nt_r = min(nt, 300)
        r_vx = torch.empty((ns, nt_r, nrec), dtype=torch.float32, device=dev)
        r_vz = torch.empty_like(r_vx)

        def rep_run():
            return D.elastic2d_batch(d_vp, d_vs, d_rho, dh=cfg["dh"], dt=cfg["dt"], nt=nt_r,
                                     nbc=cfg["nbc"], fd_order=cfg["fd_order"], v_ref=v_ref,
                                     sx=d_sx, sz=d_sz, wavelet=d_w[:nt_r], rx=d_rx, rz=d_rz,
                                     seis_vx=r_vx, seis_vz=r_vz, kernel=4, device=local)

        rep_run()
        torch.cuda.synchronize()
        e4, e5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e4.record(stream)
        for _ in range(2):
            rep_run()
        e5.record(stream)
        torch.cuda.synchronize()
        rep_ms_step = e4.elapsed_time(e5) / 2 / nt_r  # per time step of the batch
        ours_ms_step = ms / nt
        same = bool(torch.equal(r_vx, d_svx[:, :nt_r]) and torch.equal(r_vz, d_svz[:, :nt_r]))
        line["replica"] = {
            "label": "replica of Fomo's CUDA.jl elastic2d_batch step, not Fomo itself",
            "value": ns / (rep_ms_step * 1e-3 * nt), "unit": "shots/s",
            "ms_per_time_step": rep_ms_step, "ours_ms_per_time_step": ours_ms_step,
            "ratio": rep_ms_step / ours_ms_step, "nt_sampled": nt_r,
            "launches_per_time_step": 8, "seismograms_equal_ours": same}
    if rank == 0 and world == 1 and not os.environ.get("FOMO_BENCH_NO_CPU"):
        # the middle shot of the timed run over its first 800 steps vs the FP64 oracle
        mid = ns // 2
        sv = d_svx[mid].T.contiguous().cpu().numpy()  # (n_rec, nt)
        szv = d_svz[mid].T.contiguous().cpu().numpy()
        line["l2_vs_fp64"] = l2_vs_fp64(cfg, sv, szv, mid, min(nt, 800))
        nt_s, cores, run = cpu_baseline(cfg)
        t = run(nt_s)
        cv = ns / (t * nt / nt_s)
        line["cpu_baseline"] = {"value": cv, "unit": "shots/s", "cores": cores, "kind": "port",
                                "sample": f"{ns} shots x {nt_s} of {nt} time steps ({t:.1f} s), "
                                          "scaled linearly; FP32 C++/OpenMP oracle"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def secondary(args):
    """Secondary workloads through the public API: `value` from the library's
    CUDA-event time of the time loop, `e2e` from torch events around the call
    (host arrays in, seismograms out)."""
    import warnings

    import torch

    import fomo_b200 as F

    warnings.simplefilter("ignore")
    world, rank, local = _dist()
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    peak, peak_kind = _peaks()
    if args.workload == "uneven":
        from fomo_b200.synthetic import uneven_batch_config

        c = uneven_batch_config(nt=args.nt if args.nt != 3000 else 2000)
        ns = len(c["vps"])
        desc = (f"acoustic2d uneven batch: {ns} shots, nx ~ logU(200,2000), nz ~ logU(200,800), "
                f"dh 10 m, dt 1 ms, nt {c['nt']}, order 8, nbc 50, GRF vp; one graph-captured run")

        def run():
            r = F.acoustic2d_uneven(c["vps"], c["rhos"], c["dh"], c["dt"], c["nt"], c["f0"],
                                    sx=c["sx"], sz=c["sz"], rx=c["rx"], rz=c["rz"], nbc=c["nbc"],
                                    fd_order=c["fd_order"], device=local)
            # the library's count, plus the medium-preparation kernel of each shot
            launches = F.api.last_stats.gpu_launches + len(c["vps"])
            return r, r.stats.kernel_time_s, r.stats.cell_updates, 36.0 * r.stats.cell_updates, launches
        unit, metric, per = "shots/s", "shots/s", ns
        h2d = sum(2 * v.nbytes for v in c["vps"])
        d2h = sum(3 * r.size * c["nt"] * 4 for r in c["rx"])
        dtype = "f32"
    elif args.workload in ("elastic3d", "acoustic3d"):
        from fomo_b200.synthetic import elastic3d_config

        el = args.workload == "elastic3d"
        g3 = [int(v) for v in args.grid3d.split(",")]
        c = elastic3d_config(*g3)
        nt = args.nt if args.nt != 3000 else 200
        pads = [v + 2 * (c["nbc"] + c["fd_order"] // 2) for v in g3]
        desc = (f"{args.workload}: {g3[0]}x{g3[1]}x{g3[2]} (padded {pads[0]}x{pads[1]}x{pads[2]}), "
                f"dh 10 m, dt 0.8 ms, nt {nt} of 2500, order 8, nbc 40, 3D GRF vp, vacuum top, "
                f"{c['rx'].size} receivers")
        kw3 = dict(sx=c["sx"], sy=c["sy"], sz=c["sz"], rx=c["rx"], ry=c["ry"], rz=c["rz"],
                   nbc=c["nbc"], fd_order=c["fd_order"], device=local, kernel=args.kernel3d)

        def run():
            if el:
                r = F.elastic3d(c["vp"], c["vs"], c["rho"], c["dh"], c["dt"], nt, c["f0"], **kw3)
            else:
                r = F.acoustic3d(c["vp"], c["rho"], c["dh"], c["dt"], nt, c["f0"], **kw3)
            s = F.api.last_stats
            return r, s.kernel_time_s, s.cell_updates, s.alg_bytes, s.gpu_launches
        unit, metric, per = "Gcell-updates/s", "Gcell-updates/s", None
        h2d = (3 if el else 2) * c["vp"].nbytes
        d2h = 3 * c["rx"].size * nt * 4
        dtype = "f32"
    else:  # elastic-fp16
        from fomo_b200.synthetic import elastic_batch_config

        c = elastic_batch_config(n_shots=args.shots)
        c["nt"] = args.nt
        ns = c["sx"].size
        desc = WORKLOAD.replace("elastic2d_batch fp32", "elastic2d_batch fp16-storage/fp32-accumulate")

        def run():
            r = F.elastic2d_batch(c["vp"], c["vs"], c["rho"], c["dh"], c["dt"], c["nt"], c["f0"],
                                  sx=c["sx"], sz=c["sz"], rx=c["rx"], rz=c["rz"], nbc=c["nbc"],
                                  fd_order=c["fd_order"], precision="fp16", device=local)
            s = F.api.last_stats
            return r, s.kernel_time_s, s.cell_updates, s.alg_bytes, s.gpu_launches
        unit, metric, per = "shots/s", "shots/s", ns
        h2d = 3 * c["vp"].nbytes
        d2h = 2 * c["rx"].size * c["nt"] * ns * 4
        dtype = "fp16-storage/f32"
    for _ in range(args.warmup):
        run()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    kt, cells, algb, launches = [], 0.0, 0.0, 0
    res = None
    with ClockSampler(local) as clk:
        ev[0].record(stream)
        for _ in range(args.steps):
            res, t, cells, algb, nl = run()
            kt.append(t)
            launches += int(nl)
        ev[1].record(stream)
        torch.cuda.synchronize()
    wall = ev[0].elapsed_time(ev[1]) / args.steps * 1e-3
    t = float(np.mean(kt))
    if per is None:
        value, e2e = cells / t / 1e9, cells / wall / 1e9
    else:
        value, e2e = per / t, per / wall
    achieved = algb / t / 1e9
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic",
            "config": {"workload": desc, "secondary": args.workload},
            "gcell_updates_per_s": cells / t / 1e9,
            "e2e": {"value": e2e, "unit": unit, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                         "kernel": "whole time loop (library CUDA events)"},
            "gpu_launches": launches, "clocks": clk.summary()}
    if rank == 0 and not os.environ.get("FOMO_BENCH_NO_CPU"):
        nt_run = c["nt"] if args.workload not in ("elastic3d", "acoustic3d") else nt
        line["l2_vs_fp64"] = secondary_l2(args.workload, c, res, nt_run)
    if rank == 0:
        print(json.dumps(line), flush=True)


def slabs_bench(args):
    """elastic3d / acoustic3d over z-slabs (fomo_b200.slabs3d).  `value`: padded
    cell-updates of the whole model / the slowest rank's device time of the time
    loop (CUDA events around the half steps and halo exchanges); `e2e`: the same
    over the whole call (slab set-up from host arrays, seismograms back)."""
    import datetime
    import warnings

    import torch
    import torch.distributed as dist

    from fomo_b200 import slabs3d
    from fomo_b200.synthetic import elastic3d_config

    warnings.simplefilter("ignore")
    world, rank, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    stream = torch.cuda.current_stream()
    peak, peak_kind = _peaks()
    el = args.workload == "elastic3d"
    g3 = [int(v) for v in args.grid3d.split(",")]
    c = elastic3d_config(*g3)
    nt = args.nt if args.nt != 3000 else 200
    n = world if world > 1 else args.slabs
    pads = [v + 2 * (c["nbc"] + c["fd_order"] // 2) for v in g3]
    cells = float(np.prod(pads)) * nt
    desc = (f"{args.workload}: {g3[0]}x{g3[1]}x{g3[2]} (padded {pads[0]}x{pads[1]}x{pads[2]}), "
            f"dh 10 m, dt 0.8 ms, nt {nt} of 2500, order 8, nbc 40, 3D GRF vp, vacuum top, "
            f"{c['rx'].size} receivers; {n} z-slabs "
            + ("one per GPU, NCCL halo exchange" if world > 1 else "on one GPU, device-copy halos"))
    kw = dict(sx=c["sx"], sy=c["sy"], sz=c["sz"], rx=c["rx"], ry=c["ry"], rz=c["rz"],
              nbc=c["nbc"], fd_order=c["fd_order"], device=local, n_slabs=n)

    def run():
        if el:
            slabs3d.elastic3d_slabs(c["vp"], c["vs"], c["rho"], c["dh"], c["dt"], nt, c["f0"], **kw)
        else:
            slabs3d.acoustic3d_slabs(c["vp"], c["rho"], c["dh"], c["dt"], nt, c["f0"], **kw)
        return dict(slabs3d.last_run)

    try:
        for _ in range(args.warmup):
            run()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        loops, launches = [], 0
        with ClockSampler(local) as clk:
            if world > 1:
                dist.barrier()
            ev[0].record(stream)
            for _ in range(args.steps):
                lr = run()
                loops.append(lr["loop_s"])
                launches += lr["gpu_launches"]
            ev[1].record(stream)
            torch.cuda.synchronize()
        wall = max_over_ranks(ev[0].elapsed_time(ev[1]) / args.steps * 1e-3, world, "cuda")
        t = max_over_ranks(float(np.mean(loops)), world, "cuda")
    finally:
        if world > 1:
            dist.destroy_process_group()
    nfield, nmat = (9, 8) if el else (4, 4)
    achieved = 4.0 * (2 * nfield + nmat) * cells / t / 1e9
    line = {"metric": "Gcell-updates/s", "value": cells / t / 1e9, "unit": "Gcell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "secondary": args.workload + "-slabs", "slabs": n},
            "e2e": {"value": cells / wall / 1e9, "unit": "Gcell-updates/s",
                    "h2d_bytes_per_step": int((3 if el else 2) * c["vp"].nbytes),
                    "d2h_bytes_per_step": int(3 * c["rx"].size * nt * 4)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak / max(world, 1), "traffic": None,
                         "peak_kind": peak_kind,
                         "kernel": "whole time loop incl. halo exchange (CUDA events)"},
            "gpu_launches": launches, "clocks": clk.summary()}
    if rank == 0 and not os.environ.get("FOMO_BENCH_NO_CPU"):
        line["l2_vs_fp64"] = secondary_l2(args.workload, c, None, nt, slabs=max(n, 2))
    if rank == 0:
        print(json.dumps(line), flush=True)


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def secondary_l2(workload, c, r, nt, slabs=0):
    """Error statement of a secondary line against the FP64 oracle of the same
    scheme: elastic-fp16 -- the middle shot's seismograms over the first
    min(nt, 1000) steps; uneven -- the smallest shot over its whole run (and
    whether it equals the FP32 oracle bit for bit); elastic3d -- a reduced grid
    (64x64x48 interior, the same dh, dt, order, nbc and model statistics, 150
    steps), since the oracle cannot run the full volume in a bench; with slabs > 0
    that grid runs as that many z-slabs on this device, and the line also says
    whether it equals the single-device run bit for bit."""
    from oracle import oracle as O

    import fomo_b200 as F

    O.build()
    t0 = time.perf_counter()
    if workload == "elastic-fp16":
        mid = c["sx"].size // 2
        k = min(nt, 1000)
        w = F.ricker_wavelet(c["f0"], c["dt"], k).reshape(1, -1)
        o = O.elastic2d(c["vp"], c["vs"], c["rho"], c["dh"], c["dt"], k, sx=[[int(c["sx"][mid])]],
                        sz=[[int(c["sz"][mid])]], rx=c["rx"], rz=c["rz"], wavelet=w, nbc=c["nbc"],
                        fd_order=c["fd_order"], prec=64)
        out = {"vx": _rel(r.seis_vx[:, :k, mid], o["seis_vx"][:, :, 0]),
               "vz": _rel(r.seis_vz[:, :k, mid], o["seis_vz"][:, :, 0]),
               "tolerance": 1e-2, "sample": f"shot {mid}, steps 1..{k}"}
    elif workload == "uneven":
        s = int(np.argmin([v.size for v in c["vps"]]))
        w = F.ricker_wavelet(c["f0"], c["dt"], nt).reshape(1, -1)
        kw = dict(sx=[c["sx"][s]], sz=[c["sz"][s]], rx=c["rx"][s], rz=c["rz"][s], wavelet=w,
                  nbc=c["nbc"], fd_order=c["fd_order"])
        o64 = O.acoustic2d(c["vps"][s], c["rhos"][s], c["dh"], c["dt"], nt, prec=64, **kw)
        o32 = O.acoustic2d(c["vps"][s], c["rhos"][s], c["dh"], c["dt"], nt, **kw)
        p = r.shots[s][0]
        out = {"p": _rel(p, o64["seis_p"][:, :, 0]),
               "bitwise_vs_fp32_oracle": bool(np.array_equal(p, o32["seis_p"][:, :, 0])),
               "tolerance": 1e-5, "sample": f"shot {s} ({c['vps'][s].shape[0]}x"
                                            f"{c['vps'][s].shape[1]}), all {nt} steps"}
    else:  # elastic3d / acoustic3d on a reduced grid of the same configuration
        from fomo_b200.synthetic import elastic3d_config

        c3 = elastic3d_config(64, 64, 48)
        k = 150
        w = F.ricker_wavelet(c3["f0"], c3["dt"], k)
        kw = dict(sx=c3["sx"], sy=c3["sy"], sz=c3["sz"], rx=c3["rx"], ry=c3["ry"], rz=c3["rz"],
                  nbc=c3["nbc"], fd_order=c3["fd_order"])
        from fomo_b200 import slabs3d

        if workload == "elastic3d":
            g = F.elastic3d(c3["vp"], c3["vs"], c3["rho"], c3["dh"], c3["dt"], k, c3["f0"], **kw)
            o = O.elastic3d(c3["vp"], c3["vs"], c3["rho"], c3["dh"], c3["dt"], k,
                            wavelet=w.reshape(1, -1), prec=64, **kw)
            if slabs:
                gs = slabs3d.elastic3d_slabs(c3["vp"], c3["vs"], c3["rho"], c3["dh"], c3["dt"], k,
                                             c3["f0"], n_slabs=slabs, **kw)
        else:
            g = F.acoustic3d(c3["vp"], c3["rho"], c3["dh"], c3["dt"], k, c3["f0"], **kw)
            o = O.acoustic3d(c3["vp"], c3["rho"], c3["dh"], c3["dt"], k,
                             wavelet=w.reshape(1, -1), prec=64, **kw)
            if slabs:
                gs = slabs3d.acoustic3d_slabs(c3["vp"], c3["rho"], c3["dh"], c3["dt"], k, c3["f0"],
                                              n_slabs=slabs, **kw)
        sample = f"64x64x48 interior, {k} steps, same dh/dt/order/nbc"
        if slabs:
            same = all(np.array_equal(gs[q], g[q]) for q in range(3))
            g = gs
            sample += f", {slabs} z-slabs on one device"
        out = {"vz": _rel(g[2], o["seis_vz"]), "vx": _rel(g[0], o["seis_vx"]),
               "tolerance": 1e-5, "sample": sample}
        if slabs:
            out["bitwise_vs_single_device"] = bool(same)
    out["oracle"] = f"C++ restatement in FP64 ({time.perf_counter() - t0:.1f} s on the host)"
    return out


# Fomo's published throughput (README.md "Performance & Reproducibility", RTX 3060,
# Float32, HABC, fd_order 8, nbc 50): steps/s per interior grid.
README_STEPS = {
    "acoustic2d": {(240, 200): 25000, (500, 400): 11800, (1000, 800): 4400, (2000, 1600): 1300},
    "scalar2d": {(240, 200): 24400, (500, 400): 23800, (1000, 800): 11800, (2000, 1600): 4100},
    "elastic2d": {(240, 200): 17000, (500, 400): 7700, (1000, 800): 2600},
}


def readme_grids(args):
    """Steps/s of the single-shot solvers on the reference's published grids, with
    the setup of its benchmark scripts (test/bench_fused.jl, bench_batch_v2.jl):
    dh 10 m, dt 1 ms, 15 Hz, vp 3000 m/s over 3800 m/s below mid-depth, rho 2200,
    vs = vp / 1.8, source at (nx/2, 8), receivers every 5th x at depth 6, nbc 50,
    order 8.  Steps/s from the library's CUDA-event time of the time loop."""
    import warnings

    import fomo_b200 as F

    warnings.simplefilter("ignore")
    nt = args.nt if args.nt != 3000 else 1000
    for eq, table in README_STEPS.items():
        for (nx, nz), ref in table.items():
            vp = np.full((nx, nz), 3000.0, np.float32, order="F")
            vp[:, nz // 2 - 1:] = 3800.0
            rho = np.full((nx, nz), 2200.0, np.float32, order="F")
            rx = np.arange(10, nx - 9, 5)
            kw = dict(sx=[nx // 2], sz=[8], rx=rx, rz=np.full(rx.size, 6), nbc=50, fd_order=8)

            def run():
                if eq == "acoustic2d":
                    return F.acoustic2d(vp, rho, 10.0, 1e-3, nt, 15.0, **kw).stats.kernel_time_s
                if eq == "scalar2d":
                    return F.scalar2d(vp, 10.0, 1e-3, nt, 15.0, **kw).stats.kernel_time_s
                vs = (vp / np.float32(1.8)).astype(np.float32)
                return F.elastic2d(vp, vs, rho, 10.0, 1e-3, nt, 15.0, **kw).stats.kernel_time_s

            for _ in range(max(1, args.warmup)):
                run()
            t = float(np.median([run() for _ in range(max(1, args.steps))]))
            sps = nt / t
            print(json.dumps({"workload": "reference README grids", "equation": eq,
                              "grid": [nx, nz], "nt": nt, "steps_per_s": sps,
                              "reference_rtx3060_steps_per_s": ref, "ratio": sps / ref,
                              "device": "B200", "dtype": "f32"}), flush=True)


# Fomo's HABC-vs-sponge benchmark (example/benchmark/habc_vs_sponge*.jl and
# output/report*.txt, RTX 3060): wall-clock of the whole call in seconds
# (including warm-up and JIT there), and the late-time interior energy.
SPONGE_BENCH = {
    "acoustic2d": dict(nt=1500, snap=30, ref_s={"habc": 9.285, "sponge": 0.504},
                       ref_energy={"habc": 3.540e-07, "sponge": 9.363e-06}),
    "elastic2d": dict(nt=2500, snap=50, ref_s={"habc": 11.581, "sponge": 1.108},
                      ref_energy={"habc": 1.470e-08, "sponge": 2.069e-06}),
}


def sponge_bench(args):
    """401x401 homogeneous model (vp 2500, vs 1500, rho 2000), dh 10 m, dt 1 ms,
    15 Hz Ricker at the centre, receivers every 2nd x at mid-depth, nbc 50,
    order 8, snapshots every `snap` steps; the same call with boundary=:habc and
    boundary=:sponge.  `wall_s`: the public call end to end (host model in,
    seismograms and snapshots out), median of --steps after --warmup calls;
    `kernel_s`: the library's CUDA-event time of the time loop.  Energy: mean over
    the last quarter of the snapshots of sum(f^2) less a 50-cell margin,
    normalised to its peak (habc_vs_sponge.jl:98-127)."""
    import time
    import warnings

    import fomo_b200 as F

    warnings.simplefilter("ignore")
    n = 401
    vp = np.full((n, n), 2500.0, np.float32, order="F")
    vs = np.full((n, n), 1500.0, np.float32, order="F")
    rho = np.full((n, n), 2000.0, np.float32, order="F")
    rx = np.arange(1, n + 1, 2)
    for eq, c in SPONGE_BENCH.items():
        kw = dict(sx=[n // 2], sz=[n // 2], rx=rx, rz=np.full(rx.size, n // 2), nbc=50,
                  fd_order=8, snap_interval=c["snap"])
        out = {}
        for bnd in ("habc", "sponge"):
            def run():
                t0 = time.perf_counter()
                if eq == "acoustic2d":
                    r = F.acoustic2d(vp, rho, 10.0, 1e-3, c["nt"], 15.0, boundary=bnd, **kw)
                else:
                    r = F.elastic2d(vp, vs, rho, 10.0, 1e-3, c["nt"], 15.0, boundary=bnd, **kw)
                return time.perf_counter() - t0, r

            for _ in range(max(1, args.warmup)):
                run()
            runs = [run() for _ in range(max(1, args.steps))]
            snaps = np.stack(runs[-1][1].snaps, axis=2)[50:-50, 50:-50].astype(np.float64)
            e = (snaps ** 2).sum(axis=(0, 1))
            e /= e.max()
            late = float(e[3 * e.size // 4 - 1:].mean())
            out[bnd] = {"wall_s": float(np.median([t for t, _ in runs])),
                        "kernel_s": float(np.median([r.stats.kernel_time_s for _, r in runs])),
                        "late_energy": late}
        line = {"workload": "reference HABC-vs-sponge benchmark", "equation": eq,
                "grid": [n, n], "nt": c["nt"], "snap_interval": c["snap"],
                "habc": out["habc"], "sponge": out["sponge"],
                "late_energy_ratio": out["sponge"]["late_energy"] / out["habc"]["late_energy"],
                "reference_rtx3060_wall_s": c["ref_s"],
                "reference_late_energy": c["ref_energy"], "device": "B200", "dtype": "f32"}
        if not args.no_cpu:
            from oracle import oracle as O

            w = np.asarray(F.ricker_wavelet(15.0, 1e-3, c["nt"]))
            okw = {k: v for k, v in kw.items() if k != "snap_interval"}

            def orun(m):
                if eq == "acoustic2d":
                    O.acoustic2d(vp, rho, 10.0, 1e-3, m, wavelet=w[None, :m], sponge_factor=0.015,
                                 **okw)
                else:
                    O.elastic2d(vp, vs, rho, 10.0, 1e-3, m, wavelet=w[None, :m],
                                sponge_factor=0.015, **okw)

            rate, m, cores = _oracle_steps_per_s(orun, c["nt"])
            line["cpu_baseline"] = {"value": c["nt"] / rate, "unit": "s (sponge run)",
                                    "cores": cores, "kind": "port",
                                    "sample": f"{m} of {c['nt']} steps scaled linearly; FP32 "
                                    "C++/OpenMP oracle with the sponge"}
        print(json.dumps(line), flush=True)


def _oracle_steps_per_s(run, nt, target_s=4.0):
    """Steps/s of an oracle run on all host threads, timed on a bounded sample:
    run(n) runs n time steps; n is sized from a 2-step probe to about target_s."""
    import time

    from oracle import oracle as O

    O.build()
    t0 = time.perf_counter()
    run(2)
    t = time.perf_counter() - t0
    n = int(max(2, min(nt, round(2 * target_s / max(t, 1e-6)))))
    t0 = time.perf_counter()
    run(n)
    return n / (time.perf_counter() - t0), n, O.max_threads()


def _coupled_demo_models():
    """The models of example/coupled2d_simple_demo.jl (400x300, two layers) and
    example/coupled2d_demo.jl (601x601, three thin scatterers)."""
    vp1 = np.full((400, 300), 2500.0, np.float32, order="F")
    vs1 = np.full((400, 300), 1200.0, np.float32, order="F")
    vp1[:, 149:] = 3500.0
    vs1[:, 149:] = 1800.0
    vp2 = np.full((601, 601), 3000.0, np.float32, order="F")
    vs2 = np.full((601, 601), 1500.0, np.float32, order="F")
    vp2[:, 149:152] = 3300.0
    vs2[:, 299:302] = 1650.0
    vp2[:, 449:452] = 3300.0
    vs2[:, 449:452] = 1650.0
    return [
        dict(name="coupled2d_simple_demo", vp=vp1, vs=vs1, dh=10.0, dt=1e-3, nt=2000, sz=10,
             snap=50),
        dict(name="coupled2d_demo", vp=vp2, vs=vs2, dh=5.0, dt=5e-4, nt=4000, sz=5, snap=100),
    ]


def coupled_bench(args):
    """coupled2d on the two demo setups: 15 Hz Ricker at (nx/2, sz), receivers
    every 2nd x at depth sz, nbc 100, order 8, snapshots of P and S.  `wall_s`:
    the public call end to end, median of --steps after --warmup calls;
    `loop_s`: the library's CUDA-event time of the time loop; `alg_gbs`: the
    algorithmic bytes of the two update kernels (80 B per padded cell and step)
    over the loop time."""
    import time
    import warnings

    import fomo_b200 as F

    warnings.simplefilter("ignore")
    peak, pkind = _peaks()
    for c in _coupled_demo_models():
        nx, nz = c["vp"].shape
        rx = np.arange(1, nx + 1, 2)
        kw = dict(sx=[nx // 2], sz=[c["sz"]], rx=rx, rz=np.full(rx.size, c["sz"]), nbc=100,
                  fd_order=8, snap_interval=c["snap"])

        def run():
            t0 = time.perf_counter()
            r = F.coupled2d(c["vp"], c["vs"], c["dh"], c["dt"], c["nt"], 15.0, **kw)
            return time.perf_counter() - t0, r, F.api.last_stats.alg_bytes

        for _ in range(max(1, args.warmup)):
            run()
        runs = [run() for _ in range(max(1, args.steps))]
        wall = float(np.median([t for t, _, _ in runs]))
        loop = float(np.median([r.stats.kernel_time_s for _, r, _ in runs]))
        gbs = runs[-1][2] / loop / 1e9
        line = {"workload": "coupled2d demo", "demo": c["name"], "grid": [nx, nz],
                "nt": c["nt"], "snap_interval": c["snap"], "wall_s": wall,
                "loop_s": loop, "steps_per_s": c["nt"] / loop, "alg_gbs": gbs,
                "hbm_frac": gbs / peak, "peak_gbs": peak, "peak_kind": pkind,
                "device": "B200", "dtype": "f32"}
        if not args.no_cpu:
            from oracle import oracle as O

            w = np.asarray(F.ricker_wavelet(15.0, c["dt"], c["nt"]))

            def orun(n):
                O.coupled2d(c["vp"], c["vs"], c["dh"], c["dt"], n, wavelet=w[None, :n], **kw)

            rate, n, cores = _oracle_steps_per_s(orun, c["nt"])
            line["cpu_baseline"] = {"value": rate, "unit": "steps/s", "cores": cores,
                                    "kind": "port", "sample": f"{n} of {c['nt']} steps; FP32 "
                                    "C++/OpenMP oracle (run_coupled2d)"}
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    # reduced cases for profiling captures (same model, fewer shots / time steps)
    ap.add_argument("--shots", type=int, default=32)
    ap.add_argument("--nt", type=int, default=3000)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--grid3d", default="400,400,300",
                    help="elastic3d workload: interior nx,ny,nz (smaller cases for profiling)")
    ap.add_argument("--kernel3d", type=int, default=0,
                    help="elastic3d workload: fomo_opts.kernel (0 auto, 1 per-cell, 2 fused, 3 z-march)")
    ap.add_argument("--slabs", type=int, default=0,
                    help="elastic3d / acoustic3d: split the model into this many z-slabs")
    ap.add_argument("--workload", choices=["elastic-batch", "elastic-fp16", "uneven", "elastic3d", "acoustic3d",
                                           "readme", "sponge", "coupled"],
                    default="elastic-batch")
    args = ap.parse_args()
    if args.workload == "coupled":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference publishes no "
                              "coupled2d timing"}))
            return
        coupled_bench(args)
        return
    if args.workload == "sponge":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference's HABC-vs-sponge "
                              "benchmark is compared against its published RTX 3060 report"}))
            return
        sponge_bench(args)
        return
    if args.workload == "readme":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference's README grids "
                              "are compared against its published RTX 3060 figures"}))
            return
        readme_grids(args)
        return
    if args.workload in ("elastic3d", "acoustic3d") and args.slabs > 0:
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no "
                              "domain-decomposed 3D solver"}))
            return
        slabs_bench(args)
        return
    if args.workload != "elastic-batch":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "reference arm is measured on "
                              "the default elastic-batch workload only"}))
            return
        secondary(args)
        return
    world, rank, _ = _dist()
    cfg = rank_config(args.shots, world, rank)
    cfg["nt"] = args.nt
    if args.no_cpu:
        os.environ["FOMO_BENCH_NO_CPU"] = "1"
    if args.no_e2e:
        os.environ["FOMO_BENCH_NO_E2E"] = "1"
    if args.impl == "reference":
        reference_arm(args, cfg)
    else:
        ours(args, cfg)


if __name__ == "__main__":
    main()
