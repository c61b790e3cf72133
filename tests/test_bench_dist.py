"""bench.py's multi-GPU host logic on two gloo ranks (CPU): shot sharding, the
max-over-ranks time, and the reference arm running on rank 0 only."""
import contextlib
import io
import os
import socket
import sys
from datetime import timedelta
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK="0")
    for p in (ROOT, ROOT / "fomo.jl_b200"):
        if str(p) not in sys.path:
            sys.path.insert(0, str(p))
    import torch
    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        cfg = bench.rank_config(4, world, rank)
        t = bench.max_over_ranks(1.5 + rank, world, torch.device("cpu"))
        out = io.StringIO()
        with contextlib.redirect_stdout(out):
            if rank != 0:  # rank 0 would time the CPU oracle here; the others must do nothing
                bench.reference_arm(type("A", (), {"gpus": world, "steps": 1, "warmup": 0})(), cfg)
        q.put((rank, cfg["sx"].tolist(), cfg["sz"].tolist(), float(cfg["vp"].sum()), t,
               out.getvalue()))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_shard_shots_and_reduce_time():
    import torch.multiprocessing as mp

    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        rank, sx, sz, vsum, t, printed = q.get(timeout=300)
        res[rank] = (sx, sz, vsum, t, printed)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sys.path.insert(0, str(ROOT / "fomo.jl_b200"))
    from fomo_b200.synthetic import elastic_batch_config

    full = elastic_batch_config(n_shots=4 * world)
    shots = [(x, z) for r in range(world) for x, z in zip(res[r][0], res[r][1])]
    # each rank runs 4 distinct shots; together they are the global set, in order
    assert all(len(res[r][0]) == 4 for r in range(world))
    assert shots == list(zip(full["sx"].tolist(), full["sz"].tolist()))
    assert len(set(shots)) == 4 * world
    # the same model everywhere; the job time is the slowest rank's on every rank
    assert res[0][2] == res[1][2] == float(np.asarray(full["vp"]).sum())
    assert res[0][3] == res[1][3] == 2.5
    assert res[1][4] == ""
