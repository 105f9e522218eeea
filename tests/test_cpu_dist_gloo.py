"""Multi-rank path on CPU (gloo, world size 2): each rank takes its frame shard, the union
covers every frame once, and the benchmark's max-over-ranks timing agrees on all ranks."""

from __future__ import annotations

import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    sys.path[:0] = [str(root), str(root / "ultrasound-3d-reconstruction_b200")]
    import torch
    import torch.distributed as dist

    from us3d_b200.dist import max_over_ranks, shard_frames

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    mine = shard_frames(10, rank, world)
    got = [None] * world
    dist.all_gather_object(got, mine)
    t = max_over_ranks(1.5 + rank)
    dist.barrier()
    dist.destroy_process_group()
    out[rank] = (sorted(sum(got, [])), t)


def test_two_rank_sharding_and_timing():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][0] == list(range(10)) and res[1][0] == list(range(10))
    assert res[0][1] == 2.5 and res[1][1] == 2.5
