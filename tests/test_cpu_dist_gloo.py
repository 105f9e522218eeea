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


def _render_worker(rank, world, port, out):
    """Rank `rank` renders its shard of a 6-frame sweep with the C oracle (the CPU stand-in of
    the per-GPU renderer) and the images are gathered on every rank."""
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    sys.path[:0] = [str(root), str(root / "ultrasound-3d-reconstruction_b200")]
    import torch.distributed as dist

    from oracle import ultragauss_oracle as O
    from us3d_b200 import scenes
    from us3d_b200.dist import shard_frames

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    O.set_threads(1)
    sc = scenes.make_scene(600, seed=4, cube_mm=16.0)
    sweep = scenes.linear_sweep(6, 24, 28, 0.6, seed=4, cube_mm=16.0)
    images = {}
    for f in shard_frames(len(sweep), rank, world):
        fr = sweep[f]
        geo = O.geometry(fr.origin, fr.axis_lat, fr.axis_ax, fr.axis_ele, 0.6, 0.6, 0.0, fr.lateral_col_offset)
        st = O.render(sc.means, sc.precision_tril, sc.opacities, sc.intensities, fr.pixels, geo, 24, 28)
        images[f] = st["image"].tolist()
    got = [None] * world
    dist.all_gather_object(got, images)
    dist.barrier()
    dist.destroy_process_group()
    merged = {}
    for g in got:
        merged.update(g)
    out[rank] = merged


def test_two_rank_render_union_matches_single_rank():
    import numpy as np

    from oracle import ultragauss_oracle as O
    from us3d_b200 import scenes

    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_render_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(180)
            assert p.exitcode == 0
        res = dict(out)
    O.set_threads(1)
    sc = scenes.make_scene(600, seed=4, cube_mm=16.0)
    sweep = scenes.linear_sweep(6, 24, 28, 0.6, seed=4, cube_mm=16.0)
    for r in (0, 1):
        assert sorted(res[r]) == list(range(6))
    for f, fr in enumerate(sweep):
        geo = O.geometry(fr.origin, fr.axis_lat, fr.axis_ax, fr.axis_ele, 0.6, 0.6, 0.0, fr.lateral_col_offset)
        ref = O.render(sc.means, sc.precision_tril, sc.opacities, sc.intensities, fr.pixels, geo, 24, 28)["image"]
        for r in (0, 1):
            assert np.array_equal(np.asarray(res[r][f], dtype=ref.dtype), ref), (r, f)
