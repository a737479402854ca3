"""Ensembles of independent boxes.

The boxes of an ensemble share nothing, so they are advanced together: every
kernel of a step is launched once for all of them, each block finding its
box through a per-kernel tile table.  ``run_batched`` does that (one CUDA
graph per step of the whole set); ``run_plain`` advances the same boxes one
at a time to completion, with the same kernels and a graph per box.  The
ratio of the two is the benefit of batching.

Across GPUs an ensemble is sharded by box (``shard``, ``rank_share``): each
rank owns a subset and no collective is needed on the data path.
"""
from __future__ import annotations

import time

import numpy as np

from .config import BouIn
from .ic import initial_fields


def ensemble_configs(n: int = 64, seed: int = 1000) -> list[BouIn]:
    """Box sizes and physics drawn from PCG64(seed): nxm in {32, 64, 96},
    nym = nzm in {32, 48, 64, 96, 128}, aspect ratio nym/nxm clamped to
    [1, 2], Ra log-uniform in [1e5, 1e8], Pr in {0.7, 1, 4.38}."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(n):
        nxm = int(rng.choice([32, 64, 96]))
        nyz = int(rng.choice([32, 48, 64, 96, 128]))
        asp = min(max(nyz / nxm, 1.0), 2.0)
        ra = float(10 ** rng.uniform(5, 8))
        pr = float(rng.choice([0.7, 1.0, 4.38]))
        dt = 2e-4 if ra < 1e7 else 1e-4
        out.append(BouIn(nxm=nxm, nym=nyz, nzm=nyz, ylen=asp, zlen=asp, ray=ra, pra=pr, dt=dt,
                         istr3=7, idtv=0, resid=1e-10))
    return out


def cells(cfg: BouIn) -> int:
    return cfg.nxm * cfg.nym * cfg.nzm


def shard(cfgs: list, rank: int, world: int) -> list[int]:
    """Indices of the boxes rank ``rank`` owns: greedy balance of cells over
    ranks, largest boxes first (deterministic, identical on every rank)."""
    order = sorted(range(len(cfgs)), key=lambda q: (-cells(cfgs[q]), q))
    load = [0] * world
    owner = [0] * len(cfgs)
    for q in order:
        r = min(range(world), key=lambda x: (load[x], x))
        owner[q] = r
        load[r] += cells(cfgs[q])
    return [q for q in range(len(cfgs)) if owner[q] == rank]


def rank_share(per_rank: int, seed: int, rank: int, world: int) -> tuple[list, list[int]]:
    """This rank's share of one ensemble of per_rank * world boxes drawn from
    ``seed``: (configurations, their indices in the ensemble).  Every rank
    computes the same assignment without communication; a box's index is
    also the seed of its initial condition, so a box is the same whichever
    rank advances it."""
    cfgs = ensemble_configs(per_rank * world, seed=seed)
    mine = shard(cfgs, rank, world)
    return [cfgs[q] for q in mine], mine


def make_boxes(ctx, cfgs, seed0: int = 0):
    boxes = []
    for q, cfg in enumerate(cfgs):
        b = ctx.add_box(cfg)
        for k, v in initial_fields(cfg, b.xc, seed=seed0 + q).items():
            b.upload(k, v)
        boxes.append(b)
    return boxes


def reset_boxes(boxes, seed0: int = 0):
    for q, b in enumerate(boxes):
        for k, v in initial_fields(b.cfg, b.xc, seed=seed0 + q).items():
            b.upload(k, v)
        b.reset(b.cfg.dt)


def _timed(ctx, fn):
    import torch
    s = torch.cuda.ExternalStream(ctx.stream) if ctx.stream else torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ctx.synchronize()
    e0.record(s)
    fn()
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3


def run_batched(ctx, boxes, nsteps: int, graph: bool = True) -> float:
    """Seconds (device time) for nsteps of every box, batched."""
    return _timed(ctx, lambda: ctx.step(boxes, nsteps, graph=graph))


def run_plain(ctx, boxes, nsteps: int, graph: bool = True) -> float:
    """Seconds (device time) for nsteps of every box, one box at a time."""
    def go():
        for b in boxes:
            ctx.step([b], nsteps, graph=graph)
    return _timed(ctx, go)


def compare(ctx, cfgs, nsteps: int, warmup: int = 2, seed0: int = 0) -> dict:
    """Batched against plain throughput on the same boxes and steps."""
    boxes = make_boxes(ctx, cfgs, seed0)
    ncell = sum(cells(c) for c in cfgs)
    ctx.step(boxes, warmup, graph=True)
    for b in boxes:
        ctx.step([b], warmup, graph=True)
    reset_boxes(boxes, seed0)
    t_b = run_batched(ctx, boxes, nsteps)
    st_b = [b.scalars()["status"] for b in boxes]
    reset_boxes(boxes, seed0)
    t_p = run_plain(ctx, boxes, nsteps)
    for b in boxes:
        ctx.remove_box(b)
    return {"boxes": len(cfgs), "cells": ncell, "steps": nsteps,
            "batched_s": t_b, "plain_s": t_p,
            "batched_mpoint_steps_s": ncell * nsteps / t_b / 1e6,
            "plain_mpoint_steps_s": ncell * nsteps / t_p / 1e6,
            "speedup": t_p / t_b, "status": st_b,
            "when": time.strftime("%Y-%m-%dT%H:%M:%S")}


def main(argv=None) -> int:
    """``python -m afid_b200.ensemble``: advance the seeded ensemble on one
    GPU and print its device time per step (a small driver for profiling
    the batched step outside the benchmark)."""
    import argparse
    import json

    from .solver import Context
    ap = argparse.ArgumentParser(prog="python -m afid_b200.ensemble")
    ap.add_argument("--boxes", type=int, default=64)
    ap.add_argument("--seed", type=int, default=1000)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--graph", action="store_true", help="step through the per-step CUDA graph")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    cfgs = ensemble_configs(a.boxes, seed=a.seed)
    with Context(a.device) as ctx:
        boxes = make_boxes(ctx, cfgs)
        t = run_batched(ctx, boxes, a.steps, graph=a.graph)
        status = [b.scalars()["status"] for b in boxes]
        print(json.dumps({"boxes": len(cfgs), "cells": sum(cells(c) for c in cfgs), "steps": a.steps,
                          "ms_per_step": t / a.steps * 1e3, "status_ok": all(s == 0 for s in status)}))
        for b in boxes:
            ctx.remove_box(b)
    return 0 if all(s == 0 for s in status) else 1


if __name__ == "__main__":
    raise SystemExit(main())
