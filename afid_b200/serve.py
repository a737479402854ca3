"""Serving many RB solves on one GPU with continuous batching.

Requests (a box configuration, a step count, a seed) arrive over time.  The
scheduler admits waiting requests in arrival order while the device memory
they need (``afid_box_device_bytes``) fits the HBM budget and a slot is
free; each admitted request becomes a resident box.  All resident boxes
advance together, a chunk of steps at a time (one batched launch sequence
per step), so the work of requests that arrived at different times overlaps
on the device.  A finished or failed request leaves the batch at the end of
a chunk and frees its memory and slot for the next one.  Chunks are cut so
that no box runs past its own step count, which keeps each request's result
identical to running it alone.

``serve_plain`` runs the same stream one request at a time (the plain GPU
loop), for comparison.
"""
from __future__ import annotations

import collections
import dataclasses
import math
import time

import numpy as np

from .config import BouIn
from .ic import initial_fields
from .solver import device_bytes


@dataclasses.dataclass
class Request:
    rid: int
    cfg: BouIn
    nsteps: int
    seed: int
    arrival: float                 # seconds after the start of the stream
    admitted: float | None = None
    finished: float | None = None
    steps_done: int = 0
    status: int = 0
    result: dict | None = None
    box: object = None
    nbytes: int = 0

    @property
    def cells(self) -> int:
        return self.cfg.nxm * self.cfg.nym * self.cfg.nzm


def request_stream(n: int, rate: float, seed: int, steps: int, mix) -> list[Request]:
    """n requests with exponential inter-arrival gaps of mean 1/rate; ``mix``
    is a callable(rng) -> BouIn drawing one configuration."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = 0.0
    out = []
    for q in range(n):
        t += float(rng.exponential(1.0 / rate))
        out.append(Request(rid=q, cfg=mix(rng), nsteps=steps, seed=int(rng.integers(1 << 30)),
                           arrival=t))
    return out


def serve_mix(rng) -> BouIn:
    """Serving mix: 90% ensemble sizes, 10% nx=193, ny=nz=384; Ra log-uniform
    in [1e5, 1e9]; CFL-adaptive dt (CFL 1.2, dtmin 1e-8, dtmax 1e-2)."""
    if rng.uniform() < 0.1:
        nxm, nyz = 192, 384
    else:
        nxm = int(rng.choice([32, 64, 96]))
        nyz = int(rng.choice([32, 48, 64, 96, 128]))
    asp = min(max(nyz / nxm, 1.0), 2.0)
    ra = float(10 ** rng.uniform(5, 9))
    pr = float(rng.choice([0.7, 1.0, 4.38]))
    return BouIn(nxm=nxm, nym=nyz, nzm=nyz, ylen=asp, zlen=asp, ray=ra, pra=pr, dt=1e-8,
                 istr3=7, idtv=1, cflmax=1.2, dtmin=1e-8, dtmax=1e-2, resid=0.0)


def _admit(ctx, r: Request, now: float):
    b = ctx.add_box(r.cfg)
    for k, v in initial_fields(r.cfg, b.xc, seed=r.seed).items():
        b.upload(k, v)
    r.box = b
    r.admitted = now


def _finish(ctx, r: Request, now: float, keep_fields: bool):
    s = r.box.scalars()
    r.status = s["status"]
    hist = r.box.history(r.nsteps)
    r.result = {"scalars": s, "nu_bot": [h["nu_bot"] for h in hist],
                "nu_top": [h["nu_top"] for h in hist], "dt": [h["dt"] for h in hist]}
    if keep_fields:
        r.result["fields"] = {f: r.box.download(f) for f in ("vx", "vy", "vz", "temp", "pr")}
    r.finished = now
    ctx.remove_box(r.box)
    r.box = None


def serve(ctx, requests: list[Request], hbm_budget: int, max_slots: int = 256,
          quantum: int = 32, graph: bool = True, keep_fields: bool = False,
          realtime: bool = True) -> dict:
    """Run the stream with continuous batching.  ``realtime``: arrivals follow
    the wall clock; otherwise every request is available at once."""
    pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
    waiting: collections.deque = collections.deque()
    active: list[Request] = []
    used = 0
    chunk_lat = []           # (seconds per step, boxes in batch)
    t0 = time.perf_counter()
    clock = (lambda: time.perf_counter() - t0) if realtime else (lambda: math.inf)
    while pending or waiting or active:
        now = clock()
        while pending and pending[0].arrival <= now:
            waiting.append(pending.popleft())
        while waiting and len(active) < max_slots:
            r = waiting[0]
            r.nbytes = device_bytes(r.cfg)
            if used + r.nbytes > hbm_budget and active:
                break                               # wait for memory to free up
            if used + r.nbytes > hbm_budget:
                raise MemoryError(f"request {r.rid} needs {r.nbytes} B > budget {hbm_budget} B")
            waiting.popleft()
            _admit(ctx, r, clock() if realtime else time.perf_counter() - t0)
            used += r.nbytes
            active.append(r)
        if not active:
            if pending:
                time.sleep(max(0.0, min(pending[0].arrival - clock(), 0.01)))
            continue
        chunk = min(quantum, min(r.nsteps - r.steps_done for r in active))
        ts = time.perf_counter()
        ctx.step([r.box for r in active], chunk, graph=graph)
        ctx.synchronize()
        te = time.perf_counter()
        chunk_lat.append(((te - ts) / chunk, len(active)))
        done = []
        for r in active:
            r.steps_done += chunk
        stats = {r.rid: r.box.scalars()["status"] for r in active}
        for r in active:
            if r.steps_done >= r.nsteps or stats[r.rid] != 0:
                done.append(r)
        for r in done:
            _finish(ctx, r, te - t0, keep_fields)
            used -= r.nbytes
            active.remove(r)
    return summarize(requests, time.perf_counter() - t0, chunk_lat)


def serve_plain(ctx, requests: list[Request], graph: bool = True, keep_fields: bool = False,
                realtime: bool = True) -> dict:
    """The same stream, one request at a time in arrival order."""
    t0 = time.perf_counter()
    lat = []
    for r in sorted(requests, key=lambda r: r.arrival):
        if realtime:
            wait = r.arrival - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
        _admit(ctx, r, time.perf_counter() - t0)
        ts = time.perf_counter()
        ctx.step([r.box], r.nsteps, graph=graph)
        ctx.synchronize()
        te = time.perf_counter()
        lat.append(((te - ts) / r.nsteps, 1))
        r.steps_done = r.nsteps
        _finish(ctx, r, te - t0, keep_fields)
    return summarize(requests, time.perf_counter() - t0, lat)


def summarize(requests, makespan: float, chunk_lat) -> dict:
    comp = np.array([r.finished - r.arrival for r in requests if r.finished is not None])
    work = sum(r.cells * r.steps_done for r in requests)
    step_lat = np.array([x for x, _ in chunk_lat]) if chunk_lat else np.array([0.0])
    return {
        "requests": len(requests),
        "makespan_s": makespan,
        "mpoint_steps_s": work / makespan / 1e6,
        "p50_completion_s": float(np.percentile(comp, 50)) if comp.size else None,
        "p99_completion_s": float(np.percentile(comp, 99)) if comp.size else None,
        "p50_step_latency_ms": float(np.percentile(step_lat, 50) * 1e3),
        "p99_step_latency_ms": float(np.percentile(step_lat, 99) * 1e3),
        "failed": sum(1 for r in requests if r.status != 0),
        "mean_batch": float(np.mean([n for _, n in chunk_lat])) if chunk_lat else 0.0,
    }
