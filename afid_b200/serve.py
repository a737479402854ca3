"""Serving many RB solves on one GPU with continuous batching.

Requests (a box configuration, a step count, a seed) arrive over time.  The
scheduler admits waiting requests in arrival order while the device memory
they need (``afid_box_device_bytes``) fits the HBM budget and a slot is
free; each admitted request becomes a resident box whose step target is a
device-side hold (``Box.set_stop``).  All resident boxes advance together,
``quantum`` steps at a time (one CUDA graph launch per step of the whole
set); a box that reaches its target is held by the device, so the other
boxes keep their full chunk and each result is the one the request gets when
run alone.  While a chunk runs on the compute stream, the host admits the
next requests on a second stream (initial fields, box creation, uploads);
after the chunk, finished and failed requests leave the set and free their
memory, and the admitted ones join it.

``serve_plain`` runs the same stream one request at a time (the plain GPU
loop), for comparison.  ``shard_requests`` routes a stream over ranks
(each GPU serves its share; no collective on the data path).
"""
from __future__ import annotations

import collections
import dataclasses
import math
import time

import numpy as np

from . import _lib
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
                 istr3=7, idtv=1, cflmax=1.2, dtmin=1e-8, dtmax=1e-2, resid=1e-10)


def shard_requests(requests: list[Request], rank: int, world: int) -> list[Request]:
    """The requests rank ``rank`` serves: greedy balance of work (cells x
    steps) in arrival order, each request to the least-loaded rank.  The
    routing is deterministic, so every rank computes it without
    communication."""
    load = [0] * world
    mine = []
    for r in sorted(requests, key=lambda r: (r.arrival, r.rid)):
        dst = min(range(world), key=lambda x: (load[x], x))
        load[dst] += r.cells * r.nsteps
        if dst == rank:
            mine.append(r)
    return mine


def _admit(ctx, r: Request, now: float):
    b = ctx.add_box(r.cfg)
    for k, v in initial_fields(r.cfg, b.xc, seed=r.seed).items():
        b.upload(k, v)
    b.set_stop(r.nsteps)
    r.box = b
    r.admitted = now


def _finish(ctx, r: Request, now: float, keep_fields: bool):
    s = r.box.scalars()
    r.status = 0 if s["status"] == _lib.STATUS_HELD else s["status"]
    r.steps_done = s["ntime"]
    hist = r.box.history(r.nsteps)
    r.result = {"scalars": s, "nu_bot": [h["nu_bot"] for h in hist],
                "nu_top": [h["nu_top"] for h in hist], "dt": [h["dt"] for h in hist]}
    if keep_fields:
        r.result["fields"] = {f: r.box.download(f) for f in ("vx", "vy", "vz", "temp", "pr")}
    r.finished = now
    ctx.remove_box(r.box)
    r.box = None


class _Streams:
    """The compute stream (the context's own) and an admission stream, with
    an event to ask whether the chunk on the compute stream has finished."""

    def __init__(self, ctx):
        import torch
        self.torch = torch
        self.ctx = ctx
        self.compute = ctx.stream
        self.admit = torch.cuda.Stream(device=ctx.device)
        self.ev = None

    def launched(self):
        s = self.torch.cuda.ExternalStream(self.compute, device=self.ctx.device)
        self.ev = self.torch.cuda.Event()
        self.ev.record(s)

    def busy(self) -> bool:
        return self.ev is not None and not self.ev.query()

    def to_admit(self):
        self.ctx.set_stream(self.admit.cuda_stream)

    def to_compute(self):
        self.ctx.set_stream(self.compute)


def serve(ctx, requests: list[Request], hbm_budget: int, max_slots: int = 256,
          quantum: int = 32, graph: bool = True, keep_fields: bool = False,
          realtime: bool = True) -> dict:
    """Run the stream with continuous batching.  ``realtime``: arrivals follow
    the wall clock; otherwise every request is available at once."""
    pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
    waiting: collections.deque = collections.deque()
    active: list[Request] = []
    staged: list[Request] = []
    used = 0
    chunk_lat = []           # (seconds per step, boxes in batch)
    st = _Streams(ctx)
    t0 = time.perf_counter()
    clock = (lambda: time.perf_counter() - t0) if realtime else (lambda: math.inf)
    stamp = lambda: time.perf_counter() - t0

    def admit_some(only_while_busy: bool):
        nonlocal used
        st.to_admit()
        try:
            while waiting and len(active) + len(staged) < max_slots:
                if only_while_busy and not st.busy():
                    break
                r = waiting[0]
                r.nbytes = device_bytes(r.cfg)
                if used + r.nbytes > hbm_budget:
                    if active or staged:
                        break                       # wait for memory to free up
                    raise MemoryError(f"request {r.rid} needs {r.nbytes} B > budget {hbm_budget} B")
                waiting.popleft()
                _admit(ctx, r, stamp())
                used += r.nbytes
                staged.append(r)
        finally:
            st.to_compute()

    while pending or waiting or active or staged:
        now = clock()
        while pending and pending[0].arrival <= now:
            waiting.append(pending.popleft())
        if not active:
            admit_some(only_while_busy=False)
            active, staged = staged, []
            if not active:
                if pending:
                    time.sleep(max(0.0, min(pending[0].arrival - clock(), 0.01)))
                continue
        ts = time.perf_counter()
        ctx.step([r.box for r in active], quantum, graph=graph)
        st.launched()
        # admission overlaps the chunk
        now = clock()
        while pending and pending[0].arrival <= now:
            waiting.append(pending.popleft())
        admit_some(only_while_busy=True)
        ctx.synchronize()
        te = time.perf_counter()
        chunk_lat.append(((te - ts) / quantum, len(active)))
        done = []
        for r in active:
            s = r.box.scalars()
            if s["status"] != 0:        # held at its target, or failed
                done.append(r)
        for r in done:
            _finish(ctx, r, stamp(), keep_fields)
            used -= r.nbytes
            active.remove(r)
        active.extend(staged)
        staged = []
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
        r.gpu_s = te - ts
        _finish(ctx, r, te - t0, keep_fields)
    return summarize(requests, time.perf_counter() - t0, lat)


def plain_split(requests: list[Request]) -> dict:
    """Device-loop seconds of a ``serve_plain`` run by request size (the
    Amdahl split of the served speed-up)."""
    out: dict = {}
    for r in requests:
        key = f"{r.cfg.nxm + 1}x{r.cfg.nym}x{r.cfg.nzm}" if r.cfg.nxm >= 192 else "ensemble sizes"
        d = out.setdefault(key, {"requests": 0, "gpu_s": 0.0, "mpoint_steps": 0.0})
        d["requests"] += 1
        d["gpu_s"] += getattr(r, "gpu_s", 0.0)
        d["mpoint_steps"] += r.cells * r.steps_done / 1e6
    for d in out.values():
        d["mpoint_steps_s"] = d["mpoint_steps"] / d["gpu_s"] if d["gpu_s"] > 0 else None
    return out


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
