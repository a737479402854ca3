#!/usr/bin/env python3
"""Benchmark of the FP64 RK3 time step (Mpoint-steps/s) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W]
                    [--workload batch|c2|c1|c3|s384] [--impl ours|reference]
                    [--serve] [--no-serve] [--no-c2] [--no-cpu]

One "step" is one RK3 time step (CalcMaxCFL, the dt rule, three substeps
and the plate Nusselt numbers) of every box of the workload; points are
nxm*nym*nzm cells.

Default workload (``batch``): the batched ensemble of 64 independent boxes
(nx in {33, 65, 97}, ny = nz in {32, 48, 64, 96, 128}, aspect ratio 1-2,
Ra log-uniform in [1e5, 1e8], Pr in {0.7, 1, 4.38}, fixed dt), every kernel
of a step launched once for all boxes, one CUDA graph per step.  The line
also carries, on the same GPU:
  * ``batched``: the same boxes and steps one box at a time (the plain GPU
    loop) and the speed-up of batching;
  * ``serve``: a served stream (Poisson arrivals, continuous batching with
    HBM admission, CFL-adaptive dt) against the plain loop, with p50/p99
    completion and per-step latency;
  * ``c2``: the plain large box (385x768x768, Ra=1e9, dt=1e-4) with its
    per-kernel times and HBM roofline;
  * ``cpu_baseline``: the C/OpenMP restatement of the reference on the same
    ensemble, all host threads.
The ensemble's fields (~210 MB each, 9 resident) exceed L2, so no flush is
needed between timed steps.

With N > 1 GPUs (``--gpus N`` starts N ranks through torch.distributed.run
when WORLD_SIZE is unset) the ensemble holds 64 N boxes drawn from one seed
and each rank advances its share (ensemble.shard), the served stream is
routed over the ranks (serve.shard_requests); no collective runs on the
data path, times are the maximum over ranks.  The single-box workloads run
one replica per rank.

``--impl reference`` times the C/OpenMP restatement of the reference
(oracle/afid_cpu.c, all host threads) on the same workload; the Fortran
reference cannot be built in this image.
"""
from __future__ import annotations

import argparse
import json
import os
import socket
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# Streams share the device's hardware work queues (8 by default); two streams
# on one queue run in issue order.  The end-to-end leg runs two halves of the
# boxes on two streams, and a split set's halves run on two more, so ask for
# the maximum before CUDA starts (a setting of this process only).
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

METRIC_BATCH = "Mpoint-steps/s FP64 (batched/served vs plain, same B200); p50/p99 solve latency"
METRIC_BOX = "Mpoint-steps/s FP64 (RK3 step, cells = nxm*nym*nzm)"
UNIT = "Mpoint-steps/s"
# RESID of every workload: a box whose max divergence exceeds it at the start
# of a step stops with code 169, so a line whose statuses are all 0 shows the
# bound held at every timed step
DIV_RESID = 1e-10
ENSEMBLE_PER_GPU = 64

# DRAM traffic per cell of each kernel, (dram__bytes_read.sum +
# dram__bytes_write.sum) / (nxm*nym*nzm), from ncu captures of the 193x384x384
# box (bench.py --workload s384); traffic scales with the number of cells, the
# kernels having the same per-cell structure at every size.
NCU_TRAFFIC_BYTES_PER_CELL: dict[str, float] = {
    "explicit_fwd": 135.5, "implicit_bwd": 94.9, "divergence": 31.4, "fft_y_fwd": 14.3,
    "fft_z_fwd": 14.3, "poisson_x": 30.3, "fft_z_inv": 14.4, "fft_y_inv": 14.5, "diag": 32.4,
}
# the same from an ncu capture of the 64-box ensemble itself
# (python -m afid_b200.ensemble --steps 2, fourth explicit-kernel launch)
NCU_TRAFFIC_BYTES_PER_CELL_ENSEMBLE: dict[str, float] = {"explicit_fwd": 134.9}


# ----------------------------------------------------------------------------
# workloads
# ----------------------------------------------------------------------------
def single_box(name: str):
    from afid_b200 import BouIn
    spec = {
        "c2": (384, 768, 2.0, 1e9, 1e-4, "plain large box 385x768x768 Ra=1e9 Pr=1 dt=1e-4"),
        "c1": (64, 64, 1.0, 1e6, 5e-4, "plain box 65x64x64 Ra=1e6 Pr=1 dt=5e-4"),
        "c3": (512, 1280, 2.0, 1e10, 5e-5, "plain largest box 513x1280x1280 Ra=1e10 Pr=1 dt=5e-5"),
        "s384": (192, 384, 2.0, 1e9, 1e-4, "box 193x384x384 Ra=1e9 Pr=1 dt=1e-4"),
    }[name]
    nxm, nyz, asp, ra, dt, desc = spec
    cfg = BouIn(nxm=nxm, nym=nyz, nzm=nyz, ylen=asp, zlen=asp, ray=ra, pra=1.0, dt=dt, istr3=7,
                idtv=0, resid=DIV_RESID)
    return cfg, {"workload": desc, "nx": nxm + 1, "ny": nyz, "nz": nyz}


def workload(name: str, rank: int, world: int):
    """(configurations of this rank, their seeds, config record, scaling)."""
    if name == "batch":
        from afid_b200.ensemble import rank_share
        cfgs, mine = rank_share(ENSEMBLE_PER_GPU, 1000, rank, world)
        conf = {"workload": f"ensemble of {ENSEMBLE_PER_GPU * world} boxes (64 per GPU), nx in "
                            "{33,65,97}, ny=nz in {32,48,64,96,128}, aspect 1-2, Ra log-uniform "
                            "[1e5,1e8], Pr in {0.7,1,4.38}, fixed dt",
                "boxes": ENSEMBLE_PER_GPU * world, "boxes_this_rank": len(mine),
                "parallelism": f"box shards x{world}"}
        return cfgs, list(mine), conf, "weak"
    cfg, conf = single_box(name)
    conf["parallelism"] = f"replicas x{world}"
    return [cfg], [rank], conf, "weak"


def cells(cfg) -> int:
    return cfg.nxm * cfg.nym * cfg.nzm


# algorithmic (compulsory) bytes per cell of one launch of each kernel:
# inputs read once + outputs written once, FP64
def kernel_bytes_per_cell(cfg) -> dict[str, float]:
    spec = 16.0 * (cfg.nym // 2 + 1) / cfg.nym      # half-spectrum bytes per cell
    return {
        "explicit_fwd": 17 * 8.0,   # R vx vy vz temp pr rux ruy ruz rutemp, W rux ruy ruz rutemp + 4 sweeps
        "implicit_bwd": 12 * 8.0,   # R 4 sweeps + vx vy vz temp, W vx vy vz temp
        "divergence": 32.0,         # R vx vy vz, W dph
        "fft_y_fwd": 8.0 + spec,    # R dph, W spectrum
        "fft_z_fwd": 2 * spec,
        "poisson_x": 2 * spec,      # R spectrum, W solution (the pivot table is not counted)
        "fft_z_inv": 2 * spec,
        "fft_y_inv": spec + 8.0,    # R spectrum, W dph
        "correct": 9 * 8.0,         # R dph vx vy vz pr, W vx vy vz pr
        "diag": 4 * 8.0,            # R vx vy vz temp
    }


# ----------------------------------------------------------------------------
# helpers
# ----------------------------------------------------------------------------
def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region: NVML polled from a thread every 5 ms (the region can be shorter
    than nvidia-smi's start-up), nvidia-smi as the fallback.  Only samples
    taken between start() and stop() count; start() returns once the first
    sample is in."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self.th = None
        self.nv = None
        self.samples: list[tuple[float, float, int]] = []
        self.smax = None
        self.run = False
        self.t0 = self.t1 = 0.0

    def _nvml_handle(self):
        import pynvml as N
        import torch
        N.nvmlInit()
        pr = torch.cuda.get_device_properties(self.device)
        try:
            return N, N.nvmlDeviceGetHandleByPciBusId(
                f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0")
        except Exception:
            return N, N.nvmlDeviceGetHandleByIndex(self.device)

    def _poll(self, N, h):
        while self.run:
            try:
                sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
                rs = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((time.monotonic(), float(sm), int(rs)))
            except Exception:
                pass
            time.sleep(0.005)

    def start(self):
        try:
            N, h = self._nvml_handle()
            self.smax = float(N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM))
            self.nv = (N, {"hw_slowdown": N.nvmlClocksEventReasonHwSlowdown,
                           "hw_thermal_slowdown": N.nvmlClocksEventReasonHwThermalSlowdown,
                           "sw_thermal_slowdown": N.nvmlClocksEventReasonSwThermalSlowdown,
                           "sw_power_cap": N.nvmlClocksEventReasonSwPowerCap})
            self.run = True
            self.th = threading.Thread(target=self._poll, args=(N, h), daemon=True)
            self.th.start()
            t_end = time.monotonic() + 1.0
            while not self.samples and time.monotonic() < t_end:
                time.sleep(0.001)
            self.t0 = time.monotonic()
            return
        except Exception:
            self.nv = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self) -> dict:
        if self.nv is not None:
            self.t1 = time.monotonic()
            time.sleep(0.006)
            self.run = False
            self.th.join(timeout=2)
            N, bits = self.nv
            inside = [(sm, rs) for t, sm, rs in self.samples if self.t0 <= t <= self.t1]
            if not inside and self.samples:   # a region shorter than one poll: the nearest sample
                inside = [min(((abs(t - self.t0), sm, rs) for t, sm, rs in self.samples))[1:]]
            reasons = sorted({nm for _, rs in inside for nm, bit in bits.items() if rs & bit})
            return {"sm_mhz": statistics.median([sm for sm, _ in inside]) if inside else None,
                    "sm_max_mhz": self.smax, "reasons": reasons, "samples": len(inside),
                    "source": "NVML, 5 ms polling during the timed region"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.th:
            self.th.join(timeout=2)
        sm, smax, reasons = [], None, set()
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(self.NAMES, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi -lms 100"}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ----------------------------------------------------------------------------
# CPU: the C restatement of the reference on the same boxes
# ----------------------------------------------------------------------------
def cpu_run(cfgs, seeds, steps: int, warmup: int):
    """The compiled C restatement (oracle/afid_cpu.c, OpenMP over all host
    threads) advancing the given boxes one after the other.  Returns
    (Mpoint-steps/s, seconds per step of the whole set)."""
    from afid_b200 import make_grid
    from afid_b200.ic import initial_fields
    from oracle.cpu_port import CpuBox
    boxes = []
    for cfg, seed in zip(cfgs, seeds):
        xc = make_grid(cfg.nxm, cfg.istr3, cfg.str3, cfg.alx3)
        b = CpuBox(cfg, xc)
        for f, v in initial_fields(cfg, xc, seed=seed).items():
            b.set(f, v)
        boxes.append(b)
    for b, cfg in zip(boxes, cfgs):
        if warmup:
            b.step(cfg.dt, warmup)
    t0 = time.perf_counter()
    for b, cfg in zip(boxes, cfgs):
        b.step(cfg.dt, steps)
    t = time.perf_counter() - t0
    for b in boxes:
        b.close()
    n = sum(cells(c) for c in cfgs)
    return n * steps / t / 1e6, t / steps


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    cfgs, seeds, conf, scaling = workload(args.workload, 0, 1)
    steps = max(1, args.steps)
    warm = max(0, min(args.warmup, 1))
    if args.workload in ("c2", "c3"):
        steps, warm = 1, 0          # ~7 s (c2) per step on 16 host threads
    val, tps = cpu_run(cfgs, seeds, steps, warm)
    thr = cpu_threads()
    conf = dict(conf)
    conf["same_config"] = True
    line = {
        "metric": METRIC_BATCH if args.workload == "batch" else METRIC_BOX, "value": val, "unit": UNIT,
        "n_gpus": world, "steps": steps, "warmup": warm, "ms_per_step": tps * 1e3,
        "higher_is_better": True, "scaling": scaling, "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "config": conf, "impl": "reference",
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": thr, "kind": "port",
                         "sample": f"{steps} RK3 steps of the whole workload ({len(cfgs)} box(es), "
                                   f"{tps:.2f} s/step) with the C/OpenMP restatement of the reference "
                                   "(oracle/afid_cpu.c, checked against the NumPy oracle); the "
                                   "Fortran reference has no compiler in this image"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------
# GPU pieces
# ----------------------------------------------------------------------------
class Dist:
    def __init__(self):
        import torch
        self.torch = torch
        self.rank, self.world, self.local = dist_env()
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist_
            from datetime import timedelta
            torch.cuda.set_device(self.local)
            dist_.init_process_group("nccl", timeout=timedelta(seconds=300))
            self.dist = dist_

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, v: float) -> float:
        if self.dist is None:
            return v
        t = self.torch.tensor([v], device=f"cuda:{self.local}", dtype=self.torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if self.dist is None:
            return v
        t = self.torch.tensor([v], device=f"cuda:{self.local}", dtype=self.torch.float64)
        self.dist.all_reduce(t)
        return float(t.item())

    def gather(self, obj):
        if self.dist is None:
            return [obj]
        out = [None] * self.world
        self.dist.all_gather_object(out, obj)
        return out

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()


def make_boxes(ctx, cfgs, seeds):
    """New boxes with the seeded initial condition: a new box's fields are
    zero, so only the temperature is uploaded."""
    from afid_b200.ic import initial_fields
    boxes = []
    for cfg, seed in zip(cfgs, seeds):
        b = ctx.add_box(cfg)
        b.upload("temp", initial_fields(cfg, b.xc, seed=seed)["temp"])
        boxes.append(b)
    return boxes


def reset(boxes, seeds):
    from afid_b200.ic import initial_fields
    for b, seed in zip(boxes, seeds):
        for k, v in initial_fields(b.cfg, b.xc, seed=seed).items():
            b.upload(k, v)
        b.reset(b.cfg.dt)


def timed_steps(ctx, stream, boxes, nsteps, D: Dist, fn=None):
    """Device time (ms, max over ranks) of nsteps of the boxes, events on the
    launching stream, with a barrier and a synchronize on both sides."""
    torch = D.torch
    D.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    if fn is None:
        ctx.step(boxes, nsteps, graph=True)
    else:
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    D.barrier()
    return D.max(e0.elapsed_time(e1))


def roofline_of(ctx, boxes, cfgs, prof_steps=2, ensemble=False):
    prof = ctx.step_profiled(boxes, prof_steps)
    launches_per_step = sum(c for _, c in prof.values()) / prof_steps
    ncell = sum(cells(c) for c in cfgs)
    kb = {}
    for cfg in cfgs:
        for k, v in kernel_bytes_per_cell(cfg).items():
            kb[k] = kb.get(k, 0.0) + v * cells(cfg)
    ranked = sorted(((t_ms, k) for k, (t_ms, c) in prof.items() if k in kb), reverse=True)
    top_ms, top = ranked[0]
    avg_s = top_ms / 1e3 / prof[top][1]
    peak, peak_kind = load_peaks()
    achieved = kb[top] / avg_s / 1e9
    table = NCU_TRAFFIC_BYTES_PER_CELL_ENSEMBLE if ensemble else NCU_TRAFFIC_BYTES_PER_CELL
    traffic = table[top] * ncell if top in table else None
    per_kernel = {}
    for k, (t_ms, c) in prof.items():
        if c == 0:
            continue
        e = {"ms_per_step": round(t_ms / prof_steps, 4), "launches_per_step": c / prof_steps}
        if k in kb:
            e["frac_of_peak"] = round(kb[k] / (t_ms / 1e3 / c) / 1e9 / peak, 3)
        per_kernel[k] = e
    return {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": f"{peak_kind} copy bandwidth (of measured)",
            "bytes_per_launch": kb[top], "avg_launch_ms": avg_s * 1e3, "traffic": traffic,
            "traffic_source": ("ncu dram bytes per cell of a capture of the same 64 boxes, times the cells"
                               if ensemble else "ncu dram bytes per cell of a 193x384x384 capture, times the cells"),
            "kernel_ms_per_step": {k: v["ms_per_step"] for k, v in per_kernel.items()},
            "per_kernel": per_kernel}, launches_per_step


def e2e_run(ctx, boxes, cfgs, seeds, nsteps, D: Dist):
    """The same steps through the public C-ABI from pinned host buffers, the
    boxes in two halves of about equal cells, each half on its own stream
    (afid_ctx_set_stream) with the context's own set splitting off: upload
    of the half's initial fields (queued; the second half's behind the
    first's), reset, per step afid_step_graph + every box's result record of
    that step (afid_boxes_get_scalars_async, written by the device into that
    step's slot of a pinned buffer), download of the final fields (queued);
    one wait at the end.  One half's copies overlap the other half's
    steps."""
    import ctypes as C
    torch = D.torch
    from afid_b200 import _lib
    from afid_b200.ensemble import shard
    from afid_b200.ic import initial_fields
    L = _lib.lib()
    fields = ["vx", "vy", "vz", "temp", "pr"]
    host = []
    for b, cfg, seed in zip(boxes, cfgs, seeds):
        f = initial_fields(cfg, b.xc, seed=seed)
        ins = {}
        for k in fields:
            t_in = torch.empty((cfg.nzm, cfg.nym, cfg.nx), dtype=torch.float64, pin_memory=True)
            t_in.numpy()[...] = f[k].transpose(2, 1, 0)
            ins[k] = t_in          # the final fields overwrite the initial ones
        host.append(ins)
    parts = [p for p in (shard(cfgs, r, 2) for r in range(2)) if p] if len(boxes) > 1 else [[0]]
    ids = [(C.c_int * len(p))(*[boxes[q].id for q in p]) for p in parts]
    streams = [torch.cuda.Stream(device=D.local) for _ in parts]
    rec_size = C.sizeof(_lib.BoxScalars)
    h2d = sum(5 * cfg.nx * cfg.nym * cfg.nzm * 8 for cfg in cfgs)
    nb = len(boxes)
    # one pinned slot of records per step and part, read on the host after
    # the final wait
    rec_buf = torch.empty(nsteps * nb * rec_size, dtype=torch.uint8, pin_memory=True)
    recs = (_lib.BoxScalars * (nsteps * nb)).from_address(rec_buf.data_ptr())
    own = ctx.stream
    ctx.set_split_sets(False)
    for h, p in enumerate(parts):      # each part's graph on its stream, outside the timing
        ctx.set_stream(streams[h].cuda_stream)
        _lib.check(L.afid_step_graph(ctx.h, ids[h], len(p), 0))
    torch.cuda.synchronize()
    D.barrier()
    marks = {}

    def mark(name, st):                # device timeline of the leg
        e = torch.cuda.Event(enable_timing=True)
        e.record(st)
        marks[name] = e
    t0 = time.perf_counter()
    mark("start", streams[0])
    for st in streams[1:]:
        st.wait_event(marks["start"])
    uploaded = None
    for h, p in enumerate(parts):      # queued; part h + 1's copies wait for part h's
        ctx.set_stream(streams[h].cuda_stream)
        if uploaded is not None:
            streams[h].wait_event(uploaded)
        for q in p:
            for k in fields:
                _lib.check(L.afid_box_upload_async(ctx.h, boxes[q].id, _lib.FIELDS[k],
                                                   C.cast(host[q][k].data_ptr(), C.POINTER(C.c_double))))
        uploaded = torch.cuda.Event()
        uploaded.record(streams[h])
        mark(f"uploaded{h}", streams[h])
    bases = [sum(len(x) for x in parts[:h]) for h in range(len(parts))]
    for h, p in enumerate(parts):
        ctx.set_stream(streams[h].cuda_stream)
        for q in p:
            _lib.check(L.afid_box_reset(ctx.h, boxes[q].id, 0.0))
    # the parts' steps issued in turn, step by step, part h offset by `lead`
    # steps per part before it (part 0 steps while part 1's data is still
    # coming in; part 0's downloads go out while part 1 finishes); streams
    # that share a hardware queue then alternate instead of running one part
    # after the other
    lead = min(3, nsteps)
    order = sorted(((s + h * lead, h, s) for h in range(len(parts)) for s in range(nsteps)))
    done = [0] * len(parts)

    def downloads(h):
        ctx.set_stream(streams[h].cuda_stream)
        mark(f"stepped{h}", streams[h])
        for q in parts[h]:
            for k in fields:
                _lib.check(L.afid_box_download_async(ctx.h, boxes[q].id, _lib.FIELDS[k],
                                                     C.cast(host[q][k].data_ptr(), C.POINTER(C.c_double))))
        mark(f"downloaded{h}", streams[h])
    for _, h, s in order:
        p = parts[h]
        ctx.set_stream(streams[h].cuda_stream)
        _lib.check(L.afid_step_graph(ctx.h, ids[h], len(p), 1))
        slot = C.cast(C.addressof(recs) + (s * nb + bases[h]) * rec_size, C.POINTER(_lib.BoxScalars))
        _lib.check(L.afid_boxes_get_scalars_async(ctx.h, ids[h], len(p), slot))
        done[h] += 1
        if done[h] == nsteps:
            downloads(h)
    for st in streams:
        st.synchronize()
    t = D.max(time.perf_counter() - t0)
    ctx.set_stream(own)
    ctx.set_split_sets(True)
    if any(recs[(nsteps - 1) * nb + q].status != 0 for q in range(nb)) or \
            any(recs[s * nb].ntime != recs[0].ntime + s for s in range(nsteps)):
        raise RuntimeError("e2e: a box stopped with a status code, or a record is missing")
    ncell = D.sum(sum(cells(c) for c in cfgs))
    return {"value": ncell * nsteps / t / 1e6, "unit": UNIT,
            "h2d_bytes_per_step": D.sum(h2d) / nsteps,
            "d2h_bytes_per_step": D.sum(h2d + rec_size * nsteps * nb) / nsteps,
            "parts": len(parts),
            "timeline_ms": {k: round(marks["start"].elapsed_time(e), 2) for k, e in marks.items() if k != "start"},
            "what": "boxes in two halves, each on its own stream: afid_box_upload_async of the initial "
                    "fields from pinned host memory, afid_box_reset, K x (afid_step_graph + "
                    "afid_boxes_get_scalars_async: every box's record of that step into pinned host "
                    "memory), afid_box_download_async of the final fields; one wait"}


def serve_record(ctx, D: Dist, rate: float, nreq: int, steps: int, quantum: int = 32) -> dict:
    """A served stream at ``rate`` requests/s per GPU (nreq per GPU, steps
    each) with continuous batching, against the plain one-request-at-a-time
    loop on the same requests; the stream is routed over the ranks."""
    from afid_b200.serve import plain_split, request_stream, serve, serve_mix, serve_plain, shard_requests
    torch = D.torch
    free, _ = torch.cuda.mem_get_info(D.local)
    budget = int(free * 0.8)
    mk = lambda: shard_requests(request_stream(nreq * D.world, rate * D.world, seed=2000, steps=steps,
                                               mix=serve_mix), D.rank, D.world)
    mine = mk()
    D.barrier()
    res_b = serve(ctx, mine, hbm_budget=budget, quantum=quantum)
    comp_b = [r.finished - r.arrival for r in mine]
    mine_p = mk()
    D.barrier()
    res_p = serve_plain(ctx, mine_p)
    comp_p = [r.finished - r.arrival for r in mine_p]
    split = plain_split(mine_p)
    g = D.gather({"b": res_b, "p": res_p, "cb": comp_b, "cp": comp_p,
                  "wb": sum(r.cells * r.steps_done for r in mine),
                  "wp": sum(r.cells * r.steps_done for r in mine_p)})

    def agg(key, comp_key, work_key):
        span = max(x[key]["makespan_s"] for x in g)
        comp = np.concatenate([np.array(x[comp_key]) for x in g])
        d = {"requests": sum(x[key]["requests"] for x in g), "makespan_s": span,
             "mpoint_steps_s": sum(x[work_key] for x in g) / span / 1e6,
             "p50_completion_s": float(np.percentile(comp, 50)), "p99_completion_s": float(np.percentile(comp, 99)),
             "p50_step_latency_ms": max(x[key]["p50_step_latency_ms"] for x in g),
             "p99_step_latency_ms": max(x[key]["p99_step_latency_ms"] for x in g),
             "failed": sum(x[key]["failed"] for x in g),
             "mean_batch": float(np.mean([x[key]["mean_batch"] for x in g]))}
        return d
    sb, sp = agg("b", "cb", "wb"), agg("p", "cp", "wp")
    return {"rate_per_s": rate * D.world, "requests": nreq * D.world, "steps_per_request": steps,
            "hbm_budget_bytes_per_gpu": budget, "quantum": quantum,
            "served": sb, "plain": sp, "speedup_vs_plain": sb["mpoint_steps_s"] / sp["mpoint_steps_s"],
            "plain_split": split if D.world == 1 else None,
            "mix": "90% ensemble sizes + 10% 193x384x384, Ra log-uniform [1e5,1e9], CFL-adaptive dt"}


def c2_record(ctx, stream, D: Dist, steps: int) -> dict:
    """The plain large box: Mpoint-steps/s over a few steps and the
    per-kernel HBM roofline, with the built-in launch shapes (the tuner's
    choices for this size)."""
    cfg, conf = single_box("c2")
    boxes = make_boxes(ctx, [cfg], [D.rank])
    ctx.step(boxes, 2, graph=True)
    ms = timed_steps(ctx, stream, boxes, steps, D)
    status = boxes[0].scalars()["status"]
    roof, _ = roofline_of(ctx, boxes, [cfg])
    ctx.remove_box(boxes[0])
    return {"workload": conf["workload"], "steps": steps, "ms_per_step": ms / steps,
            "value": D.world * cells(cfg) * steps / (ms / 1e3) / 1e6, "status": status, "roofline": roof}


# ----------------------------------------------------------------------------
# GPU arm
# ----------------------------------------------------------------------------
def gpu_arm(args):
    import torch

    from afid_b200 import Context, autotune
    D = Dist()
    rank, world, device = D.rank, D.world, D.local
    torch.cuda.set_device(device)
    stream = torch.cuda.Stream(device=device)
    ctx = Context(device)
    ctx.set_stream(stream.cuda_stream)
    cfgs, seeds, conf, scaling = workload(args.workload, rank, world)
    boxes = make_boxes(ctx, cfgs, seeds)
    ncell_rank = sum(cells(c) for c in cfgs)
    ncell = D.sum(ncell_rank)

    tuned = {}
    if not args.no_tune:
        if len(boxes) > 1:
            tuned = {"batch": autotune.tune_batch(ctx, boxes)}
        else:
            tuned = autotune.tune(ctx, cfgs)
            for b in boxes:
                autotune.apply(b, tuned)

    # warm-up (also captures the CUDA graph of one step)
    ctx.step(boxes, max(args.warmup, 1), graph=True)
    ctx.synchronize()
    graph_kernels = ctx.graph_kernels(boxes)   # kernels of one timed step (both halves of a split set)

    # ---- timed region: K steps through the captured graph, device events
    clocks = ClockSampler(device)
    clocks.start()
    ms = timed_steps(ctx, stream, boxes, args.steps, D)
    clk = clocks.stop()
    value = ncell * args.steps / (ms / 1e3) / 1e6
    statuses = [b.scalars()["status"] for b in boxes]
    div_max = max(max(h["divmax"] for h in b.history(args.steps)) for b in boxes)

    roof, _ = roofline_of(ctx, boxes, cfgs, ensemble=(args.workload == "batch"))
    e2e = e2e_run(ctx, boxes, cfgs, seeds, args.steps, D)

    batched = None
    if args.workload == "batch" and not args.no_plain:
        if not args.no_tune:                 # each box alone runs its own class's best shapes
            per_class = autotune.tune(ctx, cfgs)
            for b in boxes:
                autotune.apply(b, per_class)
        for b in boxes:                      # capture the one-box graphs outside the timing
            ctx.step([b], 1, graph=True)
        reset(boxes, seeds)
        t_plain = timed_steps(ctx, stream, boxes, args.steps, D,
                              fn=lambda: [ctx.step([b], args.steps, graph=True) for b in boxes])
        pv = ncell * args.steps / (t_plain / 1e3) / 1e6
        batched = {"plain_value": pv, "plain_ms_per_step": t_plain / args.steps,
                   "speedup_vs_plain": value / pv,
                   "plain": "the same boxes and steps, one box at a time (a CUDA graph per box "
                            "step, each box with the launch shapes tuned for its size class), "
                            "device time"}
    for b in boxes:
        ctx.remove_box(b)

    serve_rec = None
    if args.workload == "batch" and not args.no_serve:
        serve_rec = serve_record(ctx, D, rate=args.rate, nreq=args.requests, steps=args.serve_steps)
    c2 = None
    if args.workload == "batch" and not args.no_c2 and world == 1:
        c2 = c2_record(ctx, stream, D, steps=5)

    # ---- CPU baseline (rank 0, N = 1): the same workload
    cpu = None
    if world == 1 and not args.no_cpu:
        csteps = 2 if args.workload == "batch" else 1
        v, tps = cpu_run(cfgs, seeds, csteps, 0)
        thr = cpu_threads()
        cpu = {"value": v, "unit": UNIT, "cores": thr, "kind": "port",
               "sample": f"{csteps} RK3 step(s) of the same {len(cfgs)} box(es) with the C/OpenMP "
                         f"restatement of the reference (oracle/afid_cpu.c, {tps:.2f} s/step on "
                         f"{thr} host threads)"}

    if rank == 0:
        conf = dict(conf)
        field_mb = ncell_rank * 8 / 1e6   # one field of all boxes of a rank
        conf.update({
            "global_batch": len(cfgs) * world if args.workload != "batch" else conf["boxes"],
            "l2": ("inputs larger than L2 (each field %.0f MB per GPU, 9 resident fields), no flush"
                   % field_mb if field_mb > 126 else
                   "inputs fit in L2 (each field %.1f MB), no flush: a latency measurement" % field_mb),
            "graph": "one CUDA graph per step", "grid": "istr3=7 Chebyshev-Gauss-Lobatto",
            "div_resid": DIV_RESID})
        line = {
            "metric": METRIC_BATCH if args.workload == "batch" else METRIC_BOX,
            "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": scaling, "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": conf, "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(graph_kernels * args.steps), "clocks": clk,
            "status": statuses, "max_divergence_timed": div_max,
        }
        if batched is not None:
            line["batched"] = batched
        if serve_rec is not None:
            line["serve"] = serve_rec
        if c2 is not None:
            line["c2"] = c2
        if tuned:
            line["tuning"] = {k: {q: v[q] for q in ("fft_y_lines", "fft_z_lines", "k1_minb")}
                              for k, v in tuned.items()}
        print(json.dumps(line), flush=True)
    ctx.close()
    D.close()
    return 0


def serve_arm(args):
    """Served stream at each rate against the plain loop (one line)."""
    import torch

    from afid_b200 import Context
    D = Dist()
    torch.cuda.set_device(D.local)
    ctx = Context(D.local)
    out = {}
    for rate in args.rates:
        out[str(rate)] = serve_record(ctx, D, rate=rate, nreq=args.requests, steps=args.serve_steps)
    ctx.close()
    if D.rank == 0:
        best = max(out.values(), key=lambda d: d["served"]["mpoint_steps_s"])
        line = {"metric": METRIC_BATCH + "; served stream sweep", "value": best["served"]["mpoint_steps_s"],
                "unit": UNIT, "n_gpus": D.world, "steps": args.serve_steps, "warmup": 0,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded Poisson arrivals)",
                "config": {"workload": f"served stream, {args.requests} requests per GPU per rate, "
                                       f"{args.serve_steps} CFL-adaptive steps each, 90% ensemble sizes + "
                                       "10% 193x384x384, Ra log-uniform [1e5,1e9]"},
                "rates": out}
        print(json.dumps(line), flush=True)
    D.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="batch", choices=["batch", "c1", "c2", "c3", "s384"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-tune", action="store_true", help="use the built-in launch shapes")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-stream sub-record")
    ap.add_argument("--no-c2", action="store_true", help="skip the large-box sub-record")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the one-box-at-a-time comparison of the batch workload")
    ap.add_argument("--rate", type=float, default=50.0, help="arrivals/s of the serve sub-record")
    ap.add_argument("--serve", action="store_true", help="run the served-stream sweep over --rates")
    ap.add_argument("--rates", type=float, nargs="+", default=[1.0, 10.0, 50.0, 200.0])
    ap.add_argument("--requests", type=int, default=32, help="requests per GPU of a served stream")
    ap.add_argument("--serve-steps", type=int, default=200)
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU through torch.distributed.run
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
               f"--nproc-per-node={args.gpus}", "--master-addr", "127.0.0.1",
               "--master-port", str(free_port()), os.path.abspath(__file__)] + sys.argv[1:]
        return subprocess.call(cmd)
    if args.impl == "reference":
        return reference_arm(args)
    if args.serve:
        return serve_arm(args)
    return gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
