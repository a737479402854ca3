#!/usr/bin/env python3
"""Benchmark of the FP64 RK3 time step (Mpoint-steps/s) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2|c1|c3|batch]
                    [--impl ours|reference]

One "step" is one RK3 time step (CalcMaxCFL, the dt rule, three substeps
and the plate Nusselt numbers) of every box of the workload.  The default
workload is the plain large single box (nx=385, ny=nz=768, aspect ratio 2,
Ra=1e9, Pr=1, dt=1e-4 fixed, seeded noise on the conduction profile).
Inputs (~24 GB of resident fields per box) are far larger than L2, so no
flush is needed between timed steps.

With N > 1 (torchrun) every rank advances its own replica of the workload
(the path does not shard a box across GPUs; ensemble boxes are independent),
and the time is the maximum over ranks.

``--impl reference`` times the C/OpenMP restatement of the reference
(oracle/afid_cpu.c, all host threads) on a bounded sample of the same
workload; the Fortran reference cannot be built in this image.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mpoint-steps/s FP64 (RK3 step, cells = nxm*nym*nzm)"
UNIT = "Mpoint-steps/s"

# DRAM traffic per cell of each kernel, (dram__bytes_read.sum +
# dram__bytes_write.sum) / (nxm*nym*nzm), from one ncu --set full capture of
# the 193x384x384 box (bench.py --workload s384, one step); traffic scales with
# the number of cells, the kernels having the same per-cell structure at every
# size.
NCU_TRAFFIC_BYTES_PER_CELL: dict[str, float] = {
    "explicit_fwd": 135.5, "implicit_bwd": 94.9, "divergence": 31.4, "fft_y_fwd": 14.3,
    "fft_z_fwd": 14.3, "poisson_x": 30.3, "fft_z_inv": 14.4, "fft_y_inv": 14.5, "diag": 32.4,
}


# ----------------------------------------------------------------------------
# workloads
# ----------------------------------------------------------------------------
def workload_boxes(name: str, rank: int = 0):
    from afid_b200 import BouIn
    if name == "c2":
        return [BouIn(nxm=384, nym=768, nzm=768, ylen=2.0, zlen=2.0, ray=1e9, pra=1.0, dt=1e-4,
                      istr3=7, idtv=0, resid=0.0)], {"workload": "plain large box 385x768x768 Ra=1e9 Pr=1 dt=1e-4",
                                                     "nx": 385, "ny": 768, "nz": 768}
    if name == "c1":
        return [BouIn(nxm=64, nym=64, nzm=64, ylen=1.0, zlen=1.0, ray=1e6, pra=1.0, dt=5e-4,
                      istr3=7, idtv=0, resid=0.0)], {"workload": "plain box 65x64x64 Ra=1e6 Pr=1 dt=5e-4",
                                                     "nx": 65, "ny": 64, "nz": 64}
    if name == "c3":
        return [BouIn(nxm=512, nym=1280, nzm=1280, ylen=2.0, zlen=2.0, ray=1e10, pra=1.0, dt=5e-5,
                      istr3=7, idtv=0, resid=0.0)], {"workload": "plain largest box 513x1280x1280 Ra=1e10 Pr=1 dt=5e-5",
                                                     "nx": 513, "ny": 1280, "nz": 1280}
    if name == "s384":
        return [BouIn(nxm=192, nym=384, nzm=384, ylen=2.0, zlen=2.0, ray=1e9, pra=1.0, dt=1e-4,
                      istr3=7, idtv=0, resid=0.0)], {"workload": "box 193x384x384 Ra=1e9 Pr=1 dt=1e-4",
                                                     "nx": 193, "ny": 384, "nz": 384}
    if name == "batch":
        from afid_b200.ensemble import ensemble_configs
        return ensemble_configs(64, seed=1000 + rank), {
            "workload": "ensemble of 64 boxes, nx in {33,65,97}, ny=nz in {32..128}, "
                        "Ra log-uniform [1e5,1e8], Pr in {0.7,1,4.38}", "boxes": 64}
    raise SystemExit(f"unknown workload {name}")


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
        "poisson_x": 2 * spec,
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
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self.th = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.th:
            self.th.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ----------------------------------------------------------------------------
# CPU baseline: the oracle on a bounded sample
# ----------------------------------------------------------------------------
def cpu_sample_cfg(workload: str):
    from afid_b200 import BouIn
    if workload == "c1":
        return BouIn(nxm=64, nym=64, nzm=64, ray=1e6, dt=5e-4, istr3=7), "the full 65x64x64 box"
    if workload == "batch":
        return BouIn(nxm=64, nym=48, nzm=48, ray=1e7, dt=1e-4, istr3=7), \
            "one 65x48x48 ensemble-size box"
    nxm = {"c2": 384, "c3": 512, "s384": 192}[workload]
    ra = {"c2": 1e9, "c3": 1e10, "s384": 1e9}[workload]
    dt = {"c2": 1e-4, "c3": 5e-5, "s384": 1e-4}[workload]
    return BouIn(nxm=nxm, nym=96, nzm=96, ylen=2.0 * 96 / 768, zlen=2.0 * 96 / 768, ray=ra, dt=dt,
                 istr3=7), f"a {nxm + 1}x96x96 column of the workload (same x grid, Ra, dt)"


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def run_oracle_sample(workload: str, steps: int, warmup: int):
    """The compiled C restatement (oracle/afid_cpu.c, OpenMP over all host
    threads) on a bounded sample of the workload.
    Returns (Mpoint-steps/s, seconds per step, sample description, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import oracle_state
    from oracle.cpu_port import CpuBox
    cfg, desc = cpu_sample_cfg(workload)
    s = oracle_state(cfg, seed=0)
    box = CpuBox(cfg, s.g.xc)
    for f in ("vx", "vy", "vz", "temp", "pr"):
        box.set(f, getattr(s, f))
    if warmup:
        box.step(cfg.dt, warmup)
    t0 = time.perf_counter()
    box.step(cfg.dt, steps)
    t = time.perf_counter() - t0
    box.close()
    return cells(cfg) * steps / t / 1e6, t / steps, desc, cpu_threads()


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    boxes, conf = workload_boxes(args.workload)
    steps = max(1, args.steps)
    val, tps, desc, thr = run_oracle_sample(args.workload, steps, max(0, min(args.warmup, 1)))
    conf = dict(conf)
    conf["cpu_sample"] = desc
    line = {
        "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": tps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": conf, "impl": "reference",
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": thr, "kind": "port",
                         "sample": f"{steps} RK3 steps of {desc} with the C/OpenMP restatement of "
                                   "the reference (oracle/afid_cpu.c, checked against the NumPy "
                                   "oracle); the Fortran reference has no compiler in this image"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------
# GPU arm
# ----------------------------------------------------------------------------
def gpu_arm(args):
    import ctypes as C

    import torch

    from afid_b200 import Context, _lib
    from afid_b200.ic import initial_fields

    rank, world, local = dist_env()
    dist = None
    if world > 1:
        import torch.distributed as dist_
        from datetime import timedelta
        dist = dist_
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    device = local
    torch.cuda.set_device(device)
    stream = torch.cuda.Stream(device=device)
    ctx = Context(device)
    ctx.set_stream(stream.cuda_stream)
    cfgs, conf = workload_boxes(args.workload, rank)
    boxes = []
    for q, cfg in enumerate(cfgs):
        b = ctx.add_box(cfg)
        f = initial_fields(cfg, b.xc, seed=rank * 1000 + q)
        for k, v in f.items():
            b.upload(k, v)
        boxes.append(b)
    ncell = sum(cells(c) for c in cfgs)

    # launch shapes from the autotuner (cached per GPU and size class)
    from afid_b200 import autotune
    tuned = {}
    if not args.no_tune:
        tuned = autotune.tune(ctx, cfgs)
        for b in boxes:
            autotune.apply(b, tuned)

    # warm-up (also captures the CUDA graph of one step)
    ctx.step(boxes, max(args.warmup, 1), graph=True)
    ctx.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- timed region: K steps through the captured graph, device events
    clocks = ClockSampler(device)
    clocks.start()
    barrier()
    torch.cuda.synchronize(device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.step(boxes, args.steps, graph=True)
    e1.record(stream)
    torch.cuda.synchronize(device)
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([ms], device=f"cuda:{device}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * ncell * args.steps / (ms / 1e3) / 1e6
    statuses = [b.scalars()["status"] for b in boxes]

    # ---- per-kernel device times (CUDA events on the launching stream)
    prof_steps = 2
    prof = ctx.step_profiled(boxes, prof_steps)
    launches_per_step = sum(c for _, c in prof.values()) / prof_steps
    kb = {}
    for cfg in cfgs:
        for k, v in kernel_bytes_per_cell(cfg).items():
            kb[k] = kb.get(k, 0.0) + v * cells(cfg)
    ranked = sorted(((t_ms, k) for k, (t_ms, c) in prof.items() if k in kb), reverse=True)
    top_ms, top = ranked[0]
    nlaunch = prof[top][1]
    avg_s = top_ms / 1e3 / nlaunch
    peak, peak_kind = load_peaks()
    achieved = kb[top] / avg_s / 1e9
    traffic = None
    if top in NCU_TRAFFIC_BYTES_PER_CELL:
        traffic = NCU_TRAFFIC_BYTES_PER_CELL[top] * ncell
    roofline = {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": f"{peak_kind} (copy bandwidth)",
                "bytes_per_launch": kb[top], "avg_launch_ms": avg_s * 1e3, "traffic": traffic,
                "kernel_ms_per_step": {k: round(v[0] / prof_steps, 4) for k, v in prof.items()}}

    # ---- end to end through the public C-ABI with pinned host buffers:
    # upload the initial fields, K steps with the per-step result (plate Nu
    # record) read back every step, download the final fields.
    e2e = None
    if rank == 0 or world > 1:
        L = _lib.lib()
        fields = ["vx", "vy", "vz", "temp", "pr"]
        host_in, host_out = [], []
        for q, (b, cfg) in enumerate(zip(boxes, cfgs)):
            f = initial_fields(cfg, b.xc, seed=rank * 1000 + q)
            ins, outs = {}, {}
            for k in fields:
                t_in = torch.empty((cfg.nzm, cfg.nym, cfg.nx), dtype=torch.float64, pin_memory=True)
                t_in.numpy()[...] = f[k].transpose(2, 1, 0)
                ins[k] = t_in
                outs[k] = t_in          # the final fields overwrite the initial ones
            host_in.append(ins)
            host_out.append(outs)
        ids = (C.c_int * len(boxes))(*[b.id for b in boxes])
        sc = _lib.BoxScalars()
        h2d = sum(5 * cfg.nx * cfg.nym * cfg.nzm * 8 for cfg in cfgs)
        torch.cuda.synchronize(device)
        barrier()
        t0 = time.perf_counter()
        for b, ins in zip(boxes, host_in):
            for k in fields:
                _lib.check(L.afid_box_upload(ctx.h, b.id, _lib.FIELDS[k],
                                             C.cast(ins[k].data_ptr(), C.POINTER(C.c_double))))
            _lib.check(L.afid_box_reset(ctx.h, b.id, 0.0))
        for _ in range(args.steps):
            _lib.check(L.afid_step_graph(ctx.h, ids, len(boxes), 1))
            for b in boxes:
                _lib.check(L.afid_box_get_scalars(ctx.h, b.id, C.byref(sc)))
        for b, outs in zip(boxes, host_out):
            for k in fields:
                _lib.check(L.afid_box_download(ctx.h, b.id, _lib.FIELDS[k],
                                               C.cast(outs[k].data_ptr(), C.POINTER(C.c_double))))
        t_e2e = time.perf_counter() - t0
        if dist is not None:
            t = torch.tensor([t_e2e], device=f"cuda:{device}", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            t_e2e = float(t.item())
        e2e = {"value": world * ncell * args.steps / t_e2e / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": h2d / args.steps,
               "d2h_bytes_per_step": (h2d + C.sizeof(sc) * args.steps * len(boxes)) / args.steps,
               "what": "afid_box_upload of the initial fields from pinned host memory, K x "
                       "(afid_step_graph + afid_box_get_scalars), afid_box_download of the final fields"}

    # ---- batched against the plain one-box-at-a-time loop (ensemble workload)
    batched = None
    if args.workload == "batch":
        from afid_b200.ensemble import run_plain, reset_boxes
        reset_boxes(boxes, seed0=rank * 1000)
        t_plain = run_plain(ctx, boxes, args.steps, graph=True)
        batched = {"plain_value": world * ncell * args.steps / t_plain / 1e6,
                   "plain_ms_per_step": t_plain * 1e3 / args.steps,
                   "speedup_vs_plain": (world * ncell * args.steps / t_plain / 1e6) and value / (
                       world * ncell * args.steps / t_plain / 1e6),
                   "plain": "the same boxes and steps, one box at a time, a CUDA graph per box step"}

    # ---- CPU baseline (rank 0, N = 1 only)
    cpu = None
    if world == 1 and not args.no_cpu:
        v, tps, desc, thr = run_oracle_sample(args.workload, steps=5, warmup=1)
        cpu = {"value": v, "unit": UNIT, "cores": thr, "kind": "port",
               "sample": f"5 RK3 steps of {desc} with the C/OpenMP restatement of the reference "
                         f"(oracle/afid_cpu.c, {tps:.2f} s/step on {thr} host threads)"}

    if rank == 0:
        conf = dict(conf)
        field_mb = ncell * 8 / 1e6   # one field of all boxes of a rank
        l2 = ("inputs larger than L2 (each field %.0f MB, 9 resident fields >> 126 MB), no flush" % field_mb
              if 9 * field_mb > 2 * 126 else
              "inputs fit in L2 (each field %.1f MB), no flush: a small-box latency measurement, "
              "not a bandwidth one" % field_mb)
        conf.update({"global_batch": len(cfgs) * world, "parallelism": f"replicas x{world}",
                     "l2": l2, "graph": "one CUDA graph per step", "grid": "istr3=7 Chebyshev-Gauss-Lobatto"})
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": conf, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(round(launches_per_step * args.steps)), "clocks": clk,
            "status": statuses,
        }
        if batched is not None:
            line["batched"] = batched
        if tuned:
            line["tuning"] = {k: {q: v[q] for q in ("fft_y_lines", "fft_z_lines", "k1_minb")}
                              for k, v in tuned.items()}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def serve_arm(args):
    """Served stream: Poisson arrivals at each rate, continuous batching
    against the plain one-request-at-a-time loop."""
    import torch

    from afid_b200 import Context
    from afid_b200.serve import request_stream, serve, serve_mix, serve_plain
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    ctx = Context(local)
    free, total = torch.cuda.mem_get_info(local)
    budget = int(free * 0.8)
    out = {}
    for rate in args.rates:
        reqs = request_stream(args.requests, rate, seed=2000 + rank, steps=args.serve_steps, mix=serve_mix)
        res_b = serve(ctx, reqs, hbm_budget=budget, quantum=32)
        reqs = request_stream(args.requests, rate, seed=2000 + rank, steps=args.serve_steps, mix=serve_mix)
        res_p = serve_plain(ctx, reqs)
        out[str(rate)] = {"served": res_b, "plain": res_p,
                          "speedup_vs_plain": res_b["mpoint_steps_s"] / res_p["mpoint_steps_s"]}
    ctx.close()
    if rank == 0:
        best = max(out.values(), key=lambda d: d["served"]["mpoint_steps_s"])
        line = {"metric": METRIC + "; served stream", "value": best["served"]["mpoint_steps_s"],
                "unit": UNIT, "n_gpus": world, "steps": args.serve_steps, "warmup": 0,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded Poisson arrivals)",
                "config": {"workload": f"served stream, {args.requests} requests per rate, "
                                       f"{args.serve_steps} CFL-adaptive steps each, 90% ensemble sizes + "
                                       "10% 193x384x384, Ra log-uniform [1e5,1e9]",
                           "hbm_budget_bytes": budget},
                "rates": out}
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "s384", "batch"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-tune", action="store_true", help="use the built-in launch shapes")
    ap.add_argument("--serve", action="store_true", help="run the served-stream benchmark")
    ap.add_argument("--rates", type=float, nargs="+", default=[10.0, 100.0])
    ap.add_argument("--requests", type=int, default=48)
    ap.add_argument("--serve-steps", type=int, default=200)
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.serve:
        return serve_arm(args)
    return gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
