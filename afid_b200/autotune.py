"""Autotuner of launch shapes.

For each box size class (nxm, nym, nzm) the tuner times candidate launch
shapes of the kernels whose shape is free, with device events around every
kernel (afid_step_profiled), and keeps the fastest:

* row pairs per y-FFT block (forward and inverse y transforms),
* ky columns per z-FFT block (forward and inverse z transforms),
* the variant of the explicit/forward kernel: 32x8-column tiles with 2
  resident blocks (up to 128 registers per thread), with 3 (up to 80), or
  with two x-planes per barrier; 32x4 tiles with 4, 5 or 6 blocks; 32x2
  tiles with 8 blocks.

``tune`` tunes each size class on a box of its own (for single boxes);
``tune_batch`` tunes a set of boxes that are stepped together, on the set.

Results do not depend on the shapes (tests/test_gpu_batch.py checks batched
against single-box results bit for bit), so tuning is purely a speed choice.
The choices are cached in a JSON file keyed by GPU name and size class.
"""
from __future__ import annotations

import json
import os

from .config import BouIn
from .ic import initial_fields

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "afid_b200", "tune.json")


def fft_plan(n: int) -> list[int]:
    """Radix plan of an n-point transform (the library's factor_radices)."""
    m, a, rad = n, 0, []
    while m % 2 == 0:
        m //= 2
        a += 1
    while a >= 4:
        rad.append(16)
        a -= 4
    rad += {3: [8], 2: [4], 1: [2], 0: []}[a]
    for p in (3, 5, 7):
        while m % p == 0:
            rad.append(p)
            m //= p
    if m != 1:
        raise ValueError(f"{n}: prime factor > 7")
    return rad


SMEM_MAX = 200 * 1024   # shared memory of one transform block (two copy-in slots, twiddles)
TILE_MAX = 14 * 256     # complex values of one in-place tile


TAIL_BYTES = 1024        # upper bound of the slot mbarriers and the cached box descriptor


def fft_y_bytes(n: int, pairs: int) -> int:
    return (2 * 2 * pairs * (n // 2 + 1) + n) * 16 + TAIL_BYTES


def fft_z_bytes(n: int, lines: int) -> int:
    return (2 * lines * n + n) * 16 + TAIL_BYTES


def candidates(cfg: BouIn) -> dict:
    ny = [v for v in (1, 2, 4, 8, 16, 32, 64) if fft_y_bytes(cfg.nym, v) <= SMEM_MAX and v * cfg.nym <= TILE_MAX]
    nz = [v for v in (1, 2, 4, 8, 16, 32, 64) if fft_z_bytes(cfg.nzm, v) <= SMEM_MAX and v * cfg.nzm <= TILE_MAX
          and v < 2 * (cfg.nym // 2 + 1)]
    return {"fft_y_lines": ny or [1], "fft_z_lines": nz or [1], "k1_minb": [2, 3, 4, 5, 6, 7, 8]}


def class_key(cfg: BouIn) -> str:
    return f"{cfg.nxm}x{cfg.nym}x{cfg.nzm}"


def gpu_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name()
    except Exception:
        return "unknown"


class TuneCache:
    def __init__(self, path: str | None = None):
        self.path = path or os.environ.get("AFID_TUNE_CACHE", DEFAULT_CACHE)
        self.data: dict = {}
        try:
            with open(self.path) as fh:
                self.data = json.load(fh)
        except (OSError, ValueError):
            self.data = {}

    def get(self, cfg: BouIn):
        return self.data.get(gpu_name(), {}).get(class_key(cfg))

    def put(self, cfg: BouIn, choice: dict):
        self.data.setdefault(gpu_name(), {})[class_key(cfg)] = choice

    def save(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        tmp = self.path + ".tmp"
        with open(tmp, "w") as fh:
            json.dump(self.data, fh, indent=1, sort_keys=True)
        os.replace(tmp, self.path)


def _time(ctx, box, kernels, steps):
    prof = ctx.step_profiled([box], steps)
    return sum(prof[k][0] for k in kernels)


def tune_class(ctx, cfg: BouIn, steps: int = 2) -> dict:
    """Time every candidate of each tunable kernel family on one box of the
    class and return the fastest choices with their times (ms per step)."""
    box = ctx.add_box(cfg)
    try:
        for k, v in initial_fields(cfg, box.xc, seed=0).items():
            box.upload(k, v)
        ctx.step([box], 1)
        cand = candidates(cfg)
        best = {}
        res = {}
        for fy in cand["fft_y_lines"]:
            box.set_tuning(fy, 0, 2)
            res[("y", fy)] = _time(ctx, box, ("fft_y_fwd", "fft_y_inv"), steps)
        fy = min(cand["fft_y_lines"], key=lambda v: res[("y", v)])
        for fz in cand["fft_z_lines"]:
            box.set_tuning(fy, fz, 2)
            res[("z", fz)] = _time(ctx, box, ("fft_z_fwd", "fft_z_inv"), steps)
        fz = min(cand["fft_z_lines"], key=lambda v: res[("z", v)])
        for mb in cand["k1_minb"]:
            box.set_tuning(fy, fz, mb)
            res[("k1", mb)] = _time(ctx, box, ("explicit_fwd",), steps)
        mb = min(cand["k1_minb"], key=lambda v: res[("k1", v)])
        best = {"fft_y_lines": fy, "fft_z_lines": fz, "k1_minb": mb,
                "ms_per_step": {f"{a}{b}": round(t / steps, 4) for (a, b), t in res.items()}}
        return best
    finally:
        ctx.remove_box(box)


def tune(ctx, cfgs, cache: TuneCache | None = None, steps: int = 2) -> dict:
    """Tune every size class of ``cfgs`` that the cache does not hold."""
    cache = cache or TuneCache()
    out = {}
    for cfg in cfgs:
        key = class_key(cfg)
        if key in out:
            continue
        choice = cache.get(cfg)
        if choice is None:
            choice = tune_class(ctx, cfg, steps)
            cache.put(cfg, choice)
        out[key] = choice
    try:
        cache.save()
    except OSError:
        pass
    return out


def tune_batch(ctx, boxes, steps: int = 2) -> dict:
    """Tune the launch shapes of a set of boxes stepped together: each
    candidate is applied to every box of the set (where it is valid for the
    box) and the set's own kernel times decide.  Shapes that are best for a
    box alone are not best in a batch: a transform launch takes the largest
    tile of its boxes, so one class asking for big tiles lowers the
    occupancy of all.  Returns the chosen values and their times; the boxes
    keep the chosen shapes."""
    y_all = sorted({v for b in boxes for v in candidates(b.cfg)["fft_y_lines"]})
    z_all = sorted({v for b in boxes for v in candidates(b.cfg)["fft_z_lines"]})

    def set_all(fy, fz, mb):
        for b in boxes:
            c = candidates(b.cfg)
            b.set_tuning(fy if fy in c["fft_y_lines"] else 0, fz if fz in c["fft_z_lines"] else 0, mb)

    def t(kernels):
        ctx.step(boxes, 1)
        prof = ctx.step_profiled(boxes, steps)
        return sum(prof[k][0] for k in kernels) / steps

    res = {}
    set_all(0, 0, 0)
    res[("y", 0)] = t(("fft_y_fwd", "fft_y_inv"))
    for fy in y_all:
        set_all(fy, 0, 0)
        res[("y", fy)] = t(("fft_y_fwd", "fft_y_inv"))
    fy = min([0] + y_all, key=lambda v: res[("y", v)])
    set_all(fy, 0, 0)
    res[("z", 0)] = t(("fft_z_fwd", "fft_z_inv"))
    for fz in z_all:
        set_all(fy, fz, 0)
        res[("z", fz)] = t(("fft_z_fwd", "fft_z_inv"))
    fz = min([0] + z_all, key=lambda v: res[("z", v)])
    for mb in candidates(boxes[0].cfg)["k1_minb"]:
        set_all(fy, fz, mb)
        res[("k1", mb)] = t(("explicit_fwd",))
    mb = min(candidates(boxes[0].cfg)["k1_minb"], key=lambda v: res[("k1", v)])
    set_all(fy, fz, mb)
    return {"fft_y_lines": fy, "fft_z_lines": fz, "k1_minb": mb,
            "ms_per_step": {f"{a}{b}": round(v, 4) for (a, b), v in res.items()}}


def apply(box, choices: dict):
    """Set a box's launch shapes from tuned choices (if its class is there)."""
    c = choices.get(class_key(box.cfg))
    if c:
        box.set_tuning(c["fft_y_lines"], c["fft_z_lines"], c["k1_minb"])
