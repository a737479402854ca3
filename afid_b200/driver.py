"""The time loop of main.F90:167-279 over the library (one box).

``run`` advances a box as the reference's main loop does:

* every step: CalcMaxCFL and the dt rule, TimeMarcher, time += dt
  (main.F90:167-200), on the device in CUDA graphs of up to ``chunk`` steps;
* at output times (main.F90:207: the loop's second step, then every step
  after which mod(time, tout) < dt) the box is held by the device and the
  host calls GlobalQuantities (``nu_vol.out``, ``rms_vel.out``), CalcMaxCFL,
  CheckDivergence and CalcPlateNu (``nu_plate.out``), and, once
  time > tsta, CalcStats and CalcDissipationNu (``nu_diss.out``) when STATON
  and BALANCEON are set (main.F90:208-222);
* exits (main.F90:224-275) with the reference's codes: 555 after the step
  with loop index NTST, 333 once time > TMAX, 334 past WALLTIMEMAX seconds
  of wall time, and the failure codes 165, 166, 169, 266 (or the library's
  990) of the box; when several apply to one step, the later assignment in
  main.F90 wins (555 over 334 over 333 over the output-time checks).

The output files keep the reference's columns: ``nu_plate.out`` is written
with its Fortran format 4(1x,e14.6) (CalcPlateNu.F90:48-54); the
list-directed files (nu_vol.out, rms_vel.out, nu_diss.out) are written with
17 significant digits.  ``wnus_means`` averages them as wnus.sh does.
"""
from __future__ import annotations

import math
import os
import time

import numpy as np

from . import _lib
from .config import BouIn
from .ic import initial_fields

NORMAL_EXITS = (555, 333, 334)


def fortran_e(x: float, w: int = 14, d: int = 6) -> str:
    """Fortran's Ew.d edit descriptor: 0.ddddddE+ee, right-justified in w."""
    if x == 0.0 or not math.isfinite(x):
        body = f"0.{'0' * d}E+00" if x == 0.0 else str(x)
        return body.rjust(w)
    sign = "-" if x < 0 else ""
    e = math.floor(math.log10(abs(x))) + 1
    m = round(abs(x) / 10.0 ** e, d)
    if m >= 1.0:
        m /= 10.0
        e += 1
    digits = f"{m:.{d}f}"[2:]
    return f"{sign}0.{digits}E{'+' if e >= 0 else '-'}{abs(e):02d}".rjust(w)


def _ld(*vals) -> str:
    """One list-directed output record (17 significant digits per value)."""
    return " " + " ".join(f"{v: .16E}" for v in vals) + "\n"


class OutputFiles:
    """The per-output-time logs of the reference, appended as it does."""

    def __init__(self, out_dir: str | None):
        self.dir = out_dir
        if out_dir:
            os.makedirs(out_dir, exist_ok=True)

    def _append(self, name: str, line: str):
        if self.dir:
            with open(os.path.join(self.dir, name), "a") as fh:
                fh.write(line)

    def nu_plate(self, t, lo, up):
        self._append("nu_plate.out", "".join(" " + fortran_e(v) for v in (t, lo, up)) + "\n")

    def nu_vol(self, t, nu):
        self._append("nu_vol.out", _ld(t, nu))

    def rms_vel(self, t, vz, vy, vx, v):
        self._append("rms_vel.out", _ld(t, vz, vy, vx, v))

    def nu_diss(self, t, mu, th):
        self._append("nu_diss.out", _ld(t, mu, th))


def is_output_step(ntime_done: int, t: float, dt: float, tout: float) -> bool:
    """main.F90:207 after a step: the loop index is ntime_done - 1."""
    return ntime_done == 2 or math.fmod(t, tout) < dt


def run(ctx, cfg: BouIn, box=None, seed: int | None = 0, out_dir: str | None = None,
        chunk: int = 64, walltimemax: float | None = None) -> dict:
    """Advance ``box`` (a new one with the seeded initial condition if None)
    until an exit of main.F90.  Returns the exit code, the step count, the
    output-time series and the box."""
    if box is None:
        box = ctx.add_box(cfg)
        for k, v in initial_fields(cfg, box.xc, seed=seed).items():
            box.upload(k, v)
    files = OutputFiles(out_dir)
    wall = cfg.walltimemax if walltimemax is None else walltimemax
    box.set_stop(cfg.ntst + 1, cfg.tout, cfg.tmax)
    series = {k: [] for k in ("time", "nu_bot", "nu_top", "nu_vol", "vz_rms", "vy_rms", "vx_rms",
                              "vel_rms", "divmax", "cfl", "nu_mu", "nu_th")}
    t0 = time.perf_counter()
    code = 0
    while code == 0:
        ctx.step([box], chunk, graph=True)
        s = box.scalars()
        if s["status"] not in (0, _lib.STATUS_HELD):
            code = s["status"]                     # a failure stopped the box
            break
        if s["status"] == _lib.STATUS_HELD:
            t, n, dt = s["time"], s["ntime"], s["dt"]
            if is_output_step(n, t, dt, cfg.tout):
                code = _output(box, cfg, s, files, series)
            if t > cfg.tmax:
                code = 333
            if time.perf_counter() - t0 > wall:
                code = 334
            if n >= cfg.ntst + 1:
                code = 555
            if code == 0:
                box.resume()
        elif time.perf_counter() - t0 > wall:
            code = 334
    s = box.scalars()
    out = {"code": code, "normal": code in NORMAL_EXITS, "ntime": s["ntime"], "time": s["time"],
           "wall_s": time.perf_counter() - t0, "box": box}
    out.update({k: np.array(v) for k, v in series.items()})
    return out


def _output(box, cfg: BouIn, s: dict, files: OutputFiles, series: dict) -> int:
    """The output-time calls of main.F90:208-222; returns 266 or 169 when the
    reference's checks there fail, else 0."""
    t = s["time"]
    g = box.global_quantities()
    files.nu_vol(t, g["nu_vol"])
    files.rms_vel(t, g["vz_rms"], g["vy_rms"], g["vx_rms"], g["vel_rms"])
    code = 266 if (g["vmax"][0] > cfg.vlim and g["vmax"][1] > cfg.vlim) else 0
    cfl = box.calc_max_cfl()
    dmax = box.check_divergence()
    lo, up = box.calc_plate_nu()
    files.nu_plate(t, lo, up)
    mu = th = float("nan")
    if t > cfg.tsta and cfg.staton:
        box.calc_stats()
        if cfg.balanceon:
            mu, th = box.calc_dissipation_nu()
            files.nu_diss(t, mu, th)
    if abs(dmax) > cfg.resid:
        code = 169
    for k, v in (("time", t), ("nu_bot", lo), ("nu_top", up), ("nu_vol", g["nu_vol"]),
                 ("vz_rms", g["vz_rms"]), ("vy_rms", g["vy_rms"]), ("vx_rms", g["vx_rms"]),
                 ("vel_rms", g["vel_rms"]), ("divmax", dmax), ("cfl", cfl), ("nu_mu", mu), ("nu_th", th)):
        series[k].append(v)
    return code


def wnus_means(nu_vol, nu_bot, nu_top) -> dict:
    """The averages of wnus.sh:1-15: nu_vol over the first half of its
    records and over all, the plate Nusselt numbers over all records."""
    nu_vol = np.asarray(nu_vol)
    half = len(nu_vol) // 2
    return {"half_nu_conv": float(nu_vol[:half].mean()) if half else float("nan"),
            "full_nu_conv": float(nu_vol.mean()), "full_nu_bot": float(np.mean(nu_bot)),
            "full_nu_top": float(np.mean(nu_top))}
