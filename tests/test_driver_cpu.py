"""Host logic of the run driver on the CPU: the Fortran E format of
nu_plate.out, the output-time rule of main.F90:207, wnus.sh's averages and
the exit-code precedence of main.F90:224-275, with a stand-in for the
device box that applies the library's hold rules."""
import math

import numpy as np
import pytest

from afid_b200 import BouIn, _lib
from afid_b200.driver import fortran_e, is_output_step, run, wnus_means


@pytest.mark.parametrize("x,want", [
    (0.0, "  0.000000E+00"), (1.0, "  0.100000E+01"), (0.01, "  0.100000E-01"),
    (-123.4567, " -0.123457E+03"), (9.9999999, "  0.100000E+02"), (1.5e-7, "  0.150000E-06"),
])
def test_fortran_e14_6(x, want):
    assert fortran_e(x) == want


def test_output_rule_and_wnus_means():
    dt, tout = 5e-4, 1e-2
    t, outs = 0.0, []
    for n in range(1, 101):
        t += dt
        if is_output_step(n, t, dt, tout):
            outs.append(n)
    assert outs[0] == 2 and outs[1:] == [20, 40, 60, 80, 100] or outs[1:] == [19, 39, 59, 79, 99]
    m = wnus_means([1.0, 2.0, 3.0, 4.0, 10.0], [1.0, 3.0], [2.0, 2.0])
    assert m == {"half_nu_conv": 1.5, "full_nu_conv": 4.0, "full_nu_bot": 2.0, "full_nu_top": 2.0}


class FakeBox:
    """Applies the device's per-step bookkeeping and hold rules
    (k_finalize): time += dt, ntime += 1, hold at stop_ntime / output
    times / time > tmax; a planted failure code at a given step."""

    def __init__(self, dt, fail_at=None, fail_code=266):
        self.dt, self.t, self.n, self.status = dt, 0.0, 0, 0
        self.stop, self.tout, self.tmax = 0, 0.0, 0.0
        self.fail_at, self.fail_code = fail_at, fail_code

    def set_stop(self, n, tout, tmax):
        self.stop, self.tout, self.tmax = n, tout, tmax

    def step(self, k):
        for _ in range(k):
            if self.status != 0:
                return
            if self.fail_at is not None and self.n + 1 == self.fail_at:
                self.status = self.fail_code
                return
            self.t += self.dt
            self.n += 1
            hold = self.stop > 0 and self.n >= self.stop
            hold |= self.tout > 0 and (self.n == 2 or math.fmod(self.t, self.tout) < self.dt)
            hold |= self.tmax > 0 and self.t > self.tmax
            if hold:
                self.status = _lib.STATUS_HELD

    def scalars(self):
        return {"time": self.t, "ntime": self.n, "dt": self.dt, "status": self.status}

    def resume(self):
        if self.status == _lib.STATUS_HELD:
            self.status = 0

    def global_quantities(self):
        return {"nu_vol": 1.0, "vz_rms": 0.0, "vy_rms": 0.0, "vx_rms": 0.0, "vel_rms": 0.0,
                "vmax": (0.0, 0.0, 0.0)}

    def calc_max_cfl(self):
        return 0.0

    def check_divergence(self):
        return 0.0

    def calc_plate_nu(self):
        return 1.0, 1.0


class FakeCtx:
    def step(self, boxes, n, graph=False):
        for b in boxes:
            b.step(n)


def _cfg(**kw):
    base = dict(nxm=8, nym=8, nzm=8, dt=1e-3, tout=1e-2, tmax=1e9, ntst=99, resid=1e-2)
    base.update(kw)
    return BouIn(**base)


def test_exit_555_after_ntst_plus_one_steps(tmp_path):
    cfg = _cfg()
    box = FakeBox(cfg.dt)
    res = run(FakeCtx(), cfg, box=box, out_dir=str(tmp_path), chunk=7)
    assert res["code"] == 555 and res["ntime"] == 100
    # output times: the second step, then every tout
    assert len(res["time"]) == 1 + 10
    assert np.loadtxt(tmp_path / "nu_plate.out").shape == (11, 3)


def test_exit_333_when_time_passes_tmax():
    cfg = _cfg(tmax=0.0255)
    res = run(FakeCtx(), cfg, box=FakeBox(cfg.dt), chunk=16)
    assert res["code"] == 333 and res["ntime"] == 26


def test_ntst_wins_over_tmax_on_the_same_step():
    cfg = _cfg(ntst=25, tmax=0.0255)
    res = run(FakeCtx(), cfg, box=FakeBox(cfg.dt), chunk=64)
    assert res["code"] == 555 and res["ntime"] == 26


def test_device_failure_code_ends_the_run():
    cfg = _cfg()
    res = run(FakeCtx(), cfg, box=FakeBox(cfg.dt, fail_at=37, fail_code=165), chunk=8)
    assert res["code"] == 165 and res["ntime"] == 36


def test_walltime_exit_334():
    cfg = _cfg(ntst=10 ** 6)
    res = run(FakeCtx(), cfg, box=FakeBox(cfg.dt), chunk=8, walltimemax=0.0)
    assert res["code"] == 334
