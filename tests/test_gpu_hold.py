"""Device-side holds (afid_box_set_stop / afid_box_resume).

A box stopped at step n by its hold has exactly the fields of a box stepped
n times, whatever number of steps the launch queued; the hold at output
times follows main.F90:207 (second step, then every step after which
mod(time, tout) < dt); a held box is skipped by the batch without affecting
the others."""
import math

import numpy as np
import pytest

from afid_b200 import _lib
from helpers import cfg_of, oracle_state, FIELDS

pytestmark = pytest.mark.gpu


def _box(ctx, cfg, seed):
    s = oracle_state(cfg, seed=seed)
    box = ctx.add_box(cfg, s.g.xc)
    for f in FIELDS:
        box.upload(f, getattr(s, f))
    return box


def _fields(box):
    return {f: box.download(f) for f in FIELDS}


def test_stop_step_equals_exact_step_count(ctx):
    cfg = cfg_of(24, 16, 12, ray=1e5, zlen=0.75, dt=5e-4)
    a, b, c = (_box(ctx, cfg, 4) for _ in range(3))
    b.set_stop(7)
    ctx.step([a], 7)
    ctx.step([b, c], 12, graph=True)          # c is not held: 12 steps
    sb, sc = b.scalars(), c.scalars()
    assert sb["status"] == _lib.STATUS_HELD and sb["ntime"] == 7
    assert sc["status"] == 0 and sc["ntime"] == 12
    fa, fb = _fields(a), _fields(b)
    for f in FIELDS:
        assert np.array_equal(fa[f], fb[f]), f
    # resume: three more steps equal ten steps in one go
    b.set_stop(0)
    b.resume()
    ctx.step([b], 3)
    ctx.step([a], 3)
    assert b.scalars()["status"] == 0 and b.scalars()["ntime"] == 10
    fa, fb = _fields(a), _fields(b)
    for f in FIELDS:
        assert np.array_equal(fa[f], fb[f]), f
    for x in (a, b, c):
        ctx.remove_box(x)


def test_output_time_holds_follow_main_loop(ctx):
    dt, tout = 5e-4, 2.1e-3
    cfg = cfg_of(24, 16, 12, ray=1e5, zlen=0.75, dt=dt)
    box = _box(ctx, cfg, 5)
    box.set_stop(0, tout)
    # the host restatement of main.F90:207 with the device's time sums
    t, want = 0.0, []
    for n in range(1, 31):
        t += dt
        if n == 2 or math.fmod(t, tout) < dt:
            want.append(n)
    got = []
    while len(got) < len(want):
        ctx.step([box], 8, graph=True)
        s = box.scalars()
        assert s["status"] == _lib.STATUS_HELD
        got.append(s["ntime"])
        box.resume()
    assert got == want
    ctx.remove_box(box)
