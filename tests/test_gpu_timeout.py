"""The bounded waits of the transforms' tile copies, made to run out.

With the test switch afid_box_test_skip_z_copies a box's z transform arms
the mbarrier of each tile slot for the tile's bytes but issues no copy, so
its wait gives up after a few polls: no copy is ever in flight and nothing
faults.  The box must then carry status 990, the block stops, and a box that
comes earlier in the same batch must still come out bit for bit as it does
alone; the context stays usable."""
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


def test_z_copy_timeout_sets_990_and_spares_the_other_box(ctx):
    cfg = cfg_of(24, 32, 24, ray=1e5, zlen=0.75, dt=5e-4)
    alone = _box(ctx, cfg, 5)
    ctx.step([alone], 2)
    a = _box(ctx, cfg, 5)
    b = _box(ctx, cfg, 6)
    L = _lib.lib()
    _lib.check(L.afid_box_test_skip_z_copies(ctx.h, b.id, 1, 1000))
    ctx.step([a, b], 2)
    ctx.synchronize()
    assert b.scalars()["status"] == _lib.STATUS_DEVICE_TIMEOUT
    sa = a.scalars()
    assert sa["status"] == 0 and sa["ntime"] == 2
    for f in FIELDS:
        assert np.array_equal(a.download(f), alone.download(f)), f
    # the context and the other box keep working
    _lib.check(L.afid_box_test_skip_z_copies(ctx.h, b.id, 0, 0))
    ctx.step([a], 1)
    ctx.step([alone], 1)
    assert a.scalars()["status"] == 0
    for f in FIELDS:
        assert np.array_equal(a.download(f), alone.download(f)), f
    for x in (alone, a, b):
        ctx.remove_box(x)
