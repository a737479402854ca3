"""Serving with continuous batching: each request's result is the same alone
and in the mix; admission respects the HBM budget; batched ensemble beats
the one-box-at-a-time loop."""
import numpy as np
import pytest

from afid_b200 import BouIn
from afid_b200.ensemble import compare, ensemble_configs
from afid_b200.serve import Request, serve, serve_plain
from afid_b200.solver import device_bytes

pytestmark = pytest.mark.gpu


def _mix_requests(steps=12):
    cfgs = [
        BouIn(nxm=32, nym=32, nzm=48, ylen=1.0, zlen=1.5, ray=1e5, pra=0.7, dt=1e-6, idtv=1,
              cflmax=1.2, dtmin=1e-8, dtmax=1e-3, resid=0.0),
        BouIn(nxm=64, nym=64, nzm=64, ray=3e6, pra=1.0, dt=1e-6, idtv=1, cflmax=1.2,
              dtmin=1e-8, dtmax=1e-3, resid=0.0),
        BouIn(nxm=32, nym=96, nzm=96, ylen=2.0, zlen=2.0, ray=1e8, pra=4.38, dt=1e-6, idtv=1,
              cflmax=1.2, dtmin=1e-8, dtmax=1e-3, resid=0.0),
        BouIn(nxm=96, nym=48, nzm=48, ray=1e7, pra=1.0, dt=2e-4, idtv=0, resid=0.0),
    ]
    return [Request(rid=q, cfg=c, nsteps=steps + 3 * q, seed=100 + q, arrival=0.0)
            for q, c in enumerate(cfgs)]


def test_results_alone_equal_results_in_mix(ctx):
    mixed = _mix_requests()
    serve(ctx, mixed, hbm_budget=8 << 30, quantum=5, keep_fields=True, realtime=False)
    alone = _mix_requests()
    serve_plain(ctx, alone, keep_fields=True, realtime=False)
    for a, m in zip(alone, mixed):
        assert a.status == 0 and m.status == 0
        assert m.result["scalars"]["ntime"] == a.nsteps
        assert np.array_equal(a.result["dt"], m.result["dt"])
        assert np.abs(np.array(a.result["nu_bot"]) - np.array(m.result["nu_bot"])).max() <= 1e-12
        for f, va in a.result["fields"].items():
            vm = m.result["fields"][f]
            assert np.linalg.norm(va - vm) <= 1e-11 * max(np.linalg.norm(va), 1e-30), f


def test_admission_respects_budget(ctx):
    reqs = _mix_requests(steps=4)
    budget = max(device_bytes(r.cfg) for r in reqs) + 1
    out = serve(ctx, reqs, hbm_budget=budget, quantum=2, realtime=False)
    assert out["failed"] == 0
    assert out["mean_batch"] <= 1.0 + 1e-9        # only one box fits at a time
    for r in reqs:
        assert r.finished is not None and r.steps_done == r.nsteps


def test_batched_ensemble_faster_than_plain(ctx):
    res = compare(ctx, ensemble_configs(16, seed=3), nsteps=10, warmup=1)
    assert all(s == 0 for s in res["status"])
    assert res["speedup"] > 1.0
