"""The configurations of the parity contract on the GPU.

C1  65x64x64, Ra=1e6, Pr=1, dt=5e-4, 200 RK3 steps, seeds 0, 1 and 2:
    max divergence <= 1e-10 at every step and plate Nusselt numbers within
    1e-9 of the oracle's series over steps 1-100
    (tests/golden/golden_c1_seeds.npz).  The boxes run with RESID = 1e-10,
    so the device itself stops a box with code 169 the first step its
    divergence exceeds the bound.
C2, C3 scaled down: the large-box physics (Ra=1e9, dt=1e-4 and Ra=1e10,
    dt=5e-5, aspect ratio 2) on 49x96x96 and 65x160x160 boxes, one step
    against the oracle at per-field relative L2 <= 1e-11.
C3  full size (513x1280x1280, ~91 GB resident): conduction is a fixed point
    (KAT-1) and two seeded steps keep the divergence <= 1e-10.
"""
import ctypes as C
import os

import numpy as np
import pytest

from afid_b200 import _lib
from helpers import cfg_of, compare_fields, oracle_state, FIELDS
from oracle import afid_oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
DIV_BOUND = 1e-10


def _box(ctx, cfg, s):
    box = ctx.add_box(cfg, s.g.xc)
    for f in FIELDS:
        box.upload(f, getattr(s, f))
    return box


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_c1_200_steps_divergence_and_plate_nu(ctx, seed):
    z = np.load(os.path.join(GOLDEN, "golden_c1_seeds.npz"))
    cfg = cfg_of(64, 64, 64, ray=1e6, dt=5e-4, resid=DIV_BOUND)
    s = oracle_state(cfg, seed=seed)
    box = _box(ctx, cfg, s)
    ctx.step([box], 200, graph=True)
    sc = box.scalars()
    assert sc["status"] == 0 and sc["ntime"] == 200, sc
    hist = box.history(200)
    assert len(hist) == 200
    # divmax of step n is the divergence of the velocity step n-1 left
    # (step 1 starts from rest); the last step's is read directly
    div = [h["divmax"] for h in hist[1:]] + [box.check_divergence()]
    assert max(div) <= DIV_BOUND, max(div)
    nb = np.array([h["nu_bot"] for h in hist[:100]])
    nt = np.array([h["nu_top"] for h in hist[:100]])
    assert np.abs(nb - z[f"s{seed}_nu_bot"]).max() <= 1e-9
    assert np.abs(nt - z[f"s{seed}_nu_top"]).max() <= 1e-9
    assert np.array_equal(np.array([h["dt"] for h in hist[:100]]), z[f"s{seed}_dt"])
    ctx.remove_box(box)


@pytest.mark.parametrize("name,shape,kw", [
    ("c2_scaled", (48, 96, 96), dict(ray=1e9, ylen=2.0, zlen=2.0, dt=1e-4)),
    ("c3_scaled", (64, 160, 160), dict(ray=1e10, ylen=2.0, zlen=2.0, dt=5e-5)),
])
def test_large_box_physics_scaled_down_one_step(ctx, name, shape, kw):
    cfg = cfg_of(*shape, pra=1.0, resid=DIV_BOUND, **kw)
    s = oracle_state(cfg, seed=3)
    box = _box(ctx, cfg, s)
    recs = O.run(s, 1, cfg.dt, vectorised_poisson=True)
    ctx.step([box], 1)
    err = compare_fields(box, s)
    assert all(v <= 1e-11 for v in err.values()), (name, err)
    sc = box.scalars()
    assert sc["status"] == 0
    assert abs(sc["nu_bot"] - recs[0]["nu_bot"]) <= 1e-9
    assert abs(sc["nu_top"] - recs[0]["nu_top"]) <= 1e-9
    assert box.check_divergence() <= DIV_BOUND
    ctx.remove_box(box)


def _fortran_temp(cfg, xc, seed):
    """Temperature of the seeded initial condition as the C-ABI takes it:
    Fortran order (x fastest), i.e. a C-order (nzm, nym, nx) array, built
    one z-slab at a time to bound host memory."""
    nx, nxm, nym, nzm = cfg.nx, cfg.nxm, cfg.nym, cfg.nzm
    prof = np.empty(nx)
    prof[1:nxm] = cfg.tempbp - (cfg.tempbp - cfg.temptp) * xc[1:nxm] / xc[nx - 1]
    prof[0], prof[nx - 1] = cfg.tempbp, cfg.temptp
    buf = np.empty((nzm, nym, nx))
    buf[...] = prof
    if seed is not None:
        # the draws of ic.seeded_noise, in the same order
        rng = np.random.Generator(np.random.PCG64(seed))
        for i in range(nzm):
            buf[i, :, 1:nxm] += rng.uniform(-0.01, 0.01, size=(nym, nxm - 1))
    return buf


def test_c3_full_size_invariants(ctx):
    import torch
    cfg = cfg_of(512, 1280, 1280, ray=1e10, ylen=2.0, zlen=2.0, dt=5e-5, resid=DIV_BOUND)
    free, _ = torch.cuda.mem_get_info(0)
    from afid_b200.solver import device_bytes
    need = device_bytes(cfg)
    if need > free:
        pytest.skip(f"C3 needs {need / 2**30:.1f} GiB, {free / 2**30:.1f} GiB free")
    box = ctx.add_box(cfg)
    L = _lib.lib()
    up = lambda buf: _lib.check(L.afid_box_upload(ctx.h, box.id, _lib.FIELDS["temp"],
                                                  buf.ctypes.data_as(C.POINTER(C.c_double))))
    # KAT-1: the conduction profile is a fixed point of the step
    t0 = _fortran_temp(cfg, box.xc, seed=None)
    up(t0)
    ctx.step([box], 1)
    t1 = np.empty_like(t0)
    _lib.check(L.afid_box_download(ctx.h, box.id, _lib.FIELDS["temp"], t1.ctypes.data_as(C.POINTER(C.c_double))))
    assert np.abs(t1 - t0).max() <= 1e-14
    del t1
    sc = box.scalars()
    assert sc["status"] == 0
    # plate Nu divides the temperature step of the first cell by its width
    # (9.4e-6 on this grid): one ulp of temperature is ~2e-11 of Nu
    assert sc["nu_bot"] == pytest.approx(1.0, abs=1e-10) and sc["nu_top"] == pytest.approx(1.0, abs=1e-10)
    # seeded noise, two steps: the projection keeps the divergence at roundoff
    del t0
    up(_fortran_temp(cfg, box.xc, seed=0))
    box.reset()
    ctx.step([box], 2)
    sc = box.scalars()
    assert sc["status"] == 0 and sc["ntime"] == 2, sc
    hist = box.history(2)
    assert hist[1]["divmax"] <= DIV_BOUND
    assert box.check_divergence() <= DIV_BOUND
    ctx.remove_box(box)
