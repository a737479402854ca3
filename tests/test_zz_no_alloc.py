"""The pressure solve that allocates nothing (afid_solve_pressure_correction_noalloc).

Some callers cannot allocate device memory while they run: an application
that has handed its GPU memory to its own pool, code that runs where
cudaMalloc is not allowed, or a host program that must keep a fixed device
footprint.  They pass their own dph array and the library uses a fixed
scratch array of its own.  This test checks, through the C-ABI, that two
calls in a row give the same result as the regular entry point
(afid_solve_pressure_correction on a box), within the tolerance of the
Poisson parity tests.  The test allocates its device buffer with torch; the
entry point itself allocates nothing.

The file name makes pytest collect it last."""
import ctypes as C

import numpy as np
import pytest

from afid_b200 import _lib
from helpers import cfg_of, rel_l2

pytestmark = pytest.mark.gpu


def _regular(ctx, cfg, dph_kji):
    box = ctx.add_box(cfg)
    box.upload("dph", dph_kji)
    box.solve_pressure_correction()
    out = box.download("dph")
    xc = box.xc.copy()
    ctx.remove_box(box)
    return out, xc


def _noalloc(cfg, xc, dph_kji):
    import torch
    dev = torch.from_numpy(np.ascontiguousarray(dph_kji.transpose(0, 2, 1))).cuda()  # [k][i][j]
    stream = torch.cuda.current_stream()
    rc = _lib.lib().afid_solve_pressure_correction_noalloc(
        C.c_void_p(dev.data_ptr()), cfg.nxm, cfg.nym, cfg.nzm, _lib.dptr(xc), cfg.alx3,
        cfg.ylen, cfg.zlen, C.c_void_p(stream.cuda_stream))
    _lib.check(rc)
    stream.synchronize()
    return dev.cpu().numpy().transpose(0, 2, 1).copy()


@pytest.mark.parametrize("shape,kw", [((32, 48, 40), dict(ylen=1.5, zlen=1.25)),
                                      ((24, 16, 20), dict(zlen=0.5))])
def test_noalloc_matches_regular_twice(ctx, shape, kw):
    cfg = cfg_of(*shape, **kw)
    rng = np.random.default_rng(42)
    for call in range(2):
        dph = rng.standard_normal((cfg.nxm, cfg.nym, cfg.nzm))
        want, xc = _regular(ctx, cfg, dph)
        got = _noalloc(cfg, xc, dph)
        assert rel_l2(got, want, remove_mean=True) <= 1e-12, f"call {call}"


def test_noalloc_rejects_oversize():
    xc = np.linspace(0.0, 1.0, 513)
    rc = _lib.lib().afid_solve_pressure_correction_noalloc(
        C.c_void_p(1), 512, 1024, 1024, _lib.dptr(xc), 1.0, 1.0, 1.0, None)
    assert rc == -6
    assert b"exceeds the fixed scratch" in _lib.lib().afid_last_error()


def test_noalloc_rejects_misaligned_dph():
    """The bulk copies of the transforms need a 16-byte aligned dph; a
    misaligned pointer is refused on the host before any device work."""
    xc = np.linspace(0.0, 1.0, 33)
    rc = _lib.lib().afid_solve_pressure_correction_noalloc(
        C.c_void_p(8), 32, 16, 16, _lib.dptr(xc), 1.0, 1.0, 1.0, None)
    assert rc == -1
    assert b"16-byte aligned" in _lib.lib().afid_last_error()
