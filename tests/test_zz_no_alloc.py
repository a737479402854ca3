"""The pressure solve that allocates nothing (afid_solve_pressure_correction_noalloc).

Some callers cannot allocate device memory while they run: an application
that has handed its GPU memory to its own pool, code that runs where
cudaMalloc is not allowed, or a host program that must keep a fixed device
footprint.  They pass their own dph array and the library uses a fixed
scratch array of its own.  Through the C-ABI, calls in a row on shapes A, B
(larger) and A again must each give
  * the oracle's SolvePressureCorrection to 1e-12 (volume mean removed), and
  * bit for bit the regular entry point (afid_solve_pressure_correction on a
    box), which runs the same kernels,
so that the scratch left by an earlier, larger call does no harm; the status
word they report is 0.  A call on a stream that is being captured is
refused.  The test allocates its device buffers with torch; the entry point
itself allocates nothing.

The file name makes pytest collect it last."""
import ctypes as C

import numpy as np
import pytest

from afid_b200 import _lib
from helpers import cfg_of, oracle_state, rel_l2
from oracle import afid_oracle as O

pytestmark = pytest.mark.gpu

SHAPES = {"A": ((24, 16, 20), dict(zlen=0.5)), "B": ((32, 48, 40), dict(ylen=1.5, zlen=1.25))}


def _regular(ctx, cfg, dph_kji):
    box = ctx.add_box(cfg)
    box.upload("dph", dph_kji)
    box.solve_pressure_correction()
    out = box.download("dph")
    xc = box.xc.copy()
    ctx.remove_box(box)
    return out, xc


def _call(cfg, xc, dev, stream, status):
    return _lib.lib().afid_solve_pressure_correction_noalloc(
        C.c_void_p(dev.data_ptr()), cfg.nxm, cfg.nym, cfg.nzm, _lib.dptr(xc), cfg.alx3,
        cfg.ylen, cfg.zlen, C.c_void_p(stream.cuda_stream), status)


def _noalloc(cfg, xc, dph_kji):
    import torch
    dev = torch.from_numpy(np.ascontiguousarray(dph_kji.transpose(0, 2, 1))).cuda()  # [k][i][j]
    stream = torch.cuda.current_stream()
    st = C.c_int(-7)
    _lib.check(_call(cfg, xc, dev, stream, C.byref(st)))
    stream.synchronize()
    return dev.cpu().numpy().transpose(0, 2, 1).copy(), st.value


def test_noalloc_matches_oracle_and_box_path_across_shapes(ctx):
    rng = np.random.default_rng(42)
    for call, name in enumerate(("A", "B", "A")):
        shape, kw = SHAPES[name]
        cfg = cfg_of(*shape, **kw)
        dph = rng.standard_normal((cfg.nxm, cfg.nym, cfg.nzm))
        want, xc = _regular(ctx, cfg, dph)
        got, status = _noalloc(cfg, xc, dph)
        assert status == 0, f"call {call} ({name}): status {status}"
        assert np.array_equal(got, want), f"call {call} ({name}): differs from the box path"
        s = oracle_state(cfg, seed=None)
        s.dph[...] = dph
        O.solve_pressure_correction(s)
        assert rel_l2(got, s.dph, remove_mean=True) <= 1e-12, f"call {call} ({name}) against the oracle"


def test_noalloc_refuses_a_capturing_stream():
    import torch
    cfg = cfg_of(24, 16, 20, zlen=0.5)
    xc = np.linspace(0.0, 1.0, cfg.nxm + 1)
    dev = torch.zeros((cfg.nxm, cfg.nzm, cfg.nym), dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        rc = _call(cfg, xc, dev, s, None)
    assert rc == -1
    assert b"captured" in _lib.lib().afid_last_error()


def test_noalloc_rejects_oversize():
    xc = np.linspace(0.0, 1.0, 513)
    rc = _lib.lib().afid_solve_pressure_correction_noalloc(
        C.c_void_p(1), 512, 1024, 1024, _lib.dptr(xc), 1.0, 1.0, 1.0, None, None)
    assert rc == -6
    assert b"exceeds the fixed scratch" in _lib.lib().afid_last_error()


def test_noalloc_rejects_misaligned_dph():
    """The bulk copies of the transforms need a 16-byte aligned dph; a
    misaligned pointer is refused on the host before any device work."""
    xc = np.linspace(0.0, 1.0, 33)
    rc = _lib.lib().afid_solve_pressure_correction_noalloc(
        C.c_void_p(8), 32, 16, 16, _lib.dptr(xc), 1.0, 1.0, 1.0, None, None)
    assert rc == -1
    assert b"16-byte aligned" in _lib.lib().afid_last_error()
