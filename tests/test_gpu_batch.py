"""Batched boxes of uneven size and physics advance exactly as when alone;
CUDA-graph replay is bitwise identical to direct launches; per-box status
codes retire a failing box without touching the others."""
import numpy as np
import pytest

from afid_b200 import Context
from afid_b200.ic import initial_fields
from helpers import cfg_of, FIELDS

pytestmark = pytest.mark.gpu

MIX = [
    dict(nxm=32, nym=32, nzm=48, ray=1e5, pra=0.7, ylen=1.0, zlen=1.5, dt=2e-4),
    dict(nxm=64, nym=48, nzm=48, ray=1e7, pra=4.38, dt=1e-4),
    dict(nxm=96, nym=128, nzm=96, ray=3e6, pra=1.0, ylen=1.33, zlen=1.0, dt=1e-4),
    dict(nxm=32, nym=64, nzm=64, ray=1e8, pra=1.0, ylen=2.0, zlen=2.0, dt=5e-5),
]


def _add(ctx, kw, seed):
    cfg = cfg_of(**kw)
    b = ctx.add_box(cfg)
    for k, v in initial_fields(cfg, b.xc, seed).items():
        b.upload(k, v)
    return b


def test_batch_equals_alone_and_graph_equals_direct(ctx):
    batch = [_add(ctx, kw, 10 + q) for q, kw in enumerate(MIX)]
    alone = [_add(ctx, kw, 10 + q) for q, kw in enumerate(MIX)]
    graphed = [_add(ctx, kw, 10 + q) for q, kw in enumerate(MIX)]
    ctx.step(batch, 3)
    for b in alone:
        ctx.step([b], 3)
    ctx.step(graphed, 3, graph=True)
    for a, b, g in zip(batch, alone, graphed):
        for f in FIELDS:
            fa, fb, fg = a.download(f), b.download(f), g.download(f)
            assert np.array_equal(fa, fb), f
            assert np.array_equal(fa, fg), f
        assert a.scalars() == b.scalars()
    for b in batch + alone + graphed:
        ctx.remove_box(b)


def test_nonfinite_box_is_retired_others_continue(ctx):
    good = _add(ctx, MIX[0], 1)
    ref = _add(ctx, MIX[0], 1)
    bad = _add(ctx, MIX[1], 2)
    t = bad.download("temp")
    t[5, 3, 4] = np.nan
    bad.upload("temp", t)
    ctx.step([good, bad], 2)
    ctx.step([ref], 2)
    assert bad.scalars()["status"] == 266
    assert good.scalars()["status"] == 0
    for f in FIELDS:
        assert np.array_equal(good.download(f), ref.download(f))
    for b in (good, ref, bad):
        ctx.remove_box(b)


def test_cfl_and_dtmin_codes(ctx):
    # fixed dt with CFL*dt above CFLMAX: code 165 (main.F90:186-189)
    kw = dict(MIX[0]); kw.update(dt=1.0, cflmax=1e-9)
    b = _add(ctx, kw, 3)
    v = b.download("vy"); v[:] = 1.0; b.upload("vy", v)
    ctx.step([b], 1)
    assert b.scalars()["status"] == 165
    # variable dt below dtmin: code 166 (main.F90:173-184)
    kw = dict(MIX[0]); kw.update(idtv=1, dtmin=1e-3, dtmax=2e-3, cflmax=1e-6)
    c = _add(ctx, kw, 4)
    v = c.download("vy"); v[:] = 1.0; c.upload("vy", v)
    ctx.step([c], 3)
    assert c.scalars()["status"] == 166
    for x in (b, c):
        ctx.remove_box(x)


def test_velocity_limit_code(ctx):
    kw = dict(MIX[0]); kw.update(vlim=0.5)
    b = _add(ctx, kw, 5)
    for f in ("vy", "vz"):
        v = b.download(f); v[:] = 1.0; b.upload(f, v)
    ctx.step([b], 1)
    assert b.scalars()["status"] == 266
    ctx.remove_box(b)


def test_fft_size_rule(ctx):
    from afid_b200._lib import AfidError
    with pytest.raises((AfidError, ValueError)):
        ctx.add_box(cfg_of(16, 22, 16))


@pytest.mark.parametrize("fy,fz,k1", [(1, 2, 3), (2, 1, 2), (4, 4, 5), (2, 8, 6), (1, 4, 7), (8, 2, 8)])
def test_launch_shapes_do_not_change_results(ctx, fy, fz, k1):
    """Tuned launch shapes (FFT lines per block, tile shape and occupancy of
    the explicit kernel) give bit-identical fields to the defaults (explicit
    kernel variant 4)."""
    a = _add(ctx, MIX[2], 21)
    b = _add(ctx, MIX[2], 21)
    b.set_tuning(fft_y_lines=fy, fft_z_lines=fz, k1_minb=k1)
    ctx.step([a], 3)
    ctx.step([b], 3)
    for f in FIELDS:
        assert np.array_equal(a.download(f), b.download(f)), f
    from afid_b200._lib import AfidError
    for bad in (dict(fft_y_lines=10 ** 6), dict(fft_y_lines=3), dict(fft_z_lines=6), dict(k1_minb=9)):
        with pytest.raises(AfidError):
            b.set_tuning(**bad)
    for x in (a, b):
        ctx.remove_box(x)


def test_batch_tuning_keeps_results(ctx):
    """autotune.tune_batch chooses the launch shapes on the set itself; the
    chosen shapes change no result bit."""
    from afid_b200 import autotune
    tuned = [_add(ctx, kw, 20 + q) for q, kw in enumerate(MIX)]
    plain = [_add(ctx, kw, 20 + q) for q, kw in enumerate(MIX)]
    choice = autotune.tune_batch(ctx, tuned, steps=1)
    assert choice["k1_minb"] in autotune.candidates(tuned[0].cfg)["k1_minb"]
    for b, kw, q in zip(tuned, MIX, range(len(MIX))):        # restart from the seeded state
        for k, v in initial_fields(b.cfg, b.xc, 20 + q).items():
            b.upload(k, v)
        b.reset(b.cfg.dt)
    ctx.step(tuned, 2, graph=True)
    ctx.step(plain, 2, graph=True)
    for a, b in zip(tuned, plain):
        for f in FIELDS:
            assert np.array_equal(a.download(f), b.download(f)), f
    for b in tuned + plain:
        ctx.remove_box(b)


def test_async_transfers_and_batched_scalars(ctx):
    """afid_box_upload_async / afid_box_download_async queued for several
    boxes and fields, then one wait, give the same device fields and host
    arrays as the waiting transfers; afid_boxes_get_scalars gives every
    box's afid_box_get_scalars record."""
    from afid_b200 import _lib
    L = _lib.lib()
    sync = [_add(ctx, kw, 30 + q) for q, kw in enumerate(MIX)]
    asyn = [ctx.add_box(b.cfg) for b in sync]
    keep = []
    for q, (s, a) in enumerate(zip(sync, asyn)):
        for k, v in initial_fields(s.cfg, s.xc, 30 + q).items():
            buf = np.ascontiguousarray(np.asarray(v, dtype=np.float64).transpose(2, 1, 0))
            keep.append(buf)
            _lib.check(L.afid_box_upload_async(ctx.h, a.id, _lib.FIELDS[k], _lib.dptr(buf)))
    ctx.synchronize()
    ctx.step(sync, 2)
    ctx.step(asyn, 2)
    recs = ctx.scalars(asyn)
    assert recs == [b.scalars() for b in asyn]
    assert recs == [b.scalars() for b in sync]
    # queued records: one slot per step, read after one wait
    import ctypes as C
    ids = (C.c_int * len(asyn))(*[b.id for b in asyn])
    slots = (_lib.BoxScalars * (2 * len(asyn)))()
    for q in range(2):
        ctx.step(asyn, 1)
        ptr = C.cast(C.addressof(slots) + q * len(asyn) * C.sizeof(_lib.BoxScalars), C.POINTER(_lib.BoxScalars))
        _lib.check(L.afid_boxes_get_scalars_async(ctx.h, ids, len(asyn), ptr))
    ctx.synchronize()
    assert [slots[len(asyn) + q].ntime for q in range(len(asyn))] == [r["ntime"] + 2 for r in recs]
    assert [slots[q].ntime for q in range(len(asyn))] == [r["ntime"] + 1 for r in recs]
    last = ctx.scalars(asyn)
    assert [slots[len(asyn) + q].time for q in range(len(asyn))] == [r["time"] for r in last]
    ctx.step(sync, 2)
    outs = []
    for a in asyn:
        for f in FIELDS:
            buf = np.empty((a.cfg.nzm, a.cfg.nym, a._rows(f)))
            outs.append((a, f, buf))
            _lib.check(L.afid_box_download_async(ctx.h, a.id, _lib.FIELDS[f], _lib.dptr(buf)))
    ctx.synchronize()
    for (a, f, buf), s in zip(outs, [s for s in sync for _ in FIELDS]):
        got = np.ascontiguousarray(buf.transpose(2, 1, 0))
        assert np.array_equal(got, a.download(f)), f
        assert np.array_equal(got, s.download(f)), f
    for b in sync + asyn:
        ctx.remove_box(b)
    del keep   # the upload buffers stay alive until the copies have run


def test_split_graph_equals_direct(ctx):
    """A set large enough for afid_step_graph to run it as two halves on two
    streams gives bit for bit the fields and records of the same set
    stepped by direct launches, and its graph step launches both halves'
    kernels."""
    kws = [dict(nxm=64, nym=96, nzm=96, ray=10 ** (5 + 0.4 * q), pra=(0.7, 1.0, 4.38)[q % 3], dt=1e-4)
           for q in range(8)]
    graphed = [_add(ctx, kw, 50 + q) for q, kw in enumerate(kws)]
    direct = [_add(ctx, kw, 50 + q) for q, kw in enumerate(kws)]
    ctx.step(graphed, 3, graph=True)
    ctx.step(direct, 3)
    for g, d in zip(graphed, direct):
        for f in FIELDS:
            assert np.array_equal(g.download(f), d.download(f)), f
        assert g.scalars() == d.scalars()
    one = ctx.graph_kernels(graphed[:1])
    split = ctx.graph_kernels(graphed)
    assert split > one
    ctx.set_split_sets(False)     # the whole set in one graph: one launch per stage
    try:
        assert ctx.graph_kernels(graphed) == one
        ctx.step(graphed, 1, graph=True)
        ctx.step(direct, 1)
        for g, d in zip(graphed, direct):
            assert np.array_equal(g.download("temp"), d.download("temp"))
    finally:
        ctx.set_split_sets(True)
    for b in graphed + direct:
        ctx.remove_box(b)


def test_queued_records_on_two_streams(ctx):
    """Two box sets stepped and read back on two streams of one context,
    queued one after the other with no wait between: each stream's records
    are its own set's (pageable memory through a per-stream staging array,
    pinned memory written directly), and a queued reset takes effect in
    stream order."""
    import ctypes as C

    import torch

    from afid_b200 import _lib
    L = _lib.lib()
    sets = [[_add(ctx, kw, 70 + 10 * h + q) for q, kw in enumerate(MIX[:2])] for h in range(2)]
    streams = [torch.cuda.Stream() for _ in sets]
    own = ctx.stream
    # stream 0 reads into pageable memory (a queued copy through the stream's
    # staging), stream 1 into pinned memory (written by the device itself)
    pinned = torch.empty(2 * C.sizeof(_lib.BoxScalars), dtype=torch.uint8, pin_memory=True)
    slots = [(_lib.BoxScalars * 2)(), (_lib.BoxScalars * 2).from_address(pinned.data_ptr())]
    try:
        for h, (boxes, st) in enumerate(zip(sets, streams)):
            ctx.set_stream(st.cuda_stream)
            ids = (C.c_int * 2)(*[b.id for b in boxes])
            if h == 1:
                for b in boxes:
                    b.reset(2e-5)
            ctx.step(boxes, 2 + h)
            _lib.check(L.afid_boxes_get_scalars_async(ctx.h, ids, 2, slots[h]))
        for st in streams:
            st.synchronize()
    finally:
        ctx.set_stream(own)
    for h, boxes in enumerate(sets):
        want = ctx.scalars(boxes)
        assert [slots[h][q].ntime for q in range(2)] == [r["ntime"] for r in want] == [2 + h] * 2
        assert [slots[h][q].time for q in range(2)] == [r["time"] for r in want]
    assert all(r["dt"] == 2e-5 for r in ctx.scalars(sets[1]))
    for b in sets[0] + sets[1]:
        ctx.remove_box(b)
