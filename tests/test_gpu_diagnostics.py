"""Output-time diagnostics on the device (GlobalQuantities, CalcStats,
CalcDissipationNu, SlabDumper) against the oracle on the same fields."""
import numpy as np
import pytest

from helpers import cfg_of, oracle_state, FIELDS
from oracle import afid_oracle as O
from afid_b200.ic import initial_fields

pytestmark = pytest.mark.gpu

TOL = 1e-12   # relative: sums over the same values in a different order


def _box_and_state(ctx, cfg, steps=3, seed=7):
    box = ctx.add_box(cfg)
    for k, v in initial_fields(cfg, box.xc, seed=seed).items():
        box.upload(k, v)
    ctx.step([box], steps)
    s = oracle_state(cfg, seed=None)
    for f in ("vx", "vy", "vz", "temp"):
        getattr(s, f)[...] = box.download(f)
    return box, s


def _close(a, b, tol=TOL):
    return abs(a - b) <= tol * max(abs(b), 1e-300)


def test_global_quantities(ctx):
    cfg = cfg_of(40, 32, 24, ray=1e6, zlen=0.75)
    box, s = _box_and_state(ctx, cfg)
    g = box.global_quantities()
    o = O.global_quantities(s)
    for k in ("nu_vol", "tempm", "vx_rms", "vy_rms", "vz_rms", "vel_rms"):
        assert _close(g[k], o[k]), (k, g[k], o[k])
    assert g["vmax"] == o["vmax"] and g["tempmax"] == o["tempmax"] and g["tempmin"] == o["tempmin"]
    ctx.remove_box(box)


def test_dissipation_and_stats(ctx):
    cfg = cfg_of(40, 32, 24, ray=1e6, zlen=0.75)
    box, s = _box_and_state(ctx, cfg)
    mu, th = box.calc_dissipation_nu()
    d = O.calc_dissipation_nu(s)
    assert _close(mu, d["nu_mu"]) and _close(th, d["nu_th"])
    box.calc_stats()
    box.calc_stats()
    st = box.stats()
    acc = O.calc_stats(s)
    acc = O.calc_stats(s, acc)
    assert st["nstatsamples"] == 2
    # the plane means of vx, vy, vz cancel to roundoff: compare against the
    # sums of the magnitudes of their terms
    sa = s.copy()
    for f in ("vx", "vy", "vz", "temp"):
        getattr(sa, f)[...] = np.abs(getattr(s, f))
    mag = O.calc_stats(sa)
    for name in O.STAT_NAMES[:9]:
        assert np.all(np.abs(st[name] - acc[name]) <= TOL * 2 * mag[name] + 1e-300), name
    for name in ("disste", "dissth"):
        assert np.abs(st[name] - d[name]).max() <= TOL * np.abs(d[name]).max(), name
    box.reset_stats()
    assert box.stats()["nstatsamples"] == 0 and not box.stats()["vx_me"].any()
    ctx.remove_box(box)


def test_slab_dump_is_exact(ctx):
    cfg = cfg_of(32, 24, 16, ray=1e5)
    box, s = _box_and_state(ctx, cfg, steps=2)
    ks = [2, 9, 17, 32]
    got = box.slab_dump(ks)
    want = O.slab_dump(s, ks)
    assert got.shape == (4, 4, cfg.nym, cfg.nzm)
    assert np.array_equal(got, want)
    from afid_b200._lib import AfidError
    with pytest.raises(AfidError):
        box.slab_dump([0])
    ctx.remove_box(box)
