"""Restart onto a new grid on the device (afid_box_interp_field, the
interpolation of ReadFlowField.F90:63-150 / interp.F90) against the oracle's
restatement, bit for bit, and through the continua reader."""
import numpy as np
import pytest

from afid_b200 import continua
from afid_b200._lib import AfidError
from afid_b200.ic import initial_fields
from helpers import cfg_of
from oracle import afid_oracle as O

pytestmark = pytest.mark.gpu

# old grid (nxo, nyo, nzo, istro3, stro3) -> new box: refinement with a change
# of stretching, and coarsening
CASES = [
    ((17, 17, 13, 0, 0.0), dict(nxm=24, nym=24, nzm=20, istr3=6, str3=2.0)),
    ((25, 33, 25, 6, 3.0), dict(nxm=16, nym=16, nzm=16, istr3=6, str3=3.0)),
]


@pytest.mark.parametrize("case", CASES)
def test_device_regrid_matches_oracle(ctx, case):
    (nxo, nyo, nzo, isto, sto), kw = case
    cfg = cfg_of(kw["nxm"], kw["nym"], kw["nzm"], ylen=1.5, zlen=2.0, istr3=kw["istr3"], str3=kw["str3"])
    b = ctx.add_box(cfg, validate=False)
    rng = np.random.default_rng(7)
    for name in ("vx", "vy", "vz", "temp"):
        old = rng.standard_normal((nxo, nyo - 1, nzo - 1))
        b.interp_field(name, old, nxo, nyo, nzo, isto, sto)
        want = O.interp_field(old, nxo, nyo, nzo, isto, sto, O.INTERP_FLAG[name], cfg.nxm, cfg.nym, cfg.nzm,
                              cfg.istr3, cfg.str3, cfg.ylen, cfg.zlen)
        assert np.array_equal(b.download(name), want), name
    ctx.remove_box(b)


def test_restart_on_a_finer_grid(ctx, tmp_path):
    coarse = cfg_of(16, 16, 12, ray=1e5, istr3=6, str3=2.0)
    a = ctx.add_box(coarse, validate=False)
    for k, v in initial_fields(coarse, a.xc, seed=4).items():
        a.upload(k, v)
    ctx.step([a], 2)
    continua.write_flow_field(a, str(tmp_path))
    fine = cfg_of(24, 24, 20, ray=1e5, istr3=6, str3=2.0)
    b = ctx.add_box(fine, validate=False)
    t = continua.read_flow_field(b, str(tmp_path))
    assert t == a.scalars()["time"] == b.scalars()["time"]
    m = continua.read_master(str(tmp_path))
    raw = continua.read_raw(str(tmp_path), m)
    for name in continua.FIELDS:
        want = O.interp_field(raw[name], m["nx"], m["ny"], m["nz"], m["istr3"], m["str3"], O.INTERP_FLAG[name],
                              fine.nxm, fine.nym, fine.nzm, fine.istr3, fine.str3, fine.ylen, fine.zlen)
        assert np.array_equal(b.download(name), want), name
    ctx.step([b], 2)
    assert b.scalars()["status"] == 0 and b.scalars()["time"] > t
    for x in (a, b):
        ctx.remove_box(x)


def test_regrid_conditions_on_device(ctx):
    b = ctx.add_box(cfg_of(24, 24, 20, istr3=6, str3=2.0), validate=False)
    with pytest.raises(AfidError):   # more than twice the old points in y
        b.interp_field("vx", np.zeros((17, 11, 12)), 17, 12, 13, 0, 0.0)
    with pytest.raises(AfidError):   # old wall-normal grid that gridnew does not define
        b.interp_field("vx", np.zeros((17, 16, 12)), 17, 17, 13, 4, 1.0)
    with pytest.raises(AfidError):   # pr is not a continua field
        b.interp_field("pr", np.zeros((17, 16, 12)), 17, 17, 13, 0, 0.0)
    c = ctx.add_box(cfg_of(24, 24, 20), validate=False)   # istr3 = 7 for the new grid
    with pytest.raises(AfidError):
        c.interp_field("vx", np.zeros((17, 16, 12)), 17, 17, 13, 0, 0.0)
    for x in (b, c):
        ctx.remove_box(x)
