"""Continua files (WriteFlowField / ReadFlowField layout without HDF5)."""
import json
import os

import numpy as np
import pytest

from afid_b200 import continua
from helpers import cfg_of


def _fields(cfg, seed=0):
    rng = np.random.default_rng(seed)
    return {f: rng.standard_normal((cfg.nxm + 1, cfg.nym, cfg.nzm)) for f in continua.FIELDS}


def test_roundtrip_and_layout(tmp_path):
    cfg = cfg_of(12, 8, 6)
    f = _fields(cfg)
    continua.write_fields(str(tmp_path), cfg, f, time=1.25)
    m = json.load(open(tmp_path / "continua_master.json"))
    assert (m["nx"], m["ny"], m["nz"], m["time"]) == (13, 9, 7, 1.25)
    raw = np.fromfile(tmp_path / "continua_vx.bin", dtype="<f8")
    # Fortran order of (nx, nym, nzm): x fastest, then y, then z
    assert raw[1] == f["vx"][1, 0, 0] and raw[13] == f["vx"][0, 1, 0] and raw[13 * 8] == f["vx"][0, 0, 1]
    g, t = continua.read_fields(str(tmp_path), cfg)
    assert t == 1.25
    for k in continua.FIELDS:
        assert np.array_equal(g[k], f[k])


def test_other_grid_is_refused(tmp_path):
    cfg = cfg_of(12, 8, 6)
    continua.write_fields(str(tmp_path), cfg, _fields(cfg), time=0.0)
    with pytest.raises(ValueError):
        continua.read_fields(str(tmp_path), cfg_of(16, 8, 6))
    with pytest.raises(ValueError):
        continua.write_fields(str(tmp_path), cfg, {k: np.zeros((3, 3, 3)) for k in continua.FIELDS}, 0.0)


@pytest.mark.gpu
def test_box_restart_restores_fields_and_time(ctx, tmp_path):
    from afid_b200.ic import initial_fields
    cfg = cfg_of(24, 16, 12, ray=1e5, zlen=0.75)
    a = ctx.add_box(cfg)
    for k, v in initial_fields(cfg, a.xc, seed=3).items():
        a.upload(k, v)
    ctx.step([a], 3)
    continua.write_flow_field(a, str(tmp_path))
    b = ctx.add_box(cfg)
    t = continua.read_flow_field(b, str(tmp_path))
    assert t == a.scalars()["time"] == b.scalars()["time"]
    for k in continua.FIELDS:
        assert np.array_equal(a.download(k), b.download(k)), k
    ctx.step([b], 2)
    assert b.scalars()["status"] == 0 and b.scalars()["time"] > t
    for x in (a, b):
        ctx.remove_box(x)
