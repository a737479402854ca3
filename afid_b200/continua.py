"""Continua (restart) files in the reference's layout, without HDF5.

WriteFlowField.F90:11-46 writes continua_temp, continua_vx, continua_vy and
continua_vz (the arrays (1:nx, 1:nym, 1:nzm) in Fortran order, x fastest)
and a master record continua_master with nx, ny, nz, ylen, zlen, time,
istr3 and str3.  ReadFlowField.F90 reads them back.  This image has no
HDF5, so the same content is stored as raw little-endian FP64 files
``continua_<field>.bin`` (same element order as the HDF5 datasets) and a
JSON master record ``continua_master.json`` with the same names.  A restart
on the same grid restores the four fields and the time; the reference's
interpolation onto a different grid (ReadFlowField.F90 with interp.F90) is
not provided.
"""
from __future__ import annotations

import json
import os

import numpy as np

FIELDS = ("temp", "vx", "vy", "vz")


def write_fields(path: str, cfg, fields: dict, time: float) -> None:
    """Write ``fields`` (arrays a[k, j, i] of shape (nx, nym, nzm)) and the
    master record into directory ``path``."""
    os.makedirs(path, exist_ok=True)
    shape = (cfg.nxm + 1, cfg.nym, cfg.nzm)
    for name in FIELDS:
        a = np.asarray(fields[name], dtype="<f8")
        if a.shape != shape:
            raise ValueError(f"{name}: shape {a.shape}, expected {shape}")
        # Fortran order of (nx, nym, nzm): x fastest
        a.ravel(order="F").tofile(os.path.join(path, f"continua_{name}.bin"))
    master = {"nx": cfg.nxm + 1, "ny": cfg.nym + 1, "nz": cfg.nzm + 1, "ylen": cfg.ylen,
              "zlen": cfg.zlen, "time": float(time), "istr3": cfg.istr3, "str3": cfg.str3}
    with open(os.path.join(path, "continua_master.json"), "w") as fh:
        json.dump(master, fh, indent=1)


def read_fields(path: str, cfg) -> tuple[dict, float]:
    """Read the four fields (arrays a[k, j, i]) and the time; the grid of
    the files must be the grid of ``cfg``."""
    with open(os.path.join(path, "continua_master.json")) as fh:
        m = json.load(fh)
    want = (cfg.nxm + 1, cfg.nym + 1, cfg.nzm + 1)
    got = (m["nx"], m["ny"], m["nz"])
    if got != want:
        raise ValueError(f"continua grid (nx, ny, nz) = {got} differs from {want}: "
                         "interpolation onto a new grid is not provided")
    if m["istr3"] != cfg.istr3 or m["str3"] != cfg.str3:
        raise ValueError("continua were written on another x grid (istr3/str3)")
    shape = (cfg.nxm + 1, cfg.nym, cfg.nzm)
    out = {}
    for name in FIELDS:
        a = np.fromfile(os.path.join(path, f"continua_{name}.bin"), dtype="<f8")
        if a.size != np.prod(shape):
            raise ValueError(f"continua_{name}.bin holds {a.size} values, expected {np.prod(shape)}")
        out[name] = a.reshape(shape, order="F")
    return out, float(m["time"])


def write_flow_field(box, path: str) -> None:
    """WriteFlowField: the box's temp, vx, vy, vz and its time."""
    write_fields(path, box.cfg, {f: box.download(f) for f in FIELDS}, box.scalars()["time"])


def read_flow_field(box, path: str) -> float:
    """ReadFlowField on the same grid: upload the four fields, set the time;
    returns the time."""
    fields, time = read_fields(path, box.cfg)
    for name, a in fields.items():
        box.upload(name, a)
    box.set_time(time)
    return time
