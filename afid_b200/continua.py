"""Continua (restart) files in the reference's layout, without HDF5.

WriteFlowField.F90:11-46 writes continua_temp, continua_vx, continua_vy and
continua_vz (the arrays (1:nx, 1:nym, 1:nzm) in Fortran order, x fastest)
and a master record continua_master with nx, ny, nz, ylen, zlen, time,
istr3 and str3.  ReadFlowField.F90 reads them back.  This image has no
HDF5, so the same content is stored as raw little-endian FP64 files
``continua_<field>.bin`` (same element order as the HDF5 datasets) and a
JSON master record ``continua_master.json`` with the same names.  A restart
on the same grid restores the four fields and the time; on another grid
(ReadFlowField.F90:63-150) each field is interpolated onto the box's grid by
the library (interp.F90), under the reference's conditions.
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


def read_master(path: str) -> dict:
    with open(os.path.join(path, "continua_master.json")) as fh:
        return json.load(fh)


def same_grid(m: dict, cfg) -> bool:
    """ReadFlowField.F90:75-77: no interpolation when nx, ny, nz and istr3
    match and str3 differs by at most 1e-8."""
    return (m["ny"] == cfg.nym + 1 and m["nx"] == cfg.nxm + 1 and m["nz"] == cfg.nzm + 1
            and m["istr3"] == cfg.istr3 and not abs(m["str3"] - cfg.str3) > 1e-8)


def read_raw(path: str, m: dict) -> dict:
    """The four datasets of continua files with master record ``m``, as
    arrays a[k, j, i] of shape (nx, ny-1, nz-1) of the files' grid."""
    shape = (m["nx"], m["ny"] - 1, m["nz"] - 1)
    out = {}
    for name in FIELDS:
        a = np.fromfile(os.path.join(path, f"continua_{name}.bin"), dtype="<f8")
        if a.size != np.prod(shape):
            raise ValueError(f"continua_{name}.bin holds {a.size} values, expected {np.prod(shape)}")
        out[name] = a.reshape(shape, order="F")
    return out


def read_fields(path: str, cfg) -> tuple[dict, float]:
    """Read the four fields (arrays a[k, j, i]) and the time; the grid of
    the files must be the grid of ``cfg``."""
    m = read_master(path)
    if not same_grid(m, cfg):
        raise ValueError(f"continua grid (nx, ny, nz, istr3, str3) = "
                         f"{(m['nx'], m['ny'], m['nz'], m['istr3'], m['str3'])} differs from the box's: "
                         "use read_flow_field, which interpolates")
    return read_raw(path, m), float(m["time"])


def write_flow_field(box, path: str) -> None:
    """WriteFlowField: the box's temp, vx, vy, vz and its time."""
    write_fields(path, box.cfg, {f: box.download(f) for f in FIELDS}, box.scalars()["time"])


def read_flow_field(box, path: str) -> float:
    """ReadFlowField: the four fields onto the box (uploaded as they are on
    the same grid, interpolated on the device onto the box's grid
    otherwise), then the time; returns the time."""
    m = read_master(path)
    fields = read_raw(path, m)
    if same_grid(m, box.cfg):
        for name, a in fields.items():
            box.upload(name, a)
    else:
        # ReadFlowField.F90:102-150 regrids vz, vy, vx, temp in that order
        for name in ("vz", "vy", "vx", "temp"):
            box.interp_field(name, fields[name], m["nx"], m["ny"], m["nz"], m["istr3"], m["str3"])
    box.set_time(float(m["time"]))
    return float(m["time"])
