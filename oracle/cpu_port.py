"""ctypes wrapper of oracle/afid_cpu.c (the multi-threaded C restatement).

TEST INFRASTRUCTURE ONLY: used by the tests (cross-check against the NumPy
oracle) and by the CPU-baseline leg of bench.py.  Build with ``make -C oracle``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libafid_cpu.so")
FIELD = {"vx": 0, "vy": 1, "vz": 2, "temp": 3, "pr": 4, "rux": 5, "ruy": 6, "ruz": 7, "rutemp": 8,
         "dph": 9}


class Params(C.Structure):
    _fields_ = [("nxm", C.c_int), ("nym", C.c_int), ("nzm", C.c_int), ("nsst", C.c_int),
                ("inslws", C.c_int), ("inslwn", C.c_int), ("alx3", C.c_double), ("ylen", C.c_double),
                ("zlen", C.c_double), ("ray", C.c_double), ("pra", C.c_double),
                ("tempbp", C.c_double), ("temptp", C.c_double)]


_L = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def lib() -> C.CDLL:
    global _L
    if _L is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.afid_cpu_create.restype = C.c_void_p
        L.afid_cpu_create.argtypes = [C.POINTER(Params), C.POINTER(C.c_double)]
        L.afid_cpu_destroy.argtypes = [C.c_void_p]
        L.afid_cpu_set.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double)]
        L.afid_cpu_get.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double)]
        L.afid_cpu_step.argtypes = [C.c_void_p, C.c_double, C.c_int]
        _L = L
    return _L


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class CpuBox:
    """One box advanced by the C restatement; fields cross as a[k, j, i]."""

    def __init__(self, cfg, xc):
        self.cfg = cfg
        p = Params(cfg.nxm, cfg.nym, cfg.nzm, cfg.nsst, cfg.inslws, cfg.inslwn, cfg.alx3, cfg.ylen,
                   cfg.zlen, cfg.ray, cfg.pra, cfg.tempbp, cfg.temptp)
        xc = np.ascontiguousarray(xc, dtype=np.float64)
        self.h = lib().afid_cpu_create(C.byref(p), _p(xc))
        if not self.h:
            raise ValueError("afid_cpu_create rejected the box")

    def set(self, name, a):
        buf = np.ascontiguousarray(np.asarray(a, dtype=np.float64).transpose(0, 2, 1))
        if lib().afid_cpu_set(self.h, FIELD[name], _p(buf)):
            raise ValueError(name)

    def get(self, name):
        rows = self.cfg.nxm if name == "dph" else self.cfg.nxm + 1
        buf = np.empty((rows, self.cfg.nzm, self.cfg.nym))
        if lib().afid_cpu_get(self.h, FIELD[name], _p(buf)):
            raise ValueError(name)
        return np.ascontiguousarray(buf.transpose(0, 2, 1))

    def step(self, dt, nsteps=1):
        lib().afid_cpu_step(self.h, dt, nsteps)

    def close(self):
        if self.h:
            lib().afid_cpu_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
