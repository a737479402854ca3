"""Initial conditions.

``initial_fields(cfg, xc, seed)``: velocities and pressure zero, temperature
linear between the plates (CreateInitialConditions.F90:39-52) plus uniform
noise in [-amp, amp] at the interior nodes k = 2..nxm, drawn from numpy's
PCG64(seed) in Fortran order (x fastest, then y, then z).
"""
from __future__ import annotations

import numpy as np

from .config import BouIn


def seeded_noise(nxm: int, nym: int, nzm: int, seed: int, amp: float = 0.01) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    raw = rng.uniform(-amp, amp, size=(nzm, nym, nxm - 1))
    return np.ascontiguousarray(raw.transpose(2, 1, 0))


def initial_fields(cfg: BouIn, xc: np.ndarray, seed: int | None = 0, amp: float = 0.01) -> dict:
    nx, nxm, nym, nzm = cfg.nx, cfg.nxm, cfg.nym, cfg.nzm
    tb, tt = cfg.tempbp, cfg.temptp
    temp = np.zeros((nx, nym, nzm))
    for k in range(1, nxm):
        temp[k] = tb - (tb - tt) * xc[k] / xc[nx - 1]
    temp[0] = tb
    temp[nx - 1] = tt
    if seed is not None:
        temp[1:nxm] += seeded_noise(nxm, nym, nzm, seed, amp)
    z = lambda: np.zeros((nx, nym, nzm))
    return {"vx": z(), "vy": z(), "vz": z(), "pr": z(), "temp": temp}
