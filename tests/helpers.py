"""Shared helpers of the parity tests: run the same seeded case through the
oracle and through the library."""
from __future__ import annotations

import numpy as np

from afid_b200 import BouIn
from afid_b200.ic import initial_fields
from oracle import afid_oracle as O

FIELDS = ("vx", "vy", "vz", "temp", "pr")


def cfg_of(nxm, nym, nzm, ray=1e6, pra=1.0, ylen=1.0, zlen=1.0, dt=5e-4, istr3=7, str3=0.0,
           nsst=3, inslws=1, inslwn=1, idtv=0, cflmax=1.2, dtmin=1e-8, dtmax=1e-2, resid=0.0,
           vlim=1e3):
    return BouIn(nxm=nxm, nym=nym, nzm=nzm, ray=ray, pra=pra, ylen=ylen, zlen=zlen, dt=dt,
                 istr3=istr3, str3=str3, nsst=nsst, inslws=inslws, inslwn=inslwn, idtv=idtv,
                 cflmax=cflmax, dtmin=dtmin, dtmax=dtmax, resid=resid, vlim=vlim)


def oracle_params(cfg: BouIn) -> O.Params:
    return O.Params(nxm=cfg.nxm, nym=cfg.nym, nzm=cfg.nzm, ylen=cfg.ylen, zlen=cfg.zlen,
                    ray=cfg.ray, pra=cfg.pra, alx3=cfg.alx3, istr3=cfg.istr3, str3=cfg.str3,
                    inslws=cfg.inslws, inslwn=cfg.inslwn, nsst=cfg.nsst,
                    tempbp=cfg.tempbp, temptp=cfg.temptp)


def oracle_state(cfg: BouIn, seed=0, fields=None) -> O.State:
    p = oracle_params(cfg)
    s = O.init_state(p, seed=None, ic="conduction")
    f = fields if fields is not None else initial_fields(cfg, s.g.xc, seed)
    for k, v in f.items():
        getattr(s, k)[...] = v
    return s


def rel_l2(a, b, remove_mean=False):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if remove_mean:
        a = a - a.mean()
        b = b - b.mean()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def compare_fields(box, s: O.State, nxm_pr=True):
    """Per-field relative L2 between a device box and an oracle state; pr is
    compared on rows 1..nxm after removing its volume mean."""
    out = {}
    for f in FIELDS:
        d = box.download(f)
        o = getattr(s, f)
        if f == "pr":
            out[f] = rel_l2(d[:-1], o[:-1], remove_mean=True)
        elif f in ("vy", "vz"):
            out[f] = rel_l2(d[:-1], o[:-1])
        else:
            out[f] = rel_l2(d, o)
    return out
