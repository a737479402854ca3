"""The compiled C restatement (oracle/afid_cpu.c) against the NumPy oracle."""
import numpy as np
import pytest

from helpers import cfg_of, oracle_state, rel_l2, FIELDS
from oracle import afid_oracle as O
from oracle.cpu_port import CpuBox


@pytest.mark.parametrize("shape,kw", [((24, 16, 12), dict(ray=1e5, pra=0.7, zlen=0.75)),
                                      ((16, 20, 40), dict(ray=3e6, pra=4.38, zlen=2.0)),
                                      ((18, 12, 8), dict(ray=1e6, inslws=0, istr3=6, str3=4.0))])
def test_cpu_port_matches_oracle(shape, kw):
    cfg = cfg_of(*shape, dt=5e-4, **kw)
    s = oracle_state(cfg, seed=2)
    box = CpuBox(cfg, s.g.xc)
    for f in FIELDS:
        box.set(f, getattr(s, f))
    O.run(s, 3, cfg.dt)
    box.step(cfg.dt, 3)
    for f in FIELDS:
        a, b = box.get(f), getattr(s, f)
        if f == "pr":
            a, b = a[:-1], b[:-1]
        assert rel_l2(a, b, remove_mean=(f == "pr")) <= 1e-12, f
    box.close()
