"""Generate the golden fixtures of the parity tests with the CPU oracle.

    python tests/golden/make_golden.py

golden_small.npz  box 25x16x12 (nxm=24), Ra=1e5, Pr=0.7, zlen=0.75,
                  dt=5e-4, seed 11: fields after 1 and 5 RK3 steps plus the
                  per-step records.
golden_c1_nu.npz  box 65x64x64, Ra=1e6, Pr=1, dt=5e-4, seed 0 (the plain
                  single-box configuration): per-step plate Nusselt numbers,
                  dt and max divergence for 100 steps, plus per-field
                  checksums (sum, sum of squares) after 100 steps.
golden_c1_seeds.npz  the same box for seeds 0, 1 and 2: per-step plate
                  Nusselt numbers and dt of the first 100 steps
                  (keys s<seed>_nu_bot, s<seed>_nu_top, s<seed>_dt).
The Fortran reference cannot be compiled here, so these vectors pin the
oracle against itself across changes (regression) and pin the CUDA path
against the oracle; the oracle is pinned to the reference's formulas by the
analytic known-answer tests of tests/test_oracle_kat.py.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import afid_oracle as O  # noqa: E402
from helpers import cfg_of, oracle_state, FIELDS  # noqa: E402

SMALL = dict(nxm=24, nym=16, nzm=12, ray=1e5, pra=0.7, zlen=0.75, dt=5e-4)
C1 = dict(nxm=64, nym=64, nzm=64, ray=1e6, pra=1.0, dt=5e-4)


def small():
    cfg = cfg_of(**SMALL)
    s = oracle_state(cfg, seed=11)
    out = {}
    recs = O.run(s, 1, cfg.dt)
    for f in FIELDS:
        out[f"step1_{f}"] = getattr(s, f).copy()
    recs += O.run(s, 4, cfg.dt)
    for f in FIELDS:
        out[f"step5_{f}"] = getattr(s, f).copy()
    out["nu_bot"] = np.array([r["nu_bot"] for r in recs])
    out["nu_top"] = np.array([r["nu_top"] for r in recs])
    out["div"] = np.array([r["div"] for r in recs])
    np.savez_compressed(os.path.join(HERE, "golden_small.npz"), **out)


def c1(nsteps=100):
    cfg = cfg_of(**C1)
    s = oracle_state(cfg, seed=0)
    recs = O.run(s, nsteps, cfg.dt, vectorised_poisson=True)
    out = {"nu_bot": np.array([r["nu_bot"] for r in recs]),
           "nu_top": np.array([r["nu_top"] for r in recs]),
           "dt": np.array([r["dt"] for r in recs]),
           "div": np.array([r["div"] for r in recs])}
    for f in FIELDS:
        a = getattr(s, f)
        if f == "pr":
            a = a[:-1] - a[:-1].mean()
        out[f"sum_{f}"] = np.array([a.sum(), (a * a).sum()])
    np.savez_compressed(os.path.join(HERE, "golden_c1_nu.npz"), **out)


def c1_seeds(seeds=(0, 1, 2), nsteps=100):
    cfg = cfg_of(**C1)
    out = {}
    for seed in seeds:
        s = oracle_state(cfg, seed=seed)
        recs = O.run(s, nsteps, cfg.dt, vectorised_poisson=True)
        out[f"s{seed}_nu_bot"] = np.array([r["nu_bot"] for r in recs])
        out[f"s{seed}_nu_top"] = np.array([r["nu_top"] for r in recs])
        out[f"s{seed}_dt"] = np.array([r["dt"] for r in recs])
    np.savez_compressed(os.path.join(HERE, "golden_c1_seeds.npz"), **out)


if __name__ == "__main__":
    which = sys.argv[1:] or ["small", "c1", "c1_seeds"]
    if "small" in which:
        small()
    if "c1" in which:
        c1()
    if "c1_seeds" in which:
        c1_seeds()
    print("golden fixtures written")
