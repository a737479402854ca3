"""Long-run series of the plain single-box configuration on the CPU, for the
"mean Nu within 1% over long runs" check of the GPU run driver.

    python tests/golden/make_longrun.py [nsteps]

Box 65x64x64 (Ra=1e6, Pr=1, aspect ratio 1, dt=5e-4, seed 0), advanced by
the C/OpenMP restatement of the reference (oracle/afid_cpu.c) under the host
loop of main.F90:167-279 with TOUT = 1e-2: at each output time (the loop's
second step, then every step after which mod(time, tout) < dt) the oracle's
GlobalQuantities and CalcPlateNu are evaluated on the port's fields.  Writes
golden_c1_longrun.npz: time, nu_vol, nu_bot, nu_top per output time, and the
step count.
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import afid_oracle as O  # noqa: E402
from oracle.cpu_port import CpuBox  # noqa: E402
from helpers import cfg_of, oracle_state, FIELDS  # noqa: E402

TOUT = 1e-2
NSTEPS = 30000


def main(nsteps: int = NSTEPS):
    cfg = cfg_of(64, 64, 64, ray=1e6, pra=1.0, dt=5e-4)
    s = oracle_state(cfg, seed=0)
    box = CpuBox(cfg, s.g.xc)
    for f in FIELDS:
        box.set(f, getattr(s, f))
    t, out = 0.0, {"time": [], "nu_vol": [], "nu_bot": [], "nu_top": []}
    for n in range(1, nsteps + 1):
        box.step(cfg.dt, 1)
        t += cfg.dt
        if n == 2 or math.fmod(t, TOUT) < cfg.dt:
            for f in FIELDS:
                getattr(s, f)[...] = box.get(f)
            g = O.global_quantities(s)
            lo, up = O.calc_plate_nu(s)
            out["time"].append(t)
            out["nu_vol"].append(g["nu_vol"])
            out["nu_bot"].append(lo)
            out["nu_top"].append(up)
    box.close()
    np.savez_compressed(os.path.join(HERE, "golden_c1_longrun.npz"), nsteps=nsteps, tout=TOUT,
                        **{k: np.array(v) for k, v in out.items()})
    print(f"{len(out['time'])} output times; last nu_vol {out['nu_vol'][-1]:.6f}")


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else NSTEPS)
