"""Long runs through the run driver (main.F90:167-279 over the library):
the mean Nusselt numbers, averaged as wnus.sh does, agree within 1% with the
C/OpenMP restatement of the reference run over the same steps
(tests/golden/golden_c1_longrun.npz, made by tests/golden/make_longrun.py),
and the run ends with the reference's exit code 555 after NTST."""
import os

import numpy as np
import pytest

from afid_b200 import BouIn
from afid_b200.driver import run, wnus_means

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_long_run_mean_nu_within_one_percent(ctx, tmp_path):
    z = np.load(os.path.join(GOLDEN, "golden_c1_longrun.npz"))
    nsteps = int(z["nsteps"])
    cfg = BouIn(nxm=64, nym=64, nzm=64, ylen=1.0, zlen=1.0, ray=1e6, pra=1.0, dt=5e-4, istr3=7,
                idtv=0, ntst=nsteps - 1, tout=float(z["tout"]), tmax=1e9, resid=1e-10)
    res = run(ctx, cfg, seed=0, out_dir=str(tmp_path))
    box = res.pop("box")
    assert res["code"] == 555 and res["ntime"] == nsteps, res["code"]
    assert np.array_equal(res["time"], z["time"])
    gpu = wnus_means(res["nu_vol"], res["nu_bot"], res["nu_top"])
    cpu = wnus_means(z["nu_vol"], z["nu_bot"], z["nu_top"])
    for k in gpu:
        assert abs(gpu[k] - cpu[k]) <= 0.01 * abs(cpu[k]), (k, gpu[k], cpu[k])
    # CheckDivergence at the output times, on the held box
    assert 0.0 < max(res["divmax"]) <= 1e-10
    assert max(res["cfl"]) > 1e-8
    # the log files carry the same series (nu_plate.out at its 6 digits)
    plate = np.loadtxt(tmp_path / "nu_plate.out")
    vol = np.loadtxt(tmp_path / "nu_vol.out")
    assert plate.shape == (len(z["time"]), 3) and vol.shape == (len(z["time"]), 2)
    assert np.allclose(plate[:, 1], res["nu_bot"], rtol=1e-5, atol=0)
    assert np.array_equal(vol[:, 1], res["nu_vol"])
    ctx.remove_box(box)
