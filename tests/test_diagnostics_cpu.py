"""Output-time diagnostics of the oracle (GlobalQuantities, CalcStats,
CalcDissipationNu, slab locations) against known answers, and the library's
host-side slab location rule against the oracle (no GPU)."""
import numpy as np
import pytest

from helpers import cfg_of, oracle_state
from oracle import afid_oracle as O


def test_conduction_known_answers():
    """Conduction (u = 0, T = 1 - x): volume Nu = 1, dissipation Nu_mu = 1
    and Nu_th = 1 (|grad T| = 1 everywhere, CalcDissipationNu.F90:95-111),
    rms velocities 0, mean temperature profile 1 - xc."""
    cfg = cfg_of(24, 12, 10, ray=1e5, zlen=0.8)
    s = oracle_state(cfg, seed=None)
    gq = O.global_quantities(s)
    assert gq["nu_vol"] == 1.0
    assert gq["vx_rms"] == 0.0 and gq["vel_rms"] == 0.0
    assert gq["tempmax"] == 1.0 and gq["tempmin"] == pytest.approx(1.0 - s.g.xc[cfg.nxm - 1], abs=1e-15)
    d = O.calc_dissipation_nu(s)
    assert d["nu_mu"] == 1.0
    assert d["nu_th"] == pytest.approx(1.0, rel=1e-13)
    acc = O.calc_stats(s)
    assert acc["nstatsamples"] == 1
    assert np.allclose(acc["temp_me"], 1.0 - s.g.xc[:cfg.nxm], rtol=0, atol=1e-14)
    assert np.all(acc["vx_rms"] == 0.0)
    acc = O.calc_stats(s, acc)
    assert acc["nstatsamples"] == 2
    assert np.allclose(acc["temp_me"], 2 * (1.0 - s.g.xc[:cfg.nxm]), rtol=0, atol=1e-14)


def test_dissipation_balance_sign():
    """On a seeded noisy state the dissipation rates are positive and the
    per-plane profiles sum to the volume numbers' raw sums."""
    cfg = cfg_of(24, 16, 12, ray=1e6, zlen=0.75)
    s = oracle_state(cfg, seed=3)
    O.run(s, 2, cfg.dt)
    d = O.calc_dissipation_nu(s)
    assert d["nu_mu"] > 1.0 and d["nu_th"] > 0.0
    assert np.all(d["disste"] >= 0) and np.all(d["dissth"] > 0)


def test_slab_locations_match_oracle():
    from afid_b200.solver import make_grid, slab_locations
    xc = make_grid(64, 7)
    p = O.Params(nxm=64, nym=8, nzm=8)
    g = O.create_grid(p, xc)
    xslab = [0.01, 0.05, 0.1, 0.25, 0.5, 0.75, 0.9, 0.99]
    assert slab_locations(xc, xslab) == O.slab_locations(g, 64, xslab)
    assert slab_locations(xc, xslab)[0] == 2
