"""The CPU oracle against analytic known answers of the reference's own
formulas and against its committed golden vectors (no GPU)."""
import math
import os

import numpy as np
import pytest
from scipy.linalg import lapack

from helpers import cfg_of, oracle_state, FIELDS
from oracle import afid_oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_rk3_coefficients_sum_to_one():
    # InitTimeMarchScheme.F90:16-23, 46-48
    gam, rom, alm = O.init_time_march_scheme(3)
    assert math.isclose(sum(alm), 1.0, rel_tol=0, abs_tol=1e-15)
    assert gam == [8 / 15, 5 / 12, 3 / 4] and rom == [0.0, -17 / 60, -5 / 12]
    gam, rom, alm = O.init_time_march_scheme(1)
    assert alm[0] == 1.0


@pytest.mark.parametrize("istr3,str3", [(0, 0.0), (4, 3.0), (6, 12.0), (6, 0.0), (7, 0.0)])
def test_grid_options(istr3, str3):
    xc = O.make_xc(48, istr3, str3)
    assert xc[0] == 0.0 and xc[-1] == 1.0
    assert np.all(np.diff(xc) > 0)
    if istr3 == 7:
        k = np.arange(49)
        assert np.allclose(xc, 0.5 * (1 - np.cos(np.pi * k / 48)), atol=1e-15)


def test_metric_identities():
    # acphk = -(amphk + apphk) with kmc(1) = kpc(nxm) = 0 (InitPressureSolver.F90:50-59)
    p = O.Params(nxm=32, nym=16, nzm=16)
    g = O.create_grid(p)
    assert g.amphk[0] == 0.0 and g.apphk[-1] == 0.0
    assert np.array_equal(g.acphk, -(g.amphk + g.apphk))
    # the staggered no-slip wall coefficients (CreateGrid.F90:222-242)
    assert g.am3sk[0] == 0.0 and g.ap3sk[p.nxm - 1] == 0.0


def test_conduction_state_is_a_fixed_point():
    """KAT-1: u = 0 and T linear in x are a discrete steady state; plate Nu = 1."""
    cfg = cfg_of(20, 12, 10, ray=1e5, zlen=0.8)
    s = oracle_state(cfg, seed=None)
    t0 = s.temp.copy()
    recs = O.run(s, 2, cfg.dt)
    assert np.abs(s.temp - t0).max() == 0.0
    for f in ("vx", "vy", "vz"):
        assert np.abs(getattr(s, f)).max() < 1e-18   # roundoff of the buoyancy/pressure balance
    for r in recs:
        assert r["nu_bot"] == pytest.approx(1.0, abs=1e-13)
        assert r["nu_top"] == pytest.approx(1.0, abs=1e-13)


def test_projection_is_divergence_free():
    """KAT-2: after CorrectVelocity the discrete divergence is at roundoff."""
    cfg = cfg_of(24, 16, 12, ray=1e6, zlen=0.75)
    s = oracle_state(cfg, seed=5)
    O.run(s, 3, cfg.dt)
    scale = max(np.abs(s.vx).max(), 1e-30) * s.g.udx3m.max()
    assert O.check_divergence(s) <= 1e-12 * scale + 1e-20


@pytest.mark.parametrize("m,n", [(0, 0), (1, 0), (0, 2), (3, 1), (8, 6)])
def test_poisson_manufactured_solution(m, n):
    """KAT-3: the solver inverts the discrete Laplacian it is built from
    (amphk/acphk/apphk in x, 3-point stencils in y and z)."""
    p = O.Params(nxm=24, nym=16, nzm=12, ylen=1.0, zlen=0.75)
    s = O.init_state(p, seed=None, ic="conduction")
    g = s.g
    xm = g.xm[:p.nxm]
    y = (np.arange(p.nym) + 0.5) / p.nym * p.ylen
    z = (np.arange(p.nzm) + 0.5) / p.nzm * p.zlen
    f = np.cos(np.pi * xm) + xm ** 3
    phi = (f[:, None, None] * np.cos(2 * np.pi * m * y / p.ylen)[None, :, None]
           * np.cos(2 * np.pi * n * z / p.zlen)[None, None, :])
    lap = ((np.roll(phi, -1, 2) - 2 * phi + np.roll(phi, 1, 2)) * g.dzq
           + (np.roll(phi, -1, 1) - 2 * phi + np.roll(phi, 1, 1)) * g.dyq
           + phi[g.kpv] * g.apphk[:, None, None] + phi * g.acphk[:, None, None]
           + phi[g.kmv] * g.amphk[:, None, None])
    s.dph[:] = lap
    O.solve_pressure_correction(s)
    got = s.dph - s.dph.mean()
    want = phi - phi.mean()
    assert np.abs(got - want).max() <= 1e-10 * max(np.abs(want).max(), 1.0)


def test_vectorised_poisson_matches_lapack_per_mode():
    """KAT-5 (complex tridiagonal): the vectorised Thomas sweep of the oracle
    agrees with LAPACK zgttrf/zgttrs mode by mode."""
    cfg = cfg_of(24, 16, 12, zlen=0.75)
    s1 = oracle_state(cfg, seed=2)
    rng = np.random.default_rng(0)
    s1.dph[:] = rng.standard_normal(s1.dph.shape)
    s2 = s1.copy()
    O.solve_pressure_correction(s1, vectorised=False)
    O.solve_pressure_correction(s2, vectorised=True)
    a = s1.dph - s1.dph.mean()
    b = s2.dph - s2.dph.mean()
    assert np.linalg.norm(a - b) <= 1e-12 * np.linalg.norm(a)


def test_real_tridiagonal_matches_dense_solve():
    """KAT-5 (real): the SolveImpEqnUpdate_YZ matrix solved through
    dgttrf/dgttrs equals a dense solve of the same matrix."""
    cfg = cfg_of(24, 16, 12)
    s = oracle_state(cfg, seed=1)
    g = s.g
    betadx = 3e-3
    n = cfg.nxm
    am = np.array([-g.am3sk[k] * betadx / (1 - g.ac3sk[k] * betadx) for k in range(n)])
    ap = np.array([-g.ap3sk[k] * betadx / (1 - g.ac3sk[k] * betadx) for k in range(n)])
    A = np.eye(n) + np.diag(am[1:], -1) + np.diag(ap[:-1], 1)
    b = np.random.default_rng(1).standard_normal((n, 3))
    dl, d, du, du2, ipiv, info = lapack.dgttrf(am[1:], np.ones(n), ap[:-1])
    x, info = lapack.dgttrs(dl, d, du, du2, ipiv, b)
    assert np.allclose(x, np.linalg.solve(A, b), rtol=1e-13, atol=1e-14)


def test_zero_mode_pin():
    """The (0,0) Poisson mode solves rows 1..nxm-1 with x(nxm) = 0."""
    g = O.create_grid(O.Params(nxm=16, nym=8, nzm=8))
    s_ = 1.0 / g.acphk
    dl = (g.amphk * s_)[1:].astype(complex)
    du = (g.apphk * s_)[:-1].astype(complex)
    d = np.ones(16, complex)
    b = np.random.default_rng(3).standard_normal(16) + 0j
    x = O._tridiag_pinned_zero_mode(dl, d, du, b)
    assert x[-1] == 0
    A = np.eye(16) + np.diag(dl, -1) + np.diag(du, 1)
    assert np.allclose((A @ x)[:-1], b[:-1], rtol=1e-12, atol=1e-12)


def test_oracle_reproduces_golden_small():
    z = np.load(os.path.join(GOLDEN, "golden_small.npz"))
    cfg = cfg_of(24, 16, 12, ray=1e5, pra=0.7, zlen=0.75, dt=5e-4)
    s = oracle_state(cfg, seed=11)
    recs = O.run(s, 5, cfg.dt)
    for f in FIELDS:
        a, b = getattr(s, f), z[f"step5_{f}"]
        if f == "pr":
            a, b = a[:-1] - a[:-1].mean(), b[:-1] - b[:-1].mean()
        assert np.linalg.norm(a - b) <= 1e-13 * max(np.linalg.norm(b), 1e-30), f
    assert np.allclose([r["nu_bot"] for r in recs], z["nu_bot"], rtol=0, atol=1e-13)


def test_rhs_wall_row_is_carried_state():
    """The reference's shared rhs array keeps rhs(1,:,:) = dvz(1) from the
    vz solve; the temperature solve and the next vx solve read it.  The
    oracle must keep it (the result differs if it is zeroed)."""
    cfg = cfg_of(24, 16, 12, ray=1e5, zlen=0.75)
    s1 = oracle_state(cfg, seed=4)
    O.run(s1, 2, cfg.dt)
    s2 = s1.copy()
    O.time_marcher(s1, cfg.dt)
    # variant with the wall row cleared before each implicit solve
    gam, rom, alm = O.init_time_march_scheme(3)
    beta = cfg.dt / s2.p.ren * 0.5
    for ns in range(3):
        al, ga, ro = alm[ns], gam[ns], rom[ns]
        for fn in (O.explicit_terms_vx, O.explicit_terms_vy, O.explicit_terms_vz, O.explicit_terms_temp):
            fn(s2)
        for fn in (O.implicit_and_update_vx, O.implicit_and_update_vy, O.implicit_and_update_vz,
                   O.implicit_and_update_temp):
            s2.rhs[0] = 0.0
            fn(s2, al, ga, ro, cfg.dt, beta)
        O.calc_local_divergence(s2, al, cfg.dt)
        O.solve_pressure_correction(s2)
        O.correct_velocity(s2, al, cfg.dt)
        O.correct_pressure(s2, al, beta)
    assert np.abs(s1.rhs[0]).max() > 0
    assert np.abs(s1.temp - s2.temp).max() > 0
