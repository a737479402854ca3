"""Routine-level entry points against the oracle, routine by routine.

The stencil routines (explicit terms, implicit updates with their x-solves,
divergence, pressure correction) are compared for bitwise equality: the
library is built without FMA contraction and follows the reference's
operation order, so each value is the same IEEE result.  The pressure solve
goes through a different FFT than NumPy's and is compared at 1e-12."""
import numpy as np
import pytest

from helpers import cfg_of, oracle_state, rel_l2, FIELDS
from oracle import afid_oracle as O

pytestmark = pytest.mark.gpu

CASES = [
    # nxm, nym, nzm, kw
    (24, 16, 12, dict(ray=1e5, pra=0.7, zlen=0.75)),                  # radix 4, 2, 3
    (20, 20, 40, dict(ray=3e6, pra=4.38, ylen=1.2, zlen=2.0)),        # radix 5
    (18, 12, 8, dict(ray=1e6, inslws=0, inslwn=1, istr3=6, str3=4.0)),  # stress-free wall, clipped grid
    (16, 48, 24, dict(ray=2e5, istr3=4, str3=2.0, inslwn=0)),
]


def _prepared(ctx, nxm, nym, nzm, kw, seed=3, nsteps=2):
    cfg = cfg_of(nxm, nym, nzm, dt=1e-3, **kw)
    s = oracle_state(cfg, seed=seed)
    O.run(s, nsteps, cfg.dt)          # non-trivial velocity, pressure and history
    box = ctx.add_box(cfg, s.g.xc)
    for f in FIELDS + ("rux", "ruy", "ruz", "rutemp"):
        box.upload(f, getattr(s, f))
    box.upload("wall", s.rhs[0])
    return cfg, s, box


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("ns", [0, 1, 2])
def test_routines_match_oracle(ctx, case, ns):
    nxm, nym, nzm, kw = CASES[case]
    cfg, s, box = _prepared(ctx, nxm, nym, nzm, kw)
    gam, rom, alm = O.init_time_march_scheme(3)
    dt = cfg.dt
    beta = dt / s.p.ren * 0.5
    al, ga, ro = alm[ns], gam[ns], rom[ns]
    box.time_marcher_begin_substep(ns)
    exact = [
        ("explicit_terms_vx", lambda: O.explicit_terms_vx(s), "qcap", slice(1, nxm)),
        ("explicit_terms_vy", lambda: O.explicit_terms_vy(s), "dph", slice(0, nxm)),
        ("explicit_terms_vz", lambda: O.explicit_terms_vz(s), "dq", slice(0, nxm)),
        ("explicit_terms_temp", lambda: O.explicit_terms_temp(s), "hro", slice(1, nxm)),
        ("implicit_and_update_vx", lambda: O.implicit_and_update_vx(s, al, ga, ro, dt, beta), "vx", slice(None)),
        ("implicit_and_update_vy", lambda: O.implicit_and_update_vy(s, al, ga, ro, dt, beta), "vy", slice(0, nxm)),
        ("implicit_and_update_vz", lambda: O.implicit_and_update_vz(s, al, ga, ro, dt, beta), "vz", slice(0, nxm)),
        ("implicit_and_update_temp", lambda: O.implicit_and_update_temp(s, al, ga, ro, dt, beta), "temp", slice(None)),
        ("calc_local_divergence", lambda: O.calc_local_divergence(s, al, dt), "dph", slice(None)),
    ]
    for name, ofn, field, rows in exact:
        getattr(box, name)()
        ofn()
        d = box.download(field)[rows]
        o = getattr(s, field)[rows]
        assert np.array_equal(d, o), f"{name}: max diff {np.abs(d - o).max():.3e}"
        if name.startswith("implicit"):
            assert np.array_equal(box.download("wall"), s.rhs[0]), f"{name}: rhs wall row"
    box.solve_pressure_correction()
    O.solve_pressure_correction(s)
    d = box.download("dph")
    assert rel_l2(d, s.dph, remove_mean=True) <= 1e-12
    # continue from the oracle's dph so the corrections are compared exactly
    box.upload("dph", s.dph)
    box.correct_velocity()
    O.correct_velocity(s, al, dt)
    box.correct_pressure()
    O.correct_pressure(s, al, beta)
    for f in ("vx", "vy", "vz"):
        assert np.array_equal(box.download(f)[:nxm], getattr(s, f)[:nxm]), f
    assert np.array_equal(box.download("pr")[:nxm], s.pr[:nxm])
    ctx.remove_box(box)


def test_reductions_match_oracle(ctx):
    cfg, s, box = _prepared(ctx, 24, 16, 12, dict(ray=1e6, zlen=0.75), nsteps=3)
    assert box.calc_max_cfl() == pytest.approx(O.calc_max_cfl(s), rel=1e-15)
    assert box.check_divergence() == pytest.approx(O.check_divergence(s), rel=1e-12, abs=1e-30)
    nb, nt = box.calc_plate_nu()
    ob, ot = O.calc_plate_nu(s)
    assert abs(nb - ob) <= 1e-13 and abs(nt - ot) <= 1e-13
    ctx.remove_box(box)


def test_routine_step_matches_fused_step(ctx):
    """TimeMarcher through the routine entry points and through the fused
    kernels give the same step (the fused path adds the temperature wall-row
    contribution after its forward sweep: identical up to rounding)."""
    cfg = cfg_of(24, 16, 12, ray=1e6, zlen=0.75, dt=5e-4)
    s = oracle_state(cfg, seed=9)
    O.run(s, 2, cfg.dt)
    a = ctx.add_box(cfg, s.g.xc)
    b = ctx.add_box(cfg, s.g.xc)
    for box in (a, b):
        for f in FIELDS + ("rux", "ruy", "ruz", "rutemp"):
            box.upload(f, getattr(s, f))
        box.upload("wall", s.rhs[0])
    a.time_marcher_routines()
    for ns in range(3):
        ctx.substep([b], ns)
    for f in FIELDS:
        da, db = a.download(f), b.download(f)
        assert rel_l2(db[:-1], da[:-1], remove_mean=(f == "pr")) <= 1e-13, f
    ctx.remove_box(a)
    ctx.remove_box(b)


@pytest.mark.parametrize("nxm", [24, 40, 100, 200, 300, 384, 500, 530])
def test_pressure_solve_x_sizes(ctx, nxm):
    """SolvePressureCorrection on white-noise dph over a range of x sizes,
    each mode pair (kz, nzm - kz) solved by one thread, against the oracle
    at the parity tolerance 1e-11: on the tallest Chebyshev grids the wall
    cells are ~1e-5 of the mid cells, and white noise in x excites the
    ill-conditioned end of the solve (the physical fields of the other tests
    agree to 1e-12)."""
    cfg = cfg_of(nxm, 16, 12, ray=1e6, ylen=1.5, zlen=0.75)
    s = oracle_state(cfg, seed=None)
    s.dph[...] = np.random.default_rng(nxm).standard_normal(s.dph.shape)
    box = ctx.add_box(cfg, s.g.xc)
    box.upload("dph", s.dph)
    box.solve_pressure_correction()
    O.solve_pressure_correction(s)
    assert rel_l2(box.download("dph"), s.dph, remove_mean=True) <= 1e-11
    ctx.remove_box(box)


@pytest.mark.parametrize("nym,nzm", [(8, 12), (12, 8), (16, 24), (8, 8), (24, 16)])
def test_pressure_solve_short_lines(ctx, nym, nzm):
    """SolvePressureCorrection on the shortest transform lines: 8 and
    12 points are one warp lane per line in the z transform (32 lines per
    warp) and leave the y transform to the tile kernel (its staged rows need
    at least two lanes per line); 16 and 24 points are two lanes per line."""
    cfg = cfg_of(20, nym, nzm, ray=1e6, ylen=1.3, zlen=0.9)
    s = oracle_state(cfg, seed=None)
    s.dph[...] = np.random.default_rng(nym * 100 + nzm).standard_normal(s.dph.shape)
    box = ctx.add_box(cfg, s.g.xc)
    box.upload("dph", s.dph)
    box.solve_pressure_correction()
    O.solve_pressure_correction(s)
    assert rel_l2(box.download("dph"), s.dph, remove_mean=True) <= 1e-12
    ctx.remove_box(box)
