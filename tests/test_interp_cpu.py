"""Restart onto a new grid (ReadFlowField.F90:63-150, interp.F90): the
oracle's vectorised restatement against a loop-for-loop one, the grids
against CreateGrid's, and the reference's conditions on a regrid."""
import numpy as np
import pytest

from afid_b200 import _lib, continua
from helpers import cfg_of
from oracle import afid_oracle as O


def interp_loops(old, nxo, nyo, nzo, istro3, stro3, flag, nxm, nym, nzm, istr3, str3, ylen, zlen):
    """interp.F90:11-227 statement by statement (Fortran indices kept)."""
    nx, ny, nz = nxm + 1, nym + 1, nzm + 1
    nyom, nzom = nyo - 1, nzo - 1
    tcold, tmold = O.gridnew(nzo, zlen, 0, 1.0)
    rcold, rmold = O.gridnew(nyo, ylen, 0, 1.0)
    zzold, zmold = O.gridnew(nxo, 1.0, istro3, stro3)
    tcnew, tmnew = O.gridnew(nz, zlen, 0, 1.0)
    rcnew, rmnew = O.gridnew(ny, ylen, 0, 1.0)
    zznew, zmnew = O.gridnew(nx, 1.0, istr3, str3)
    if flag == 1:
        xold, yold, zold, xnew, ynew, znew = tcold, rmold, zmold, tcnew, rmnew, zmnew
    elif flag == 2:
        xold, yold, zold, xnew, ynew, znew = tmold, rcold, zmold, tmnew, rcnew, zmnew
    elif flag == 3:
        xold, yold, zold, xnew, ynew, znew = tmold, rmold, zzold, tmnew, rmnew, zznew
    else:
        xold, yold, zold, xnew, ynew, znew = tmold, rmold, zmold, tmnew, rmnew, zmnew
    arrold = np.zeros((nxo + 2, nyom + 2, nzom + 2))   # edges and corners stay zero
    arrold[1:nxo + 1, 1:nyom + 1, 1:nzom + 1] = old
    for i in range(1, nzom + 1):
        for j in range(1, nyom + 1):
            arrold[0, j, i] = 2.0 * arrold[1, j, i] - arrold[2, j, i]
            arrold[nxo + 1, j, i] = 2.0 * arrold[nxo, j, i] - arrold[nxo - 1, j, i]
    for j in range(1, nyom + 1):
        for k in range(1, nxo + 1):
            arrold[k, j, 0] = 2.0 * arrold[k, j, 1] - arrold[k, j, 2]
            arrold[k, j, nzom + 1] = 2.0 * arrold[k, j, nzom] - arrold[k, j, nzom - 1]
    for i in range(1, nzom + 1):
        for k in range(1, nxo + 1):
            arrold[k, 0, i] = 2.0 * arrold[k, 1, i] - arrold[k, 2, i]
            arrold[k, nyom + 1, i] = 2.0 * arrold[k, nyom, i] - arrold[k, nyom - 1, i]
    arrnew = np.zeros((nx, nym, nzm))
    for i in range(1, nzm + 1):
        for j in range(1, nym + 1):
            for k in range(1, nx + 1):
                bix, biy, biz = xnew[i], ynew[j], znew[k]
                bifi, bici = nzo - 1, nzo
                for l in range(1, nzo + 1):
                    if xold[l] >= bix:
                        bifi, bici = l - 1, l
                        break
                bifj, bicj = nyo - 1, nyo
                for l in range(1, nyo + 1):
                    if yold[l] >= biy:
                        bifj, bicj = l - 1, l
                        break
                bifk, bick = nxo - 1, nxo
                for l in range(1, nxo + 1):
                    if zold[l] >= biz:
                        bifk, bick = l - 1, l
                        break
                bix1, bix2 = xold[bifi], xold[bici]
                biy1, biy2 = yold[bifj], yold[bicj]
                biz1, biz2 = zold[bifk], zold[bick]
                an = [arrold[bifk, bicj, bifi], arrold[bifk, bifj, bifi], arrold[bifk, bicj, bici],
                      arrold[bifk, bifj, bici], arrold[bick, bicj, bifi], arrold[bifk, bifj, bifi],
                      arrold[bifk, bicj, bici], arrold[bifk, bifj, bici]]
                dxdydz = 1.0 / ((bix2 - bix1) * (biy2 - biy1) * (biz2 - biz1))
                arrnew[k - 1, j - 1, i - 1] = (
                    an[0] * (bix2 - bix) * (biy - biy1) * (biz2 - biz)
                    + an[1] * (bix2 - bix) * (biy2 - biy) * (biz2 - biz)
                    + an[2] * (bix - bix1) * (biy - biy1) * (biz2 - biz)
                    + an[3] * (bix - bix1) * (biy2 - biy) * (biz2 - biz)
                    + an[4] * (bix2 - bix) * (biy - biy1) * (biz - biz1)
                    + an[5] * (bix2 - bix) * (biy2 - biy) * (biz - biz1)
                    + an[6] * (bix - bix1) * (biy - biy1) * (biz - biz1)
                    + an[7] * (bix - bix1) * (biy2 - biy) * (biz - biz1)) * dxdydz
    return arrnew


# (nxo, nyo, nzo, istro3, stro3) -> (nxm, nym, nzm, istr3, str3): refinement,
# coarsening and a change of wall-normal stretching
CASES = [
    ((9, 9, 7, 0, 0.0), (12, 12, 10, 6, 2.0)),
    ((13, 13, 9, 6, 3.0), (8, 10, 6, 6, 3.0)),
    ((11, 7, 9, 6, 1.0), (16, 12, 12, 0, 0.0)),
]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("flag", [1, 2, 3, 4])
def test_vectorised_regrid_matches_the_loops(case, flag):
    (nxo, nyo, nzo, isto, sto), (nxm, nym, nzm, istn, stn) = case
    old = np.random.default_rng(flag).standard_normal((nxo, nyo - 1, nzo - 1))
    a = O.interp_field(old, nxo, nyo, nzo, isto, sto, flag, nxm, nym, nzm, istn, stn, 1.5, 2.0)
    b = interp_loops(old, nxo, nyo, nzo, isto, sto, flag, nxm, nym, nzm, istn, stn, 1.5, 2.0)
    assert a.shape == (nxm + 1, nym, nzm)
    assert np.array_equal(a, b)


def test_linear_fields_are_reproduced_away_from_the_stencil_quirks():
    # a field linear in y and z only (constant in x) is reproduced exactly
    # wherever the stencil's corners are interior: the reference's
    # lower-x corners do not matter for a field constant in x
    nxo, nyo, nzo = 9, 9, 9
    rc, rm = O.gridnew(nyo, 1.0, 0, 1.0)
    tc, tm = O.gridnew(nzo, 1.0, 0, 1.0)
    old = (3.0 * rm[1:nyo][None, :, None] - 2.0 * tm[1:nzo][None, None, :]) * np.ones((nxo, 1, 1))
    new = O.interp_field(old, nxo, nyo, nzo, 0, 0.0, 4, 12, 12, 12, 0, 0.0, 1.0, 1.0)
    rcn, rmn = O.gridnew(13, 1.0, 0, 1.0)
    tcn, tmn = O.gridnew(13, 1.0, 0, 1.0)
    want = 3.0 * rmn[1:13][None, :, None] - 2.0 * tmn[1:13][None, None, :]
    inner = np.s_[1:-1, 1:-1, 1:-1]
    assert np.allclose(new[inner], np.broadcast_to(want, new.shape)[inner], rtol=0, atol=1e-12)


@pytest.mark.parametrize("istr,st", [(0, 0.0), (6, 2.0), (6, 5.0)])
@pytest.mark.parametrize("n", [5, 17, 64])
def test_library_grid_is_gridnew(built_lib, istr, st, n):
    """The library builds interp's grids with afid_make_grid: for istr 0 and
    6 its nodes are gridnew's (interp.F90:229-296)."""
    xc = np.zeros(n)
    assert _lib.lib().afid_make_grid(n - 1, istr, st, 1.0, _lib.dptr(xc)) == 0
    rc, rm = O.gridnew(n, 1.0, istr, st)
    assert np.array_equal(xc, rc[1:n + 1])


def test_regrid_conditions():
    old = np.zeros((9, 8, 6))
    with pytest.raises(ValueError):      # more than twice the old points (ReadFlowField.F90:88-99)
        O.interp_field(old, 9, 9, 7, 0, 0.0, 4, 12, 18, 10, 0, 0.0, 1.0, 1.0)
    for bad in (4, 7):                   # gridnew defines istr 0 and 6 only
        with pytest.raises(ValueError):
            O.interp_field(old, 9, 9, 7, bad, 1.0, 4, 12, 12, 10, 0, 0.0, 1.0, 1.0)
        with pytest.raises(ValueError):
            O.interp_field(old, 9, 9, 7, 0, 0.0, 4, 12, 12, 10, bad, 1.0, 1.0, 1.0)


def test_same_grid_rule():
    cfg = cfg_of(12, 8, 6, istr3=6, str3=2.0)
    m = {"nx": 13, "ny": 9, "nz": 7, "istr3": 6, "str3": 2.0 + 5e-9}
    assert continua.same_grid(m, cfg)
    assert not continua.same_grid(dict(m, str3=2.0 + 2e-8), cfg)
    assert not continua.same_grid(dict(m, nz=9), cfg)
    assert not continua.same_grid(dict(m, istr3=0), cfg)


def test_interp_entry_point_is_exported(built_lib):
    assert "afid_box_interp_field" in _lib.EXPORTS
    assert hasattr(_lib.lib(), "afid_box_interp_field")
