"""Host logic without a GPU: bou.in format, FFT-size rule, C-ABI exports."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from afid_b200 import BouIn, largest_factor, read_bou_in, write_bou_in
from afid_b200 import _lib
from oracle import afid_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SAMPLE_BOU = """ NXM  NYM  NZM   NSST(>1=RK,else AB) NREAD
 48 96 72       3                   0
 NTST   WALLTIMEMAX    TOUT      TMAX     IRESET
 1000     3600          1e-2      20.0      0
 ALX3D      ISTR3   STR3
 1.0000       6     12.0
 YLEN ZLEN
 2.0   1.5
   RA   PRA      DT      RESID    CFLMAX
 1e+8  0.7   1d-4   1.e-2    1.2
 STATON  BALANCEON  TSTA  STAREAD
 0        0            0    0
 inslws   inslwn
  1          0
 IDTV(0=dt fixed,1=var.)   DTMIN(for dt var.)  DTMAX(for dt var.)     VLIM
   1                       1e-8                0.01                    1e3
 SLABDUMP(STST3)
   0
"""


def test_read_bou_in(tmp_path):
    p = tmp_path / "bou.in"
    p.write_text(SAMPLE_BOU)
    c = read_bou_in(str(p))
    assert (c.nxm, c.nym, c.nzm, c.nsst) == (48, 96, 72, 3)
    assert (c.istr3, c.str3, c.ylen, c.zlen) == (6, 12.0, 2.0, 1.5)
    assert (c.ray, c.pra, c.dt, c.cflmax) == (1e8, 0.7, 1e-4, 1.2)
    assert (c.inslws, c.inslwn, c.idtv, c.dtmin, c.dtmax, c.vlim) == (1, 0, 1, 1e-8, 0.01, 1e3)
    assert c.ren == pytest.approx(np.sqrt(1e8 / 0.7))
    c.validate()


def test_bou_in_roundtrip(tmp_path):
    c = BouIn(nxm=32, nym=48, nzm=40, ray=3e5, istr3=4, str3=2.5, idtv=1)
    p = tmp_path / "bou.in"
    write_bou_in(c, str(p))
    d = read_bou_in(str(p))
    for f in ("nxm", "nym", "nzm", "ray", "istr3", "str3", "idtv", "dt"):
        assert getattr(c, f) == getattr(d, f)


@pytest.mark.parametrize("n,out", [(64, 3), (768, 5), (1280, 7), (96, 5), (7, 9), (22, 13), (45, 7)])
def test_largest_factor_follows_factorize(n, out):
    # Factorize.F90:8-34 returns the divisor after the last one removed
    assert largest_factor(n) == out


def test_validate_rejects_inefficient_fft():
    with pytest.raises(ValueError):
        BouIn(nym=44).validate()     # 11 -> code 444
    with pytest.raises(ValueError):
        BouIn(nym=14).validate()     # factor 7 gives 9 > 7 in the reference rule


def test_choose_dt_rules():
    # main.F90:171-189
    assert O.choose_dt(0, 0.5, 1e-3, 1, 1.2, 1e-8, 1e-2) == (1e-8, 0.5, 0)
    dt, cfl, err = O.choose_dt(5, 100.0, 1e-3, 1, 1.2, 1e-8, 1e-2)
    assert dt == pytest.approx(0.012 / 1.0 * 1) or dt == 1e-2
    assert O.choose_dt(5, 1e-9, 1e-3, 1, 1.2, 1e-8, 1e-2)[0] == 1e-2
    assert O.choose_dt(5, 1e12, 1e-3, 1, 1.2, 1e-8, 1e-2)[2] == 166
    assert O.choose_dt(5, 2000.0, 1e-3, 0, 1.2, 1e-8, 1e-2)[2] == 165


def _declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "afid_gpu.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(afid_\w+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol(built_lib):
    L = _lib.lib()
    declared = _declared_symbols()
    assert len(declared) >= 30
    for name in declared:
        assert hasattr(L, name), name
    assert set(declared) == set(_lib.EXPORTS)


def test_grid_and_sizes_need_no_gpu(built_lib):
    L = _lib.lib()
    xc = np.zeros(65)
    assert L.afid_make_grid(64, 7, 0.0, 1.0, _lib.dptr(xc)) == 0
    assert np.array_equal(xc, O.make_xc(64, 7, 0.0))
    p = _lib.BoxParams(nxm=384, nym=768, nzm=768, nsst=3, alx3=1.0, ylen=2.0, zlen=2.0,
                       ray=1e9, pra=1.0, inslws=1, inslwn=1, tempbp=1.0, temptp=0.0, dt=1e-4)
    nbytes = L.afid_box_device_bytes(C.byref(p))
    field = 385 * 768 * 768 * 8
    assert 13 * field < nbytes < 14 * field


def test_bad_grid_arguments_rejected(built_lib):
    L = _lib.lib()
    assert L.afid_make_grid(1, 7, 0.0, 1.0, _lib.dptr(np.zeros(2))) == -1
    assert b"nxm" in L.afid_last_error()
