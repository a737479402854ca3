"""bou.in reader/writer with the reference's fixed layout (ReadInputFile.F90:16-37).

bou.in alternates a header line (read as ``a4`` and ignored) with a line of
list-directed values, nine times:

    NXM NYM NZM NSST NREAD | NTST WALLTIMEMAX TOUT TMAX IRESET |
    ALX3D ISTR3 STR3 | YLEN ZLEN | RA PRA DT RESID CFLMAX |
    STATON BALANCEON TSTA STAREAD | INSLWS INSLWN |
    IDTV DTMIN DTMAX VLIM | SLABDUMP

``istr3 = 7`` (pure Chebyshev-Gauss-Lobatto nodes) is accepted in addition
to the reference's 0, 4 and 6.
"""
from __future__ import annotations

import dataclasses
import math

_LAYOUT = [
    ("NXM  NYM  NZM  NSST NREAD", [("nxm", int), ("nym", int), ("nzm", int), ("nsst", int), ("nread", int)]),
    ("NTST WALLTIMEMAX TOUT TMAX IRESET", [("ntst", int), ("walltimemax", float), ("tout", float),
                                           ("tmax", float), ("ireset", int)]),
    ("ALX3D ISTR3 STR3", [("alx3", float), ("istr3", int), ("str3", float)]),
    ("YLEN ZLEN", [("ylen", float), ("zlen", float)]),
    ("RA PRA DT RESID CFLMAX", [("ray", float), ("pra", float), ("dt", float), ("resid", float),
                                ("cflmax", float)]),
    ("STATON BALANCEON TSTA STAREAD", [("staton", int), ("balanceon", int), ("tsta", float),
                                       ("staread", int)]),
    ("INSLWS INSLWN", [("inslws", int), ("inslwn", int)]),
    ("IDTV DTMIN DTMAX VLIM", [("idtv", int), ("dtmin", float), ("dtmax", float), ("vlim", float)]),
    ("SLABDUMP", [("slabdump", int)]),
]


@dataclasses.dataclass
class BouIn:
    nxm: int = 64
    nym: int = 64
    nzm: int = 64
    nsst: int = 3
    nread: int = 0
    ntst: int = 200
    walltimemax: float = 83000.0
    tout: float = 1e-2
    tmax: float = 50.0
    ireset: int = 0
    alx3: float = 1.0
    istr3: int = 7
    str3: float = 0.0
    ylen: float = 1.0
    zlen: float = 1.0
    ray: float = 1e6
    pra: float = 1.0
    dt: float = 5e-4
    resid: float = 1e-2
    cflmax: float = 1.2
    staton: int = 0
    balanceon: int = 0
    tsta: float = 0.0
    staread: int = 0
    inslws: int = 1
    inslwn: int = 1
    idtv: int = 0
    dtmin: float = 1e-8
    dtmax: float = 1e-2
    vlim: float = 1e3
    slabdump: int = 0
    tempbp: float = 1.0
    temptp: float = 0.0

    # derived quantities of ReadInputFile.F90:38-48
    @property
    def nx(self) -> int:
        return self.nxm + 1

    @property
    def ren(self) -> float:
        return math.sqrt(self.ray / self.pra)

    @property
    def pec(self) -> float:
        return math.sqrt(self.pra * self.ray)

    def validate(self) -> None:
        """Checks the reference makes at start-up (main.F90:156-165,
        CreateGrid.F90:66-119) plus the even-nym rule of the real y-FFT."""
        if self.istr3 not in (0, 4, 6, 7):
            raise ValueError(f"istr3={self.istr3}: supported grids are 0, 4, 6, 7")
        for name in ("nym", "nzm"):
            n = getattr(self, name)
            if largest_factor(n) > 7:
                raise ValueError(f"{name}={n}: FFT size not efficient (largest factor > 7, code 444)")
        if self.nym % 2:
            raise ValueError("nym must be even")
        if self.nsst not in (1, 3):
            raise ValueError("nsst must be 3 (RK3) or 1 (AB2)")


def largest_factor(n: int) -> int:
    """Factorize.F90:8-34: strips 2s, then odd divisors, returns the last
    divisor tried (the largest prime factor when n > 1)."""
    m = n
    while m % 2 == 0 and m != 1:
        m //= 2
    d = 3
    while d <= m:
        while m % d == 0 and m != 1:
            m //= d
        d += 2
    return d


def _convert(tok: str, typ):
    t = tok.strip().replace("d", "e").replace("D", "e")
    return typ(float(t)) if typ is int else typ(t)


def read_bou_in(path: str) -> BouIn:
    with open(path) as fh:
        lines = [ln for ln in fh.read().splitlines()]
    cfg = BouIn()
    pos = 0
    for _, fields in _LAYOUT:
        pos += 1                       # header line (format a4, ignored)
        while pos < len(lines) and not lines[pos].strip():
            pos += 1
        if pos >= len(lines):
            raise ValueError(f"{path}: truncated bou.in")
        toks = lines[pos].split()
        if len(toks) < len(fields):
            raise ValueError(f"{path}:{pos + 1}: expected {len(fields)} values, got {len(toks)}")
        for (name, typ), tok in zip(fields, toks):
            setattr(cfg, name, _convert(tok, typ))
        pos += 1
    return cfg


def write_bou_in(cfg: BouIn, path: str) -> None:
    out = []
    for header, fields in _LAYOUT:
        out.append(" " + header)
        out.append(" " + "  ".join(repr(getattr(cfg, n)) if t is float else str(getattr(cfg, n))
                                   for n, t in fields))
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")
