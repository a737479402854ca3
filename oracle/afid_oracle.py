"""CPU oracle: a NumPy/SciPy restatement of AFiD's RK3 time-step hot path.

TEST INFRASTRUCTURE ONLY.  This module is the checker for the CUDA path.
Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it.  The product path (``afid_b200``) never routes
through it.

Parity status: the Fortran reference cannot be compiled in this image (no
Fortran compiler, MPI, FFTW3 or HDF5), and the reference ships no tests or
golden vectors.  The restatement is therefore pinned by analytic
known-answer tests derived from the reference's own formulas (conduction
fixed point, manufactured Poisson solution, RK3 coefficient sums,
projection to zero divergence) and by using the same LAPACK routines the
reference calls (dgttrf/dgttrs/zgttrf/zgttrs, through SciPy).  Against
executed reference output, parity is unpinned.

Array convention: every 3-D field is indexed ``a[k, j, i]`` (x = wall-normal,
y, z) with shape ``(nx, nym, nzm)``, 0-based, where the reference uses
``a(k, j, i)`` 1-based with a one-cell periodic halo in y and z.  Periodic
halos are ``np.roll`` wraps.  Floating-point operation order follows the
Fortran source expression by expression (x86-64 -O2 evaluates left to
right, without fused multiply-add).

Differences from the reference, each deliberate:
* The (ky, kz) = (0, 0) pressure mode is an exactly singular Neumann system.
  The reference hands it to zgttrf unpinned (it aborts when the pivot is an
  exact zero, SolvePressureCorrection.F90:130-134).  Here that mode drops
  its last equation and sets its last unknown to zero, which fixes the
  arbitrary additive constant of the pressure correction.
* ``istr3 = 7`` adds the pure Chebyshev-Gauss-Lobatto grid
  x_k = 0.5 (1 - cos(pi (k-1) / nxm)); options 0, 4 and 6 follow
  CreateGrid.F90:66-119.
* FFTW is replaced by NumPy's pocketfft (the same discrete transforms).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np
from scipy.linalg import lapack

__all__ = [
    "Params", "Grid", "State", "create_grid", "init_time_march_scheme",
    "init_state", "explicit_terms_vx", "explicit_terms_vy", "explicit_terms_vz",
    "explicit_terms_temp", "implicit_and_update_vx", "implicit_and_update_vy",
    "implicit_and_update_vz", "implicit_and_update_temp",
    "calc_local_divergence", "solve_pressure_correction", "correct_velocity",
    "correct_pressure", "time_marcher", "calc_max_cfl", "check_divergence",
    "calc_plate_nu", "global_quantities", "choose_dt", "run",
]


# ----------------------------------------------------------------------------
# parameters and grid
# ----------------------------------------------------------------------------
@dataclasses.dataclass
class Params:
    """The bou.in values that the hot path reads (ReadInputFile.F90:16-56)."""
    nxm: int
    nym: int
    nzm: int
    ylen: float = 1.0
    zlen: float = 1.0
    ray: float = 1e6
    pra: float = 1.0
    alx3: float = 1.0
    istr3: int = 7
    str3: float = 0.0
    inslws: int = 1
    inslwn: int = 1
    nsst: int = 3
    tempbp: float = 1.0   # SetTempBCs.F90:16-21 (bottom plate)
    temptp: float = 0.0   # (top plate)

    @property
    def nx(self):
        return self.nxm + 1

    @property
    def ren(self):
        return math.sqrt(self.ray / self.pra)      # ReadInputFile.F90:46

    @property
    def pec(self):
        return math.sqrt(self.pra * self.ray)      # ReadInputFile.F90:47


@dataclasses.dataclass
class Grid:
    xc: np.ndarray
    xm: np.ndarray
    g3rc: np.ndarray
    g3rm: np.ndarray
    udx3c: np.ndarray
    udx3m: np.ndarray
    kmv: np.ndarray
    kpv: np.ndarray
    kmc: np.ndarray
    kpc: np.ndarray
    ap3ck: np.ndarray
    ac3ck: np.ndarray
    am3ck: np.ndarray
    ap3sk: np.ndarray
    ac3sk: np.ndarray
    am3sk: np.ndarray
    ap3ssk: np.ndarray
    ac3ssk: np.ndarray
    am3ssk: np.ndarray
    amphk: np.ndarray
    acphk: np.ndarray
    apphk: np.ndarray
    ak1: np.ndarray
    ak2: np.ndarray
    yc: np.ndarray
    ym: np.ndarray
    zc: np.ndarray
    zm: np.ndarray
    dx: float
    dy: float
    dz: float
    dxq: float
    dyq: float
    dzq: float


def make_xc(nxm: int, istr3: int, str3: float, alx3: float = 1.0) -> np.ndarray:
    """Wall-normal node positions xc(1..nx) (CreateGrid.F90:66-119; istr3=7 new)."""
    nx = nxm + 1
    pi = 2.0 * math.asin(1.0)
    xc = np.zeros(nx)
    if istr3 == 0:
        for kc in range(1, nx + 1):
            x3 = float(kc - 1) / float(nxm)
            xc[kc - 1] = alx3 * x3
    elif istr3 == 4:
        tstr3 = math.tanh(str3)
        xc[0] = 0.0
        for kc in range(2, nx + 1):
            z2dp = float(2 * kc - nx - 1) / float(nxm)
            xc[kc - 1] = (1 + math.tanh(str3 * z2dp) / tstr3) * 0.5 * alx3
            if xc[kc - 1] < 0 or xc[kc - 1] > alx3:
                raise ValueError("grid is too stretched")
    elif istr3 == 6:
        nclip = int(str3)
        nxmo = nx + nclip + nclip
        etazm = np.array([math.cos(pi * (float(kc) - 0.5) / float(nxmo))
                          for kc in range(1, nxmo + 1)])
        etaz = etazm[nclip:nclip + nx].copy()
        delet = etaz[0] - etaz[nx - 1]
        etaz = etaz / (0.5 * delet)
        xc[0] = 0.0
        for kc in range(2, nxm + 1):
            xc[kc - 1] = alx3 * (1.0 - etaz[kc - 1]) * 0.5
        xc[nx - 1] = alx3
    elif istr3 == 7:
        for kc in range(1, nx + 1):
            xc[kc - 1] = alx3 * 0.5 * (1.0 - math.cos(pi * float(kc - 1) / float(nxm)))
        xc[0] = 0.0
        xc[nx - 1] = alx3
    else:
        raise ValueError(f"istr3={istr3} not supported (0, 4, 6, 7)")
    return xc


def create_grid(p: Params, xc: np.ndarray | None = None) -> Grid:
    """Index maps, metrics and difference coefficients (CreateGrid.F90:27-266)
    plus the Poisson tables of InitPressureSolver.F90:22-59."""
    nxm, nym, nzm = p.nxm, p.nym, p.nzm
    nx, ny, nz = nxm + 1, nym + 1, nzm + 1
    pi = 2.0 * math.asin(1.0)
    if xc is None:
        xc = make_xc(nxm, p.istr3, p.str3, p.alx3)
    xc = np.asarray(xc, dtype=np.float64)
    # index maps (CreateGrid.F90:27-37); stored 0-based
    kmv = np.array([kc - 1 for kc in range(1, nxm + 1)])
    kpv = np.array([kc + 1 for kc in range(1, nxm + 1)])
    kmv[0] = 1
    kpv[nxm - 1] = nxm
    kc1 = np.arange(1, nxm + 1)
    kpc = kpv - kc1
    kmc = kc1 - kmv
    kmv0 = kmv - 1
    kpv0 = kpv - 1
    # uniform horizontal grid (CreateGrid.F90:43-59)
    zc = np.array([p.zlen * (float(i - 1) / float(nzm)) for i in range(1, nz + 1)])
    zm = (zc[:-1] + zc[1:]) * 0.5
    yc = np.array([p.ylen * (float(j - 1) / float(nym)) for j in range(1, ny + 1)])
    ym = (yc[:-1] + yc[1:]) * 0.5
    # metrics (CreateGrid.F90:129-159)
    dx = float(nxm) / p.alx3
    dy = float(nym) / p.ylen
    dz = float(nzm) / p.zlen
    dxq, dyq, dzq = dx * dx, dy * dy, dz * dz
    xm = np.zeros(nx)
    g3rm = np.zeros(nx)
    g3rc = np.zeros(nx)
    for kc in range(1, nxm + 1):
        xm[kc - 1] = (xc[kc - 1] + xc[kc]) * 0.5
        g3rm[kc - 1] = (xc[kc] - xc[kc - 1]) * dx
    for kc in range(2, nxm + 1):
        g3rc[kc - 1] = (xc[kc] - xc[kc - 2]) * dx * 0.5
    g3rc[0] = (xc[1] - xc[0]) * dx
    g3rc[nx - 1] = (xc[nx - 1] - xc[nxm - 1]) * dx
    udx3m = np.zeros(nx)
    udx3c = np.zeros(nx)
    for kc in range(1, nxm + 1):
        udx3m[kc - 1] = dx / g3rm[kc - 1]
        udx3c[kc - 1] = dx / g3rc[kc - 1]
    udx3c[nx - 1] = dx / g3rc[nx - 1]
    # centred (CreateGrid.F90:186-202)
    am3ck = np.zeros(nx); ap3ck = np.zeros(nx); ac3ck = np.zeros(nx)
    ac3ck[0] = 1.0; ac3ck[nx - 1] = 1.0
    for kc in range(2, nxm + 1):
        a33 = dxq / g3rc[kc - 1]
        a33p = 1.0 / g3rm[kc - 1]
        a33m = 1.0 / g3rm[kc - 2]
        ap3ck[kc - 1] = a33 * a33p
        am3ck[kc - 1] = a33 * a33m
        ac3ck[kc - 1] = -(ap3ck[kc - 1] + am3ck[kc - 1])
    # staggered (CreateGrid.F90:209-242)
    am3sk = np.zeros(nx); ap3sk = np.zeros(nx); ac3sk = np.zeros(nx)
    for kc in range(2, nxm):
        a33 = dxq / g3rm[kc - 1]
        a33p = +a33 / g3rc[kc]
        a33m = +a33 / g3rc[kc - 1]
        ap3sk[kc - 1] = a33p
        am3sk[kc - 1] = a33m
        ac3sk[kc - 1] = -(ap3sk[kc - 1] + am3sk[kc - 1])
    kc = 1
    a33 = dxq / g3rm[kc - 1]
    a33p = +a33 / g3rc[kc]
    a33m = +a33 / g3rc[kc - 1]
    ap3sk[kc - 1] = a33p
    am3sk[kc - 1] = 0.0
    ac3sk[kc - 1] = -(a33p + p.inslws * a33m * 2.0)
    kc = nxm
    a33 = dxq / g3rm[kc - 1]
    a33p = +a33 / g3rc[kc]
    a33m = +a33 / g3rc[kc - 1]
    am3sk[kc - 1] = a33m
    ap3sk[kc - 1] = 0.0
    ac3sk[kc - 1] = -(a33m + p.inslwn * a33p * 2.0)
    # temperature (CreateGrid.F90:244-266)
    am3ssk = np.zeros(nx); ap3ssk = np.zeros(nx); ac3ssk = np.zeros(nx)
    ac3ssk[0] = 1.0
    for kc in range(2, nxm + 1):
        a33 = dxq / g3rc[kc - 1]
        a33p = 1.0 / g3rm[kc - 1]
        a33m = 1.0 / g3rm[kc - 2]
        ap3ssk[kc - 1] = a33 * a33p
        am3ssk[kc - 1] = a33 * a33m
        ac3ssk[kc - 1] = -(ap3ssk[kc - 1] + am3ssk[kc - 1])
    ac3ssk[nx - 1] = 1.0
    # Poisson tables (InitPressureSolver.F90:22-59)
    nymh = nym // 2 + 1
    nzmh = nzm // 2 + 1
    ao = np.zeros(nzm)
    for i in range(1, nzmh + 1):
        ao[i - 1] = (i - 1) * 2.0 * pi
    for i in range(nzmh + 1, nzm + 1):
        ao[i - 1] = -(nzm - i + 1) * 2.0 * pi
    ak1 = np.array([2.0 * (1.0 - math.cos(ao[i] / nzm)) * (float(nzm) / p.zlen) ** 2
                    for i in range(nzm)])
    ap_ = np.zeros(nym)
    for j in range(1, nymh + 1):
        ap_[j - 1] = (j - 1) * 2.0 * pi
    for j in range(nymh + 1, nym + 1):
        ap_[j - 1] = -(nym - j + 1) * 2.0 * pi
    ak2 = np.array([2.0 * (1.0 - math.cos(ap_[j] / nym)) * (float(nym) / p.ylen) ** 2
                    for j in range(nym)])
    amphk = np.zeros(nxm); apphk = np.zeros(nxm); acphk = np.zeros(nxm)
    for kc in range(1, nxm + 1):
        kp = kpv[kc - 1]
        a33icc = kmc[kc - 1] * dxq / g3rc[kc - 1]
        a33icp = kpc[kc - 1] * dxq / g3rc[kp - 1]
        ugmmm = 1.0 / g3rm[kc - 1]
        amphk[kc - 1] = a33icc * ugmmm
        apphk[kc - 1] = a33icp * ugmmm
        acphk[kc - 1] = -(amphk[kc - 1] + apphk[kc - 1])
    return Grid(xc=xc, xm=xm, g3rc=g3rc, g3rm=g3rm, udx3c=udx3c, udx3m=udx3m,
                kmv=kmv0, kpv=kpv0, kmc=kmc, kpc=kpc,
                ap3ck=ap3ck, ac3ck=ac3ck, am3ck=am3ck,
                ap3sk=ap3sk, ac3sk=ac3sk, am3sk=am3sk,
                ap3ssk=ap3ssk, ac3ssk=ac3ssk, am3ssk=am3ssk,
                amphk=amphk, acphk=acphk, apphk=apphk, ak1=ak1, ak2=ak2,
                yc=yc, ym=ym, zc=zc, zm=zm,
                dx=dx, dy=dy, dz=dz, dxq=dxq, dyq=dyq, dzq=dzq)


def init_time_march_scheme(nsst: int):
    """gam, rom, alm (InitTimeMarchScheme.F90:16-48)."""
    if nsst > 1:
        gam = [8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0]
        rom = [0.0, -17.0 / 60.0, -5.0 / 12.0]
    else:
        gam = [1.5, 0.0, 0.0]
        rom = [-0.5, 0.0, 0.0]
    alm = [gam[n] + rom[n] for n in range(3)]
    return gam, rom, alm


# ----------------------------------------------------------------------------
# state
# ----------------------------------------------------------------------------
FIELDS = ("vx", "vy", "vz", "temp", "pr")
HISTORY = ("rux", "ruy", "ruz", "rutemp")
SCRATCH = ("rhs", "qcap", "dph", "dq", "hro")


@dataclasses.dataclass
class State:
    p: Params
    g: Grid
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray
    temp: np.ndarray
    pr: np.ndarray
    rux: np.ndarray
    ruy: np.ndarray
    ruz: np.ndarray
    rutemp: np.ndarray
    rhs: np.ndarray
    qcap: np.ndarray
    dph: np.ndarray
    dq: np.ndarray
    hro: np.ndarray
    time: float = 0.0

    def copy(self) -> "State":
        kw = {f.name: getattr(self, f.name) for f in dataclasses.fields(self)}
        for k, v in kw.items():
            if isinstance(v, np.ndarray):
                kw[k] = v.copy()
        return State(**kw)


def seeded_noise(p: Params, seed: int, amp: float = 0.01) -> np.ndarray:
    """Uniform [-amp, amp] noise for the interior nodes k=2..nxm.

    Drawn from numpy's PCG64(seed) in Fortran order (x fastest, then y,
    then z), returned as a [k, j, i] array of shape (nxm-1, nym, nzm)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    raw = rng.uniform(-amp, amp, size=(p.nzm, p.nym, p.nxm - 1))
    return np.ascontiguousarray(raw.transpose(2, 1, 0))


def init_state(p: Params, seed: int | None = 0, ic: str = "noise",
               xc: np.ndarray | None = None) -> State:
    """Allocate (all zero, AuxiliaryRoutines.F90:79-97) and fill the initial
    condition.  ``ic='noise'``: u=v=w=0, p=0, T linear between the plates
    (CreateInitialConditions.F90:39-52) plus seeded noise at k=2..nxm.
    ``ic='reference'``: the reference's deterministic perturbation
    (CreateInitialConditions.F90:20-53)."""
    g = create_grid(p, xc)
    nx, nxm, nym, nzm = p.nx, p.nxm, p.nym, p.nzm
    z = lambda: np.zeros((nx, nym, nzm))
    s = State(p=p, g=g, vx=z(), vy=z(), vz=z(), temp=z(), pr=z(),
              rux=z(), ruy=z(), ruz=z(), rutemp=z(), rhs=z(), qcap=z(),
              dph=np.zeros((nxm, nym, nzm)), dq=z(), hro=z())
    xc = g.xc
    tb, tt = p.tempbp, p.temptp
    for k in range(1, nxm):
        s.temp[k] = tb - (tb - tt) * xc[k] / xc[nx - 1]
    s.temp[0] = tb
    s.temp[nx - 1] = tt
    if ic == "noise":
        if seed is not None:
            s.temp[1:nxm] += seeded_noise(p, seed)
    elif ic == "reference":
        eps = 0.01
        for k in range(nxm):
            yyy = g.xm[k]
            s.vy[k] = ((2.0 * yyy - 6.0 * yyy ** 2 + 4.0 * yyy ** 3)
                       * np.sin(3 * g.yc[:nym]) * eps)[:, None]
            yyy = xc[k]
            s.vx[k] = (-yyy ** 2 * (1.0 - yyy) ** 2 * np.cos(3.1 * g.ym) * eps)[:, None]
    elif ic == "conduction":
        pass
    else:
        raise ValueError(ic)
    return s


# periodic neighbours
def _jp(a):
    return np.roll(a, -1, axis=1)


def _jm(a):
    return np.roll(a, 1, axis=1)


def _ip(a):
    return np.roll(a, -1, axis=2)


def _im(a):
    return np.roll(a, 1, axis=2)


# ----------------------------------------------------------------------------
# explicit terms
# ----------------------------------------------------------------------------
def explicit_terms_vx(s: State):
    """qcap at k=2..nxm (ExplicitTermsVX.F90:23-104)."""
    p, g = s.p, s.g
    nxm = p.nxm
    ren = p.ren
    udy = g.dy * 0.25
    udz = g.dz * 0.25
    udyq = g.dyq / ren
    udzq = g.dzq / ren
    kc = slice(1, nxm)
    km = slice(0, nxm - 1)
    kp = slice(2, nxm + 1)
    vx, vy, vz, temp = s.vx, s.vy, s.vz, s.temp
    vxc = vx[kc]
    hxz = (((_ip(vz[kc]) + _ip(vz[km])) * (_ip(vxc) + vxc))
           - ((vz[kc] + vz[km]) * (vxc + _im(vxc)))) * udz
    hxy = (((_jp(vy[kc]) + _jp(vy[km])) * (_jp(vxc) + vxc))
           - ((vy[kc] + vy[km]) * (vxc + _jm(vxc)))) * udy
    a = vx[kp] + vxc
    b = vxc + vx[km]
    hxx = (a * a - b * b) * g.udx3c[kc, None, None] * 0.25
    tempit = temp[kc]
    dzzvx = (_im(vxc) - 2.0 * vxc + _ip(vxc)) * udzq
    dyyvx = (_jm(vxc) - 2.0 * vxc + _jp(vxc)) * udyq
    s.qcap[kc] = -(hxx + hxy + hxz) + dyyvx + dzzvx + tempit


def explicit_terms_vy(s: State):
    """dph at k=1..nxm (ExplicitTermsVY.F90:23-100)."""
    p, g = s.p, s.g
    nxm = p.nxm
    ren = p.ren
    udyq = g.dyq / ren
    udzq = g.dzq / ren
    udy = g.dy * 0.25
    udz = g.dz * 0.25
    kc = slice(0, nxm)
    kmm = g.kmv
    kpp = g.kpv
    kp = slice(1, nxm + 1)
    vx, vy, vz = s.vx, s.vy, s.vz
    vyc = vy[kc]
    hyx = ((vx[kp] + _jm(vx[kp])) * (vy[kpp] + vyc)
           - (vx[kc] + _jm(vx[kc])) * (vyc + vy[kmm])) * g.udx3m[kc, None, None] * 0.25
    a = _jp(vyc) + vyc
    b = _jm(vyc) + vyc
    hyy = (a * a - b * b) * udy
    hyz = ((_ip(vyc) + vyc) * (_ip(vz[kc]) + _ip(_jm(vz[kc])))
           - (vyc + _im(vyc)) * (vz[kc] + _jm(vz[kc]))) * udz
    dyyvy = (_jp(vyc) - 2.0 * vyc + _jm(vyc)) * udyq
    dzzvy = (_ip(vyc) - 2.0 * vyc + _im(vyc)) * udzq
    s.dph[:] = -(hyx + hyy + hyz) + dyyvy + dzzvy


def explicit_terms_vz(s: State):
    """dq at k=1..nxm (ExplicitTermsVZ.F90:23-104)."""
    p, g = s.p, s.g
    nxm = p.nxm
    ren = p.ren
    udyq = g.dyq / ren
    udzq = g.dzq / ren
    udy = g.dy * 0.25
    udz = g.dz * 0.25
    kc = slice(0, nxm)
    kmm = g.kmv
    kpp = g.kpv
    kp = slice(1, nxm + 1)
    vx, vy, vz = s.vx, s.vy, s.vz
    vzc = vz[kc]
    a = _ip(vzc) + vzc
    b = _im(vzc) + vzc
    hzz = (a * a - b * b) * udz
    hzy = ((_jp(vy[kc]) + _im(_jp(vy[kc]))) * (_jp(vzc) + vzc)
           - (vy[kc] + _im(vy[kc])) * (vzc + _jm(vzc))) * udy
    hzx = ((vx[kp] + _im(vx[kp])) * (vz[kpp] + vzc)
           - (vx[kc] + _im(vx[kc])) * (vzc + vz[kmm])) * g.udx3m[kc, None, None] * 0.25
    dzzvz = (_ip(vzc) - 2.0 * vzc + _im(vzc)) * udzq
    dyyvz = (_jp(vzc) - 2.0 * vzc + _jm(vzc)) * udyq
    s.dq[kc] = -(hzx + hzy + hzz) + dyyvz + dzzvz


def explicit_terms_temp(s: State):
    """hro at k=2..nxm (ExplicitTermsTemp.F90:22-96)."""
    p, g = s.p, s.g
    nxm = p.nxm
    pec = p.pec
    udz = g.dz * 0.25
    udy = g.dy * 0.25
    udzq = g.dzq / pec
    udyq = g.dyq / pec
    kc = slice(1, nxm)
    km = slice(0, nxm - 1)
    kp = slice(2, nxm + 1)
    vx, vy, vz, t = s.vx, s.vy, s.vz, s.temp
    tc = t[kc]
    htz = ((_ip(vz[km]) + _ip(vz[kc])) * (_ip(tc) + tc)
           - (vz[km] + vz[kc]) * (tc + _im(tc))) * udz
    hty = ((_jp(vy[kc]) + _jp(vy[km])) * (_jp(tc) + tc)
           - (vy[kc] + vy[km]) * (tc + _jm(tc))) * udy
    htx = ((vx[kp] + vx[kc]) * (t[kp] + tc)
           - (vx[kc] + vx[km]) * (tc + t[km])) * g.udx3c[kc, None, None] * 0.25
    dzzt = (_ip(tc) - 2.0 * tc + _im(tc)) * udzq
    dyyt = (_jp(tc) - 2.0 * tc + _jm(tc)) * udyq
    s.hro[kc] = -(htx + hty + htz) + dyyt + dzzt


# ----------------------------------------------------------------------------
# implicit (Crank-Nicolson) updates
# ----------------------------------------------------------------------------
def _dgt_solve(dl, d, du, b2d):
    """LAPACK dgttrf + dgttrs('N') on all columns of ``b2d`` (n, nrhs)."""
    dl_, d_, du_, du2, ipiv, info = lapack.dgttrf(dl, d, du)
    if info != 0:
        raise np.linalg.LinAlgError(f"dgttrf info={info}")
    x, info = lapack.dgttrs(dl_, d_, du_, du2, ipiv, b2d)
    if info != 0:
        raise np.linalg.LinAlgError(f"dgttrs info={info}")
    return x


def solve_imp_eqn_update_x(s: State, al: float, beta: float):
    """SolveImpEqnUpdate_X.F90:25-64 (size nx, identity wall rows)."""
    p, g = s.p, s.g
    nx, nxm = p.nx, p.nxm
    betadx = beta * al
    amkl = np.zeros(nx); apkl = np.zeros(nx); ackl = np.ones(nx)
    sc = np.ones(nx)
    for kc in range(2, nxm + 1):
        ackl_b = 1.0 / (1.0 - g.ac3ck[kc - 1] * betadx)
        amkl[kc - 1] = -g.am3ssk[kc - 1] * betadx * ackl_b
        apkl[kc - 1] = -g.ap3ssk[kc - 1] * betadx * ackl_b
        sc[kc - 1] = ackl_b
    s.rhs[1:nxm] *= sc[1:nxm, None, None]
    b = s.rhs.reshape(nx, -1)
    x = _dgt_solve(amkl[1:nx], ackl.copy(), apkl[0:nx - 1], b)
    s.rhs[:] = x.reshape(s.rhs.shape)
    s.vx[1:nxm] = s.vx[1:nxm] + s.rhs[1:nxm]


def solve_imp_eqn_update_yz(s: State, q: np.ndarray, al: float, beta: float):
    """SolveImpEqnUpdate_YZ.F90:25-58 (size nxm on rows 1..nxm of rhs)."""
    p, g = s.p, s.g
    nxm = p.nxm
    betadx = beta * al
    amkl = np.zeros(nxm); apkl = np.zeros(nxm); ackl = np.ones(nxm)
    sc = np.ones(nxm)
    for kc in range(1, nxm + 1):
        ackl_b = 1.0 / (1.0 - g.ac3sk[kc - 1] * betadx)
        amkl[kc - 1] = -g.am3sk[kc - 1] * betadx * ackl_b
        apkl[kc - 1] = -g.ap3sk[kc - 1] * betadx * ackl_b
        sc[kc - 1] = ackl_b
    s.rhs[0:nxm] *= sc[:, None, None]
    b = s.rhs[0:nxm].reshape(nxm, -1)
    x = _dgt_solve(amkl[1:nxm], ackl.copy(), apkl[0:nxm - 1], b)
    s.rhs[0:nxm] = x.reshape((nxm,) + s.rhs.shape[1:])
    q[0:nxm] = q[0:nxm] + s.rhs[0:nxm]


def solve_imp_eqn_update_temp(s: State, al: float, dt: float):
    """SolveImpEqnUpdate_Temp.F90:25-67 (size nx; betadx = al dt / (2 Pe))."""
    p, g = s.p, s.g
    nx, nxm = p.nx, p.nxm
    betadx = 0.5 * al * dt / p.pec
    amkl = np.zeros(nx); apkl = np.zeros(nx); ackl = np.ones(nx)
    sc = np.ones(nx)
    for kc in range(2, nxm + 1):
        ackl_b = 1.0 / (1.0 - g.ac3ssk[kc - 1] * betadx)
        amkl[kc - 1] = -g.am3ssk[kc - 1] * betadx * ackl_b
        apkl[kc - 1] = -g.ap3ssk[kc - 1] * betadx * ackl_b
        sc[kc - 1] = ackl_b
    s.rhs[1:nxm] *= sc[1:nxm, None, None]
    b = s.rhs.reshape(nx, -1)
    x = _dgt_solve(amkl[1:nx], ackl.copy(), apkl[0:nx - 1], b)
    s.rhs[:] = x.reshape(s.rhs.shape)
    s.temp[1:nxm] = s.temp[1:nxm] + s.rhs[1:nxm]


def implicit_and_update_vx(s: State, al, ga, ro, dt, beta):
    """ImplicitAndUpdateVX.F90:24-77.  Rows 1 and nx of ``rhs`` keep whatever
    the previous solve left there, as in the reference (the module array is
    shared by all four implicit updates)."""
    p, g = s.p, s.g
    nxm = p.nxm
    alre = al / p.ren
    kc = slice(1, nxm)
    km = slice(0, nxm - 1)
    kp = slice(2, nxm + 1)
    udx3 = (al * g.udx3c[kc])[:, None, None]
    amm = g.am3ck[kc, None, None]
    acc = g.ac3ck[kc, None, None]
    app = g.ap3ck[kc, None, None]
    dxxvx = s.vx[kp] * app + s.vx[kc] * acc + s.vx[km] * amm
    dxp = (s.pr[kc] - s.pr[km]) * udx3
    s.rhs[kc] = (ga * s.qcap[kc] + ro * s.rux[kc] + alre * dxxvx - dxp) * dt
    s.rux[kc] = s.qcap[kc]
    solve_imp_eqn_update_x(s, al, beta)
    s.vx[0] = 0.0
    s.vx[p.nx - 1] = 0.0


def implicit_and_update_vy(s: State, al, ga, ro, dt, beta):
    """ImplicitAndUpdateVY.F90:26-75."""
    p, g = s.p, s.g
    nxm = p.nxm
    alre = al / p.ren
    udy = g.dy * al
    kc = slice(0, nxm)
    amm = g.am3sk[kc, None, None]
    acc = g.ac3sk[kc, None, None]
    app = g.ap3sk[kc, None, None]
    vy = s.vy
    dxxvy = vy[g.kpv] * app + vy[kc] * acc + vy[g.kmv] * amm
    dyp = (s.pr[kc] - _jm(s.pr[kc])) * udy
    s.rhs[kc] = (ga * s.dph + ro * s.ruy[kc] + alre * dxxvy - dyp) * dt
    s.ruy[kc] = s.dph
    solve_imp_eqn_update_yz(s, s.vy, al, beta)


def implicit_and_update_vz(s: State, al, ga, ro, dt, beta):
    """ImplicitAndUpdateVZ.F90:24-71."""
    p, g = s.p, s.g
    nxm = p.nxm
    alre = al / p.ren
    kc = slice(0, nxm)
    amm = g.am3sk[kc, None, None]
    acc = g.ac3sk[kc, None, None]
    app = g.ap3sk[kc, None, None]
    vz = s.vz
    dxxvz = vz[g.kpv] * app + vz[kc] * acc + vz[g.kmv] * amm
    dzp = (s.pr[kc] - _im(s.pr[kc])) * g.dz * al
    s.rhs[kc] = (ga * s.dq[kc] + ro * s.ruz[kc] + alre * dxxvz - dzp) * dt
    s.ruz[kc] = s.dq[kc]
    solve_imp_eqn_update_yz(s, s.vz, al, beta)


def implicit_and_update_temp(s: State, al, ga, ro, dt, beta):
    """ImplicitAndUpdateTemp.F90:23-73."""
    p, g = s.p, s.g
    nxm, nx = p.nxm, p.nx
    alpec = al / p.pec
    kc = slice(1, nxm)
    t = s.temp
    dxxt = (t[2:nxm + 1] * g.ap3ck[kc, None, None] + t[kc] * g.ac3ck[kc, None, None]
            + t[0:nxm - 1] * g.am3ck[kc, None, None])
    s.rhs[kc] = (ga * s.hro[kc] + ro * s.rutemp[kc] + alpec * dxxt) * dt
    s.rutemp[kc] = s.hro[kc]
    solve_imp_eqn_update_temp(s, al, dt)
    s.temp[0] = p.tempbp
    s.temp[nx - 1] = p.temptp


# ----------------------------------------------------------------------------
# pressure projection
# ----------------------------------------------------------------------------
def calc_local_divergence(s: State, al: float, dt: float):
    """dph = div(u*) / (al dt) at k=1..nxm (CalcLocalDivergence.F90:20-40)."""
    g = s.g
    nxm = s.p.nxm
    usdtal = 1.0 / (dt * al)
    kc = slice(0, nxm)
    kp = slice(1, nxm + 1)
    dqcap = ((_ip(s.vz[kc]) - s.vz[kc]) * g.dz
             + (_jp(s.vy[kc]) - s.vy[kc]) * g.dy
             + (s.vx[kp] - s.vx[kc]) * g.udx3m[kc, None, None])
    s.dph[:] = dqcap * usdtal


def _tridiag_pinned_zero_mode(dl, d, du, b):
    """Solve rows 1..n-1 of the singular (0,0) system with x(n) = 0."""
    n = d.shape[0]
    x = np.zeros_like(b)
    dl_, d_, du_, du2, ipiv, info = lapack.zgttrf(dl[:n - 2], d[:n - 1], du[:n - 2])
    if info != 0:
        raise np.linalg.LinAlgError(f"zgttrf (pinned) info={info}")
    xs, info = lapack.zgttrs(dl_, d_, du_, du2, ipiv, b[:n - 1].reshape(n - 1, 1))
    x[:n - 1] = xs[:, 0]
    return x


def solve_pressure_correction(s: State, vectorised: bool = False):
    """FFT(y,z) + per-mode complex tridiagonal in x + inverse FFT
    (SolvePressureCorrection.F90:35-151).  ``dph`` is updated in place."""
    p, g = s.p, s.g
    nxm, nym, nzm = p.nxm, p.nym, p.nzm
    nymh = nym // 2 + 1
    cy = np.fft.rfft(s.dph, axis=1)              # r2c along y (:98)
    cz = np.fft.fft(cy, axis=2)                  # c2c forward along z (:102)
    cz = cz / (nzm * nym)                        # normalise (:105)
    out = np.empty_like(cz)
    if vectorised:
        out[:] = _poisson_thomas_vectorised(g, cz, nxm, nymh, nzm)
    else:
        for i in range(nzm):
            for j in range(nymh):
                acphT_b = 1.0 / (g.acphk - g.ak2[j] - g.ak1[i])
                rhs = cz[:, j, i] * acphT_b
                apph = g.apphk * acphT_b
                amph = g.amphk * acphT_b
                d = np.ones(nxm, dtype=np.complex128)
                dl = amph[1:].astype(np.complex128)
                du = apph[:-1].astype(np.complex128)
                if i == 0 and j == 0:
                    out[:, j, i] = _tridiag_pinned_zero_mode(dl, d, du, rhs)
                    continue
                dl_, d_, du_, du2, ipiv, info = lapack.zgttrf(dl, d, du)
                if info > 0:
                    raise np.linalg.LinAlgError(f"zgttrf info={info} at mode {(j, i)}")
                x, info = lapack.zgttrs(dl_, d_, du_, du2, ipiv, rhs.reshape(nxm, 1))
                out[:, j, i] = x[:, 0]
    cz = np.fft.ifft(out, axis=2, norm="forward")             # backward z (:145)
    s.dph[:] = np.fft.irfft(cz, n=nym, axis=1, norm="forward")  # c2r y (:149)


def _poisson_thomas_vectorised(g: Grid, cz, nxm, nymh, nzm):
    """Tridiagonal solve without pivoting, vectorised over all modes, in the
    dgttrf/dgttrs operation order.  Used for sizes where one LAPACK call per
    mode is too slow; it agrees with the per-mode path to roundoff."""
    s_ = 1.0 / ((g.acphk[:, None, None] - g.ak2[None, :nymh, None]) - g.ak1[None, None, :])
    b = cz * s_
    am = g.amphk[:, None, None] * s_
    ap = g.apphk[:, None, None] * s_
    d = np.ones((nxm, nymh, nzm))
    fact = np.zeros((nxm, nymh, nzm))
    for k in range(nxm - 1):
        fact[k] = am[k + 1] / d[k]
        d[k + 1] = d[k + 1] - fact[k] * ap[k]
        b[k + 1] = b[k + 1] - fact[k] * b[k]
    x = np.empty_like(b)
    with np.errstate(divide="ignore", invalid="ignore"):
        x[nxm - 1] = b[nxm - 1] / d[nxm - 1]
    x[nxm - 1, 0, 0] = 0.0
    for k in range(nxm - 2, -1, -1):
        x[k] = (b[k] - ap[k] * x[k + 1]) / d[k]
    return x


def correct_velocity(s: State, al: float, dt: float):
    """CorrectVelocity.F90:19-44."""
    g = s.g
    nxm = s.p.nxm
    udy = al * dt * g.dy
    udz = al * dt * g.dz
    kc = slice(0, nxm)
    usukm = (al * dt * g.udx3c[kc])[:, None, None]
    dph = s.dph
    s.vx[kc] = s.vx[kc] - (dph - dph[g.kmv]) * usukm
    s.vy[kc] = s.vy[kc] - (dph - _jm(dph)) * udy
    s.vz[kc] = s.vz[kc] - (dph - _im(dph)) * udz


def correct_pressure(s: State, al: float, beta: float):
    """CorrectPressure.F90:19-51."""
    g = s.g
    nxm = s.p.nxm
    be = al * beta
    dph = s.dph
    kc = slice(0, nxm)
    amm = g.amphk[:, None, None]
    acc = g.acphk[:, None, None]
    app = g.apphk[:, None, None]
    s.pr[kc] = s.pr[kc] + dph - be * (
        (_ip(dph) - 2.0 * dph + _im(dph)) * g.dzq
        + (_jp(dph) - 2.0 * dph + _jm(dph)) * g.dyq
        + (dph[g.kpv] * app + dph * acc + dph[g.kmv] * amm))


# ----------------------------------------------------------------------------
# integrator and diagnostics
# ----------------------------------------------------------------------------
def substep(s: State, ns: int, dt: float, vectorised_poisson: bool = False):
    """One substep ns (0-based) of TimeMarcher.F90:28-72."""
    p = s.p
    gam, rom, alm = init_time_march_scheme(p.nsst)
    beta = dt / p.ren * 0.5
    al, ga, ro = alm[ns], gam[ns], rom[ns]
    explicit_terms_vx(s)
    explicit_terms_vy(s)
    explicit_terms_vz(s)
    explicit_terms_temp(s)
    implicit_and_update_vx(s, al, ga, ro, dt, beta)
    implicit_and_update_vy(s, al, ga, ro, dt, beta)
    implicit_and_update_vz(s, al, ga, ro, dt, beta)
    implicit_and_update_temp(s, al, ga, ro, dt, beta)
    calc_local_divergence(s, al, dt)
    solve_pressure_correction(s, vectorised=vectorised_poisson)
    correct_velocity(s, al, dt)
    correct_pressure(s, al, beta)


def time_marcher(s: State, dt: float, vectorised_poisson: bool = False):
    """TimeMarcher.F90:22-74: nsst substeps."""
    for ns in range(s.p.nsst):
        substep(s, ns, dt, vectorised_poisson)


def calc_max_cfl(s: State) -> float:
    """CalcMaxCFL.F90:21-45."""
    g = s.g
    nxm = s.p.nxm
    kc = slice(0, nxm)
    kp = slice(1, nxm + 1)
    qcf = (np.abs((s.vz[kc] + _ip(s.vz[kc])) * 0.5 * g.dz)
           + np.abs((s.vy[kc] + _jp(s.vy[kc])) * 0.5 * g.dy)
           + np.abs((s.vx[kc] + s.vx[kp]) * 0.5 * g.udx3m[kc, None, None]))
    return max(0.00000001, float(qcf.max()))


def check_divergence(s: State) -> float:
    """Max |div u| (CheckDivergence.F90:21-44)."""
    g = s.g
    nxm = s.p.nxm
    kc = slice(0, nxm)
    kp = slice(1, nxm + 1)
    dqcap = ((_ip(s.vz[kc]) - s.vz[kc]) * g.dz
             + (_jp(s.vy[kc]) - s.vy[kc]) * g.dy
             + (s.vx[kp] - s.vx[kc]) * g.udx3m[kc, None, None])
    return float(np.abs(dqcap).max())


def calc_plate_nu(s: State):
    """(Nu_bottom, Nu_top) (CalcPlateNu.F90:22-43)."""
    p, g = s.p, s.g
    nx, nxm = p.nx, p.nxm
    dl = 1.0 / (g.xc[1] - g.xc[0])
    dn = 1.0 / (g.xc[nx - 1] - g.xc[nxm - 1])
    nuslow = float(((s.temp[0] - s.temp[1]) * dl).sum()) / (p.nzm * p.nym)
    nusupp = float(((s.temp[nxm - 1] - s.temp[nx - 1]) * dn).sum()) / (p.nzm * p.nym)
    return nuslow, nusupp


def global_quantities(s: State):
    """Volume Nu, max velocities, mean/min/max T, rms velocities
    (GlobalQuantities.F90:23-97)."""
    p, g = s.p, s.g
    nxm = p.nxm
    kc = slice(0, nxm)
    kp = slice(1, nxm + 1)
    vol = 1.0 / (p.alx3 * g.dx * float(p.nzm) * float(p.nym))
    fac2 = g.g3rc[kc, None, None]
    vxcen = (s.vx[kc] + s.vx[kp]) * 0.5
    tcen = (s.temp[kc] + s.temp[kp]) * 0.5
    anusin = float((tcen * vxcen * fac2).sum())
    tempm = float((tcen * fac2).sum())
    vxr = float((fac2 * s.vx[kc] ** 2).sum())
    vyr = float((fac2 * s.vy[kc] ** 2).sum())
    vzr = float((fac2 * s.vz[kc] ** 2).sum())
    rr = math.sqrt(p.ray / p.pra)
    return dict(
        nu_vol=1.0 + math.sqrt(p.pra * p.ray) * anusin * vol,
        vmax=(float(np.abs(s.vz[kc]).max()), float(np.abs(s.vy[kc]).max()),
              float(np.abs(s.vx[kc]).max())),
        tempm=tempm * vol, tempmax=float(s.temp[kc].max()),
        tempmin=float(s.temp[kc].min()),
        vx_rms=math.sqrt(vxr * vol) * rr, vy_rms=math.sqrt(vyr * vol) * rr,
        vz_rms=math.sqrt(vzr * vol) * rr,
        vel_rms=math.sqrt((vzr + vyr + vxr) * vol) * rr)


def dissipation_metrics(g: Grid, nxm: int):
    """dxm, dxc, lem, lec of CalcDissipationNu.F90:32-40 (0-based k)."""
    xm, xc, dx = g.xm, g.xc, g.dx
    dxm = np.empty(nxm)
    dxc = np.empty(nxm)
    lem = np.empty(nxm)
    lec = np.empty(nxm)
    for k in range(nxm):
        dxm[k] = 1.0 / (xm[k + 1] - xm[k]) if k < nxm - 1 else 0.0
        dxc[k] = 1.0 / (xc[k + 1] - xc[k])
        lem[k] = (xc[k + 1] - xc[k]) * dx
        lec[k] = (xm[k + 1] - xm[k]) * dx
    lec[nxm - 1] = (xm[nxm - 1] - xm[nxm - 2]) * dx
    dxm[nxm - 1] = 1.0 / (xm[nxm - 1] - xm[nxm - 2])
    return dxm, dxc, lem, lec


def calc_dissipation_nu(s: State):
    """Nusselt numbers from the viscous and thermal dissipation rates and
    their per-plane profiles (CalcDissipationNu.F90:42-117).  Returns nu_mu,
    nu_th and the per-plane increments of the disste and dissth
    accumulators (the stat arrays of the reference)."""
    p, g = s.p, s.g
    nxm, nym, nzm = p.nxm, p.nym, p.nzm
    dxm, dxc, lem, lec = dissipation_metrics(g, nxm)
    kc, kp = slice(0, nxm), slice(1, nxm + 1)
    c3 = (slice(None), None, None)
    vx, vy, vz, t = s.vx[kc], s.vy[kc], s.vz[kc], s.temp[kc]
    hxx = (s.vx[kp] - vx) * dxc[c3]
    hxy = (_jp(vx) - vx) * g.dy
    hxz = (_ip(vx) - vx) * g.dz
    hyx = (s.vy[kp] - vy) * dxm[c3]
    hyy = (_jp(vy) - vy) * g.dy
    hyz = (_ip(vy) - vy) * g.dz
    hzx = (s.vz[kp] - vz) * dxm[c3]
    hzy = (_jp(vz) - vz) * g.dy
    hzz = (_ip(vz) - vz) * g.dz
    dissipte = hxx * hxx + hxy * hxy + hxz * hxz
    dissipte2 = (hyx * hyx + hyy * hyy + hyz * hyz) + (hzx * hzx + hzy * hzy + hzz * hzz)
    nu_mu = float((dissipte * lem[c3] * p.pra + dissipte2 * lec[c3] * p.pra).sum())
    tx = (s.temp[kp] - t) * dxc[c3]
    ty = (_jp(t) - t) * g.dy
    tz = (_ip(t) - t) * g.dz
    dissipth = tx * tx + ty * ty + tz * tz
    nu_th = float((dissipth * lem[c3]).sum())
    disste = ((dissipte + dissipte2) / (p.ren * float(nym) * float(nzm))).sum(axis=(1, 2))
    dissth = (dissipth / (p.pec * float(nym) * float(nzm))).sum(axis=(1, 2))
    volt = 1.0 / (float(nxm) * float(nzm) * float(nym))
    return dict(nu_mu=nu_mu * volt + 1, nu_th=nu_th * volt, disste=disste, dissth=dissth)


STAT_NAMES = ("vx_me", "vy_me", "vz_me", "temp_me", "vx_rms", "vy_rms", "vz_rms", "temp_rms",
              "tempvx_me", "disste", "dissth")


def calc_stats(s: State, acc: dict | None = None) -> dict:
    """Horizontal means of CalcStats (StatRoutines.F90:21-43), added to the
    accumulators ``acc`` (created zeroed on first use, with the sample count
    ``nstatsamples``)."""
    p = s.p
    nxm = p.nxm
    if acc is None:
        acc = {k: np.zeros(nxm) for k in STAT_NAMES}
        acc["nstatsamples"] = 0
    acc["nstatsamples"] += 1
    usnym, usnzm = 1.0 / p.nym, 1.0 / p.nzm
    kc = slice(0, nxm)
    vx, vy, vz, t = s.vx[kc], s.vy[kc], s.vz[kc], s.temp[kc]
    for name, q in (("vx_me", vx), ("vy_me", vy), ("vz_me", vz), ("temp_me", t),
                    ("vx_rms", vx ** 2), ("vy_rms", vy ** 2), ("vz_rms", vz ** 2),
                    ("temp_rms", t ** 2), ("tempvx_me", t * vx)):
        acc[name] += (q * usnzm * usnym).sum(axis=(1, 2))
    return acc


def slab_locations(g: Grid, nxm: int, xslab) -> list[int]:
    """kslab(1..9) of InitializeSlabDump (SlabDumpRoutines.F90:52-67), 1-based:
    slab m = 2..9 sits at the first k whose cell centre interval
    (xm(k-1), xm(k)) contains xslab(m); kslab(1) = 2."""
    kslab = [2] * 9
    for k in range(2, nxm + 1):
        for m in range(2, 10):
            if g.xm[k - 1] > xslab[m - 2] and g.xm[k - 2] < xslab[m - 2]:
                kslab[m - 1] = k
    return kslab


def slab_dump(s: State, kslab) -> np.ndarray:
    """The four horizontal slabs of SlabDumper (SlabDumpRoutines.F90:15-24)
    at each 1-based kslab: (vx(k) + vx(k+1)) / 2, vy(k), vz(k), temp(k).
    Returns an array (len(kslab), 4, nym, nzm)."""
    out = []
    for k in kslab:
        kk = k - 1
        out.append(np.stack([(s.vx[kk] + s.vx[kk + 1]) * 0.5, s.vy[kk], s.vz[kk], s.temp[kk]]))
    return np.array(out)


def choose_dt(ntime: int, instcfl: float, dt: float, idtv: int, cflmax: float,
              dtmin: float, dtmax: float):
    """main.F90:171-189: returns (dt, cfl*dt or cfl, errorcode)."""
    err = 0
    if idtv:
        if ntime > 1:
            if instcfl < 1.0e-8:
                dt = dtmax
            else:
                dt = cflmax / instcfl
            if dt > dtmax:
                dt = dtmax
        else:
            dt = dtmin
        if dt < dtmin:
            err = 166
    else:
        instcfl = instcfl * dt
        if instcfl > cflmax:
            err = 165
    return dt, instcfl, err


def run(s: State, nsteps: int, dt: float, idtv: int = 0, cflmax: float = 1.2,
        dtmin: float = 1e-8, dtmax: float = 1e-2, vectorised_poisson: bool = False):
    """``nsteps`` passes of main.F90:167-200 (CFL, dt rule, TimeMarcher,
    time += dt); returns per-step records (dt, cfl, plate Nu, max div)."""
    recs = []
    for ntime in range(nsteps):
        cfl = calc_max_cfl(s)
        dt, cfl_used, err = choose_dt(ntime, cfl, dt, idtv, cflmax, dtmin, dtmax)
        time_marcher(s, dt, vectorised_poisson)
        s.time += dt
        nub, nut = calc_plate_nu(s)
        recs.append(dict(ntime=ntime, dt=dt, cfl=cfl_used, err=err,
                         nu_bot=nub, nu_top=nut, div=check_divergence(s)))
    return recs


# ----------------------------------------------------------------------------
# Restart onto a new grid: ReadFlowField.F90:63-150 with interp.F90:11-227
# ----------------------------------------------------------------------------
# interp.F90's case selector per field, as ReadFlowField.F90:70-73 passes it
# (vxflag = 1 ... teflag = 4).  Case 1 interpolates on the z nodes and case 3
# on the x nodes (interp.F90:65-94), so vx is regridded with vz's staggering
# and vz with vx's: the reference's behaviour, kept.
INTERP_FLAG = {"vx": 1, "vy": 2, "vz": 3, "temp": 4}


def gridnew(n: int, rext: float, istr: int, stri: float) -> tuple[np.ndarray, np.ndarray]:
    """interp.F90:229-296 with the halo extrapolation of interp.F90:45-60:
    nodes rc and centres rm of an n-point grid on [0, rext], as arrays indexed
    like the Fortran ones, 0..n+1 (rc(0), rc(n+1), rm(0), rm(n+1) extrapolated
    to second order).  gridnew defines istr 0 (uniform) and 6 (clipped
    Chebyshev) only; for those its nodes are CreateGrid's."""
    if istr not in (0, 6):
        raise ValueError(f"interp.F90's gridnew defines istr 0 and 6 only (got {istr})")
    rc = np.zeros(n + 2)
    rm = np.zeros(n + 2)
    rc[1:n + 1] = make_xc(n - 1, istr, stri, rext)
    for i in range(1, n):
        rm[i] = (rc[i] + rc[i + 1]) * 0.5
    rm[n] = 2 * rc[n] - rm[n - 1]
    for a in (rc, rm):
        a[0] = 2 * a[1] - a[2]
        a[n + 1] = 2 * a[n] - a[n - 1]
    return rc, rm


def interp_check(nxo: int, nyo: int, nzo: int, istro3: int, nx: int, ny: int, nz: int, istr3: int) -> None:
    """The conditions ReadFlowField.F90:88-99 and interp.F90's gridnew put
    on a regrid (point counts nx = nxm + 1, ny = nym + 1, nz = nzm + 1)."""
    if nz > nzo * 2 or ny > nyo * 2 or nx > nxo * 2:
        raise ValueError("new grid resolution cannot be more than twice the old resolution")
    if min(nxo, nyo, nzo) < 3:
        raise ValueError("old grid too small to extrapolate its halo")
    for s in (istro3, istr3):
        if s not in (0, 6):
            raise ValueError(f"interp.F90's gridnew defines istr 0 and 6 only (got {s})")


def _bracket(old: np.ndarray, n: int, new: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """interp.F90:137-169: for each new coordinate the first old index l in
    1..n with old(l) >= new, returned as (l-1, l); (n-1, n) when there is none."""
    ge = old[None, 1:n + 1] >= new[:, None]
    has = ge.any(axis=1)
    l = np.where(has, ge.argmax(axis=1) + 1, n)
    return np.where(has, l - 1, n - 1), l


def interp_field(old: np.ndarray, nxo: int, nyo: int, nzo: int, istro3: int, stro3: float,
                 flag: int, nxm: int, nym: int, nzm: int, istr3: int, str3: float,
                 ylen: float, zlen: float) -> np.ndarray:
    """One field of a snapshot interpolated onto the grid (nxm, nym, nzm)
    (interp.F90:11-227).  ``old`` is a[k, j, i] of shape (nxo, nyo-1, nzo-1)
    (the continua dataset); the result has shape (nxm+1, nym, nzm).

    As in the reference: the old array's halo is filled by linear
    extrapolation on its six faces only (interp.F90:95-117); the stencil
    reads the lower x index in three of its four upper-x corners
    (interp.F90:184-191, sffc/sccc/scfc); the x grids are built with
    extent 1 whatever alx3 (interp.F90:42,64).  The halo's edges and corners,
    which the reference never writes yet reads for new points below the
    first old point in two directions, are zero here (what a fresh
    allocation holds)."""
    nx, ny, nz = nxm + 1, nym + 1, nzm + 1
    interp_check(nxo, nyo, nzo, istro3, nx, ny, nz, istr3)
    nyom, nzom = nyo - 1, nzo - 1
    if old.shape != (nxo, nyom, nzom):
        raise ValueError(f"old field shape {old.shape}, expected {(nxo, nyom, nzom)}")
    tco, tmo = gridnew(nzo, zlen, 0, 1.0)
    rco, rmo = gridnew(nyo, ylen, 0, 1.0)
    zzo, zmo = gridnew(nxo, 1.0, istro3, stro3)
    tcn, tmn = gridnew(nz, zlen, 0, 1.0)
    rcn, rmn = gridnew(ny, ylen, 0, 1.0)
    zzn, zmn = gridnew(nx, 1.0, istr3, str3)
    xold, yold, zold, xnew, ynew, znew = {
        1: (tco, rmo, zmo, tcn, rmn, zmn),
        2: (tmo, rco, zmo, tmn, rcn, zmn),
        3: (tmo, rmo, zzo, tmn, rmn, zzn),
        4: (tmo, rmo, zmo, tmn, rmn, zmn)}[flag]
    # padded old array a(0:nxo+1, 0:nyom+1, 0:nzom+1)
    a = np.zeros((nxo + 2, nyom + 2, nzom + 2))
    a[1:nxo + 1, 1:nyom + 1, 1:nzom + 1] = old
    a[0, 1:nyom + 1, 1:nzom + 1] = 2.0 * a[1, 1:nyom + 1, 1:nzom + 1] - a[2, 1:nyom + 1, 1:nzom + 1]
    a[nxo + 1, 1:nyom + 1, 1:nzom + 1] = 2.0 * a[nxo, 1:nyom + 1, 1:nzom + 1] - a[nxo - 1, 1:nyom + 1, 1:nzom + 1]
    a[1:nxo + 1, 1:nyom + 1, 0] = 2.0 * a[1:nxo + 1, 1:nyom + 1, 1] - a[1:nxo + 1, 1:nyom + 1, 2]
    a[1:nxo + 1, 1:nyom + 1, nzom + 1] = 2.0 * a[1:nxo + 1, 1:nyom + 1, nzom] - a[1:nxo + 1, 1:nyom + 1, nzom - 1]
    a[1:nxo + 1, 0, 1:nzom + 1] = 2.0 * a[1:nxo + 1, 1, 1:nzom + 1] - a[1:nxo + 1, 2, 1:nzom + 1]
    a[1:nxo + 1, nyom + 1, 1:nzom + 1] = 2.0 * a[1:nxo + 1, nyom, 1:nzom + 1] - a[1:nxo + 1, nyom - 1, 1:nzom + 1]
    # interp's x, y, z are the z, y, x directions: i (nzm), j (nym), k (nx)
    bix = xnew[1:nzm + 1]
    biy = ynew[1:nym + 1]
    biz = znew[1:nx + 1]
    fi, ci = _bracket(xold, nzo, bix)
    fj, cj = _bracket(yold, nyo, biy)
    fk, ck = _bracket(zold, nxo, biz)
    bix1, bix2 = xold[fi], xold[ci]
    biy1, biy2 = yold[fj], yold[cj]
    biz1, biz2 = zold[fk], zold[ck]
    K = (slice(None), None, None)
    J = (None, slice(None), None)
    I = (None, None, slice(None))
    FK, CK, FJ, CJ, FI, CI = fk[K], ck[K], fj[J], cj[J], fi[I], ci[I]
    aficjfk = a[FK, CJ, FI]
    afifjfk = a[FK, FJ, FI]
    acicjfk = a[FK, CJ, CI]
    acifjfk = a[FK, FJ, CI]
    aficjck = a[CK, CJ, FI]
    afifjck = a[FK, FJ, FI]
    acicjck = a[FK, CJ, CI]
    acifjck = a[FK, FJ, CI]
    X, X1, X2 = bix[I], bix1[I], bix2[I]
    Y, Y1, Y2 = biy[J], biy1[J], biy2[J]
    Z, Z1, Z2 = biz[K], biz1[K], biz2[K]
    dxdydz = 1.0 / ((X2 - X1) * (Y2 - Y1) * (Z2 - Z1))
    ans = (aficjfk * (X2 - X) * (Y - Y1) * (Z2 - Z)
           + afifjfk * (X2 - X) * (Y2 - Y) * (Z2 - Z)
           + acicjfk * (X - X1) * (Y - Y1) * (Z2 - Z)
           + acifjfk * (X - X1) * (Y2 - Y) * (Z2 - Z)
           + aficjck * (X2 - X) * (Y - Y1) * (Z - Z1)
           + afifjck * (X2 - X) * (Y2 - Y) * (Z - Z1)
           + acicjck * (X - X1) * (Y - Y1) * (Z - Z1)
           + acifjck * (X - X1) * (Y2 - Y) * (Z - Z1)) * dxdydz
    return np.ascontiguousarray(ans)
