"""Host-side mirror of the reference's hot-path interface, over the C-ABI.

``Context`` owns device memory and a CUDA stream (afid_ctx).  ``Box`` is one
simulation: the state the reference keeps in its modules, resident in HBM.
Its methods carry the names of the reference subroutines they replace
(ExplicitTermsVX -> ``explicit_terms_vx`` ...); ``Context.step`` advances
many boxes together through the fused kernels.

Arrays cross the boundary indexed ``a[k, j, i]`` (x, y, z), shape
``(nx, nym, nzm)`` (``(nxm, nym, nzm)`` for dph), float64.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .config import BouIn

FIELD_ROWS_NXM = {"dph"}


def make_grid(nxm: int, istr3: int = 7, str3: float = 0.0, alx3: float = 1.0) -> np.ndarray:
    """xc(1..nx) of CreateGrid.F90:66-119 (plus istr3 = 7), computed by the library."""
    xc = np.zeros(nxm + 1)
    _lib.check(_lib.lib().afid_make_grid(nxm, istr3, str3, alx3, _lib.dptr(xc)))
    return xc


def slab_locations(xc: np.ndarray, xslab) -> list[int]:
    """kslab(1..9) of InitializeSlabDump from the eight x positions of
    stst3.in (1-based planes), computed by the library."""
    nxm = len(xc) - 1
    xs = np.ascontiguousarray(xslab, dtype=np.float64)
    if xs.shape != (8,):
        raise ValueError("xslab holds the eight positions of slabs 2..9")
    ks = np.zeros(9, dtype=np.int32)
    _lib.check(_lib.lib().afid_slab_locations(nxm, _lib.dptr(np.ascontiguousarray(xc, dtype=np.float64)),
                                              _lib.dptr(xs), ks.ctypes.data_as(C.POINTER(C.c_int))))
    return [int(k) for k in ks]


def box_params(cfg: BouIn) -> _lib.BoxParams:
    p = _lib.BoxParams()
    for name in ("nxm", "nym", "nzm", "nsst", "alx3", "ylen", "zlen", "ray", "pra", "inslws",
                 "inslwn", "tempbp", "temptp", "dt", "idtv", "cflmax", "dtmin", "dtmax", "vlim",
                 "resid"):
        setattr(p, name, getattr(cfg, name))
    return p


def device_bytes(cfg: BouIn) -> int:
    p = box_params(cfg)
    return int(_lib.lib().afid_box_device_bytes(C.byref(p)))


class Context:
    def __init__(self, device: int = 0):
        self._L = _lib.lib()
        h = C.c_void_p()
        _lib.check(self._L.afid_ctx_create(C.byref(h), device))
        self.h = h
        self.device = device
        self.boxes: dict[int, Box] = {}

    # -- lifetime
    def close(self):
        if self.h:
            self._L.afid_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- streams
    @property
    def stream(self) -> int:
        return int(self._L.afid_ctx_stream(self.h) or 0)

    def set_stream(self, handle: int | None):
        _lib.check(self._L.afid_ctx_set_stream(self.h, C.c_void_p(handle or 0)))

    def set_split_sets(self, on: bool):
        """Run large box sets as two halves on two streams in graph steps
        (the default) or whole (see afid_ctx_set_split_sets)."""
        _lib.check(self._L.afid_ctx_set_split_sets(self.h, 1 if on else 0))

    def synchronize(self):
        _lib.check(self._L.afid_ctx_synchronize(self.h))

    # -- boxes
    def add_box(self, cfg: BouIn, xc: np.ndarray | None = None, validate: bool = True) -> "Box":
        """A box for ``cfg``.  ``validate`` applies the reference's start-up
        checks (ReadInputFile/main.F90); without it only the library's own
        limits apply (e.g. its transforms also take a largest factor of 7,
        which the reference's Factorize rejects)."""
        if validate:
            cfg.validate()
        if xc is None:
            xc = make_grid(cfg.nxm, cfg.istr3, cfg.str3, cfg.alx3)
        xc = np.ascontiguousarray(xc, dtype=np.float64)
        p = box_params(cfg)
        bid = C.c_int()
        _lib.check(self._L.afid_box_add(self.h, C.byref(p), _lib.dptr(xc), C.byref(bid)))
        b = Box(self, bid.value, cfg, xc)
        self.boxes[b.id] = b
        return b

    def remove_box(self, box: "Box"):
        _lib.check(self._L.afid_box_remove(self.h, box.id))
        self.boxes.pop(box.id, None)

    @staticmethod
    def _ids(boxes):
        ids = (C.c_int * len(boxes))(*[b.id for b in boxes])
        return ids, len(boxes)

    def step(self, boxes, nsteps: int = 1, graph: bool = False):
        """nsteps of main.F90:171-200 for every box, batched."""
        ids, n = self._ids(boxes)
        f = self._L.afid_step_graph if graph else self._L.afid_step
        _lib.check(f(self.h, ids, n, nsteps))

    def graph_kernels(self, boxes) -> int:
        """Kernels one graph step of ``boxes`` launches (see Context.step)."""
        ids, n = self._ids(boxes)
        k = C.c_int(0)
        _lib.check(self._L.afid_step_graph_kernels(self.h, ids, n, C.byref(k)))
        return k.value

    def scalars(self, boxes) -> list[dict]:
        """Box.scalars() of every box of ``boxes``, read with one copy."""
        ids, n = self._ids(boxes)
        out = (_lib.BoxScalars * n)()
        _lib.check(self._L.afid_boxes_get_scalars(self.h, ids, n, out))
        return [dict(dt=s.dt, time=s.time, cfl=s.cfl, cfl_used=s.cfl_used, divmax=s.divmax,
                     vmax=tuple(s.vmax), nu_bot=s.nu_bot, nu_top=s.nu_top, ntime=s.ntime,
                     status=s.status) for s in out]

    def step_profiled(self, boxes, nsteps: int = 1) -> dict:
        """Per-kernel device time (ms, summed over nsteps) and launch counts."""
        ids, n = self._ids(boxes)
        nk = len(_lib.KERNELS)
        ms = (C.c_double * nk)()
        cnt = (C.c_int * nk)()
        _lib.check(self._L.afid_step_profiled(self.h, ids, n, nsteps, ms, cnt, nk))
        return {k: (ms[q], cnt[q]) for q, k in enumerate(_lib.KERNELS)}

    def substep(self, boxes, ns: int):
        ids, n = self._ids(boxes)
        _lib.check(self._L.afid_substep(self.h, ids, n, ns))


class Box:
    def __init__(self, ctx: Context, bid: int, cfg: BouIn, xc: np.ndarray):
        self.ctx = ctx
        self.id = bid
        self.cfg = cfg
        self.xc = xc

    @property
    def _L(self):
        return self.ctx._L

    def _rows(self, field: str) -> int:
        return self.cfg.nxm if field in FIELD_ROWS_NXM else self.cfg.nx

    # -- data movement (Fortran order across the C-ABI)
    def upload(self, field: str, a: np.ndarray):
        c = self.cfg
        if field == "wall":
            buf = np.ascontiguousarray(np.asarray(a, dtype=np.float64).T)   # (j, i) -> i-major
            if buf.shape != (c.nzm, c.nym):
                raise ValueError("wall plane must be (nym, nzm)")
        else:
            a = np.asarray(a, dtype=np.float64)
            if a.shape != (self._rows(field), c.nym, c.nzm):
                raise ValueError(f"{field}: shape {a.shape} != {(self._rows(field), c.nym, c.nzm)}")
            buf = np.ascontiguousarray(a.transpose(2, 1, 0))
        _lib.check(self._L.afid_box_upload(self.ctx.h, self.id, _lib.FIELDS[field], _lib.dptr(buf)))

    def download(self, field: str) -> np.ndarray:
        c = self.cfg
        if field == "wall":
            buf = np.empty((c.nzm, c.nym))
            _lib.check(self._L.afid_box_download(self.ctx.h, self.id, _lib.FIELDS[field], _lib.dptr(buf)))
            return buf.T.copy()
        buf = np.empty((c.nzm, c.nym, self._rows(field)))
        _lib.check(self._L.afid_box_download(self.ctx.h, self.id, _lib.FIELDS[field], _lib.dptr(buf)))
        return np.ascontiguousarray(buf.transpose(2, 1, 0))

    def set_tuning(self, fft_y_lines: int = 0, fft_z_lines: int = 0, k1_minb: int = 0):
        """Launch shapes of this box's kernels (results do not depend on them)."""
        _lib.check(self._L.afid_box_set_tuning(self.ctx.h, self.id, fft_y_lines, fft_z_lines, k1_minb))
        self.tuning = (fft_y_lines, fft_z_lines, k1_minb)

    def set_time(self, time: float):
        """Simulation time of the box (as restored from continua files)."""
        _lib.check(self._L.afid_box_set_time(self.ctx.h, self.id, float(time)))

    def interp_field(self, field: str, old: np.ndarray, nxo: int, nyo: int, nzo: int,
                     istro3: int, stro3: float):
        """One continua dataset of a run on another grid (nxo, nyo, nzo points,
        wall-normal grid istro3/stro3), interpolated onto this box's grid on
        the device as ReadFlowField.F90:63-150 / interp.F90 do.  ``old`` is
        a[k, j, i] of shape (nxo, nyo-1, nzo-1)."""
        a = np.asarray(old, dtype=np.float64)
        if a.shape != (nxo, nyo - 1, nzo - 1):
            raise ValueError(f"old field shape {a.shape}, expected {(nxo, nyo - 1, nzo - 1)}")
        buf = np.ascontiguousarray(a.ravel(order="F"))
        _lib.check(self._L.afid_box_interp_field(self.ctx.h, self.id, _lib.FIELDS[field], _lib.dptr(buf),
                                                 nxo, nyo, nzo, int(istro3), float(stro3),
                                                 int(self.cfg.istr3), float(self.cfg.str3)))

    def set_stop(self, stop_ntime: int = 0, tout: float = 0.0, tmax: float = 0.0):
        """Hold the box after the step that brings its step count to
        ``stop_ntime``, with ``tout`` > 0 at every output time of
        main.F90:207, and with ``tmax`` > 0 once time > tmax; a held box has
        status ``_lib.STATUS_HELD``."""
        _lib.check(self._L.afid_box_set_stop(self.ctx.h, self.id, int(stop_ntime), float(tout),
                                             float(tmax)))

    def resume(self):
        """Release the box from a hold (queued on the context's stream)."""
        _lib.check(self._L.afid_box_resume(self.ctx.h, self.id))

    def reset(self, dt: float = 0.0):
        _lib.check(self._L.afid_box_reset(self.ctx.h, self.id, dt))

    def scalars(self) -> dict:
        s = _lib.BoxScalars()
        _lib.check(self._L.afid_box_get_scalars(self.ctx.h, self.id, C.byref(s)))
        return dict(dt=s.dt, time=s.time, cfl=s.cfl, cfl_used=s.cfl_used, divmax=s.divmax,
                    vmax=tuple(s.vmax), nu_bot=s.nu_bot, nu_top=s.nu_top, ntime=s.ntime,
                    status=s.status)

    def history(self, max_records: int = 4096) -> list[dict]:
        recs = (_lib.StepRecord * max_records)()
        n = _lib.check(self._L.afid_box_history(self.ctx.h, self.id, recs, max_records))
        return [{k: getattr(recs[r], k) for k, _ in _lib.StepRecord._fields_} for r in range(n)]

    # -- routine-level entry points (reference names)
    def time_marcher_begin_substep(self, ns: int):
        _lib.check(self._L.afid_time_marcher_begin_substep(self.ctx.h, self.id, ns))

    def _call(self, name: str):
        _lib.check(getattr(self._L, "afid_" + name)(self.ctx.h, self.id))

    def explicit_terms_vx(self): self._call("explicit_terms_vx")
    def explicit_terms_vy(self): self._call("explicit_terms_vy")
    def explicit_terms_vz(self): self._call("explicit_terms_vz")
    def explicit_terms_temp(self): self._call("explicit_terms_temp")
    def implicit_and_update_vx(self): self._call("implicit_and_update_vx")
    def implicit_and_update_vy(self): self._call("implicit_and_update_vy")
    def implicit_and_update_vz(self): self._call("implicit_and_update_vz")
    def implicit_and_update_temp(self): self._call("implicit_and_update_temp")
    def calc_local_divergence(self): self._call("calc_local_divergence")
    def solve_pressure_correction(self): self._call("solve_pressure_correction")
    def correct_velocity(self): self._call("correct_velocity")
    def correct_pressure(self): self._call("correct_pressure")

    def calc_max_cfl(self) -> float:
        v = C.c_double()
        _lib.check(self._L.afid_calc_max_cfl(self.ctx.h, self.id, C.byref(v)))
        return v.value

    def check_divergence(self) -> float:
        v = C.c_double()
        _lib.check(self._L.afid_check_divergence(self.ctx.h, self.id, C.byref(v)))
        return v.value

    def calc_plate_nu(self) -> tuple[float, float]:
        a, b = C.c_double(), C.c_double()
        _lib.check(self._L.afid_calc_plate_nu(self.ctx.h, self.id, C.byref(a), C.byref(b)))
        return a.value, b.value

    # ---- output-time diagnostics (main.F90:202-216) ----------------------
    def global_quantities(self) -> dict:
        """GlobalQuantities.F90: volume Nu, max |v|, temperature mean and
        extrema, rms velocities (times sqrt(Ra/Pr))."""
        q = _lib.GlobalQ()
        _lib.check(self._L.afid_global_quantities(self.ctx.h, self.id, C.byref(q)))
        return dict(nu_vol=q.nu_vol, vmax=tuple(q.vmax), tempm=q.tempm, tempmax=q.tempmax,
                    tempmin=q.tempmin, vz_rms=q.vz_rms, vy_rms=q.vy_rms, vx_rms=q.vx_rms,
                    vel_rms=q.vel_rms)

    def calc_stats(self):
        """CalcStats (StatRoutines.F90): add this state's horizontal means to
        the box's profiles."""
        _lib.check(self._L.afid_calc_stats(self.ctx.h, self.id))

    def calc_dissipation_nu(self) -> tuple[float, float]:
        """CalcDissipationNu.F90: (nu_mu, nu_th); adds the dissipation
        profiles to the box's disste and dissth."""
        a, b = C.c_double(), C.c_double()
        _lib.check(self._L.afid_calc_dissipation_nu(self.ctx.h, self.id, C.byref(a), C.byref(b)))
        return a.value, b.value

    def stats(self) -> dict:
        """Accumulated profiles (one array of nxm per name) and nstatsamples."""
        nxm = self.cfg.nxm
        buf = np.zeros(len(_lib.STATS) * nxm)
        n = C.c_int()
        _lib.check(self._L.afid_box_get_stats(self.ctx.h, self.id, _lib.dptr(buf), C.byref(n)))
        out = {name: buf[q * nxm:(q + 1) * nxm].copy() for q, name in enumerate(_lib.STATS)}
        out["nstatsamples"] = n.value
        return out

    def reset_stats(self):
        _lib.check(self._L.afid_box_reset_stats(self.ctx.h, self.id))

    def slab_dump(self, kslab) -> np.ndarray:
        """SlabDumper: for each 1-based plane k of ``kslab``, the slabs
        (vx(k)+vx(k+1))/2, vy(k), vz(k), temp(k); array (n, 4, nym, nzm)."""
        ks = np.ascontiguousarray(kslab, dtype=np.int32)
        c = self.cfg
        buf = np.empty((len(ks), 4, c.nzm, c.nym))
        _lib.check(self._L.afid_slab_dump(self.ctx.h, self.id, ks.ctypes.data_as(C.POINTER(C.c_int)),
                                          len(ks), _lib.dptr(buf)))
        return np.ascontiguousarray(buf.transpose(0, 1, 3, 2))

    def time_marcher_routines(self):
        """One TimeMarcher step (TimeMarcher.F90:24-74) through the
        routine-level entry points, in the reference's call order, with the
        box's current dt."""
        for ns in range(self.cfg.nsst):
            self.time_marcher_begin_substep(ns)
            self.explicit_terms_vx()
            self.explicit_terms_vy()
            self.explicit_terms_vz()
            self.explicit_terms_temp()
            self.implicit_and_update_vx()
            self.implicit_and_update_vy()
            self.implicit_and_update_vz()
            self.implicit_and_update_temp()
            self.calc_local_divergence()
            self.solve_pressure_correction()
            self.correct_velocity()
            self.correct_pressure()
