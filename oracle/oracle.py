"""ctypes wrapper of the FP64 CPU restatement (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` as the checker
and by bench.py's CPU-baseline leg.  The product package never imports it.

Parity status: unpinned by the reference's own tests (the reference ships none and cannot
be built here); see pip_oracle.h.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional, Tuple

import numpy as np

from pip_b200.params import PipParams, Settings

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile."""
    src = os.path.join(_HERE, "pip_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.POINTER
        d = ctypes.c_double
        dp = P(d)
        vp = ctypes.c_void_p
        L.orc_create.argtypes = [P(PipParams), P(ctypes.c_int)]
        L.orc_create.restype = vp
        L.orc_destroy.argtypes = [vp]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_get_threads.restype = ctypes.c_int
        L.orc_set_state.argtypes = [vp, dp, dp]
        L.orc_get_state.argtypes = [vp, dp, dp]
        L.orc_set_time.argtypes = [vp, d]
        L.orc_get_time.argtypes = [vp]
        L.orc_get_time.restype = d
        L.orc_get_cmax.argtypes = [vp]
        L.orc_get_cmax.restype = d
        L.orc_set_cmax.argtypes = [vp, d]
        L.orc_cfl.argtypes = [vp, dp, dp]
        L.orc_run_solver.argtypes = [vp, d]
        L.orc_stage.argtypes = [vp, ctypes.c_int, d]
        L.orc_set_neighbors.argtypes = [vp, P(ctypes.c_int)]
        L.orc_flux.argtypes = [vp, ctypes.c_int, dp, dp]
        L.orc_source.argtypes = [vp, d, dp, dp]
        L.orc_bnd.argtypes = [vp]
        L.orc_run.argtypes = [vp, ctypes.c_long, d, dp, P(ctypes.c_long), dp, ctypes.c_long]
        L.orc_run.restype = ctypes.c_int
        L.orc_has_nan.argtypes = [vp]
        L.orc_conduction.argtypes = [vp, d, P(ctypes.c_int), dp]
        L.orc_conduction.restype = ctypes.c_int
        L.orc_has_nan.restype = ctypes.c_int
        L.orc_coefficients.argtypes = [vp]
        L.orc_set_resistivity.argtypes = [vp, dp]
        L.orc_resistivity.argtypes = [vp, dp]
        L.orc_resistivity.restype = None
        L.orc_ir_rates.argtypes = [vp, dp, dp]
        L.orc_alpha_c.argtypes = [vp, dp]
        L.orc_alpha_c.restype = ctypes.c_int
        L.orc_expint_table.argtypes = [ctypes.c_long, dp]
        L.orc_expint_table.restype = None
        L.orc_set_nlevel.argtypes = [vp, ctypes.c_int, d, d, d, dp, ctypes.c_long]
        L.orc_set_nlevel.restype = ctypes.c_int
        L.orc_set_nexcite.argtypes = [vp, dp]
        L.orc_get_nexcite.argtypes = [vp, dp]
        L.orc_get_colrat.argtypes = [vp, dp]
        L.orc_get_ion_pot.argtypes = [vp, dp]
        L.orc_gm_rec_ref.argtypes = [vp]
        L.orc_gm_rec_ref.restype = d
        L.orc_nlevel_status.argtypes = [vp]
        L.orc_nlevel_status.restype = ctypes.c_int
        L.orc_hcd_begin.argtypes = [vp, d, dp]
        L.orc_hcd_begin.restype = ctypes.c_int
        L.orc_hcd_phase.argtypes = [vp, ctypes.c_int, dp, dp]
        L.orc_hcd_phase.restype = ctypes.c_int
        L.orc_hcd_get_row.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
        L.orc_hcd_set_row.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
        L.orc_hcd_end.argtypes = [vp]
        L.orc_hcd_end.restype = ctypes.c_int
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def expint_table(nsamps: int = 100000) -> np.ndarray:
    """colexpintcalc.f90's exponential-integral table, shape (nsamps+1, 4): yn, E0, E1, E2."""
    t = np.empty((nsamps + 1, 4))
    lib().orc_expint_table(int(nsamps), _ptr(t))
    return t


class Oracle:
    """One simulation on the CPU restatement; mirrors the C ABI's call set."""

    def __init__(self, s: Settings, U_h: np.ndarray, U_m: np.ndarray):
        self.s = s
        self.params, self._keep = s.to_params()
        st = ctypes.c_int(0)
        self.h = lib().orc_create(ctypes.byref(self.params), ctypes.byref(st))
        if not self.h:
            raise ValueError("oracle rejected the parameters (status %d)" % st.value)
        self.shape_h = U_h.shape
        self.shape_m = U_m.shape
        self.set_state(U_h, U_m)

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, U_h, U_m):
        U_h = np.ascontiguousarray(U_h, dtype=np.float64)
        U_m = np.ascontiguousarray(U_m, dtype=np.float64)
        lib().orc_set_state(self.h, _ptr(U_h), _ptr(U_m))

    def state(self) -> Tuple[np.ndarray, np.ndarray]:
        U_h = np.empty(self.shape_h)
        U_m = np.empty(self.shape_m)
        lib().orc_get_state(self.h, _ptr(U_h), _ptr(U_m))
        return U_h, U_m

    @property
    def time(self) -> float:
        return lib().orc_get_time(self.h)

    @time.setter
    def time(self, t: float):
        lib().orc_set_time(self.h, float(t))

    @property
    def cmax(self) -> float:
        return lib().orc_get_cmax(self.h)

    @cmax.setter
    def cmax(self, v: float):
        lib().orc_set_cmax(self.h, float(v))

    def cfl(self) -> Tuple[float, float]:
        dt = ctypes.c_double()
        cm = ctypes.c_double()
        lib().orc_cfl(self.h, ctypes.byref(dt), ctypes.byref(cm))
        return dt.value, cm.value

    def run_solver(self, dt: float) -> None:
        lib().orc_run_solver(self.h, float(dt))

    def stage(self, istep: int, dt: float) -> None:
        """One stage of run_solver with the stage's PIPbnd (physical faces only)."""
        lib().orc_stage(self.h, int(istep), float(dt))

    def set_neighbors(self, neighbor) -> None:
        """set_mpi_neighbor: faces with a neighbouring rank are left to the halo exchange."""
        nb = (ctypes.c_int * 4)(*[int(v) for v in neighbor])
        lib().orc_set_neighbors(self.h, nb)

    def flux(self, direction: int):
        F_h = np.zeros(self.shape_h)
        F_m = np.zeros(self.shape_m)
        lib().orc_flux(self.h, int(direction), _ptr(F_h), _ptr(F_m))
        return F_h, F_m

    def source(self, dt_coll: float):
        S_h = np.zeros(self.shape_h)
        S_m = np.zeros(self.shape_m)
        lib().orc_source(self.h, float(dt_coll), _ptr(S_h), _ptr(S_m))
        return S_h, S_m

    def conduction(self, dt: float):
        """HC(U_m,nvar_m,1) over dt; returns (status, iterations, relative residual)."""
        it = ctypes.c_int()
        rr = ctypes.c_double()
        st = lib().orc_conduction(self.h, float(dt), ctypes.byref(it), ctypes.byref(rr))
        return st, it.value, rr.value

    def fill_ghosts(self) -> None:
        lib().orc_bnd(self.h)

    def coefficients(self) -> None:
        """set_coefficients' collision part: flag_col 2..7 rewrites the energies, sets alpha_c."""
        lib().orc_coefficients(self.h)

    def set_resistivity(self, eta: np.ndarray) -> None:
        """The eta field (jx, ix) of flag_resi 1 (eta_0 everywhere until set)."""
        e = np.ascontiguousarray(eta, dtype=np.float64).reshape(self.shape_h[1:])
        lib().orc_set_resistivity(self.h, _ptr(e))

    def resistivity(self) -> np.ndarray:
        """The current eta field (jx, ix)."""
        e = np.empty(self.shape_h[1:])
        lib().orc_resistivity(self.h, _ptr(e))
        return e

    def ir_rates(self):
        """(Gm_ion, Gm_rec) of the last set_IR, each shaped like one plane."""
        ion = np.empty(self.shape_h[1:])
        rec = np.empty(self.shape_h[1:])
        lib().orc_ir_rates(self.h, _ptr(ion), _ptr(rec))
        return ion, rec

    def alpha_c(self) -> np.ndarray:
        """alpha_c of every cell, shaped like one plane of the state."""
        a = np.empty(self.shape_h[1:])
        lib().orc_alpha_c(self.h, _ptr(a))
        return a

    def prologue(self) -> None:
        """The prologue's cfl and ghost fill (Initial_rot.f90:152-160)."""
        dt, cm = self.cfl()
        self.cmax = cm
        self.fill_ghosts()

    def run(self, nsteps: int = 0, t_end: float = 0.0, max_hist: int = 0):
        t = ctypes.c_double()
        n = ctypes.c_long()
        hist = np.zeros(max(max_hist, 1))
        status = lib().orc_run(self.h, int(nsteps), float(t_end), ctypes.byref(t), ctypes.byref(n),
                               _ptr(hist), int(max_hist))
        return status, t.value, n.value, hist[: min(n.value, max_hist)]

    def has_nan(self) -> bool:
        return bool(lib().orc_has_nan(self.h))

    # ---- BiCGstabMPI in phases (orc_hcd_*): vector 0 x, 1 r, 2 Ap
    def hcd_begin(self, dt: float):
        s = (ctypes.c_double * 2)()
        lib().orc_hcd_begin(self.h, float(dt), s)
        return s[0], s[1]

    def hcd_phase(self, phase: int, c0: float = 0.0, c1: float = 0.0):
        coef = (ctypes.c_double * 2)(float(c0), float(c1))
        s = (ctypes.c_double * 2)()
        if lib().orc_hcd_phase(self.h, int(phase), coef, s):
            raise ValueError("phase %d" % phase)
        return s[0], s[1]

    def hcd_get_row(self, vec: int, row: int) -> np.ndarray:
        out = np.empty(self.shape_h[2])
        lib().orc_hcd_get_row(self.h, int(vec), int(row), _ptr(out))
        return out

    def hcd_set_row(self, vec: int, row: int, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        lib().orc_hcd_set_row(self.h, int(vec), int(row), _ptr(v))

    def hcd_end(self) -> None:
        lib().orc_hcd_end(self.h)

    # ---- set_IR type 4 (the 6-level hydrogen model)
    def set_nlevel(self, table: np.ndarray, deriv: int = 1, n0fac: float = 1.0,
                   f_p_ini: float = 1.0, f_p_p_ini: float = 1.0) -> None:
        """expinttab (rows yn, E0, E1, E2) and the model's settings."""
        t = np.ascontiguousarray(table, dtype=np.float64)
        st = lib().orc_set_nlevel(self.h, int(deriv), float(n0fac), float(f_p_ini),
                                  float(f_p_p_ini), _ptr(t), int(t.shape[0]))
        if st:
            raise ValueError("orc_set_nlevel rejected the settings (%d)" % st)

    def set_nexcite(self, nex: np.ndarray) -> None:
        """Nexcite, shape (6, jx, ix): levels 1-5 then the ions."""
        n = np.ascontiguousarray(nex, dtype=np.float64).reshape((6,) + self.shape_h[1:])
        lib().orc_set_nexcite(self.h, _ptr(n))

    def nexcite(self) -> np.ndarray:
        n = np.empty((6,) + self.shape_h[1:])
        lib().orc_get_nexcite(self.h, _ptr(n))
        return n

    def colrat(self) -> np.ndarray:
        """colrat of the last set_IR as [a, b] = colrat(a+1, b+1), shape (6, 6, jx, ix)."""
        c = np.empty((6, 6) + self.shape_h[1:])
        lib().orc_get_colrat(self.h, _ptr(c))
        return np.ascontiguousarray(c.transpose(1, 0, 2, 3))

    def ion_pot(self) -> np.ndarray:
        a = np.empty(self.shape_h[1:])
        lib().orc_get_ion_pot(self.h, _ptr(a))
        return a

    @property
    def gm_rec_ref(self) -> float:
        return lib().orc_gm_rec_ref(self.h)

    @property
    def nlevel_status(self) -> int:
        return lib().orc_nlevel_status(self.h)


def run_case(s: Settings, U_h, U_m, nsteps: int = 0, t_end: Optional[float] = None,
             threads: int = 1, max_hist: int = 0):
    """prologue + time loop; returns (status, time, steps, U_h, U_m, dt_hist)."""
    set_threads(threads)
    o = Oracle(s, U_h, U_m)
    o.prologue()
    status, t, n, hist = o.run(nsteps, t_end if t_end is not None else 0.0, max_hist)
    Uh, Um = o.state()
    o.close()
    return status, t, n, Uh, Um, hist
