"""ctypes binding of the C ABI (include/pip_gpu.h) in pip_b200/libpipgpu.so.

This is the reference-facing surface in Python form: the same calls the Fortran driver
makes through an ISO_C_BINDING interface module.  There is no CPU fallback: if the CUDA
library is missing or no GPU is visible the calls raise.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Tuple

import numpy as np

from .params import PipParams, Settings

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpipgpu.so")

PIP_OK = 0
PIP_ERR_PARAM = 1
PIP_ERR_CUDA = 2
PIP_ERR_NAN = 3
PIP_ERR_DT = 4
PIP_ERR_ITER = 5
PIP_ERR_STATE = 6
PIP_ERR_NOMEM = 7
PIP_ERR_NULL = 8
PIP_ERR_RATE = 9

# every extern "C" symbol include/pip_gpu.h declares
EXPORTS = (
    "pip_ctx_create", "pip_ctx_destroy", "pip_upload", "pip_download", "pip_cfl", "pip_step",
    "pip_run", "pip_set_time", "pip_get_time", "pip_flux", "pip_source", "pip_fill_ghosts",
    "pip_status", "pip_conduction", "pip_last_cuda_error", "pip_strerror",
    "pip_step_noalloc", "pip_set_neighbors", "pip_stage", "pip_halo_bytes", "pip_halo_pack",
    "pip_halo_unpack", "pip_ctx_stream", "pip_set_cmax_scale", "pip_dev_begin", "pip_dev_stage",
    "pip_dev_stage_split", "pip_set_halo_stream",
    "pip_dev_candidates", "pip_dev_poll", "pip_coefficients", "pip_get_alpha_c",
    "pip_set_alpha_c", "pip_set_resistivity", "pip_set_hc_wait_limit", "pip_set_hc_loop",
    "pip_resi_dt",
    "pip_colexp_table", "pip_set_nlevel", "pip_set_nexcite", "pip_get_nexcite",
    "pip_get_colrat", "pip_get_ion_pot", "pip_nlevel_gm_rec_ref", "pip_get_ir_rates",
    "pip_hcd_begin", "pip_hcd_phase", "pip_hcd_row_bytes", "pip_hcd_pack", "pip_hcd_unpack",
    "pip_hcd_end",
    # include/pip_bench.h
    "pip_run_timed", "pip_bench_stage_ms", "pip_kernels_per_run", "pip_conduction_iterations",
    # include/pip_ensemble.h
    "pip_ensemble_create", "pip_ensemble_destroy", "pip_ensemble_upload", "pip_ensemble_run",
    "pip_ensemble_member", "pip_ensemble_set_config", "pip_ensemble_tune",
    "pip_ensemble_timings", "pip_ensemble_slots", "pip_ensemble_blocks",
    "pip_ensemble_set_cluster", "pip_ensemble_plan",
    # include/pip_adjoint.h
    "pip_adj_create", "pip_adj_destroy", "pip_adj_set_col", "pip_adj_forward",
    "pip_adj_backward", "pip_adj_dt", "pip_adj_stage_vjp", "pip_adj_fold",
)

_lib = None


class PipError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        msg = "%s failed: %s (%d)" % (where, strerror(code), code)
        if code == PIP_ERR_CUDA:
            msg += ", cudaError %d" % lib().pip_last_cuda_error()
        super().__init__(msg)


def lib(path: Optional[str] = None):
    """Load libpipgpu.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise RuntimeError("libpipgpu.so is missing: run `python -m pip_b200.build` "
                           "(or __graft_entry__.build()) first")
    L = ctypes.CDLL(path)
    P = ctypes.POINTER
    d = ctypes.c_double
    dp = P(d)
    vp = ctypes.c_void_p
    i = ctypes.c_int
    L.pip_ctx_create.argtypes = [P(PipParams), P(vp)]
    L.pip_ctx_create.restype = i
    L.pip_ctx_destroy.argtypes = [vp]
    L.pip_ctx_destroy.restype = None
    L.pip_upload.argtypes = [vp, dp, dp]
    L.pip_download.argtypes = [vp, dp, dp]
    L.pip_cfl.argtypes = [vp, dp, dp]
    L.pip_step.argtypes = [vp, d]
    L.pip_run.argtypes = [vp, ctypes.c_int64, d, dp, P(ctypes.c_int64)]
    L.pip_set_time.argtypes = [vp, d]
    L.pip_get_time.argtypes = [vp, dp]
    L.pip_flux.argtypes = [vp, i, dp, dp]
    L.pip_source.argtypes = [vp, d, dp, dp]
    L.pip_fill_ghosts.argtypes = [vp]
    L.pip_coefficients.argtypes = [vp]
    L.pip_get_alpha_c.argtypes = [vp, dp]
    L.pip_set_alpha_c.argtypes = [vp, dp]
    L.pip_set_resistivity.argtypes = [vp, dp]
    L.pip_resi_dt.argtypes = [vp, dp]
    L.pip_status.argtypes = [vp, P(i), P(i)]
    L.pip_conduction.argtypes = [vp, d, P(i), dp]
    L.pip_set_hc_wait_limit.argtypes = [vp, i]
    L.pip_set_hc_loop.argtypes = [vp, i]
    L.pip_step_noalloc.argtypes = [P(PipParams), vp, d, d, vp]
    L.pip_set_neighbors.argtypes = [vp, P(i)]
    L.pip_stage.argtypes = [vp, i, d, d]
    L.pip_halo_bytes.argtypes = [vp, i]
    L.pip_halo_bytes.restype = ctypes.c_int64
    L.pip_halo_pack.argtypes = [vp, i, vp, P(ctypes.c_int64)]
    L.pip_halo_unpack.argtypes = [vp, i, vp, ctypes.c_int64]
    L.pip_ctx_stream.argtypes = [vp, P(vp)]
    L.pip_set_cmax_scale.argtypes = [vp, d]
    L.pip_dev_begin.argtypes = [vp, ctypes.c_int64, d]
    L.pip_dev_stage.argtypes = [vp, i]
    L.pip_dev_stage_split.argtypes = [vp, i, P(vp)]
    L.pip_set_halo_stream.argtypes = [vp, vp]
    L.pip_dev_candidates.argtypes = [vp, P(vp), P(vp)]
    L.pip_dev_poll.argtypes = [vp, P(i), dp, P(ctypes.c_int64)]
    L.pip_step_noalloc.restype = i
    L.pip_colexp_table.argtypes = [ctypes.c_int64, dp]
    L.pip_set_nlevel.argtypes = [vp, P(PipNlevel), dp, ctypes.c_int64]
    L.pip_set_nexcite.argtypes = [vp, dp]
    L.pip_get_nexcite.argtypes = [vp, dp]
    L.pip_get_colrat.argtypes = [vp, dp]
    L.pip_get_ion_pot.argtypes = [vp, dp]
    L.pip_nlevel_gm_rec_ref.argtypes = [vp, dp]
    L.pip_get_ir_rates.argtypes = [vp, dp, dp]
    L.pip_hcd_begin.argtypes = [vp, d, dp]
    L.pip_hcd_phase.argtypes = [vp, i, dp, dp]
    L.pip_hcd_row_bytes.argtypes = [vp]
    L.pip_hcd_row_bytes.restype = ctypes.c_int64
    L.pip_hcd_pack.argtypes = [vp, i, i, vp]
    L.pip_hcd_unpack.argtypes = [vp, i, i, vp]
    L.pip_hcd_end.argtypes = [vp, i]
    for name in ("pip_hcd_begin", "pip_hcd_phase", "pip_hcd_pack", "pip_hcd_unpack", "pip_hcd_end"):
        getattr(L, name).restype = i
    for name in ("pip_colexp_table", "pip_set_nlevel", "pip_set_nexcite", "pip_get_nexcite",
                 "pip_get_colrat", "pip_get_ion_pot", "pip_nlevel_gm_rec_ref",
                 "pip_get_ir_rates"):
        getattr(L, name).restype = i
    L.pip_last_cuda_error.argtypes = []
    L.pip_strerror.argtypes = [i]
    L.pip_strerror.restype = ctypes.c_char_p
    # measurement hooks (include/pip_bench.h)
    L.pip_run_timed.argtypes = [vp, ctypes.c_int64, d, dp, P(ctypes.c_int64), P(ctypes.c_float)]
    L.pip_bench_stage_ms.argtypes = [vp, i, P(ctypes.c_float), P(ctypes.c_float), P(ctypes.c_float)]
    L.pip_kernels_per_run.argtypes = [vp, ctypes.c_int64]
    L.pip_conduction_iterations.argtypes = [vp]
    L.pip_conduction_iterations.restype = ctypes.c_int64
    # batched ensembles (include/pip_ensemble.h)
    L.pip_ensemble_create.argtypes = [P(PipParams), i, P(vp)]
    L.pip_ensemble_destroy.argtypes = [vp]
    L.pip_ensemble_destroy.restype = None
    L.pip_ensemble_upload.argtypes = [vp, i, dp, dp]
    L.pip_ensemble_run.argtypes = [vp, d, ctypes.c_int64, P(ctypes.c_float)]
    L.pip_ensemble_member.argtypes = [vp, i, dp, dp, dp, P(ctypes.c_int64), P(i)]
    L.pip_ensemble_set_config.argtypes = [vp, i, i]
    L.pip_ensemble_tune.argtypes = [vp, d, P(i), P(i), P(ctypes.c_float)]
    L.pip_ensemble_timings.argtypes = [vp, dp, dp]
    L.pip_ensemble_slots.argtypes = [vp, P(i)]
    L.pip_ensemble_blocks.argtypes = [vp, P(i)]
    L.pip_ensemble_set_cluster.argtypes = [vp, i, d]
    L.pip_ensemble_plan.argtypes = [vp, P(i), P(i), P(i)]
    L.pip_adj_create.argtypes = [P(PipParams), ctypes.c_int64, i, P(vp)]
    L.pip_adj_destroy.argtypes = [vp]
    L.pip_adj_destroy.restype = None
    L.pip_adj_set_col.argtypes = [vp, d]
    L.pip_adj_forward.argtypes = [vp, vp, vp, ctypes.c_int64, P(ctypes.c_float)]
    L.pip_adj_backward.argtypes = [vp, vp, vp, dp, P(ctypes.c_float)]
    L.pip_adj_dt.argtypes = [vp, dp, ctypes.c_int64, P(ctypes.c_int64)]
    L.pip_adj_stage_vjp.argtypes = [vp, i, vp, vp, vp, d, dp, dp]
    L.pip_adj_fold.argtypes = [vp, vp]
    for name in ("pip_ensemble_create", "pip_ensemble_upload", "pip_ensemble_run",
                 "pip_ensemble_member", "pip_ensemble_set_config", "pip_ensemble_tune",
                 "pip_ensemble_timings", "pip_ensemble_slots", "pip_ensemble_blocks",
                 "pip_ensemble_set_cluster", "pip_ensemble_plan"):
        getattr(L, name).restype = i
    L.pip_kernels_per_run.restype = ctypes.c_int64
    for name in ("pip_upload", "pip_download", "pip_cfl", "pip_step", "pip_run", "pip_set_time",
                 "pip_get_time", "pip_flux", "pip_source", "pip_fill_ghosts", "pip_status",
                 "pip_conduction", "pip_last_cuda_error", "pip_run_timed", "pip_bench_stage_ms",
                 "pip_coefficients", "pip_get_alpha_c", "pip_set_alpha_c",
                 "pip_set_resistivity"):
        getattr(L, name).restype = i
    _lib = L
    return L


def strerror(code: int) -> str:
    return lib().pip_strerror(int(code)).decode()


class PipNlevel(ctypes.Structure):
    """ctypes mirror of ``struct pip_nlevel`` (set_IR type 4's settings)."""

    _fields_ = [
        ("n_levels", ctypes.c_int32),
        ("flag_rad", ctypes.c_int32),
        ("deriv", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("n0fac", ctypes.c_double),
        ("f_p_ini", ctypes.c_double),
        ("f_p_p_ini", ctypes.c_double),
    ]


def colexp_table(nsamps: int = 100000) -> np.ndarray:
    """expintcalc/colexp.dat's table as expintread holds it, shape (nsamps+1, 4): rows
    (yn, E0(yn), E1(yn), E2(yn)) by the algorithm of expintcalc/colexpintcalc.f90."""
    t = np.empty((int(nsamps) + 1, 4))
    _check(lib().pip_colexp_table(int(nsamps), _ptr(t)), "pip_colexp_table")
    return t


def _ptr(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise TypeError("arrays must be C-contiguous float64 (Fortran U(ix,jx,kx,nvar) order)")
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _check(code: int, where: str) -> int:
    if code != PIP_OK:
        raise PipError(code, where)
    return code


class Context:
    """One device-resident two-fluid simulation (a ``pip_ctx``).

    Method names follow the Fortran routines they replace: ``cfl`` (Scheme_rot.f90:183),
    ``run_solver`` (Solver_rot.f90:42), ``set_flux`` (:124), ``source_pip``
    (PIP_rot.f90:1309), ``pipbnd`` (Boundary_rot.f90:34).
    """

    def __init__(self, s: Settings):
        self.s = s
        self.params, self._keep = s.to_params()
        h = ctypes.c_void_p()
        _check(lib().pip_ctx_create(ctypes.byref(self.params), ctypes.byref(h)), "pip_ctx_create")
        self.h = h
        ix, jx, _ = s.shape
        self.shape_h = (s.nvar_h, jx, ix)
        self.shape_m = (s.nvar_m, jx, ix)

    def close(self) -> None:
        if getattr(self, "h", None) is not None and self.h.value:
            lib().pip_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------ state
    def upload(self, U_h: np.ndarray, U_m: np.ndarray) -> None:
        U_h = np.ascontiguousarray(U_h, dtype=np.float64)
        U_m = np.ascontiguousarray(U_m, dtype=np.float64)
        if U_h.shape != self.shape_h or U_m.shape != self.shape_m:
            raise ValueError("state shapes %s/%s, expected %s/%s"
                             % (U_h.shape, U_m.shape, self.shape_h, self.shape_m))
        _check(lib().pip_upload(self.h, _ptr(U_h), _ptr(U_m)), "pip_upload")

    def download(self, out_h: Optional[np.ndarray] = None,
                 out_m: Optional[np.ndarray] = None) -> Tuple[np.ndarray, np.ndarray]:
        U_h = out_h if out_h is not None else np.empty(self.shape_h)
        U_m = out_m if out_m is not None else np.empty(self.shape_m)
        _check(lib().pip_download(self.h, _ptr(U_h), _ptr(U_m)), "pip_download")
        return U_h, U_m

    # ------------------------------------------------------------------ the step
    def cfl(self) -> Tuple[float, float]:
        dt = ctypes.c_double()
        cm = ctypes.c_double()
        _check(lib().pip_cfl(self.h, ctypes.byref(dt), ctypes.byref(cm)), "pip_cfl")
        return dt.value, cm.value

    def run_solver(self, dt: float) -> None:
        _check(lib().pip_step(self.h, float(dt)), "pip_step")

    def run(self, nsteps: int = 0, t_end: float = 0.0, check: bool = True) -> Tuple[int, float, int]:
        """Time loop on the device; returns (status, time, steps)."""
        t = ctypes.c_double()
        n = ctypes.c_int64()
        st = lib().pip_run(self.h, int(nsteps), float(t_end), ctypes.byref(t), ctypes.byref(n))
        if check and st not in (PIP_OK, PIP_ERR_NAN, PIP_ERR_DT):
            raise PipError(st, "pip_run")
        return st, t.value, n.value

    def conduction(self, dt: float) -> Tuple[int, int, float]:
        """HC(U_m,nvar_m,1) over dt (flag_heat = 1 contexts): (status, iterations, relative
        residual); status PIP_OK or PIP_ERR_ITER."""
        it = ctypes.c_int()
        rr = ctypes.c_double()
        st = lib().pip_conduction(self.h, float(dt), ctypes.byref(it), ctypes.byref(rr))
        if st not in (PIP_OK, PIP_ERR_ITER):
            raise PipError(st, "pip_conduction")
        return st, it.value, rr.value

    def set_hc_wait_limit(self, polls: int) -> None:
        """Polls of the BiCGstab staging waits from the next solve on (< 0: the default)."""
        _check(lib().pip_set_hc_wait_limit(self.h, int(polls)), "pip_set_hc_wait_limit")

    def set_hc_loop(self, device_loop: bool) -> None:
        """BiCGstab iterations as one device-side loop (True, the default) or in host-checked
        groups (False)."""
        _check(lib().pip_set_hc_loop(self.h, 1 if device_loop else 0), "pip_set_hc_loop")

    @property
    def conduction_iterations(self) -> int:
        return int(lib().pip_conduction_iterations(self.h))

    @property
    def time(self) -> float:
        t = ctypes.c_double()
        _check(lib().pip_get_time(self.h, ctypes.byref(t)), "pip_get_time")
        return t.value

    @time.setter
    def time(self, t: float) -> None:
        _check(lib().pip_set_time(self.h, float(t)), "pip_set_time")

    # ------------------------------------------------------------------ unit entry points
    def set_flux(self, direction: int) -> Tuple[np.ndarray, np.ndarray]:
        F_h = np.empty(self.shape_h)
        F_m = np.empty(self.shape_m)
        _check(lib().pip_flux(self.h, int(direction), _ptr(F_h), _ptr(F_m)), "pip_flux")
        return F_h, F_m

    def source_pip(self, dt_coll: float) -> Tuple[np.ndarray, np.ndarray]:
        S_h = np.empty(self.shape_h)
        S_m = np.empty(self.shape_m)
        _check(lib().pip_source(self.h, float(dt_coll), _ptr(S_h), _ptr(S_m)), "pip_source")
        return S_h, S_m

    def pipbnd(self) -> None:
        _check(lib().pip_fill_ghosts(self.h), "pip_fill_ghosts")

    def coefficients(self) -> None:
        """set_coefficients' collision part (flag_col 2..7: energies rewritten, alpha_c set)."""
        _check(lib().pip_coefficients(self.h), "pip_coefficients")

    def alpha_c(self) -> np.ndarray:
        """alpha_c of every cell, shaped like one plane of the state."""
        a = np.empty(self.shape_h[1:])
        _check(lib().pip_get_alpha_c(self.h, _ptr(a)), "pip_get_alpha_c")
        return a

    def set_resistivity(self, eta: np.ndarray) -> None:
        """The eta field (jx, ix) of flag_resi 1 (set_resistivity; eta_0 everywhere until set)."""
        e = np.ascontiguousarray(eta, dtype=np.float64).reshape(self.shape_h[1:])
        _check(lib().pip_set_resistivity(self.h, _ptr(e)), "pip_set_resistivity")

    def resi_dt(self) -> float:
        """cfl_resi's bound of the current eta (pip_resi_dt)."""
        b = ctypes.c_double()
        _check(lib().pip_resi_dt(self.h, ctypes.byref(b)), "pip_resi_dt")
        return b.value

    def set_alpha_c(self, ac: np.ndarray) -> None:
        """The field of a restart output (its "ac" dataset) for the next cfl."""
        a = np.ascontiguousarray(ac, dtype=np.float64).reshape(self.shape_h[1:])
        _check(lib().pip_set_alpha_c(self.h, _ptr(a)), "pip_set_alpha_c")

    # ------------------------------------------------------------------ domain decomposition
    def set_neighbors(self, neighbor) -> None:
        """set_mpi_neighbor (MPI_rot.f90:90-126): rank across faces x-, x+, y-, y+ or -1."""
        nb = (ctypes.c_int * 4)(*[int(v) for v in neighbor])
        _check(lib().pip_set_neighbors(self.h, nb), "pip_set_neighbors")

    def stage(self, stage: int, dt: float, cmax: float) -> None:
        """One RK stage of run_solver (Solver_rot.f90:59-71)."""
        _check(lib().pip_stage(self.h, int(stage), float(dt), float(cmax)), "pip_stage")

    @property
    def stream(self) -> int:
        """The context's cudaStream_t (pip_ctx_stream), as an integer handle."""
        h = ctypes.c_void_p()
        _check(lib().pip_ctx_stream(self.h, ctypes.byref(h)), "pip_ctx_stream")
        return int(h.value or 0)

    def set_cmax_scale(self, sg: float) -> None:
        _check(lib().pip_set_cmax_scale(self.h, float(sg)), "pip_set_cmax_scale")

    def dev_begin(self, nsteps: int = 0, t_end: float = 0.0) -> None:
        _check(lib().pip_dev_begin(self.h, int(nsteps), float(t_end)), "pip_dev_begin")

    def dev_stage(self, stage: int) -> None:
        _check(lib().pip_dev_stage(self.h, int(stage)), "pip_dev_stage")

    def dev_stage_split(self, stage: int) -> int:
        """A device stage with its boundary tile rows on a high-priority stream of the
        context, concurrent with the middle rows; returns that stream (an int handle)."""
        bs = ctypes.c_void_p()
        _check(lib().pip_dev_stage_split(self.h, int(stage), ctypes.byref(bs)),
               "pip_dev_stage_split")
        return bs.value or 0

    def set_halo_stream(self, stream: int) -> None:
        """The stream of pip_halo_pack / pip_halo_unpack (0: the context stream)."""
        _check(lib().pip_set_halo_stream(self.h, ctypes.c_void_p(stream or None)),
               "pip_set_halo_stream")

    def dev_candidates(self) -> Tuple[int, int]:
        """Device addresses of the cfl candidates: (2 int64 to MIN, 4 int64 to MAX)."""
        a, b = ctypes.c_void_p(), ctypes.c_void_p()
        _check(lib().pip_dev_candidates(self.h, ctypes.byref(a), ctypes.byref(b)),
               "pip_dev_candidates")
        return int(a.value), int(b.value)

    def dev_poll(self) -> Tuple[int, int, float, int]:
        """(status, done, time, steps) of the device-driven loop, after waiting for it."""
        done = ctypes.c_int()
        t = ctypes.c_double()
        n = ctypes.c_int64()
        st = lib().pip_dev_poll(self.h, ctypes.byref(done), ctypes.byref(t), ctypes.byref(n))
        if st not in (PIP_OK, PIP_ERR_NAN, PIP_ERR_DT):
            raise PipError(st, "pip_dev_poll")
        return st, done.value, t.value, n.value

    def halo_bytes(self, face: int) -> int:
        return int(lib().pip_halo_bytes(self.h, int(face)))

    def halo_pack(self, face: int, send_ptr: int) -> int:
        """mpi_bnd's send side of face f into device memory at send_ptr (queued on the
        context stream); returns the message length in bytes."""
        n = ctypes.c_int64()
        _check(lib().pip_halo_pack(self.h, int(face), ctypes.c_void_p(send_ptr), ctypes.byref(n)),
               "pip_halo_pack")
        return n.value

    def halo_unpack(self, face: int, recv_ptr: int, nbytes: int) -> None:
        """mpi_bnd's receive side: the message at recv_ptr into the ghost layers of face f
        (queued on the context stream)."""
        _check(lib().pip_halo_unpack(self.h, int(face), ctypes.c_void_p(recv_ptr), int(nbytes)),
               "pip_halo_unpack")

    def status(self) -> Tuple[int, int]:
        stop = ctypes.c_int()
        nan = ctypes.c_int()
        _check(lib().pip_status(self.h, ctypes.byref(stop), ctypes.byref(nan)), "pip_status")
        return stop.value, nan.value

    # ---- set_IR type 4 (the 6-level hydrogen model)
    def set_nlevel(self, table: np.ndarray, **override) -> None:
        """The exponential-integral table (rows yn, E0, E1, E2) and the model's settings:
        n_levels, flag_rad, deriv (the settings' nlev_deriv), n0fac, f_p_ini, f_p_p_ini from
        the context's Settings unless given."""
        t = np.ascontiguousarray(table, dtype=np.float64)
        if t.ndim != 2 or t.shape[1] != 4:
            raise ValueError("the table has rows of 4 values (yn, E0, E1, E2)")
        s = self.s
        v = dict(n_levels=s.n_levels, flag_rad=s.flag_rad, deriv=s.nlev_deriv, n0fac=s.n0fac,
                 f_p_ini=s.f_p_ini, f_p_p_ini=s.f_p_p_ini)
        unknown = set(override) - set(v)
        if unknown:
            raise TypeError("unknown settings %s" % sorted(unknown))
        v.update(override)
        cfg = PipNlevel(int(v["n_levels"]), int(v["flag_rad"]), int(v["deriv"]), 0,
                        float(v["n0fac"]), float(v["f_p_ini"]), float(v["f_p_p_ini"]))
        _check(lib().pip_set_nlevel(self.h, ctypes.byref(cfg), _ptr(t), t.shape[0]),
               "pip_set_nlevel")

    def set_nexcite(self, nex: np.ndarray) -> None:
        """Nexcite, shape (6, jx, ix): levels 1-5 then the ions."""
        n = np.ascontiguousarray(nex, dtype=np.float64).reshape((6,) + self.shape_h[1:])
        _check(lib().pip_set_nexcite(self.h, _ptr(n)), "pip_set_nexcite")

    def nexcite(self) -> np.ndarray:
        n = np.empty((6,) + self.shape_h[1:])
        _check(lib().pip_get_nexcite(self.h, _ptr(n)), "pip_get_nexcite")
        return n

    def colrat(self) -> np.ndarray:
        """colrat of the last set_IR as [a, b] = colrat(a+1, b+1), shape (6, 6, jx, ix)."""
        c = np.empty((6, 6) + self.shape_h[1:])
        _check(lib().pip_get_colrat(self.h, _ptr(c)), "pip_get_colrat")
        return np.ascontiguousarray(c.transpose(1, 0, 2, 3))

    def ion_pot(self) -> np.ndarray:
        a = np.empty(self.shape_h[1:])
        _check(lib().pip_get_ion_pot(self.h, _ptr(a)), "pip_get_ion_pot")
        return a

    def ir_rates(self) -> Tuple[np.ndarray, np.ndarray]:
        """(Gm_ion, Gm_rec) of the last set_IR, each shaped like one plane (set_IR types 1, 4)."""
        ion = np.empty(self.shape_h[1:])
        rec = np.empty(self.shape_h[1:])
        _check(lib().pip_get_ir_rates(self.h, _ptr(ion), _ptr(rec)), "pip_get_ir_rates")
        return ion, rec

    # ---- conduction of a decomposed run (BiCGstabMPI in phases, pip_hcd_*)
    def hcd_begin(self, dt: float) -> Tuple[float, float]:
        s = (ctypes.c_double * 2)()
        _check(lib().pip_hcd_begin(self.h, float(dt), s), "pip_hcd_begin")
        return s[0], s[1]

    def hcd_phase(self, phase: int, c0: float = 0.0, c1: float = 0.0) -> Tuple[float, float]:
        coef = (ctypes.c_double * 2)(float(c0), float(c1))
        s = (ctypes.c_double * 2)()
        _check(lib().pip_hcd_phase(self.h, int(phase), coef, s), "pip_hcd_phase")
        return s[0], s[1]

    def hcd_row_bytes(self) -> int:
        return int(lib().pip_hcd_row_bytes(self.h))

    def hcd_pack(self, vec: int, face: int, send_ptr: int) -> None:
        _check(lib().pip_hcd_pack(self.h, int(vec), int(face), ctypes.c_void_p(send_ptr)),
               "pip_hcd_pack")

    def hcd_unpack(self, vec: int, face: int, recv_ptr: int) -> None:
        _check(lib().pip_hcd_unpack(self.h, int(vec), int(face), ctypes.c_void_p(recv_ptr)),
               "pip_hcd_unpack")

    def hcd_end(self, iters: int) -> None:
        _check(lib().pip_hcd_end(self.h, int(iters)), "pip_hcd_end")

    def gm_rec_ref(self) -> float:
        v = ctypes.c_double()
        _check(lib().pip_nlevel_gm_rec_ref(self.h, ctypes.byref(v)), "pip_nlevel_gm_rec_ref")
        return v.value

    def prologue(self) -> None:
        """The prologue's cfl and ghost fill (Initial_rot.f90:152-160)."""
        self.cfl()
        self.pipbnd()

    # ------------------------------------------------------------------ measurement hooks
    def run_timed(self, nsteps: int = 0, t_end: float = 0.0) -> Tuple[int, float, int, float]:
        """pip_run plus the device time of the loop (ms, CUDA events on the context stream)."""
        t = ctypes.c_double()
        n = ctypes.c_int64()
        ms = ctypes.c_float()
        st = lib().pip_run_timed(self.h, int(nsteps), float(t_end), ctypes.byref(t),
                                 ctypes.byref(n), ctypes.byref(ms))
        if st not in (PIP_OK, PIP_ERR_NAN, PIP_ERR_DT):
            raise PipError(st, "pip_run_timed")
        return st, t.value, n.value, ms.value

    def stage_ms(self, nsteps: int) -> Tuple[float, float, float]:
        """Mean device time of one stage-1 launch, one stage-2 launch and one step (ms)."""
        a, b, c = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        _check(lib().pip_bench_stage_ms(self.h, int(nsteps), ctypes.byref(a), ctypes.byref(b),
                                        ctypes.byref(c)), "pip_bench_stage_ms")
        return a.value, b.value, c.value

    def kernels_per_run(self, nsteps: int) -> int:
        return int(lib().pip_kernels_per_run(self.h, int(nsteps)))
