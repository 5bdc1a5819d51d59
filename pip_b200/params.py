"""Parameter block of the PIP two-fluid step (mirror of ``pip_params`` in include/pip_gpu.h).

``Settings`` reads a PIP ``setting.txt`` the way ``get_parameters`` does
(Model_rot.f90:39-253, lines of the form ``value:key;comment`` split by ``get_word``,
Util_rot.f90:5-12), derives the sizes (Model_rot.f90:254-333) and builds the uniform grid
of ``set_coordinate`` (Model_rot.f90:394-458).  ``Settings.to_params()`` returns the
ctypes structure the C ABI takes.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import List, Tuple

import numpy as np

PIP_ABI_VERSION = 1
PIP_FP64 = 0
PIP_MIXED = 1
PIP_IR_NONE = 0
PIP_IR_JEFFERY = 1              # set_IR type 1 (PIP_rot.f90:135-149)
PIP_IR_POPESCU = 2              # set_IR type 2 (PIP_rot.f90:148-170)
PIP_IR_POPESCU_EQ = 3           # set_IR type 3 (PIP_rot.f90:173-228)
PIP_IR_NLEVEL = 4               # set_IR type 4, the 6-level hydrogen model (PIP_rot.f90:232-311)
PIP_IR_POWERLAW = 5

# boundary codes the C ABI accepts (boundary_control types 1, 2 and 10, and the codes
# MHDbnd/HDbnd map onto type 2, Boundary_rot.f90:62-80)
SUPPORTED_BND = (1, 2, 3, 4, 5, 6, 7, 10, 11)


class PipParams(ctypes.Structure):
    """ctypes mirror of ``struct pip_params`` (field order and types must match)."""

    _fields_ = [
        ("abi_version", ctypes.c_int32),
        ("ndim", ctypes.c_int32),
        ("ix", ctypes.c_int32),
        ("jx", ctypes.c_int32),
        ("kx", ctypes.c_int32),
        ("margin", ctypes.c_int32 * 3),
        ("nvar_h", ctypes.c_int32),
        ("nvar_m", ctypes.c_int32),
        ("flag_sch", ctypes.c_int32),
        ("flag_hll", ctypes.c_int32),
        ("s_order", ctypes.c_int32),
        ("t_order", ctypes.c_int32),
        ("flag_time", ctypes.c_int32),
        ("flag_divb", ctypes.c_int32),
        ("flag_col", ctypes.c_int32),
        ("flag_pip_imp", ctypes.c_int32),
        ("flag_ir", ctypes.c_int32),
        ("flag_ir_type", ctypes.c_int32),
        ("flag_heat", ctypes.c_int32),
        ("hc_max", ctypes.c_int32),
        ("flag_bnd", ctypes.c_int32 * 6),
        ("precision", ctypes.c_int32),
        ("fp_exact", ctypes.c_int32),
        ("flag_resi", ctypes.c_int32),
        ("resi_type", ctypes.c_int32),
        ("reserved_i", ctypes.c_int32 * 4),
        ("gm", ctypes.c_double),
        ("safety", ctypes.c_double),
        ("ro_lim", ctypes.c_double),
        ("pr_lim", ctypes.c_double),
        ("col", ctypes.c_double),
        ("db_clean", ctypes.c_double),
        ("pip_imp_factor", ctypes.c_double),
        ("t_ir", ctypes.c_double),
        ("ir_chi", ctypes.c_double),
        ("ir_ion_coef", ctypes.c_double),
        ("ir_rec_coef", ctypes.c_double),
        ("kapper", ctypes.c_double),
        ("hc_error", ctypes.c_double),
        ("beta", ctypes.c_double),
        ("eta_0", ctypes.c_double),
        ("t_norm", ctypes.c_double),
        ("n_norm", ctypes.c_double),
        ("j_cri", ctypes.c_double),
        ("vd_cri", ctypes.c_double),
        ("reserved_d", ctypes.c_double * 1),
        ("dx", ctypes.POINTER(ctypes.c_double)),
        ("dy", ctypes.POINTER(ctypes.c_double)),
        ("dz", ctypes.POINTER(ctypes.c_double)),
    ]


def get_word(line: str) -> Tuple[str, str]:
    """``get_word`` (Util_rot.f90:5-12): key between ':' and ';', value before ':'."""
    ind_s = line.find(":")
    ind_e = line.find(";")
    if ind_s < 0:
        return "", ""
    key = line[ind_s + 1: ind_e if ind_e >= 0 else len(line)].strip()
    return key, line[:ind_s].strip()


def _fortran_real(text: str) -> float:
    # list-directed read accepts 1.d0 / 1.0e-3 / 0001.d0
    return float(text.strip().lower().replace("d", "e"))


@dataclasses.dataclass
class Settings:
    """The subset of ``globalvar`` the two-fluid step reads, with PIP's defaults."""

    flag_eqs: str = "PIP"
    ndim: int = 1
    ix0: int = 64               # interior cells (setting.txt ``ix``)
    jx0: int = 1
    kx0: int = 1
    gm_d: float = 5.0
    gm_n: float = 3.0
    safety: float = 0.3
    flag_sch: int = 0
    flag_hll: int = 2
    s_order: int = 2
    t_order: int = 2
    flag_time: int = 0
    flag_divb: int = 0
    db_clean: float = 0.7
    ro_lim: float = 1.0e-8
    pr_lim: float = 1.0e-8
    flag_bnd: List[int] = dataclasses.field(default_factory=lambda: [10, 10, 10, 10, 10, 10])
    n_fraction: float = 0.5
    col: float = 100.0
    flag_col: int = 1
    beta: float = 0.1
    flag_pip_imp: int = 0
    pip_imp_factor: float = 10.0
    flag_ir: int = 0
    flag_ir_type: int = 1
    t_ir: float = 1.0
    ir_chi: float = 5.0
    ir_ion_coef: float = 0.0
    ir_rec_coef: float = 0.0
    flag_heat: int = 0
    kapper: float = 0.0
    hc_max: int = 500
    hc_error: float = 1.0e-10
    flag_resi: int = 0          # 10*resi_type + flag (Res_rot.f90:8-15): 1 uniform, 11 localised;
                                # 21/31 anomalous eta set once at the prologue, 22/32 at every stage
    eta_0: float = 0.0
    j_cri: float = 0.0          # resi_type 2 threshold on |curl B|
    vd_cri: float = 0.0         # resi_type 3 threshold on the drift |curl B|/rho_i
    t_norm: float = 0.0         # setting key T_norm (K)
    n_norm: float = 0.0         # setting key n_norm
    # set_IR type 4: nlevels and flag_rad of setting.txt; the convective derivative of the
    # excitation update (1 two-point, 4 five-point, 0 none: the reference's s_order 2 leaves
    # it unset); n0fac, f_p_ini, f_p_p_ini as the initial condition sets them
    n_levels: int = 5
    flag_rad: int = 0
    nlev_deriv: int = 1
    n0fac: float = 1.0
    f_p_ini: float = 1.0
    f_p_p_ini: float = 1.0
    debug_parameter: float = 0.0
    flag_amb: int = 0
    flag_visc: int = 0
    flag_grav: int = 0
    tend: float = -1.0
    precision: int = PIP_FP64
    fp_exact: int = 0
    start: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    end: Tuple[float, float, float] = (1.0, 1.0, 1.0)

    # ---------------------------------------------------------------- derived values
    @property
    def gm(self) -> float:
        return self.gm_d / float(self.gm_n)

    @property
    def margin(self) -> Tuple[int, int, int]:
        """Ghost layers (Model_rot.f90:282-289,319-330), HLL branch."""
        m = self.s_order + min(self.flag_resi, 1) + min(self.flag_amb, 1)
        if self.flag_heat >= 1:
            m += 1
        if self.ndim == 1:
            return (m, 0, 0)
        if self.ndim == 2:
            return (m, m, 0)
        return (m, m, m)

    @property
    def divb(self) -> int:
        return 0 if self.ndim == 1 else self.flag_divb   # Model_rot.f90:309

    @property
    def nvar_m(self) -> int:
        return 8 + (1 if self.divb in (1, 2) else 0)

    @property
    def nvar_h(self) -> int:
        return 5

    @property
    def shape(self) -> Tuple[int, int, int]:
        """(ix, jx, kx) including ghosts (Model_rot.f90:331-333)."""
        m = self.margin
        jx0 = self.jx0 if self.ndim >= 2 else 1
        kx0 = self.kx0 if self.ndim >= 3 else 1
        return (self.ix0 + 2 * m[0], jx0 + 2 * m[1], kx0 + 2 * m[2])

    # ---------------------------------------------------------------- grid
    def coordinates(self):
        """``set_coordinate`` (Model_rot.f90:394-458) for one rank: returns
        (x, y, z, dx, dy, dz) with the cumulative-sum construction of the reference."""
        ix, jx, kx = self.shape
        m = self.margin
        start = list(self.start)
        end = list(self.end)
        if self.ndim <= 2:
            start[2] = 0.0
            end[2] = 0.0
            if self.ndim <= 1:
                start[1] = 0.0
                end[1] = 0.0
        dr = [(end[0] - start[0]) / (ix - 2 * m[0]),
              (end[1] - start[1]) / (jx - 2 * m[1]),
              (end[2] - start[2]) / (kx - 2 * m[2])]
        dx = np.full(ix, dr[0])
        dy = np.full(jx, dr[1])
        dz = np.full(kx, dr[2])
        if self.ndim <= 2:
            dz[0] = 100.0
            if self.ndim <= 1:
                dy[0] = 100.0
        out = []
        for n, (n_cells, d) in enumerate(((ix, dx), (jx, dy), (kx, dz))):
            c = np.zeros(n_cells)
            z0 = m[n]                       # Fortran zeros(n) = margin+1, 0-based margin
            c[z0] = start[n] + 0.5 * dr[n]
            for i in range(z0 + 1, n_cells):
                c[i] = c[i - 1] + d[i - 1]
            for i in range(z0 - 1, -1, -1):
                c[i] = c[i + 1] - d[i]
            out.append(c)
        return out[0], out[1], out[2], dx, dy, dz

    @property
    def resi_type(self) -> int:
        """initialize_resistivity's resi_type = mod(flag_resi/10, 10) (Res_rot.f90:12)."""
        return (self.flag_resi // 10) % 10

    def eta_field(self, U_m: np.ndarray = None) -> np.ndarray:
        """set_resistivity's eta (Res_rot.f90:16-60) as (jx, ix): resi_type 0 eta_0
        everywhere, resi_type 1 eta_0*exp(-((x/0.8)**2 + ((y-debug_parameter)/0.8)**2)),
        resi_type 2 and 3 from |curl B| of the ion state U_m (nvar_m, jx, ix) (get_rotation's
        central differences, zero on the outermost layer): type 2 11 eta_0 where
        |curl B| >= j_cri, else eta_0; type 3 eta_0 (vd/vd_cri - 1)**2 where
        vd = |curl B|/rho_i >= vd_cri, else 0."""
        x, y, _, _, _, _ = self.coordinates()
        ix, jx, _ = self.shape
        if self.resi_type in (2, 3):
            if U_m is None:
                raise ValueError("resi_type %d: eta depends on the state; pass U_m" % self.resi_type)
            _, _, _, dx, dy, _ = self.coordinates()
            bx, by, bz = (np.asarray(U_m[n], dtype=np.float64) for n in (5, 6, 7))
            r1 = np.zeros_like(bx)
            r2 = np.zeros_like(bx)
            r3 = np.zeros_like(bx)
            if self.ndim == 1:
                d2 = (2.0 * dx[1:-1])[None, :]
                r2[:, 1:-1] = -(bz[:, 2:] - bz[:, :-2]) / d2
                r3[:, 1:-1] = (by[:, 2:] - by[:, :-2]) / d2
            else:
                dx2 = (2.0 * dx[1:-1])[None, :]
                dy2 = (2.0 * dy[1:-1])[:, None]
                c = (slice(1, -1), slice(1, -1))
                r1[c] = (bz[2:, 1:-1] - bz[:-2, 1:-1]) / dy2
                r2[c] = -(bz[1:-1, 2:] - bz[1:-1, :-2]) / dx2
                r3[c] = (by[1:-1, 2:] - by[1:-1, :-2]) / dx2 - (bx[2:, 1:-1] - bx[:-2, 1:-1]) / dy2
            c2 = np.sqrt(r1 * r1 + r2 * r2 + r3 * r3)
            if self.resi_type == 2:
                return np.where(c2 >= self.j_cri, self.eta_0 * 11.0, self.eta_0)
            vd = c2 / np.asarray(U_m[0], dtype=np.float64)
            a = vd / self.vd_cri - 1.0
            return np.where(vd >= self.vd_cri, self.eta_0 * (a * a), 0.0)
        if self.resi_type == 1:
            ax = x / 0.8
            ay = (y - self.debug_parameter) / 0.8
            return self.eta_0 * np.exp(-(ax[None, :] * ax[None, :] + ay[:, None] * ay[:, None]))
        return np.full((jx, ix), float(self.eta_0))

    # ---------------------------------------------------------------- checks
    def validate(self) -> None:
        """Raise ValueError for settings outside the supported two-fluid path."""
        bad = []
        if self.flag_eqs != "PIP":
            bad.append("flag_eqs must be PIP (two-fluid)")
        if self.ndim not in (1, 2):
            bad.append("ndim must be 1 or 2")
        if self.flag_sch != 0 or self.flag_hll != 2:
            bad.append("only flag_sch=0, flag_hll=2 (HLLD/HLLC) is supported")
        if self.s_order != 2 or self.t_order != 2 or self.flag_time != 0:
            bad.append("only s_order=2, t_order=2, flag_time=0 is supported")
        if self.flag_col not in range(1, 8):
            bad.append("flag_col must be 1..7 (set_collisional col_type 0..6)")
        elif self.flag_col >= 2 and self.precision != PIP_FP64:
            bad.append("flag_col 2..7 (alpha_c per cell) needs precision PIP_FP64")
        elif self.flag_col in (2, 4, 6) and not self.beta > 0.0:
            bad.append("flag_col %d divides by sqrt(beta*gm/2): beta must be > 0" % self.flag_col)
        if self.flag_resi % 10 not in (0, 1, 2) or self.resi_type not in (0, 1, 2, 3) or \
                self.flag_resi >= 100:
            bad.append("flag_resi must be 10*resi_type + 1 or 2 with resi_type 0..3")
        elif self.flag_resi and (self.precision != PIP_FP64 or self.flag_heat):
            bad.append("resistivity needs precision PIP_FP64 and no conduction")
        elif self.resi_type == 3 and not self.vd_cri > 0.0:
            bad.append("resi_type 3 divides by vd_cri: vd_cri must be > 0")
        if self.flag_amb or self.flag_visc or self.flag_grav:
            bad.append("ambipolar diffusion, viscosity and gravity are not supported")
        set_ir_laws = (PIP_IR_JEFFERY, PIP_IR_POPESCU, PIP_IR_POPESCU_EQ, PIP_IR_NLEVEL)
        if self.flag_ir not in (PIP_IR_NONE, PIP_IR_POWERLAW) + set_ir_laws:
            bad.append("flag_ir must be 0, 1, 2, 3, 4 (set_IR types 1-4) or %d" % PIP_IR_POWERLAW)
        elif self.flag_ir in set_ir_laws:
            if not (self.t_norm > 0.0 and self.n_norm > 0.0):
                bad.append("set_IR types 1-4 need T_norm > 0 and n_norm > 0")
            if self.precision != PIP_FP64:
                bad.append("set_IR types 1-4 need precision PIP_FP64")
        if self.flag_ir == PIP_IR_NLEVEL:
            if self.n_levels != 5:
                bad.append("the 6-level model has nlevels = 5")
            if self.flag_rad not in (0, 1):
                bad.append("flag_rad >= 2 (radiative rates, get_radrat_fixed) is not built")
            if self.nlev_deriv not in (0, 1, 4):
                bad.append("nlev_deriv must be 0, 1 or 4")
            if self.flag_col % 2 == 0 and not self.beta > 0.0:
                bad.append("set_IR type 4 with an even flag_col divides by beta")
        if self.flag_ir and self.flag_ir_type not in (1, 2) and \
                not (self.flag_ir == PIP_IR_NLEVEL and self.flag_ir_type == 0):
            bad.append("flag_ir_type must be 1 or 2 (0 with set_IR type 4)")
        for f in range(2 * self.ndim):
            if self.flag_bnd[f] not in SUPPORTED_BND:
                bad.append("flag_bnd[%d]=%d unsupported" % (f, self.flag_bnd[f]))
        if bad:
            raise ValueError("; ".join(bad))

    # ---------------------------------------------------------------- C struct
    def to_params(self) -> Tuple[PipParams, tuple]:
        """Return (PipParams, keepalive) where keepalive holds the dx/dy/dz buffers."""
        ix, jx, kx = self.shape
        _, _, _, dx, dy, dz = self.coordinates()
        dx = np.ascontiguousarray(dx, dtype=np.float64)
        dy = np.ascontiguousarray(dy, dtype=np.float64)
        dz = np.ascontiguousarray(dz, dtype=np.float64)
        p = PipParams()
        p.abi_version = PIP_ABI_VERSION
        p.ndim = self.ndim
        p.ix, p.jx, p.kx = ix, jx, kx
        for n, m in enumerate(self.margin):
            p.margin[n] = m
        p.nvar_h = self.nvar_h
        p.nvar_m = self.nvar_m
        p.flag_sch = self.flag_sch
        p.flag_hll = self.flag_hll
        p.s_order = self.s_order
        p.t_order = self.t_order
        p.flag_time = self.flag_time
        p.flag_divb = self.divb
        p.flag_col = self.flag_col
        p.flag_pip_imp = self.flag_pip_imp
        p.flag_ir = self.flag_ir
        p.flag_ir_type = self.flag_ir_type
        p.flag_heat = self.flag_heat
        p.hc_max = self.hc_max
        for n in range(6):
            p.flag_bnd[n] = self.flag_bnd[n]
        p.precision = self.precision
        p.fp_exact = self.fp_exact
        p.gm = self.gm
        p.safety = self.safety
        p.ro_lim = self.ro_lim
        p.pr_lim = self.pr_lim
        p.col = self.col
        p.db_clean = self.db_clean
        p.pip_imp_factor = self.pip_imp_factor
        p.t_ir = self.t_ir
        p.ir_chi = self.ir_chi
        p.ir_ion_coef = self.ir_ion_coef
        p.ir_rec_coef = self.ir_rec_coef
        p.kapper = self.kapper
        p.hc_error = self.hc_error
        p.beta = self.beta
        # per-stage eta only where it depends on the state; a per-stage resi_type 0 or 1
        # field is the same at every stage, a fixed field
        flag = self.flag_resi % 10
        p.flag_resi = 2 if (flag == 2 and self.resi_type in (2, 3)) else (1 if flag else 0)
        p.resi_type = self.resi_type
        p.j_cri = self.j_cri
        p.vd_cri = self.vd_cri
        p.eta_0 = self.eta_0
        p.t_norm = self.t_norm
        p.n_norm = self.n_norm
        dptr = ctypes.POINTER(ctypes.c_double)
        p.dx = dx.ctypes.data_as(dptr)
        p.dy = dy.ctypes.data_as(dptr)
        p.dz = dz.ctypes.data_as(dptr)
        return p, (dx, dy, dz)

    # ---------------------------------------------------------------- setting.txt
    @classmethod
    def from_setting_text(cls, text: str) -> "Settings":
        """Parse ``setting.txt`` content like ``get_parameters`` (Model_rot.f90:39-253)."""
        s = cls()
        ints = {"ndim": "ndim", "ix": "ix0", "jx": "jx0", "kx": "kx0",
                "flag_sch": "flag_sch", "s_order": "s_order", "t_order": "t_order",
                "flag_divb": "flag_divb", "flag_pip_imp": "flag_pip_imp",
                "flag_col": "flag_col", "flag_IR": "flag_ir", "flag_IR_type": "flag_ir_type",
                "flag_heat": "flag_heat", "hc_max": "hc_max", "flag_hll": "flag_hll",
                "flag_time": "flag_time", "flag_resi": "flag_resi", "flag_amb": "flag_amb",
                "flag_visc": "flag_visc", "flag_grav": "flag_grav", "nlevels": "n_levels",
                "flag_rad": "flag_rad"}
        reals = {"gm_d": "gm_d", "gm_n": "gm_n", "safety": "safety", "db_clean": "db_clean",
                 "ro_lim": "ro_lim", "pr_lim": "pr_lim", "n_fraction": "n_fraction",
                 "col": "col", "pip_imp_factor": "pip_imp_factor", "t_IR": "t_ir",
                 "kapper": "kapper", "tend": "tend", "beta": "beta", "eta_0": "eta_0",
                 "debug_parameter": "debug_parameter", "T_norm": "t_norm", "n_norm": "n_norm",
                 "j_cri": "j_cri", "vd_cri": "vd_cri"}
        bnd = {"flag_bnd_x_l": 0, "flag_bnd_x_r": 1, "flag_bnd_y_l": 2, "flag_bnd_y_r": 3,
               "flag_bnd_z_l": 4, "flag_bnd_z_r": 5}
        for raw in text.splitlines():
            key, val = get_word(raw)
            if not key:
                continue
            if key == "flag_eqs":
                s.flag_eqs = val.strip()
            elif key in ints:
                setattr(s, ints[key], int(_fortran_real(val)))
            elif key in reals:
                setattr(s, reals[key], _fortran_real(val))
            elif key in bnd:
                s.flag_bnd[bnd[key]] = int(_fortran_real(val))
        return s

    def overrides(self, **kw) -> "Settings":
        return dataclasses.replace(self, **kw)

