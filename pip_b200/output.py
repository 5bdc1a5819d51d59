"""IO_rot's output layout and restart (IO_rot.f90) as raw binary files.

The reference writes, at every output time, one parallel HDF5 file ``outdir/tNNNN.h5``
(``output``, IO_rot.f90:39-105) holding the grid (``xgrid ygrid zgrid dx dy dz``,
``save_coordinates`` :194-203), the scalar ``time`` (``write_time`` :180-192) and the state
in ``save_varfiles`` order (:282-333): ``ro_p mx_p my_p mz_p en_p bx by bz [ps]``, the
ionisation/recombination rates ``ion rec`` when flag_ir >= 1, then ``ro_n mx_n my_n mz_n
en_n`` (names from ``set_initial_out`` :362-374).  Every 3D dataset is FP64 of the global
dimensions with ghost cells, Fortran order (x fastest); each rank writes a hyperslab
(``create_write_dataspaces`` :127-164): its interior, plus its ghost layers on the sides
where it touches the global boundary.  With alpha_c per cell (flag_col 2..7) the file opens
its variables with ``ac``, the field of the last set_collisional, and with resistivity
(flag_resi) with ``et``, the eta field, as ``def_varfiles`` (:231-259) writes them before
the state at every output; restart reads them back (``reread_variables`` :566-572).  ``config.txt`` (``mk_config`` :377-402) records the
setting lines, the equation flags, variable counts, grid, margins, gamma and flag_bnd, and
``restart`` (:405-459) reads them back with the state of output ``flag_restart``.

HDF5 is not in this image, so the files here are the same datasets in the same order as
a raw binary file ``tNNNN.bin`` (little-endian FP64, datasets back to back) with a text
index ``tNNNN.idx`` giving each dataset's name, byte offset and Fortran dimensions -- the
table of contents an HDF5 reader would take from the file.  ``write_output`` writes a whole
state; ``write_output_block`` lets each rank of a decomposed run write its own hyperslab
into the shared file, as the parallel HDF5 writes do.

The time loop with outputs (``main.f90``'s call of ``output`` after each step, with
``get_next_output`` type 0 of IOT_rot.f90:18-41: output n at n*dtout) is
``run_with_output``: the device runs until the next output time, the state is downloaded
(``pip_download``) and written.
"""
from __future__ import annotations

import os
from typing import Dict, Optional, Sequence, Tuple

import numpy as np

from .params import (PIP_IR_JEFFERY, PIP_IR_NLEVEL, PIP_IR_NONE, PIP_IR_POPESCU,
                     PIP_IR_POPESCU_EQ, Settings)

VAR_M = ("ro_p", "mx_p", "my_p", "mz_p", "en_p", "bx", "by", "bz", "ps")
VAR_H = ("ro_n", "mx_n", "my_n", "mz_n", "en_n")
GRID = ("xgrid", "ygrid", "zgrid", "dx", "dy", "dz")


def file_stem(outdir: str, nout: int) -> str:
    return os.path.join(outdir, "t%04d" % nout)


def variables(s: Settings) -> Tuple[str, ...]:
    """The 3D datasets of def_varfiles and save_varfiles, in order."""
    names = ["ac"] if s.flag_col >= 2 else []
    if s.flag_resi:
        names.append("et")
    names += list(VAR_M[: s.nvar_m])
    if s.flag_ir != PIP_IR_NONE:
        names += ["ion", "rec"]
    if s.flag_ir == PIP_IR_NLEVEL:
        # the 6-level model's populations and rates (IO_rot.f90:301-310)
        for i in range(1, 7):
            names.append("nexcite%d" % i)
            names += ["colrat%d%d" % (i, j) for j in range(1, 7)]
        if s.flag_ir_type == 0:
            names.append("ion_loss")
    return tuple(names) + VAR_H


def layout(s: Settings, global_shape: Tuple[int, int, int]):
    """[(name, byte offset, Fortran dims)] of one output file, and its size in bytes."""
    ix, jx, kx = global_shape
    entries = []
    off = 0
    for name, n in zip(GRID, (ix, jx, kx, ix, jx, kx)):
        entries.append((name, off, (n,)))
        off += 8 * n
    entries.append(("time", off, ()))
    off += 8
    for name in variables(s):
        entries.append((name, off, (ix, jx, kx)))
        off += 8 * ix * jx * kx
    return entries, off


def ir_rates(s: Settings, U_m: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Gm_ion, Gm_rec from the ion state: the temperature of get_Te_MHD (get_Pr_MHD's
    pressure with its floor), then PIP_IR_POWERLAW or set_IR type 1, 2 or 3
    (PIP_rot.f90:134-228; the Fortran's single-precision literals rounded to float).  The
    rates are recomputed from the state as written; the run's last set_IR took them from
    the state before the cfl's rewrite, so they agree to round-off."""
    gm = s.gm
    u = U_m
    pr = (gm - 1.0) * (u[4] - 0.5 * ((u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0] +
                                     u[5] * u[5] + u[6] * u[6] + u[7] * u[7]))
    pr = np.maximum(pr, s.pr_lim)
    te = 0.5 * gm * (pr / u[0])
    if s.flag_ir == PIP_IR_JEFFERY:
        T0, n0 = s.t_norm, s.n_norm
        f32 = lambda x: float(np.float32(x))
        factor = np.exp(-13.2 / (T0 / 11605.0))
        f2 = f32(2.7) * (13.2 * 11605.0) ** -2.0 * T0 ** 0.5 * n0
        f3 = f32(5.6e-16) * (13.2 * 11605.0) ** -2.0 * T0 ** -1.0 * n0 ** 2.0
        rec = te ** -0.5 * (u[0] * u[0]) * (f2 / f3) * (f3 / s.t_ir)
        ion = te ** 0.5 * u[0] * factor ** (1.0 / te) * (f3 / s.t_ir)
        return ion, rec
    if s.flag_ir in (PIP_IR_POPESCU, PIP_IR_POPESCU_EQ):
        f32 = lambda x: float(np.float32(x))
        te0 = s.t_norm / f32(1.1604e4)
        n6 = s.n_norm * f32(1.0e6)
        c26, c291 = f32(2.6e-19), f32(2.91e-14)
        if s.flag_ir == PIP_IR_POPESCU:
            a = 13.6 / te0 / te
            rec = u[0] / np.sqrt(te) * (c26 * n6 / np.sqrt(te0) * s.t_ir)
            ion = (n6 * u[0]) * c291 * np.exp(-a) * a ** 0.39 / (0.232 + a) * s.t_ir
            return ion, rec
        ioneq = (c26 / np.sqrt(te0)) / (c291 / (0.232 + 13.6 / te0) * (13.6 / te0) ** 0.39 *
                                         np.exp(-13.6 / te0))
        f_n = ioneq / (ioneq + 1.0)
        f_p = 1.0 - f_n
        f_p_p = 2.0 * f_p / (f_n + 2.0 * f_p)
        tfac = 0.5 * f_p_p / f_p if s.flag_col % 2 == 1 else s.beta / 2.0 * f_p_p * 5.0 / 6.0 / f_p
        b = 13.6 / te0 / te * tfac
        rec = u[0] / np.sqrt(te) * s.t_ir / f_p * np.sqrt(tfac)
        ion = c291 * n6 * u[0] * np.exp(-b) * b ** 0.39 / (0.232 + b) / (c26 * n6 / np.sqrt(te0)) / f_p * s.t_ir
        return ion, rec
    rs = 1.0 / np.sqrt(te)
    return s.ir_ion_coef * rs * np.exp(-s.ir_chi / te), s.ir_rec_coef * rs


def _write_index(stem: str, entries) -> None:
    with open(stem + ".idx", "w") as f:
        for name, off, dims in entries:
            f.write("%s f8 %d %s\n" % (name, off, ",".join(str(d) for d in dims) or "scalar"))


def _create(stem: str, s: Settings, global_shape, time: float, grid) -> Dict[str, Tuple[int, tuple]]:
    entries, size = layout(s, global_shape)
    mm = np.memmap(stem + ".bin", dtype=np.uint8, mode="w+", shape=(size,))
    where = {name: (off, dims) for name, off, dims in entries}
    for name, arr in zip(GRID, grid):
        off, dims = where[name]
        mm[off: off + 8 * dims[0]] = np.ascontiguousarray(arr, dtype="<f8").view(np.uint8)
    off, _ = where["time"]
    mm[off: off + 8] = np.array([time], dtype="<f8").view(np.uint8)
    mm.flush()
    del mm
    _write_index(stem, entries)
    return where


def _state_planes(s: Settings, U_h: np.ndarray, U_m: np.ndarray, ac: Optional[np.ndarray],
                  eta: Optional[np.ndarray] = None, nlevel: Optional[Dict[str, np.ndarray]] = None):
    planes = {}
    if s.flag_col >= 2:
        if ac is None:
            raise ValueError("flag_col %d writes the alpha_c field: pass ac" % s.flag_col)
        planes["ac"] = np.asarray(ac).reshape(U_h.shape[1:])
    if s.flag_resi:
        # resi_type 2 and 3: eta of the written state by default (the reference writes the
        # eta of its last set_resistivity, from the last RK stage's state)
        if eta is None:
            eta = s.eta_field(U_m if s.resi_type in (2, 3) else None)
        planes["et"] = np.asarray(eta).reshape(U_h.shape[1:])
    planes.update({VAR_M[n]: U_m[n] for n in range(s.nvar_m)})
    if s.flag_ir == PIP_IR_NLEVEL:
        if nlevel is None:
            raise ValueError("set_IR type 4 writes its populations and rates: pass nlevel")
        shp = U_h.shape[1:]
        planes["ion"] = np.asarray(nlevel["ion"]).reshape(shp)
        planes["rec"] = np.asarray(nlevel["rec"]).reshape(shp)
        nx = np.asarray(nlevel["nexcite"]).reshape((6,) + shp)
        cr = np.asarray(nlevel["colrat"]).reshape((6, 6) + shp)
        for i in range(6):
            planes["nexcite%d" % (i + 1)] = nx[i]
            for j in range(6):
                planes["colrat%d%d" % (i + 1, j + 1)] = cr[i, j]
        if s.flag_ir_type == 0:
            planes["ion_loss"] = np.asarray(nlevel["ion_loss"]).reshape(shp)
    elif s.flag_ir != PIP_IR_NONE:
        planes["ion"], planes["rec"] = ir_rates(s, U_m)
    for n, name in enumerate(VAR_H):
        planes[name] = U_h[n]
    return planes


def write_output(outdir: str, nout: int, s: Settings, time: float, U_h: np.ndarray,
                 U_m: np.ndarray, ac: Optional[np.ndarray] = None,
                 eta: Optional[np.ndarray] = None,
                 nlevel: Optional[Dict[str, np.ndarray]] = None) -> str:
    """output() of a whole state (global arrays with ghosts, layout (planes, jx, ix)); ac is
    the alpha_c field (pip_get_alpha_c), needed with flag_col 2..7; eta the resistivity
    field (default: the settings' set_resistivity field); nlevel, with set_IR type 4, the
    arrays of nlevel_planes (the rates, Nexcite, colrat, ion_pot)."""
    os.makedirs(outdir, exist_ok=True)
    stem = file_stem(outdir, nout)
    x, y, z, dx, dy, dz = s.coordinates()
    where = _create(stem, s, s.shape, time, (x, y, z, dx, dy, dz))
    mm = np.memmap(stem + ".bin", dtype=np.uint8, mode="r+")
    for name, plane in _state_planes(s, U_h, U_m, ac, eta, nlevel).items():
        off, dims = where[name]
        raw = np.ascontiguousarray(plane, dtype="<f8").view(np.uint8).reshape(-1)
        mm[off: off + raw.size] = raw
    mm.flush()
    del mm
    return stem + ".bin"


def create_output(outdir: str, nout: int, s: Settings, time: float) -> str:
    """Rank 0's part of a decomposed output: the file at full size with grid and time (the
    other ranks then write their hyperslabs with write_output_block)."""
    os.makedirs(outdir, exist_ok=True)
    stem = file_stem(outdir, nout)
    _create(stem, s, s.shape, time, s.coordinates())
    return stem + ".bin"


def write_output_block(outdir: str, nout: int, s: Settings, block, U_h: np.ndarray,
                       U_m: np.ndarray, ac: Optional[np.ndarray] = None,
                       eta: Optional[np.ndarray] = None) -> None:
    """One rank's hyperslab (create_write_dataspaces, IO_rot.f90:127-164) of a decomposed
    output into the file create_output made: the block's interior rows (1D: columns),
    plus its ghost layers on a side where it touches the global boundary.  s is the global
    settings, block the rank's pip_b200.decomp.Block, U_h/U_m its local state."""
    from .decomp import split_axis
    stem = file_stem(outdir, nout)
    entries, _ = layout(s, s.shape)
    ix, jx, _ = s.shape
    ax = split_axis(s)
    m = s.margin[ax]
    lo_local = 0 if block.rank == 0 else m
    hi_local = m + block.n + (m if block.rank == block.world - 1 else 0)
    g0 = block.lo + lo_local                 # first global index written
    mm = np.memmap(stem + ".bin", dtype=np.uint8, mode="r+")
    if s.flag_resi and eta is None:                  # the block's part of the global field
        from .decomp import scatter
        eta = scatter(s, s.eta_field()[None], block.world, block.rank)[0]
    planes = _state_planes(block.settings, U_h, U_m, ac, eta)
    for name, off, dims in entries:
        if name not in planes:
            continue
        P = planes[name]
        if ax == 1:                          # whole rows: one contiguous run per dataset
            part = np.ascontiguousarray(P[lo_local:hi_local, :], dtype="<f8")
            start = off + 8 * g0 * ix
            mm[start: start + part.nbytes] = part.view(np.uint8).reshape(-1)
        else:                                # 1D: a run of columns of the single row
            part = np.ascontiguousarray(P[:, lo_local:hi_local], dtype="<f8")
            start = off + 8 * g0
            mm[start: start + part.nbytes] = part.view(np.uint8).reshape(-1)
    mm.flush()
    del mm


def read_output(path: str) -> Dict[str, np.ndarray]:
    """Every dataset of tNNNN.bin (path with or without the suffix): 1D grids, the scalar
    time, and 3D fields as (kx, jx, ix) arrays (Fortran order read back)."""
    stem = path[:-4] if path.endswith(".bin") else path
    raw = np.fromfile(stem + ".bin", dtype="<f8")
    out = {}
    with open(stem + ".idx") as f:
        for line in f:
            name, _, off, dims = line.split()
            off = int(off) // 8
            if dims == "scalar":
                out[name] = float(raw[off])
                continue
            d = tuple(int(v) for v in dims.split(","))
            n = int(np.prod(d))
            out[name] = raw[off: off + n].reshape(d[::-1]).copy()
    return out


def mk_config(outdir: str, s: Settings, setting_text: str = "",
              mpi_siz: Optional[Sequence[int]] = None) -> str:
    """config.txt of mk_config (IO_rot.f90:377-402): the setting lines as key:value up to
    ENDSETTING, then the flags, counts, the writing rank's grid (s: the settings of that
    rank's block), margins, gamma and flag_bnd (and the MPI domain size of a decomposed
    run)."""
    os.makedirs(outdir, exist_ok=True)
    from .params import get_word
    lines = []
    for raw in setting_text.splitlines():
        key, value = get_word(raw)
        if key and value:
            lines.append("%s:%s" % (key, value))
    lines.append("ENDSETTING")
    lines.append(" %d %d  #mhd and pip flag" % (1, 1))
    lines.append(" %d %d  #number of variables" % (s.nvar_h, s.nvar_m))
    lines.append(" %d %d %d  # used grid numbers" % s.shape)
    lines.append(" %d %d %d  # used margin grid numbers" % s.margin)
    lines.append(" %r #Abiabatic constant" % s.gm)
    lines.append(" " + " ".join(str(int(b)) for b in s.flag_bnd))
    if mpi_siz is not None:
        lines.append(" " + " ".join(str(int(v)) for v in mpi_siz) + " #mpi domain size")
    path = os.path.join(outdir, "config.txt")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


def read_config(outdir: str) -> Dict[str, object]:
    """restart's reading of config.txt (IO_rot.f90:405-441): the values after ENDSETTING."""
    with open(os.path.join(outdir, "config.txt")) as f:
        lines = f.read().splitlines()
    k = lines.index("ENDSETTING")
    nums = lambda ln: ln.split("#")[0].split()
    flag_mhd, flag_pip = (int(v) for v in nums(lines[k + 1]))
    nvar_h, nvar_m = (int(v) for v in nums(lines[k + 2]))
    shape = tuple(int(v) for v in nums(lines[k + 3]))
    margin = tuple(int(v) for v in nums(lines[k + 4]))
    gm = float(nums(lines[k + 5])[0])
    flag_bnd = [int(v) for v in nums(lines[k + 6])]
    return dict(flag_mhd=flag_mhd, flag_pip=flag_pip, nvar_h=nvar_h, nvar_m=nvar_m, shape=shape,
                margin=margin, gm=gm, flag_bnd=flag_bnd)


def restart(outdir: str, nout: int, s: Settings) -> Tuple[float, np.ndarray, np.ndarray]:
    """restart (IO_rot.f90:405-459): checks config.txt against the settings and returns
    (time, U_h, U_m) of output nout, global arrays (planes, jx, ix) with ghosts."""
    cfg = read_config(outdir)
    # like the reference, the grid line (the writing rank's block) is not compared
    if (cfg["nvar_h"], cfg["nvar_m"]) != (s.nvar_h, s.nvar_m) or tuple(cfg["margin"]) != s.margin \
            or cfg["flag_bnd"] != list(s.flag_bnd) or cfg["gm"] != s.gm:
        raise ValueError("config.txt of %s does not match the settings" % outdir)
    d = read_output(file_stem(outdir, nout))
    ix, jx, _ = s.shape
    if d[VAR_H[0]].shape != (1, jx, ix):
        raise ValueError("output %d of %s has dimensions %s, the settings %s"
                         % (nout, outdir, d[VAR_H[0]].shape[::-1], s.shape))
    U_m = np.stack([d[VAR_M[n]][0] for n in range(s.nvar_m)]).reshape(s.nvar_m, jx, ix)
    U_h = np.stack([d[v][0] for v in VAR_H]).reshape(5, jx, ix)
    return d["time"], np.ascontiguousarray(U_h), np.ascontiguousarray(U_m)


def restart_resistivity(outdir: str, nout: int, s: Settings) -> Optional[np.ndarray]:
    """The eta field of output nout (jx, ix) that restart reads with flag_resi (IO_rot.f90:
    566-568), for pip_set_resistivity; None without resistivity."""
    if not s.flag_resi:
        return None
    d = read_output(file_stem(outdir, nout))
    ix, jx, _ = s.shape
    return np.ascontiguousarray(d["et"][0].reshape(jx, ix))


def nlevel_planes(ctx, s: Settings) -> Optional[Dict[str, np.ndarray]]:
    """The 6-level model's output arrays from a context (set_IR type 4): the rates of the last
    set_IR, Nexcite, colrat and ion_pot; None for the other laws."""
    if s.flag_ir != PIP_IR_NLEVEL:
        return None
    ion, rec = ctx.ir_rates()
    out = dict(ion=ion, rec=rec, nexcite=ctx.nexcite(), colrat=ctx.colrat())
    if s.flag_ir_type == 0:
        out["ion_loss"] = ctx.ion_pot()
    return out


def restart_nexcite(outdir: str, nout: int, s: Settings) -> Optional[np.ndarray]:
    """Nexcite (6, jx, ix) of output nout, for pip_set_nexcite (set_IR type 4); None for the
    other laws.  The reference's restart does not read the populations back
    (reread_variables, IO_rot.f90:574-581); this completes it."""
    if s.flag_ir != PIP_IR_NLEVEL:
        return None
    d = read_output(file_stem(outdir, nout))
    ix, jx, _ = s.shape
    return np.ascontiguousarray(np.stack([d["nexcite%d" % i][0].reshape(jx, ix)
                                          for i in range(1, 7)]))


def restart_alpha_c(outdir: str, nout: int, s: Settings) -> Optional[np.ndarray]:
    """The alpha_c field of output nout (jx, ix) that restart reads with flag_col 2..7
    (IO_rot.f90:570-572), for pip_set_alpha_c; None for a constant alpha_c."""
    if s.flag_col < 2:
        return None
    d = read_output(file_stem(outdir, nout))
    ix, jx, _ = s.shape
    return np.ascontiguousarray(d["ac"][0].reshape(jx, ix))


def run_with_output(ctx, s: Settings, outdir: str, dtout: float, tend: float,
                    nout0: int = 0, setting_text: str = "") -> Tuple[int, int, float]:
    """main.f90's loop with output (IO_rot.f90:39-105; get_next_output type 0: output n at
    time n*dtout): writes config.txt and output nout0 of the current state, then runs the
    device loop (pip_run) to each next output time, downloads the state and writes it,
    until tend.  Returns (status, last output number, time)."""
    if nout0 == 0:
        mk_config(outdir, s, setting_text)
    nout = nout0
    field = (lambda: ctx.alpha_c()) if s.flag_col >= 2 else (lambda: None)
    U_h, U_m = ctx.download()
    write_output(outdir, nout, s, ctx.time, U_h, U_m, field(), nlevel=nlevel_planes(ctx, s))
    st = 0
    while ctx.time < tend:
        nxt = min((nout + 1) * dtout, tend)
        st, t, n = ctx.run(t_end=nxt)
        U_h, U_m = ctx.download()
        nout += 1
        write_output(outdir, nout, s, t, U_h, U_m, field(), nlevel=nlevel_planes(ctx, s))
        if st != 0:
            break
    return st, nout, ctx.time
