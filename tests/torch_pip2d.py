"""Differentiable torch restatement of the 2D two-fluid FP64 step (test infrastructure).

A third transcription of main.f90:31-68 / run_solver (Solver_rot.f90:42-81) for the case
the discrete adjoint supports (flag_sch=0, flag_hll=2, s_order=2, t_order=2, ndim=2,
flag_divb=0, explicit collisions flag_pip_imp=0, no IR), ndim 1 or 2, written with
whole-array torch operations in float64 so that ``torch.autograd`` gives an FP64 reference
gradient of a short run.  Branches (minmod, HLLD fan regions, HLLC-G fallback, min/max of
wave speeds, floors, the CFL minimum) are explicit ``torch.where`` selections with the tie
rules of the hand-written adjoint it checks (minmod slope 0 when min(|X|, sign(X) Y) <= 0,
else X when |X| <= sign(X) Y; the left operand of a min/max on a tie; the first cell of a
CFL minimum), so that autograd differentiates the same branch even on a kink (ties are exact
at reflecting and outflow boundaries and wherever two limited slopes coincide).  Expressions follow the literal Fortran forms (HLL_rot.f90,
Scheme_rot.f90, PIP_rot.f90) like the C oracle.

State: tensor (13, jx, ix) -- ion planes ro, mx, my, mz, en, bx, by, bz then neutral planes
ro, mx, my, mz, en; margin 2 (jx = 1 in 1D).  Boundary codes 1, 2 and 10.
"""
import torch

TINY = 1e-20
EPSI = 1e-10
ACC = 1.03
HLLG = 1.001
MU_P, MU_N = 0.5, 1.0
NVM = 8
M = 2  # margin


def _sgn1(x):
    return torch.copysign(torch.ones_like(x), x)


def _min(a, b):
    """min with the left operand on a tie."""
    return torch.where(a <= b, a, b)


def _max(a, b):
    """max with the left operand on a tie."""
    return torch.where(a >= b, a, b)


def u2v_mhd(U, gm, ro_lim, pr_lim):                       # HLL_rot.f90:1159-1186
    ro = torch.clamp(U[0], min=ro_lim)
    roi = 1.0 / ro
    pr = (gm - 1.0) * (U[4] - 0.5 * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) * roi
                       - 0.5 * (U[5] * U[5] + U[6] * U[6] + U[7] * U[7]))
    pr = torch.where(pr < pr_lim, torch.full_like(pr, pr_lim), pr)
    return torch.stack([ro, U[1] * roi, U[2] * roi, U[3] * roi, pr, U[5], U[6], U[7]])


def u2v_hd(U, gm, ro_lim, pr_lim):                        # HLL_rot.f90:1136-1156
    ro = torch.clamp(U[0], min=ro_lim)
    roi = 1.0 / ro
    pr = (gm - 1.0) * (U[4] - 0.5 * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) * roi)
    pr = torch.where(pr < pr_lim, torch.full_like(pr, pr_lim), pr)
    return torch.stack([ro, U[1] * roi, U[2] * roi, U[3] * roi, pr])


def face_states(V, ro_lim):
    """get_Side + minmod_func (Util_rot.f90:59-76) along the last axis: left and right states
    of the faces between cells f and f+1 for f = 1 .. n-3."""
    X = V[..., 2:] - V[..., 1:-1]
    Y = V[..., 1:-1] - V[..., :-2]
    SX = _sgn1(X)
    m = torch.minimum(torch.abs(X), SX * Y)
    du = torch.where(m > 0.0, torch.where(torch.abs(X) <= SX * Y, X, Y), torch.zeros_like(X))
    VLs = V[..., 1:-1] + 0.5 * du     # VL at cells 1 .. n-2
    VRs = V[..., 1:-1] - 0.5 * du     # VR at faces 0 .. n-3
    L = VLs[..., :-1]
    R = VRs[..., 1:]
    L = torch.cat([torch.clamp(L[:1], min=ro_lim), L[1:]], dim=0)
    R = torch.cat([torch.clamp(R[:1], min=ro_lim), R[1:]], dim=0)
    return L, R


def hllc(vl, vr, gm):                                     # HLL_rot.f90:615-687
    gm1 = gm - 1.0

    def cons(v):
        return torch.stack([v[0], v[0] * v[1], v[0] * v[2], v[0] * v[3],
                            v[4] / gm1 + 0.5 * v[0] * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3])])
    ul, ur = cons(vl), cons(vr)
    prl, prr = vl[4], vr[4]

    def phys(u, pr):
        return torch.stack([u[1], pr + u[1] * u[1] / u[0], u[1] * u[2] / u[0], u[1] * u[3] / u[0],
                            u[1] * (u[4] + pr) / u[0]])
    fl, fr = phys(ul, prl), phys(ur, prr)
    csl = torch.sqrt(gm * prl / ul[0])
    csr = torch.sqrt(gm * prr / ur[0])
    vnl = ul[1] / ul[0]
    vnr = ur[1] / ur[0]
    sl = ACC * _min(vnl - csl, vnr - csr)
    sr = ACC * _max(vnl + csl, vnr + csr)
    sm = ((ur[1] * (sr - vnr) - ul[1] * (sl - vnl) + prl - prr) /
          (ur[0] * (sr - vnr) - ul[0] * (sl - vnl)))
    prm = sm * ul[0] * (sl - vnl) - ul[1] * (sl - vnl) + prl
    stl0 = ul[0] * (sl - vnl) / (sl - sm)
    str0 = ur[0] * (sr - vnr) / (sr - sm)
    stl = torch.stack([stl0, stl0 * sm, stl0 * ul[2] / ul[0], stl0 * ul[3] / ul[0],
                       ((sl - vnl) * ul[4] - prl * vnl + prm * sm) / (sl - sm)])
    st_r = torch.stack([str0, str0 * sm, str0 * ur[2] / ur[0], str0 * ur[3] / ur[0],
                        ((sr - vnr) * ur[4] - prr * vnr + prm * sm) / (sr - sm)])

    def th(s):
        # (|s| + s) / max(2 s, 1e-10) as a selection: the same values, and a gradient without
        # the 1e10-scaled terms that cancel in the quotient form
        return torch.where(s >= 0.5 * EPSI, torch.ones_like(s),
                           torch.where(s > 0.0, 2.0 * s / EPSI, torch.zeros_like(s)))
    thl, thm = th(sl), th(sm)
    thr = 1.0 - th(sr)
    return (thr * fr + thl * fl + (1.0 - thl - thr) *
            (thm * (fl + sl * (stl - ul)) + (1.0 - thm) * (fr + sr * (st_r - ur))))


def hlld(vl, vr, gm):                                     # HLL_rot.f90:691-910, 8 variables
    gm1 = gm - 1.0
    el = (vl[4] / gm1 + 0.5 * vl[0] * (vl[1] ** 2 + vl[2] ** 2 + vl[3] ** 2)
          + 0.5 * (vl[5] ** 2 + vl[6] ** 2 + vl[7] ** 2))
    er = (vr[4] / gm1 + 0.5 * vr[0] * (vr[1] ** 2 + vr[2] ** 2 + vr[3] ** 2)
          + 0.5 * (vr[5] ** 2 + vr[6] ** 2 + vr[7] ** 2))
    ul = torch.stack([vl[0], vl[0] * vl[1], vl[0] * vl[2], vl[0] * vl[3], el, vl[5], vl[6], vl[7]])
    ur = torch.stack([vr[0], vr[0] * vr[1], vr[0] * vr[2], vr[0] * vr[3], er, vr[5], vr[6], vr[7]])

    def phys(v, u):
        b2 = v[5] * v[5] + v[6] * v[6] + v[7] * v[7]
        pt = v[4] + 0.5 * b2
        vb = v[1] * v[5] + v[2] * v[6] + v[3] * v[7]
        f = torch.stack([v[0] * v[1], v[0] * (v[1] * v[1]) + v[4] + 0.5 * b2 - v[5] * v[5],
                         v[0] * v[1] * v[2] - v[5] * v[6], v[0] * v[1] * v[3] - v[5] * v[7],
                         (u[4] + pt) * v[1] - vb * v[5], torch.zeros_like(v[0]),
                         v[1] * v[6] - v[5] * v[2], v[1] * v[7] - v[5] * v[3]])
        return f, b2, pt, vb
    fl, b2l, ptl, vbl = phys(vl, ul)
    fr, b2r, ptr, vbr = phys(vr, ur)

    def vfast(v, b2):
        f1 = gm * v[4]
        f2 = 4.0 * f1 * (v[5] * v[5])
        disc = (f1 + b2) * (f1 + b2) - f2
        disc = torch.where(disc > 0.0, disc, torch.zeros_like(disc))
        dd = torch.where(disc > 0.0, torch.sqrt(torch.where(disc > 0.0, disc, torch.ones_like(disc))),
                         torch.zeros_like(disc))
        return torch.sqrt(((f1 + b2) + dd) / (2.0 * v[0]))
    vf = _max(vfast(vl, b2l), vfast(vr, b2r))
    sl = _min(vl[1], vr[1]) - vf
    sr = _max(vl[1], vr[1]) + vf
    f1 = 1.0 / (sr - sl)
    uh = f1 * (sr * ur - sl * ul - fr + fl)
    sm = uh[1] / uh[0]
    pt = ptl + vl[0] * (sl - vl[1]) * (sm - vl[1])
    ro_l1 = vl[0] * (sl - vl[1]) / (sl - sm)
    ro_r1 = vr[0] * (sr - vr[1]) / (sr - sm)
    bn = uh[5]
    sal = torch.abs(bn) / torch.sqrt(ro_l1)
    sar = torch.abs(bn) / torch.sqrt(ro_r1)

    # HLLC-G (HLL_rot.f90:776-807)
    vy2g = uh[2] / uh[0]
    vz2g = uh[3] / uh[0]

    def hllg_side(v, u, f, S, ro1, pts, vb):
        e2 = ((S - v[1]) * u[4] - pts * v[1] + pt * sm +
              bn * (vb - sm * bn - vy2g * uh[6] - vz2g * uh[7])) / (S - sm)
        st = torch.stack([ro1, ro1 * sm, ro1 * vy2g, ro1 * vz2g, e2, uh[5], uh[6], uh[7]])
        return S * (st - u) + f
    out_gl = hllg_side(vl, ul, fl, sl, ro_l1, ptl, vbl)
    out_gr = hllg_side(vr, ur, fr, sr, ro_r1, ptr, vbr)

    # single-star states (HLL_rot.f90:813-843)
    def star(v, u, S, ro1, pts, vb):
        f = 1.0 / (v[0] * (S - v[1]) * (S - sm) - uh[5] * uh[5])
        u6 = v[6] * f * (v[0] * ((S - v[1]) * (S - v[1])) - uh[5] * uh[5])
        u7 = v[7] * f * (v[0] * ((S - v[1]) * (S - v[1])) - uh[5] * uh[5])
        vy1 = v[2] - f * uh[5] * v[6] * (sm - v[1])
        vz1 = v[3] - f * uh[5] * v[7] * (sm - v[1])
        e1 = ((S - v[1]) * u[4] - pts * v[1] + pt * sm +
              uh[5] * (vb - sm * uh[5] - vy1 * u6 - vz1 * u7)) / (S - sm)
        return torch.stack([ro1, ro1 * sm, ro1 * vy1, ro1 * vz1, e1, uh[5], u6, u7]), vy1, vz1
    ul1, vy_l1, vz_l1 = star(vl, ul, sl, ro_l1, ptl, vbl)
    ur1, vy_r1, vz_r1 = star(vr, ur, sr, ro_r1, ptr, vbr)
    sl1 = sm - sal
    sr1 = sm + sar
    out_ls = sl * (ul1 - ul) + fl
    out_rs = sr * (ur1 - ur) + fr

    # central states (HLL_rot.f90:861-898)
    ro_ls = torch.sqrt(ro_l1)
    ro_rs = torch.sqrt(ro_r1)
    fc = 1.0 / (ro_ls + ro_rs)
    f2 = _sgn1(uh[5])
    vy2 = fc * (ro_ls * vy_l1 + ro_rs * vy_r1 + (ur1[6] - ul1[6]) * f2)
    vz2 = fc * (ro_ls * vz_l1 + ro_rs * vz_r1 + (ur1[7] - ul1[7]) * f2)
    u26 = fc * (ro_ls * ur1[6] + ro_rs * ul1[6] + ro_ls * ro_rs * (vy_r1 - vy_l1) * f2)
    u27 = fc * (ro_ls * ur1[7] + ro_rs * ul1[7] + ro_ls * ro_rs * (vz_r1 - vz_l1) * f2)
    e2l = ul1[4] - ro_ls * (vy_l1 * ul1[6] + vz_l1 * ul1[7] - vy2 * u26 - vz2 * u27) * f2
    e2r = ur1[4] + ro_rs * (vy_r1 * ur1[6] + vz_r1 * ur1[7] - vy2 * u26 - vz2 * u27) * f2
    u2l = torch.stack([ro_l1, ro_l1 * sm, ro_l1 * vy2, ro_l1 * vz2, e2l, uh[5], u26, u27])
    u2r = torch.stack([ro_r1, ro_r1 * sm, ro_r1 * vy2, ro_r1 * vz2, e2r, uh[5], u26, u27])
    out_lss = sl1 * u2l - (sl1 - sl) * ul1 - sl * ul + fl
    out_rss = sr1 * u2r - (sr1 - sr) * ur1 - sr * ur + fr

    hllg = (sl >= (sm - HLLG * sal)) | ((sm + HLLG * sar) >= sr)
    pos = sm >= 0.0
    hlld_out = torch.where(sl1 >= 0.0, out_ls,
                           torch.where(sr1 <= 0.0, out_rs, torch.where(pos, out_lss, out_rss)))
    fan = torch.where(hllg, torch.where(pos, out_gl, out_gr), hlld_out)
    return torch.where(sl >= 0.0, fl, torch.where(sr <= 0.0, fr, fan))


PERM_M_Y = [0, 2, 1, 3, 4, 6, 5, 7]
PERM_H_Y = [0, 2, 1, 3, 4]


class Geom:
    """Grid and boundary description of a run: ndim, margin, boundary codes (1 periodic,
    2 reflecting, 10 outflow; Boundary_rot.f90:323-402 with set_sym_mhd/hd :239-320) and the
    cell widths."""

    def __init__(self, s):
        self.ndim = s.ndim
        self.flag_bnd = list(s.flag_bnd)
        _, _, _, dx, dy, _ = s.coordinates()
        self.dx = torch.from_numpy(dx)
        self.dy = torch.from_numpy(dy)
        self.gm, self.safety, self.ro_lim, self.pr_lim = s.gm, s.safety, s.ro_lim, s.pr_lim

    def sl(self):
        """Interior slice of a (13, jx, ix) array."""
        return (slice(None), slice(M, -M) if self.ndim == 2 else slice(None), slice(M, -M))


def _ghost_sources(code, n, upper):
    """0-based source index of each ghost layer (lower: layers 0..M-1, upper: n-M..n-1)."""
    if code == 1:
        return [n - 2 * M + l for l in range(M)] if not upper else [M + l for l in range(M)]
    if code == 2:
        return [2 * M - 1 - l for l in range(M)] if not upper else [n - M - 1 - l for l in range(M)]
    if code == 10:
        return [M] * M if not upper else [n - M - 1] * M
    raise ValueError("boundary code %d not covered" % code)


def _sym(code, direction):
    """Per-plane signs of the ghost copies (13 planes) for a face of the given direction."""
    sg = [1.0] * 13
    if code == 2:
        sg[direction] = -1.0            # normal momentum (ions)
        sg[4 + direction] = -1.0        # normal field
        sg[NVM + direction] = -1.0      # normal momentum (neutrals)
    return torch.tensor(sg, dtype=torch.float64)


def fill(Ui, g):
    """PIPbnd: ghost cells of the interior array Ui (13, ny, nx) -- x faces, then y faces
    (whole rows, so corners take both copies)."""
    n = Ui.shape[2] + 2 * M
    U = torch.cat([Ui[:, :, :M], Ui, Ui[:, :, :M]], dim=2)      # placeholder ghost columns
    lo = _ghost_sources(g.flag_bnd[0], n, False)
    hi = _ghost_sources(g.flag_bnd[1], n, True)
    U = torch.cat([_sym(g.flag_bnd[0], 1)[:, None, None] * U[:, :, lo],
                   U[:, :, M:n - M],
                   _sym(g.flag_bnd[1], 1)[:, None, None] * U[:, :, hi]], dim=2)
    if g.ndim == 1:
        return U
    m = U.shape[1] + 2 * M
    U = torch.cat([U[:, :M], U, U[:, :M]], dim=1)
    lo = _ghost_sources(g.flag_bnd[2], m, False)
    hi = _ghost_sources(g.flag_bnd[3], m, True)
    return torch.cat([_sym(g.flag_bnd[2], 2)[:, None, None] * U[:, lo, :],
                      U[:, M:m - M, :],
                      _sym(g.flag_bnd[3], 2)[:, None, None] * U[:, hi, :]], dim=1)


def fill_periodic(Ui):
    """Ghost cells by periodic copy (flag_bnd = 1): x first, then y."""
    U = torch.cat([Ui[:, :, -M:], Ui, Ui[:, :, :M]], dim=2)
    return torch.cat([U[:, -M:, :], U, U[:, :M, :]], dim=1)


def fluxes(U, g):
    """x and y face fluxes adjacent to interior cells: Fx (13, ny, ix-3), Fy (13, jx-3, nx)."""
    gm, ro_lim, pr_lim = g.gm, g.ro_lim, g.pr_lim
    Vm = u2v_mhd(U[:NVM], gm, ro_lim, pr_lim)
    Vh = u2v_hd(U[NVM:], gm, ro_lim, pr_lim)
    rows = slice(M, -M) if g.ndim == 2 else slice(None)
    Lm, Rm = face_states(Vm[:, rows, :], ro_lim)
    Lh, Rh = face_states(Vh[:, rows, :], ro_lim)
    Fx = torch.cat([hlld(Lm, Rm, gm), hllc(Lh, Rh, gm)], dim=0)
    if g.ndim == 1:
        return Fx, None
    Vmy = Vm[PERM_M_Y][:, :, M:-M].transpose(1, 2)
    Vhy = Vh[PERM_H_Y][:, :, M:-M].transpose(1, 2)
    Lm, Rm = face_states(Vmy, ro_lim)
    Lh, Rh = face_states(Vhy, ro_lim)
    Fy = torch.cat([hlld(Lm, Rm, gm)[PERM_M_Y], hllc(Lh, Rh, gm)[PERM_H_Y]], dim=0).transpose(1, 2)
    return Fx, Fy


def cq2pv(u, gm, ro_lim, pr_lim, mhd):                    # Scheme_rot.f90:132-179
    de = u[0]
    vx, vy, vz = u[1] / de, u[2] / de, u[3] / de
    if mhd:
        bb = u[5] * u[5] + u[6] * u[6] + u[7] * u[7]
        pr = (gm - 1.0) * (u[4] - 0.5 * de * (vx * vx + vy * vy + vz * vz) - 0.5 * bb)
    else:
        pr = (gm - 1.0) * (u[4] - 0.5 * de * (vx * vx + vy * vy + vz * vz))
    pr = torch.clamp(pr, min=pr_lim)
    de = torch.clamp(de, min=ro_lim)
    e = pr / (gm - 1.0) + 0.5 * de * (vx * vx + vy * vy + vz * vz)
    if mhd:
        e = e + 0.5 * bb
        w = torch.stack([de, vx * de, vy * de, vz * de, e, u[5], u[6], u[7]])
    else:
        w = torch.stack([de, vx * de, vy * de, vz * de, e])
    return w, (de, vx, vy, vz, pr)


def source(Ui, gm, ac, ro_lim, pr_lim):
    """Explicit collision source S (PIP_rot.f90:1333-1368) on cells of Ui (13, ...)."""
    um, qm = cq2pv(Ui[:NVM], gm, ro_lim, pr_lim, True)
    uh, qh = cq2pv(Ui[NVM:], gm, ro_lim, pr_lim, False)
    de, vx, vy, vz, pr = qm
    nde, nvx, nvy, nvz, npr = qh
    te = pr / de * gm * MU_P
    nte = npr / nde * gm * MU_N
    ds1 = ac * (um[0] * uh[1] - uh[0] * um[1])
    ds2 = ac * (um[0] * uh[2] - uh[0] * um[2])
    ds3 = ac * (um[0] * uh[3] - uh[0] * um[3])
    ds4 = ac * nde * de * (0.5 * ((nvx * nvx - vx * vx) + (nvy * nvy - vy * vy) + (nvz * nvz - vz * vz))
                           + 3.0 / gm / 2.0 * (nte - te))
    z = torch.zeros_like(ds1)
    ds = torch.stack([z, ds1, ds2, ds3, ds4])
    Sm = torch.cat([ds, torch.zeros_like(Ui[5:NVM])], dim=0)
    return torch.cat([Sm, -ds], dim=0)


def stage(Us, U0, dt_sub, ac, g):
    """One RK stage (add_flux_rk x then y, add_source) and the ghost fill."""
    Fx, Fy = fluxes(Us, g)
    sl = g.sl()
    S = source(Us[sl], g.gm, ac, g.ro_lim, g.pr_lim)
    u = U0[sl] - (dt_sub / g.dx[M:-M][None, None, :]) * (Fx[:, :, 1:] - Fx[:, :, :-1])
    if g.ndim == 2:
        u = u - (dt_sub / g.dy[M:-M][None, :, None]) * (Fy[:, 1:, :] - Fy[:, :-1, :])
    u = u + S * dt_sub
    return fill(u, g)


def rewrite(U, g):
    um, qm = cq2pv(U[:NVM], g.gm, g.ro_lim, g.pr_lim, True)
    uh, qh = cq2pv(U[NVM:], g.gm, g.ro_lim, g.pr_lim, False)
    return torch.cat([um, uh], dim=0), qm, qh


def cfl_dt(U, ac, g):
    """cfl (Scheme_rot.f90:183-213) for a state; returns (rewritten state, dt)."""
    W, qm, qh = rewrite(U, g)
    sl = g.sl()[1:]
    gm, safety = g.gm, g.safety
    de, vx, vy, vz, pr = [q[sl] for q in qm]
    bx, by, bz = [W[n][sl] for n in (5, 6, 7)]
    if g.ndim == 2:
        gmin = torch.minimum(g.dx[M:-M][None, :], g.dy[M:-M][:, None])
    else:
        gmin = torch.minimum(g.dx[M:-M], g.dy[0:1])[None, :]
    dm = torch.clamp(de, min=TINY)
    cs2 = gm * pr / dm
    valf2 = (bx * bx + by * by + bz * bz) / dm
    vabs = torch.sqrt(vx * vx + vy * vy + vz * vz)
    cand_m = safety * gmin / (vabs + torch.sqrt(cs2 + valf2))
    nde, nvx, nvy, nvz, npr = [q[sl] for q in qh]
    cs = torch.sqrt(gm * npr / nde)
    nvabs = torch.sqrt(torch.clamp(nvx * nvx + nvy * nvy + nvz * nvz, min=TINY))
    cand_h = safety * gmin / (nvabs + cs)
    cand = _min(cand_m, cand_h).reshape(-1)
    dt = cand[torch.argmin(cand)]                       # the first cell on a tie
    rcell = _max(W[0][sl] * ac, W[NVM][sl] * ac).reshape(-1)
    rho = rcell[torch.argmax(rcell)]
    dtc = min(safety, 0.3) / rho
    dt = torch.where(dtc < dt, dtc, dt)
    return W, dt


def run(U0, ac, nsteps, g):
    """nsteps steps of the time loop from U0 (13, jx, ix); returns the final state (after the
    last cfl rewrite) and the list of dt."""
    dts = []
    W, dt = cfl_dt(U0, ac, g)
    for n in range(nsteps):
        U1 = stage(W, W, dt / 2.0, ac, g)
        U2 = stage(U1, W, dt / 1.0, ac, g)
        dts.append(dt)
        W1, _, _ = rewrite(U2, g)                      # cfl after run_solver
        if n + 1 == nsteps:
            return W1, dts
        W, dt = cfl_dt(W1, ac, g)                      # cfl of the next step
    return W, dts
