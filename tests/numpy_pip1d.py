"""Independent numpy restatement of the 1D two-fluid step (test infrastructure).

A second transcription of the same Fortran, vectorised over faces and cells with numpy's
IEEE double arithmetic (no FMA), used to cross-check the C oracle bit for bit on 1D runs.
It follows main.f90:31-68 / run_solver (Solver_rot.f90:42-81) for flag_sch=0, flag_hll=2,
s_order=2, t_order=2, ndim=1, explicit or exponential collisions, boundary types 1/2/10.
"""
import math

import numpy as np

TINY = 1e-20


def _exp(a):
    """libm's exp element by element (numpy's vectorised exp may differ by an ulp)."""
    a = np.asarray(a, dtype=np.float64)
    return np.array([math.exp(v) for v in a.ravel()]).reshape(a.shape)


EPSI = 1e-10
ACC = 1.03
HLLG = 1.001


def u2v_mhd(U, gm, ro_lim, pr_lim):                       # HLL_rot.f90:1159-1186
    V = np.empty_like(U)
    V[0] = np.maximum(U[0], ro_lim)
    roi = 1.0 / V[0]
    V[1] = U[1] * roi
    V[2] = U[2] * roi
    V[3] = U[3] * roi
    V[4] = (gm - 1.0) * (U[4] - 0.5 * (U[1] ** 2 + U[2] ** 2 + U[3] ** 2) * roi
                         - 0.5 * (U[5] ** 2 + U[6] ** 2 + U[7] ** 2))
    V[4] = np.where(V[4] < pr_lim, pr_lim, V[4])
    V[5:8] = U[5:8]
    return V


def u2v_hd(U, gm, ro_lim, pr_lim):                        # HLL_rot.f90:1136-1156
    V = np.empty_like(U)
    V[0] = np.maximum(U[0], ro_lim)
    roi = 1.0 / V[0]
    V[1] = U[1] * roi
    V[2] = U[2] * roi
    V[3] = U[3] * roi
    V[4] = (gm - 1.0) * (U[4] - 0.5 * (U[1] ** 2 + U[2] ** 2 + U[3] ** 2) * roi)
    V[4] = np.where(V[4] < pr_lim, pr_lim, V[4])
    return V


def sides(V, ro_lim):                                     # get_Side + minmod_func
    X = V[:, 2:] - V[:, 1:-1]
    Y = V[:, 1:-1] - V[:, :-2]
    SX = np.copysign(1.0, X)
    dU = SX * np.maximum(0.0, np.minimum(np.abs(X), SX * Y))
    VL = np.zeros_like(V)
    VR = np.zeros_like(V)
    VL[:, 1:-1] = V[:, 1:-1] + 0.5 * dU
    VR[:, :-2] = V[:, 1:-1] - 0.5 * dU
    VL[0] = np.maximum(VL[0], ro_lim)
    VR[0] = np.maximum(VR[0], ro_lim)
    return VL, VR


def hllc(vl, vr, gm):                                     # HLL_rot.f90:615-687
    def cons(v):
        u = np.empty_like(v)
        u[0] = v[0]
        u[1] = v[0] * v[1]
        u[2] = v[0] * v[2]
        u[3] = v[0] * v[3]
        u[4] = v[4] / (gm - 1.0) + 0.5 * v[0] * (v[1] ** 2 + v[2] ** 2 + v[3] ** 2)
        return u
    ul, ur = cons(vl), cons(vr)
    pl, pr = vl[4], vr[4]

    def flux(u, p):
        f = np.empty_like(u)
        f[0] = u[1]
        f[1] = p + u[1] ** 2 / u[0]
        f[2] = u[1] * u[2] / u[0]
        f[3] = u[1] * u[3] / u[0]
        f[4] = u[1] * (u[4] + p) / u[0]
        return f
    fl, fr = flux(ul, pl), flux(ur, pr)
    csl = np.sqrt(gm * pl / ul[0])
    csr = np.sqrt(gm * pr / ur[0])
    vnl = ul[1] / ul[0]
    vnr = ur[1] / ur[0]
    sl = ACC * np.minimum(vnl - csl, vnr - csr)
    sr = ACC * np.maximum(vnl + csl, vnr + csr)
    sm = (ur[1] * (sr - vnr) - ul[1] * (sl - vnl) + pl - pr) / (ur[0] * (sr - vnr) - ul[0] * (sl - vnl))
    pm = sm * ul[0] * (sl - vnl) - ul[1] * (sl - vnl) + pl
    stl = np.empty_like(ul)
    str_ = np.empty_like(ur)
    stl[0] = ul[0] * (sl - vnl) / (sl - sm)
    str_[0] = ur[0] * (sr - vnr) / (sr - sm)
    stl[1] = stl[0] * sm
    str_[1] = str_[0] * sm
    stl[2] = stl[0] * ul[2] / ul[0]
    str_[2] = str_[0] * ur[2] / ur[0]
    stl[3] = stl[0] * ul[3] / ul[0]
    str_[3] = str_[0] * ur[3] / ur[0]
    stl[4] = ((sl - vnl) * ul[4] - pl * vnl + pm * sm) / (sl - sm)
    str_[4] = ((sr - vnr) * ur[4] - pr * vnr + pm * sm) / (sr - sm)
    thl = (np.abs(sl) + sl) / np.maximum(2.0 * sl, EPSI)
    thm = (np.abs(sm) + sm) / np.maximum(2.0 * sm, EPSI)
    thr = 1.0 - (np.abs(sr) + sr) / np.maximum(2.0 * sr, EPSI)
    return (thr * fr + thl * fl + (1.0 - thl - thr) *
            (thm * (fl + sl * (stl - ul)) + (1.0 - thm) * (fr + sr * (str_ - ur))))


def hlld(vl, vr, gm):                                     # HLL_rot.f90:691-910 (8 variables)
    def cons(v):
        u = np.empty_like(v)
        u[0] = v[0]
        u[1] = v[0] * v[1]
        u[2] = v[0] * v[2]
        u[3] = v[0] * v[3]
        u[5:8] = v[5:8]
        u[4] = (v[4] / (gm - 1.0) + 0.5 * v[0] * (v[1] ** 2 + v[2] ** 2 + v[3] ** 2)
                + 0.5 * (v[5] ** 2 + v[6] ** 2 + v[7] ** 2))
        return u

    def flux(v, u):
        b2 = v[5] ** 2 + v[6] ** 2 + v[7] ** 2
        pt = v[4] + 0.5 * b2
        vb = v[1] * v[5] + v[2] * v[6] + v[3] * v[7]
        f = np.zeros_like(v)
        f[0] = v[0] * v[1]
        f[1] = v[0] * v[1] ** 2 + v[4] + 0.5 * b2 - v[5] ** 2
        f[2] = v[0] * v[1] * v[2] - v[5] * v[6]
        f[3] = v[0] * v[1] * v[3] - v[5] * v[7]
        f[4] = (u[4] + pt) * v[1] - vb * v[5]
        f[6] = v[1] * v[6] - v[5] * v[2]
        f[7] = v[1] * v[7] - v[5] * v[3]
        return f, b2, pt, vb

    ul, ur = cons(vl), cons(vr)
    fl, b2l, ptl, vbl = flux(vl, ul)
    fr, b2r, ptr, vbr = flux(vr, ur)

    def fast(v, b2):
        f1 = gm * v[4]
        f2 = 4.0 * f1 * v[5] ** 2
        return np.sqrt(((f1 + b2) + np.sqrt(np.maximum((f1 + b2) ** 2 - f2, 0.0))) / (2.0 * v[0]))
    vfl, vfr = fast(vl, b2l), fast(vr, b2r)
    sl = np.minimum(vl[1], vr[1]) - np.maximum(vfl, vfr)
    sr = np.maximum(vl[1], vr[1]) + np.maximum(vfl, vfr)
    with np.errstate(all="ignore"):
        f1 = 1.0 / (sr - sl)
        uh = f1 * (sr * ur - sl * ul - fr + fl)
        sm = uh[1] / uh[0]
        pt = ptl + vl[0] * (sl - vl[1]) * (sm - vl[1])
        rol1 = vl[0] * (sl - vl[1]) / (sl - sm)
        ror1 = vr[0] * (sr - vr[1]) / (sr - sm)
        sal = np.abs(uh[5]) / np.sqrt(rol1)
        sar = np.abs(uh[5]) / np.sqrt(ror1)
        # HLLC-G
        vy2 = uh[2] / uh[0]
        vz2 = uh[3] / uh[0]
        gl = np.empty_like(vl)
        e2 = ((sl - vl[1]) * ul[4] - ptl * vl[1] + pt * sm
              + uh[5] * (vbl - sm * uh[5] - vy2 * uh[6] - vz2 * uh[7])) / (sl - sm)
        gl[0] = sl * (rol1 - vl[0]) + fl[0]
        gl[1] = sl * (rol1 * sm - ul[1]) + fl[1]
        gl[2] = sl * (rol1 * vy2 - ul[2]) + fl[2]
        gl[3] = sl * (rol1 * vz2 - ul[3]) + fl[3]
        gl[4] = sl * (e2 - ul[4]) + fl[4]
        gl[5:8] = sl * (uh[5:8] - vl[5:8]) + fl[5:8]
        gr = np.empty_like(vr)
        e2r = ((sr - vr[1]) * ur[4] - ptr * vr[1] + pt * sm
               + uh[5] * (vbr - sm * uh[5] - vy2 * uh[6] - vz2 * uh[7])) / (sr - sm)
        gr[0] = sr * (ror1 - vr[0]) + fr[0]
        gr[1] = sr * (ror1 * sm - ur[1]) + fr[1]
        gr[2] = sr * (ror1 * vy2 - ur[2]) + fr[2]
        gr[3] = sr * (ror1 * vz2 - ur[3]) + fr[3]
        gr[4] = sr * (e2r - ur[4]) + fr[4]
        gr[5:8] = sr * (uh[5:8] - vr[5:8]) + fr[5:8]
        hllcg = np.where(sm >= 0.0, gl, gr)

        def star(v, u, s, ro1, ptx, vbx):
            f = 1.0 / (v[0] * (s - v[1]) * (s - sm) - uh[5] ** 2)
            w = np.empty_like(v)
            w[5] = uh[5]
            w[6] = v[6] * f * (v[0] * (s - v[1]) ** 2 - uh[5] ** 2)
            w[7] = v[7] * f * (v[0] * (s - v[1]) ** 2 - uh[5] ** 2)
            vy1 = v[2] - f * uh[5] * v[6] * (sm - v[1])
            vz1 = v[3] - f * uh[5] * v[7] * (sm - v[1])
            w[0] = ro1
            w[4] = ((s - v[1]) * u[4] - ptx * v[1] + pt * sm
                    + uh[5] * (vbx - sm * uh[5] - vy1 * w[6] - vz1 * w[7])) / (s - sm)
            w[1] = ro1 * sm
            w[2] = ro1 * vy1
            w[3] = ro1 * vz1
            return w, vy1, vz1
        ul1, vyl1, vzl1 = star(vl, ul, sl, rol1, ptl, vbl)
        ur1, vyr1, vzr1 = star(vr, ur, sr, ror1, ptr, vbr)
        sl1 = sm - sal
        sr1 = sm + sar
        fls = np.empty_like(vl)
        fls[0] = sl * (ul1[0] - vl[0]) + fl[0]
        fls[1:5] = sl * (ul1[1:5] - ul[1:5]) + fl[1:5]
        fls[5:8] = sl * (ul1[5:8] - vl[5:8]) + fl[5:8]
        frs = np.empty_like(vr)
        frs[0] = sr * (ur1[0] - vr[0]) + fr[0]
        frs[1:5] = sr * (ur1[1:5] - ur[1:5]) + fr[1:5]
        frs[5:8] = sr * (ur1[5:8] - vr[5:8]) + fr[5:8]
        rls = np.sqrt(rol1)
        rrs = np.sqrt(ror1)
        f1c = 1.0 / (rls + rrs)
        f2 = np.copysign(1.0, uh[5])
        vy2c = f1c * (rls * vyl1 + rrs * vyr1 + (ur1[6] - ul1[6]) * f2)
        vz2c = f1c * (rls * vzl1 + rrs * vzr1 + (ur1[7] - ul1[7]) * f2)
        u2 = np.empty_like(vl)
        u2[5] = uh[5]
        u2[6] = f1c * (rls * ur1[6] + rrs * ul1[6] + rls * rrs * (vyr1 - vyl1) * f2)
        u2[7] = f1c * (rls * ur1[7] + rrs * ul1[7] + rls * rrs * (vzr1 - vzl1) * f2)
        cl = np.empty_like(vl)
        u2l = u2.copy()
        u2l[0] = rol1
        u2l[4] = ul1[4] - rls * (vyl1 * ul1[6] + vzl1 * ul1[7] - vy2c * u2[6] - vz2c * u2[7]) * f2
        u2l[1] = rol1 * sm
        u2l[2] = rol1 * vy2c
        u2l[3] = rol1 * vz2c
        cl[0] = sl1 * u2l[0] - (sl1 - sl) * ul1[0] - sl * vl[0] + fl[0]
        cl[1:5] = sl1 * u2l[1:5] - (sl1 - sl) * ul1[1:5] - sl * ul[1:5] + fl[1:5]
        cl[5:8] = sl1 * u2l[5:8] - (sl1 - sl) * ul1[5:8] - sl * vl[5:8] + fl[5:8]
        cr = np.empty_like(vr)
        u2r = u2.copy()
        u2r[0] = ror1
        u2r[4] = ur1[4] + rrs * (vyr1 * ur1[6] + vzr1 * ur1[7] - vy2c * u2[6] - vz2c * u2[7]) * f2
        u2r[1] = ror1 * sm
        u2r[2] = ror1 * vy2c
        u2r[3] = ror1 * vz2c
        cr[0] = sr1 * u2r[0] - (sr1 - sr) * ur1[0] - sr * vr[0] + fr[0]
        cr[1:5] = sr1 * u2r[1:5] - (sr1 - sr) * ur1[1:5] - sr * ur[1:5] + fr[1:5]
        cr[5:8] = sr1 * u2r[5:8] - (sr1 - sr) * ur1[5:8] - sr * vr[5:8] + fr[5:8]
        central = np.where(sm >= 0.0, cl, cr)
        hlldf = np.where(sl1 >= 0.0, fls, np.where(sr1 <= 0.0, frs, central))
        revert = (sl >= (sm - HLLG * sal)) | ((sm + HLLG * sar) >= sr)
        sub = np.where(revert, hllcg, hlldf)
    return np.where(sl >= 0.0, fl, np.where(sr <= 0.0, fr, sub))


def cq2pv(U, gm, ro_lim, pr_lim, mhd):                    # Scheme_rot.f90:132-179
    de = U[0].copy()
    vx, vy, vz = U[1] / de, U[2] / de, U[3] / de
    if mhd:
        pr = (gm - 1.0) * (U[4] - 0.5 * de * (vx ** 2 + vy ** 2 + vz ** 2)
                           - 0.5 * (U[5] ** 2 + U[6] ** 2 + U[7] ** 2))
    else:
        pr = (gm - 1.0) * (U[4] - 0.5 * de * (vx ** 2 + vy ** 2 + vz ** 2))
    pr = np.maximum(pr, pr_lim)
    de = np.maximum(de, ro_lim)
    U[0] = de
    U[1] = vx * de
    U[2] = vy * de
    U[3] = vz * de
    if mhd:
        U[4] = (pr / (gm - 1.0) + 0.5 * de * (vx ** 2 + vy ** 2 + vz ** 2)
                + 0.5 * (U[5] ** 2 + U[6] ** 2 + U[7] ** 2))
    else:
        U[4] = pr / (gm - 1.0) + 0.5 * de * (vx ** 2 + vy ** 2 + vz ** 2)
    return de, vx, vy, vz, pr


class Run1D:
    def __init__(self, s, U_h, U_m):
        self.s = s
        self.gm = s.gm
        self.Uh = U_h[:, 0, :].copy()
        self.Um = U_m[:, 0, :].copy()
        self.dx = s.coordinates()[3]
        self.m = s.margin[0]
        self.ac = s.col
        self.time = 0.0
        self.cmax = 0.0

    def bnd(self, U, mhd):                               # boundary_control, 1D faces
        m, n = self.m, U.shape[1]
        for side in (0, 1):
            code = self.s.flag_bnd[side]
            t = 2 if code in (3, 4, 5, 6, 7, 11) else code
            sym = np.ones(U.shape[0])
            if code == 2:
                sym[1] = -1.0
                if mhd:
                    sym[5] = -1.0
            for l in range(m):
                dst = l if side == 0 else n - m + l
                if t == 1:
                    src = n - 2 * m + l if side == 0 else m + l
                elif t == 2:
                    src = 2 * m - 1 - l if side == 0 else n - m - 1 - l
                else:
                    src = m if side == 0 else n - m - 1
                U[:, dst] = (sym * U[:, src]) if t != 10 else U[:, src]

    def pipbnd(self):
        self.bnd(self.Um, True)
        self.bnd(self.Uh, False)

    def cfl(self):                                       # Scheme_rot.f90:183-313
        s, gm, m = self.s, self.gm, self.m
        de, vx, vy, vz, pr = cq2pv(self.Um, gm, s.ro_lim, s.pr_lim, True)
        gmin = np.minimum(np.minimum(self.dx, 100.0), 100.0)
        cs2 = gm * pr / np.maximum(de, TINY)
        va2 = (self.Um[5] ** 2 + self.Um[6] ** 2 + self.Um[7] ** 2) / np.maximum(de, TINY)
        vabs = np.sqrt(vx ** 2 + vy ** 2 + vz ** 2)
        dtm = s.safety * gmin / (vabs + np.sqrt(cs2 + va2))
        de, vx, vy, vz, pr = cq2pv(self.Uh, gm, s.ro_lim, s.pr_lim, False)
        cs = np.sqrt(gm * pr / de)
        vabs = np.sqrt(np.maximum(vx ** 2 + vy ** 2 + vz ** 2, TINY))
        dth = s.safety * gmin / (vabs + cs)
        dt = min(10.0, dtm[m:-m].min(), dth[m:-m].min())
        mx = max((self.Um[0] * self.ac).max(), (self.Uh[0] * self.ac).max())
        if s.flag_pip_imp == 1:
            dt = min(dt, s.pip_imp_factor / mx)
        else:
            dt = min(dt, min(s.safety, 0.3) / mx)
        return dt

    def source(self, Uh0, Um0, dt_coll):                 # PIP_rot.f90:1309-1368
        gm, ac = self.gm, self.ac
        nde, nvx, nvy, nvz, npr = cq2pv(self.Uh, gm, self.s.ro_lim, self.s.pr_lim, False)
        de, vx, vy, vz, pr = cq2pv(self.Um, gm, self.s.ro_lim, self.s.pr_lim, True)
        te = pr / de * gm * 0.5
        nte = npr / nde * gm * 1.0
        uh, um = self.Uh, self.Um
        ds = np.zeros((5,) + de.shape)
        Sh = np.zeros_like(self.Uh)
        Sm = np.zeros_like(self.Um)
        if self.s.flag_pip_imp == 1:
            temp = dt_coll * (uh[0] + um[0])
            e = (1.0 - _exp(-ac * temp))
            for k in (1, 2, 3):
                ds[k] = (um[0] * uh[k] - uh[0] * um[k]) * e / temp
            lam = ac * (nde + de)
            kap = 3.0 * (gm - 1.0) * ac * (0.5 * nde + 1.0 * de)
            B = -(1.0 / 3.0 * gm * kap / ((nde + de) * (kap - lam)) *
                  (de * ((nvx - vx) * vx + (nvy - vy) * vy + (nvz - vz) * nvz) +
                   nde * ((nvx - vx) * nvx + (nvy - vy) * nvy + (nvz - vz) * nvz)))
            D = -(gm / 6.0 * kap * (de - nde) / ((de + nde) * (kap - 2 * lam)) *
                  ((nvx - vx) ** 2 + (nvy - vy) ** 2 + (nvz - vz) ** 2))
            ds[4] = -((3.0 / gm) * ac * de * nde / kap *
                      (+(_exp(-kap * dt_coll) - 1.0) * (nte - te) - (B + D) * _exp(-kap * dt_coll)
                       + B * _exp(-lam * dt_coll) + D * _exp(-2.0 * lam * dt_coll)) / dt_coll)
            Uh0[:5] = Uh0[:5] - dt_coll * ds
            Um0[:5] = Um0[:5] + dt_coll * ds
        else:
            for k in (1, 2, 3):
                ds[k] = ac * (um[0] * uh[k] - uh[0] * um[k])
            ds[4] = ac * nde * de * (0.5 * ((nvx ** 2 - vx ** 2) + (nvy ** 2 - vy ** 2) +
                                            (nvz ** 2 - vz ** 2)) + 3.0 / gm / 2.0 * (nte - te))
            Sh[:5] = Sh[:5] - ds
            Sm[:5] = Sm[:5] + ds
        return Sh, Sm

    def run_solver(self, dt):
        s, gm = self.s, self.gm
        Uh0, Um0 = self.Uh.copy(), self.Um.copy()
        Fh = np.zeros_like(self.Uh)
        Fm = np.zeros_like(self.Um)
        for istep in (1, 2):
            dt_coll = dt * 0.5
            V = u2v_mhd(self.Um, gm, s.ro_lim, s.pr_lim)
            VL, VR = sides(V, s.ro_lim)
            Fm[:, :-1] = hlld(VL[:, :-1], VR[:, :-1], gm)
            V = u2v_hd(self.Uh, gm, s.ro_lim, s.pr_lim)
            VL, VR = sides(V, s.ro_lim)
            Fh[:, :-1] = hllc(VL[:, :-1], VR[:, :-1], gm)
            Sh, Sm = self.source(Uh0, Um0, dt_coll)
            dt_sub = dt / float(2 - istep + 1)
            c = dt_sub / self.dx[1:]
            self.Uh[:, 1:] = Uh0[:, 1:] - c * (Fh[:, 1:] - Fh[:, :-1])
            self.Uh = self.Uh + Sh * dt_sub
            self.Um[:, 1:] = Um0[:, 1:] - c * (Fm[:, 1:] - Fm[:, :-1])
            self.Um = self.Um + Sm * dt_sub
            self.pipbnd()
        self.pipbnd()

    def step(self):
        dt = self.cfl()
        self.run_solver(dt)
        self.cfl()
        self.time = self.time + dt
        return dt

    def prologue(self):
        self.cfl()
        self.pipbnd()
