"""Independent numpy restatement of the 6-level hydrogen model (test infrastructure).

A second transcription of the Fortran of set_IR type 4, written from PIP_rot.f90 directly:
get_col_ion_coeff (:361-616) with ionexpfitinterp2 (:919-946), IRgetionpot (:1162-1235),
hydrogen_excitation_update (:1026-1159) for 1D, and the trapezoid of
expintcalc/colexpintcalc.f90.  Vectorised over cells; exp, log and pow go through libm one
value at a time (numpy's vectorised versions may differ in the last bit), so it can be
compared with the C oracle bit for bit.
"""
import math

import numpy as np

PI = 3.1415926535897932
F32 = np.float32


def _f(x):
    """A Fortran default-real literal: the nearest float, widened."""
    return float(F32(x))


KB = _f(1.38064852e-23)
ME = _f(9.10938356e-31)
A0 = _f(5.29e-11)
E14 = _f(1.0e14)
KBHAT, MEHAT, HHAT = 1.38064852, 9.10938356, 6.62607004


def _map(fn, *arrs):
    arrs = [np.asarray(a, dtype=np.float64) for a in arrs]
    shape = np.broadcast(*arrs).shape
    flat = [np.broadcast_to(a, shape).ravel() for a in arrs]
    return np.array([fn(*v) for v in zip(*flat)], dtype=np.float64).reshape(shape)


def exp(a):
    return _map(math.exp, a)


def log(a):
    return _map(math.log, a)


def powr(a, b):
    return _map(math.pow, a, b)


def trapezoid(zhat, istar, vectorised_exp=np.exp):
    """colexpintcalc.f90's ionexpfittest for an array of zhat; the abscissae a, b advance
    the same way for every row, so the rows share them and stop one by one."""
    z = np.asarray(zhat, dtype=np.float64)
    step, tol = 0.001, 0.0001
    a = 1.0
    b = a + step
    fa = vectorised_exp(-z * a) * math.pow(a, -istar)
    fb = vectorised_exp(-z * b) * math.pow(b, -istar)
    sol0 = 0.5 * (b - a) * (fa + fb)
    sol = sol0.copy()
    active = np.ones(z.shape, dtype=bool)
    while active.any():
        a = b
        b = a + step
        pa, pb = math.pow(a, -istar), math.pow(b, -istar)
        za = z[active]
        solt = 0.5 * (b - a) * (vectorised_exp(-za * a) * pa + vectorised_exp(-za * b) * pb)
        sol[active] = sol[active] + solt
        done = (solt / sol0[active]) <= tol
        idx = np.flatnonzero(active)
        active[idx[done]] = False
    return sol


class Rates:
    """Cell-independent coefficients, then rates of cells (te [K], ne), from the Fortran."""

    def __init__(self, table):
        self.tab = np.asarray(table, dtype=np.float64)      # (n, 4): yn, E0, E1, E2
        self.gw = np.array([2.0, 8.0, 18.0, 32.0, 50.0, 1.0])
        ev = np.array([13.6, 3.4, 1.51, 0.85, 0.54, 0.0])
        self.eion = ev / 13.6 * _f(2.18e-18)
        self.rn = np.array([0.45] + [1.94 * math.pow(float(k), -1.57) for k in range(2, 7)])
        self.bn = np.array([-0.603] + [(1.0 / k) * (4.0 - 18.63 / k + 36.24 / (k ** 2) -
                                                     28.09 / (k ** 3)) for k in
                                       (2.0, 3.0, 4.0, 5.0, 6.0)])

    def pair(self, ii, jj):
        """xrat, Enn, rnn, Ann, Bnn, log term for levels ii < jj (1-based)."""
        i, j = float(ii), float(jj)
        x = 1.0 - (i / j) * (i / j)
        if ii == 1:
            g = 1.1330 - 0.4059 / x + 0.07014 / (x * x)
        elif ii == 2:
            g = 1.0785 - 0.2319 / x + 0.02947 / (x * x)
        else:
            g = (0.9935 + 0.2328 / i - 0.1296 / (i * i)
                 - (1.0 / x) * (1.0 / i) * (0.6282 - 0.5598 / i + 0.5299 / (i * i))
                 + (1.0 / x) * (1.0 / x) * (1.0 / (i * i)) * (0.3887 - 1.181 / i + 1.470 / (i * i)))
        fnn = 32.0 / 3.0 / math.sqrt(3.0) / PI * i / (j * j * j) / (x * x * x) * g
        ann = 2.0 * (i * i) / x * fnn
        bnn = 4.0 * ((i * i) * (i * i)) / (j * j * j) / (x * x) * \
            (1.0 + 4.0 / 3.0 / x + self.bn[ii - 1] / (x * x))
        return (x, self.eion[ii - 1] - self.eion[jj - 1], self.rn[ii - 1] * x, ann, bnn,
                math.log(2.0 * (i * i) / x))

    def level(self, ii):
        i = float(ii)
        if ii == 1:
            g = (1.1330, -0.4059, 0.07014)
        elif ii == 2:
            g = (1.0785, -0.2319, 0.02947)
        else:
            g = (0.9935 + 0.2328 / i - 0.1296 / (i * i),
                 (-1.0 / i) * (0.6282 - 0.5598 / i + 0.5299 / (i * i)),
                 (1.0 / i) * (1.0 / i) * (0.3887 - 1.181 / i + 1.470 / (i * i)))
        an0 = 32.0 / 3.0 / math.sqrt(3.0) / PI * i + g[0] / 3.0 + g[1] / 4.0 + g[2] / 5.0
        bn0 = 2.0 / 3.0 * (i * i) * (5.0 + self.bn[ii - 1])
        return an0, bn0, math.log(2.0 * (i * i))

    def interp(self, z, col):
        """ionexpfitinterp2 (rad 0) of E_col at z (array); xindex stops at n-2."""
        t = self.tab
        n = t.shape[0]
        xmin, xmax = t[0, 0], t[-1, 0]
        f = np.floor((z - xmin) / (xmax - xmin) * float(n))
        xi = np.where(~(f > 0.0), 1, np.where(f >= n, n - 1, np.nan_to_num(f, nan=1.0)))
        xi = np.minimum(xi.astype(np.int64), n - 2)
        x0, x1, x2 = t[xi - 1, 0], t[xi, 0], t[xi + 1, 0]
        w0 = ((z - x1) * (z - x2)) / ((x0 - x1) * (x0 - x2))
        w1 = ((z - x0) * (z - x2)) / ((x1 - x0) * (x1 - x2))
        w2 = ((z - x0) * (z - x1)) / ((x2 - x0) * (x2 - x1))
        return w0 * t[xi - 1, col + 1] + w1 * t[xi, col + 1] + w2 * t[xi + 1, col + 1]

    def colrat(self, te, ne):
        """colrat (6, 6, ...) with [a, b] = colrat(a+1, b+1) for cells (te, ne)."""
        te = np.asarray(te, dtype=np.float64)
        ne = np.asarray(ne, dtype=np.float64)
        cr = np.zeros((6, 6) + te.shape)
        s = np.sqrt(8.0 * KB * te / PI / ME)
        colex = {}
        for ii in range(1, 6):
            for jj in range(ii + 1, 6):
                x, enn, rnn, ann, bnn, lgt = self.pair(ii, jj)
                yhat = enn / KB / te
                zhat = rnn + enn / KB / te
                E1y, E1z = self.interp(yhat, 1), self.interp(zhat, 1)
                E2y, E2z = self.interp(yhat, 2), self.interp(zhat, 2)
                colex[ii, jj] = (ne * s * 2.0 * float(ii) ** 2 / x * PI * (A0 * A0) * (yhat * yhat) *
                                 (ann * ((1.0 / yhat + 0.5) * E1y - (1.0 / zhat + 0.5) * E1z) +
                                  (bnn - ann * lgt) * (E2y / yhat - E2z / zhat)))
            an0, bn0, lgi = self.level(ii)
            yn = self.eion[ii - 1] / KB / te
            zn = self.rn[ii - 1] + self.eion[ii - 1] / KB / te
            E1y, E1z = self.interp(yn, 1), self.interp(zn, 1)
            E2y, E2z = self.interp(yn, 2), self.interp(zn, 2)
            E0y, E0z = self.interp(yn, 0), self.interp(zn, 0)
            ziyn = E0y - 2.0 * E1y + E2y
            zizn = E0z - 2.0 * E1z + E2z
            colex[ii, 6] = (ne * s * 2.0 * float(ii) ** 2 * PI * (A0 * A0) * (yn * yn) *
                            (an0 * (E1y / yn - E1z / zn) + (bn0 - an0 * lgi) * (ziyn - zizn)))
        for ii in range(1, 6):
            for jj in range(1, 6):
                if jj > ii:
                    cr[ii - 1, jj - 1] = self.gw[ii - 1] / self.gw[jj - 1] * colex[ii, jj]
                elif jj < ii:
                    cr[ii - 1, jj - 1] = colex[jj, ii] * exp(
                        -((self.eion[jj - 1] - self.eion[ii - 1]) / KB / te))
            cr[ii - 1, 5] = colex[ii, 6] * exp(-((self.eion[5] - self.eion[ii - 1]) / KB / te))
        saha = powr(2.0 * PI * MEHAT * KBHAT * te / HHAT / HHAT * E14, -1.5)
        for ii in range(1, 6):
            cr[5, ii - 1] = (ne * cr[ii - 1, 5] * self.gw[ii - 1] / self.gw[5] / 2.0 * saha *
                             exp(self.eion[ii - 1] / KB / te))
        return cr

    @staticmethod
    def sums(cr, nex):
        """Gm_ion and Gm_rec before normalisation: sums of max(.,0) over levels 1-5."""
        gi = np.zeros(cr.shape[2:])
        gr = np.zeros(cr.shape[2:])
        for a in range(5):
            gi = gi + np.maximum(nex[a] * cr[a, 5], 0.0)
            gr = gr + np.maximum(nex[5] * cr[5, a], 0.0)
        return gi, gr


def ion_pot(cr, nex, gm, t0, beta, flag_col, gref, t_ir):
    """IRgetionpot (PIP_rot.f90:1162-1235)."""
    eev = [float(F32(v)) for v in (13.6, 3.4, 1.51, 0.85, 0.54, 0.0)]
    il = np.zeros(cr.shape[2:])
    ig = np.zeros(cr.shape[2:])
    for i in range(5):
        il = il + cr[i, 5] * eev[i] * nex[i]
        ig = ig + cr[5, i] * eev[i] * nex[5]
        for j in range(1, 5):
            il = il + nex[i] * cr[i, j] * (eev[i] - eev[j])
            ig = ig + nex[j] * (cr[j, i] * (eev[i] - eev[j]))
    if flag_col % 2 == 1:
        en = (il - ig) / gm / t0 / _f(8.6173e-5)
    else:
        en = (il - ig) / (beta / t0 / 2.0 / _f(8.6173e-5))
    return en / gref * t_ir


def excitation_update_1d(nex, cr, rho_n, rho_i, mx_n, dx, dt, gref, t_ir, deriv):
    """hydrogen_excitation_update on a 1D row (interior result for every cell whose
    derivative stencil fits; the caller applies the boundary)."""
    n = nex.shape[-1]
    w = {1: 1, 4: 2}.get(deriv, 0)
    d = np.zeros((6, n))
    for jj in range(5):
        d[5] = d[5] + nex[jj] * cr[jj, 5] / gref * t_ir - nex[5] * cr[5, jj] / gref * t_ir
    for ii in range(5):
        d[ii] = d[ii] + nex[5] * cr[5, ii] / gref * t_ir - nex[ii] * cr[ii, 5] / gref * t_ir
    for ii in range(5):
        for jj in range(5):
            d[ii] = d[ii] + nex[jj] * cr[jj, ii] / gref * t_ir - nex[ii] * cr[ii, jj] / gref * t_ir
    out = nex.copy()
    for ii in range(5):
        der = np.zeros(n)
        if deriv == 1:
            der[1:-1] = (nex[ii, 2:] - nex[ii, :-2]) / (2.0 * dx[1:-1])
        elif deriv == 4:
            der[2:-2] = (-nex[ii, 4:] + 8.0 * nex[ii, 3:-1] - 8.0 * nex[ii, 1:-3] + nex[ii, :-4]) / \
                (12.0 * dx[2:-2])
        conv = der * mx_n / rho_n
        v = nex[ii] + dt * (d[ii] - conv)
        out[ii] = np.where(v > _f(1.e-16), v, _f(1.e-16))
    tot = out[0] + out[1] + out[2] + out[3] + out[4] - rho_n
    out[0] = out[0] - tot
    out[5] = rho_i
    return out
