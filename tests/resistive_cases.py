"""The resistive decay case of the resistivity tests: a 1D periodic two-fluid rest state
with By = 1e-4 sin(2 pi x), whose field diffuses at the rate eta*sin(k dx)^2/dx^2 of the
discrete operator (resistive_flux's face average of the central-difference curl)."""
import math

import numpy as np

from pip_b200 import ics
from pip_b200.params import Settings


def decay_case(n, eta, **kw):
    """1D periodic two-fluid rest state with By = 1e-4 sin(2 pi x): the field diffuses."""
    s = Settings(ndim=1, ix0=n, start=(0.0, -1.0, -1.0), end=(1.0, 1.0, 1.0), flag_bnd=[1] * 6,
                 n_fraction=0.5, col=1.0, safety=0.3, flag_divb=0, flag_resi=1, eta_0=eta)
    s = s.overrides(**kw)
    X, _ = ics._grid(s)
    f_n, f_p, f_p_n, f_p_p = ics.fractions(s.n_fraction)
    one, zero = np.ones_like(X), np.zeros_like(X)
    by = 1e-4 * np.sin(2.0 * math.pi * X)
    Uh = ics.pv2cq_hd(s, f_n * one, zero, zero, zero, f_p_n * one)
    Um = ics.pv2cq_mhd(s, f_p * one, zero, zero, zero, f_p_p * one, zero, by, zero)
    return s, Uh, Um


def decay_factor(s, Um, t):
    m = s.margin[0]
    X, _ = ics._grid(s)
    x = X[0, m:-m]
    amp = 2.0 * np.mean(Um[6, 0, m:-m] * np.sin(2.0 * math.pi * x)) / 1e-4
    n = s.ix0
    dx = 1.0 / n
    return amp, math.exp(-s.eta_0 * math.sin(2.0 * math.pi * dx) ** 2 / dx ** 2 * t)
