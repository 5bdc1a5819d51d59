"""Small seeded cases for the decomposition tests: periodic 2D with Dedner cleaning
(Orszag-Tang), 2D with reflecting walls at the ends of the split axis and ionisation/
recombination (Kelvin-Helmholtz), and 1D with outflow ends (Brio-Wu); the ``_col`` cases
use alpha_c per cell (set_collisional), ``ot_resi`` adds a uniform resistivity, ``kh_ir1``
and ``kh_ir3`` use set_IR types 1 and 3, ``kh_hc`` and ``kh_hc_generic`` implicit conduction."""
from generic_state import generic_state
from pip_b200 import ics


def make_case(case):
    if case == "ot":
        s, Uh, Um = ics.orszag_tang(16)
    elif case == "kh":
        s, Uh, Um = ics.kelvin_helmholtz(16, 16)
    elif case == "bw":
        s, Uh, Um = ics.brio_wu(64)
    elif case == "ot_col":
        s, Uh, Um = ics.orszag_tang(16, flag_col=6)   # alpha_c per cell, col_type 5
    elif case == "kh_col":
        s, Uh, Um = ics.kelvin_helmholtz(16, 16, flag_col=4)
    elif case == "kh_ir1":
        s, Uh, Um = ics.kelvin_helmholtz(16, 16, flag_ir=1, t_norm=1.5e4, n_norm=1.0e11, t_ir=10.0)
    elif case == "kh_ir3":
        s, Uh, Um = ics.kelvin_helmholtz(16, 16, flag_ir=3, t_norm=1.5e4, n_norm=1.0e11, t_ir=10.0,
                                         flag_col=5)
    elif case == "ot_resi":
        s, Uh, Um = ics.orszag_tang(16, flag_resi=1, eta_0=2e-3, flag_col=3)
    elif case == "kh_hc":
        s, Uh, Um = ics.kelvin_helmholtz(16, 16, flag_heat=1, kapper=0.1, hc_error=1e-12,
                                         hc_max=400)
    elif case == "kh_hc_generic":
        s, _, _ = ics.kelvin_helmholtz(24, 32, flag_heat=1, kapper=1.0, hc_error=1e-12,
                                       hc_max=800)
        Uh, Um = generic_state(s, 5)
    elif case == "ot_generic":
        s, _, _ = ics.orszag_tang(16)
        Uh, Um = generic_state(s, 11)
    else:
        raise ValueError(case)
    return s, Uh, Um
