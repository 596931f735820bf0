"""Physical constants and unit conversions (constants.py:11-29 of the
reference): SciPy's CODATA values, so the B200 backend multiplies by the same
doubles the reference does."""

from scipy import constants as _c

ELEMENTARY_CHARGE = _c.e
SPEED_OF_LIGHT = _c.c
VACUUM_PERMITTIVITY = _c.epsilon_0
COULOMB_CONSTANT = 1.0 / (4.0 * _c.pi * VACUUM_PERMITTIVITY)


def ev_c_to_si_momentum(p_ev_c):
    return p_ev_c * ELEMENTARY_CHARGE / SPEED_OF_LIGHT


def si_momentum_to_ev_c(p_si):
    return p_si * SPEED_OF_LIGHT / ELEMENTARY_CHARGE


def ev_to_kg(mass_ev):
    return mass_ev * ELEMENTARY_CHARGE / SPEED_OF_LIGHT**2
