"""Oracle: constants, pair forces, analytic fields, kill masks (float64, NumPy).

Test infrastructure only -- see ``oracle/__init__.py``.  Each function
names the reference function it restates; operation order follows the
reference wherever it changes rounding (sum of squares before adding the
softening, ``r2*sqrt(r2)`` for the cube, left-to-right charge products).
"""

import numpy as np
from scipy import constants as _sc

# constants.py:11-14 -- SciPy CODATA values, the same objects the reference reads.
ELEMENTARY_CHARGE = _sc.e
SPEED_OF_LIGHT = _sc.c
VACUUM_PERMITTIVITY = _sc.epsilon_0
COULOMB_CONSTANT = 1.0 / (4.0 * _sc.pi * VACUUM_PERMITTIVITY)
ELECTRON_MASS_EV = 510998.95069  # mass of the electron species used by every fixture [eV]


def ev_to_kg(mass_ev):
    """constants.py:27-29."""
    return mass_ev * ELEMENTARY_CHARGE / SPEED_OF_LIGHT**2


def ev_c_to_si(p_ev_c):
    """constants.py:17-19."""
    return p_ev_c * ELEMENTARY_CHARGE / SPEED_OF_LIGHT


def pair_sum(targets, sources, q_targets, q_sources, live, soft):
    """Softened pair sum restricted to live-live pairs (forces.py:16-29).

    targets, sources: (G, E, 3); q_*: (G, E); live: (G, E) bool.
    Returns sum_j k q_i q_j (r_i - r_j) / (|r_i - r_j|^2 + a^2)^1.5.
    """
    sep = targets[:, :, np.newaxis, :] - sources[:, np.newaxis, :, :]
    r2 = np.sum(sep * sep, axis=-1) + soft**2
    r3 = r2 * np.sqrt(r2)
    both = live[:, :, np.newaxis] & live[:, np.newaxis, :]
    c = COULOMB_CONSTANT * q_targets[:, :, np.newaxis] * q_sources[:, np.newaxis, :] / r3
    c = np.where(both, c, 0.0)
    return np.einsum("gij,gijc->gic", c, sep)


def coulomb(pos, q, live, soft):
    """forces.py:32-57 -- real-real repulsion within each group."""
    return pair_sum(pos, pos, q, q, live, soft)


def flat_image(pos, q, live, z0, soft):
    """forces.py:60-98 -- images mirrored through the plane z = -z0."""
    mirrored = pos.copy()
    mirrored[..., 2] = -2.0 * z0 - pos[..., 2]
    return pair_sum(pos, mirrored, q, -q, live, soft)


def tip_images(pos, q, live, sphere_radius, soft, plane_z0):
    """forces.py:101-191 -- sphere image, plane image, plane image of the
    sphere image; sphere centred at the origin of ``pos``."""
    a = sphere_radius
    d2 = np.sum(pos * pos, axis=-1)
    d = np.sqrt(d2)
    d_ok = np.where(d > 0.0, d, a)
    shrink = (a * a) / (d_ok * d_ok)
    s_pos = pos * shrink[..., np.newaxis]
    s_q = -q * (a / d_ok)
    p_pos = pos.copy()
    p_pos[..., 2] = -2.0 * plane_z0 - pos[..., 2]
    ps_pos = s_pos.copy()
    ps_pos[..., 2] = -2.0 * plane_z0 - s_pos[..., 2]
    f1 = pair_sum(pos, s_pos, q, s_q, live, soft)
    f2 = pair_sum(pos, p_pos, q, -q, live, soft)
    f3 = pair_sum(pos, ps_pos, q, -s_q, live, soft)
    return f1 + f2 + f3


def gun_field(pos, Ez):
    """fields.py:43-59 -- uniform Ez for z >= 0, zero below."""
    out = np.zeros_like(pos)
    out[..., 2] = np.where(pos[..., 2] >= 0.0, Ez, 0.0)
    return out


def tip_field(pos, Ez, R):
    """fields.py:119-160 -- grounded sphere in a uniform field, outside
    r >= R(1-1e-6) and z >= 0, zero elsewhere."""
    x, y, z = pos[..., 0], pos[..., 1], pos[..., 2]
    r = np.sqrt(x * x + y * y + z * z)
    ok = (r >= R * (1.0 - 1e-6)) & (z >= 0.0)
    rs = np.where(ok, r, R)
    r3 = rs * rs * rs
    r5 = r3 * rs * rs
    R3 = R * R * R
    ex = 3.0 * Ez * R3 * x * z / r5
    ey = 3.0 * Ez * R3 * y * z / r5
    ez = Ez * (1.0 - R3 / r3 + 3.0 * R3 * z * z / r5)
    return np.where(ok[..., np.newaxis], np.stack([ex, ey, ez], axis=-1), 0.0)


def inside_sphere(pos, R):
    """geometry.py:238-248 -- the tip kill radius R(1-1e-6)."""
    rk = R * (1.0 - 1e-6)
    return np.sum(pos * pos, axis=-1) <= rk * rk


def well_contains(rho, z, R, H, bottom_fillet, rim_fillet):
    """bem/fields.py:89-136 -- inside (or on) the real well conductor."""
    eps = 1e-6 * R
    outside = rho >= R * (1.0 - 1e-6)
    solid = np.where(outside, z <= 0.0, z <= -H * (1.0 + 1e-6))
    if rim_fillet > 0.0:
        cr, cz = R + rim_fillet, -rim_fillet
        zone = (rho >= R - eps) & (rho <= R + rim_fillet + eps) & (z >= -rim_fillet - eps) & (z <= eps)
        solid = np.where(zone, np.hypot(rho - cr, z - cz) <= rim_fillet, solid)
    if bottom_fillet > 0.0:
        cr, cz = R - bottom_fillet, -H + bottom_fillet
        zone = ((rho <= R + eps) & (rho >= R - bottom_fillet - eps)
                & (z <= -H + bottom_fillet + eps) & (z >= -H - eps))
        solid = np.where(zone, np.hypot(rho - cr, z - cz) >= bottom_fillet, solid)
    return solid


def smoothstep_weight(z, z_lo, z_hi):
    """bem/image_charge.py:333-342 -- 1 below z_lo, 0 above z_hi, cubic between."""
    s = np.clip((z_hi - z) / (z_hi - z_lo), 0.0, 1.0)
    return s * s * (3.0 - 2.0 * s)
