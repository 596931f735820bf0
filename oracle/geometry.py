"""Oracle: field / image force / kill mask per geometry spec, and the stage
acceleration (geometry.py:265-322, bem/geometry.py:44-55, 319-344, 429-436,
779-812).  Test infrastructure only -- see ``oracle/__init__.py``.

A *spec* is a plain dict (``kind`` plus parameters; BEM kinds also carry
``profile``, ``sigma``, ``n_subdiv``, ``z_handoff``).  Kinds:

* ``flat``     -- geometry.FlatCathode
* ``tip``      -- geometry.HemisphericalTip (analytic field, 3-image force)
* ``tip_bem``  -- bem.geometry.HemisphericalTipBEMGeometry; with ``z0`` the
  spec also carries ``image_profile``, ``image_n_max``, ``image_d_lo``,
  ``image_d_hi``, ``image_mirror_symmetric`` (optional ``image_A``) for the
  BEM image-charge force
* ``well_bem`` -- bem.geometry.CylindricalWellBEMGeometry (the same image keys)
* ``post_bem`` -- hemisphere of radius R on a cylindrical post of height L:
  BEM field of the mirror-doubled capsule blended with the flat fallback,
  and the 3-image force of forces.hemispherical_tip_image_force applied in
  the apex frame (z' = z - L, plane_z0 = L + z0).  Composed only from
  reference functions; no reference class of its own.
"""

import numpy as np

from . import bem as _bem
from . import physics as _ph


def _post_inside(pos, R, L):
    rk = R * (1.0 - 1e-6)
    x, y, z = pos[..., 0], pos[..., 1], pos[..., 2]
    shank = (x * x + y * y <= rk * rk) & (z <= L)
    zc = z - L
    cap = x * x + y * y + zc * zc <= rk * rk
    return shank | cap


def field(spec, pos):
    k = spec["kind"]
    Ez = spec["E_gun"]
    if k == "flat":
        return _ph.gun_field(pos, Ez)
    if k == "tip":
        return _ph.tip_field(pos, Ez, spec["R"])
    z = pos[..., 2]
    if k == "tip_bem":
        r = np.linalg.norm(pos, axis=-1)
        ok = (r >= spec["R"] * (1.0 - 1e-6)) & (z >= 0.0)
    elif k == "well_bem":
        rho = np.linalg.norm(pos[..., :2], axis=-1)
        ok = ~_ph.well_contains(rho, z, spec["R"], spec["H"],
                                spec.get("bottom_fillet_radius") or 0.0, spec.get("rim_fillet_radius") or 0.0)
    elif k == "post_bem":
        ok = (~_post_inside(pos, spec["R"], spec["L"])) & (z >= 0.0)
    else:
        raise ValueError(f"unknown geometry kind {k!r}")
    uniform = np.zeros_like(pos)
    uniform[..., 2] = Ez
    pert = _bem.field(pos, spec["profile"], spec["sigma"], spec.get("n_subdiv", 8))
    near = np.where(ok[..., None], uniform + pert, 0.0)
    far = _ph.gun_field(pos, Ez)
    zh = spec["z_handoff"]
    w = _ph.smoothstep_weight(z, 0.5 * zh, zh)
    return w[..., None] * near + (1.0 - w[..., None]) * far


def image_force(spec, pos, q, live, soft):
    k = spec["kind"]
    z0 = spec.get("z0")
    if z0 is None:
        return np.zeros_like(pos)
    if k == "flat":
        return _ph.flat_image(pos, q, live, z0, soft)
    if k == "tip":
        return _ph.tip_images(pos, q, live, spec["R"] - z0, soft, plane_z0=z0)
    if k == "post_bem":
        shifted = pos.copy()
        shifted[..., 2] = pos[..., 2] - spec["L"]
        return _ph.tip_images(shifted, q, live, spec["R"] - z0, soft, plane_z0=spec["L"] + z0)
    if k in ("tip_bem", "well_bem"):
        # bem/geometry.py:326-344, 780-797: the BEM image-charge solve (oracle/image_charge.py)
        from . import image_charge as _ic
        sol = spec.get("_image_oracle")
        if sol is None:
            sol = _ic.ImageSolution(spec["image_profile"], spec["image_n_max"], A=spec.get("image_A"))
            spec["_image_oracle"] = sol
        return _ic.geometry_image_force(sol, pos, q, live, z0, spec["R"], spec["image_d_lo"], spec["image_d_hi"],
                                        z_handoff=spec["z_handoff"],
                                        mirror_symmetric=spec.get("image_mirror_symmetric", False), soft=soft)
    raise ValueError(f"unknown geometry kind {k!r}")


def kill_mask(spec, pos, z_max=None):
    """geometry.py:152-155, 238-248, 304-322; bem/geometry.py:429-436, 803-812."""
    k = spec["kind"]
    kz = spec.get("kill_z_below", 0.0)
    z = pos[..., 2]
    if k == "flat":
        m = np.zeros(pos.shape[:-1], dtype=bool) if kz is None else z <= kz
    elif k in ("tip", "tip_bem"):
        m = _ph.inside_sphere(pos, spec["R"])
        if kz is not None:
            m = m | (z <= kz)
    elif k == "well_bem":
        rho = np.linalg.norm(pos[..., :2], axis=-1)
        m = _ph.well_contains(rho, z, spec["R"], spec["H"],
                              spec.get("bottom_fillet_radius") or 0.0, spec.get("rim_fillet_radius") or 0.0)
    elif k == "post_bem":
        m = _post_inside(pos, spec["R"], spec["L"])
        if kz is not None:
            m = m | (z <= kz)
    else:
        raise ValueError(k)
    if z_max is not None:
        m = m | (z >= z_max)
    return m


def make_accel(spec, charge, mass, charge_to_mass, soft):
    """geometry.py:265-301 -- accel(pos, vel, active, group_idx)."""

    def accel(pos, vel, active, gidx):
        c = charge[gidx]
        m = mass[gidx]
        a_field = charge_to_mass * field(spec, pos)
        a_coul = 0.0 if pos.shape[1] == 1 else _ph.coulomb(pos, c, active, soft) / m[..., None]
        a_img = image_force(spec, pos, c, active, soft) / m[..., None]
        return np.where(active[..., None], a_field + a_coul + a_img, 0.0)

    return accel


def make_kill(spec, z_max=None):
    return lambda pos: kill_mask(spec, pos, z_max)
