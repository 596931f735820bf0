"""Generating profiles (rho, z) for the axisymmetric BEM geometries.

A profile is an (n, 2) float64 array of nodes ordered along the surface so
that the left normal of every segment, (-dz, drho)/|.|, points into the
vacuum (the convention of bem/axisymmetric.py:329-338).  Pure NumPy.

* ``sphere_profile``  -- full sphere pole to pole (the mirror-doubled
  hemisphere tip, bem/fields.py:178-184).
* ``capsule_profile`` -- hemisphere of radius R on a cylindrical post of
  height L, mirror-doubled through z = 0: apex cap, shank down to z = -L,
  mirrored cap.  Odd Dirichlet data Ez*z on this closed surface gives a
  solution that vanishes on the plane z = 0, the same symmetry argument the
  reference uses for the hemisphere (bem/fields.py:21-33).
* ``well_profile``    -- cylindrical recess of radius R and depth H cut into
  the plane z = 0: floor, wall, optional corner fillets, graded plane out to
  ``plane_radius`` (the shape of bem/mesh.py:317-417).
"""

import numpy as np


def points_for_length(arc, max_length, min_points=2):
    """Node count so that each of the (n-1) segments is at most max_length."""
    if max_length <= 0.0:
        raise ValueError(f"segment length bound {max_length!r} is not > 0")
    return max(min_points, max(1, int(np.ceil(arc / max_length))) + 1)


def arc_profile(center_rho, center_z, radius, th0, th1, n):
    """Nodes (center_rho + radius sin th, center_z + radius cos th), th0..th1."""
    th = np.linspace(th0, th1, n)
    return np.column_stack([center_rho + radius * np.sin(th), center_z + radius * np.cos(th)])


def sphere_profile(R, n_theta):
    return arc_profile(0.0, 0.0, R, 0.0, np.pi, n_theta)


def capsule_profile(R, L, n_cap, n_wall):
    """2*n_cap + 2*n_wall segments: apex cap (n_cap), shank from z = L to
    z = 0 (n_wall) and its mirror images below z = 0."""
    cap = arc_profile(0.0, L, R, 0.0, 0.5 * np.pi, n_cap + 1)
    wall = np.column_stack([np.full(n_wall + 1, R), np.linspace(L, 0.0, n_wall + 1)])
    upper = np.concatenate([cap, wall[1:]], axis=0)
    lower = upper[-2::-1].copy()
    lower[:, 1] = -lower[:, 1]
    prof = np.concatenate([upper, lower], axis=0)
    prof[np.abs(prof[:, 1]) < 1e-300, 1] = 0.0
    return prof


def graded_plane(r0, r1, z, first, growth=1.15):
    """Annulus nodes from r0 to r1 with spacing starting at ``first`` and
    growing geometrically; a last gap shorter than half the previous one is
    merged into it."""
    r = [r0]
    step = first
    while r[-1] + step < r1:
        r.append(r[-1] + step)
        step *= growth
    if len(r) > 1 and r1 - r[-1] < 0.5 * (r[-1] - r[-2]):
        r[-1] = r1
    else:
        r.append(r1)
    r = np.asarray(r, dtype=float)
    return np.column_stack([r, np.full_like(r, z)])


def well_profile(R, H, plane_radius, max_length, bottom_fillet_radius=0.0, rim_fillet_radius=0.0,
                 plane_growth=1.15, min_fillet_segments=5):
    bf = float(bottom_fillet_radius or 0.0)
    rf = float(rim_fillet_radius or 0.0)
    if bf < 0.0 or rf < 0.0 or bf + rf >= H:
        raise ValueError("fillet radii must be >= 0 with bottom + rim < H")
    r_floor = R - bf
    pieces = [np.column_stack([np.linspace(0.0, r_floor, points_for_length(r_floor, max_length)),
                               np.full(points_for_length(r_floor, max_length), -H)])]
    if bf > 0.0:
        n = points_for_length(bf * np.pi / 2, max_length, min_fillet_segments + 1)
        ph = np.linspace(-0.5 * np.pi, 0.0, n)[1:]
        pieces.append(np.column_stack([r_floor + bf * np.cos(ph), -H + bf + bf * np.sin(ph)]))
    z_lo, z_hi = -H + bf, -rf
    n = points_for_length(z_hi - z_lo, max_length)
    pieces.append(np.column_stack([np.full(n, R), np.linspace(z_lo, z_hi, n)])[1:])
    if rf > 0.0:
        n = points_for_length(rf * np.pi / 2, max_length, min_fillet_segments + 1)
        ph = np.linspace(np.pi, 0.5 * np.pi, n)[1:]
        pieces.append(np.column_stack([R + rf + rf * np.cos(ph), -rf + rf * np.sin(ph)]))
    pieces.append(graded_plane(R + rf, plane_radius, 0.0, max_length, plane_growth)[1:])
    return np.concatenate(pieces, axis=0)


def well_profile_with_segments(R, H, plane_radius, n_segments, **kw):
    """well_profile with max_length chosen (bisection) so the profile has
    n_segments segments, or the nearest count above it."""
    lo, hi = 1e-6 * min(R, H), max(R, H)
    for _ in range(200):
        mid = np.sqrt(lo * hi)
        n = len(well_profile(R, H, plane_radius, mid, **kw)) - 1
        if n > n_segments:
            lo = mid
        else:
            hi = mid
    return well_profile(R, H, plane_radius, hi, **kw)
