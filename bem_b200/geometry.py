"""Cathode geometries for the B200 backend.

Same constructor arguments and meaning as the reference's Geometry
subclasses (geometry.py:97-256, bem/geometry.py:58-885); each object turns
itself into the C-ABI parameter block (``to_struct``) and, for BEM shapes,
into device tables (``bem_tables``).  ``spec()`` returns the plain-data
description (kind, parameters, profile, sigma) -- the one format shared with
anything that needs to restate the physics independently.

``from_reference(geometry)`` converts a reference Geometry object (anything
with the reference's ``worker_args()`` tuple, geometry.py:61-65) without
importing the reference: for the BEM shapes it reads the already-solved
``field_solver.solution.profile/.sigma``, so no BEM solve is repeated.
"""

import numpy as np

from . import _lib
from . import mesh

DEFAULT_Z0 = 3.0e-9  # geometry.py:34


class Geometry:
    kind = None
    is_bem = False

    def to_struct(self, z_max=None):
        g = _lib.SptGeometry()
        g.kind = self.kind
        g.E_gun = float(self.E_gun)
        z0 = getattr(self, "z0", None)
        g.has_image = int(z0 is not None)
        g.z0 = float(z0) if z0 is not None else 0.0
        kz = getattr(self, "kill_z_below", None)
        g.has_kill_below = int(kz is not None)
        g.kill_z_below = float(kz) if kz is not None else 0.0
        g.has_z_max = int(z_max is not None)
        g.z_max = float(z_max) if z_max is not None else 0.0
        g.R = float(getattr(self, "R", 0.0))
        g.H = float(getattr(self, "H", 0.0))
        g.L = float(getattr(self, "L", 0.0))
        g.z_handoff = float(getattr(self, "z_handoff", 0.0))
        g.bottom_fillet = float(getattr(self, "bottom_fillet_radius", 0.0) or 0.0)
        g.rim_fillet = float(getattr(self, "rim_fillet_radius", 0.0) or 0.0)
        return g

    def bem_tables(self, device="cuda"):
        return None

    def field_accel_scale_field(self):
        return abs(self.E_gun)


class FlatCathode(Geometry):
    """geometry.FlatCathode: the plane z = 0 in a uniform field E_gun."""

    kind = _lib.GEOM_FLAT

    def __init__(self, E_gun, z0=DEFAULT_Z0, kill_z_below=0.0):
        self.E_gun = float(E_gun)
        self.z0 = z0
        self.kill_z_below = kill_z_below

    def spec(self):
        return dict(kind="flat", E_gun=self.E_gun, z0=self.z0, kill_z_below=self.kill_z_below)


class HemisphericalTip(Geometry):
    """geometry.HemisphericalTip: analytic field, exact 3-image force."""

    kind = _lib.GEOM_TIP

    def __init__(self, E_gun, R, z0=DEFAULT_Z0, kill_z_below=0.0):
        if z0 is not None and R <= z0:
            raise ValueError(f"R ({R!r}) must be greater than z0 ({z0!r})")
        self.E_gun = float(E_gun)
        self.R = float(R)
        self.z0 = z0
        self.kill_z_below = kill_z_below

    def spec(self):
        return dict(kind="tip", E_gun=self.E_gun, R=self.R, z0=self.z0, kill_z_below=self.kill_z_below)


class _BemGeometry(Geometry):
    is_bem = True

    def _set_solution(self, profile, sigma, n_subdiv):
        self.profile = np.asarray(profile, dtype=np.float64)
        self.sigma = np.asarray(sigma, dtype=np.float64)
        self.n_subdiv = int(n_subdiv)
        self._tables = {}

    def bem_tables(self, device="cuda"):
        import torch

        key = str(torch.device(device))
        if key not in self._tables:
            from .tables import BemTables
            self._tables[key] = BemTables(self.profile, self.sigma, self.n_subdiv, device=device)
        return self._tables[key]

    def _spec_common(self, kind):
        return dict(kind=kind, E_gun=self.E_gun, R=self.R, profile=self.profile, sigma=self.sigma,
                    n_subdiv=self.n_subdiv, z_handoff=self.z_handoff,
                    kill_z_below=getattr(self, "kill_z_below", None))


def _solve_or_take(profile, sigma, E_gun):
    if sigma is not None:
        return np.asarray(sigma, dtype=np.float64)
    from .bem_solve import solve_dirichlet
    return solve_dirichlet(profile, lambda rho, z: E_gun * z)


class HemisphericalTipBEMGeometry(_BemGeometry):
    """bem.geometry.HemisphericalTipBEMGeometry with z0=None (no image force):
    BEM field of the mirror-doubled sphere, blended with the flat fallback
    between z_handoff/2 and z_handoff."""

    kind = _lib.GEOM_TIP_BEM

    def __init__(self, E_gun, R, field_max_length=None, n_subdiv=8, z0=None, z_handoff=None, kill_z_below=0.0,
                 profile=None, sigma=None):
        if z0 is not None:
            raise NotImplementedError("z0 (the BEM image-charge solve) is not on the B200 path; use z0=None")
        self.E_gun = float(E_gun)
        self.R = float(R)
        self.z0 = None
        self.field_max_length = field_max_length
        self.z_handoff = 20.0 * self.R if z_handoff is None else float(z_handoff)
        self.kill_z_below = kill_z_below
        if profile is None:
            ml = self.R * np.pi / 39.0 if field_max_length is None else field_max_length
            profile = mesh.sphere_profile(self.R, mesh.points_for_length(self.R * np.pi, ml))
        self._set_solution(profile, _solve_or_take(profile, sigma, self.E_gun), n_subdiv)

    def spec(self):
        return self._spec_common("tip_bem")


class CylindricalWellBEMGeometry(_BemGeometry):
    """bem.geometry.CylindricalWellBEMGeometry with z0=None (image force zero,
    bem/geometry.py:786-790)."""

    kind = _lib.GEOM_WELL_BEM

    def __init__(self, E_gun, R, H, field_plane_radius=None, field_max_length=None, n_subdiv=8,
                 bottom_fillet_radius=None, rim_fillet_radius=None, z0=None, z_handoff=None,
                 profile=None, sigma=None, n_segments=None):
        if z0 is not None:
            raise NotImplementedError("z0 (the BEM image-charge solve) is not on the B200 path; use z0=None")
        self.E_gun = float(E_gun)
        self.R = float(R)
        self.H = float(H)
        self.z0 = None
        self.kill_z_below = None
        self.bottom_fillet_radius = bottom_fillet_radius
        self.rim_fillet_radius = rim_fillet_radius
        self.z_handoff = 20.0 * max(self.R, self.H) if z_handoff is None else float(z_handoff)
        self.field_plane_radius = self.z_handoff if field_plane_radius is None else float(field_plane_radius)
        if profile is None:
            kw = dict(bottom_fillet_radius=bottom_fillet_radius or 0.0, rim_fillet_radius=rim_fillet_radius or 0.0)
            if n_segments is not None:
                profile = mesh.well_profile_with_segments(self.R, self.H, self.field_plane_radius, n_segments, **kw)
            else:
                ml = min(self.R, self.H) / 19.0 if field_max_length is None else field_max_length
                profile = mesh.well_profile(self.R, self.H, self.field_plane_radius, ml, **kw)
        self._set_solution(profile, _solve_or_take(profile, sigma, self.E_gun), n_subdiv)

    def spec(self):
        s = self._spec_common("well_bem")
        s.update(H=self.H, bottom_fillet_radius=self.bottom_fillet_radius or 0.0,
                 rim_fillet_radius=self.rim_fillet_radius or 0.0, kill_z_below=None)
        return s


class PostTipBEMGeometry(_BemGeometry):
    """Hemisphere of radius R on a cylindrical post of height L, in a uniform
    field E_gun: BEM field of the mirror-doubled capsule (odd Dirichlet data
    E_gun*z makes the plane z = 0 an equipotential), blended with the flat
    fallback between z_handoff/2 and z_handoff (default 20 (L + R)); image
    force = forces.hemispherical_tip_image_force in the apex frame
    (z' = z - L, sphere radius R - z0, plane_z0 = L + z0); killed inside the
    conductor or at z <= kill_z_below."""

    kind = _lib.GEOM_POST_BEM

    def __init__(self, E_gun, R, L, n_cap=100, n_wall=900, n_subdiv=8, z0=DEFAULT_Z0, z_handoff=None,
                 kill_z_below=0.0, profile=None, sigma=None):
        if z0 is not None and R <= z0:
            raise ValueError("R must exceed z0")
        self.E_gun = float(E_gun)
        self.R = float(R)
        self.L = float(L)
        self.z0 = z0
        self.kill_z_below = kill_z_below
        self.z_handoff = 20.0 * (self.L + self.R) if z_handoff is None else float(z_handoff)
        if profile is None:
            profile = mesh.capsule_profile(self.R, self.L, n_cap, n_wall)
        self._set_solution(profile, _solve_or_take(profile, sigma, self.E_gun), n_subdiv)

    def spec(self):
        s = self._spec_common("post_bem")
        s.update(L=self.L, z0=self.z0)
        return s


def from_reference(geometry):
    """Convert a reference Geometry (geometry.FlatCathode, HemisphericalTip,
    bem.geometry.HemisphericalTipBEMGeometry / CylindricalWellBEMGeometry with
    z0=None) into the B200 equivalent, reusing its solved BEM density."""
    if isinstance(geometry, Geometry):
        return geometry
    args = geometry.worker_args()
    kind = args[0]
    if kind == "flat":
        _, E_gun, z0, kz = args
        return FlatCathode(E_gun, z0=z0, kill_z_below=kz)
    if kind == "hemispherical_tip":
        _, E_gun, R, z0, kz = args
        return HemisphericalTip(E_gun, R, z0=z0, kill_z_below=kz)
    if kind == "hemispherical_tip_bem":
        E_gun, R, fml, n_subdiv, z0 = args[1:6]
        z_handoff, kz = args[14], args[15]
        sol = geometry.field_solver.solution
        return HemisphericalTipBEMGeometry(E_gun, R, fml, n_subdiv, z0=z0, z_handoff=z_handoff, kill_z_below=kz,
                                           profile=sol.profile, sigma=sol.sigma)
    if kind == "cylindrical_well_bem":
        E_gun, R, H, fpr, fml, n_subdiv, bfr, rfr, z0 = args[1:10]
        z_handoff = args[20]
        sol = geometry.field_solver.solution
        return CylindricalWellBEMGeometry(E_gun, R, H, fpr, fml, n_subdiv, bfr, rfr, z0=z0, z_handoff=z_handoff,
                                          profile=sol.profile, sigma=sol.sigma)
    raise ValueError(f"geometry kind {kind!r} has no B200 equivalent")
