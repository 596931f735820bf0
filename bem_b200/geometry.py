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
            t = BemTables(self.profile, self.sigma, self.n_subdiv, device=device)
            if getattr(self, "image_profile", None) is not None:
                t.attach_image(self.image_solution(device))
            self._tables[key] = t
        return self._tables[key]

    def image_solution(self, device="cuda"):
        """The image-charge solve of a geometry built with z0 (per device,
        built on first use: operators assembled on the GPU, inverted once)."""
        import torch

        from .image_charge import ImageChargeSolution
        key = str(torch.device(device))
        cache = self.__dict__.setdefault("_image", {})
        if key not in cache:
            cache[key] = ImageChargeSolution(self.image_profile, self.image_n_max, self.image_d_lo * self.R,
                                             self.image_d_hi * self.R,
                                             mirror_symmetric=getattr(self, "image_mirror_symmetric", False),
                                             device=device)
        return cache[key]

    def _image_spec(self, s):
        if getattr(self, "image_profile", None) is not None:
            s.update(z0=self.z0, image_profile=self.image_profile, image_n_max=self.image_n_max,
                     image_d_lo=self.image_d_lo, image_d_hi=self.image_d_hi,
                     image_mirror_symmetric=bool(getattr(self, "image_mirror_symmetric", False)))
        return s

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
    """bem.geometry.HemisphericalTipBEMGeometry (bem/geometry.py:58-507):
    BEM field of the mirror-doubled sphere, blended with the flat fallback
    between z_handoff/2 and z_handoff.  With z0 the image force is the BEM
    image-charge solve on the recessed surface (cap of radius R - z0, ridge
    fillet, plane at -z0 out to 5 R; or, with image_mirror_symmetric, that
    surface mirror-doubled through -z0), blended with the flat plane image
    at z0 the same way (image_charge.py via spt_image_force, and inside
    every stage of the trace).  profile / sigma / image_profile: take these
    instead of meshing (and solving) here."""

    kind = _lib.GEOM_TIP_BEM

    def __init__(self, E_gun, R, field_max_length=None, n_subdiv=8, z0=None, image_max_length=None,
                 image_cap_max_length=None, image_fillet_max_length=None, image_plane_max_length=None,
                 image_n_max=16, image_d_lo=0.1, image_d_hi=0.5, image_mirror_symmetric=False, z_handoff=None,
                 kill_z_below=0.0, profile=None, sigma=None, image_profile=None):
        from . import image_charge as ic
        self.E_gun = float(E_gun)
        self.R = float(R)
        self.z0 = z0
        self.image_profile = None
        if z0 is not None:
            z0 = float(z0)
            ml = (self.R - z0) * np.pi / 2.0 / 29.0 if image_max_length is None else float(image_max_length)
            self.image_max_length = ml
            self.image_n_max, self.image_d_lo, self.image_d_hi = int(image_n_max), float(image_d_lo), float(image_d_hi)
            self.image_mirror_symmetric = bool(image_mirror_symmetric)
            if image_profile is not None:
                self.image_profile = np.asarray(image_profile, dtype=np.float64)
            elif self.image_mirror_symmetric:
                self.image_profile = ic.tip_image_doubled_profile(self.R, z0, ml, image_cap_max_length,
                                                                  image_fillet_max_length)
            else:
                self.image_profile = ic.tip_image_profile(self.R, z0, 5.0 * self.R, ml, image_cap_max_length,
                                                          image_fillet_max_length, image_plane_max_length)
        self.field_max_length = field_max_length
        self.z_handoff = 20.0 * self.R if z_handoff is None else float(z_handoff)
        self.kill_z_below = kill_z_below
        if profile is None:
            ml = self.R * np.pi / 39.0 if field_max_length is None else field_max_length
            profile = mesh.sphere_profile(self.R, mesh.points_for_length(self.R * np.pi, ml))
        self._set_solution(profile, _solve_or_take(profile, sigma, self.E_gun), n_subdiv)

    def spec(self):
        return self._image_spec(self._spec_common("tip_bem"))


class CylindricalWellBEMGeometry(_BemGeometry):
    """bem.geometry.CylindricalWellBEMGeometry (bem/geometry.py:510-885).
    Without z0 the image force is zero (bem/geometry.py:786-790); with z0
    both corners are rounded by default (bem/geometry.py:661-680) and the
    image force is the BEM image-charge solve on the well's surface eroded
    by z0, blended with the flat plane image (spt_image_force).  profile /
    sigma / image_profile: take these instead of meshing (and solving)."""

    kind = _lib.GEOM_WELL_BEM

    def __init__(self, E_gun, R, H, field_plane_radius=None, field_max_length=None, n_subdiv=8,
                 bottom_fillet_radius=None, rim_fillet_radius=None, z0=None, image_plane_radius=None,
                 image_max_length=None, image_bottom_max_length=None, image_fillet_max_length=None,
                 image_wall_max_length=None, image_rim_fillet_max_length=None, image_plane_max_length=None,
                 image_n_max=16, image_d_lo=0.1, image_d_hi=0.5, z_handoff=None, profile=None, sigma=None,
                 n_segments=None, image_profile=None):
        from . import image_charge as ic
        self.E_gun = float(E_gun)
        self.R = float(R)
        self.H = float(H)
        self.z0 = z0
        self.kill_z_below = None
        self.image_profile = None
        if z0 is not None:
            room = min(0.5 * float(z0), 0.2 * (self.H - float(z0)))
            bottom_fillet_radius = room if bottom_fillet_radius is None else float(bottom_fillet_radius)
            rim_fillet_radius = float(z0) + room if rim_fillet_radius is None else float(rim_fillet_radius)
            self.image_n_max, self.image_d_lo, self.image_d_hi = int(image_n_max), float(image_d_lo), float(image_d_hi)
            self.image_plane_radius = 5.0 * max(self.R, self.H) if image_plane_radius is None else float(
                image_plane_radius)
            self.image_max_length = min(self.R, self.H) / 14.0 if image_max_length is None else float(image_max_length)
            if image_profile is not None:
                self.image_profile = np.asarray(image_profile, dtype=np.float64)
            else:
                self.image_profile = ic.well_image_profile(
                    self.R, self.H, float(z0), self.image_plane_radius, self.image_max_length, bottom_fillet_radius,
                    rim_fillet_radius, image_bottom_max_length, image_fillet_max_length, image_wall_max_length,
                    image_rim_fillet_max_length, image_plane_max_length)
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
        return self._image_spec(s)


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
    bem.geometry.HemisphericalTipBEMGeometry / CylindricalWellBEMGeometry)
    into the B200 equivalent, reusing its solved BEM density and its image
    profile (the image operators are assembled again on the device)."""
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
        E_gun, R, fml, n_subdiv, z0, iml, icml, ifml, ipml, n_max, d_lo, d_hi, sym, z_handoff, kz = args[1:16]
        sol = geometry.field_solver.solution
        img = geometry.image_solution
        return HemisphericalTipBEMGeometry(E_gun, R, fml, n_subdiv, z0, iml, icml, ifml, ipml, n_max, d_lo, d_hi, sym,
                                           z_handoff=z_handoff, kill_z_below=kz, profile=sol.profile, sigma=sol.sigma,
                                           image_profile=None if img is None else img.profile)
    if kind == "cylindrical_well_bem":
        (E_gun, R, H, fpr, fml, n_subdiv, bfr, rfr, z0, ipr, iml, ibml, ifml, iwml, irml, ipml, n_max, d_lo,
         d_hi, z_handoff) = args[1:21]
        sol = geometry.field_solver.solution
        img = geometry.image_solution
        return CylindricalWellBEMGeometry(E_gun, R, H, fpr, fml, n_subdiv, bfr, rfr, z0, ipr, iml, ibml, ifml, iwml,
                                          irml, ipml, n_max, d_lo, d_hi, z_handoff=z_handoff, profile=sol.profile,
                                          sigma=sol.sigma, image_profile=None if img is None else img.profile)
    raise ValueError(f"geometry kind {kind!r} has no B200 equivalent")
