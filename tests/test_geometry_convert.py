"""from_reference: a reference Geometry (any object with the reference's
worker_args() tuple, bem/geometry.py:438-469, 814-837, and its solved
field_solver.solution / image_solution) becomes the B200 geometry with the
same parameters, reusing the reference's density and image profile.  CPU
only: stand-in objects carry exactly the attributes the conversion reads."""

import numpy as np

from bem_b200 import _lib
from bem_b200 import geometry as bg
from bem_b200 import image_charge as bic


class _Solution:
    def __init__(self, profile, sigma=None):
        self.profile = profile
        self.sigma = sigma


class _RefGeometry:
    def __init__(self, args, profile, sigma, image_profile):
        self._args = args
        self.field_solver = type("F", (), {"solution": _Solution(profile, sigma)})()
        self.image_solution = None if image_profile is None else _Solution(image_profile)

    def worker_args(self):
        return self._args


def _sphere(R, n=31):
    th = np.linspace(0.0, np.pi, n)
    return np.column_stack([R * np.sin(th), R * np.cos(th)])


def test_tip_with_image_plane():
    R, z0 = 50e-9, 3e-9
    prof = _sphere(R)
    img = bic.tip_image_doubled_profile(R, z0, R / 40)
    args = ("hemispherical_tip_bem", -1e8, R, R * np.pi / 30, 8, z0, R / 40, None, None, None, 12, 0.2, 0.6, True,
            1.5e-6, 0.0)
    g = bg.from_reference(_RefGeometry(args, prof, np.ones(len(prof)), img))
    assert isinstance(g, bg.HemisphericalTipBEMGeometry)
    np.testing.assert_array_equal(g.image_profile, img)
    assert (g.image_n_max, g.image_d_lo, g.image_d_hi, g.image_mirror_symmetric) == (12, 0.2, 0.6, True)
    s = g.to_struct()
    assert (s.kind, s.has_image, s.z0, s.z_handoff) == (_lib.GEOM_TIP_BEM, 1, z0, 1.5e-6)
    assert g.spec()["image_mirror_symmetric"] is True


def test_tip_without_image_plane():
    R = 50e-9
    prof = _sphere(R)
    args = ("hemispherical_tip_bem", -1e8, R, None, 8, None, None, None, None, None, 16, 0.1, 0.5, False, 1e-6, 0.0)
    g = bg.from_reference(_RefGeometry(args, prof, np.ones(len(prof)), None))
    assert g.image_profile is None and g.to_struct().has_image == 0
    assert "image_profile" not in g.spec()


def test_well_with_image_plane():
    R, H, z0 = 200e-9, 100e-9, 3e-9
    room = min(0.5 * z0, 0.2 * (H - z0))
    img = bic.well_image_profile(R, H, z0, 5 * R, min(R, H) / 14, room, z0 + room)
    prof = np.column_stack([np.linspace(0, 4 * R, 9), np.zeros(9)])
    args = ("cylindrical_well_bem", -1e7, R, H, 4 * R, None, 8, room, z0 + room, z0, 5 * R, min(R, H) / 14, None, None,
            None, None, None, 16, 0.1, 0.5, 4e-6)
    g = bg.from_reference(_RefGeometry(args, prof, np.ones(9), img))
    assert isinstance(g, bg.CylindricalWellBEMGeometry)
    np.testing.assert_array_equal(g.image_profile, img)
    s = g.to_struct()
    assert (s.kind, s.has_image, s.bottom_fillet, s.rim_fillet) == (_lib.GEOM_WELL_BEM, 1, room, z0 + room)
