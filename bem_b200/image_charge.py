"""BEM image-charge force on B200: the induced charge of an axisymmetric
grounded conductor, by azimuthal Fourier modes (bem/image_charge.py,
bem/ring_modes.py, bem/toroidal.py of the reference).

``ImageChargeSolution`` is the B200 counterpart of
``ImageChargeBEMSolution`` (bem/image_charge.py:457-620): the recessed image
profile, its per-mode collocation operators assembled on the GPU
(``spt_image_assemble``) and inverted once (torch.linalg.inv: cuSOLVER,
setup only), and the device tables ``spt_image_force`` reads on every call.
The profile builders restate bem/mesh.py's image surfaces (the recessed
hemisphere-on-plane, its mirror-doubled variant and the recessed well).
"""

import ctypes

import numpy as np

from . import _lib
from .mesh import arc_profile, graded_plane, points_for_length

GAUSS4_X, GAUSS4_W = np.polynomial.legendre.leggauss(4)
MIN_FILLET_SEGMENTS = 5  # bem/mesh.py:163-170: every 90-degree fillet gets at least 5 segments


def _cap(max_length, region):
    """bem/mesh.py:153-160: a region's length bound, tightened (never relaxed) by its own override."""
    return max_length if region is None else min(max_length, region)


def _fillet(major, tube, ph0, ph1, n):
    """Torus-tube slice (major + tube cos ph, tube sin ph), bem/mesh.py:118-124."""
    ph = np.linspace(ph0, ph1, n)
    return np.column_stack([major + tube * np.cos(ph), tube * np.sin(ph)])


def tip_image_profile(R, z0, plane_radius, max_length, cap_max_length=None, fillet_max_length=None,
                      plane_max_length=None, plane_growth=1.15):
    """bem/mesh.py:200-240: cap of radius R - z0, quarter-torus fillet (tube z0,
    major radius R) around the ridge, graded plane at z = -z0 out to plane_radius."""
    if not (0.0 < z0 < R):
        raise ValueError(f"z0 must satisfy 0 < z0 < R (got z0={z0!r}, R={R!r})")
    cap = arc_profile(0.0, 0.0, R - z0, 0.0, 0.5 * np.pi,
                      points_for_length((R - z0) * np.pi / 2, _cap(max_length, cap_max_length)))
    n_f = points_for_length(z0 * np.pi / 2, _cap(max_length, fillet_max_length), MIN_FILLET_SEGMENTS + 1)
    fillet = _fillet(R, z0, np.pi, 1.5 * np.pi, n_f)[1:]
    plane = graded_plane(R, plane_radius, -z0, _cap(max_length, plane_max_length), plane_growth)[1:]
    return np.concatenate([cap, fillet, plane], axis=0)


def tip_image_doubled_profile(R, z0, max_length, cap_max_length=None, fillet_max_length=None):
    """bem/mesh.py:243-315: cap + fillet of tip_image_profile, then the same
    piece reflected through z = -z0 (pole to pole, no plane)."""
    if not (0.0 < z0 < R):
        raise ValueError(f"z0 must satisfy 0 < z0 < R (got z0={z0!r}, R={R!r})")
    cap = arc_profile(0.0, 0.0, R - z0, 0.0, 0.5 * np.pi,
                      points_for_length((R - z0) * np.pi / 2, _cap(max_length, cap_max_length)))
    n_f = points_for_length(z0 * np.pi / 2, _cap(max_length, fillet_max_length), MIN_FILLET_SEGMENTS + 1)
    upper = np.concatenate([cap, _fillet(R, z0, np.pi, 1.5 * np.pi, n_f)[1:]], axis=0)
    lower = upper[-2::-1].copy()
    lower[:, 1] = -2.0 * z0 - lower[:, 1]
    return np.concatenate([upper, lower], axis=0)


def well_image_profile(R, H, z0, plane_radius, max_length, bottom_fillet_radius=None, rim_fillet_radius=None,
                       bottom_max_length=None, bottom_fillet_max_length=None, wall_max_length=None,
                       rim_fillet_max_length=None, plane_max_length=None, plane_growth=1.15):
    """bem/mesh.py:412-530: the well's surface eroded by z0 -- floor at
    -H - z0, bottom fillet of radius bottom + z0, wall at R + z0, the rim
    fillet of radius rim - z0 (a sharp mitre at (R + z0, -z0) when rim <= z0),
    graded plane at -z0."""
    if not (0.0 < z0 < min(R, H)):
        raise ValueError(f"z0 must satisfy 0 < z0 < min(R, H) (got z0={z0!r}, R={R!r}, H={H!r})")
    bf = 0.0 if bottom_fillet_radius is None else float(bottom_fillet_radius)
    rf = 0.0 if rim_fillet_radius is None else float(rim_fillet_radius)
    if bf < 0.0 or rf < 0.0:
        raise ValueError("fillet radii must be >= 0")
    top = max(rf, z0)
    if bf + top >= H:
        raise ValueError(f"bottom_fillet_radius + max(rim_fillet_radius, z0) must be < H (got {bf!r} + {top!r})")
    r_floor = R - bf
    n = points_for_length(r_floor, _cap(max_length, bottom_max_length))
    pieces = [np.column_stack([np.linspace(0.0, r_floor, n), np.full(n, -H - z0)])]
    n = points_for_length((bf + z0) * np.pi / 2, _cap(max_length, bottom_fillet_max_length), MIN_FILLET_SEGMENTS + 1)
    f = _fillet(r_floor, bf + z0, -0.5 * np.pi, 0.0, n)[1:]
    f[:, 1] += -H + bf
    pieces.append(f)
    z_lo, z_hi = -H + bf, -top
    n = points_for_length(z_hi - z_lo, _cap(max_length, wall_max_length))
    pieces.append(np.column_stack([np.full(n, R + z0), np.linspace(z_lo, z_hi, n)])[1:])
    if rf - z0 > 0.0:
        n = points_for_length((rf - z0) * np.pi / 2, _cap(max_length, rim_fillet_max_length),
                              MIN_FILLET_SEGMENTS + 1)
        f = _fillet(R + rf, rf - z0, np.pi, 0.5 * np.pi, n)[1:]
        f[:, 1] += -rf
        pieces.append(f)
        r0 = R + rf
    else:
        r0 = R + z0
    pieces.append(graded_plane(r0, plane_radius, -z0, _cap(max_length, plane_max_length), plane_growth)[1:])
    return np.concatenate(pieces, axis=0)


def quadrature(profile, n_subdiv):
    """bem/image_charge.py:418-452: n_subdiv sub-panels x Gauss-4 per
    segment -> rows rho, z, length weight, t along the segment, segment index."""
    p = np.asarray(profile, dtype=np.float64)
    p0, p1 = p[:-1], p[1:]
    length = np.linalg.norm(p1 - p0, axis=-1)
    k = np.arange(n_subdiv)
    t = ((k[:, None] + 0.5 * (GAUSS4_X[None, :] + 1.0)) / n_subdiv).reshape(-1)  # per segment, sub-panel major
    w = np.tile(0.5 * GAUSS4_W, n_subdiv)
    rho = p0[:, None, 0] + t[None, :] * (p1 - p0)[:, None, 0]
    z = p0[:, None, 1] + t[None, :] * (p1 - p0)[:, None, 1]
    lw = (length / n_subdiv)[:, None] * w[None, :]
    seg = np.repeat(np.arange(len(p0)), t.size).astype(np.float64)
    return np.stack([rho.reshape(-1), z.reshape(-1), lw.reshape(-1), np.tile(t, len(p0)), seg])


class ImageChargeSolution:
    """Per-mode operators and device tables of one image profile
    (ImageChargeBEMSolution.solve, bem/image_charge.py:493-496, with the
    cached inverse of image_charge.py:209-237).

    profile: (P, 2) recessed image profile; n_max: highest mode; d_lo, d_hi:
    mirror-charge blend distances [m]; n_subdiv: reconstruction sub-panels
    (image_force's default 4); mirror_symmetric: the profile is
    mirror-doubled through z = -z0 (phantom sources, see spt_image_force).
    A: optional precomputed operators (n_max+1, P, P); otherwise assembled on
    the device."""

    def __init__(self, profile, n_max, d_lo, d_hi, n_subdiv=4, mirror_symmetric=False, device="cuda",
                 refine_ratio=1.0, max_depth=20, A=None):
        import torch
        if not (0 <= int(n_max) <= _lib.IMAGE_MAX_MODES):
            raise ValueError(f"n_max must be in [0, {_lib.IMAGE_MAX_MODES}]")
        self.profile = np.asarray(profile, dtype=np.float64)
        self.n_max = int(n_max)
        self.d_lo, self.d_hi = float(d_lo), float(d_hi)
        self.n_subdiv = int(n_subdiv)
        self.mirror_symmetric = bool(mirror_symmetric)
        self.device = torch.device(device)
        P = len(self.profile)
        self.rho_floor = 1e-6 * max(float(np.max(self.profile[:, 0])), 1e-300)
        dev = self.device
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
        self.node = t(np.stack([np.maximum(self.profile[:, 0], self.rho_floor), self.profile[:, 1]]))
        p0 = self.profile[:-1]
        tan = self.profile[1:] - p0
        nrm = np.stack([-tan[:, 1], tan[:, 0]], -1)
        nrm = nrm / np.linalg.norm(nrm, axis=-1, keepdims=True)
        self.seg = t(np.stack([p0[:, 0], p0[:, 1], tan[:, 0], tan[:, 1], nrm[:, 0], nrm[:, 1]]))
        self.quad = t(quadrature(self.profile, self.n_subdiv))
        if A is None:
            A = self.assemble(refine_ratio, max_depth)
        else:
            A = t(np.asarray(A)[: self.n_max + 1, :P, :P])
        self.A = A
        self.a_inv = torch.linalg.inv(A).contiguous()
        self.struct = _lib.SptImage(n_nodes=P, n_max=self.n_max, n_quad=self.quad.shape[1],
                                    mirror_symmetric=int(self.mirror_symmetric), node=self.node.data_ptr(),
                                    seg=self.seg.data_ptr(), quad=self.quad.data_ptr(), a_inv=self.a_inv.data_ptr(),
                                    rho_floor=self.rho_floor, d_lo=self.d_lo, d_hi=self.d_hi)

    def assemble(self, refine_ratio=1.0, max_depth=20):
        """spt_image_assemble: (n_max+1, P, P) operators on the device."""
        import torch
        P = len(self.profile)
        dev = self.device
        pr = torch.as_tensor(np.ascontiguousarray(self.profile[:, 0]), device=dev)
        pz = torch.as_tensor(np.ascontiguousarray(self.profile[:, 1]), device=dev)
        gx = torch.as_tensor(GAUSS4_X, device=dev)
        gw = torch.as_tensor(GAUSS4_W, device=dev)
        A = torch.empty((self.n_max + 1, P, P), dtype=torch.float64, device=dev)
        with torch.cuda.device(dev):
            st = torch.cuda.current_stream(dev)
            rc = _lib.lib().spt_image_assemble(_lib.ptr(pr), _lib.ptr(pz), P, self.n_max, self.rho_floor,
                                               float(refine_ratio), int(max_depth), _lib.ptr(gx), _lib.ptr(gw),
                                               _lib.ptr(A), ctypes.c_void_p(st.cuda_stream))
            _lib.check(rc, "spt_image_assemble")
            st.synchronize()  # the argument tensors above are freed on return
        return A

    def force(self, pos, charge, active, group_offset, max_group_size, geometry=None, coulomb_constant=None,
              plummer_radius=1e-12, out=None, stream=None):
        """spt_image_force on device tensors: pos (N, 3) or x, y, z columns,
        charge (N,), active (N,) uint8, group_offset (G+1,) int64.  geometry:
        None (the solution-level ImageChargeBEMSolution.image_force) or an
        SptGeometry (the geometry-level force).  Returns (N, 3)."""
        import torch
        from .constants import COULOMB_CONSTANT
        k = COULOMB_CONSTANT if coulomb_constant is None else coulomb_constant
        dev = self.device
        x, y, z = (pos[:, i].contiguous() for i in range(3))
        n = x.shape[0]
        f = torch.empty((3, n), dtype=torch.float64, device=dev) if out is None else out
        st = torch.cuda.current_stream(dev) if stream is None else stream
        G = group_offset.shape[0] - 1
        rc = _lib.lib().spt_image_force(_lib.ptr(x), _lib.ptr(y), _lib.ptr(z), _lib.ptr(charge), _lib.ptr(active),
                                        _lib.ptr(group_offset), G, int(max_group_size), ctypes.byref(self.struct),
                                        None if geometry is None else ctypes.byref(geometry), float(k),
                                        float(plummer_radius), _lib.ptr(f[0]), _lib.ptr(f[1]), _lib.ptr(f[2]),
                                        ctypes.c_void_p(st.cuda_stream))
        _lib.check(rc, "spt_image_force")
        return f.T
