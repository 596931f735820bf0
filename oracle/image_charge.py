"""Oracle: the BEM image-charge force by azimuthal Fourier modes (float64,
NumPy/SciPy).

Test infrastructure only -- see ``oracle/__init__.py``.  Restates:

* ``bem/toroidal.py:180-219`` (+ ``:120-178``): Q_{m-1/2}(chi) and dQ/dchi,
  elliptic seeds for m = 0, 1, upward recurrence where M*eta <= 1, downward
  ratio recurrence elsewhere (per-element padding, as the reference's
  device kernel does, ``toroidal.py:43-88``);
* ``bem/ring_modes.py:66-158``: the single-layer mode kernel Phi_m and its
  (rho, z) gradient, and the point-charge excitation g_m;
* ``bem/image_charge.py:333-495``: mirror-charge weight and reflection, the
  per-mode collocation operators (adaptive bisection, Gauss-4 leaves), the
  fixed reconstruction quadrature;
* ``bem/image_charge.py:987-1056, 1296-1347, 1369-1395``
  (``ImageChargeBEMSolution.image_force``): the joint per-group solve,
  field reconstruction and the direct mirror-charge term;
* ``bem/geometry.py:326-415, 780-797``: the geometry-level image force
  (flat fallback blended above z_handoff/2; mirror-doubled profile with
  phantom sources).
"""

import numpy as np

from .bem import GAUSS4_W, GAUSS4_X, ellip_k_e_complement, segments
from .physics import VACUUM_PERMITTIVITY, flat_image, smoothstep_weight


# ---------------------------------------------------------------------------
# toroidal harmonics

def toroidal_q(chi, n_max, pad_min=50, pad_const=40.0):
    """Q_{n-1/2}(chi), dQ_{n-1/2}/dchi for n = 0..n_max, shape (n_max+1,) +
    chi.shape (bem/toroidal.py:180-219).  chi is clipped to the next double
    above 1; M = max(n_max, 1) modes are built and the first n_max+1
    returned."""
    if not isinstance(n_max, (int, np.integer)) or n_max < 0:
        raise ValueError("n_max must be a nonnegative integer")
    chi = np.maximum(np.asarray(chi, dtype=float), np.nextafter(1.0, 2.0))
    shape = chi.shape
    c = chi.reshape(-1)
    M = max(int(n_max), 1)
    # elliptic seeds (toroidal.py:167-176): K, E of the complementary parameter
    K, E = ellip_k_e_complement((c - 1.0) / (c + 1.0))
    root = np.sqrt(2.0 / (c + 1.0))
    q0 = root * K
    q1 = c * q0 - np.sqrt(2.0 * (c + 1.0)) * E
    dq0 = -root * E / (2.0 * (c - 1.0))
    eta = np.arccosh(c)
    q = np.empty((M + 1, c.size))
    q[0] = q0
    up = M * eta <= 1.0
    if up.any():
        cu = c[up]
        prev, cur = q0[up], q1[up]
        q[1, up] = cur
        for n in range(1, M):
            nxt = (2.0 * n * cu * cur - (n - 0.5) * prev) / (n + 0.5)
            q[n + 1, up] = nxt
            prev, cur = cur, nxt
    down = ~up
    if down.any():
        cd = c[down]
        pad = np.maximum(pad_min, np.ceil(pad_const / eta[down])).astype(np.int64)
        ratios = np.ones((M + 1, cd.size))
        r_next = np.zeros(cd.size)
        top = M + pad
        for n in range(int(top.max()), 0, -1):
            live = n <= top  # each element starts its own descent at M + pad
            rn = (n - 0.5) / (2.0 * n * cd - (n + 0.5) * r_next)
            r_next = np.where(live, rn, 0.0)
            if n <= M:
                ratios[n] = r_next
        val = q0[down].copy()
        for n in range(1, M + 1):
            val = val * ratios[n]
            q[n, down] = val
    dq = np.empty_like(q)
    dq[0] = dq0
    denom = (c - 1.0) * (c + 1.0)
    for n in range(1, M + 1):
        dq[n] = (n - 0.5) * (c * q[n] - q[n - 1]) / denom
    return q[: n_max + 1].reshape((n_max + 1,) + shape), dq[: n_max + 1].reshape((n_max + 1,) + shape)


# ---------------------------------------------------------------------------
# mode kernels (bem/ring_modes.py)

def chi_of(rho, z, a, za):
    """ring_modes.py:81-89: 1 + ((rho-a)^2 + (z-za)^2) / (2 rho a)."""
    return 1.0 + ((rho - a) ** 2 + (z - za) ** 2) / (2.0 * rho * a)


def mode_prefactors(n_max):
    """ring_modes.py:92-95: C_0 = 1/(4 pi^2), C_m = 1/(2 pi^2)."""
    c = np.full(n_max + 1, 1.0 / (2.0 * np.pi ** 2))
    c[0] = 1.0 / (4.0 * np.pi ** 2)
    return c


def ring_potential_modes(rho, z, a, za, n_max):
    """ring_modes.py:98-113: Phi_m = sqrt(a/rho) Q_{m-1/2}(chi) / (2 pi)."""
    rho, z, a, za = np.broadcast_arrays(*(np.asarray(v, dtype=float) for v in (rho, z, a, za)))
    q, _ = toroidal_q(chi_of(rho, z, a, za), n_max)
    return np.sqrt(a / rho)[None] * q / (2.0 * np.pi)


def ring_field_modes(rho, z, a, za, n_max):
    """ring_modes.py:116-135, 138-158: (Phi_m, dPhi_m/drho, dPhi_m/dz)."""
    rho, z, a, za = np.broadcast_arrays(*(np.asarray(v, dtype=float) for v in (rho, z, a, za)))
    q, dq = toroidal_q(chi_of(rho, z, a, za), n_max)
    dchi_drho = (rho ** 2 - a ** 2 - (z - za) ** 2) / (2.0 * a * rho ** 2)
    dchi_dz = (z - za) / (a * rho)
    s = np.sqrt(a / rho)[None]
    phi = s * q / (2.0 * np.pi)
    dphi_drho = (-s / (2.0 * rho[None]) * q + s * dq * dchi_drho[None]) / (2.0 * np.pi)
    dphi_dz = s * dq * dchi_dz[None] / (2.0 * np.pi)
    return phi, dphi_drho, dphi_dz


def point_charge_potential_modes(rho, z, rho0, z0, n_max):
    """ring_modes.py:138-158 (excitation): g_m = C_m Q_{m-1/2}(chi) / sqrt(rho rho0)."""
    rho, z, rho0, z0 = np.broadcast_arrays(*(np.asarray(v, dtype=float) for v in (rho, z, rho0, z0)))
    q, _ = toroidal_q(chi_of(rho, z, rho0, z0), n_max)
    c = mode_prefactors(n_max).reshape((n_max + 1,) + (1,) * rho.ndim)
    return c * q / np.sqrt(rho * rho0)[None]


# ---------------------------------------------------------------------------
# mirror charge (bem/image_charge.py:333-378)

def image_charge_weight(d, d_lo, d_hi):
    """image_charge.py:333-342: 1 at d <= d_lo, 0 at d >= d_hi, cubic smoothstep."""
    if d_hi <= d_lo:
        raise ValueError(f"d_hi must be > d_lo (got d_lo={d_lo!r}, d_hi={d_hi!r})")
    t = np.clip((d_hi - np.asarray(d, dtype=float)) / (d_hi - d_lo), 0.0, 1.0)
    return t * t * (3.0 - 2.0 * t)


def closest_on_profile(rho, z, seg):
    """image_charge.py:587-620 on bem/axisymmetric.py:341-389: closest point,
    unit tangent, unit normal and distance, first strict minimum over segments."""
    p0, tan, nrm = seg["p0"], seg["tangent"], seg["normal"]
    best = np.full(rho.shape, np.inf)
    arg = np.zeros(rho.shape, dtype=np.int64)
    tb = np.zeros(rho.shape)
    for j in range(len(p0)):
        ab2 = float(tan[j, 0] * tan[j, 0] + tan[j, 1] * tan[j, 1])
        t = np.clip(((rho - p0[j, 0]) * tan[j, 0] + (z - p0[j, 1]) * tan[j, 1]) / ab2, 0.0, 1.0)
        d2 = (rho - (p0[j, 0] + t * tan[j, 0])) ** 2 + (z - (p0[j, 1] + t * tan[j, 1])) ** 2
        better = d2 < best
        best = np.where(better, d2, best)
        arg = np.where(better, j, arg)
        tb = np.where(better, t, tb)
    closest = p0[arg] + tb[:, None] * tan[arg]
    unit = tan[arg] / np.linalg.norm(tan[arg], axis=-1, keepdims=True)
    return closest, unit, nrm[arg], np.sqrt(best)


def mirror_points(rho, z, closest, unit_t, unit_n):
    """image_charge.py:364-378: reflection through the tangent line in the
    meridian plane; side = -1 where the image crosses the axis."""
    dr, dz = rho - closest[:, 0], z - closest[:, 1]
    d_t = dr * unit_t[:, 0] + dz * unit_t[:, 1]
    d_n = dr * unit_n[:, 0] + dz * unit_n[:, 1]
    r_img = closest[:, 0] + d_t * unit_t[:, 0] - d_n * unit_n[:, 0]
    z_img = closest[:, 1] + d_t * unit_t[:, 1] - d_n * unit_n[:, 1]
    side = np.where(r_img < 0.0, -1.0, 1.0)
    return np.abs(r_img), z_img, side


# ---------------------------------------------------------------------------
# one-time operators

def _leaves(rho_f, z_f, p0, p1, refine_ratio, max_depth):
    """image_charge.py:379-411, the bisection only: the leaves [ta, tb] of the
    segment p0 -> p1 (parameter t of the whole segment) that the reference
    integrates with Gauss-4 for the field point (rho_f, z_f).  The subdivision
    decision (length > ratio * distance to the midpoint, depth < max_depth)
    does not depend on the mode."""
    out = []
    stack = [(0.0, 1.0, 0)]
    while stack:
        ta, tb, depth = stack.pop()
        a = p0 + ta * (p1 - p0)
        b = p0 + tb * (p1 - p0)
        mid = 0.5 * (a + b)
        length = np.linalg.norm(b - a)
        dist = np.hypot(rho_f - mid[0], z_f - mid[1])
        if depth < max_depth and length > refine_ratio * dist:
            tm = 0.5 * (ta + tb)
            stack.append((tm, tb, depth + 1))
            stack.append((ta, tm, depth + 1))
        else:
            out.append((ta, tb))
    return out


def assemble_mode_operators(profile, n_max, refine_ratio=1.0, max_depth=20):
    """image_charge.py:470-495: A[m, i, j] = mode-m potential at node i of the
    P1 hat density of node j, (n_max+1, P, P).  Collocation at the pole uses
    rho_floor = 1e-6 max(rho) (image_charge.py:482-489).  Leaves are gathered
    first and evaluated in one vectorised call (the sums differ from the
    reference's recursive order only in rounding)."""
    profile = np.asarray(profile, dtype=float)
    P = len(profile)
    rho_floor = 1e-6 * max(float(np.max(profile[:, 0])), 1e-300)
    rows, cols, rf, zf, rs, zs, wt = [], [], [], [], [], [], []
    for i in range(P):
        rho_f = max(profile[i, 0], rho_floor)
        z_f = profile[i, 1]
        for j in range(P - 1):
            p0, p1 = profile[j], profile[j + 1]
            seg_len = np.linalg.norm(p1 - p0)
            for ta, tb in _leaves(rho_f, z_f, p0, p1, refine_ratio, 0 if max_depth is None else max_depth):
                for x, w in zip(GAUSS4_X, GAUSS4_W):
                    t = ta + 0.5 * (tb - ta) * (x + 1.0)
                    pt = p0 + t * (p1 - p0)
                    ww = seg_len * (tb - ta) * 0.5 * w
                    for col, dens in ((j, 1.0 - t), (j + 1, t)):
                        rows.append(i)
                        cols.append(col)
                        rf.append(rho_f)
                        zf.append(z_f)
                        rs.append(pt[0])
                        zs.append(pt[1])
                        wt.append(dens * ww)
    phi = ring_potential_modes(np.array(rf), np.array(zf), np.array(rs), np.array(zs), n_max)
    A = np.zeros((n_max + 1, P, P))
    flat = np.array(rows) * P + np.array(cols)
    for m in range(n_max + 1):
        A[m].reshape(-1)[:] += np.bincount(flat, weights=phi[m] * np.array(wt), minlength=P * P)
    return A


def quadrature(profile, n_subdiv):
    """image_charge.py:418-452: fixed reconstruction nodes (rho, z, length
    weight, segment, t) -- n_subdiv sub-panels x Gauss-4 per segment."""
    profile = np.asarray(profile, dtype=float)
    rq, zq, lq, sq, tq = [], [], [], [], []
    for j in range(len(profile) - 1):
        p0, p1 = profile[j], profile[j + 1]
        length = np.linalg.norm(p1 - p0)
        for k in range(n_subdiv):
            ta, tb = k / n_subdiv, (k + 1) / n_subdiv
            for x, w in zip(GAUSS4_X, GAUSS4_W):
                t = ta + 0.5 * (tb - ta) * (x + 1.0)
                rq.append(p0[0] + t * (p1[0] - p0[0]))
                zq.append(p0[1] + t * (p1[1] - p0[1]))
                lq.append((length / n_subdiv) * 0.5 * w)
                sq.append(j)
                tq.append(t)
    return np.array(rq), np.array(zq), np.array(lq), np.array(sq, dtype=np.int64), np.array(tq)


# ---------------------------------------------------------------------------
# per-call force

class ImageSolution:
    """ImageChargeBEMSolution (image_charge.py:457-620): the image profile, its
    per-mode operators A and their inverses (image_charge.py:209-237)."""

    def __init__(self, profile, n_max, A=None, refine_ratio=1.0, max_depth=20):
        self.profile = np.asarray(profile, dtype=float)
        self.n_max = int(n_max)
        self.A = assemble_mode_operators(self.profile, n_max, refine_ratio, max_depth) if A is None else A
        self.A_inv = np.linalg.inv(self.A[: self.n_max + 1])
        self.seg = segments(self.profile)
        self.rho_floor = 1e-6 * max(float(np.max(self.profile[:, 0])), 1e-300)

    def image_force(self, pos, q, active, d_lo, d_hi, n_max=None, n_subdiv=4, n_eval=None, mirror_plane_z=None):
        """image_charge.py:987-1056: force (G, n_eval, 3) [N] on each group's
        first n_eval sources from the conductor's induced charge (joint
        per-group solve + local mirror charges), natural units divided by
        eps0 at the end."""
        n_max = self.n_max if n_max is None else int(n_max)
        pos = np.asarray(pos, dtype=float)
        G, E, _ = pos.shape
        ne = E if n_eval is None else int(n_eval)
        q_eff = np.where(active, q, 0.0)
        x, y, z = pos[..., 0], pos[..., 1], pos[..., 2]
        rho = np.hypot(x, y)
        phi = np.arctan2(y, x)
        rs = np.maximum(rho, self.rho_floor)
        closest, ut, un, dist = closest_on_profile(rs.reshape(-1), z.reshape(-1), self.seg)
        w = image_charge_weight(dist, d_lo, d_hi) if d_hi > d_lo else np.zeros_like(dist)
        if mirror_plane_z is not None:  # image_charge.py:538-585
            w = np.where(np.abs(z.reshape(-1) - mirror_plane_z) > dist, w, 0.0)
        r_img, z_img, side = mirror_points(rs.reshape(-1), z.reshape(-1), closest, ut, un)
        phi_img = np.where(side > 0, phi.reshape(-1), phi.reshape(-1) + np.pi).reshape(G, E)
        q_img = (-q_eff.reshape(-1) * w).reshape(G, E)
        r_img, z_img = r_img.reshape(G, E), z_img.reshape(G, E)
        prho = np.maximum(self.profile[:, 0], self.rho_floor)
        pz = self.profile[:, 1]
        m = np.arange(n_max + 1, dtype=float)

        def excitation(sr, sz, sphi, sq):
            g = point_charge_potential_modes(prho[None, None, :], pz[None, None, :], sr[:, :, None], sz[:, :, None],
                                             n_max)  # (M+1, G, E, P)
            wq = sq[None, :, :, None] * g
            gc = np.sum(wq * np.cos(m[:, None, None] * sphi[None])[..., None], axis=2)
            gs = np.sum(wq * np.sin(m[:, None, None] * sphi[None])[..., None], axis=2)
            return gc, gs

        c1, s1 = excitation(rs, z, phi, q_eff)
        c2, s2 = excitation(r_img, z_img, phi_img, q_img)
        rhs_c, rhs_s = -(c1 + c2), -(s1 + s2)  # (M+1, G, P)
        Ainv = self.A_inv[: n_max + 1]
        sig_c = np.einsum("mpk,mgk->mgp", Ainv, rhs_c)
        sig_s = np.einsum("mpk,mgk->mgp", Ainv, rhs_s)
        e_res = self._field(sig_c, sig_s, rs[:, :ne], phi[:, :ne], z[:, :ne], n_max, n_subdiv)
        qx = np.stack([rs[:, :ne] * np.cos(phi[:, :ne]), rs[:, :ne] * np.sin(phi[:, :ne]), z[:, :ne]], -1)
        mx = np.stack([r_img * np.cos(phi_img), r_img * np.sin(phi_img), z_img], -1)
        diff = qx[:, :, None, :] - mx[:, None, :, :]
        r = np.linalg.norm(diff, axis=-1)
        coef = np.where(r > 0.0, q_img[:, None, :] / (4.0 * np.pi * np.where(r > 0.0, r, 1.0) ** 3), 0.0)
        e_mir = np.einsum("gnm,gnmc->gnc", coef, diff)
        force = q_eff[:, :ne, None] * (e_res + e_mir) / VACUUM_PERMITTIVITY
        return np.where(active[:, :ne, None], force, 0.0)

    def _field(self, sig_c, sig_s, rq, phq, zq, n_max, n_subdiv):
        """image_charge.py:1296-1347: field of the joint mode density at each
        group's own query points, on the fixed quadrature."""
        rn, zn, ln, sn, tn = quadrature(self.profile, n_subdiv)
        dc = (sig_c[..., sn] + tn * (sig_c[..., sn + 1] - sig_c[..., sn])) * ln  # (M+1, G, Nq)
        ds = (sig_s[..., sn] + tn * (sig_s[..., sn + 1] - sig_s[..., sn])) * ln
        ph, dr, dz = ring_field_modes(rq[:, :, None], zq[:, :, None], rn[None, None, :], zn[None, None, :], n_max)
        m = np.arange(n_max + 1, dtype=float)
        cm = np.cos(m[:, None, None] * phq[None])[..., None]
        sm = np.sin(m[:, None, None] * phq[None])[..., None]
        dens = dc[:, :, None, :] * cm + ds[:, :, None, :] * sm
        ang = dc[:, :, None, :] * sm - ds[:, :, None, :] * cm
        e_rho = np.sum(np.sum(-dens * dr, axis=-1), axis=0)
        e_z = np.sum(np.sum(-dens * dz, axis=-1), axis=0)
        e_phi = np.sum(np.sum(ang * ph, axis=-1) * m[:, None, None] / rq[None], axis=0)
        return np.stack([e_rho * np.cos(phq) - e_phi * np.sin(phq), e_rho * np.sin(phq) + e_phi * np.cos(phq), e_z], -1)


def geometry_image_force(sol, pos, q, active, z0, R, d_lo=0.1, d_hi=0.5, n_max=None, z_handoff=None,
                         mirror_symmetric=False, soft=1e-12):
    """bem/geometry.py:326-344 (tip) and :780-797 (well): the image force of a
    BEM geometry built with z0 -- the flat plane image at z0
    (forces.image_charge_force) above z_handoff, the BEM image solve below
    z_handoff/2, smoothstep between.  mirror_symmetric (bem/geometry.py:
    346-415): the solve on the mirror-doubled profile excited by each source
    and its phantom (z -> -2 z0 - z, -q), plus the direct plane image."""
    pos = np.asarray(pos, dtype=float)
    far = flat_image(pos, q, active, z0, soft)
    if mirror_symmetric:
        mpos = pos.copy()
        mpos[..., 2] = -2.0 * z0 - pos[..., 2]
        near = sol.image_force(np.concatenate([pos, mpos], 1), np.concatenate([q, -q], 1),
                               np.concatenate([active, active], 1), d_lo * R, d_hi * R, n_max=n_max,
                               n_eval=pos.shape[1], mirror_plane_z=-z0) + far
    else:
        near = sol.image_force(pos, q, active, d_lo * R, d_hi * R, n_max=n_max)
    if z_handoff is None:
        z_handoff = 20.0 * R
    w = smoothstep_weight(pos[..., 2], 0.5 * z_handoff, z_handoff)[..., None]
    return w * near + (1.0 - w) * far
