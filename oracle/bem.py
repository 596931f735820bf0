"""Oracle: axisymmetric BEM ring-charge field (float64, NumPy/SciPy).

Test infrastructure only -- see ``oracle/__init__.py``.  Restates
``bem/axisymmetric.py`` (ring field, fixed quadrature, closest point,
on-surface offset, near-segment sinh quadrature) and the field half of
``bem/fields.py`` / ``bem/geometry.py``.  K and E come from SciPy's
``ellipkm1`` / ``ellipe`` exactly as ``bem/_elliptic.py:28-39`` does.
"""

import numpy as np
from scipy import special

GAUSS4_X, GAUSS4_W = np.polynomial.legendre.leggauss(4)  # bem/axisymmetric.py:98
GAUSS8_X, GAUSS8_W = np.polynomial.legendre.leggauss(8)  # bem/axisymmetric.py:94


def ellip_k_e_complement(p):
    """bem/_elliptic.py:28-39: K(1-p), E(1-p)."""
    return special.ellipkm1(p), special.ellipe(1.0 - p)


def ring_field(rho, z, a):
    """bem/axisymmetric.py:248-265 -- (E_rho, E_z) of a unit-charge ring of
    radius a at height 0, field point (rho, z); near-axis Taylor branch."""
    D = (rho + a) ** 2 + z**2
    d2 = (rho - a) ** 2 + z**2
    K, E = ellip_k_e_complement(d2 / D)
    on_axis = rho**2 < 1e-10 * (a * a + z * z)
    rho_ok = np.where(on_axis, 1.0, rho)
    with np.errstate(divide="ignore", invalid="ignore"):
        er = (K - (a * a - rho * rho + z * z) * E / d2) / (4 * np.pi**2 * rho_ok * np.sqrt(D))
        ez = z * E / (2 * np.pi**2 * np.sqrt(D) * d2)
    ax2 = a * a + z * z
    er_ax = rho * (2 * z * z - a * a) / (8 * np.pi * ax2**2.5)
    ez_ax = z / (4 * np.pi * ax2**1.5) + 3 * rho * rho * z * (3 * a * a - 2 * z * z) / (16 * np.pi * ax2**3.5)
    return np.where(on_axis, er_ax, er), np.where(on_axis, ez_ax, ez)


def far_nodes(profile, sigma, n_subdiv):
    """bem/axisymmetric.py:305-326 -- Gauss-4 nodes on n_subdiv equal
    sub-panels of every segment: (rho_q, z_q, area_q, sigma_q), segment-major."""
    profile = np.asarray(profile, dtype=float)
    sigma = np.asarray(sigma, dtype=float)
    out = [[], [], [], []]
    for j in range(len(profile) - 1):
        p0, p1 = profile[j], profile[j + 1]
        s0, s1 = sigma[j], sigma[j + 1]
        length = np.linalg.norm(p1 - p0)
        for k in range(n_subdiv):
            ta, tb = k / n_subdiv, (k + 1) / n_subdiv
            for xi, wi in zip(GAUSS4_X, GAUSS4_W):
                t = ta + 0.5 * (tb - ta) * (xi + 1.0)
                r = p0[0] + t * (p1[0] - p0[0])
                out[0].append(r)
                out[1].append(p0[1] + t * (p1[1] - p0[1]))
                out[2].append(2.0 * np.pi * r * ((length / n_subdiv) * 0.5 * wi))
                out[3].append(s0 + t * (s1 - s0))
    return tuple(np.array(v) for v in out)


def segments(profile):
    """bem/axisymmetric.py:329-338 plus lengths/unit tangents (:490-498)."""
    profile = np.asarray(profile, dtype=float)
    p0 = profile[:-1]
    tangent = profile[1:] - p0
    normal = np.stack([-tangent[:, 1], tangent[:, 0]], axis=-1)
    normal = normal / np.linalg.norm(normal, axis=-1, keepdims=True)
    length = np.linalg.norm(tangent, axis=-1)
    return dict(p0=p0, tangent=tangent, normal=normal, length=length, unit=tangent / length[:, None])


def closest_point(rho, z, seg):
    """bem/axisymmetric.py:341-389 -- first strict minimum over segments."""
    p0, tan = seg["p0"], seg["tangent"]
    best = np.full(rho.shape, np.inf)
    arg = np.zeros(rho.shape, dtype=np.int64)
    for j in range(len(p0)):
        ab2 = float(tan[j, 0] * tan[j, 0] + tan[j, 1] * tan[j, 1])
        t = np.clip(((rho - p0[j, 0]) * tan[j, 0] + (z - p0[j, 1]) * tan[j, 1]) / ab2, 0.0, 1.0)
        d2 = (rho - (p0[j, 0] + t * tan[j, 0])) ** 2 + (z - (p0[j, 1] + t * tan[j, 1])) ** 2
        better = d2 < best
        best = np.where(better, d2, best)
        arg = np.where(better, j, arg)
    return best, arg


def _near_segment_sum(rho_e, z_e, seg, sigma, j, s0, d):
    """bem/axisymmetric.py:571-600 for one (point, segment) pair: sinh map
    s = s0 + d sinh(v), Gauss-8 on ceil(width/0.5) equal v-intervals, P1 density."""
    L = seg["length"][j]
    lo = np.arcsinh(-s0 / d)
    hi = np.arcsinh((L - s0) / d)
    count = max(1, int(np.ceil((hi - lo) / 0.5)))
    width = (hi - lo) / count
    k = np.arange(count)[:, None]
    v = lo + (k + 0.5 * (GAUSS8_X[None, :] + 1.0)) * width
    s = s0 + d * np.sinh(v)
    src_r = seg["p0"][j, 0] + s * seg["unit"][j, 0]
    src_z = seg["p0"][j, 1] + s * seg["unit"][j, 1]
    dens = sigma[j] + (s / L) * (sigma[j + 1] - sigma[j])
    w = dens * (2 * np.pi * src_r) * d * np.cosh(v) * (0.5 * (hi - lo) / count) * GAUSS8_W[None, :]
    er, ez = ring_field(rho_e, z_e - src_z, src_r)
    return np.sum(w * er), np.sum(w * ez)


def field(points, profile, sigma, n_subdiv=8, chunk=256):
    """bem/axisymmetric.py:501-605 -- E = -grad S[sigma] at points (..., 3)."""
    points = np.asarray(points, dtype=float)
    shape = points.shape
    flat = points.reshape(-1, 3)
    sigma = np.asarray(sigma, dtype=float)
    seg = segments(profile)
    rq, zq, aq, sq = far_nodes(profile, sigma, n_subdiv)
    wq = aq * sq
    nseg = len(seg["p0"])
    per = len(rq) // nseg
    out = np.empty_like(flat)
    for c0 in range(0, len(flat), chunk):
        f = flat[c0:c0 + chunk]
        rho = np.hypot(f[:, 0], f[:, 1])
        z = f[:, 2].copy()
        phi = np.arctan2(f[:, 1], f[:, 0])
        d2best, j = closest_point(rho, z, seg)
        Lj = seg["length"][j]
        off = np.where(d2best < (1e-9 * Lj) ** 2, 1e-4 * Lj, 0.0)
        rho_e = rho + off * seg["normal"][j, 0]
        rho_e = np.where(rho == 0.0, 0.0, rho_e)
        z = z + off * seg["normal"][j, 1]
        er, ez = ring_field(rho_e[:, None], z[:, None] - zq[None, :], rq[None, :])
        er_s = (er * wq[None, :]).reshape(-1, nseg, per).sum(axis=-1)
        ez_s = (ez * wq[None, :]).reshape(-1, nseg, per).sum(axis=-1)
        delta = np.stack([rho_e, z], axis=-1)[:, None, :] - seg["p0"][None, :, :]
        along = np.sum(delta * seg["unit"][None, :, :], axis=-1)
        proj = np.clip(along, 0.0, seg["length"][None, :])
        dist = np.linalg.norm(delta - proj[..., None] * seg["unit"][None, :, :], axis=-1)
        pi, si = np.nonzero(dist < seg["length"][None, :])
        for p, s in zip(pi, si):
            d = max(dist[p, s], 1e-15 * seg["length"][s])
            er_s[p, s], ez_s[p, s] = _near_segment_sum(rho_e[p], z[p], seg, sigma, s, proj[p, s], d)
        e_rho = er_s.sum(axis=-1)
        e_z = ez_s.sum(axis=-1)
        out[c0:c0 + chunk, 0] = np.where(rho == 0.0, 0.0, e_rho * np.cos(phi))
        out[c0:c0 + chunk, 1] = np.where(rho == 0.0, 0.0, e_rho * np.sin(phi))
        out[c0:c0 + chunk, 2] = e_z
    return out.reshape(shape)


def near_pair_count(points, profile):
    """Number of (point, segment) pairs the near-segment quadrature handles
    (the ``distance < length`` test of bem/axisymmetric.py:566-570)."""
    flat = np.asarray(points, dtype=float).reshape(-1, 3)
    seg = segments(profile)
    rho = np.hypot(flat[:, 0], flat[:, 1])
    z = flat[:, 2]
    delta = np.stack([rho, z], axis=-1)[:, None, :] - seg["p0"][None, :, :]
    along = np.sum(delta * seg["unit"][None, :, :], axis=-1)
    proj = np.clip(along, 0.0, seg["length"][None, :])
    dist = np.linalg.norm(delta - proj[..., None] * seg["unit"][None, :, :], axis=-1)
    return int(np.count_nonzero(dist < seg["length"][None, :]))
