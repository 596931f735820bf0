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
GAUSS2_X, GAUSS2_W = np.polynomial.legendre.leggauss(2)  # adaptive far rule only (not in the reference)


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


def whole_segment_nodes(profile, sigma, gx, gw):
    """Gauss rule (gx, gw) over each whole segment: (rho_q, z_q, area_q *
    sigma_q), each [n_seg, len(gx)].  Used by the adaptive far rule."""
    profile = np.asarray(profile, dtype=float)
    sigma = np.asarray(sigma, dtype=float)
    p0, p1 = profile[:-1], profile[1:]
    length = np.linalg.norm(p1 - p0, axis=-1)
    t = 0.5 * (np.asarray(gx) + 1.0)[None, :]
    r = p0[:, :1] + t * (p1[:, :1] - p0[:, :1])
    z = p0[:, 1:] + t * (p1[:, 1:] - p0[:, 1:])
    w = 2.0 * np.pi * r * (length[:, None] * 0.5 * np.asarray(gw)[None, :])
    return r, z, w * (sigma[:-1, None] + t * (sigma[1:, None] - sigma[:-1, None]))


def run_rule_nodes(profile, sigma, block=32, n=8):
    """Run rule (adaptive far rule, not in the reference): for each run of
    `block` consecutive segments, n nodes at the Gauss points of its
    arclength and product-integration weights w_i = integral of
    sigma 2 pi rho l_i over the run (l_i the Lagrange polynomial of node i).
    Returns (rho [n_run, n], z, w, centre [n_run, 2], radius, arclength)."""
    profile = np.asarray(profile, dtype=float)
    sigma = np.asarray(sigma, dtype=float)
    nseg = len(profile) - 1
    length = np.linalg.norm(profile[1:] - profile[:-1], axis=-1)
    s_node = np.concatenate([[0.0], np.cumsum(length)])
    gx, _ = np.polynomial.legendre.leggauss(n)
    g5x, g5w = np.polynomial.legendre.leggauss(5)
    nrun = (nseg + block - 1) // block
    R, Z, W = np.zeros((nrun, n)), np.zeros((nrun, n)), np.zeros((nrun, n))
    cen, rad, arc = np.zeros((nrun, 2)), np.zeros(nrun), np.zeros(nrun)
    for q in range(nrun):
        a, b = q * block, min((q + 1) * block, nseg)
        pts = profile[a:b + 1]
        cen[q] = 0.5 * (pts.min(axis=0) + pts.max(axis=0))
        rad[q] = np.sqrt(((pts - cen[q]) ** 2).sum(axis=-1)).max()
        arc[q] = s_node[b] - s_node[a]
        sq = s_node[a] + 0.5 * (gx + 1.0) * arc[q]
        for i, sv in enumerate(sq):
            j = min(max(int(np.searchsorted(s_node, sv, side="right")) - 1, a), b - 1)
            t = (sv - s_node[j]) / length[j]
            R[q, i] = profile[j, 0] + t * (profile[j + 1, 0] - profile[j, 0])
            Z[q, i] = profile[j, 1] + t * (profile[j + 1, 1] - profile[j, 1])
        for j in range(a, b):
            t = 0.5 * (g5x + 1.0)
            sv = s_node[j] + t * length[j]
            f = (2.0 * np.pi * (profile[j, 0] + t * (profile[j + 1, 0] - profile[j, 0]))
                 * (sigma[j] + t * (sigma[j + 1] - sigma[j])) * 0.5 * length[j] * g5w)
            for i in range(n):
                lag = np.ones_like(sv)
                for m in range(n):
                    if m != i:
                        lag *= (sv - sq[m]) / (sq[i] - sq[m])
                W[q, i] += np.sum(lag * f)
    return R, Z, W, cen, rad, arc


def _run_override(er_s, ez_s, rho_e, z_e, runs, run_flags, ratio_run, round_size, block=32):
    """Run rule: for each round, a flagged run whose bounding circle is at
    least ratio_run arclengths from every point of the round contributes its
    n-node sum (kept in its first segment's slot, the others zeroed)."""
    R, Z, W, cen, rad, arc = runs
    nseg = er_s.shape[1]
    for a in range(0, len(rho_e), round_size):
        b = min(a + round_size, len(rho_e))
        lb = np.full(len(arc), np.inf)
        for p in range(a, b):
            lb = np.minimum(lb, np.hypot(rho_e[p] - cen[:, 0], z_e[p] - cen[:, 1]) - rad)
        for q in np.nonzero(np.asarray(run_flags, dtype=bool) & (lb >= ratio_run * arc))[0]:
            s0, s1 = q * block, min((q + 1) * block, nseg)
            for p in range(a, b):
                er, ez = ring_field(rho_e[p], z_e[p] - Z[q], R[q])
                er_s[p, s0:s1] = 0.0
                ez_s[p, s0:s1] = 0.0
                er_s[p, s0] = np.sum(W[q] * er)
                ez_s[p, s0] = np.sum(W[q] * ez)


def _adaptive_override(er_s, ez_s, rho_e, z_e, dist, seg, coarse, ratio4, ratio2, round_size):
    """The adaptive far rule: for each round of `round_size` consecutive
    points, a segment whose smallest distance over the round is at least
    ratio4 lengths takes the whole-segment Gauss-4 rule, at least ratio2 the
    Gauss-2 rule (replacing the sub-panel sums for every point of the round)."""
    L = seg["length"]
    (r4, z4, w4), (r2, z2, w2) = coarse
    for a in range(0, len(rho_e), round_size):
        b = min(a + round_size, len(rho_e))
        dmin = dist[a:b].min(axis=0)
        for lvl, (rq, zq, wq) in ((1, (r4, z4, w4)), (2, (r2, z2, w2))):
            sel = (dmin >= ratio4 * L) & (dmin < ratio2 * L) if lvl == 1 else dmin >= ratio2 * L
            js = np.nonzero(sel)[0]
            if len(js) == 0:
                continue
            for p in range(a, b):
                er, ez = ring_field(rho_e[p], z_e[p] - zq[js], rq[js])
                er_s[p, js] = np.sum(wq[js] * er, axis=-1)
                ez_s[p, js] = np.sum(wq[js] * ez, axis=-1)


def cluster_table(profile, sigma, n_subdiv=8, n_terms=32, block=32):
    """Cluster expansions of the adaptive rule (not in the reference; the
    product's tables restate this): a binary tree over the runs of `block`
    segments, level l the clusters of 2^l consecutive runs, each with its
    centre (0, z_c) (the middle of its z range), the radius r_max of the
    sphere about it through its farthest segment end, and the moments
    M_n = sum_q w_q (r_q / r_max)^n P_n(cos theta_q) of its far nodes (the
    axisymmetric term of the addition theorem: a ring's potential about a
    centre on the axis is sum_n r'^n / r^(n+1) P_n(u') P_n(u)).  Returns a
    list of levels, each a list of (z_c, r_max, M, s0, s1)."""
    from scipy.special import eval_legendre
    profile = np.asarray(profile, dtype=float)
    rq, zq, aq, sq = far_nodes(profile, sigma, n_subdiv)
    wq = aq * sq
    n_seg = len(profile) - 1
    per = 4 * n_subdiv
    n_run = (n_seg + block - 1) // block
    levels, size = [], 1
    while True:
        n_cl = (n_run + size - 1) // size
        lev = []
        for k in range(n_cl):
            s0, s1 = k * size * block, min((k + 1) * size * block, n_seg)
            ends = profile[s0:s1 + 1]
            zc = 0.5 * (ends[:, 1].min() + ends[:, 1].max())
            rmax = np.sqrt(ends[:, 0] ** 2 + (ends[:, 1] - zc) ** 2).max()
            r, z, w = rq[s0 * per:s1 * per], zq[s0 * per:s1 * per], wq[s0 * per:s1 * per]
            rr = np.hypot(r, z - zc)
            u = (z - zc) / rr
            M = np.array([np.sum(w * (rr / rmax) ** n * eval_legendre(n, u)) for n in range(n_terms)])
            lev.append((zc, rmax, M, s0, s1))
        levels.append(lev)
        if n_cl == 1:
            return levels
        size *= 2


def cluster_field(zc, rmax, M, rho, z):
    """(E_rho, E_z) of a cluster's expansion at (rho, z):
    E = -grad (1/4 pi) sum_n M_n rmax^n P_n(u) / r^(n+1)."""
    from scipy.special import eval_legendre
    dz = z - zc
    r = np.hypot(rho, dz)
    u, s = dz / r, rho / r
    n = np.arange(len(M))
    x = (rmax / r) ** n
    P = eval_legendre(n, u)
    # P_n'(u) by P'_(n+1) = P'_(n-1) + (2n+1) P_n
    D = np.zeros(len(M))
    for k in range(1, len(M)):
        D[k] = (D[k - 2] if k >= 2 else 0.0) + (2 * k - 1) * P[k - 1]
    e_r = np.sum((n + 1) * M * x * P) / (4 * np.pi * r * r)
    e_t = s * np.sum(M * x * D) / (4 * np.pi * r * r)
    return e_r * s + e_t * u, e_r * u - e_t * s


def _cluster_override(er_s, ez_s, rho_e, z_e, levels, kappa, block=32):
    """Cluster rule: for each point, every run takes its highest ancestor
    cluster at least kappa r_max from the point; the segments of a covered
    cluster give way to its expansion (kept in its first segment's slot)."""
    n_seg = er_s.shape[1]
    n_run = (n_seg + block - 1) // block
    for p in range(len(rho_e)):
        cover = {}
        for q in range(n_run):
            best = None
            for l, lev in enumerate(levels):
                zc, rmax, M, s0, s1 = lev[q >> l]
                if np.hypot(rho_e[p], z_e[p] - zc) >= kappa * rmax:
                    best = (l, q >> l)
            if best is not None:
                cover[best] = levels[best[0]][best[1]]
        for (l, k), (zc, rmax, M, s0, s1) in cover.items():
            er_s[p, s0:s1] = 0.0
            ez_s[p, s0:s1] = 0.0
            er_s[p, s0], ez_s[p, s0] = cluster_field(zc, rmax, M, rho_e[p], z_e[p])


def field(points, profile, sigma, n_subdiv=8, chunk=256, far_rule="reference", ratio4=8.0, ratio2=300.0,
          round_size=1, run_flags=None, ratio_run=4.0, clusters=None, cluster_kappa=3.0):
    """bem/axisymmetric.py:501-605 -- E = -grad S[sigma] at points (..., 3).

    far_rule="adaptive" swaps the sub-panel sums of distant segments for the
    whole-segment rules of ``_adaptive_override`` (chunk must be a multiple
    of round_size so rounds are consecutive points of the input), and, with
    ``run_flags`` (which runs of 32 segments may take it), distant flagged
    runs for the run rule of ``_run_override``, and, with ``clusters`` (a
    ``cluster_table``), runs covered by a distant cluster for its expansion
    (``_cluster_override``)."""
    points = np.asarray(points, dtype=float)
    shape = points.shape
    flat = points.reshape(-1, 3)
    sigma = np.asarray(sigma, dtype=float)
    seg = segments(profile)
    rq, zq, aq, sq = far_nodes(profile, sigma, n_subdiv)
    wq = aq * sq
    nseg = len(seg["p0"])
    per = len(rq) // nseg
    if far_rule == "adaptive":
        coarse = (whole_segment_nodes(profile, sigma, GAUSS4_X, GAUSS4_W),
                  whole_segment_nodes(profile, sigma, GAUSS2_X, GAUSS2_W))
        runs = run_rule_nodes(profile, sigma) if run_flags is not None else None
        assert chunk % round_size == 0
    elif far_rule != "reference":
        raise ValueError(far_rule)
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
        if far_rule == "adaptive":
            _adaptive_override(er_s, ez_s, rho_e, z, dist, seg, coarse, ratio4, ratio2, round_size)
            if runs is not None:
                _run_override(er_s, ez_s, rho_e, z, runs, run_flags, ratio_run, round_size)
            if clusters is not None:
                _cluster_override(er_s, ez_s, rho_e, z, clusters, cluster_kappa)
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
