"""Device tables of a solved axisymmetric BEM problem (profile, sigma).

Built once per geometry, like the reference's per-device field cache
(bem/axisymmetric.py:474-498, backend.py:49-51):

* segment table  [11, n_seg]: p0 (rho, z), tangent p1 - p0, length, unit
  tangent, unit left normal, density at both ends (bem/axisymmetric.py:329-338,
  490-498);
* far-node table [3, stride]: rho_q, z_q, w_q = area_q * sigma_q of the
  Gauss-4 rule on n_subdiv equal sub-panels per segment, segment-major
  (bem/axisymmetric.py:305-326, 561).  Rows are padded to a multiple of 32
  nodes so every row starts 16-byte aligned for the TMA bulk copies;
* coarse-node table [3, stride]: the same (rho_q, z_q, w_q) for the 4-point
  and the 2-point Gauss rules over each whole segment (6 nodes per segment),
  read by the adaptive far rule for distant segments.  Not in the
  reference, whose far sum always takes the n_subdiv sub-panels;
* run table [6, n_run]: centre, radius, largest segment length, arclength
  and a run-rule flag of each run of 32 consecutive segments, for skipping
  runs in the per-point segment scans (an acceleration only: results are
  unchanged) and for the adaptive rule's run classes;
* run-node table [3, n_run * 8]: the 8-point Gauss rule over the arclength
  of each whole run.  A run is flagged for it only when it is straight and,
  at probe points RATIO_RUN arclengths away, its 8-point sum matches the
  segment-wise Gauss-4 sum to RUN_TOL;
* cluster table [n_cluster, CLUSTER_TERMS + 2]: a binary tree over the runs
  (level l: clusters of 2^l consecutive runs) with, per cluster, its centre
  on the axis, its radius and the axisymmetric multipole moments of its
  far-node weights, for the adaptive rule's cluster expansions.  Not in the
  reference.
"""

import ctypes

import numpy as np

from . import _lib

GAUSS4_X, GAUSS4_W = np.polynomial.legendre.leggauss(4)
GAUSS8_X, GAUSS8_W = np.polynomial.legendre.leggauss(8)
GAUSS2_X, GAUSS2_W = np.polynomial.legendre.leggauss(2)
# default thresholds of the adaptive far rule (distance / segment length,
# distance / run arclength) and the run-rule acceptance tolerance
RATIO4, RATIO2, RATIO_RUN = 8.0, 300.0, 4.0
RUN_TOL = 1e-10
GAUSS_RUN_X, GAUSS_RUN_W = np.polynomial.legendre.leggauss(_lib.RUN_NODES)
# cluster expansions: terms kept, and separation (distance from the centre
# over the cluster's radius) beyond which a cluster is summed by them
CLUSTER_TERMS, CLUSTER_KAPPA = 32, 3.0
MAX_CLUSTER_RUNS = 256


def segment_table(profile, sigma):
    prof = np.asarray(profile, dtype=np.float64)
    sig = np.asarray(sigma, dtype=np.float64)
    if prof.ndim != 2 or prof.shape[1] != 2 or len(prof) < 2:
        raise ValueError("profile must be an (n >= 2, 2) array of (rho, z) nodes")
    if sig.shape != (len(prof),):
        raise ValueError("sigma must have one value per profile node")
    p0 = prof[:-1]
    tan = prof[1:] - p0
    length = np.linalg.norm(tan, axis=-1)
    if np.any(length <= 0.0):
        raise ValueError("profile has a zero-length segment")
    unit = tan / length[:, None]
    nrm = np.stack([-tan[:, 1], tan[:, 0]], axis=-1)
    nrm = nrm / np.linalg.norm(nrm, axis=-1, keepdims=True)
    return np.stack([p0[:, 0], p0[:, 1], tan[:, 0], tan[:, 1], length, unit[:, 0], unit[:, 1],
                     nrm[:, 0], nrm[:, 1], sig[:-1], sig[1:]])


def far_nodes(profile, sigma, n_subdiv):
    """(rho_q, z_q, area_q, sigma_q), each [n_seg * 4 * n_subdiv], segment-major."""
    prof = np.asarray(profile, dtype=np.float64)
    sig = np.asarray(sigma, dtype=np.float64)
    p0, p1 = prof[:-1], prof[1:]
    length = np.array([np.linalg.norm(b - a) for a, b in zip(p0, p1)])
    k = np.arange(n_subdiv, dtype=np.float64)
    ta = k / n_subdiv
    tb = (k + 1) / n_subdiv
    t = ta[:, None] + 0.5 * (tb - ta)[:, None] * (GAUSS4_X[None, :] + 1.0)     # [n_subdiv, 4]
    t = t.reshape(1, -1)                                                        # node order k-major, gauss-minor
    w = np.tile(GAUSS4_W, n_subdiv).reshape(1, -1)
    rho = p0[:, 0:1] + t * (p1[:, 0:1] - p0[:, 0:1])
    z = p0[:, 1:2] + t * (p1[:, 1:2] - p0[:, 1:2])
    seg_len = (length[:, None] / n_subdiv) * 0.5 * w
    area = 2.0 * np.pi * rho * seg_len
    sq = sig[:-1, None] + t * (sig[1:, None] - sig[:-1, None])
    return rho.ravel(), z.ravel(), area.ravel(), sq.ravel()


def coarse_nodes(profile, sigma):
    """[3, n_seg * 6]: per segment the Gauss-4 then the Gauss-2 nodes over the
    whole segment, as (rho_q, z_q, area_q * sigma_q)."""
    prof = np.asarray(profile, dtype=np.float64)
    sig = np.asarray(sigma, dtype=np.float64)
    p0, p1 = prof[:-1], prof[1:]
    length = np.linalg.norm(p1 - p0, axis=-1)
    x = np.concatenate([GAUSS4_X, GAUSS2_X])
    w = np.concatenate([GAUSS4_W, GAUSS2_W])
    t = 0.5 * (x + 1.0)[None, :]
    rho = p0[:, 0:1] + t * (p1[:, 0:1] - p0[:, 0:1])
    z = p0[:, 1:2] + t * (p1[:, 1:2] - p0[:, 1:2])
    area = 2.0 * np.pi * rho * (length[:, None] * 0.5 * w[None, :])
    sq = sig[:-1, None] + t * (sig[1:, None] - sig[:-1, None])
    return np.stack([rho.ravel(), z.ravel(), (area * sq).ravel()])


def _ring_field(rho, z, a):
    """(E_rho, E_z) of unit-charge rings of radius a at height 0, off the
    axis and off the ring (host-side checks only)."""
    from scipy import special
    D = (rho + a) ** 2 + z * z
    d2 = (rho - a) ** 2 + z * z
    m = 4.0 * rho * a / D
    K, E = special.ellipk(m), special.ellipe(m)
    er = (K - (a * a - rho * rho + z * z) * E / d2) / (4.0 * np.pi**2 * rho * np.sqrt(D))
    ez = z * E / (2.0 * np.pi**2 * np.sqrt(D) * d2)
    return er, ez


def run_tables(profile, sigma, block=_lib.BLOCK_SEGS, ratio_run=RATIO_RUN, tol=RUN_TOL):
    """(bounds [6, n_run], run nodes [3, n_run * 8]).  Bounds rows: centre
    (rho, z), radius covering every endpoint of the run (segments are the
    convex hulls of their endpoints), largest segment length, arclength, and
    the run-rule flag."""
    prof = np.asarray(profile, dtype=np.float64)
    sig = np.asarray(sigma, dtype=np.float64)
    n_seg = len(prof) - 1
    n_blk = (n_seg + block - 1) // block
    out = np.zeros((6, n_blk))
    nodes = np.zeros((3, n_blk * _lib.RUN_NODES))
    length = np.linalg.norm(prof[1:] - prof[:-1], axis=-1)
    s_node = np.concatenate([[0.0], np.cumsum(length)])
    gx4, gw4 = GAUSS4_X, GAUSS4_W
    for b in range(n_blk):
        s0, s1 = b * block, min((b + 1) * block, n_seg)
        pts = prof[s0:s1 + 1]
        c = 0.5 * (pts.min(axis=0) + pts.max(axis=0))
        out[0, b], out[1, b] = c
        out[2, b] = np.sqrt(((pts - c) ** 2).sum(axis=-1)).max()
        out[3, b] = length[s0:s1].max()
        arc = s_node[s1] - s_node[s0]
        out[4, b] = arc
        # 8 nodes at the Gauss points of the run's arclength (on the polyline);
        # weights by product integration: w_i = integral over the run of
        # sigma(s) 2 pi rho(s) l_i(s) ds, l_i the Lagrange polynomial of node i,
        # exact segment by segment (the integrand is a polynomial of degree 9
        # on each segment: 5-point Gauss), so the rule integrates the
        # piecewise-linear density exactly against any degree-7 kernel
        sq = s_node[s0] + 0.5 * (GAUSS_RUN_X + 1.0) * arc
        j = np.clip(np.searchsorted(s_node, sq, side="right") - 1, s0, s1 - 1)
        t = (sq - s_node[j]) / length[j]
        r = prof[j, 0] + t * (prof[j + 1, 0] - prof[j, 0])
        z = prof[j, 1] + t * (prof[j + 1, 1] - prof[j, 1])
        k = slice(b * _lib.RUN_NODES, (b + 1) * _lib.RUN_NODES)
        nodes[0, k], nodes[1, k] = r, z
        g5x, g5w = np.polynomial.legendre.leggauss(5)
        tt = 0.5 * (g5x + 1.0)
        ss = (s_node[s0:s1, None] + tt[None, :] * length[s0:s1, None]).ravel()
        rr = (prof[s0:s1, 0:1] + tt * (prof[s0 + 1:s1 + 1, 0:1] - prof[s0:s1, 0:1])).ravel()
        dd = (sig[s0:s1, None] + tt * (sig[s0 + 1:s1 + 1, None] - sig[s0:s1, None])).ravel()
        ww = (0.5 * length[s0:s1, None] * g5w[None, :]).ravel()
        lag = np.ones((_lib.RUN_NODES, len(ss)))
        for i in range(_lib.RUN_NODES):
            for m in range(_lib.RUN_NODES):
                if m != i:
                    lag[i] *= (ss - sq[m]) / (sq[i] - sq[m])
        nodes[2, k] = lag @ (ww * 2.0 * np.pi * rr * dd)
        # flag: a straight run whose run-rule sum matches the segment-wise Gauss-4 sum at
        # probe points ratio_run arclengths beyond its bounding circle, around it
        u = (pts[-1] - pts[0]) / np.linalg.norm(pts[-1] - pts[0])
        straight = np.abs((pts - pts[0]) @ np.array([-u[1], u[0]])).max() <= 1e-9 * arc
        ok = bool(straight) and ratio_run > 0
        if ok:
            tq = 0.5 * (gx4 + 1.0)
            sr = (prof[s0:s1, 0:1] + tq * (prof[s0 + 1:s1 + 1, 0:1] - prof[s0:s1, 0:1])).ravel()
            sz = (prof[s0:s1, 1:2] + tq * (prof[s0 + 1:s1 + 1, 1:2] - prof[s0:s1, 1:2])).ravel()
            sw = (2.0 * np.pi * (prof[s0:s1, 0:1] + tq * (prof[s0 + 1:s1 + 1, 0:1] - prof[s0:s1, 0:1]))
                  * (length[s0:s1, None] * 0.5 * gw4) * (sig[s0:s1, None] + tq * (sig[s0 + 1:s1 + 1, None] - sig[s0:s1, None]))).ravel()
            dist = out[2, b] + ratio_run * arc
            for ang in np.linspace(0.0, 2.0 * np.pi, 16, endpoint=False):
                pr_, pz_ = c[0] + dist * np.cos(ang), c[1] + dist * np.sin(ang)
                if pr_ <= 1e-3 * dist:
                    continue  # the axis side of the run: rho <= 0 is not a field point
                a_r, a_z = _ring_field(pr_, pz_ - sz, sr)
                b_r, b_z = _ring_field(pr_, pz_ - z, r)
                ref = np.array([np.sum(sw * a_r), np.sum(sw * a_z)])
                got = np.array([np.sum(nodes[2, k] * b_r), np.sum(nodes[2, k] * b_z)])
                scale = np.sum(np.abs(sw) * np.hypot(a_r, a_z))
                if not np.abs(got - ref).max() <= tol * scale:
                    ok = False
                    break
        out[5, b] = 1.0 if ok else 0.0
    return out, nodes


def cluster_tables(profile, sigma, n_subdiv, n_terms=CLUSTER_TERMS, block=_lib.BLOCK_SEGS):
    """(table [n_cluster, n_terms + 2], n_levels).  Level l holds
    ceil(n_run / 2^l) clusters of 2^l consecutive runs (the last one shorter),
    levels one after another, up to the level with a single cluster.  Record:
    centre z_c (on the axis: the middle of the cluster's z range), radius
    r_max (largest distance from (0, z_c) to an end of its segments, which
    bounds every ring of the cluster), moments M_n = sum_q w_q (r_q/r_max)^n
    P_n(u_q) over its far nodes q, with r_q, u_q the distance from (0, z_c) and
    the cosine of the polar angle (the potential of a ring about a centre on
    the axis is sum_n r'^n / r^(n+1) P_n(u') P_n(u), the addition theorem's
    axisymmetric term)."""
    prof = np.asarray(profile, dtype=np.float64)
    rq, zq, aq, sq = far_nodes(prof, sigma, n_subdiv)
    wq = aq * sq
    n_seg = len(prof) - 1
    per = 4 * n_subdiv
    n_run = (n_seg + block - 1) // block
    rows = []
    levels = 0
    size = 1
    while True:
        n_cl = (n_run + size - 1) // size
        for k in range(n_cl):
            s0, s1 = k * size * block, min((k + 1) * size * block, n_seg)
            ends = prof[s0:s1 + 1]
            zc = 0.5 * (ends[:, 1].min() + ends[:, 1].max())
            rmax = np.sqrt(ends[:, 0] ** 2 + (ends[:, 1] - zc) ** 2).max()
            r, z, w = rq[s0 * per:s1 * per], zq[s0 * per:s1 * per], wq[s0 * per:s1 * per]
            rr = np.sqrt(r * r + (z - zc) ** 2)
            u = np.where(rr > 0.0, (z - zc) / np.where(rr > 0.0, rr, 1.0), 1.0)
            x = rr / rmax
            M = np.zeros(n_terms)
            p_prev, p = np.ones_like(u), u
            xn = np.ones_like(u)
            for n in range(n_terms):
                pn = p_prev if n == 0 else p
                M[n] = np.sum(w * xn * pn)
                if n >= 1:
                    p_prev, p = p, ((2 * n + 1) * u * p - n * p_prev) / (n + 1)
                xn = xn * x
            rows.append(np.concatenate([[zc, rmax], M]))
        levels += 1
        if n_cl == 1:
            break
        size *= 2
    return np.array(rows), levels


class BemTables:
    """Segment and far-node tables on a CUDA device, plus the SptBem view."""

    def __init__(self, profile, sigma, n_subdiv=8, device="cuda"):
        import torch

        if not (1 <= n_subdiv <= 64):
            raise ValueError("n_subdiv must be in [1, 64]")
        self.profile = np.asarray(profile, dtype=np.float64)
        self.sigma = np.asarray(sigma, dtype=np.float64)
        self.n_subdiv = int(n_subdiv)
        seg = segment_table(self.profile, self.sigma)
        rq, zq, aq, sq = far_nodes(self.profile, self.sigma, self.n_subdiv)
        n_seg = seg.shape[1]
        nps = 4 * self.n_subdiv
        stride = ((n_seg * nps + 31) // 32) * 32
        node = np.zeros((3, stride))
        node[0, : len(rq)] = rq
        node[1, : len(rq)] = zq
        node[2, : len(rq)] = aq * sq
        self.n_seg = n_seg
        self.nodes_per_seg = nps
        self.seg = torch.as_tensor(np.ascontiguousarray(seg), device=device)
        self.node = torch.as_tensor(node, device=device)
        cn = coarse_nodes(self.profile, self.sigma)
        cstride = ((cn.shape[1] + 1) // 2) * 2
        coarse = np.zeros((3, cstride))
        coarse[:, : cn.shape[1]] = cn
        self.coarse = torch.as_tensor(coarse, device=device)
        blk, rn = run_tables(self.profile, self.sigma)
        self.blk = torch.as_tensor(blk, device=device)
        self.run_nodes = torch.as_tensor(rn, device=device)
        self.n_run_rule = int(blk[5].sum())
        n_run = blk.shape[1]
        self.clusters = None
        if n_run <= MAX_CLUSTER_RUNS:
            ct, levels = cluster_tables(self.profile, self.sigma, self.n_subdiv)
            self.clusters = torch.as_tensor(np.ascontiguousarray(ct), device=device)
            self.cluster_levels = levels
        self.struct = _lib.SptBem()
        s = self.struct
        s.n_seg = n_seg
        s.nodes_per_seg = nps
        s.seg_stride = n_seg
        s.node_stride = stride
        s.seg = self.seg.data_ptr()
        s.node = self.node.data_ptr()
        for i in range(8):
            s.gauss8_x[i] = GAUSS8_X[i]
            s.gauss8_w[i] = GAUSS8_W[i]
        s.far_rule = _lib.FAR_REFERENCE
        s.ratio4, s.ratio2 = RATIO4, RATIO2
        s.coarse = self.coarse.data_ptr()
        s.coarse_stride = cstride
        s.blk = self.blk.data_ptr()
        s.blk_stride = self.blk.shape[1]
        s.ratio_run = RATIO_RUN
        s.run_nodes = self.run_nodes.data_ptr()
        s.run_stride = self.run_nodes.shape[1]
        if self.clusters is not None:
            s.clusters = self.clusters.data_ptr()
            s.cluster_levels = self.cluster_levels
            s.cluster_terms = CLUSTER_TERMS
            s.cluster_kappa = CLUSTER_KAPPA

    def attach_image(self, solution):
        """Add the image-charge tables of a geometry built with z0 (an
        image_charge.ImageChargeSolution on the same device): every view then
        carries them, and the trace adds the image force at every stage."""
        if solution.n_max > _lib.TRACE_IMAGE_MODES:
            raise ValueError(f"image_n_max {solution.n_max} above {_lib.TRACE_IMAGE_MODES} is not offered in the trace")
        self.image = solution
        self.struct.image = solution.struct

    def view(self, far_rule="reference", ratio4=RATIO4, ratio2=RATIO2, ratio_run=RATIO_RUN, bounds=True,
             cluster_kappa=None):
        """An SptBem over these tables with the given far rule (the tables
        must outlive it); ratio_run <= 0 turns the run rule off; bounds=False
        leaves out the run bounds, so every per-point scan visits every
        segment (and the run rule and the clusters are off);
        cluster_kappa <= 0 turns the cluster expansions off."""
        v = _lib.SptBem()
        ctypes.pointer(v)[0] = self.struct
        v.far_rule = _lib.FAR_RULES[far_rule] if isinstance(far_rule, str) else int(far_rule)
        v.ratio4, v.ratio2, v.ratio_run = float(ratio4), float(ratio2), float(ratio_run)
        if cluster_kappa is not None:
            v.cluster_kappa = float(cluster_kappa)
        if not bounds:
            v.blk, v.blk_stride = None, 0
            v.clusters, v.cluster_kappa = None, 0.0
        return v

    @property
    def n_far_nodes(self):
        return self.n_seg * self.nodes_per_seg
