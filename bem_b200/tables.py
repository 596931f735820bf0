"""Device tables of a solved axisymmetric BEM problem (profile, sigma).

Built once per geometry, like the reference's per-device field cache
(bem/axisymmetric.py:474-498, backend.py:49-51):

* segment table  [11, n_seg]: p0 (rho, z), tangent p1 - p0, length, unit
  tangent, unit left normal, density at both ends (bem/axisymmetric.py:329-338,
  490-498);
* far-node table [3, stride]: rho_q, z_q, w_q = area_q * sigma_q of the
  Gauss-4 rule on n_subdiv equal sub-panels per segment, segment-major
  (bem/axisymmetric.py:305-326, 561).  Rows are padded to a multiple of 32
  nodes so every row starts 16-byte aligned for the TMA bulk copies.
"""

import numpy as np

from . import _lib

GAUSS4_X, GAUSS4_W = np.polynomial.legendre.leggauss(4)
GAUSS8_X, GAUSS8_W = np.polynomial.legendre.leggauss(8)


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

    @property
    def n_far_nodes(self):
        return self.n_seg * self.nodes_per_seg
