"""The adaptive far rule (whole-segment Gauss-4 / Gauss-2 for distant
segments) in the oracle, against the reference's sub-panel rule: the two
agree far below the tolerance of every form, on the fixtures' geometries and
on the 2000-segment benchmark tip (profile and solved density fixture)."""

import numpy as np
import pytest

from conftest import load_golden
from oracle import bem as ob


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("fixture", ["bem_sphere", "bem_well", "bem_post"])
def test_adaptive_matches_reference_rule_on_fixtures(fixture):
    g = load_golden(fixture)
    ref = ob.field(g["points"], g["profile"], g["sigma"], int(g["n_subdiv"]))
    ada = ob.field(g["points"], g["profile"], g["sigma"], int(g["n_subdiv"]), far_rule="adaptive")
    assert _rel(ada, g["e_pert"]) < 1e-10
    assert _rel(ada, ref) < 1e-10


def test_adaptive_matches_reference_rule_on_benchmark_tip():
    """Points 2 nm .. 10 um from the apex of the 50 nm / 5 um tip, on and off
    the axis: relative to the perturbation field at each point."""
    g = load_golden("sigma_c1")
    prof, sig = g["profile"], g["sigma"]
    apex = prof[:, 1].max()
    R = 50e-9
    pts = []
    for d in (2e-9, 1e-8, 1e-7, 1e-6, 1e-5):
        for th in (0.0, 0.5):
            pts.append([(R + d) * np.sin(th), 0.0, apex - R + (R + d) * np.cos(th)])
    pts = np.array(pts)
    ref = ob.field(pts, prof, sig, 8)
    ada = ob.field(pts, prof, sig, 8, far_rule="adaptive")
    rel = np.abs(ada - ref).max(axis=-1) / np.linalg.norm(ref, axis=-1)
    assert rel.max() < 1e-12, rel


def test_run_rule_matches_reference_rule_on_benchmark_tip():
    """The run rule (product-integration weights on flagged straight runs)
    on top of the segment rules: still within 1e-12 of the reference rule
    relative to the whole field (uniform 1e6 V/m plus perturbation)."""
    from bem_b200.tables import run_tables
    g = load_golden("sigma_c1")
    prof, sig = g["profile"], g["sigma"]
    blk, nodes = run_tables(prof, sig)
    R, Z, W, _, _, _ = ob.run_rule_nodes(prof, sig)
    np.testing.assert_allclose(W.ravel(), nodes[2], rtol=1e-12, atol=1e-12 * np.abs(nodes[2]).max())
    assert blk[5].sum() >= 50
    apex = prof[:, 1].max()
    pts = np.array([[0.0, 0.0, apex + d] for d in (2e-9, 1e-7, 1e-6, 1e-5, 1e-4)]
                   + [[3e-7, 0.0, apex - 1e-7], [1e-6, 0.0, 0.5 * apex]])
    ref = ob.field(pts, prof, sig, 8)
    ada = ob.field(pts, prof, sig, 8, far_rule="adaptive", run_flags=blk[5] > 0)
    tot = np.linalg.norm(ref + np.array([0.0, 0.0, float(g["E_gun"])]), axis=-1)
    assert (np.abs(ada - ref).max(axis=-1) / tot).max() < 1e-12


def test_adaptive_uses_fewer_nodes_on_benchmark_tip():
    """Node count of the adaptive rule for one round of points near the apex:
    a small fraction of the reference's n_seg * 32."""
    g = load_golden("sigma_c1")
    prof = g["profile"]
    seg = ob.segments(prof)
    apex = prof[:, 1].max()
    p = np.array([0.0, apex + 5e-9])
    delta = p[None, :] - seg["p0"]
    proj = np.clip(np.sum(delta * seg["unit"], axis=1), 0.0, seg["length"])
    dist = np.linalg.norm(delta - proj[:, None] * seg["unit"], axis=1)
    r = dist / seg["length"]
    nodes = np.where(r < 8.0, 32, np.where(r < 300.0, 4, 2)).sum()
    assert nodes < len(seg["length"]) * 32 / 10, nodes


def test_cluster_expansion_matches_reference_far_sum():
    """A cluster's multipole expansion (32 terms) against its own reference
    nodes, at points 3 to 20 radii away in every direction: within 1e-13 of
    the cluster's field scale sum |w| / (4 pi d^2)."""
    g = load_golden("sigma_c1")
    prof, sig = g["profile"], g["sigma"]
    levels = ob.cluster_table(prof, sig)
    rq, zq, aq, sq = ob.far_nodes(prof, sig, 8)
    wq = aq * sq
    rng = np.random.default_rng(3)
    for l, k in ((0, 0), (0, 2), (2, 1), (3, 0), (len(levels) - 1, 0)):
        zc, rmax, M, s0, s1 = levels[l][k]
        sl = slice(s0 * 32, s1 * 32)
        for _ in range(12):
            d = 3.0 * rmax * np.exp(rng.uniform(0.0, np.log(20.0 / 3.0)))
            ang = rng.uniform(0.02, np.pi - 0.02)
            rho, z = d * np.sin(ang), zc + d * np.cos(ang)
            got = np.array(ob.cluster_field(zc, rmax, M, rho, z))
            er, ez = ob.ring_field(rho, z - zq[sl], rq[sl])
            ref = np.array([np.sum(wq[sl] * er), np.sum(wq[sl] * ez)])
            scale = np.sum(np.abs(wq[sl])) / (4 * np.pi * d * d)
            assert np.abs(got - ref).max() <= 1e-13 * scale


def test_adaptive_rule_with_clusters_matches_reference_rule():
    """The adaptive rule with run rule and cluster expansions, against the
    reference quadrature, on the C1 tip from 2 nm to 30 um away: within
    1e-12 of the whole field (uniform included)."""
    from bem_b200 import tables
    g = load_golden("sigma_c1")
    prof, sig = g["profile"], g["sigma"]
    rng = np.random.default_rng(4)
    n = 24
    d = np.exp(rng.uniform(np.log(2e-9), np.log(3e-5), n))
    th = rng.uniform(0.0, 1.2, n)
    pts = np.stack([(50e-9 + d) * np.sin(th), np.zeros(n), 5e-6 + (50e-9 + d) * np.cos(th)], -1)
    ref = ob.field(pts, prof, sig)
    blk, _ = tables.run_tables(prof, sig)
    got = ob.field(pts, prof, sig, far_rule="adaptive", run_flags=blk[5] > 0, clusters=ob.cluster_table(prof, sig))
    tot = np.linalg.norm(ref + np.array([0.0, 0.0, float(g["E_gun"])]), axis=-1)
    assert (np.abs(got - ref).max(axis=-1) / tot).max() <= 1e-12
