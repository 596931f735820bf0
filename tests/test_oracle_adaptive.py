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
