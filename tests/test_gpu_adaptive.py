"""Adaptive far rule on the GPU (SptBem.far_rule = SPT_FAR_ADAPTIVE): the
kernel against the oracle's restatement of the same rule, against the
reference's fixtures, and in traces (float64 and mixed forms)."""

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from bem_b200 import engine  # noqa: E402
from bem_b200.tables import BemTables  # noqa: E402
from oracle import bem as ob  # noqa: E402

import gpu_util as gu  # noqa: E402


def _rel_rows(a, b):
    return np.abs(a - b).max(axis=-1) / np.maximum(np.abs(b).max(axis=-1), 1e-30)


@pytest.mark.parametrize("fixture", ["bem_sphere", "bem_well", "bem_post"])
def test_bem_field_adaptive_fp64(fixture):
    g = load_golden(fixture)
    tab = BemTables(g["profile"], g["sigma"], int(g["n_subdiv"]))
    e = engine.bem_field(tab, g["points"], far_rule="adaptive").cpu().numpy()
    ora = ob.field(g["points"], g["profile"], g["sigma"], int(g["n_subdiv"]), far_rule="adaptive",
                   run_flags=tab.blk[5].cpu().numpy() > 0,
                   clusters=ob.cluster_table(g["profile"], g["sigma"], int(g["n_subdiv"])))
    # near-surface fixture points lose digits to cancellation (the reference
    # rule's parity test allows 1e-10 for the same reason)
    assert _rel_rows(e, ora).max() < 1e-11
    assert _rel_rows(e, g["e_pert"]).max() < 1e-10


@pytest.mark.parametrize("fixture", ["bem_sphere", "bem_well", "bem_post"])
def test_bem_field_adaptive_mixed(fixture):
    g = load_golden(fixture)
    tab = BemTables(g["profile"], g["sigma"], int(g["n_subdiv"]))
    e = engine.bem_field(tab, g["points"], form="mixed", far_rule="adaptive").cpu().numpy()
    assert _rel_rows(e, g["e_pert"]).max() < 1e-5


def test_bem_field_adaptive_benchmark_tip():
    """2000-segment tip: kernel (both rules) against the oracle's adaptive
    rule (run rule and cluster expansions included) at points 2 nm .. 10 um
    from the apex; the rule without the run rule, and without the cluster
    expansions, against the reference rule."""
    g = load_golden("sigma_c1")
    prof, sig = g["profile"], g["sigma"]
    apex = prof[:, 1].max()
    rng = np.random.default_rng(5)
    d = 10 ** rng.uniform(np.log10(2e-9), -5, 64)
    th = rng.uniform(0, 0.6, 64)
    ph = rng.uniform(0, 2 * np.pi, 64)
    r = 50e-9 + d
    pts = np.stack([r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), apex - 50e-9 + r * np.cos(th)], -1)
    tab = BemTables(prof, sig, 8)
    assert tab.n_run_rule > 40  # the straight wall runs
    ada = engine.bem_field(tab, pts, far_rule="adaptive").cpu().numpy()
    seg_only = engine.bem_field(tab, pts, far_rule="adaptive", ratio_run=0.0).cpu().numpy()
    no_cl = engine.bem_field(tab, pts, far_rule="adaptive", cluster_kappa=0.0).cpu().numpy()
    ref = engine.bem_field(tab, pts).cpu().numpy()
    ora = ob.field(pts, prof, sig, 8, far_rule="adaptive", run_flags=tab.blk[5].cpu().numpy() > 0,
                   clusters=ob.cluster_table(prof, sig))
    norm = np.linalg.norm(ora, axis=-1)
    assert (np.abs(ada - ora).max(axis=-1) / norm).max() < 1e-12
    assert (np.abs(ada - ref).max(axis=-1) / norm).max() < 1e-12
    assert (np.abs(seg_only - ref).max(axis=-1) / norm).max() < 1e-12
    # without the expansions the run rule alone: 5e-12 at the few points
    # where the field nearly cancels (~2e5 V/m out of ~1e8 V/m terms)
    assert (np.abs(no_cl - ref).max(axis=-1) / norm).max() < 5e-12
    assert not np.array_equal(no_cl, ada)  # the expansions did take part


def _tip_points(n, seed):
    g = load_golden("sigma_c1")
    apex = g["profile"][:, 1].max()
    rng = np.random.default_rng(seed)
    d = 10 ** rng.uniform(-11, -5, n)
    th = rng.uniform(0, 1.5, n)
    ph = rng.uniform(0, 2 * np.pi, n)
    r = 50e-9 + d
    pts = np.stack([r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), apex - 50e-9 + r * np.cos(th)], -1)
    return g, pts


def test_bem_field_mixed_near_axis_benchmark_tip():
    """Mixed form on the benchmark tip at points near the axis (where the
    float32 Legendre branch takes almost every ring) from 2 nm to 1 mm above
    the apex: within 1e-6 of the float64 reference rule, relative to the whole
    field (uniform 1e6 V/m plus perturbation)."""
    g = load_golden("sigma_c1")
    prof, sig = g["profile"], g["sigma"]
    apex = prof[:, 1].max()
    rng = np.random.default_rng(12)
    d = 10 ** rng.uniform(np.log10(2e-9), -3, 256)
    rho = d * 10 ** rng.uniform(-4, -0.5, 256)
    ph = rng.uniform(0, 2 * np.pi, 256)
    pts = np.stack([rho * np.cos(ph), rho * np.sin(ph), apex + d], -1)
    tab = BemTables(prof, sig, 8)
    ref = engine.bem_field(tab, pts).cpu().numpy()
    tot = np.linalg.norm(ref + np.array([0.0, 0.0, float(g["E_gun"])]), axis=-1)
    for rule in ("reference", "adaptive"):
        mix = engine.bem_field(tab, pts, form="mixed", far_rule=rule).cpu().numpy()
        err = np.abs(mix - ref).max(axis=-1) / tot
        assert err.max() < 1e-6, (rule, err.max())


def test_run_bounds_leave_reference_rule_results_unchanged():
    """The closest-segment search and the near test skip runs of segments by
    their bounds; with the reference rule the field is bit-identical to the
    full scan (points down to 10 pm from the surface, on-surface offsets and
    near segments included)."""
    g, pts = _tip_points(512, 8)
    tab = BemTables(g["profile"], g["sigma"], 8)
    out = []
    for bounds in (True, False):
        view = tab.view("reference", bounds=bounds)
        x, y, z = (torch.as_tensor(np.ascontiguousarray(pts[:, k]), device="cuda") for k in range(3))
        e = [torch.empty_like(x) for _ in range(3)]
        import ctypes
        from bem_b200 import _lib
        _lib.check(_lib.lib().spt_bem_field(x.data_ptr(), y.data_ptr(), z.data_ptr(), len(pts), ctypes.byref(view), 0,
                                            e[0].data_ptr(), e[1].data_ptr(), e[2].data_ptr(), None), "spt_bem_field")
        torch.cuda.synchronize()
        out.append(torch.stack(e, -1).cpu().numpy())
    np.testing.assert_array_equal(out[0], out[1])


def _spec(g, kind):
    spec = dict(kind=kind, E_gun=float(g["E_gun"]), R=float(g["R"]), profile=g["profile"], sigma=g["sigma"],
                n_subdiv=int(g["n_subdiv"]), z_handoff=float(g["z_handoff"]), kill_z_below=0.0)
    if kind == "well_bem":
        spec["H"] = float(g["H"])
    else:
        spec["L"] = float(g["L"])
        spec["z0"] = float(g["z0"])
    return spec


@pytest.mark.parametrize("fixture,form,tol", [("trace_post", "fp64", 1e-8), ("trace_well", "fp64", 1e-8),
                                              ("trace_post", "mixed", 1e-6), ("trace_well", "mixed", 1e-6)])
def test_trace_adaptive_endpoint(fixture, form, tol):
    g = load_golden(fixture)
    spec = _spec(g, dict(trace_post="post_bem", trace_well="well_bem")[fixture])
    out = gu.device_trace(spec, g["pos0"], g["vel0"], g["t_birth"], float(g["t_max"]), float(g["rtol"]),
                          float(g["atol"]), float(g["z_max"]), form=form, far_rule="adaptive")
    rel = np.abs(out["pos"] - g["pos"]).max() / np.abs(g["pos"]).max()
    relv = np.abs(out["vel"] - g["vel"]).max() / np.abs(g["vel"]).max()
    assert rel <= tol and relv <= tol, (rel, relv)
