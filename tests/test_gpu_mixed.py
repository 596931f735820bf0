"""Precision form (SPT_FORM_MIXED): float32 + Kahan pair and far-panel sums,
float64 elsewhere.  Checked against the float64 oracle/fixtures at the
accuracy the form promises: stage quantities to 1e-5 of their scale, trace
endpoints to 1e-6 relative (the chosen-form criterion) on well-conditioned
traces."""

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from bem_b200 import engine  # noqa: E402
from bem_b200.tables import BemTables  # noqa: E402

import gpu_util as gu  # noqa: E402


def test_elliptic_float32_matches_scipy():
    """Float32 K(1-p), E(1-p): the DLMF 19.12 series below p = 1e-2, the
    Hastings approximations (A&S 17.3.34 / 17.3.36, |error| <= 2e-8) above;
    against SciPy's values recorded by the reference, within float32
    rounding (5e-7 relative) for p in [1e-6, 1]."""
    g = load_golden("ellip")
    sel = (g["p"] >= 1e-6)
    K, E = engine.ellip_ke(g["p"][sel], form="mixed")
    np.testing.assert_allclose(K.cpu().numpy(), g["K"][sel], rtol=5e-7, atol=0)
    np.testing.assert_allclose(E.cpu().numpy(), g["E"][sel], rtol=5e-7, atol=0)


@pytest.mark.parametrize("fixture", ["bem_sphere", "bem_well", "bem_post"])
def test_bem_field_mixed(fixture):
    g = load_golden(fixture)
    tab = BemTables(g["profile"], g["sigma"], int(g["n_subdiv"]))
    e = engine.bem_field(tab, g["points"], form="mixed").cpu().numpy()
    ref = g["e_pert"]
    err = np.abs(e - ref).max(axis=-1) / np.maximum(np.abs(ref).max(axis=-1), 1e-30)
    assert err.max() < 1e-5, err.max()


@pytest.mark.parametrize("name,spec", [
    ("flat", dict(kind="flat", E_gun=-1e7, z0=3e-9, kill_z_below=0.0)),
    ("tip", dict(kind="tip", E_gun=-1e8, R=50e-9, z0=3e-9, kill_z_below=0.0)),
])
def test_accel_mixed(name, spec):
    g = load_golden("accel")
    pos, live = g[f"{name}_pos"], g[f"{name}_live"]
    G, E, _ = pos.shape
    acc = engine.accel(gu.device_geometry(spec), pos.reshape(-1, 3), live.reshape(-1), np.full(G * E, gu.Q_E),
                       np.full(G * E, gu.M_E), [E] * G, gu.CM, 1e-12, form="mixed").cpu().numpy().reshape(G, E, 3)
    ref = g[f"{name}_acc"]
    np.testing.assert_allclose(acc, ref, rtol=1e-5, atol=1e-5 * np.abs(ref).max())


@pytest.mark.parametrize("fixture", ["trace_post", "trace_well"])
def test_trace_mixed_endpoint_1e6(fixture):
    g = load_golden(fixture)
    kind = dict(trace_post="post_bem", trace_well="well_bem")[fixture]
    spec = dict(kind=kind, E_gun=float(g["E_gun"]), R=float(g["R"]), profile=g["profile"], sigma=g["sigma"],
                n_subdiv=int(g["n_subdiv"]), z_handoff=float(g["z_handoff"]), kill_z_below=0.0)
    if kind == "well_bem":
        spec["H"] = float(g["H"])
    else:
        spec["L"] = float(g["L"])
        spec["z0"] = float(g["z0"])
    out = gu.device_trace(spec, g["pos0"], g["vel0"], g["t_birth"], float(g["t_max"]), float(g["rtol"]),
                          float(g["atol"]), float(g["z_max"]), form="mixed")
    rel = np.abs(out["pos"] - g["pos"]).max() / np.abs(g["pos"]).max()
    relv = np.abs(out["vel"] - g["vel"]).max() / np.abs(g["vel"]).max()
    assert rel <= 1e-6 and relv <= 1e-6, (rel, relv)


def test_trace_mixed_tip_no_kill_1e6():
    from bem_b200 import workloads as w
    d = w.tip_c2(n_groups=3, n_emit=16, R=50e-9, L=0.0, seed=42)
    spec = dict(kind="tip", E_gun=-1e8, R=50e-9, z0=3e-9, kill_z_below=0.0)
    pos0 = np.stack([d["x"], d["y"], d["z"]], -1).reshape(3, 16, 3)
    vel0 = np.stack([d[k] for k in ("px", "py", "pz")], -1).reshape(3, 16, 3) * (
        gu.ophys.ELEMENTARY_CHARGE / gu.ophys.SPEED_OF_LIGHT) / gu.M_E
    tb = d["t"].reshape(3, 16)
    p, v, td, t, h, log = gu.oracle_trace(spec, pos0, vel0, tb, 1.2e-12, 1e-9, 1e-12, None)
    out = gu.device_trace(spec, pos0, vel0, tb, 1.2e-12, 1e-9, 1e-12, None, form="mixed")
    assert np.abs(out["pos"] - p).max() / np.abs(p).max() <= 1e-6
    assert np.abs(out["vel"] - v).max() / np.abs(v).max() <= 1e-6


def _post_trace(form, far_rule="adaptive", attempts=40, **tracer_attrs):
    g = load_golden("trace_post")
    spec = dict(kind="post_bem", E_gun=float(g["E_gun"]), R=float(g["R"]), L=float(g["L"]), z0=float(g["z0"]),
                profile=g["profile"], sigma=g["sigma"], n_subdiv=int(g["n_subdiv"]), z_handoff=float(g["z_handoff"]),
                kill_z_below=0.0)
    G, E, _ = g["pos0"].shape
    tr = engine.Tracer(gu.device_geometry(spec), form=form, z_max=float(g["z_max"]), far_rule=far_rule)
    for k, v in tracer_attrs.items():
        setattr(tr, k, v)
    b = engine.GroupBatch(g["pos0"].reshape(-1, 3), g["vel0"].reshape(-1, 3), g["t_birth"].reshape(-1),
                          np.full(G * E, gu.Q_E), np.full(G * E, gu.M_E), [E] * G)
    tr.launch(b, tr.params(float(g["t_max"]), 1e-8, 1e-12, 1e-12, gu.CM, attempts))
    torch.cuda.synchronize()
    return b.positions().cpu().numpy(), tr.counter_dict()


@pytest.mark.parametrize("far_rule", ["reference", "adaptive"])
def test_mixed_form_redoes_ill_conditioned_sums_in_float64(far_rule):
    """kappa_max -> 0 declares every float32 sum ill-conditioned: every far
    sum and pair sum is recomputed by the float64 code, so the mixed form
    lands on the float64 form, far closer than the mixed form does without
    the recomputation.  (The two forms are separate kernel instantiations,
    whose float64 multiply-adds the compiler may contract differently; the
    40-attempt trace carries such ulp differences to ~1e-9.)"""
    p64, _ = _post_trace("fp64", far_rule)
    pmx, c = _post_trace("mixed", far_rule, kappa_max=1e-300)
    pf32, _ = _post_trace("mixed", far_rule)
    assert c["fp64_rounds"] > 0 and c["fp64_targets"] > 0
    scale = np.abs(p64).max()
    np.testing.assert_allclose(pmx, p64, rtol=1e-8, atol=1e-8 * scale)
    assert np.abs(pmx - p64).max() < 0.1 * np.abs(pf32 - p64).max()


def test_round_points_changes_the_far_tile_only():
    """A far-sum round of 1 point instead of 4 (reference far rule): other
    summation order, same trace to 1e-10."""
    p4, _ = _post_trace("fp64", "reference")
    p1, _ = _post_trace("fp64", "reference", round_points=1)
    assert not np.array_equal(p1, p4)
    np.testing.assert_allclose(p1, p4, rtol=1e-10, atol=1e-10 * np.abs(p4).max())
