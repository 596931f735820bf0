"""GPU parity: the CUDA path (through the C ABI) against the reference's
golden fixtures and the CPU oracle on the same seeded inputs."""

import numpy as np
import pytest

from conftest import load_golden
from oracle import bem as obem
from oracle import geometry as ogeo

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from bem_b200 import engine  # noqa: E402
from bem_b200.tables import BemTables  # noqa: E402

import gpu_util as gu  # noqa: E402


def test_elliptic_fp64_matches_scipy():
    g = load_golden("ellip")
    K, E = engine.ellip_ke(g["p"])
    np.testing.assert_allclose(K.cpu().numpy(), g["K"], rtol=2e-15, atol=0)
    np.testing.assert_allclose(E.cpu().numpy(), g["E"], rtol=2e-15, atol=0)


def test_ring_field_fp64_matches_reference():
    g = load_golden("ring")
    er, ez = engine.ring_field(g["rho"], g["z"], g["a"])
    np.testing.assert_allclose(er.cpu().numpy(), g["er"], rtol=1e-12, atol=1e-12 * np.abs(g["er"]).max())
    np.testing.assert_allclose(ez.cpu().numpy(), g["ez"], rtol=1e-12, atol=1e-12 * np.abs(g["ez"]).max())


@pytest.mark.parametrize("fixture", ["bem_sphere", "bem_well", "bem_post"])
def test_bem_field_matches_reference(fixture):
    g = load_golden(fixture)
    tab = BemTables(g["profile"], g["sigma"], int(g["n_subdiv"]))
    e = engine.bem_field(tab, g["points"]).cpu().numpy()
    scale = np.abs(g["e_pert"]).max()
    np.testing.assert_allclose(e, g["e_pert"], rtol=1e-11, atol=1e-12 * scale)


@pytest.mark.parametrize("name,spec", [
    ("flat", dict(kind="flat", E_gun=-1e7, z0=3e-9, kill_z_below=0.0)),
    ("flat_noimg", dict(kind="flat", E_gun=-1e7, z0=None, kill_z_below=0.0)),
    ("tip", dict(kind="tip", E_gun=-1e8, R=50e-9, z0=3e-9, kill_z_below=0.0)),
])
def test_accel_matches_reference(name, spec):
    g = load_golden("accel")
    pos, live = g[f"{name}_pos"], g[f"{name}_live"]
    G, E, _ = pos.shape
    acc = engine.accel(gu.device_geometry(spec), pos.reshape(-1, 3), live.reshape(-1), np.full(G * E, gu.Q_E),
                       np.full(G * E, gu.M_E), [E] * G, gu.CM, 1e-12).cpu().numpy().reshape(G, E, 3)
    ref = g[f"{name}_acc"]
    np.testing.assert_allclose(acc, ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())


def _bem_spec(fixture, kind):
    g = load_golden(fixture)
    s = dict(kind=kind, E_gun=float(g["E_gun"]), R=float(g["R"]), profile=g["profile"], sigma=g["sigma"],
             n_subdiv=int(g["n_subdiv"]), z_handoff=float(g["z_handoff"]), kill_z_below=0.0)
    if kind == "well_bem":
        s["H"] = float(g["H"])
    if kind == "post_bem":
        s["L"] = float(g["L"])
        s["z0"] = float(g["z0"])
    return s, g


@pytest.mark.parametrize("fixture,kind", [("bem_sphere", "tip_bem"), ("bem_well", "well_bem"), ("bem_post", "post_bem")])
def test_bem_accel_matches_oracle(fixture, kind):
    spec, g = _bem_spec(fixture, kind)
    rng = np.random.default_rng(5)
    pts = g["points"]
    G, E = 4, 9
    idx = rng.integers(0, len(pts), G * E)
    pos = pts[idx].reshape(G, E, 3) * (1 + 1e-3 * rng.uniform(size=(G, E, 1)))
    live = rng.uniform(size=(G, E)) < 0.85
    q = np.full((G, E), gu.Q_E)
    m = np.full((G, E), gu.M_E)
    ref = ogeo.make_accel(spec, q, m, gu.CM, 1e-12)(pos, None, live, np.arange(G))
    acc = engine.accel(gu.device_geometry(spec), pos.reshape(-1, 3), live.reshape(-1), q.reshape(-1), m.reshape(-1),
                       [E] * G, gu.CM, 1e-12).cpu().numpy().reshape(G, E, 3)
    np.testing.assert_allclose(acc, ref, rtol=1e-10, atol=1e-11 * np.abs(ref).max())


def _trace_spec(name, g):
    if name.startswith("trace_flat"):
        return dict(kind="flat", E_gun=-1e7, z0=3e-9, kill_z_below=0.0)
    if name == "trace_tip":
        return dict(kind="tip", E_gun=-1e8, R=50e-9, z0=3e-9, kill_z_below=0.0)
    kind = dict(trace_tip_bem="tip_bem", trace_well="well_bem", trace_post="post_bem")[name]
    s = dict(kind=kind, E_gun=float(g["E_gun"]), R=float(g["R"]), profile=g["profile"], sigma=g["sigma"],
             n_subdiv=int(g["n_subdiv"]), z_handoff=float(g["z_handoff"]), kill_z_below=0.0)
    if kind == "well_bem":
        s["H"] = float(g["H"])
    if kind == "post_bem":
        s["L"] = float(g["L"])
        s["z0"] = float(g["z0"])
    return s


# Endpoint tolerance per fixture, set from the oracle's own sensitivity:
# scaling vel0 by (1 + 1e-15) moves the oracle's endpoints by 7.3e-9
# (trace_flat), 2.2e-10 (trace_tip), 1.4e-7 (trace_tip_bem) and < 1e-14
# (trace_post, trace_well) -- particles killed at z_max freeze at a
# step-grid-dependent point.  The bound is 1e-10 where the problem allows it.
TRACE_RTOL = dict(trace_flat=1e-6, trace_flat_c0=1e-6, trace_tip=1e-7, trace_tip_bem=1e-5, trace_post=1e-10,
                  trace_well=1e-10)


# trace_well emits on the well floor itself: stage points land within the
# reference's on-surface threshold dist^2 < (1e-9 L)^2 or just outside it
# depending on the last ulp, and the field is evaluated at the 1e-4 L offset
# point in one case and not in the other.  Early step sizes then differ by
# up to 1e-4 (the decisions stay identical).  trace_tip_bem, the fixture
# whose endpoints move 1.4e-7 under a 1e-15 change of its inputs, has step
# times within 2.3e-6 once the far sums take rounds of 4 points (the
# summation order): checked at 1e-5, its endpoint tolerance.
T_ACC_RTOL = dict(trace_well=1e-3, trace_tip_bem=1e-5)


@pytest.mark.parametrize("name", sorted(TRACE_RTOL))
def test_trace_matches_reference(name):
    g = load_golden(name)
    spec = _trace_spec(name, g)
    out = gu.device_trace(spec, g["pos0"], g["vel0"], g["t_birth"], float(g["t_max"]), float(g["rtol"]),
                          float(g["atol"]), float(g["z_max"]))
    assert np.all(out["status"] == 2)
    attempts = out["n_acc"] + out["n_rej"]
    same = (attempts == g["attempts"]) & (out["n_acc"] == g["n_acc"])
    assert same.mean() >= 0.99, (attempts, g["attempts"], out["n_acc"], g["n_acc"])
    # Accepted step end times, reconstructed from the attempt log.  The
    # embedded error estimate h*sum(E_j k_j) cancels to ~rtol of the slopes,
    # so ulp-level slope differences become up to ~1e-3 relative differences
    # of the error norm and ~1e-7 of the next step size; the decisions above
    # are exact, the step times agree to 1e-6.
    for k in range(len(attempts)):
        hs, errs = out["log_h"][k, :attempts[k]], out["log_err"][k, :attempts[k]]
        acc = errs <= 1.0
        t_acc = float(g["t_birth"][k].min()) + np.cumsum(np.where(acc, hs, 0.0))[acc]
        ref = g["t_acc"][k, : g["n_acc"][k]]
        np.testing.assert_allclose(t_acc, ref, rtol=T_ACC_RTOL.get(name, 1e-6))
    rt = TRACE_RTOL[name]
    np.testing.assert_allclose(out["pos"], g["pos"], rtol=rt, atol=rt * np.abs(g["pos"]).max())
    np.testing.assert_allclose(out["vel"], g["vel"], rtol=rt, atol=rt * np.abs(g["vel"]).max())


@pytest.mark.parametrize("kind", ["flat", "tip"])
def test_trace_well_conditioned_1e10(kind):
    """No particle is killed before t_max: the endpoints meet 1e-10 relative
    and the step-acceptance sequences are identical."""
    from bem_b200 import workloads as w
    rng_seed = dict(flat=41, tip=42)[kind]
    if kind == "flat":
        d = w.flat_c0(n_groups=3, n_emit=16, seed=rng_seed)
        # no image force: with it, slow electrons fall back onto their own
        # image (a softened singularity) unless a kill plane stops them
        spec = dict(kind="flat", E_gun=-1e7, z0=None, kill_z_below=None)
        t_max = 1.5e-12
    else:
        d = w.tip_c2(n_groups=3, n_emit=16, R=50e-9, L=0.0, seed=rng_seed)
        spec = dict(kind="tip", E_gun=-1e8, R=50e-9, z0=3e-9, kill_z_below=0.0)
        t_max = 1.2e-12
    pos0 = np.stack([d["x"], d["y"], d["z"]], -1).reshape(3, 16, 3)
    vel0 = np.stack([d[k] for k in ("px", "py", "pz")], -1).reshape(3, 16, 3) * (gu.ophys.ELEMENTARY_CHARGE / gu.ophys.SPEED_OF_LIGHT) / gu.M_E
    tb = d["t"].reshape(3, 16)
    p, v, td, t, h, log = gu.oracle_trace(spec, pos0, vel0, tb, t_max, 1e-8, 1e-12, None)
    assert np.all(np.isinf(td))
    out = gu.device_trace(spec, pos0, vel0, tb, t_max, 1e-8, 1e-12, None)
    np.testing.assert_allclose(out["pos"], p, rtol=1e-10, atol=1e-10 * np.abs(p).max())
    for k in range(3):
        n = len(log[k][0])
        assert out["n_acc"][k] + out["n_rej"][k] == n
        np.testing.assert_array_equal(out["log_err"][k, :n] <= 1.0, log[k][2])
        np.testing.assert_allclose(out["log_h"][k, :n], log[k][0], rtol=1e-6)
    np.testing.assert_allclose(out["vel"], v, rtol=1e-10, atol=1e-10 * np.abs(v).max())


def test_bounded_slice_matches_oracle():
    """spt_trace with max_attempts stops every group after that many
    attempts, exactly where the oracle stops with the same budget."""
    g = load_golden("trace_post")
    spec = _trace_spec("trace_post", g)
    args = (g["pos0"], g["vel0"], g["t_birth"], float(g["t_max"]), 1e-8, 1e-12, float(g["z_max"]))
    p, v, td, t, h, log = gu.oracle_trace(spec, *args, max_attempts=30)
    out = gu.device_trace(spec, *args, max_attempts=30)
    assert out["n_acc"][0] + out["n_rej"][0] == 30
    np.testing.assert_allclose(out["t"], t, rtol=1e-12)
    np.testing.assert_allclose(out["pos"], p, rtol=1e-10, atol=1e-10 * np.abs(p).max())


@pytest.mark.parametrize("fixture", ["bem_sphere", "bem_well", "bem_post", "sigma_c1"])
def test_bem_solve_matches_reference(fixture):
    """GPU collocation assembly + LU reproduces the reference's solved density."""
    from bem_b200.bem_solve import solve_dirichlet
    g = load_golden(fixture)
    Ez = float(g["E_gun"])
    sigma = solve_dirichlet(g["profile"], lambda rho, z: Ez * z)
    np.testing.assert_allclose(sigma, g["sigma"], rtol=1e-9, atol=1e-11 * np.abs(g["sigma"]).max())
