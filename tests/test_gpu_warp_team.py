"""One group per warp (SptTraceParams.team = SPT_TEAM_WARP) against one
group per CTA and against the reference.

The warp team evaluates each BEM point with the CTA team's own warp routines
(closest segment, near quadrature, adaptive far sum), so the two differ only
in the order of the pair sums (sources in order on one lane, against the CTA
team's sources split over several lanes and added by shuffles): ulp-level
slope differences, which the embedded error estimate turns into ~1e-7
relative step-size differences.  Compared, therefore, like two forms: the
same attempt counts on almost every group, endpoints at the common end time
within 1e-6, screens and output snapshots alike.  The library's automatic
choice (team 0) must be the warp team bit for bit where it is offered.
"""

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from bem_b200 import _lib, autotune, engine, workloads  # noqa: E402

import gpu_util as gu  # noqa: E402


def _c1():
    g = load_golden("trace_c1")
    spec = dict(kind="post_bem", E_gun=float(g["E_gun"]), R=float(g["R"]), L=float(g["L"]), z0=float(g["z0"]),
                profile=g["profile"], sigma=g["sigma"], n_subdiv=int(g["n_subdiv"]), z_handoff=float(g["z_handoff"]),
                kill_z_below=0.0)
    return g, gu.device_geometry(spec)


def _groups(g, sizes, seed):
    d = workloads.tip_c4(g["profile"], g["sigma"], n_groups=len(sizes), seed=seed, sizes=sizes)
    pos = np.stack([d["x"], d["y"], d["z"]], -1)
    vel = np.stack([d["px"], d["py"], d["pz"]], -1) * gu.ophys.ELEMENTARY_CHARGE / gu.ophys.SPEED_OF_LIGHT / gu.M_E
    return pos, vel, d["t"], np.asarray(d["group_sizes"])


def _trace(geo, team, pos, vel, tb, sizes, t_max, screens=None, output_times=None):
    tr = engine.Tracer(geo, form="fp64", far_rule="adaptive", z_max=1e-3)
    tr.team = team
    n = len(pos)
    b = engine.GroupBatch(pos, vel, tb, np.full(n, gu.Q_E), np.full(n, gu.M_E), sizes)
    rec = tr.run(b, t_max, 1e-9, 1e-12, 1e-12, gu.CM, screens=screens, output_times=output_times)
    torch.cuda.synchronize()
    out = dict(pos=b.positions().cpu().numpy(), vel=b.velocities().cpu().numpy(), t_death=b.t_death.cpu().numpy(),
               t=b.t.cpu().numpy(), att=(b.n_accepted + b.n_rejected).cpu().numpy(), counters=tr.counter_dict())
    if screens is not None or output_times is not None:
        out["screens"], out["outputs"] = rec.screen_records(), rec.output_records()
    return out


def _rel(a, b):
    return np.linalg.norm(a - b, axis=-1) / np.maximum(np.linalg.norm(b, axis=-1), 1e-300)


def _same_trace(a, b, t_max):
    assert np.all(a["t"] == t_max) and np.all(b["t"] == t_max)
    assert np.mean(a["att"] == b["att"]) >= 0.9, (a["att"], b["att"])
    np.testing.assert_array_equal(np.isfinite(a["t_death"]), np.isfinite(b["t_death"]))
    alive = np.isinf(b["t_death"])
    assert _rel(a["pos"][alive], b["pos"][alive]).max() < 1e-6
    assert _rel(a["vel"][alive], b["vel"][alive]).max() < 1e-6
    dead = ~alive
    if dead.any():
        assert np.all(np.abs(a["t_death"][dead] - b["t_death"][dead]) <= 1e-6 * np.abs(b["t_death"][dead]))


def test_warp_team_matches_cta_team():
    """64 groups of 32 and 32 groups of 1 to 31 particles on the 2000-panel
    C1 capsule, traced to 2 ps by both teams.  So few groups leave most of
    the GPU's warps without one, so the library's own choice is the CTA
    team (bit for bit)."""
    g, geo = _c1()
    rng = np.random.default_rng(5)
    sizes = np.concatenate([np.full(64, 32), rng.integers(1, 32, 32)])
    pos, vel, tb, sizes = _groups(g, sizes, seed=11)
    t_max = 2e-12
    warp = _trace(geo, _lib.TEAM_WARP, pos, vel, tb, sizes, t_max)
    auto = _trace(geo, _lib.TEAM_AUTO, pos, vel, tb, sizes, t_max)
    cta = _trace(geo, _lib.TEAM_CTA, pos, vel, tb, sizes, t_max)
    for k in ("pos", "vel", "t_death", "t", "att"):
        np.testing.assert_array_equal(auto[k], cta[k], err_msg=k)
    _same_trace(warp, cta, t_max)
    # the same BEM work: ring evaluations per accepted particle-step within 1 %
    rw = warp["counters"]["ring_far"] / warp["counters"]["particle_steps"]
    rc = cta["counters"]["ring_far"] / cta["counters"]["particle_steps"]
    assert abs(rw / rc - 1.0) < 0.01


def test_automatic_choice_is_the_warp_team_when_the_groups_fill_the_gpu():
    """As many groups of 32 as the GPU holds warps (SMs x 16), four attempts
    each: the library's own choice is the warp team, bit for bit."""
    g, geo = _c1()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    pos, vel, tb, sizes = _groups(g, np.full(16 * sms, 32), seed=14)
    n = len(pos)
    out = {}
    for team in (_lib.TEAM_WARP, _lib.TEAM_AUTO, _lib.TEAM_CTA):
        tr = engine.Tracer(geo, form="fp64", far_rule="adaptive", z_max=1e-3)
        tr.team = team
        b = engine.GroupBatch(pos, vel, tb, np.full(n, gu.Q_E), np.full(n, gu.M_E), sizes)
        tr.launch(b, tr.params(2e-12, 1e-9, 1e-12, 1e-12, gu.CM, 4))
        torch.cuda.synchronize()
        out[team] = (b.positions().cpu().numpy(), b.velocities().cpu().numpy(), b.t.cpu().numpy(),
                     (b.n_accepted + b.n_rejected).cpu().numpy())
    for a, b in zip(out[_lib.TEAM_AUTO], out[_lib.TEAM_WARP]):
        np.testing.assert_array_equal(a, b)
    assert np.all(out[_lib.TEAM_WARP][3] == 4)
    # the CTA team's pair sums add in another order: same steps, last digits
    np.testing.assert_allclose(out[_lib.TEAM_CTA][2], out[_lib.TEAM_WARP][2], rtol=1e-6)


def test_warp_team_screens_and_outputs_match_cta_team():
    g, geo = _c1()
    pos, vel, tb, sizes = _groups(g, np.full(24, 32), seed=12)
    L = float(g["L"])
    t_max = 1.5e-12
    kw = dict(screens=[L + 60e-9, L + 400e-9], output_times=[0.4e-12, 0.9e-12, 1.2e-12])
    warp = _trace(geo, _lib.TEAM_WARP, pos, vel, tb, sizes, t_max, **kw)
    cta = _trace(geo, _lib.TEAM_CTA, pos, vel, tb, sizes, t_max, **kw)
    _same_trace(warp, cta, t_max)
    n_cross = 0
    for a, b in zip(warp["screens"], cta["screens"]):
        assert (a is None) == (b is None)
        if a is None:
            continue
        ia, ib = np.argsort(a["particle"], kind="stable"), np.argsort(b["particle"], kind="stable")
        np.testing.assert_array_equal(a["particle"][ia], b["particle"][ib])
        np.testing.assert_allclose(a["t"][ia], b["t"][ib], rtol=1e-6)
        pa = np.stack([a["x"], a["y"], a["z"]], -1)[ia]
        pb = np.stack([b["x"], b["y"], b["z"]], -1)[ib]
        assert _rel(pa, pb).max() < 1e-6
        n_cross += len(ia)
    assert n_cross > 0
    for a, b in zip(warp["outputs"], cta["outputs"]):
        assert (a is None) == (b is None)
        if a is None:
            continue
        np.testing.assert_array_equal(a["particle"], b["particle"])
        np.testing.assert_array_equal(a["t"], b["t"])
        pa, pb = np.stack([a["x"], a["y"], a["z"]], -1), np.stack([b["x"], b["y"], b["z"]], -1)
        assert _rel(pa, pb).max() < 1e-6


def test_warp_team_small_sizes_match_reference():
    """The C4 size bins 1, 2 and 7 (reference fixtures, traced to 20 ps) in one
    warp-team launch: the reference's attempt counts on at least 99 % of
    groups (its quadrature against the adaptive rule's, ~1e-13 of the field
    apart) and endpoints within 1e-6."""
    fx = [load_golden(f"trace_c4_s{E}") for E in (1, 2, 7)]
    f0 = fx[0]
    spec = dict(kind="post_bem", E_gun=float(f0["E_gun"]), R=float(f0["R"]), L=float(f0["L"]), z0=float(f0["z0"]),
                profile=f0["profile"], sigma=f0["sigma"], n_subdiv=int(f0["n_subdiv"]),
                z_handoff=float(f0["z_handoff"]), kill_z_below=0.0)
    geo = gu.device_geometry(spec)
    pos = np.concatenate([f["pos0"].reshape(-1, 3) for f in fx])
    vel = np.concatenate([f["vel0"].reshape(-1, 3) for f in fx])
    tb = np.concatenate([f["t_birth"].reshape(-1) for f in fx])
    sizes = np.concatenate([[f["pos0"].shape[1]] * f["pos0"].shape[0] for f in fx])
    o = _trace(geo, _lib.TEAM_WARP, pos, vel, tb, sizes, float(f0["t_max"]))
    att = np.concatenate([f["attempts"] for f in fx])
    assert np.mean(o["att"] == att) >= 0.99, (o["att"], att)
    ref_pos = np.concatenate([f["pos"].reshape(-1, 3) for f in fx])
    ref_vel = np.concatenate([f["vel"].reshape(-1, 3) for f in fx])
    ref_td = np.concatenate([f["t_death"].reshape(-1) for f in fx])
    np.testing.assert_array_equal(np.isfinite(o["t_death"]), np.isfinite(ref_td))
    alive = np.isinf(ref_td)
    assert _rel(o["pos"][alive], ref_pos[alive]).max() < 1e-6
    assert _rel(o["vel"][alive], ref_vel[alive]).max() < 1e-6


def test_autotuner_offers_the_team_choice():
    g, geo = _c1()
    pos, vel, tb, sizes = _groups(g, np.full(32, 32), seed=13)
    tr = engine.Tracer(geo, form="fp64", far_rule="adaptive", z_max=1e-3)
    assert autotune.warp_team_offered(tr, sizes)
    n = len(pos)
    res = autotune.tune(tr, pos, vel, tb, np.full(n, gu.Q_E), np.full(n, gu.M_E), sizes, 2e-12, 1e-9, 1e-12, 1e-12,
                        gu.CM, n_sample=32, warm=8, attempts=4, repeats=1, threads=(256,))
    assert res["team"] in (_lib.TEAM_WARP, _lib.TEAM_CTA)
    assert "team=warp" in res["timings"] and "team=cta" in res["timings"]
    mixed = engine.Tracer(geo, form="mixed", far_rule="adaptive", z_max=1e-3)
    assert not autotune.warp_team_offered(mixed, sizes)


def test_tuned_warp_team_is_not_applied_to_other_forms():
    g, geo = _c1()
    cfg = dict(team=_lib.TEAM_WARP, cta_threads=256, round_points=4, ratios=[8.0, 300.0, 4.0], order="largest_first")
    mixed = engine.Tracer(geo, form="mixed", far_rule="adaptive", z_max=1e-3)
    autotune.apply(cfg, mixed)
    assert mixed.team == _lib.TEAM_AUTO
    fp64 = engine.Tracer(geo, form="fp64", far_rule="adaptive", z_max=1e-3)
    autotune.apply(cfg, fp64)
    assert fp64.team == _lib.TEAM_AUTO  # the library then gives the warp team the launches it fills
    autotune.apply(dict(cfg, team=_lib.TEAM_CTA), fp64)
    assert fp64.team == _lib.TEAM_CTA
