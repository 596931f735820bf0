"""Learned form: the surrogate MLP evaluated with tcgen05 inside the stage
kernel, exact BEM sums inside the near-surface band and for spot checks.
Trained here (small) on the post-tip fixture geometry.

Checks: the in-kernel network agrees with the standalone one
(FieldSurrogate.predict); with every point exact (band covering all, or
spot = 1) the learned form reproduces the mixed form; a trace
driven by the surrogate stays close to the exact one and does a fraction of
its ring evaluations (the ablation); and, trained at the full learned-form
specification on the C1 tip, the measured comparison with the chosen form
on C4-sized groups (time to the same end time, attempts, endpoint error
against the plain float64 form)."""

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from bem_b200 import engine, surrogate as sg  # noqa: E402

import gpu_util as gu  # noqa: E402


@pytest.fixture(scope="module")
def post():
    g = load_golden("trace_post")
    spec = dict(kind="post_bem", E_gun=float(g["E_gun"]), R=float(g["R"]), L=float(g["L"]), z0=float(g["z0"]),
                profile=g["profile"], sigma=g["sigma"], n_subdiv=int(g["n_subdiv"]), z_handoff=float(g["z_handoff"]),
                kill_z_below=0.0)
    geo = gu.device_geometry(spec)
    model = sg.train(geo, n_points=400_000, steps=6000, batch=8192, seed=4)
    return g, geo, model


def _points(geo, n, seed, d_min=5e-9, d_max=1e-6):
    rng = np.random.default_rng(seed)
    rho, z, _, _, _ = sg.sample_points(geo, n, rng, d_min=d_min, d_max=d_max)
    phi = rng.uniform(0, 2 * np.pi, n)
    return rho, z, np.stack([rho * np.cos(phi), rho * np.sin(phi), z], -1)


def _rho_z(E, pts):
    rho = np.hypot(pts[:, 0], pts[:, 1])
    return (E[:, 0] * pts[:, 0] + E[:, 1] * pts[:, 1]) / rho, E[:, 2]


def _run(g, geo, form, model=None, band=5e-9, spot=0.01, attempts=40):
    G, E, _ = g["pos0"].shape
    tr = engine.Tracer(geo, form=form, z_max=float(g["z_max"]), surrogate=model, band=band, spot=spot)
    b = engine.GroupBatch(g["pos0"].reshape(-1, 3), g["vel0"].reshape(-1, 3), g["t_birth"].reshape(-1),
                          np.full(G * E, gu.Q_E), np.full(G * E, gu.M_E), [E] * G)
    tr.launch(b, tr.params(float(g["t_max"]), 1e-8, 1e-12, 1e-12, gu.CM, attempts))
    torch.cuda.synchronize()
    return tr, b.positions().cpu().numpy(), b.status.cpu().numpy()


def test_surrogate_fit_is_usable(post):
    """A small fit (the kernel path is what these tests check); the full
    training reaches about 1% median error near the surface."""
    g, geo, model = post
    rho, z, _ = _points(geo, 4000, 7)
    E = sg.label(geo, rho, z)
    pr, pz = model.predict(rho, z)
    err = np.hypot(pr - E[:, 0], pz - E[:, 1]) / np.hypot(E[:, 0], E[:, 1])
    assert np.median(err) < 0.25, np.median(err)


def test_kernel_network_matches_standalone(post):
    """spt_surrogate_field with no band and no spot checks is the network
    alone: same BF16 weights and activations as FieldSurrogate.predict, so the
    two agree up to FP32 summation order and BF16 rounding ties."""
    g, geo, model = post
    rho, z, pts = _points(geo, 3000, 11, d_min=1e-9, d_max=1e-4)
    bind = engine.SurrogateBinding(model, band=0.0, spot=0.0)
    E = engine.surrogate_field(geo.bem_tables("cuda"), bind, pts).cpu().numpy()
    kr, kz = _rho_z(E, pts)
    hr, hz = model.predict(rho, z)
    rel = np.hypot(kr - hr, kz - hz) / np.hypot(hr, hz)
    assert np.median(rel) < 1e-3, np.median(rel)
    assert np.quantile(rel, 0.99) < 2e-2, np.quantile(rel, 0.99)
    n_sur, n_band, n_spot, _ = bind.stats()
    assert (n_sur, n_band, n_spot) == (len(pts), 0, 0)


def test_band_covering_everything_is_the_exact_field(post):
    g, geo, model = post
    _, _, pts = _points(geo, 1024, 13)
    tables = geo.bem_tables("cuda")
    bind = engine.SurrogateBinding(model, band=1.0, spot=0.0)
    E = engine.surrogate_field(tables, bind, pts).cpu().numpy()
    ref = engine.bem_field(tables, pts, form="mixed").cpu().numpy()
    # same device code in another kernel: equal up to the compiler's
    # contraction choices in the float32 sums (the network is off by percents)
    np.testing.assert_allclose(E, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    assert bind.stats()[:3] == (0, len(pts), 0)


def test_band_partition_selects_per_point(post):
    """A band splitting the points: each one gets the exact field inside the
    band and the network's outside it, whatever the order of the mix."""
    g, geo, model = post
    band = 2e-8
    rho, z, pts = _points(geo, 1000, 19, d_min=2e-9, d_max=2e-7)
    _, _, d = model.closest(rho, z)
    keep = np.abs(d - band) > 1e-3 * band
    rho, z, pts, d = rho[keep], z[keep], pts[keep], d[keep]
    inside = d < band
    assert 0.2 < inside.mean() < 0.8
    tables = geo.bem_tables("cuda")
    bind = engine.SurrogateBinding(model, band=band, spot=0.0)
    E = engine.surrogate_field(tables, bind, pts).cpu().numpy()
    E_net = engine.surrogate_field(tables, engine.SurrogateBinding(model, 0.0, 0.0), pts).cpu().numpy()
    E_ex = engine.bem_field(tables, pts, form="mixed").cpu().numpy()
    np.testing.assert_array_equal(E[~inside], E_net[~inside])
    scale = np.abs(E_ex[inside]).max()
    np.testing.assert_allclose(E[inside], E_ex[inside], rtol=1e-6, atol=1e-9 * scale)
    assert bind.stats()[:3] == (int((~inside).sum()), int(inside.sum()), 0)


def test_spot_checks_record_the_surrogate_error(post):
    """spot = 1: every point exact, each one compared with the network."""
    g, geo, model = post
    rho, z, pts = _points(geo, 1024, 17, d_min=5e-8, d_max=1e-6)
    tables = geo.bem_tables("cuda")
    bind = engine.SurrogateBinding(model, band=0.0, spot=1.0)
    E = engine.surrogate_field(tables, bind, pts).cpu().numpy()
    ref = engine.bem_field(tables, pts, form="mixed").cpu().numpy()
    np.testing.assert_allclose(E, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    n_sur, n_band, n_spot, err = bind.stats()
    assert (n_sur, n_band, n_spot) == (0, 0, len(pts))
    # the recorded maximum is the network's error against the exact field
    kr, kz = _rho_z(engine.surrogate_field(tables, engine.SurrogateBinding(model, 0.0, 0.0), pts).cpu().numpy(), pts)
    er, ez = _rho_z(E, pts)
    host = np.max(np.hypot(kr - er, kz - ez) / np.hypot(er, ez))
    assert abs(err - host) <= 1e-5 * host + 1e-6, (err, host)


def test_all_points_spot_checked_reproduce_exact_trace(post):
    """spot = 1 in the stage kernel: every point takes the exact (mixed)
    sum, so the trace to t_max lands where the mixed form's does.  (The two
    are separate kernel instantiations, which may contract float32
    multiply-adds differently; the controller resolves float32 noise at
    rtol 1e-8, so their step sequences may part, and the comparison is at
    t_max, to the mixed form's 1e-6.)"""
    g, geo, model = post
    tr_ref, b_ref = _complete(g, geo, "mixed")
    tr, b = _complete(g, geo, "surrogate", model, band=0.0, spot=1.0)
    n_sur, n_band, n_spot, err = tr.surrogate_stats()
    assert n_sur == 0 and n_spot > 0
    assert np.isfinite(err)
    np.testing.assert_array_equal(b.status.cpu().numpy(), b_ref.status.cpu().numpy())
    p_ref, p = b_ref.positions().cpu().numpy(), b.positions().cpu().numpy()
    np.testing.assert_allclose(p, p_ref, rtol=1e-6, atol=1e-6 * np.abs(p_ref).max())


def _complete(g, geo, form, model=None, band=5e-9, spot=0.0):
    G, E, _ = g["pos0"].shape
    tr = engine.Tracer(geo, form=form, z_max=float(g["z_max"]), surrogate=model, band=band, spot=spot)
    b = engine.GroupBatch(g["pos0"].reshape(-1, 3), g["vel0"].reshape(-1, 3), g["t_birth"].reshape(-1),
                          np.full(G * E, gu.Q_E), np.full(G * E, gu.M_E), [E] * G)
    tr.run(b, float(g["t_max"]), 1e-8, 1e-12, 1e-12, gu.CM, max_steps=200_000)
    torch.cuda.synchronize()
    return tr, b


def test_surrogate_points_drive_the_trace(post):
    """Both traces run to t_max.  The small fit moves the particles the right
    way; its endpoint error is a property of the fit (printed), the bound
    here only catches a broken path.  Ablation: the network replaces most of
    the ring evaluations per stage."""
    g, geo, model = post
    tr_ref, b_ref = _complete(g, geo, "mixed")
    tr, b = _complete(g, geo, "surrogate", model, band=5e-9)
    n_sur, n_band, n_spot, err = tr.surrogate_stats()
    assert n_sur > 0 and n_spot == 0
    p_ref, p = b_ref.positions().cpu().numpy(), b.positions().cpu().numpy()
    assert np.all(np.isfinite(p))
    disp = np.abs(p_ref - g["pos0"].reshape(-1, 3)).max()
    rel = np.abs(p - p_ref).max() / disp
    c_ref, c = tr_ref.counter_dict(), tr.counter_dict()
    per_stage = lambda c: (c["ring_far"] + c["ring_near"]) / max(1, c["stage_evals"])
    print(f"surrogate points {n_sur}, band points {n_band}; endpoint error / displacement {rel:.3e}; "
          f"attempts {c['attempts']} vs {c_ref['attempts']}; ring evals per stage {per_stage(c):.0f} vs {per_stage(c_ref):.0f}")
    assert rel < 0.5, rel
    assert per_stage(c) < 0.5 * per_stage(c_ref)


def test_learned_form_measured_against_chosen_form():
    """The learned form at its full specification (4 x 128 SiLU MLP, BF16;
    2M training points log-uniform 1 nm - 1 mm from the surface, labelled by
    the float64 BEM evaluator; Adam, lr 1e-3 cosine, 20k steps, batch 8192;
    exact BEM within 5 nm, 1 % spot checks) on the C1 tip, against the chosen
    form (float64, adaptive far rule, no network) and the float32 form
    (float32 + Kahan, adaptive far rule), all tracing 148 C4-sized groups
    (sizes logU[1, 128], seed 4) to t = 0.1 ps.  Measured:
    CUDA-event time to reach t_end, attempts, accepted particle-steps and the
    endpoint error against the plain float64 form.  Particle-steps per second
    alone would reward a form that takes more, smaller steps, so the verdict
    is on time to the same end time at <= 1e-6 endpoint error.

    What this measures (printed): the network replaces most ring
    evaluations, but its BF16 output is not smooth at the 1e-9 level the
    rtol = 1e-9 controller resolves, so the controller takes far more steps
    and the endpoints miss 1e-6 -- the learned form does not beat the chosen
    form.  This test asserts that finding; a network that changes it makes
    the test fail, and the chosen form should then be revisited."""
    from bem_b200 import geometry as bg, workloads as w
    g = load_golden("sigma_c1")
    geo = bg.PostTipBEMGeometry(-1e6, 50e-9, 5e-6, profile=g["profile"], sigma=g["sigma"])
    model = sg.train(geo, seed=4)  # the full specification (the defaults)
    d = w.tip_c4(geo.profile, geo.sigma, n_groups=148, seed=4)
    pos = np.stack([d["x"], d["y"], d["z"]], -1)
    vel = np.stack([d[k] for k in ("px", "py", "pz")], -1) * (gu.ophys.ELEMENTARY_CHARGE / gu.ophys.SPEED_OF_LIGHT
                                                              / gu.M_E)
    n = len(pos)
    t_end = 0.1e-12
    out = {}
    for name, form, rule, kw in (("plain", "fp64", "reference", {}), ("chosen", "fp64", "adaptive", {}),
                                 ("mixed", "mixed", "adaptive", {}),
                                 ("learned", "surrogate", "adaptive", dict(surrogate=model, band=5e-9, spot=0.01))):
        tr = engine.Tracer(geo, form=form, far_rule=rule, z_max=1e-3, **kw)
        b = engine.GroupBatch(pos, vel, d["t"], np.full(n, gu.Q_E), np.full(n, gu.M_E), d["group_sizes"])
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        tr.run(b, t_end, 1e-9, 1e-12, 1e-12, gu.CM, max_steps=2_000_000, attempt_chunk=2_000_000)
        e.record()
        e.synchronize()
        out[name] = dict(t=s.elapsed_time(e) * 1e-3, c=tr.counter_dict(), pos=b.positions().cpu().numpy(),
                         td=b.t_death.cpu().numpy())
    ref = out["plain"]
    alive = np.isinf(ref["td"])
    for name in ("chosen", "mixed", "learned"):
        o = out[name]
        ok = alive & np.isinf(o["td"])
        o["err"] = float((np.linalg.norm(o["pos"] - ref["pos"], axis=-1)[ok] /
                          np.linalg.norm(ref["pos"], axis=-1)[ok]).max())
        c = o["c"]
        o["per_stage"] = (c["ring_far"] + c["ring_near"]) / max(1, c["stage_evals"])
        print(f"{name}: {o['t']:.3f} s to t_end, {c['attempts']} attempts, {c['particle_steps']} particle-steps "
              f"({c['particle_steps'] / o['t']:.3e}/s), ring evals per stage {o['per_stage']:.0f}, "
              f"max endpoint error vs plain {o['err']:.2e}")
    C, L = out["chosen"], out["learned"]
    assert C["err"] <= 1e-6                         # the chosen form meets the bar
    assert L["per_stage"] < 0.5 * C["per_stage"]    # the network does replace most ring evaluations ...
    assert L["err"] > 1e-6 or L["t"] > C["t"]       # ... but does not beat the chosen form within 1e-6
