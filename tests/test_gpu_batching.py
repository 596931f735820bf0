"""Batching form: compaction of retired groups on the device, the trace
captured as a CUDA graph, uneven group sizes in one launch.  Groups are
independent, so every variant must give the plain run's results bit for bit."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from bem_b200 import _lib, engine, workloads  # noqa: E402

import gpu_util as gu  # noqa: E402

FIELDS = ("x", "y", "z", "vx", "vy", "vz", "t_death", "t", "h", "status", "n_accepted", "n_rejected")


def test_compact_groups_matches_numpy():
    rng = np.random.default_rng(3)
    for n in (1, 7, 1024, 1025, 5000):
        status = torch.as_tensor(rng.integers(0, 3, n).astype(np.int32), device="cuda")
        order = torch.as_tensor(rng.permutation(n).astype(np.int32), device="cuda")
        out = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
        for base in (order, None):
            _lib.check(_lib.lib().spt_compact_groups(None if base is None else base.data_ptr(), n,
                                                     status.data_ptr(), out.data_ptr(), cnt.data_ptr(), None), "compact")
            torch.cuda.synchronize()
            o = order.cpu().numpy() if base is not None else np.arange(n, dtype=np.int32)
            want = o[status.cpu().numpy()[o] < _lib.GROUP_DONE]
            assert int(cnt.item()) == len(want)
            np.testing.assert_array_equal(out.cpu().numpy()[: len(want)], want)


def _uneven(seed=5, n_groups=40):
    """Flat-cathode groups of log-uniform sizes 1..48 (C3-like unevenness)."""
    rng = np.random.default_rng(seed)
    sizes = np.round(np.exp(rng.uniform(0, np.log(48), n_groups))).astype(int)
    n = int(sizes.sum())
    x, y = rng.normal(0, 10e-6, n), rng.normal(0, 10e-6, n)
    s = np.sqrt(workloads.ELECTRON_MC2_EV * 0.1)
    p = np.stack([rng.normal(0, s, n), rng.normal(0, s, n), np.abs(rng.normal(0, s, n))], -1)
    vel = p * gu.ophys.ELEMENTARY_CHARGE / gu.ophys.SPEED_OF_LIGHT / gu.M_E
    pos = np.stack([x, y, np.zeros(n)], -1)
    tb = rng.uniform(0, 1e-12, n)
    return pos, vel, tb, sizes


def _trace(run_kw, form="fp64"):
    pos, vel, tb, sizes = _uneven()
    geo = gu.device_geometry(dict(kind="flat", E_gun=-1e7, z0=3e-9, kill_z_below=0.0))
    tr = engine.Tracer(geo, form=form, z_max=2e-5)
    n = len(pos)
    b = engine.GroupBatch(pos, vel, tb, np.full(n, gu.Q_E), np.full(n, gu.M_E), sizes)
    tr.run(b, 3e-12, 1e-8, 1e-12, 1e-12, gu.CM, attempt_chunk=64, **run_kw)
    torch.cuda.synchronize()
    return {f: getattr(b, f).cpu().numpy() for f in FIELDS}, tr.counter_dict()


@pytest.mark.parametrize("kw", [dict(compact=True), dict(graph=True, graph_launches=3)])
def test_compacted_and_graph_runs_match_plain_run(kw):
    ref, c_ref = _trace({})
    got, c = _trace(kw)
    assert np.all(ref["status"] == _lib.GROUP_DONE)
    for f in FIELDS:
        np.testing.assert_array_equal(got[f], ref[f], err_msg=f)
    assert c["accepted"] == c_ref["accepted"] and c["attempts"] == c_ref["attempts"]


def test_graph_run_respects_max_steps():
    pos, vel, tb, sizes = _uneven()
    geo = gu.device_geometry(dict(kind="flat", E_gun=-1e7, z0=3e-9, kill_z_below=0.0))
    tr = engine.Tracer(geo, z_max=2e-5)
    n = len(pos)
    b = engine.GroupBatch(pos, vel, tb, np.full(n, gu.Q_E), np.full(n, gu.M_E), sizes)
    with pytest.raises(RuntimeError, match="did not converge within 200 steps"):
        tr.run(b, 3e-12, 1e-8, 1e-12, 1e-12, gu.CM, max_steps=200, attempt_chunk=64, graph=True, graph_launches=2)
    att = (b.n_accepted + b.n_rejected).cpu().numpy()
    assert att.max() <= 200


def test_autotune_picks_a_guarded_config_and_keeps_results():
    """The tuner times its candidates on the post-tip fixture, applies the
    winner, and the tuned trace agrees with the default one (round size and
    rule thresholds change rounding only: within the mixed form's 1e-6)."""
    from conftest import load_golden
    from bem_b200 import autotune

    g = load_golden("trace_post")
    spec = dict(kind="post_bem", E_gun=float(g["E_gun"]), R=float(g["R"]), L=float(g["L"]), z0=float(g["z0"]),
                profile=g["profile"], sigma=g["sigma"], n_subdiv=int(g["n_subdiv"]), z_handoff=float(g["z_handoff"]),
                kill_z_below=0.0)
    geo = gu.device_geometry(spec)
    G, E, _ = g["pos0"].shape
    arrays = (g["pos0"].reshape(-1, 3), g["vel0"].reshape(-1, 3), g["t_birth"].reshape(-1),
              np.full(G * E, gu.Q_E), np.full(G * E, gu.M_E), [E] * G)
    args = (float(g["t_max"]), 1e-8, 1e-12, 1e-12, gu.CM)

    def trace(tuned):
        tr = engine.Tracer(geo, form="mixed", z_max=float(g["z_max"]), far_rule="adaptive")
        b = engine.GroupBatch(*arrays)
        res = None
        if tuned:
            res = autotune.tune(tr, *arrays, *args, warm=8, attempts=4, tune_ratios=True)
            autotune.apply(res, tr, b)
        tr.launch(b, tr.params(*args, 30))
        torch.cuda.synchronize()
        return b.positions().cpu().numpy(), res

    p_ref, _ = trace(False)
    p, res = trace(True)
    assert res["round_points"] in autotune.ROUND_POINTS and res["order"] in autotune.ORDERS
    assert tuple(res["ratios"]) in autotune.RATIOS
    assert any(isinstance(v, float) for v in res["timings"].values())
    # mixed form: a different round size reorders float32 sums, so the two
    # traces agree to the form's 1e-6 bar, not bit for bit
    assert np.abs(p - p_ref).max() <= 1e-6 * np.abs(p_ref).max()


def test_group_born_after_t_max_is_done_untouched():
    """A group whose every member is born after t_max has nothing to
    integrate: it finishes with no attempt and its particles unchanged,
    while the other groups of the launch run normally."""
    pos, vel, tb, sizes = _uneven(n_groups=4)
    tb = tb.copy()
    first = slice(0, int(sizes[0]))
    tb[first] = 5e-12  # the first group: born after t_max below
    geo = gu.device_geometry(dict(kind="flat", E_gun=-1e7, z0=3e-9, kill_z_below=0.0))
    tr = engine.Tracer(geo, z_max=2e-5)
    n = len(pos)
    b = engine.GroupBatch(pos, vel, tb, np.full(n, gu.Q_E), np.full(n, gu.M_E), sizes)
    tr.run(b, 3e-12, 1e-8, 1e-12, 1e-12, gu.CM)
    assert np.all(b.status.cpu().numpy() == _lib.GROUP_DONE)
    assert int(b.n_accepted[0].item() + b.n_rejected[0].item()) == 0
    np.testing.assert_array_equal(b.positions().cpu().numpy()[first], pos[first])
    assert int(b.n_accepted[1:].sum().item()) > 0
