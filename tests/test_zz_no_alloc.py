"""spt_trace_noalloc -- the trace entry point for callers that cannot
allocate device memory (a binding with no device allocator of its own, or
code that must not trigger the device-wide synchronisation a cudaMalloc can
cause) -- gives the same results as spt_trace, call after call.

Collected last on purpose (test_zz_*): if it fails, a run that stops at the
first failure has already run every other test.  It passes alone in a fresh
process as well as after the rest of the suite.
"""

import ctypes

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from bem_b200 import _lib, engine  # noqa: E402

import gpu_util as gu  # noqa: E402

FIELDS = ("x", "y", "z", "vx", "vy", "vz", "t_death", "t", "h", "status", "n_accepted", "n_rejected")


def _noalloc(tracer, batch, params):
    stream = torch.cuda.current_stream()
    bem = ctypes.byref(tracer.tables.struct) if tracer.tables is not None else None
    rc = _lib.lib().spt_trace_noalloc(ctypes.byref(batch.struct()), ctypes.byref(params), ctypes.byref(tracer.geom),
                                      bem, ctypes.c_void_p(stream.cuda_stream))
    _lib.check(rc, "spt_trace_noalloc")


def _compare(a, b):
    torch.cuda.synchronize()
    for f in FIELDS:
        x = getattr(a, f).cpu().numpy()
        y = getattr(b, f).cpu().numpy()
        if x.dtype.kind == "f":
            scale = np.abs(x[np.isfinite(x)]).max() if np.isfinite(x).any() else 1.0
            np.testing.assert_allclose(y, x, rtol=1e-10, atol=1e-10 * scale, err_msg=f)
        else:
            np.testing.assert_array_equal(y, x, err_msg=f)


def _two_calls(spec, pos, vel, tb, sizes, t_max, rtol, z_max, attempts):
    geo = gu.device_geometry(spec)
    tracer = engine.Tracer(geo, z_max=z_max)
    n = len(pos)
    mk = lambda: engine.GroupBatch(pos, vel, tb, np.full(n, gu.Q_E), np.full(n, gu.M_E), sizes)
    ref, test = mk(), mk()
    params = tracer.params(t_max, rtol, 1e-12, 1e-12, gu.CM, attempts)
    for _ in range(2):
        tracer.launch(ref, params)
        _noalloc(tracer, test, params)
        _compare(ref, test)
    assert int(test.n_accepted.sum() + test.n_rejected.sum()) > 0


def test_noalloc_matches_trace_bem_two_calls():
    g = load_golden("trace_post")
    spec = dict(kind="post_bem", E_gun=float(g["E_gun"]), R=float(g["R"]), L=float(g["L"]), z0=float(g["z0"]),
                profile=g["profile"], sigma=g["sigma"], n_subdiv=int(g["n_subdiv"]), z_handoff=float(g["z_handoff"]),
                kill_z_below=0.0)
    G, E, _ = g["pos0"].shape
    _two_calls(spec, g["pos0"].reshape(-1, 3), g["vel0"].reshape(-1, 3), g["t_birth"].reshape(-1), [E] * G,
               float(g["t_max"]), 1e-8, float(g["z_max"]), 12)


def test_noalloc_matches_trace_large_groups_two_calls():
    """Groups above 256 particles use slope buffers in the fixed scratch."""
    from bem_b200 import workloads as w
    d = w.flat_c0(n_groups=3, n_emit=300, seed=9)
    pos = np.stack([d["x"], d["y"], d["z"]], -1)
    vel = np.stack([d["px"], d["py"], d["pz"]], -1) * gu.ophys.ELEMENTARY_CHARGE / gu.ophys.SPEED_OF_LIGHT / gu.M_E
    spec = dict(kind="flat", E_gun=-1e7, z0=3e-9, kill_z_below=0.0)
    _two_calls(spec, pos, vel, d["t"], [300] * 3, w.default_t_max(-1e7, 1e-3, 1e-12), 1e-8, 1e-3, 6)


def test_noalloc_more_groups_than_scratch_slots_two_calls():
    """12 groups of 1024 particles: the scratch holds 9 slope buffers of
    that size, so the persistent grid is capped at 9 CTAs and the work
    queue hands the other 3 groups to CTAs that finished (and 40 groups of
    300 against 32 buffers)."""
    from bem_b200 import workloads as w
    spec = dict(kind="flat", E_gun=-1e7, z0=3e-9, kill_z_below=0.0)
    for n_groups, E, attempts in ((12, 1024, 3), (40, 300, 4)):
        d = w.flat_c0(n_groups=n_groups, n_emit=E, seed=10, t_spread=2e-15)
        pos = np.stack([d["x"], d["y"], d["z"]], -1)
        vel = np.stack([d["px"], d["py"], d["pz"]], -1) * gu.ophys.ELEMENTARY_CHARGE / gu.ophys.SPEED_OF_LIGHT / gu.M_E
        _two_calls(spec, pos, vel, d["t"], [E] * n_groups, w.default_t_max(-1e7, 1e-3, 1e-12), 1e-8, 1e-3, attempts)


def test_noalloc_rejects_the_learned_form():
    s = _lib.SptState()
    s.n_groups = 1
    s.max_group_size = 8
    p = _lib.SptTraceParams()
    p.form = _lib.FORM_SURROGATE
    g = _lib.SptGeometry()
    g.kind = _lib.GEOM_POST_BEM
    rc = _lib.lib().spt_trace_noalloc(ctypes.byref(s), ctypes.byref(p), ctypes.byref(g), None, None)
    assert rc == _lib.SPT_ERR_ARG
    assert "learned form is not offered" in _lib.last_error()


def test_noalloc_rejects_groups_above_limit():
    s = _lib.SptState()
    s.n_groups = 1
    s.max_group_size = 2000
    p = _lib.SptTraceParams()
    p.form = 0
    g = _lib.SptGeometry()
    g.kind = _lib.GEOM_FLAT
    rc = _lib.lib().spt_trace_noalloc(ctypes.byref(s), ctypes.byref(p), ctypes.byref(g), None, None)
    assert rc == _lib.SPT_ERR_CAPACITY
    assert "max_group_size" in _lib.last_error()
