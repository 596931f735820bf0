"""GPU parity of the BEM image-charge force (spt_toroidal_q,
spt_image_assemble, spt_image_force) against fixtures produced by the
reference itself (tests/golden/make_golden.py: toroidal, image_tip,
image_well) and against the oracle.

Tolerances: Q 1e-13 relative (the downward recurrence starts fewer terms
above the last mode than the reference, both converged to rounding); dQ/dchi
1e-13 times the cancellation of its formula near chi = 1; operators 1e-13 of the largest entry (summation order);
forces 1e-11 of the group's largest force (rounding through the per-mode
inverse and the ~1000-node reconstruction)."""

import ctypes

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from bem_b200 import _lib  # noqa: E402
from bem_b200 import image_charge as bic  # noqa: E402
from oracle import image_charge as oic  # noqa: E402

DEV = "cuda"


def _t(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=DEV)


@pytest.mark.parametrize("n_max", [0, 1, 16, 24, 40])
def test_toroidal_q_matches_reference(n_max):
    g = load_golden("toroidal")
    chi = _t(g["chi"])
    n = chi.shape[0]
    q = torch.empty((n_max + 1, n), dtype=torch.float64, device=DEV)
    dq = torch.empty_like(q)
    rc = _lib.lib().spt_toroidal_q(_lib.ptr(chi), n, n_max, _lib.ptr(q), _lib.ptr(dq), None)
    _lib.check(rc, "spt_toroidal_q")
    torch.cuda.synchronize()
    k = min(n_max, g["q"].shape[0] - 1) + 1  # the fixture holds modes 0..24
    qr, dqr = g["q"][:k], g["dq"][:k]
    np.testing.assert_allclose(q.cpu().numpy()[:k], qr, rtol=1e-13, atol=0)
    # dQ_n = (n - 1/2)(chi Q_n - Q_{n-1}) / (chi^2 - 1) cancels near chi = 1: its rounding error is
    # that of Q times |chi Q_n| / |chi Q_n - Q_{n-1}|, the bound scaled here
    chi = np.maximum(g["chi"], np.nextafter(1.0, 2.0))
    cond = np.ones_like(qr)
    cond[1:] = np.abs(chi * qr[1:]) / np.maximum(np.abs(chi * qr[1:] - qr[:-1]), 1e-300)
    err = np.abs(dq.cpu().numpy()[:k] - dqr) / np.abs(dqr)
    assert (err <= 1e-13 * np.maximum(cond, 1.0)).all(), float((err / np.maximum(cond, 1.0)).max())


def test_toroidal_q_rejects_too_many_modes():
    rc = _lib.lib().spt_toroidal_q(None, 1, _lib.IMAGE_MAX_MODES + 1, None, None, None)
    assert rc == _lib.SPT_ERR_CAPACITY


@pytest.mark.parametrize("name,key", [("image_tip", "trunc"), ("image_tip", "doubled"), ("image_well", "")])
def test_mode_operators_match_reference(name, key):
    g = load_golden(name)
    pre = f"{key}_" if key else ""
    prof, ref = g[pre + "profile"], g[pre + "A"]
    sol = bic.ImageChargeSolution(prof, int(g[pre + "n_max"]), 0.0, 1.0, device=DEV)
    A = sol.A.cpu().numpy()
    for m in range(ref.shape[0]):
        np.testing.assert_allclose(A[m], ref[m], rtol=0, atol=1e-13 * np.abs(ref[m]).max(), err_msg=f"mode {m}")


def _device_force(sol, pos, q, active, geometry=None):
    G, E, _ = pos.shape
    off = _t(np.arange(G + 1) * E).to(torch.int64)
    act = torch.as_tensor(active.reshape(-1).astype(np.uint8), device=DEV)
    f = sol.force(_t(pos.reshape(-1, 3)), _t(q.reshape(-1)), act, off, E, geometry=geometry)
    torch.cuda.synchronize()
    return f.cpu().numpy().reshape(G, E, 3)


def _close(got, ref, tol=1e-11):
    for g in range(ref.shape[0]):
        scale = np.abs(ref[g]).max()
        np.testing.assert_allclose(got[g], ref[g], rtol=0, atol=tol * max(scale, 1e-300), err_msg=f"group {g}")


def _geometry(kind, g, R, z0, z_handoff, H=0.0):
    geo = _lib.SptGeometry()
    geo.kind = kind
    geo.has_image = 1
    geo.R, geo.H, geo.z0, geo.z_handoff = R, H, z0, z_handoff
    return geo


def test_solution_force_matches_reference():
    g = load_golden("image_tip")
    R = float(g["R"])
    for d_hi, key in ((0.5 * R, "trunc_solution_force"), (0.1 * R, "trunc_solution_force_nomirror")):
        sol = bic.ImageChargeSolution(g["trunc_profile"], int(g["trunc_n_max"]), 0.1 * R, d_hi, device=DEV)
        _close(_device_force(sol, g["pos"], g["q"], g["active"]), g[key])


@pytest.mark.parametrize("kind", ["trunc", "doubled"])
def test_tip_geometry_force_matches_reference(kind):
    g = load_golden("image_tip")
    R, z0 = float(g["R"]), float(g["z0"])
    sol = bic.ImageChargeSolution(g[f"{kind}_profile"], int(g[f"{kind}_n_max"]), 0.1 * R, 0.5 * R,
                                  mirror_symmetric=kind == "doubled", device=DEV)
    geo = _geometry(_lib.GEOM_TIP_BEM, g, R, z0, float(g[f"{kind}_z_handoff"]))
    _close(_device_force(sol, g["pos"], g["q"], g["active"], geo), g[f"{kind}_force"])


def test_well_geometry_force_matches_reference():
    g = load_golden("image_well")
    R, z0 = float(g["R"]), float(g["z0"])
    sol = bic.ImageChargeSolution(g["profile"], int(g["n_max"]), float(g["d_lo"]) * R, float(g["d_hi"]) * R,
                                  device=DEV)
    geo = _geometry(_lib.GEOM_WELL_BEM, g, R, z0, float(g["z_handoff"]), float(g["H"]))
    _close(_device_force(sol, g["pos"], g["q"], g["active"], geo), g["force"])


def test_blend_and_many_groups_match_oracle():
    """Points across the whole blend (BEM below z_handoff/2, plane image
    above z_handoff), uneven activity, 40 groups of 9 (more groups than a
    single CTA pass handles at once on a small grid is not needed: every CTA
    loops over groups) against the oracle's geometry-level force."""
    g = load_golden("image_tip")
    R, z0 = float(g["R"]), float(g["z0"])
    zh = 20.0 * R
    rng = np.random.default_rng(5)
    G, E = 40, 9
    th = rng.uniform(0, np.radians(70), (G, E))
    ph = rng.uniform(-np.pi, np.pi, (G, E))
    r = R + np.exp(rng.uniform(np.log(2e-9), np.log(1.5 * zh), (G, E)))
    pos = np.stack([r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), r * np.cos(th)], -1)
    q = np.full((G, E), -1.602176634e-19)
    active = rng.uniform(size=(G, E)) > 0.25
    ref_sol = oic.ImageSolution(g["trunc_profile"], 16, A=g["trunc_A"])
    ref = oic.geometry_image_force(ref_sol, pos, q, active, z0, R, z_handoff=zh)
    sol = bic.ImageChargeSolution(g["trunc_profile"], 16, 0.1 * R, 0.5 * R, device=DEV)
    got = _device_force(sol, pos, q, active, _geometry(_lib.GEOM_TIP_BEM, g, R, z0, zh))
    _close(got, ref)
    assert np.all(got[~active] == 0.0)


def test_rejects_bad_arguments():
    g = load_golden("image_tip")
    sol = bic.ImageChargeSolution(g["trunc_profile"], 16, 5e-9, 25e-9, device=DEV)
    x = _t(np.zeros(4))
    off = torch.tensor([0, 4], dtype=torch.int64, device=DEV)
    act = torch.ones(4, dtype=torch.uint8, device=DEV)
    L = _lib.lib()
    args = lambda n_e, geo: (_lib.ptr(x), _lib.ptr(x), _lib.ptr(x), _lib.ptr(x), _lib.ptr(act), _lib.ptr(off), 1,
                             n_e, ctypes.byref(sol.struct), geo, 8.98e9, 1e-12, _lib.ptr(x), _lib.ptr(x),
                             _lib.ptr(x), None)
    assert L.spt_image_force(*args(513, None)) == _lib.SPT_ERR_CAPACITY
    flat = _lib.SptGeometry()
    flat.kind = _lib.GEOM_FLAT
    flat.has_image = 1
    flat.z_handoff = 1e-6
    assert L.spt_image_force(*args(4, ctypes.byref(flat))) == _lib.SPT_ERR_ARG


def _image_spec(g, kind):
    s = dict(kind=kind, E_gun=float(g["E_gun"]), R=float(g["R"]), profile=g["profile"], sigma=g["sigma"],
             n_subdiv=int(g["n_subdiv"]), z_handoff=float(g["z_handoff"]), z0=float(g["z0"]),
             image_profile=g["image_profile"], image_n_max=int(g["image_n_max"]),
             image_d_lo=float(g["image_d_lo"]), image_d_hi=float(g["image_d_hi"]),
             image_mirror_symmetric=bool(g["image_mirror_symmetric"]))
    if kind == "tip_bem":
        s["kill_z_below"] = 0.0
    else:
        s.update(H=float(g["H"]), bottom_fillet_radius=float(g["bottom_fillet_radius"]),
                 rim_fillet_radius=float(g["rim_fillet_radius"]), kill_z_below=None)
    return s


@pytest.mark.parametrize("name,kind", [("trace_image_tip_trunc", "tip_bem"), ("trace_image_tip_doubled", "tip_bem"),
                                       ("trace_image_well", "well_bem")])
def test_trace_with_image_force_matches_reference(name, kind):
    """The persistent trace with the BEM image force in every stage (plain
    form) against the reference's integrate on its HemisphericalTipBEMGeometry
    / CylindricalWellBEMGeometry built with z0: the same attempt and
    acceptance sequence, endpoints within 1e-10 of the reference's."""
    import gpu_util as gu
    g = load_golden(name)
    spec = _image_spec(g, kind)
    o = gu.device_trace(spec, g["pos0"], g["vel0"], g["t_birth"], float(g["t_max"]), float(g["rtol"]),
                        float(g["atol"]), float(g["z_max"]))
    np.testing.assert_array_equal(o["n_acc"] + o["n_rej"], g["attempts"])
    np.testing.assert_array_equal(o["n_acc"], g["n_acc"])
    np.testing.assert_array_equal(np.isfinite(o["t_death"]), np.isfinite(g["t_death"]))
    alive = np.isinf(g["t_death"])
    rel = lambda a, b: np.linalg.norm(a - b, axis=-1) / np.linalg.norm(b, axis=-1)
    if alive.any():
        assert rel(o["pos"][alive], g["pos"][alive]).max() < 1e-10
        assert rel(o["vel"][alive], g["vel"][alive]).max() < 1e-10
    # killed at z_max or on the conductor: the same step of a step grid that moves by ~1e-8 (the error
    # norm's cancellation turns ulp-level slope differences into ~1e-7 of the next step size)
    dead = ~alive
    np.testing.assert_allclose(o["t_death"][dead], g["t_death"][dead], rtol=1e-7)


def test_accel_with_image_force_matches_oracle():
    """spt_accel (one stage) on the image-tip fixture's geometry at scattered
    live/dead states against the oracle's stage acceleration (1e-11)."""
    import gpu_util as gu
    from bem_b200 import engine
    from oracle import geometry as ogeo
    g = load_golden("trace_image_tip_trunc")
    spec = _image_spec(g, "tip_bem")
    rng = np.random.default_rng(8)
    G, E = 5, 6
    R = spec["R"]
    th = rng.uniform(0, 1.2, (G, E))
    ph = rng.uniform(-np.pi, np.pi, (G, E))
    r = R + np.exp(rng.uniform(np.log(1e-9), np.log(2e-6), (G, E)))
    pos = np.stack([r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), r * np.cos(th)], -1)
    live = rng.uniform(size=(G, E)) > 0.2
    q = np.full((G, E), gu.Q_E)
    m = np.full((G, E), gu.M_E)
    ref = ogeo.make_accel(spec, q, m, gu.CM, 1e-12)(pos, np.zeros_like(pos), live, np.arange(G))
    got = engine.accel(gu.device_geometry(spec), pos.reshape(-1, 3), live.reshape(-1), q.reshape(-1), m.reshape(-1),
                       [E] * G, gu.CM, 1e-12)
    got = got.cpu().numpy().reshape(G, E, 3)
    for k in range(G):
        np.testing.assert_allclose(got[k], ref[k], rtol=0, atol=1e-11 * np.abs(ref[k]).max())
