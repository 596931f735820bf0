"""Pin the CPU oracle against fixtures produced by the reference itself
(tests/golden/make_golden.py).  CPU only."""

import numpy as np
import pytest

from oracle import bem as obem
from oracle import geometry as ogeo
from oracle import physics as ophys
from oracle import rk45 as ork

from conftest import load_golden


def test_elliptic_matches_reference():
    g = load_golden("ellip")
    K, E = obem.ellip_k_e_complement(g["p"])
    np.testing.assert_array_equal(K, g["K"])
    np.testing.assert_array_equal(E, g["E"])


def test_ring_field_matches_reference():
    g = load_golden("ring")
    er, ez = obem.ring_field(g["rho"], g["z"], g["a"])
    np.testing.assert_allclose(er, g["er"], rtol=1e-15, atol=0)
    np.testing.assert_allclose(ez, g["ez"], rtol=1e-15, atol=0)


@pytest.mark.parametrize("name,spec", [
    ("flat", dict(kind="flat", E_gun=-1e7, z0=3e-9, kill_z_below=0.0)),
    ("flat_noimg", dict(kind="flat", E_gun=-1e7, z0=None, kill_z_below=0.0)),
    ("tip", dict(kind="tip", E_gun=-1e8, R=50e-9, z0=3e-9, kill_z_below=0.0)),
])
def test_accel_matches_reference(name, spec):
    g = load_golden("accel")
    pos, vel, live = g[f"{name}_pos"], g[f"{name}_vel"], g[f"{name}_live"]
    G, E, _ = pos.shape
    m = ophys.ev_to_kg(ophys.ELECTRON_MASS_EV)
    q = np.full((G, E), -ophys.ELEMENTARY_CHARGE)
    acc = ogeo.make_accel(spec, q, np.full((G, E), m), -ophys.ELEMENTARY_CHARGE / m, 1e-12)(pos, vel, live, np.arange(G))
    np.testing.assert_allclose(acc, g[f"{name}_acc"], rtol=1e-14, atol=0)
    np.testing.assert_array_equal(ogeo.kill_mask(spec, pos, 1e-6), g[f"{name}_kill"])


def _bem_spec(g, kind):
    s = dict(kind=kind, E_gun=float(g["E_gun"]), R=float(g["R"]), profile=g["profile"], sigma=g["sigma"],
             n_subdiv=int(g["n_subdiv"]), z_handoff=float(g["z_handoff"]), kill_z_below=0.0)
    if kind == "well_bem":
        s["H"] = float(g["H"])
    if kind == "post_bem":
        s["L"] = float(g["L"])
        s["z0"] = float(g["z0"])
    return s


@pytest.mark.parametrize("fixture,kind", [("bem_sphere", "tip_bem"), ("bem_well", "well_bem"),
                                          ("bem_post", "post_bem")])
def test_bem_field_matches_reference(fixture, kind):
    g = load_golden(fixture)
    e = obem.field(g["points"], g["profile"], g["sigma"], int(g["n_subdiv"]))
    scale = np.max(np.abs(g["e_pert"]))
    np.testing.assert_allclose(e, g["e_pert"], rtol=1e-11, atol=1e-13 * scale)
    spec = _bem_spec(g, kind)
    eg = ogeo.field(spec, g["points"])
    np.testing.assert_allclose(eg, g["e_geo"], rtol=1e-11, atol=1e-13 * np.max(np.abs(g["e_geo"])))
    np.testing.assert_array_equal(ogeo.kill_mask(spec, g["points"]), g["kill"])


def _trace_spec(name, g):
    if name == "trace_flat" or name == "trace_flat_c0":
        return dict(kind="flat", E_gun=-1e7, z0=3e-9, kill_z_below=0.0)
    if name == "trace_tip":
        return dict(kind="tip", E_gun=-1e8, R=50e-9, z0=3e-9, kill_z_below=0.0)
    if name == "trace_tip_bem":
        return _bem_spec(g, "tip_bem")
    if name == "trace_well":
        return _bem_spec(g, "well_bem")
    if name == "trace_post":
        return _bem_spec(g, "post_bem")
    raise KeyError(name)


def run_oracle_trace(name, g):
    spec = _trace_spec(name, g)
    pos0 = g["pos0"]
    G, E, _ = pos0.shape
    m = ophys.ev_to_kg(ophys.ELECTRON_MASS_EV)
    q = np.full((G, E), -ophys.ELEMENTARY_CHARGE)
    acc = ogeo.make_accel(spec, q, np.full((G, E), m), -ophys.ELEMENTARY_CHARGE / m, 1e-12)
    z_max = float(g["z_max"])
    return ork.integrate(acc, pos0, g["vel0"], g["t_birth"], float(g["t_max"]), float(g["rtol"]), float(g["atol"]),
                         kill=ogeo.make_kill(spec, z_max))


# Endpoint tolerance per fixture.  trace_tip_bem ends with every particle
# killed at z_max; its frozen positions depend on the step grid, and the
# oracle itself moves them by 1.4e-7 (relative) when vel0 is scaled by
# (1 + 1e-15).  The oracle's per-call accelerations agree with the
# reference to 2.3e-16 along that whole trace, so the 1.3e-8 endpoint gap
# is this sensitivity, not an algorithmic difference.
TRACE_RTOL = dict(trace_flat=1e-12, trace_tip=1e-12, trace_tip_bem=1e-6, trace_post=1e-12, trace_well=1e-12)


@pytest.mark.parametrize("name", sorted(TRACE_RTOL))
def test_trace_matches_reference(name):
    g = load_golden(name)
    pos, vel, td, t, h, log = run_oracle_trace(name, g)
    attempts = np.array([len(l[0]) for l in log])
    n_acc = np.array([int(np.sum(l[2])) for l in log])
    np.testing.assert_array_equal(attempts, g["attempts"])
    np.testing.assert_array_equal(n_acc, g["n_acc"])
    rt = TRACE_RTOL[name]
    np.testing.assert_allclose(pos, g["pos"], rtol=rt, atol=rt * np.max(np.abs(g["pos"])))
    np.testing.assert_allclose(vel, g["vel"], rtol=rt, atol=rt * np.max(np.abs(g["vel"])))
