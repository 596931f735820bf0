"""Pin the image-charge oracle (oracle/image_charge.py) and the image
profile builders (bem_b200/image_charge.py) against fixtures produced by the
reference itself (tests/golden/make_golden.py: toroidal, image_tip,
image_well), and against the physics the reference's own tests use: the
classical image of a point charge in a grounded plane, and the joint
solve's group isolation.  CPU only."""

import numpy as np
import pytest

from oracle import image_charge as oic
from oracle import physics as ophys

from conftest import load_golden
from bem_b200 import image_charge as bic


def test_toroidal_q_matches_reference():
    g = load_golden("toroidal")
    q, dq = oic.toroidal_q(g["chi"], 24)
    np.testing.assert_allclose(q, g["q"], rtol=4e-15, atol=0)
    np.testing.assert_allclose(dq, g["dq"], rtol=1e-14, atol=0)


def test_mode_kernels_match_reference():
    g = load_golden("toroidal")
    ph, dr, dz = oic.ring_field_modes(g["rho"], g["z"], g["a"], g["za"], 16)
    for got, ref in ((ph, g["phi_m"]), (dr, g["dphi_drho"]), (dz, g["dphi_dz"])):
        scale = np.abs(ref).max(axis=0, keepdims=True)  # per pair: the largest mode
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-14 * scale.max())
        assert (np.abs(got - ref) <= 1e-13 * scale).all()
    gm = oic.point_charge_potential_modes(g["rho"], g["z"], g["a"], g["za"], 16)
    np.testing.assert_allclose(gm, g["g"], rtol=1e-14, atol=0)


@pytest.mark.parametrize("kind", ["trunc", "doubled"])
def test_tip_image_profiles_match_reference(kind):
    g = load_golden("image_tip")
    R, z0 = float(g["R"]), float(g["z0"])
    ml = (R - z0) * np.pi / 2 / 29  # HemisphericalTipBEMGeometry's default image_max_length
    p = bic.tip_image_profile(R, z0, 5 * R, ml) if kind == "trunc" else bic.tip_image_doubled_profile(R, z0, ml)
    np.testing.assert_array_equal(p, g[f"{kind}_profile"])


def test_well_image_profile_matches_reference():
    g = load_golden("image_well")
    R, H, z0 = float(g["R"]), float(g["H"]), float(g["z0"])
    room = min(0.5 * z0, 0.2 * (H - z0))  # CylindricalWellBEMGeometry's default corner roundings with z0
    p = bic.well_image_profile(R, H, z0, 5 * max(R, H), min(R, H) / 14, room, z0 + room)
    np.testing.assert_array_equal(p, g["profile"])


def test_mode_operators_match_reference():
    g = load_golden("image_tip")
    A = oic.assemble_mode_operators(g["trunc_profile"], int(g["trunc_n_max"]))
    ref = g["trunc_A"]
    # the sums differ from the reference's recursive order only in rounding
    np.testing.assert_allclose(A, ref, rtol=0, atol=1e-14 * np.abs(ref).max())


def _solution(g, kind):
    return oic.ImageSolution(g[f"{kind}_profile"], int(g[f"{kind}_n_max"]), A=g[f"{kind}_A"])


def test_image_force_matches_reference():
    g = load_golden("image_tip")
    sol = _solution(g, "trunc")
    R = float(g["R"])
    for d_hi, key in ((0.5 * R, "trunc_solution_force"), (0.1 * R, "trunc_solution_force_nomirror")):
        f = sol.image_force(g["pos"], g["q"], g["active"], 0.1 * R, d_hi)
        np.testing.assert_allclose(f, g[key], rtol=0, atol=1e-13 * np.abs(g[key]).max())


@pytest.mark.parametrize("kind", ["trunc", "doubled"])
def test_geometry_image_force_matches_reference(kind):
    g = load_golden("image_tip")
    sol = _solution(g, kind)
    f = oic.geometry_image_force(sol, g["pos"], g["q"], g["active"], float(g["z0"]), float(g["R"]),
                                 z_handoff=float(g[f"{kind}_z_handoff"]), mirror_symmetric=kind == "doubled")
    ref = g[f"{kind}_force"]
    np.testing.assert_allclose(f, ref, rtol=0, atol=1e-13 * np.abs(ref).max())


def test_well_geometry_image_force_matches_reference():
    g = load_golden("image_well")
    sol = oic.ImageSolution(g["profile"], int(g["n_max"]), A=g["A"])
    f = oic.geometry_image_force(sol, g["pos"], g["q"], g["active"], float(g["z0"]), float(g["R"]),
                                 float(g["d_lo"]), float(g["d_hi"]), z_handoff=float(g["z_handoff"]))
    np.testing.assert_allclose(f, g["force"], rtol=0, atol=1e-13 * np.abs(g["force"]).max())


def test_groups_never_interact():
    """The fixture's group 2 sits where group 0 does, with other charges:
    each group's force comes from its own joint solve only
    (test_image_force_groups_never_interact of the reference)."""
    g = load_golden("image_tip")
    sol = _solution(g, "trunc")
    R = float(g["R"])
    f = sol.image_force(g["pos"], g["q"], g["active"], 0.1 * R, 0.5 * R)
    alone = sol.image_force(g["pos"][:1], g["q"][:1], g["active"][:1], 0.1 * R, 0.5 * R)
    np.testing.assert_array_equal(f[0], alone[0])


def test_flat_plane_mirror_is_the_classical_image():
    """A grounded plane (a flat profile out to 40 x the standoff) and a
    charge whose local mirror has full weight: the residual solve is ~0 and
    the force is the classical image force q^2 / (16 pi eps0 d^2) toward the
    plane, to the truncation of the finite disk."""
    rs = [0.0]
    r = 1e-9
    while r < 400e-9:
        rs.append(r)
        r *= 1.15
    rs.append(400e-9)
    prof = np.column_stack([np.array(rs)[::-1], np.zeros(len(rs))])  # outer edge first: normal points to +z
    sol = oic.ImageSolution(prof, 4)
    d = 10e-9
    q = -ophys.ELEMENTARY_CHARGE
    pos = np.array([[[3e-9, 2e-9, d]]])
    f = sol.image_force(pos, np.array([[q]]), np.array([[True]]), 1e-6, 2e-6)[0, 0]
    classical = q * q / (16.0 * np.pi * ophys.VACUUM_PERMITTIVITY * d * d)
    assert abs(f[2] + classical) < 2e-3 * classical
    assert np.hypot(f[0], f[1]) < 1e-3 * classical


def test_oracle_trace_with_image_force_matches_reference():
    """The oracle's integrator with the BEM image force of a
    HemisphericalTipBEMGeometry built with z0 against the reference's own
    trace: the same attempt and acceptance counts, endpoints to 1e-10."""
    from oracle import geometry as ogeo
    from oracle import rk45 as ork
    g = load_golden("trace_image_tip_trunc")
    spec = dict(kind="tip_bem", E_gun=float(g["E_gun"]), R=float(g["R"]), profile=g["profile"], sigma=g["sigma"],
                n_subdiv=int(g["n_subdiv"]), z_handoff=float(g["z_handoff"]), kill_z_below=0.0, z0=float(g["z0"]),
                image_profile=g["image_profile"], image_n_max=int(g["image_n_max"]),
                image_d_lo=float(g["image_d_lo"]), image_d_hi=float(g["image_d_hi"]), image_mirror_symmetric=False)
    G, E, _ = g["pos0"].shape
    m = ophys.ev_to_kg(ophys.ELECTRON_MASS_EV)
    q = -ophys.ELEMENTARY_CHARGE
    acc = ogeo.make_accel(spec, np.full((G, E), q), np.full((G, E), m), q / m, 1e-12)
    pos, vel, td, t, h, log = ork.integrate(acc, g["pos0"], g["vel0"], g["t_birth"], float(g["t_max"]),
                                            float(g["rtol"]), float(g["atol"]),
                                            kill=ogeo.make_kill(spec, float(g["z_max"])))
    attempts = np.array([len(log[k][0]) for k in range(G)])
    np.testing.assert_array_equal(attempts, g["attempts"])
    alive = np.isinf(g["t_death"])
    rel = np.linalg.norm(pos - g["pos"], axis=-1)[alive] / np.linalg.norm(g["pos"], axis=-1)[alive]
    assert rel.max() < 1e-10
