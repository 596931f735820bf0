"""Generate the golden fixtures by running the REFERENCE implementation.

Run in the development container, where the reference package
(``specific_particle_tracer`` from AdamCBartnik/BEM) is importable from its
source tree:

    python tests/golden/make_golden.py --ref <reference source tree> [names...]

(or SPT_REFERENCE=<tree> instead of --ref)

It puts ``tests/golden/_stub`` (a minimal ParticleGroup stand-in, since
openpmd-beamphysics is not installed) and the reference tree on sys.path,
calls the reference's own functions on seeded inputs, and writes one
compressed ``.npz`` per fixture next to this script.  The GPU box never
runs this; tests only read the ``.npz`` files.
"""

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _setup(ref):
    sys.path.insert(0, os.path.join(HERE, "_stub"))
    sys.path.insert(0, ref)
    sys.path.insert(0, REPO)


def _save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({os.path.getsize(path)} bytes)")


def gen_ellip():
    from specific_particle_tracer.bem._elliptic import ellip_ke_complement
    p = np.concatenate([np.logspace(-300, -1, 400), np.linspace(0.1, 1.0, 200), [1.0, 0.5, 1e-3, 1e-3 * (1 + 1e-15)]])
    K, E = ellip_ke_complement(p, np)
    _save("ellip", p=p, K=K, E=E)


def gen_ring():
    from specific_particle_tracer.bem.axisymmetric import ring_field
    rng = np.random.default_rng(11)
    n = 600
    a = rng.uniform(1e-9, 1e-7, n)
    rho = a * np.exp(rng.uniform(-3, 3, n))
    z = a * rng.normal(0, 1.0, n)
    # near the ring itself, near the axis, exactly on the axis
    rho[:100] = a[:100] * (1 + rng.normal(0, 1e-3, 100))
    z[:100] = a[:100] * rng.normal(0, 1e-3, 100)
    rho[100:150] = a[100:150] * 1e-6
    rho[150:170] = 0.0
    er, ez = ring_field(rho, z, a, np)
    _save("ring", rho=rho, z=z, a=a, er=er, ez=ez)


def _states(rng, G, E, scale, zoff=0.0, live_frac=0.8):
    pos = rng.normal(0, scale, (G, E, 3))
    pos[..., 2] = np.abs(pos[..., 2]) + zoff
    vel = rng.normal(0, 1e5, (G, E, 3))
    live = rng.uniform(0, 1, (G, E)) < live_frac
    return pos, vel, live


def gen_accel():
    from specific_particle_tracer import geometry as g
    from specific_particle_tracer.constants import ELEMENTARY_CHARGE, ev_to_kg
    rng = np.random.default_rng(12)
    m = ev_to_kg(510998.95069)
    out = {}
    for name, geo, scale, zoff in [
        ("flat", g.FlatCathode(-1e7, z0=3e-9), 5e-8, 0.0),
        ("flat_noimg", g.FlatCathode(-1e7, z0=None), 5e-8, 0.0),
        ("tip", g.HemisphericalTip(-1e8, 50e-9, z0=3e-9), 3e-8, 50e-9),
    ]:
        G, E = 3, 7
        pos, vel, live = _states(rng, G, E, scale, zoff)
        charge = np.full((G, E), -ELEMENTARY_CHARGE)
        mass = np.full((G, E), m)
        acc = g.make_accel_fn(charge, mass, -ELEMENTARY_CHARGE / m, geo, 1e-12)(pos, vel, live, np.arange(G))
        kill = g.make_kill_fn(geo, 1e-6)(pos)
        out.update({f"{name}_pos": pos, f"{name}_vel": vel, f"{name}_live": live, f"{name}_acc": acc,
                    f"{name}_kill": kill})
    _save("accel", **out)


def _surface_points(rng, profile, n, out_scale):
    """Points on, just off, and away from the profile's surface of revolution."""
    prof = np.asarray(profile)
    seg = rng.integers(0, len(prof) - 1, n)
    t = rng.uniform(0, 1, n)
    p = prof[seg] + t[:, None] * (prof[seg + 1] - prof[seg])
    tan = prof[seg + 1] - prof[seg]
    nrm = np.stack([-tan[:, 1], tan[:, 0]], -1)
    nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
    k = np.arange(n) % 4
    off = np.where(k == 0, 0.0, np.where(k == 1, 1e-3, np.where(k == 2, 0.3, 3.0))) * out_scale
    rz = p + off[:, None] * nrm
    ph = rng.uniform(0, 2 * np.pi, n)
    pts = np.stack([rz[:, 0] * np.cos(ph), rz[:, 0] * np.sin(ph), rz[:, 1]], -1)
    return pts


def gen_bem_sphere():
    from specific_particle_tracer.bem.geometry import HemisphericalTipBEMGeometry
    rng = np.random.default_rng(13)
    R = 50e-9
    geo = HemisphericalTipBEMGeometry(-1e8, R, field_max_length=R * np.pi / 40)
    sol = geo.field_solver.solution
    pts = _surface_points(rng, sol.profile, 64, R / 40)
    pts = np.concatenate([pts, [[0, 0, R], [0, 0, 1.5 * R], [1e-12, 0, 2 * R], [3 * R, 0, 5 * R],
                                [0, 0, 15 * R], [2 * R, 1 * R, 12 * R], [0, 0, 25 * R]]])
    pts = pts[pts[:, 2] >= 0]
    e_pert = sol.field(pts)
    e_geo = geo.field(pts[None])[0]
    kill = geo.kill_mask(pts)
    _save("bem_sphere", profile=sol.profile, sigma=sol.sigma, R=R, E_gun=-1e8, z_handoff=geo.z_handoff,
          n_subdiv=geo.n_subdiv, points=pts, e_pert=e_pert, e_geo=e_geo, kill=kill)


def gen_bem_well():
    from specific_particle_tracer.bem.geometry import CylindricalWellBEMGeometry
    rng = np.random.default_rng(14)
    R, H = 2e-6, 1e-6
    geo = CylindricalWellBEMGeometry(-2.5e6, R, H, field_max_length=H / 6)
    sol = geo.field_solver.solution
    pts = _surface_points(rng, sol.profile[: len(sol.profile) // 2], 48, H / 6)
    pts = np.concatenate([pts, [[0, 0, -H], [0, 0, -0.5 * H], [0.5 * R, 0, 0.0], [3 * R, 0, 5 * H], [0, 0, 30 * H]]])
    e_pert = sol.field(pts)
    e_geo = geo.field(pts[None])[0]
    kill = geo.kill_mask(pts)
    _save("bem_well", profile=sol.profile, sigma=sol.sigma, R=R, H=H, E_gun=-2.5e6, z_handoff=geo.z_handoff,
          n_subdiv=geo.n_subdiv, points=pts, e_pert=e_pert, e_geo=e_geo, kill=kill)


class _PostTip:
    """Hemisphere on a post, composed only of reference functions: BEM field
    of the mirror-doubled capsule (AxisymmetricBEMSolution), blend with the
    flat fallback (bem.geometry._blend_with_flat_fallback), 3-image force of
    forces.hemispherical_tip_image_force in the apex frame."""

    def __init__(self, E_gun, R, L, profile, z0, z_handoff, n_subdiv=8, sigma=None):
        from specific_particle_tracer.bem.axisymmetric import AxisymmetricBEMSolution
        from specific_particle_tracer.fields import GunField
        self.E_gun, self.R, self.L, self.z0, self.z_handoff, self.n_subdiv = E_gun, R, L, z0, z_handoff, n_subdiv
        if sigma is None:
            self.solution = AxisymmetricBEMSolution.solve(profile, dirichlet_fn=lambda rho, z: E_gun * z)
        else:
            # a density the reference solved earlier (sigma_c1.npz: 221 s to solve)
            self.solution = AxisymmetricBEMSolution(np.asarray(profile, dtype=float), np.asarray(sigma, dtype=float))
        self.gun = GunField(E_gun)

    def inside(self, pos):
        rk = self.R * (1.0 - 1e-6)
        x, y, z = pos[..., 0], pos[..., 1], pos[..., 2]
        return ((x * x + y * y <= rk * rk) & (z <= self.L)) | (x * x + y * y + (z - self.L) ** 2 <= rk * rk)

    def field(self, pos):
        from specific_particle_tracer.bem.geometry import _blend_with_flat_fallback
        ok = (~self.inside(pos)) & (pos[..., 2] >= 0.0)
        uni = np.zeros_like(pos)
        uni[..., 2] = self.E_gun
        near = np.where(ok[..., None], uni + self.solution.field(pos, n_subdiv=self.n_subdiv), 0.0)
        return _blend_with_flat_fallback(near, self.gun.evaluate(pos), pos[..., 2], 0.5 * self.z_handoff,
                                         self.z_handoff, np)

    def image_force(self, pos, charge, active, soft):
        from specific_particle_tracer.forces import hemispherical_tip_image_force
        sh = pos.copy()
        sh[..., 2] -= self.L
        return hemispherical_tip_image_force(sh, charge, active, self.R - self.z0, soft,
                                             plane_z0=self.L + self.z0, xp=np)

    def kill_mask(self, pos):
        return self.inside(pos) | (pos[..., 2] <= 0.0)


def _post_case():
    from bem_b200.mesh import capsule_profile
    R, L = 50e-9, 400e-9
    prof = capsule_profile(R, L, 10, 20)
    return _PostTip(-1e7, R, L, prof, 3e-9, 20 * (L + R))


def gen_bem_post():
    rng = np.random.default_rng(15)
    geo = _post_case()
    sol = geo.solution
    pts = _surface_points(rng, sol.profile[: len(sol.profile) // 2], 48, 5e-9)
    pts = pts[pts[:, 2] >= 0]
    e_pert = sol.field(pts)
    e_geo = geo.field(pts[None])[0]
    _save("bem_post", profile=sol.profile, sigma=sol.sigma, R=geo.R, L=geo.L, E_gun=geo.E_gun, z0=geo.z0,
          z_handoff=geo.z_handoff, n_subdiv=8, points=pts, e_pert=e_pert, e_geo=e_geo, kill=geo.kill_mask(pts))


def _trace(geo, pos0, vel0, tb, t_max, rtol, atol, z_max, soft=1e-12):
    from specific_particle_tracer import batched_rk45, geometry as g
    from specific_particle_tracer.constants import ELEMENTARY_CHARGE, ev_to_kg
    G, E, _ = pos0.shape
    m = ev_to_kg(510998.95069)
    charge = np.full((G, E), -ELEMENTARY_CHARGE)
    mass = np.full((G, E), m)
    acc = g.make_accel_fn(charge, mass, -ELEMENTARY_CHARGE / m, geo, soft)
    calls = np.zeros(G, dtype=np.int64)

    def counted(pos, vel, active, gidx):
        calls[gidx] += 1
        return acc(pos, vel, active, gidx)

    steps = [[] for _ in range(G)]

    def on_step(gi, t_old, p_old, v_old, t_new, p_new, v_new):
        for k, gg in enumerate(gi):
            steps[gg].append(t_new[k])

    kill = g.make_kill_fn(geo, z_max)
    t0 = time.time()
    pos, vel = batched_rk45.integrate(counted, pos0, vel0, tb, t_max, rtol, atol, on_step=on_step, kill_fn=kill)
    print(f"  trace {G}x{E}: {time.time() - t0:.1f}s, attempts {calls // 7}")
    n_acc = np.array([len(s) for s in steps])
    t_acc = np.zeros((G, n_acc.max()))
    for k, s in enumerate(steps):
        t_acc[k, :len(s)] = s
    return dict(pos0=pos0, vel0=vel0, t_birth=tb, t_max=t_max, rtol=rtol, atol=atol, z_max=z_max,
                pos=pos, vel=vel, attempts=calls // 7, n_acc=n_acc, t_acc=t_acc)


def _grouped(d, G, E, mass):
    from specific_particle_tracer.constants import ev_c_to_si_momentum
    sl = slice(0, G * E)
    pos = np.stack([d["x"][sl], d["y"][sl], d["z"][sl]], -1).reshape(G, E, 3)
    vel = np.stack([ev_c_to_si_momentum(d[k][sl]) / mass for k in ("px", "py", "pz")], -1).reshape(G, E, 3)
    return pos, vel, d["t"][sl].reshape(G, E)


def gen_trace_flat(n_groups=2):
    from specific_particle_tracer import geometry as g
    from specific_particle_tracer.constants import ev_to_kg
    from bem_b200 import workloads as w
    d = w.flat_c0()
    pos, vel, tb = _grouped(d, n_groups, 64, ev_to_kg(510998.95069))
    t_max = w.default_t_max(-1e7, 1e-3, 1e-12)
    res = _trace(g.FlatCathode(-1e7, z0=3e-9, kill_z_below=0.0), pos, vel, tb, t_max, 1e-8, 1e-12, 1e-3)
    _save("trace_flat" if n_groups == 2 else "trace_flat_c0", **res)


def gen_trace_tip():
    from specific_particle_tracer import geometry as g
    from specific_particle_tracer.constants import ev_to_kg
    from bem_b200 import workloads as w
    R = 50e-9
    d = w.tip_c2(n_groups=2, n_emit=12, R=R, L=0.0, seed=21)
    pos, vel, tb = _grouped(d, 2, 12, ev_to_kg(510998.95069))
    res = _trace(g.HemisphericalTip(-1e8, R, z0=3e-9), pos, vel, tb, 2e-12, 1e-8, 1e-12, 2e-6)
    _save("trace_tip", **res)


def gen_trace_bem():
    from specific_particle_tracer.bem.geometry import HemisphericalTipBEMGeometry
    from specific_particle_tracer.constants import ev_to_kg
    from bem_b200 import workloads as w
    R = 50e-9
    geo = HemisphericalTipBEMGeometry(-1e8, R, field_max_length=R * np.pi / 30)
    d = w.tip_c2(n_groups=1, n_emit=4, R=R, L=0.0, seed=22, t_spread=0.2e-12)
    pos, vel, tb = _grouped(d, 1, 4, ev_to_kg(510998.95069))
    res = _trace(geo, pos, vel, tb, 0.4e-12, 1e-8, 1e-12, 3e-7)
    sol = geo.field_solver.solution
    _save("trace_tip_bem", profile=sol.profile, sigma=sol.sigma, R=R, E_gun=-1e8, z_handoff=geo.z_handoff,
          n_subdiv=8, **res)


def gen_trace_post():
    from specific_particle_tracer.constants import ev_to_kg
    from bem_b200 import workloads as w
    geo = _post_case()
    d = w.tip_c2(n_groups=1, n_emit=4, R=geo.R, L=geo.L, seed=23, t_spread=0.2e-12)
    pos, vel, tb = _grouped(d, 1, 4, ev_to_kg(510998.95069))
    res = _trace(geo, pos, vel, tb, 0.4e-12, 1e-8, 1e-12, 2e-6)
    _save("trace_post", profile=geo.solution.profile, sigma=geo.solution.sigma, R=geo.R, L=geo.L,
          E_gun=geo.E_gun, z0=geo.z0, z_handoff=geo.z_handoff, n_subdiv=8, **res)


def gen_trace_well():
    from specific_particle_tracer.bem.geometry import CylindricalWellBEMGeometry
    from specific_particle_tracer.constants import ev_to_kg
    from bem_b200 import workloads as w
    R, H = 2e-6, 1e-6
    geo = CylindricalWellBEMGeometry(-2.5e7, R, H, field_max_length=H / 6)
    d = w.well_c3(n_groups=40, seed=24, R=R, H=H, t_spread=0.5e-12)
    n = 3
    pos, vel, tb = _grouped(d, 1, n, ev_to_kg(510998.95069))
    res = _trace(geo, pos, vel, tb, 1.0e-12, 1e-8, 1e-12, 5e-6)
    sol = geo.field_solver.solution
    _save("trace_well", profile=sol.profile, sigma=sol.sigma, R=R, H=H, E_gun=-2.5e7, z_handoff=geo.z_handoff,
          n_subdiv=8, **res)


def gen_trace_image():
    """Traces with the BEM image-charge force: HemisphericalTipBEMGeometry
    (R = 50 nm, z0 = 3 nm; the truncated-plane image surface and the
    mirror-doubled one) and CylindricalWellBEMGeometry (R = 200 nm,
    H = 100 nm, z0 = 3 nm), 2 groups of 4 electrons each, emitted 1 nm off
    the real surface, through the reference's integrate to a short t_max."""
    from specific_particle_tracer.bem.geometry import CylindricalWellBEMGeometry, HemisphericalTipBEMGeometry
    from specific_particle_tracer.constants import ev_to_kg
    from bem_b200 import workloads as w
    m = ev_to_kg(510998.95069)
    R, z0 = 50e-9, 3e-9
    for tag, sym in (("trunc", False), ("doubled", True)):
        geo = HemisphericalTipBEMGeometry(-1e8, R, field_max_length=R * np.pi / 30, z0=z0, image_mirror_symmetric=sym)
        d = w.tip_c2(n_groups=2, n_emit=4, R=R, L=0.0, seed=25, t_spread=0.1e-12)
        pos, vel, tb = _grouped(d, 2, 4, m)
        pos = pos * (1.0 + 1e-9 / R)  # 1 nm off the sphere along its normal
        res = _trace_groups(geo, pos, vel, tb, 0.25e-12, 1e-8, 1e-12, 3e-7, procs=2)
        sol, img = geo.field_solver.solution, geo.image_solution
        _save(f"trace_image_tip_{tag}", profile=sol.profile, sigma=sol.sigma, R=R, E_gun=-1e8, z0=z0,
              z_handoff=geo.z_handoff, n_subdiv=8, image_profile=img.profile, image_n_max=geo.image_n_max, image_d_lo=geo.image_d_lo, image_d_hi=geo.image_d_hi,
              image_mirror_symmetric=sym, **res)
    R, H = 200e-9, 100e-9
    geo = CylindricalWellBEMGeometry(-1e8, R, H, field_max_length=H / 8, z0=z0)
    d = w.well_c3(n_groups=8, seed=26, R=R, H=H, t_spread=0.1e-12)
    pos, vel, tb = _grouped(d, 2, 4, m)
    pos = pos + np.array([0.0, 0.0, 1e-9])
    res = _trace_groups(geo, pos, vel, tb, 0.25e-12, 1e-8, 1e-12, 3e-6, procs=2)
    sol, img = geo.field_solver.solution, geo.image_solution
    _save("trace_image_well", profile=sol.profile, sigma=sol.sigma, R=R, H=H, E_gun=-1e8, z0=z0,
          z_handoff=geo.z_handoff, n_subdiv=8, bottom_fillet_radius=geo.bottom_fillet_radius,
          rim_fillet_radius=geo.rim_fillet_radius, image_profile=img.profile, image_n_max=geo.image_n_max, image_d_lo=geo.image_d_lo, image_d_hi=geo.image_d_hi,
          image_mirror_symmetric=False, **res)


def gen_tracker():
    """Tracker-level outputs (screens, t_out) for a small flat case."""
    from specific_particle_tracer import SpecificParticleTracer, geometry as g
    from beamphysics import ParticleGroup
    from bem_b200 import workloads as w
    d = w.flat_c0(n_groups=3, n_emit=6, seed=31)
    pg = ParticleGroup(data={k: v for k, v in d.items() if k != "group_sizes"})
    tr = SpecificParticleTracer(pg, 6, g.FlatCathode(-1e7), screens=[1e-7, 5e-6], t_out=[0.5e-12, 1.5e-12],
                                rtol=1e-8, z_max=2e-5)
    scr, trj = tr.run()
    out = dict(t_max=tr.t_max)
    for k, s in enumerate(scr):
        for key in ("x", "y", "z", "px", "py", "pz", "t", "id"):
            out[f"screen{k}_{key}"] = np.asarray(getattr(s, key))
    for k, s in enumerate(trj):
        for key in ("x", "y", "z", "px", "py", "pz", "t", "id"):
            out[f"traj{k}_{key}"] = np.asarray(getattr(s, key))
    _save("tracker_flat", **out)


def gen_sigma_c1():
    """Reference solve of the 2000-panel hemisphere-on-post capsule
    (R = 50 nm, L = 5 um, 100 cap + 900 wall segments per half), Ez = -1e6."""
    from specific_particle_tracer.bem.axisymmetric import AxisymmetricBEMSolution
    from bem_b200.mesh import capsule_profile
    prof = capsule_profile(50e-9, 5e-6, 100, 900)
    sol = AxisymmetricBEMSolution.solve(prof, dirichlet_fn=lambda rho, z: -1e6 * z)
    _save("sigma_c1", profile=prof, sigma=sol.sigma, E_gun=-1e6)


# ---------------------------------------------------------------------------
# Fixtures at the benchmark configurations (C1-C4 scale: 2000- and
# ~3000-panel BEM solutions, groups of 32 and 1024 particles, uneven sizes).
# Each group is traced by its own call of the reference's integrate, in a
# pool of processes: groups never interact in the reference (one group per
# call gives the numbers a batched call gives), and the per-point BEM sums
# make a 2000-panel trace cost ~10 ms per particle-stage on one core.

def _one_group(job):
    """Reference integrate on one group, for at most max_attempts attempts
    (None: to t_max).  The state after the last accepted step, the death
    times, the accepted step end times and the attempt count are rebuilt
    from on_step and the counted accel calls, exactly as integrate applies
    them (kill after an accepted step, only for particles active at its
    start; batched_rk45.py:260-293)."""
    from specific_particle_tracer import batched_rk45, geometry as g
    from specific_particle_tracer.constants import ELEMENTARY_CHARGE, ev_to_kg
    pos0, vel0, tb, t_max, rtol, atol, z_max, max_attempts = job
    geo = _POOL_GEO  # set before the pool forks (geometry objects hold modules, which do not pickle)
    E = pos0.shape[1]
    m = ev_to_kg(510998.95069)
    acc = g.make_accel_fn(np.full((1, E), -ELEMENTARY_CHARGE), np.full((1, E), m), -ELEMENTARY_CHARGE / m, geo, 1e-12)
    calls = [0]

    def counted(pos, vel, active, gidx):
        calls[0] += 1
        return acc(pos, vel, active, gidx)

    kill = g.make_kill_fn(geo, z_max)
    st = dict(pos=pos0.copy(), vel=vel0.copy(), t=float(tb.min()), td=np.full((1, E), np.inf), t_acc=[])

    def on_step(gi, t_old, p_old, v_old, t_new, p_new, v_new):
        was = (t_old[:, None] >= tb) & (t_old[:, None] < st["td"])
        newly = was & kill(p_new)
        st["td"] = np.where(newly, t_new[:, None], st["td"])
        st["pos"], st["vel"], st["t"] = p_new.copy(), v_new.copy(), float(t_new[0])
        st["t_acc"].append(float(t_new[0]))

    t0 = time.time()
    done = True
    try:
        batched_rk45.integrate(counted, pos0, vel0, tb, t_max, rtol, atol, on_step=on_step, kill_fn=kill,
                               max_steps=max_attempts if max_attempts else 10_000_000)
    except RuntimeError:
        done = False  # the attempt budget ran out: the state after max_attempts attempts
    return dict(pos=st["pos"][0], vel=st["vel"][0], t=st["t"], t_death=st["td"][0], attempts=calls[0] // 7,
                n_acc=len(st["t_acc"]), t_acc=np.asarray(st["t_acc"]), done=done, seconds=time.time() - t0)


_POOL_GEO = None


def _trace_groups(geo, pos0, vel0, tb, t_max, rtol, atol, z_max, max_attempts=None, procs=8):
    import multiprocessing as mp
    global _POOL_GEO
    _POOL_GEO = geo
    G = pos0.shape[0]
    jobs = [(pos0[k:k + 1], vel0[k:k + 1], tb[k:k + 1], t_max, rtol, atol, z_max, max_attempts) for k in range(G)]
    with mp.get_context("fork").Pool(min(procs, G)) as pool:
        res = pool.map(_one_group, jobs)
    n_acc = np.array([r["n_acc"] for r in res])
    t_acc = np.zeros((G, max(1, n_acc.max())))
    for k, r in enumerate(res):
        t_acc[k, :len(r["t_acc"])] = r["t_acc"]
    print(f"  {G} groups x {pos0.shape[1]}: attempts {[r['attempts'] for r in res]}, "
          f"{max(r['seconds'] for r in res):.0f} s")
    return dict(pos0=pos0, vel0=vel0, t_birth=tb, t_max=t_max, rtol=rtol, atol=atol, z_max=z_max,
                max_attempts=-1 if max_attempts is None else max_attempts,
                pos=np.stack([r["pos"] for r in res]), vel=np.stack([r["vel"] for r in res]),
                t=np.array([r["t"] for r in res]), t_death=np.stack([r["t_death"] for r in res]),
                attempts=np.array([r["attempts"] for r in res]), n_acc=n_acc, t_acc=t_acc,
                done=np.array([r["done"] for r in res]))


def _c1_geometry():
    """The C1 tip (R = 50 nm on a 5 um post, 2000-panel capsule, E = -1e6
    V/m, z0 = 3 nm, z_handoff = 20 (L + R)) with the density the reference
    solved (sigma_c1.npz)."""
    g = np.load(os.path.join(HERE, "sigma_c1.npz"))
    R, L = 50e-9, 5e-6
    return _PostTip(-1e6, R, L, g["profile"], 3e-9, 20 * (L + R), sigma=g["sigma"]), g


def _vel(d, mass):
    from specific_particle_tracer.constants import ev_c_to_si_momentum
    return np.stack([ev_c_to_si_momentum(d[k]) / mass for k in ("px", "py", "pz")], -1)


def _bench_groups(d, first, n, E):
    from specific_particle_tracer.constants import ev_to_kg
    sl = slice(first * E, (first + n) * E)
    pos = np.stack([d["x"][sl], d["y"][sl], d["z"][sl]], -1).reshape(n, E, 3)
    vel = _vel({k: d[k][sl] for k in ("px", "py", "pz")}, ev_to_kg(510998.95069)).reshape(n, E, 3)
    return pos, vel, d["t"][sl].reshape(n, E)


def _post_fields(geo, g):
    return dict(profile=g["profile"], sigma=g["sigma"], R=geo.R, L=geo.L, E_gun=geo.E_gun, z0=geo.z0,
                z_handoff=geo.z_handoff, n_subdiv=8)


def gen_trace_c1():
    """C1 exactly: the first 4 groups x 32 of the C1 sampler (seed 1, drawn
    at the full 4096 x 32 size), traced from emission to t = 20 ps."""
    from bem_b200 import workloads as w
    geo, g = _c1_geometry()
    d = w.tip_c1(g["profile"], g["sigma"], seed=1)
    pos, vel, tb = _bench_groups(d, 0, 4, 32)
    res = _trace_groups(geo, pos, vel, tb, 20e-12, 1e-9, 1e-12, 1e-3)
    _save("trace_c1", **_post_fields(geo, g), **res)


def gen_trace_c2():
    """C2 scale: one group of 1024 from the C2 sampler (seed 2) on the C1
    tip, every member born at t = 0 (so all 1024 interact from the first
    stage), traced to t = 2e-18 s (with 1024 electrons 1 nm apart the
    reference's steps stay near 5e-19 s, and its field of 1024 points takes
    ~12 s a stage, so a longer trace takes it hours).  Traced to t_max, not cut
    after a number of attempts: both runs end at the same time, so the
    endpoints do not carry the step sizes' last digits (a budget-cut run's
    end time does).  The sites are lifted 1 nm off the apex
    along its normal: a point on the surface itself sits ~1e-13 m from the
    chords of the profile, where the near-segment quadrature depends on that
    distance to ~1e-8 relative through the rounding of 5 um coordinates --
    a property of the point, not of either implementation."""
    from bem_b200 import workloads as w
    geo, g = _c1_geometry()
    d = w.tip_c2(n_groups=1, seed=2)
    d["t"] = np.zeros_like(d["t"])
    pos, vel, tb = _bench_groups(d, 0, 1, 1024)
    apex = np.array([0.0, 0.0, geo.L])
    nrm = (pos - apex) / np.linalg.norm(pos - apex, axis=-1, keepdims=True)
    pos = pos + 1e-9 * nrm
    res = _trace_groups(geo, pos, vel, tb, 2e-18, 1e-9, 1e-12, 1e-3)
    _save("trace_c2", **_post_fields(geo, g), **res)


def _lift_cap(pos, L, dz=1e-9):
    """Emission sites on the apex sphere moved dz along its normal (a point on
    the surface itself sits ~1e-13 m from the chords of the profile, where
    the near-segment quadrature depends on that distance to ~1e-8 relative
    through the rounding of 5 um coordinates -- a property of the point, not
    of either implementation; it dominates a comparison cut after a few
    attempts, while the particles are still at the surface)."""
    apex = np.array([0.0, 0.0, L])
    nrm = (pos - apex) / np.linalg.norm(pos - apex, axis=-1, keepdims=True)
    return pos + dz * nrm


C4_BINS = ((1, 8, None), (2, 4, None), (7, 2, None), (128, 1, 150))
C3_BINS = ((1, 8, None), (2, 4, None), (129, 1, 60), (256, 1, 60))


def gen_trace_c4(bins=C4_BINS):
    """C4 size bins on the C1 tip (C4 sampler, seed 4, fixed sizes): 8 groups
    of 1, 4 of 2, 2 of 7 traced to t = 20 ps, one of 128 for 150 attempts
    (its sites lifted 1 nm off the surface, see _lift_cap).  One fixture per
    bin (the reference needs one size per call)."""
    from bem_b200 import workloads as w
    geo, g = _c1_geometry()
    for E, n, att in bins:
        d = w.tip_c4(g["profile"], g["sigma"], seed=4, sizes=[E] * n)
        pos, vel, tb = _bench_groups(d, 0, n, E)
        if att:
            pos = _lift_cap(pos, geo.L)
        res = _trace_groups(geo, pos, vel, tb, 20e-12, 1e-9, 1e-12, 1e-3, max_attempts=att)
        _save(f"trace_c4_s{E}", **_post_fields(geo, g), **res)


def gen_trace_c3(bins=C3_BINS):
    """C3 size bins on the reference's own ~3000-segment well (R = 2 um,
    H = 1 um, E = -2.5e6 V/m, max_length H/980): the C3 sampler (seed 3,
    fixed sizes), 8 groups of 1 and 4 of 2 traced to t = 30 ps (with two
    more reference runs at vel0 x (1 -+ 1e-15) that record its own
    sensitivity), one group each of 129 and 256 for 60 attempts; every site
    lifted 1 nm off the floor (for the reason of _lift_cap: on the floor itself a point sits on
    the on-surface offset threshold, which moves the early step sizes and
    with them the death time of a particle that returns to the floor)."""
    from specific_particle_tracer.bem.geometry import CylindricalWellBEMGeometry
    from bem_b200 import workloads as w
    R, H = 2e-6, 1e-6
    t0 = time.time()
    geo = CylindricalWellBEMGeometry(-2.5e6, R, H, field_max_length=H / 980)
    sol = geo.field_solver.solution
    print(f"  well solve ({len(sol.profile) - 1} segments): {time.time() - t0:.0f} s")
    _save("sigma_c3", profile=sol.profile, sigma=sol.sigma, E_gun=-2.5e6, R=R, H=H, z_handoff=geo.z_handoff)
    for E, n, att in bins:
        d = w.well_c3(seed=3, sizes=[E] * n)
        pos, vel, tb = _bench_groups(d, 0, n, E)
        pos = pos + np.array([0.0, 0.0, 1e-9])
        res = _trace_groups(geo, pos, vel, tb, 30e-12, 1e-9, 1e-12, 2e-3, max_attempts=att)
        if not att:
            # the reference's own sensitivity: the same groups with vel0 scaled by 1 -+ 1e-15 (a group whose
            # attempt sequence changes under it returns to the floor, where the decisions are ill-conditioned)
            pert = [_trace_groups(geo, pos, vel * (1.0 + e), tb, 30e-12, 1e-9, 1e-12, 2e-3) for e in (1e-15, -1e-15)]
            res.update(attempts_pert=np.stack([r["attempts"] for r in pert]),
                       t_death_pert=np.stack([r["t_death"] for r in pert]),
                       pos_pert=np.stack([r["pos"] for r in pert]), vel_pert=np.stack([r["vel"] for r in pert]))
        _save(f"trace_c3_s{E}", profile=sol.profile, sigma=sol.sigma, R=R, H=H, E_gun=-2.5e6,
              z_handoff=geo.z_handoff, n_subdiv=8, **res)


def gen_toroidal():
    """Q_{m-1/2}, dQ/dchi (both recurrence branches, near coincidence to far)
    and the mode kernels on random (field, source) pairs."""
    from specific_particle_tracer.bem.ring_modes import point_charge_potential_modes, ring_field_modes
    from specific_particle_tracer.bem.toroidal import toroidal_Q
    rng = np.random.default_rng(21)
    chi = np.concatenate([1.0 + np.logspace(-14, 3, 300), [1.0, np.nextafter(1.0, 2.0), 1.0 + 1e-300]])
    q, dq = toroidal_Q(chi, 24)
    n = 400
    a = rng.uniform(1e-9, 1e-7, n)
    za = rng.normal(0.0, 5e-8, n)
    rho = a * np.exp(rng.uniform(-4.0, 3.0, n))
    z = za + a * rng.normal(0.0, 1.0, n) * np.exp(rng.uniform(-6.0, 1.0, n))
    ph, dr, dz = ring_field_modes(rho, z, a, za, 16)
    g = point_charge_potential_modes(rho, z, a, za, 16)
    _save("toroidal", chi=chi, q=q, dq=dq, rho=rho, z=z, a=a, za=za, phi_m=ph, dphi_drho=dr, dphi_dz=dz, g=g)


def _image_states(rng, G, E, R, lift_lo, lift_hi, theta_max):
    """Points above the real hemisphere-on-plane surface: lifted off the cap
    by lift in [lift_lo, lift_hi] at polar angles below theta_max, random
    azimuths; a fifth of them inactive."""
    th = rng.uniform(0.0, theta_max, (G, E))
    ph = rng.uniform(-np.pi, np.pi, (G, E))
    r = R + rng.uniform(lift_lo, lift_hi, (G, E))
    pos = np.stack([r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), r * np.cos(th)], -1)
    active = rng.uniform(0.0, 1.0, (G, E)) > 0.2
    q = np.full((G, E), -1.602176634e-19) * rng.uniform(0.5, 2.0, (G, E))
    return pos, q, active


def gen_image_tip():
    """The BEM image-charge force on the hemisphere-on-plane tip (R = 50 nm,
    z0 = 3 nm): the truncated-plane image profile (operators, per-call
    ImageChargeBEMSolution.image_force) and the geometry-level force of
    HemisphericalTipBEMGeometry(z0=3 nm) in both image modes."""
    from specific_particle_tracer.bem.geometry import HemisphericalTipBEMGeometry
    R, z0 = 50e-9, 3e-9
    rng = np.random.default_rng(22)
    out = {}
    pos, q, active = _image_states(rng, 3, 5, R, 1e-9, 4e-8, np.radians(60.0))
    pos[2, :, :] = pos[0, :, :]  # group 2 = group 0 with other charges: groups are independent
    out.update(pos=pos, q=q, active=active, R=R, z0=z0, d_lo=0.1, d_hi=0.5)
    for tag, sym in (("trunc", False), ("doubled", True)):
        geo = HemisphericalTipBEMGeometry(-1e8, R, z0=z0, image_mirror_symmetric=sym)
        sol = geo.image_solution
        out[f"{tag}_profile"] = sol.profile
        out[f"{tag}_A"] = sol.A
        out[f"{tag}_n_max"] = sol.n_max
        out[f"{tag}_z_handoff"] = geo.z_handoff
        out[f"{tag}_force"] = geo.image_force(pos, q, active, 1e-12)
        if not sym:
            out["trunc_solution_force"] = sol.image_force(pos, q, active, 0.1 * R, 0.5 * R, n_max=sol.n_max)
            out["trunc_solution_force_nomirror"] = sol.image_force(pos, q, active, 0.1 * R, 0.1 * R,
                                                                   n_max=sol.n_max)
    _save("image_tip", **out)


def gen_image_well():
    """CylindricalWellBEMGeometry(z0=3 nm) on a small well (R = 200 nm,
    H = 100 nm): its image profile's operators and the geometry-level image
    force at points inside and above the recess."""
    from specific_particle_tracer.bem.geometry import CylindricalWellBEMGeometry
    R, H, z0 = 200e-9, 100e-9, 3e-9
    rng = np.random.default_rng(23)
    geo = CylindricalWellBEMGeometry(-1e7, R, H, z0=z0)
    sol = geo.image_solution
    G, E = 3, 4
    rho = R * np.sqrt(rng.uniform(0.0, 0.8, (G, E)))
    ph = rng.uniform(-np.pi, np.pi, (G, E))
    z = rng.uniform(-H + 5e-9, 60e-9, (G, E))
    pos = np.stack([rho * np.cos(ph), rho * np.sin(ph), z], -1)
    active = rng.uniform(0.0, 1.0, (G, E)) > 0.2
    q = np.full((G, E), -1.602176634e-19)
    force = geo.image_force(pos, q, active, 1e-12)
    _save("image_well", profile=sol.profile, A=sol.A, n_max=sol.n_max, z_handoff=geo.z_handoff, R=R, H=H, z0=z0,
          d_lo=geo.image_d_lo, d_hi=geo.image_d_hi, pos=pos, q=q, active=active, force=force)


GENERATORS = dict(sigma_c1=gen_sigma_c1, toroidal=gen_toroidal, image_tip=gen_image_tip, image_well=gen_image_well, ellip=gen_ellip, ring=gen_ring, accel=gen_accel, bem_sphere=gen_bem_sphere,
                  bem_well=gen_bem_well, bem_post=gen_bem_post, trace_flat=gen_trace_flat,
                  trace_tip=gen_trace_tip, trace_tip_bem=gen_trace_bem, trace_post=gen_trace_post,
                  trace_well=gen_trace_well, tracker=gen_tracker,
                  trace_flat_c0=lambda: gen_trace_flat(16), trace_c1=gen_trace_c1, trace_c2=gen_trace_c2,
                  trace_c3=gen_trace_c3, trace_c4=gen_trace_c4,
                  trace_c3_budget=lambda: gen_trace_c3(C3_BINS[2:]), trace_c4_budget=lambda: gen_trace_c4(C4_BINS[3:]),
                  trace_c3_small=lambda: gen_trace_c3(C3_BINS[:2]), trace_image=gen_trace_image)

# generated only when named (minutes to an hour of CPU each)
ON_REQUEST = ("trace_flat_c0", "sigma_c1", "trace_c1", "trace_c2", "trace_c3", "trace_c4", "trace_c3_budget",
              "trace_c4_budget", "trace_c3_small", "trace_image")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("SPT_REFERENCE"),
                    help="source tree of the reference project (or set SPT_REFERENCE)")
    ap.add_argument("names", nargs="*")
    a = ap.parse_args()
    if not a.ref:
        ap.error("give the reference source tree with --ref or SPT_REFERENCE")
    _setup(a.ref)
    for name in a.names or [k for k in GENERATORS if k not in ON_REQUEST]:
        t0 = time.time()
        GENERATORS[name]()
        print(f"{name}: {time.time() - t0:.1f}s")


if __name__ == "__main__":
    main()
