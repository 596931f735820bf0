"""Seeded synthetic emission workloads (the five benchmark configurations).

No public dataset exists for this tracer; these samplers stand in for the
distgen inputs the reference's notebooks use (``distgen/distgen.in.yaml``).
Every sampler returns a plain dict of float64 arrays in the openPMD
ParticleGroup convention -- x, y, z [m], px, py, pz [eV/c], t [s],
weight [C], id -- plus ``group_sizes`` (members per emission group, in id
order).  Pure NumPy; importing this module never loads the CUDA library.

Configurations (sizes as stated for each):

* C0  flat cathode, E = -1e7 V/m, 16 groups x 64, x,y ~ N(0, 10 um), z = 0,
      half-Maxwellian MTE 100 meV, t ~ U(0, 1 ps), seed 0.
* C1  hemisphere (R = 50 nm) on a 5 um post, E = -1e6 V/m, 4096 x 32;
      sites on the apex cap within 30 deg, accepted with probability
      (sigma/sigma_max)^2 (|E_surface| = |sigma| for this single-layer
      normalisation), KE ~ U(0, 0.5 eV), Lambertian about the normal,
      t ~ U(0, 1 ps), seed 1.
* C2  the C1 tip, 512 x 1024, (x, y) ~ N(0, 15 nm) truncated to rho < R and
      projected onto the apex sphere, momenta as C1, seed 2.
* C3  cylindrical well R = 2 um, H = 1 um, 65,536 groups of size
      round(logU[1, 256]), uniform over the floor, MTE 50 meV,
      t ~ U(0, 10 ps), seed 3.
* C4  the C1 tip, 65,536 groups of size round(logU[1, 128]), seed 4.
"""

import numpy as np

ELECTRON_MC2_EV = 510998.95069
E_CHARGE = 1.602176634e-19


def _half_maxwellian(rng, n, mte_ev):
    s = np.sqrt(ELECTRON_MC2_EV * mte_ev)
    return rng.normal(0.0, s, n), rng.normal(0.0, s, n), np.abs(rng.normal(0.0, s, n))


def _rotate_z_to(normal, vec):
    """Rodrigues rotation taking +z onto each unit ``normal`` row, applied to ``vec``."""
    axis = np.stack([-normal[:, 1], normal[:, 0], np.zeros(len(normal))], axis=-1)
    s = np.linalg.norm(axis, axis=-1)
    c = normal[:, 2]
    flat = s < 1e-12
    u = axis / np.where(flat, 1.0, s)[:, None]
    dot = np.sum(u * vec, axis=-1, keepdims=True)
    rot = vec * c[:, None] + np.cross(u, vec) * s[:, None] + u * dot * (1.0 - c[:, None])
    return np.where(flat[:, None], np.where(c[:, None] > 0, vec, -vec), rot)


def _lambertian_momenta(rng, normal, ke_max_ev):
    n = len(normal)
    ke = rng.uniform(0.0, ke_max_ev, n)
    p = np.sqrt(2.0 * ELECTRON_MC2_EV * ke)
    ct = np.sqrt(rng.uniform(0.0, 1.0, n))
    st = np.sqrt(1.0 - ct * ct)
    ph = rng.uniform(0.0, 2.0 * np.pi, n)
    local = np.stack([p * st * np.cos(ph), p * st * np.sin(ph), p * ct], axis=-1)
    return _rotate_z_to(normal, local)


def _pack(x, y, z, px, py, pz, t, sizes):
    n = len(x)
    return dict(x=x, y=y, z=z, px=px, py=py, pz=pz, t=t,
                weight=np.full(n, E_CHARGE), id=np.arange(1, n + 1),
                group_sizes=np.asarray(sizes, dtype=np.int64), species="electron")


def flat_c0(n_groups=16, n_emit=64, seed=0, sigma_xy=10e-6, mte_ev=0.1, t_spread=1e-12):
    rng = np.random.default_rng(seed)
    n = n_groups * n_emit
    x = rng.normal(0.0, sigma_xy, n)
    y = rng.normal(0.0, sigma_xy, n)
    px, py, pz = _half_maxwellian(rng, n, mte_ev)
    t = rng.uniform(0.0, t_spread, n)
    return _pack(x, y, np.zeros(n), px, py, pz, t, [n_emit] * n_groups)


def _cap_sites(rng, n, R, apex_z, sigma_of_theta, theta_max=np.pi / 6):
    """Sites on the apex sphere within theta_max, uniform in solid angle,
    thinned by (sigma/sigma_max)^2."""
    grid = np.linspace(0.0, theta_max, 257)
    smax = np.max(np.abs(sigma_of_theta(grid)))
    th_out = np.empty(0)
    cmin = np.cos(theta_max)
    while th_out.size < n:
        m = 2 * (n - th_out.size) + 64
        th = np.arccos(rng.uniform(cmin, 1.0, m))
        keep = rng.uniform(0.0, 1.0, m) < (sigma_of_theta(th) / smax) ** 2
        th_out = np.concatenate([th_out, th[keep]])
    th = th_out[:n]
    ph = rng.uniform(0.0, 2.0 * np.pi, n)
    normal = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], axis=-1)
    pos = normal * R
    pos[:, 2] += apex_z
    return pos, normal


def sigma_on_cap(profile, sigma, R, apex_z):
    """P1 surface density along the apex cap as a function of polar angle."""
    prof = np.asarray(profile, dtype=float)
    th_nodes = np.arctan2(prof[:, 0], prof[:, 1] - apex_z)
    on_cap = prof[:, 1] >= apex_z - 1e-15
    tn, sn = th_nodes[on_cap], np.asarray(sigma)[on_cap]
    order = np.argsort(tn)
    return lambda th: np.interp(th, tn[order], sn[order])


def tip_c1(profile, sigma, n_groups=4096, n_emit=32, seed=1, R=50e-9, L=5e-6, ke_max=0.5, t_spread=1e-12):
    rng = np.random.default_rng(seed)
    n = n_groups * n_emit
    pos, normal = _cap_sites(rng, n, R, L, sigma_on_cap(profile, sigma, R, L))
    mom = _lambertian_momenta(rng, normal, ke_max)
    t = rng.uniform(0.0, t_spread, n)
    return _pack(pos[:, 0], pos[:, 1], pos[:, 2], mom[:, 0], mom[:, 1], mom[:, 2], t, [n_emit] * n_groups)


def tip_c2(n_groups=512, n_emit=1024, seed=2, R=50e-9, L=5e-6, sigma_xy=15e-9, ke_max=0.5, t_spread=1e-12):
    rng = np.random.default_rng(seed)
    n = n_groups * n_emit
    xy = np.empty((0, 2))
    while len(xy) < n:
        c = rng.normal(0.0, sigma_xy, (2 * (n - len(xy)) + 64, 2))
        xy = np.concatenate([xy, c[np.sum(c * c, axis=1) < R * R]])
    x, y = xy[:n, 0], xy[:n, 1]
    zc = np.sqrt(R * R - (x * x + y * y))
    normal = np.stack([x, y, zc], axis=-1) / R
    mom = _lambertian_momenta(rng, normal, ke_max)
    t = rng.uniform(0.0, t_spread, n)
    return _pack(x, y, L + zc, mom[:, 0], mom[:, 1], mom[:, 2], t, [n_emit] * n_groups)


def log_uniform_sizes(rng, n_groups, lo, hi):
    return np.clip(np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), n_groups))), lo, hi).astype(np.int64)


def well_c3(n_groups=65536, seed=3, R=2e-6, H=1e-6, max_size=256, mte_ev=0.05, t_spread=10e-12, sizes=None):
    """``sizes``: fixed group sizes instead of the log-uniform draw (one
    size bin at a time, for fixtures of a per-size reference run)."""
    rng = np.random.default_rng(seed)
    sizes = log_uniform_sizes(rng, n_groups, 1, max_size) if sizes is None else np.asarray(sizes, dtype=np.int64)
    n = int(sizes.sum())
    r = R * np.sqrt(rng.uniform(0.0, 1.0, n))
    ph = rng.uniform(0.0, 2.0 * np.pi, n)
    px, py, pz = _half_maxwellian(rng, n, mte_ev)
    t = rng.uniform(0.0, t_spread, n)
    return _pack(r * np.cos(ph), r * np.sin(ph), np.full(n, -H), px, py, pz, t, sizes)


def tip_c4(profile, sigma, n_groups=65536, seed=4, R=50e-9, L=5e-6, max_size=128, ke_max=0.5, t_spread=1e-12,
           sizes=None):
    """``sizes``: fixed group sizes instead of the log-uniform draw."""
    rng = np.random.default_rng(seed)
    sizes = log_uniform_sizes(rng, n_groups, 1, max_size) if sizes is None else np.asarray(sizes, dtype=np.int64)
    n = int(sizes.sum())
    pos, normal = _cap_sites(rng, n, R, L, sigma_on_cap(profile, sigma, R, L))
    mom = _lambertian_momenta(rng, normal, ke_max)
    t = rng.uniform(0.0, t_spread, n)
    return _pack(pos[:, 0], pos[:, 1], pos[:, 2], mom[:, 0], mom[:, 1], mom[:, 2], t, sizes)


def default_t_max(E_gun, z_far, t_spread):
    """t_max = emission spread + 2 x single-electron transit time to z_far
    in the uniform field E_gun."""
    a = E_CHARGE * abs(E_gun) / (ELECTRON_MC2_EV * E_CHARGE / 299792458.0**2)
    return t_spread + 2.0 * np.sqrt(2.0 * z_far / a)
