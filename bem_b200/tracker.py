"""SpecificParticleTracer on the B200 backend.

Same constructor arguments, defaults, validation, warnings and return value
as the reference driver (tracker.py:42-417); the whole
``batched_rk45.integrate`` loop (tracker.py:368-372) is replaced by the
persistent CUDA kernel behind the C ABI, with the geometry's physics
(fields, pair forces, kill test) evaluated inside it rather than through
Python callbacks.  Screen crossings and output-time snapshots are produced on
the device as well and returned as ParticleGroup objects.
"""

import os
import warnings

import numpy as np

from . import backend as backend_module
from . import engine
from . import geometry as geometry_module
from .constants import ev_c_to_si_momentum, ev_to_kg, si_momentum_to_ev_c

DEFAULT_PLUMMER_RADIUS = 1e-12  # tracker.py:22
DEFAULT_RTOL = 1e-7             # tracker.py:23
DEFAULT_ATOL = 1e-12            # tracker.py:39


def _particle_group_class():
    try:
        from beamphysics import ParticleGroup
        return ParticleGroup
    except ImportError:
        try:
            from pmd_beamphysics import ParticleGroup
            return ParticleGroup
        except ImportError:
            return ParticleData


class ParticleData:
    """Stand-in for openPMD-beamphysics' ParticleGroup when that package is
    absent: the same data dict exposed as attributes."""

    def __init__(self, data):
        self._data = dict(data)
        self.species = data.get("species", "electron")

    def __getattr__(self, name):
        d = self.__dict__.get("_data", {})
        if name in d:
            return d[name]
        raise AttributeError(name)

    def __len__(self):
        return len(self._data["x"])


def group_indices(particle_group, n_emit):
    """emission.py:6-38: ids sorted ascending, chunked into groups of n_emit."""
    n = len(particle_group)
    if n_emit < 1:
        raise ValueError(f"n_emit must be a positive integer, got {n_emit}")
    if n % n_emit != 0:
        raise ValueError(f"Number of particles ({n}) is not evenly divisible by n_emit ({n_emit}).")
    ids = np.asarray(particle_group.id)
    if len(np.unique(ids)) != n:
        raise ValueError("particle_group.id must contain unique values.")
    return np.argsort(ids, kind="stable").reshape(n // n_emit, n_emit)


class SpecificParticleTracer:
    def __init__(self, initial_particles, n_emit, geometry, screens, t_out=None,
                 plummer_radius=DEFAULT_PLUMMER_RADIUS, backend="b200", n_workers=1, rtol=None, atol=None,
                 t_max=None, z_max=None, form="fp64", device="cuda", far_rule="reference"):
        if n_workers != 1:
            raise ValueError(
                f"n_workers is only supported for backend='cpu' (got backend={backend!r}, n_workers={n_workers!r})")
        self.initial_particles = initial_particles
        self.n_emit = n_emit
        self.screen_positions = list(screens)
        self.output_times_host = None if t_out is None else np.sort(np.asarray(t_out, dtype=float))
        self.plummer_radius = plummer_radius
        self.z_max = z_max
        if z_max is not None and self.screen_positions and z_max < max(self.screen_positions):
            warnings.warn(
                f"z_max={z_max!r} is below the furthest screen ({max(self.screen_positions)!r}): particles are "
                "killed before reaching it, so crossings recorded at screens beyond z_max are spurious and their "
                "number will vary with step size. Raise z_max above every screen, or drop those screens.",
                stacklevel=2)
        self.n_workers = 1
        self.backend_name = backend
        self.xp, self.dtype = backend_module.resolve_backend(backend)
        self.geometry = geometry_module.from_reference(geometry)
        self.rtol = rtol if rtol is not None else DEFAULT_RTOL
        self.atol = atol if atol is not None else DEFAULT_ATOL
        self.form = form
        self.far_rule = far_rule
        self.device = device
        self._setup_state()
        self.t_max = t_max if t_max is not None else self._default_t_max()

    def _setup_state(self):
        """tracker.py:214-288."""
        pg = self.initial_particles
        idx = group_indices(pg, self.n_emit)
        self.n_groups, self.n_per_group = idx.shape
        self.mass = ev_to_kg(pg.mass)
        self.charge_to_mass = float(pg.species_charge) / self.mass
        qmag = abs(pg.species_charge)
        weight = np.asarray(pg.weight, dtype=float)
        if not np.allclose(weight, qmag, rtol=1e-9, atol=0):
            warnings.warn(
                "SpecificParticleTracer models individual real particles, not statistical macroparticles: "
                f"overriding initial_particles.weight (which was not uniformly {qmag:.6e} C, the species' "
                "elementary charge) so every particle carries exactly one elementary charge of weight.",
                stacklevel=2)
            weight = np.full_like(weight, qmag)
        charge = np.sign(pg.species_charge) * weight
        pmass = self.mass * (weight / qmag)
        flat = idx.reshape(-1)
        self.pos0 = np.stack([np.asarray(pg.x)[flat], np.asarray(pg.y)[flat], np.asarray(pg.z)[flat]], -1)
        self.vel0 = np.stack([ev_c_to_si_momentum(np.asarray(getattr(pg, k)))[flat] / self.mass
                              for k in ("px", "py", "pz")], -1)
        self.t_birth = np.asarray(pg.t, dtype=float)[flat]
        self.charge = charge[flat]
        self.particle_mass = pmass[flat]
        self.weight = weight[flat]
        self.ids = np.asarray(pg.id)[flat]
        self.species = pg.species

    def _default_t_max(self):
        """tracker.py:290-307."""
        a0 = abs(self.geometry.E_gun) * abs(self.charge_to_mass)
        z = np.array(self.screen_positions, dtype=float)
        zp = z[z > 0]
        t_transit = np.sqrt(2 * zp.max() / a0) if len(zp) > 0 and a0 > 0 else 1e-12
        t = float(self.t_birth.max()) + 3.0 * t_transit
        if self.output_times_host is not None:
            t = max(t, float(self.output_times_host.max()))
        return t

    def run(self, verbose=False):
        """tracker.py:312-386 -> (screen ParticleGroups, trajectory ParticleGroups)."""
        tracer = engine.Tracer(self.geometry, device=self.device, form=self.form, z_max=self.z_max,
                               far_rule=self.far_rule)
        batch = engine.GroupBatch(self.pos0, self.vel0, self.t_birth, self.charge, self.particle_mass,
                                  [self.n_per_group] * self.n_groups, device=self.device)
        rec = tracer.run(batch, self.t_max, self.rtol, self.atol, self.plummer_radius, self.charge_to_mass,
                         screens=self.screen_positions, output_times=self.output_times_host)
        if verbose:
            c = tracer.counter_dict()
            print(f"{c['accepted']} accepted group-steps across {self.n_groups} groups (backend={self.backend_name})")
        self.final_state = dict(pos=batch.positions().cpu().numpy(), vel=batch.velocities().cpu().numpy(),
                                t_death=batch.t_death.cpu().numpy())
        screens = [self._build(r) for r in rec.screen_records()] if self.screen_positions else []
        trajs = [self._build(r) for r in rec.output_records()] if self.output_times_host is not None else []
        return screens, trajs

    def _build(self, rec):
        """tracker.py:388-417."""
        PG = _particle_group_class()
        if rec is None or len(rec["t"]) == 0:
            data = dict(x=np.array([]), y=np.array([]), z=np.array([]), px=np.array([]), py=np.array([]),
                        pz=np.array([]), t=np.array([]), weight=np.array([]), status=np.array([]),
                        id=np.array([], dtype=int), species=self.species)
            return PG(data=data) if PG is not ParticleData else ParticleData(data)
        p = rec["particle"]
        data = dict(x=rec["x"], y=rec["y"], z=rec["z"],
                    px=si_momentum_to_ev_c(rec["vx"] * self.mass), py=si_momentum_to_ev_c(rec["vy"] * self.mass),
                    pz=si_momentum_to_ev_c(rec["vz"] * self.mass), t=rec["t"], weight=self.weight[p],
                    status=np.ones_like(rec["t"]), id=self.ids[p].astype(int), species=self.species)
        return PG(data=data) if PG is not ParticleData else ParticleData(data)
