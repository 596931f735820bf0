"""Shared helpers for the GPU parity tests: build oracle specs and device
geometries from the golden fixtures, run the oracle on the same inputs."""

import numpy as np

from bem_b200 import geometry as bg
from oracle import geometry as ogeo
from oracle import physics as ophys
from oracle import rk45 as ork

M_E = ophys.ev_to_kg(ophys.ELECTRON_MASS_EV)
Q_E = -ophys.ELEMENTARY_CHARGE
CM = Q_E / M_E


def device_geometry(spec):
    k = spec["kind"]
    if k == "flat":
        return bg.FlatCathode(spec["E_gun"], z0=spec.get("z0"), kill_z_below=spec.get("kill_z_below", 0.0))
    if k == "tip":
        return bg.HemisphericalTip(spec["E_gun"], spec["R"], z0=spec.get("z0"), kill_z_below=spec.get("kill_z_below", 0.0))
    img = {}
    if spec.get("z0") is not None and k in ("tip_bem", "well_bem"):  # the BEM image-charge force
        img = dict(z0=spec["z0"], image_n_max=spec["image_n_max"], image_d_lo=spec["image_d_lo"],
                   image_d_hi=spec["image_d_hi"], image_profile=spec["image_profile"])
        if k == "tip_bem":
            img["image_mirror_symmetric"] = spec.get("image_mirror_symmetric", False)
    if k == "tip_bem":
        return bg.HemisphericalTipBEMGeometry(spec["E_gun"], spec["R"], n_subdiv=spec["n_subdiv"],
                                              z_handoff=spec["z_handoff"], kill_z_below=spec.get("kill_z_below", 0.0),
                                              profile=spec["profile"], sigma=spec["sigma"], **img)
    if k == "well_bem":
        return bg.CylindricalWellBEMGeometry(spec["E_gun"], spec["R"], spec["H"], n_subdiv=spec["n_subdiv"],
                                             bottom_fillet_radius=spec.get("bottom_fillet_radius"),
                                             rim_fillet_radius=spec.get("rim_fillet_radius"),
                                             z_handoff=spec["z_handoff"], profile=spec["profile"], sigma=spec["sigma"],
                                             **img)
    if k == "post_bem":
        return bg.PostTipBEMGeometry(spec["E_gun"], spec["R"], spec["L"], n_subdiv=spec["n_subdiv"], z0=spec.get("z0"),
                                     z_handoff=spec["z_handoff"], kill_z_below=spec.get("kill_z_below", 0.0),
                                     profile=spec["profile"], sigma=spec["sigma"])
    raise KeyError(k)


def oracle_trace(spec, pos0, vel0, tb, t_max, rtol, atol, z_max, max_attempts=None):
    G, E, _ = pos0.shape
    q = np.full((G, E), Q_E)
    m = np.full((G, E), M_E)
    acc = ogeo.make_accel(spec, q, m, CM, 1e-12)
    return ork.integrate(acc, pos0, vel0, tb, t_max, rtol, atol, kill=ogeo.make_kill(spec, z_max),
                         max_attempts=max_attempts)


def device_trace(spec, pos0, vel0, tb, t_max, rtol, atol, z_max, max_attempts=None, log_capacity=4096,
                 form="fp64", far_rule="reference"):
    import torch
    from bem_b200 import engine

    G, E, _ = pos0.shape
    geo = device_geometry(spec)
    tr = engine.Tracer(geo, form=form, z_max=z_max, far_rule=far_rule)
    batch = engine.GroupBatch(pos0.reshape(-1, 3), vel0.reshape(-1, 3), tb.reshape(-1), np.full(G * E, Q_E),
                              np.full(G * E, M_E), [E] * G)
    if max_attempts is None:
        log = tr.run(batch, t_max, rtol, atol, 1e-12, CM, log_capacity=log_capacity)
    else:
        log = (torch.full((G, log_capacity), float("nan"), dtype=torch.float64, device="cuda"),
               torch.full((G, log_capacity), float("nan"), dtype=torch.float64, device="cuda"))
        tr.launch(batch, tr.params(t_max, rtol, atol, 1e-12, CM, max_attempts, log=log))
    torch.cuda.synchronize()
    pos = batch.positions().cpu().numpy().reshape(G, E, 3)
    vel = batch.velocities().cpu().numpy().reshape(G, E, 3)
    td = batch.t_death.cpu().numpy().reshape(G, E)
    out = dict(pos=pos, vel=vel, t_death=td, t=batch.t.cpu().numpy(), h=batch.h.cpu().numpy(),
               n_acc=batch.n_accepted.cpu().numpy(), n_rej=batch.n_rejected.cpu().numpy(),
               status=batch.status.cpu().numpy(), log_h=log[0].cpu().numpy(), log_err=log[1].cpu().numpy(),
               counters=tr.counter_dict())
    return out
