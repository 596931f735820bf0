"""Autotuner for the trace's launch configuration.

The knobs change speed, not physics:

* ``cta_threads`` -- the CTA width (64, 128, 256 threads on one group at a
  time): narrower CTAs put more groups on an SM and fewer warps behind each
  barrier; wider ones spread a large group's work.  Results agree to the
  summation order of the reductions.
* ``team`` -- one group per warp (lane i = particle i, several groups per
  CTA, no CTA barrier inside a group's step) or one group per CTA, where
  the warp team is offered (BEM geometry without the image-charge force,
  float64, adaptive far rule, groups of at most 32).  Results agree to the
  summation order of the pair sums.
* ``round_points`` -- the far-sum tile shape: evaluation points per round
  (1, 2, 4).  Fewer points give each thread more nodes in flight per
  point; more points share node loads and the adaptive rule's
  classification.  Results agree to rounding.
* ``ratios`` -- thresholds (ratio4, ratio2, ratio_run) of the adaptive far
  rule, tuned only with ``tune_ratios=True``.  Candidates pass an accuracy
  guard first: at the sample's own trajectory points their float64 field
  must match the reference quadrature to ``tol`` of the whole field; a
  candidate that does not is never timed.  The guard is necessary, not
  sufficient: on the whole C1 trace the (6, 150, 3) thresholds passed it and
  still moved one group's endpoints by 2.6e-5 from the plain form (the
  defaults: 2e-7), so by default the thresholds stay the defaults, whose
  endpoint error is measured on whole traces.

The group processing order is not tuned: it sets the load balance of the
tail of the full grid, which a sample of groups cannot measure, so it stays
largest first (a sample once preferred the given order, which then cost the
full C1 launch 8 %).

Procedure: a sample of groups (every k-th group, so that every size range is
represented; 2368 = 16 per SM, enough to fill the GPU at every CTA width) is
advanced `warm` attempts from emission, the warmed state is saved, and each
candidate runs `attempts` attempts from that state, timed with CUDA events
(best of `repeats`).  Coordinate descent: team, cta_threads, round_points, then
ratios; a candidate replaces the current choice only if it is faster by more
than `margin` (timing noise on a sample is a few per cent).  The winner
is applied to a Tracer / GroupBatch with ``apply``.  Results can be cached
in a JSON file keyed by the geometry, form, rule and group-size mix.
"""

import json
import os

import numpy as np

from . import _lib, engine, tables

CTA_THREADS = (64, 128, 256)
ROUND_POINTS = (4, 2, 1)
RATIOS = ((tables.RATIO4, tables.RATIO2, tables.RATIO_RUN), (6.0, 150.0, 3.0), (12.0, 600.0, 6.0),
          (16.0, 1000.0, 8.0))
ORDERS = ("largest_first",)


def _torch():
    import torch
    return torch


def signature(tracer, sizes):
    """Cache key: geometry kind and panel count, form, rule, size mix."""
    sizes = np.asarray(sizes)
    hist = np.histogram(np.log2(np.maximum(sizes, 1)), bins=[0, 2, 4, 6, 8, 11])[0]
    n_seg = tracer.tables.n_seg if tracer.tables is not None else 0
    frac = tuple(int(round(100 * h / len(sizes))) for h in hist)
    return f"kind{tracer.geom.kind}-seg{n_seg}-form{tracer.form}-{tracer.far_rule}-sizes{frac}"


class TuneResult(dict):
    """config (team, cta_threads, round_points, ratios, order) plus the timings behind it."""


def warp_team_offered(tracer, sizes):
    """Whether the library offers the warp team for this tracer and group
    sizes (the predicate of the C ABI's team selection)."""
    if tracer.tables is None or tracer.bem is None or tracer.far_rule != "adaptive" or tracer.form != _lib.FORM_FP64:
        return False
    if int(np.max(sizes)) > 32:
        return False
    bem_image = (tracer.geom.kind in (_lib.GEOM_TIP_BEM, _lib.GEOM_WELL_BEM) and tracer.geom.has_image
                 and tracer.bem.image.n_nodes >= 2)
    return not bem_image


def _sample(sizes, n_sample):
    G = len(sizes)
    if G <= n_sample:
        return np.arange(G)
    return np.linspace(0, G - 1, n_sample).round().astype(np.int64)


def _accuracy_ok(tracer, pos, ratios, tol):
    """Float64 field of the candidate adaptive rule against the reference
    rule at the given points, relative to the whole field there."""
    if tracer.tables is None or tracer.far_rule != "adaptive":
        return True
    geo = tracer.geometry
    pts = pos[(pos[:, 2] >= 0.0) & np.isfinite(pos).all(axis=1)]
    if len(pts) == 0:
        return True
    ref = engine.bem_field(tracer.tables, pts).cpu().numpy()
    got = engine.bem_field(tracer.tables, pts, far_rule="adaptive", ratio4=ratios[0], ratio2=ratios[1],
                           ratio_run=ratios[2]).cpu().numpy()
    tot = np.linalg.norm(ref + np.array([0.0, 0.0, float(geo.E_gun)]), axis=-1)
    return bool(np.all(np.abs(got - ref).max(axis=-1) <= tol * tot))


def tune(tracer, pos, vel, t_birth, charge, mass, sizes, t_max, rtol, atol, plummer_radius, charge_to_mass,
         n_sample=2368, warm=200, attempts=32, repeats=3, tol=1e-11, margin=0.03, cache=None, threads=CTA_THREADS,
         tune_ratios=False):
    """Choose the CTA width, round_points (and with tune_ratios the adaptive rule's ratios) for `tracer` on
    this workload (arrays as for GroupBatch; the order stays largest first).  Returns a
    TuneResult; `apply` sets it.  `cache`: a JSON file path (read if it holds
    this signature, updated otherwise)."""
    torch = _torch()
    sizes = np.asarray(sizes, dtype=np.int64)
    key = signature(tracer, sizes)
    if cache and os.path.exists(cache):
        with open(cache) as f:
            stored = json.load(f)
        if key in stored:
            return TuneResult(stored[key], cached=True)
    groups = _sample(sizes, n_sample)
    offs = np.concatenate([[0], np.cumsum(sizes)])
    rows = np.concatenate([np.arange(offs[g], offs[g + 1]) for g in groups])
    sub = (np.asarray(pos)[rows], np.asarray(vel)[rows], np.asarray(t_birth)[rows], np.asarray(charge)[rows],
           np.asarray(mass)[rows], sizes[groups])
    base = engine.GroupBatch(*sub, device=tracer.device)
    prm = lambda a, rp=None, th=None, tm=None: tracer.params(t_max, rtol, atol, plummer_radius, charge_to_mass, a,
                                                             round_points=rp, cta_threads=th, team=tm)
    tracer.launch(base, prm(warm))
    torch.cuda.synchronize()
    work = engine.GroupBatch(*sub, device=tracer.device)
    saved_bem, saved_rp, saved_th, saved_tm = tracer.bem, tracer.round_points, tracer.cta_threads, tracer.team

    def timed(order, rp, ratios, th=0, tm=None):
        tm = cfg["team"] if tm is None else tm
        if tracer.tables is not None:
            tracer.bem = tracer.tables.view(tracer.far_rule, ratio4=ratios[0], ratio2=ratios[1], ratio_run=ratios[2])
        work.set_order(order)
        best = float("inf")
        steps = 0
        for _ in range(repeats):
            work.copy_state_from(base)
            c0 = tracer.counter_dict()["particle_steps"]
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            tracer.launch(work, prm(attempts, rp, th, tm))
            e.record()
            e.synchronize()
            best = min(best, s.elapsed_time(e) * 1e-3)
            steps = tracer.counter_dict()["particle_steps"] - c0
        return steps / best

    timings = {}
    cfg = dict(team=_lib.TEAM_AUTO, cta_threads=0, round_points=4, ratios=list(RATIOS[0]), order="largest_first")

    def pick(rates, current):
        best = max(rates, key=rates.get)
        return best if rates[best] > (1.0 + margin) * rates[current] else current

    try:
        if warp_team_offered(tracer, sizes):
            rates = {}
            for tm, name in ((_lib.TEAM_WARP, "warp"), (_lib.TEAM_CTA, "cta")):
                rates[tm] = timings[f"team={name}"] = timed(cfg["order"], cfg["round_points"], cfg["ratios"], 0, tm)
            cfg["team"] = max(rates, key=rates.get)
        if len(threads) > 1 or threads[0]:
            rates = {}
            for th in threads:
                rates[th] = timings[f"cta_threads={th}"] = timed(cfg["order"], cfg["round_points"], cfg["ratios"], th)
            cfg["cta_threads"] = max(rates, key=rates.get)
        rates = {}
        for rp in ROUND_POINTS:
            rates[rp] = timings[f"round_points={rp}"] = timed(cfg["order"], rp, cfg["ratios"], cfg["cta_threads"])
        cfg["round_points"] = pick(rates, 4)
        if tune_ratios and tracer.tables is not None and tracer.far_rule == "adaptive":
            sample_pos = base.positions().cpu().numpy()
            rates = {}
            for r in RATIOS:
                if not _accuracy_ok(tracer, sample_pos, r, tol):
                    timings[f"ratios={r}"] = "rejected by the accuracy guard"
                    continue
                rates[r] = timings[f"ratios={r}"] = timed(cfg["order"], cfg["round_points"], r, cfg["cta_threads"])
            if RATIOS[0] in rates:
                cfg["ratios"] = list(pick(rates, RATIOS[0]))
            elif rates:
                cfg["ratios"] = list(max(rates, key=rates.get))
    finally:
        tracer.bem, tracer.round_points, tracer.cta_threads, tracer.team = saved_bem, saved_rp, saved_th, saved_tm
    res = TuneResult(cfg, timings=timings, key=key, sample_groups=len(groups), attempts=attempts, warm=warm)
    if cache:
        stored = {}
        if os.path.exists(cache):
            with open(cache) as f:
                stored = json.load(f)
        stored[key] = dict(cfg)
        with open(cache, "w") as f:
            json.dump(stored, f, indent=1)
    return res


def apply(config, tracer, batch=None):
    """Set a tuned configuration on a Tracer (and a GroupBatch's order)."""
    tracer.round_points = int(config["round_points"])
    tracer.cta_threads = int(config.get("cta_threads", 0))
    # the warp team as the library's choice: it takes launches whose groups fill
    # every resident warp (and only the forms it serves), the CTA team the rest
    team = int(config.get("team", _lib.TEAM_AUTO))
    tracer.team = _lib.TEAM_CTA if team == _lib.TEAM_CTA else _lib.TEAM_AUTO
    if tracer.tables is not None:
        r = config["ratios"]
        tracer.bem = tracer.tables.view(tracer.far_rule, ratio4=r[0], ratio2=r[1], ratio_run=r[2])
    if batch is not None:
        batch.set_order(config["order"])
    return tracer
