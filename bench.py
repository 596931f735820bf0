"""Benchmark: accepted RK45 particle-steps per second of the photoemission
tracer's hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload c1|c0|c2|c3|c4] [--span trace|slice] [--t-end T]
                    [--form mixed|fp64] [--far-rule adaptive|reference]
                    [--cta-threads 64|128|256] [--bins] [--no-tune] ...

The chosen form (the default): float64 arithmetic with the adaptive
far-field rule (the BEM far sum ~1e-14 from the reference's quadrature;
the plain form's step sequence on ~99 % of groups), its launch
configuration chosen first by the project's autotuner on a sample of the
workload (untimed; `--no-tune` keeps the defaults).  `--form mixed` times
the float32 + Kahan form instead; on the whole C1 trace it misses the 1e-6
endpoint bar in a few groups, so the default run reports it beside the
chosen form (accuracy.mixed_form) rather than as the headline.

Workload (default c1, the largest single-GPU configuration with a BEM
field): hemisphere R = 50 nm on a 5 um post, E = -1e6 V/m, 2000-panel BEM
capsule (64,000 far nodes), 4096 groups x 32 electrons, Coulomb + 3-image
forces, rtol 1e-9, atol 1e-12, z_max = 1 mm, seed 1.  Synthetic, seeded
inputs (workloads.py) stand in for a distgen distribution.

A step (--span trace, the default) is one WHOLE trace of the workload: every
group from its emission to t_end (C1: 20 ps, 19 ps past the last birth; the
integrator's t_max is t_end), in one persistent spt_trace launch (one per
size bin with --bins), from the same initial state each step (restored
untimed).  W warm-up steps, then K timed steps; L2 is flushed (256 MiB
write) before each step and each step is timed alone with CUDA events on the
launch stream.  value = accepted particle-steps (device counter: sum over
accepted group-steps of the group size) / summed step time.
`live_particle_steps_per_s` counts only the particles alive at each
accepted step.  --span slice times --attempts attempts per group per step
instead, continuing from the previous step (labelled in config).

In the same run (rank 0):
  plain_fp64  the plain form (float64, the reference's quadrature) traces the
              first --plain-groups groups over the same span; the chosen form
              traces the same groups; ratio = chosen / plain on that subset.
  accuracy    endpoint error of the chosen form against the plain form on
              that subset (alive particles by position and velocity, killed
              ones by death time), and their attempt counts; beside it the
              plain form's own sensitivity (the same subset with vel0 x
              (1 + 1e-15)), and the error over the particles that sensitivity
              shows to be well conditioned (moved < 1e-7 by it).
  e2e         the same whole traces through the public API with the state in
              pinned host memory: H2D of the initial state, the trace, D2H of
              the final state, every step.
  cpu_baseline  the oracle port (the reference's algorithm) on the host
              cores, on a bounded prefix of the same trace.
  image_force the BEM image-charge force per call (spt_image_force) at the
              batch shapes the reference published timings for.

N > 1 (torchrun): the workload is N x the groups (one draw of N x 4096
groups for C1), split into contiguous group ranges balanced by estimated
cost (partition.py; weak scaling); each rank traces its range; the final
state is all-gathered (NCCL) inside each timed step; times are the max over
ranks.
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "accepted RK45 particle-steps/s at ≤1e-6 rel endpoint err: chosen form vs plain FP64"
UNIT = "particle-steps/s"
FLOP_PER_RING = 64.0   # nominal FLOPs of one ring-kernel evaluation (26 algebra + 38 for K, E)
FLOP_PER_PAIR = 20.0   # nominal FLOPs of one softened pair interaction
FLOP_PER_CLUSTER = 12.0 * 32  # nominal FLOPs of one 32-term cluster expansion (12 per term)
WHOLE_TRACE = 1_000_000  # attempt budget of a whole-trace launch (every group reaches t_end far sooner)
T_END = dict(c0=None, c1=20e-12, c2=20e-12, c3=30e-12, c4=20e-12)


# ---------------------------------------------------------------------------
# workloads

def build_workload(name, n_copies=1):
    """Returns dict(geometry, data, rtol, atol, t_max, z_max, config).
    n_copies > 1: the same sampler drawn at n_copies x the groups (the
    multi-GPU workload, partitioned across ranks)."""
    from bem_b200 import geometry as bg
    from bem_b200 import workloads as w

    if name == "c0":
        geo = bg.FlatCathode(-1e7, z0=3e-9, kill_z_below=0.0)
        data = w.flat_c0(n_groups=16 * n_copies, seed=0)
        return dict(geometry=geo, data=data, rtol=1e-8, atol=1e-12, t_max=w.default_t_max(-1e7, 1e-3, 1e-12),
                    z_max=1e-3, config=dict(workload=f"C0 flat cathode, {16 * n_copies} groups x 64, rtol 1e-8",
                                            groups=16 * n_copies, group_size=64, bem_panels=0))
    if name in ("c1", "c2", "c4"):
        geo = bg.PostTipBEMGeometry(-1e6, 50e-9, 5e-6, n_cap=100, n_wall=900, n_subdiv=8, z0=3e-9)
        if name == "c1":
            G = 4096 * n_copies
            data = w.tip_c1(geo.profile, geo.sigma, n_groups=G, seed=1)
            cfg = dict(workload=f"C1 hemisphere-on-post BEM tip, {G} groups x 32, 2000 panels, rtol 1e-9",
                       groups=G, group_size=32)
        elif name == "c2":
            G = 512 * n_copies
            data = w.tip_c2(n_groups=G, seed=2)
            cfg = dict(workload=f"C2 post tip, {G} groups x 1024, 2000 panels, rtol 1e-9", groups=G, group_size=1024)
        else:
            G = 65536 * n_copies
            data = w.tip_c4(geo.profile, geo.sigma, n_groups=G, seed=4)
            cfg = dict(workload=f"C4 post tip, {G} groups of size logU[1,128], rtol 1e-9", groups=G,
                       group_size="1-128")
        cfg.update(bem_panels=geo.profile.shape[0] - 1, far_nodes=(geo.profile.shape[0] - 1) * 32,
                   particles=int(np.sum(data["group_sizes"])))
        return dict(geometry=geo, data=data, rtol=1e-9, atol=1e-12, t_max=w.default_t_max(-1e6, 1e-3, 1e-12),
                    z_max=1e-3, config=cfg)
    if name == "c3":
        geo = bg.CylindricalWellBEMGeometry(-2.5e6, 2e-6, 1e-6, n_segments=3000)
        G = 65536 * n_copies
        data = w.well_c3(n_groups=G, seed=3)
        return dict(geometry=geo, data=data, rtol=1e-9, atol=1e-12, t_max=w.default_t_max(-2.5e6, 2e-3, 10e-12),
                    z_max=2e-3, config=dict(workload=f"C3 cylindrical well, {G} groups of size logU[1,256], rtol 1e-9",
                                            groups=G, group_size="1-256", bem_panels=geo.profile.shape[0] - 1,
                                            particles=int(np.sum(data["group_sizes"]))))
    raise ValueError(name)


def first_groups(data, n):
    """The workload cut to its first n emission groups."""
    from bem_b200.partition import shard
    if n is None or n >= len(data["group_sizes"]):
        return data
    return shard(data, 0, n)


def particle_arrays(data):
    from bem_b200.constants import ELEMENTARY_CHARGE, SPEED_OF_LIGHT, ev_to_kg
    m = ev_to_kg(510998.95069)
    pos = np.stack([data["x"], data["y"], data["z"]], -1)
    vel = np.stack([data["px"], data["py"], data["pz"]], -1) * ELEMENTARY_CHARGE / SPEED_OF_LIGHT / m
    n = len(pos)
    return pos, vel, data["t"], np.full(n, -ELEMENTARY_CHARGE), np.full(n, m), -ELEMENTARY_CHARGE / m


def _default_t_max(name):
    from bem_b200 import workloads as w
    return dict(c0=w.default_t_max(-1e7, 1e-3, 1e-12))[name]


def span_t_max(args):
    """The integrator's t_max for this run: t_end of the trace span."""
    t = args.t_end if args.t_end is not None else T_END[args.workload]
    return _default_t_max(args.workload) if t is None else float(t)


# ---------------------------------------------------------------------------
# CPU leg (oracle port; spawn pool, started before any CUDA use)

def _cpu_job(args):
    g, attempts = args
    import numpy as _np
    from oracle import geometry as ogeo
    from oracle import rk45 as ork
    wl = _cpu_blob()
    data = wl["data"]
    sizes = data["group_sizes"]
    offs = _np.concatenate([[0], _np.cumsum(sizes)])
    sl = slice(offs[g], offs[g + 1])
    pos, vel, tb, q, m, cm = particle_arrays({k: (v[sl] if k not in ("group_sizes", "species") else v)
                                              for k, v in data.items()})
    E = len(pos)
    spec = wl["spec"]
    acc = ogeo.make_accel(spec, q.reshape(1, E), m.reshape(1, E), cm, 1e-12)
    t0 = time.perf_counter()
    _, _, _, _, _, log = ork.integrate(acc, pos.reshape(1, E, 3), vel.reshape(1, E, 3), tb.reshape(1, E),
                                       wl["t_max"], wl["rtol"], wl["atol"],
                                       kill=ogeo.make_kill(spec, wl["z_max"]), max_attempts=attempts)
    dt = time.perf_counter() - t0
    accepted = int(_np.sum(log[0][2]))
    return accepted * E, len(log[0][0]), dt


_CPU_CACHE = {}


def _cpu_blob():
    path = os.environ["SPT_BENCH_CPU_BLOB"]
    if path not in _CPU_CACHE:
        _CPU_CACHE[path] = np.load(path, allow_pickle=True)["wl"].item()
    return _CPU_CACHE[path]


def cpu_leg(n_procs, attempts, groups):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(n_procs) as pool:
        res = pool.map(_cpu_job, [(g, attempts) for g in groups])
    wall = time.perf_counter() - t0
    steps = sum(r[0] for r in res)
    return steps / wall, steps, wall, sum(r[1] for r in res)


def _make_blob(name, t_max):
    wl = build_workload(name)
    spec = wl["geometry"].spec()
    blob = dict(spec=spec, data=dict(wl["data"]), rtol=wl["rtol"], atol=wl["atol"], t_max=t_max, z_max=wl["z_max"],
                config=wl["config"])
    import tempfile
    path = os.path.join(tempfile.gettempdir(), f"spt_bench_cpu_{name}_{os.getpid()}.npz")
    np.savez(path, wl=np.array(blob, dtype=object))
    return path


def prepare_cpu(name, t_max):
    """Workload for the CPU legs, built in a spawned child (BEM workloads
    need the device solve; this process stays CUDA-free for the spawn pool)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        path = pool.apply(_make_blob, (name, t_max))
    os.environ["SPT_BENCH_CPU_BLOB"] = path
    return _cpu_blob()


def physical_cores():
    """Worker processes for the CPU legs: the physical cores, at most 64, and
    no more than the available host memory allows at ~2 GiB per worker (a
    worker's float64 ring-sum temporaries over 64,000 nodes)."""
    n = os.cpu_count() or 1
    try:
        import psutil
        n = psutil.cpu_count(logical=False) or n
        n = min(n, max(1, int(psutil.virtual_memory().available / 2**30) // 2))
    except Exception:
        pass
    return max(1, min(n, 64))


def cpu_sample(wl):
    procs = min(physical_cores(), 64)
    groups = list(range(min(procs, len(wl["data"]["group_sizes"]))))
    return procs, groups


def cpu_baseline(args, t_max):
    """The oracle port on the host cores, on a bounded sample of the same
    trace: the first `procs` groups (one per process) for --cpu-attempts
    attempts each from emission, with the same t_max as the GPU span."""
    wl = prepare_cpu(args.workload, t_max)
    procs, groups = cpu_sample(wl)
    value, steps, wall, attempts = cpu_leg(procs, args.cpu_attempts, groups)
    return dict(value=value, unit=UNIT, cores=procs, kind="port",
                sample=f"first {len(groups)} groups of the workload, {args.cpu_attempts} attempts each from "
                       f"emission toward t_max = {t_max:.3g} s (the GPU trace's span), one group per process; "
                       f"{steps} accepted particle-steps in {wall:.1f} s")


# ---------------------------------------------------------------------------
# clocks

class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return dict(sm_mhz=float(np.median(sm)) if sm else None, sm_max_mhz=mx, reasons=sorted(reasons),
                    samples=len(sm))


# ---------------------------------------------------------------------------
# GPU leg

def _gemm_peak(torch, dev, dtype, n):
    a = torch.randn(n, n, dtype=dtype, device=dev)
    b = torch.randn(n, n, dtype=dtype, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) * 1e-3)
    del a, b
    return 2.0 * n**3 / best / 1e12


def fp64_peak_tflops(torch, dev):
    """Measured float64 GEMM rate (cuBLAS DGEMM, 4096^3, best of 5): the
    FP64 denominator (no FP64 figure in the measured-peaks file)."""
    return _gemm_peak(torch, dev, torch.float64, 4096)


def fp32_peak_tflops(torch, dev):
    """Float32 CUDA-core peak measured in-run: a float32 GEMM with TF32 off."""
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        return _gemm_peak(torch, dev, torch.float32, 8192)
    finally:
        torch.backends.cuda.matmul.allow_tf32 = old


def combine_ranks(t_total, particle_steps, world, device):
    """Whole-job numbers of a multi-rank run: the slowest rank's timed region
    (max) and the particle-steps of all ranks (sum), by collectives on the
    initialised process group (NCCL on the GPU path; any backend)."""
    if world == 1:
        return float(t_total), float(particle_steps)
    import torch
    import torch.distributed as dist
    tt = torch.tensor([float(t_total)], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    st = torch.tensor([float(particle_steps)], dtype=torch.float64, device=device)
    dist.all_reduce(st)
    return float(tt.item()), float(st.item())


TEAMS = dict(auto=0, cta=1, warp=2)
TEAM_NAMES = {0: "library's choice (one group per warp where offered)", 1: "one group per CTA",
              2: "one group per warp"}


def make_tracer(args, wl, dev, form=None, far_rule=None):
    from bem_b200 import engine
    tr = engine.Tracer(wl["geometry"], device=dev, form=form or args.form, z_max=wl["z_max"],
                       far_rule=far_rule or args.far_rule)
    tr.kappa_max = args.kappa
    if form is None and far_rule is None:
        tr.team = TEAMS[args.team]
    return tr


class Runner:
    """One workload on one device: a pristine copy of the initial state, the
    working batch, and whole-trace (or slice) launches, binned or not."""

    def __init__(self, tracer, pos, vel, tb, q, m, sizes, dev, binned=False):
        from bem_b200 import engine
        self.tracer = tracer
        self.batch = engine.GroupBatch(pos, vel, tb, q, m, sizes, device=dev)
        self.init = engine.GroupBatch(pos, vel, tb, q, m, sizes, device=dev)
        self.plan = self.batch.bin_plan() if binned else None

    def reset(self):
        self.batch.copy_state_from(self.init)

    def launch(self, params, stream):
        if self.plan is not None:
            self.tracer.launch_binned(self.batch, params, self.plan, stream)
        else:
            self.tracer.launch(self.batch, params, stream)

    def check_done(self):
        from bem_b200 import engine
        if not engine.Tracer._check_done(self.batch):
            raise RuntimeError("a whole-trace launch left groups unfinished")


def run_gpu(args, rank, world):
    import torch
    from bem_b200 import partition

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    wl = build_workload(args.workload, n_copies=world)
    data = wl["data"]
    if args.groups:
        data = first_groups(data, args.groups * world)
        wl["config"] = dict(wl["config"], groups=args.groups * world,
                            workload=wl["config"]["workload"] + f" (first {args.groups * world} groups)")
    all_sizes = np.asarray(data["group_sizes"])
    ranges = partition.partition(all_sizes, world)
    g0, g1 = ranges[rank]
    local = partition.shard(data, g0, g1)
    pos, vel, tb, q, m, cm = particle_arrays(local)
    wl["cm"] = cm
    sizes = local["group_sizes"]
    t_max = span_t_max(args)
    trace = args.span == "trace"
    budget = WHOLE_TRACE if trace else args.attempts

    tracer = make_tracer(args, wl, dev)
    if args.cta_threads:
        tracer.cta_threads = args.cta_threads
    tuned = None
    if args.tune:
        from bem_b200 import autotune
        t0 = time.perf_counter()
        threads = (args.cta_threads,) if (args.cta_threads or args.bins) else autotune.CTA_THREADS
        res = autotune.tune(tracer, pos, vel, tb, q, m, sizes, t_max, wl["rtol"], wl["atol"], 1e-12, cm,
                            threads=threads)
        autotune.apply(res, tracer)
        if args.team != "auto":
            tracer.team = TEAMS[args.team]
        args.tuned_config = res
        tuned = dict(res, seconds=round(time.perf_counter() - t0, 2),
                     timings={k: (round(v) if isinstance(v, float) else v) for k, v in res.get("timings", {}).items()})
    run = Runner(tracer, pos, vel, tb, q, m, sizes, dev, binned=args.bins)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    counts = [int(np.sum(all_sizes[a:b])) for a, b in ranges]
    gcounts = [b - a for a, b in ranges]
    prm = lambda: tracer.params(t_max, wl["rtol"], wl["atol"], 1e-12, cm, budget)

    def step():
        if trace:
            run.reset()
        flush.fill_(1.0)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        run.launch(prm(), stream)
        if world > 1:
            b = run.batch
            partition.gather_state({k: getattr(b, k) for k in partition.STATE_PARTICLE + partition.STATE_GROUP},
                                   counts, gcounts)
        e.record(stream)
        e.synchronize()
        if trace:
            run.check_done()
        return s.elapsed_time(e) * 1e-3

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    c0 = tracer.counter_dict()
    times = []
    with ClockSampler(dev.index) as clk:
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            times.append(step())
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
    c1 = tracer.counter_dict()
    dc = {k: c1[k] - c0[k] for k in c1}
    t_total = float(np.sum(times))
    t_max_ranks, steps_all = combine_ranks(t_total, dc["particle_steps"], world, dev)
    _, live_all = combine_ranks(t_total, dc["live_steps"], world, dev)

    e2e = plain = acc = None
    if rank == 0 and not args.no_e2e:
        e2e = e2e_leg(args, wl, tracer, pos, vel, tb, q, m, sizes, dev, t_max, budget)
    if rank == 0 and not args.no_plain and (args.form, args.far_rule) != ("fp64", "reference"):
        plain, acc = plain_and_accuracy(args, wl, pos, vel, tb, q, m, sizes, dev, t_max, budget)
    img = image_force_leg(dev) if rank == 0 and not args.no_image else None
    peak = (fp64_peak_tflops if args.form == "fp64" else fp32_peak_tflops)(torch, dev) if rank == 0 else None
    flops = (dc["ring_far"] * FLOP_PER_RING + dc["ring_near"] * FLOP_PER_RING + dc["pair_evals"] * FLOP_PER_PAIR
             + dc["cluster_evals"] * FLOP_PER_CLUSTER)
    achieved = flops / t_total / 1e12
    return dict(value=steps_all / t_max_ranks, live=live_all / t_max_ranks, t_total=t_max_ranks, times=times,
                counters=dc, clocks=clk.summary(), e2e=e2e, peak=peak, achieved=achieved, config=wl["config"],
                plain=plain, accuracy=acc, tuned=tuned, t_max=t_max, ranges=ranges, image_force=img,
                team=TEAM_NAMES[tracer.team],
                launches_per_step=len(run.plan) if run.plan else 1)


# The reference's own per-call image-force timings (docs/gpu_performance.md:21-29; RTX 5070 Ti, CuPy),
# samples 1 nm outside the tip or above the well bottom: (geometry, G, E) -> ms per call
IMAGE_PUBLISHED_MS = {("tip", 1, 1): 4.51, ("tip", 32, 4): 5.15, ("tip", 256, 4): 21.18,
                      ("well", 1, 1): 4.28, ("well", 32, 4): 6.35, ("well", 256, 4): 19.81}


def image_force_leg(dev, reps=7):
    """spt_image_force per call (geometry level, the tables of
    HemisphericalTipBEMGeometry(R = 50 nm, z0 = 3 nm) and
    CylindricalWellBEMGeometry(R = 2 um, H = 1 um, z0 = 3 nm) with the
    reference's default image parameters) at the batch shapes the reference
    published, points 1 nm outside the tip / above the well floor: median of
    `reps` CUDA-event-timed calls after a warm-up, inputs resident."""
    import torch
    from bem_b200 import _lib
    from bem_b200 import image_charge as ic
    from bem_b200.constants import COULOMB_CONSTANT, ELEMENTARY_CHARGE
    rng = np.random.default_rng(7)
    out = []
    for geo_name in ("tip", "well"):
        z0 = 3e-9
        g = _lib.SptGeometry()
        g.has_image, g.z0 = 1, z0
        if geo_name == "tip":
            R = 50e-9
            prof = ic.tip_image_profile(R, z0, 5 * R, (R - z0) * np.pi / 2 / 29)
            g.kind, g.R, g.z_handoff = _lib.GEOM_TIP_BEM, R, 20 * R
        else:
            R, H = 2e-6, 1e-6
            room = min(0.5 * z0, 0.2 * (H - z0))
            prof = ic.well_image_profile(R, H, z0, 5 * R, min(R, H) / 14, room, z0 + room)
            g.kind, g.R, g.H, g.z_handoff = _lib.GEOM_WELL_BEM, R, H, 20 * R
        sol = ic.ImageChargeSolution(prof, 16, 0.1 * R, 0.5 * R, device=dev)
        for G, E in ((1, 1), (32, 4), (256, 4)):
            n = G * E
            if geo_name == "tip":
                th = rng.uniform(0, np.radians(60), n)
                ph = rng.uniform(-np.pi, np.pi, n)
                r = R + 1e-9
                pts = np.stack([r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), r * np.cos(th)], -1)
            else:
                rr = 0.8 * R * np.sqrt(rng.uniform(0, 1, n))
                ph = rng.uniform(-np.pi, np.pi, n)
                pts = np.stack([rr * np.cos(ph), rr * np.sin(ph), np.full(n, -H + 1e-9)], -1)
            pos = torch.as_tensor(pts, device=dev)
            q = torch.full((n,), -ELEMENTARY_CHARGE, dtype=torch.float64, device=dev)
            act = torch.ones(n, dtype=torch.uint8, device=dev)
            off = torch.arange(0, n + 1, E, dtype=torch.int64, device=dev)
            f = torch.empty((3, n), dtype=torch.float64, device=dev)
            call = lambda: sol.force(pos, q, act, off, E, geometry=g, coulomb_constant=COULOMB_CONSTANT, out=f)
            call()
            torch.cuda.synchronize()
            ts = []
            st = torch.cuda.current_stream(dev)
            for _ in range(reps):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(st)
                call()
                b.record(st)
                b.synchronize()
                ts.append(a.elapsed_time(b))
            ms = float(np.median(ts))
            pub = IMAGE_PUBLISHED_MS[(geo_name, G, E)]
            out.append(dict(geometry=geo_name, groups=G, group_size=E, ms_per_call=ms,
                            reference_published_ms=pub, ratio=pub / ms))
    return dict(what="geometry-level BEM image-charge force per call (spt_image_force, n_max 16); reference: "
                     "its own published per-call times (RTX 5070 Ti, CuPy), not the same hardware", calls=out)


def plain_and_accuracy(args, wl, pos, vel, tb, q, m, sizes, dev, t_max, budget):
    """The plain form (float64, the reference's quadrature) and the chosen
    form over the same span on the first --plain-groups groups: the ratio of
    their rates, and the chosen form's endpoint error against the plain one
    (alive particles by position and velocity; particles killed at the
    emitter or at z_max keep the state of the step that crossed, which moves
    with the step sequence: compared by death time)."""
    import torch
    n = min(args.plain_groups, len(sizes))
    k = int(np.sum(sizes[:n]))
    sub = (pos[:k], vel[:k], tb[:k], q[:k], m[:k], sizes[:n])
    out = {}
    stream = torch.cuda.current_stream(dev)
    legs = [("plain", "fp64", "reference"), ("chosen", args.form, args.far_rule)]
    if args.form == "fp64" and args.far_rule == "adaptive":
        legs.append(("mixed", "mixed", "adaptive"))  # the float32 form, reported beside the chosen one
    if not args.no_sensitivity:
        legs.append(("plain_pert", "fp64", "reference"))  # the plain form's own sensitivity (vel0 x (1 + 1e-15))
    for name, form, rule in legs:
        tracer = make_tracer(args, wl, dev, form, rule)
        binned = False
        if name != "plain":
            binned = args.bins
            if getattr(args, "tuned_config", None):
                from bem_b200 import autotune
                autotune.apply(args.tuned_config, tracer)
            elif args.cta_threads:
                tracer.cta_threads = args.cta_threads
        leg = sub if name != "plain_pert" else (sub[0], sub[1] * (1.0 + 1e-15)) + sub[2:]
        run = Runner(tracer, *leg, dev, binned=binned)
        prm = lambda a: tracer.params(t_max, wl["rtol"], wl["atol"], 1e-12, wl["cm"], a)
        # warm-up: a short slice, then the timed span from the initial state
        run.launch(prm(4), stream)
        torch.cuda.synchronize()
        run.reset()
        c0 = tracer.counter_dict()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        run.launch(prm(budget), stream)
        e.record(stream)
        e.synchronize()
        c = {kk: v - c0[kk] for kk, v in tracer.counter_dict().items()}
        b = run.batch
        out[name] = dict(t=s.elapsed_time(e) * 1e-3, c=c, pos=b.positions().cpu().numpy(),
                         vel=b.velocities().cpu().numpy(), td=b.t_death.cpu().numpy())
    P, C = out["plain"], out["chosen"]
    rate = lambda o: o["c"]["particle_steps"] / o["t"]

    def errors(C):
        d0, d1 = P["td"], C["td"]
        alive = ~np.isfinite(d0) & ~np.isfinite(d1)
        ex = np.linalg.norm(C["pos"] - P["pos"], axis=-1)[alive] / np.linalg.norm(P["pos"], axis=-1)[alive]
        return ex
    span = f"whole trace to t = {t_max:.3g} s" if budget == WHOLE_TRACE else f"{budget} attempts from emission"
    plain = dict(value=rate(P), unit=UNIT, seconds=P["t"], form="fp64", far_rule="reference", groups=n,
                 chosen_value_same_groups=rate(C), chosen_seconds=C["t"], ratio=rate(C) / rate(P),
                 time_ratio=P["t"] / C["t"], span=f"first {n} groups, {span}")
    d0, d1 = P["td"], C["td"]
    alive = ~np.isfinite(d0) & ~np.isfinite(d1)
    dead = np.isfinite(d0) & np.isfinite(d1)
    ex = np.linalg.norm(C["pos"] - P["pos"], axis=-1)[alive] / np.linalg.norm(P["pos"], axis=-1)[alive]
    ev = np.linalg.norm(C["vel"] - P["vel"], axis=-1)[alive] / np.linalg.norm(P["vel"], axis=-1)[alive]
    et = np.abs(d1[dead] - d0[dead]) / d0[dead]
    acc = dict(groups=n, particles=k, t_end=t_max, against="plain fp64 (reference quadrature) on the GPU",
               alive=int(alive.sum()), max_rel_pos=float(ex.max()) if ex.size else None,
               median_rel_pos=float(np.median(ex)) if ex.size else None,
               max_rel_vel=float(ev.max()) if ev.size else None,
               killed=int(dead.sum()), killed_in_one_only=int((np.isfinite(d0) != np.isfinite(d1)).sum()),
               max_rel_t_death=float(et.max()) if et.size else None,
               attempts_plain=int(P["c"]["attempts"]), attempts_chosen=int(C["c"]["attempts"]),
               accepted_steps_ratio=float(C["c"]["accepted"] / max(P["c"]["accepted"], 1)))
    if "plain_pert" in out:
        # endpoints are only as well defined as the trajectory allows: a 1e-15 change of vel0 moves the
        # plain form's own endpoints by `sens`; the chosen form is held to 1e-6 where sens < 1e-7
        d0, d1, d2 = P["td"], C["td"], out["plain_pert"]["td"]
        alive_all = ~np.isfinite(d0) & ~np.isfinite(d1) & ~np.isfinite(d2)
        rel = lambda X: np.linalg.norm(X["pos"] - P["pos"], axis=-1)[alive_all] / \
            np.linalg.norm(P["pos"], axis=-1)[alive_all]
        sens, err = rel(out["plain_pert"]), rel(C)
        well = sens < 1e-7
        acc["plain_self_sensitivity"] = dict(
            what="plain form against itself with vel0 x (1 + 1e-15), alive particles", max_rel_pos=float(sens.max()),
            particles_above_1e6=int((sens > 1e-6).sum()), seconds=out["plain_pert"]["t"])
        acc["max_rel_pos_well_conditioned"] = float(err[well].max()) if well.any() else None
        acc["well_conditioned_particles"] = int(well.sum())
        acc["max_error_over_sensitivity"] = float((err / np.maximum(sens, 1e-7)).max())
    if "mixed" in out:
        X = out["mixed"]
        e = errors(X)
        acc["mixed_form"] = dict(
            note="float32 + Kahan pair and far sums, adaptive far rule: faster, but over 1e-6 on this span, so "
                 "not the chosen form", value=rate(X), ratio_to_plain=rate(X) / rate(P),
            max_rel_pos=float(e.max()) if e.size else None, particles_above_1e6=int((e > 1e-6).sum()),
            accepted_steps_ratio=float(X["c"]["accepted"] / max(P["c"]["accepted"], 1)))
    return plain, acc


def e2e_leg(args, wl, tracer, pos, vel, tb, q, m, sizes, dev, t_max, budget):
    """The same traces through the public API with the state in pinned host
    memory: every step copies the initial state host -> device, traces, and
    copies the final state device -> host.  min(K, 3) steps after one
    warm-up."""
    import torch
    from bem_b200 import engine

    run = Runner(tracer, pos, vel, tb, q, m, sizes, dev, binned=args.bins)
    batch = run.batch
    names = list(engine.GroupBatch.STATE)
    host_in = {k: torch.empty_like(getattr(batch, k), device="cpu").pin_memory() for k in names}
    host_out = {k: torch.empty_like(getattr(batch, k), device="cpu").pin_memory() for k in names}
    for k in names:
        host_in[k].copy_(getattr(batch, k))
    stream = torch.cuda.current_stream(dev)
    prm = lambda: tracer.params(t_max, wl["rtol"], wl["atol"], 1e-12, wl["cm"], budget)
    nbytes = sum(host_in[k].numel() * host_in[k].element_size() for k in names)
    n_steps = max(1, min(args.steps, 3))
    c_total, wall = 0, 0.0
    for it in range(1 + n_steps):
        c0 = tracer.counter_dict()["particle_steps"]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in names:
            getattr(batch, k).copy_(host_in[k], non_blocking=True)
        run.launch(prm(), stream)
        for k in names:
            host_out[k].copy_(getattr(batch, k), non_blocking=True)
        stream.synchronize()
        dt = time.perf_counter() - t0
        if it > 0:
            wall += dt
            c_total += tracer.counter_dict()["particle_steps"] - c0
    return dict(value=c_total / wall, unit=UNIT, h2d_bytes_per_step=int(nbytes), d2h_bytes_per_step=int(nbytes),
                steps=n_steps)


def load_traffic(workload, form, far_rule):
    """DRAM bytes per trace launch from the committed ncu summary of this
    workload and form (profiles/), or None."""
    for name in (f"trace_kernel_{workload}_{form}_{far_rule}.json", f"trace_kernel_{workload}_{form}.json"):
        path = os.path.join(REPO, "profiles", name)
        if os.path.exists(path) and (far_rule == "reference" or name.endswith(f"_{far_rule}.json")):
            with open(path) as f:
                return json.load(f)
    return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="c1", choices=["c0", "c1", "c2", "c3", "c4"])
    ap.add_argument("--span", default="trace", choices=["trace", "slice"],
                    help="trace: a step is a whole trace from emission to t_end; slice: --attempts per group")
    ap.add_argument("--t-end", type=float, default=None, help="end of the trace span [s] (default per workload)")
    ap.add_argument("--attempts", type=int, default=16, help="--span slice: RK45 attempts per group per step")
    ap.add_argument("--form", default="fp64", choices=["fp64", "mixed"],
                    help="arithmetic of the chosen form (fp64: the only form within 1e-6 on the whole C1 trace)")
    ap.add_argument("--far-rule", default="adaptive", choices=["reference", "adaptive"],
                    help="far-field quadrature of the BEM sum (adaptive: whole-segment Gauss-4/2 when distant)")
    ap.add_argument("--cta-threads", type=int, default=0, help="CTA width (0: autotuned, or the library's choice)")
    ap.add_argument("--team", default="auto", choices=list(TEAMS),
                    help="one group per warp (groups <= 32, float64 + adaptive rule) or per CTA; auto: autotuned "
                         "where both are offered, else the library's choice")
    ap.add_argument("--bins", action="store_true",
                    help="size-binned scheduling: one launch per group-size bin on concurrent streams")
    ap.add_argument("--cpu-attempts", type=int, default=16)
    ap.add_argument("--groups", type=int, default=None, help="first N emission groups only (a smaller case)")
    ap.add_argument("--plain-groups", type=int, default=592,
                    help="groups traced by both forms for the ratio and the endpoint error")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-form and accuracy leg")
    ap.add_argument("--tune", dest="tune", action="store_true", default=True,
                    help="autotune the launch configuration first (untimed; the default)")
    ap.add_argument("--no-tune", dest="tune", action="store_false", help="time the default launch configuration")
    ap.add_argument("--kappa", type=float, default=0.0,
                    help="mixed form: conditioning bound above which float32 sums are redone in float64 (0: 16)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-image", action="store_true", help="skip the per-call BEM image-charge force leg")
    ap.add_argument("--no-sensitivity", action="store_true",
                    help="skip the perturbed plain run that measures the trajectories' own conditioning")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))

    if args.impl == "reference":
        return reference_arm(args, rank, world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args, span_t_max(args))

    if world > 1:
        import torch
        import datetime
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    r = run_gpu(args, rank, world)
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()
    if rank != 0:
        return 0
    t = load_traffic(args.workload, args.form, args.far_rule)
    mean_ms = 1e3 * r["t_total"] / args.steps
    fp64 = args.form == "fp64"
    span = (f"whole trace: every group from emission to t_end = {r['t_max']:.3g} s (integrator t_max), one launch "
            f"{'per size bin ' if args.bins else ''}per step, initial state restored untimed"
            if args.span == "trace" else f"slices of {args.attempts} attempts per group per step, continuing")
    line = dict(
        metric=METRIC, value=r["value"], unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup,
        ms_per_step=mean_ms, higher_is_better=True, scaling="weak", vs_baseline=None,
        dtype="f64" if fp64 else "f32+f64", data="synthetic (seeded samplers, workloads.py)",
        config=dict(r["config"], form=args.form, far_rule=args.far_rule, span=span, t_end=r["t_max"],
                    kappa_max=args.kappa or 16.0, autotuned=r["tuned"], size_binned=bool(args.bins),
                    cta_threads=(r["tuned"] or {}).get("cta_threads") or args.cta_threads or "library default",
                    team=r["team"],
                    parallelism=f"contiguous group ranges balanced by cost, {world} GPU(s)",
                    l2="flushed between steps (256 MiB write); each step timed alone with CUDA events"),
        live_particle_steps_per_s=r["live"],
        clocks=r["clocks"], gpu_launches=args.steps * r["launches_per_step"],
        roofline=dict(bound="fp64" if fp64 else "fp32", achieved=r["achieved"], peak=r["peak"], unit="TFLOP/s",
                      frac=(r["achieved"] / r["peak"]) if r["peak"] else None,
                      traffic=(t or {}).get("dram_bytes_per_launch"),
                      peak_source=("measured in-run: cuBLAS DGEMM 4096^3" if fp64 else
                                   "measured in-run: cuBLAS SGEMM 8192^3, TF32 off")
                      + " (no FP32/FP64 figure in the measured-peaks file)",
                      flop_model=f"{FLOP_PER_RING:g} FLOP/ring eval, {FLOP_PER_PAIR:g} FLOP/pair, "
                                 f"{FLOP_PER_CLUSTER:g} FLOP/cluster expansion (nominal)"),
        plain_fp64=r["plain"],
        accuracy=r["accuracy"],
        counters=r["counters"],
        e2e=r["e2e"],
        image_force=r["image_force"],
        cpu_baseline=cpu,
    )
    print(json.dumps(line))
    return 0


def reference_arm(args, rank, world):
    """The reference's algorithm for this path on the host cores (the NumPy
    oracle port, float64, the reference's quadrature), on the same workload
    and trace span (t_max = t_end): each step is a bounded sample -- the first
    `procs` groups, one per process, --cpu-attempts attempts each from
    emission.  Under torchrun only rank 0 runs."""
    if rank != 0:
        return 0
    t_max = span_t_max(args)
    wl = prepare_cpu(args.workload, t_max)
    procs, groups = cpu_sample(wl)
    total_steps, total_wall = 0, 0.0
    for _ in range(args.steps):
        value, steps, wall, _ = cpu_leg(procs, args.cpu_attempts, groups)
        total_steps += steps
        total_wall += wall
    value = total_steps / total_wall
    cpu = dict(value=value, unit=UNIT, cores=procs, kind="port",
               sample=f"per step the first {len(groups)} groups, {args.cpu_attempts} attempts each from emission "
                      f"toward t_max = {t_max:.3g} s, one group per process; {args.steps} steps, {total_steps} "
                      f"accepted particle-steps in {total_wall:.1f} s")
    line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps, warmup=0,
                ms_per_step=1e3 * total_wall / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f64", data="synthetic (seeded samplers, workloads.py)", impl="reference",
                config=dict(wl.get("config", {}), form="fp64 (reference algorithm, NumPy port)", t_end=t_max,
                            span=f"{args.cpu_attempts} attempts per group from emission (a bounded prefix of the "
                                 f"GPU arm's whole trace)"),
                cpu_baseline=cpu, e2e=dict(value=value, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
