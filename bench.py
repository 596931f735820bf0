"""Benchmark: accepted RK45 particle-steps per second of the photoemission
tracer's hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload c1|c0|c2|c3|c4] [--attempts A] [--form fp64|mixed]
                    [--far-rule reference|adaptive] [--no-tune]

The chosen form (the default): float32 + Kahan BEM and pair sums (float64
state, stage combination, error norm and controller, float64 for points
close to a ring and for ill-conditioned sums) with the adaptive far-field
rule, its launch configuration chosen first by the project's autotuner on a
sample of the workload (untimed; `--no-tune` keeps the defaults).  The plain form (float64,
the reference's quadrature) is timed in the same run on the same workload
(`plain_fp64`), and `accuracy` reports the chosen form's endpoint error
against it on a sample of groups traced to a fixed time.

Workload (default c1, the largest single-GPU configuration with a BEM
field): hemisphere R = 50 nm on a 5 um post, E = -1e6 V/m, 2000-panel BEM
capsule (64,000 far nodes), 4096 groups x 32 electrons, Coulomb + 3-image
forces, rtol 1e-9, atol 1e-12, z_max = 1 mm, seed 1.  Synthetic, seeded
inputs (workloads.py) stand in for a distgen distribution.

A step is one spt_trace call that advances every group by at most A
Dormand-Prince attempts, continuing from the state the previous step left
(the trace is cut into slices, the way a long run is checkpointed).  W warm-up
steps are followed by K timed steps; L2 is flushed (256 MiB write) between
steps and each step is timed alone with CUDA events on the launch stream.
value = accepted particle-steps (device counter: sum over accepted
group-steps of the group size) / summed step time.

N > 1 (torchrun): weak scaling -- every rank traces its own 4096 groups
(seed + rank); there is no data-path collective, only a barrier and a max
of the per-rank times.
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


# ---------------------------------------------------------------------------
# workloads

def build_workload(name, rank=0):
    """Returns dict(geometry, data, rtol, atol, t_max, z_max, label, config)."""
    from bem_b200 import geometry as bg
    from bem_b200 import workloads as w

    if name == "c0":
        geo = bg.FlatCathode(-1e7, z0=3e-9, kill_z_below=0.0)
        data = w.flat_c0(seed=0 + rank)
        return dict(geometry=geo, data=data, rtol=1e-8, atol=1e-12, t_max=w.default_t_max(-1e7, 1e-3, 1e-12),
                    z_max=1e-3, config=dict(workload="C0 flat cathode, 16 groups x 64, rtol 1e-8", groups=16,
                                            group_size=64, bem_panels=0))
    if name in ("c1", "c2", "c4"):
        geo = bg.PostTipBEMGeometry(-1e6, 50e-9, 5e-6, n_cap=100, n_wall=900, n_subdiv=8, z0=3e-9)
        if name == "c1":
            data = w.tip_c1(geo.profile, geo.sigma, seed=1 + rank)
            cfg = dict(workload="C1 hemisphere-on-post BEM tip, 4096 groups x 32, 2000 panels, rtol 1e-9",
                       groups=4096, group_size=32)
        elif name == "c2":
            data = w.tip_c2(seed=2 + rank)
            cfg = dict(workload="C2 post tip, 512 groups x 1024, 2000 panels", groups=512, group_size=1024)
        else:
            data = w.tip_c4(geo.profile, geo.sigma, seed=4 + rank)
            cfg = dict(workload="C4 post tip, 65536 groups of size logU[1,128]", groups=65536, group_size="1-128")
        cfg.update(bem_panels=geo.profile.shape[0] - 1, far_nodes=(geo.profile.shape[0] - 1) * 32)
        return dict(geometry=geo, data=data, rtol=1e-9, atol=1e-12, t_max=w.default_t_max(-1e6, 1e-3, 1e-12),
                    z_max=1e-3, config=cfg)
    if name == "c3":
        geo = bg.CylindricalWellBEMGeometry(-2.5e6, 2e-6, 1e-6, n_segments=3000)
        data = w.well_c3(seed=3 + rank)
        return dict(geometry=geo, data=data, rtol=1e-9, atol=1e-12, t_max=w.default_t_max(-2.5e6, 2e-3, 10e-12),
                    z_max=2e-3, config=dict(workload="C3 cylindrical well, 65536 groups of size logU[1,256]",
                                            groups=65536, group_size="1-256", bem_panels=geo.profile.shape[0] - 1))
    raise ValueError(name)


def first_groups(data, n):
    """The workload cut to its first n emission groups (a smaller case of the
    same kernel, for profiling)."""
    sizes = np.asarray(data["group_sizes"])
    if n is None or n >= len(sizes):
        return data
    k = int(sizes[:n].sum())
    out = {key: (v[:k] if isinstance(v, np.ndarray) and v.shape[:1] == (int(sizes.sum()),) else v) for key, v in data.items()}
    out["group_sizes"] = sizes[:n]
    return out


def particle_arrays(data):
    from bem_b200.constants import ELEMENTARY_CHARGE, SPEED_OF_LIGHT, ev_to_kg
    m = ev_to_kg(510998.95069)
    pos = np.stack([data["x"], data["y"], data["z"]], -1)
    vel = np.stack([data["px"], data["py"], data["pz"]], -1) * ELEMENTARY_CHARGE / SPEED_OF_LIGHT / m
    n = len(pos)
    return pos, vel, data["t"], np.full(n, -ELEMENTARY_CHARGE), np.full(n, m), -ELEMENTARY_CHARGE / m


# ---------------------------------------------------------------------------
# CPU leg (oracle port; spawn pool, started before any CUDA use)

def _cpu_job(args):
    name, g, attempts = args
    import numpy as _np
    from oracle import geometry as ogeo
    from oracle import rk45 as ork
    wl = build_workload_cpu(name)
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
    return int(_np.sum(log[0][2])) * E, len(log[0][0]), dt


_CPU_CACHE = {}


def build_workload_cpu(name):
    """Same workload as build_workload, with the BEM solution taken from the
    cached device solve (the CPU leg never solves)."""
    if name in _CPU_CACHE:
        return _CPU_CACHE[name]
    blob = np.load(os.environ["SPT_BENCH_CPU_BLOB"], allow_pickle=True)
    wl = blob["wl"].item()
    _CPU_CACHE[name] = wl
    return wl


def cpu_leg(name, n_procs, attempts, groups):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(n_procs) as pool:
        res = pool.map(_cpu_job, [(name, g, attempts) for g in groups])
    wall = time.perf_counter() - t0
    steps = sum(r[0] for r in res)
    return steps / wall, steps, wall, sum(r[1] for r in res)


def prepare_cpu_blob(name, wl):
    spec = wl["geometry"].spec()
    d = {k: v for k, v in wl["data"].items()}
    blob = dict(spec=spec, data=d, rtol=wl["rtol"], atol=wl["atol"], t_max=wl["t_max"], z_max=wl["z_max"],
                config=wl["config"])
    import tempfile
    path = os.path.join(tempfile.gettempdir(), f"spt_bench_cpu_{name}_{os.getpid()}.npz")
    np.savez(path, wl=np.array(blob, dtype=object))
    os.environ["SPT_BENCH_CPU_BLOB"] = path
    return path


def physical_cores():
    """Worker processes for the CPU legs: the physical cores, at most 64, and
    no more than the available host memory allows at ~1 GiB per worker (a
    worker's float64 ring-sum temporaries over 64,000 nodes)."""
    n = os.cpu_count() or 1
    try:
        import psutil
        n = psutil.cpu_count(logical=False) or n
        n = min(n, max(1, int(psutil.virtual_memory().available / 2**30) // 2))
    except Exception:
        pass
    return max(1, min(n, 64))


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

def fp64_peak_tflops(torch, dev):
    """Measured float64 GEMM rate (cuBLAS DGEMM, 4096^3, best of 5): the
    FP64 denominator, since the driver's peak file has no FP64 figure."""
    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
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


def fp32_peak_tflops(torch, dev, n=8192):
    """Float32 CUDA-core peak measured in-run: a float32 GEMM with TF32 off."""
    old = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        a = torch.randn(n, n, dtype=torch.float32, device=dev)
        b = torch.randn(n, n, dtype=torch.float32, device=dev)
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
    finally:
        torch.backends.cuda.matmul.allow_tf32 = old


def combine_ranks(t_total, particle_steps, world, device):
    """Whole-job numbers of a weak-scaling run: the slowest rank's timed
    region (max) and the particle-steps of all ranks (sum), by collectives
    on the initialised process group (NCCL on the GPU path; any backend)."""
    if world == 1:
        return float(t_total), float(particle_steps)
    import torch
    import torch.distributed as dist
    tt = torch.tensor([float(t_total)], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    st = torch.tensor([float(particle_steps)], dtype=torch.float64, device=device)
    dist.all_reduce(st)
    return float(tt.item()), float(st.item())


def run_gpu(args, rank, world):
    import torch
    from bem_b200 import engine

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    wl = build_workload(args.workload, rank)
    if args.groups:
        wl["data"] = first_groups(wl["data"], args.groups)
        wl["config"] = dict(wl["config"], groups=args.groups, workload=wl["config"]["workload"] + f" (first {args.groups} groups)")
    pos, vel, tb, q, m, cm = particle_arrays(wl["data"])
    sizes = wl["data"]["group_sizes"]
    tracer = engine.Tracer(wl["geometry"], device=dev, form=args.form, z_max=wl["z_max"], far_rule=args.far_rule)
    tracer.kappa_max = args.kappa
    batch = engine.GroupBatch(pos, vel, tb, q, m, sizes, device=dev)
    tuned = None
    if args.tune:
        # launch configuration chosen by the project's autotuner on a sample of this workload (untimed)
        from bem_b200 import autotune
        t0 = time.perf_counter()
        res = autotune.tune(tracer, pos, vel, tb, q, m, sizes, wl["t_max"], wl["rtol"], wl["atol"], 1e-12, cm)
        autotune.apply(res, tracer, batch)
        tracer.tuned_order = res["order"]
        args.tuned_config = res
        tuned = dict(res, seconds=round(time.perf_counter() - t0, 2), sample_groups=res.get("sample_groups"),
                     timings={k: (round(v) if isinstance(v, float) else v) for k, v in res.get("timings", {}).items()})
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    prm = lambda: tracer.params(wl["t_max"], wl["rtol"], wl["atol"], 1e-12, cm, args.attempts)

    for _ in range(args.warmup):
        tracer.launch(batch, prm(), stream)
    torch.cuda.synchronize()

    c0 = tracer.counter_dict()
    times = []
    with ClockSampler(dev.index) as clk:
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush.fill_(1.0)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            tracer.launch(batch, prm(), stream)
            e.record(stream)
            e.synchronize()
            times.append(s.elapsed_time(e) * 1e-3)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
    c1 = tracer.counter_dict()
    dc = {k: c1[k] - c0[k] for k in c1}
    t_total = float(np.sum(times))
    t_max_ranks, steps_all = combine_ranks(t_total, dc["particle_steps"], world, dev)

    # end-to-end leg: host (pinned) state in, host state out, every step
    e2e = None
    if rank == 0 and not args.no_e2e:
        e2e = e2e_leg(args, wl, tracer, pos, vel, tb, q, m, cm, sizes, dev)

    plain = None
    acc = None
    if rank == 0 and not args.no_plain and (args.form, args.far_rule) != ("fp64", "reference"):
        plain = plain_leg(args, wl, pos, vel, tb, q, m, cm, sizes, dev)
    if rank == 0 and not args.no_accuracy and (args.form, args.far_rule) != ("fp64", "reference"):
        acc = accuracy_leg(args, wl, pos, vel, tb, q, m, cm, sizes, dev)
    peak = (fp64_peak_tflops if args.form == "fp64" else fp32_peak_tflops)(torch, dev) if rank == 0 else None
    flops = dc["ring_far"] * FLOP_PER_RING + dc["ring_near"] * FLOP_PER_RING + dc["pair_evals"] * FLOP_PER_PAIR
    achieved = flops / t_total / 1e12
    return dict(value=steps_all / t_max_ranks, t_total=t_max_ranks, times=times, counters=dc, clocks=clk.summary(),
                e2e=e2e, peak=peak, achieved=achieved, config=wl["config"], wl=wl, plain=plain, accuracy=acc,
                tuned=tuned)


def plain_leg(args, wl, pos, vel, tb, q, m, cm, sizes, dev):
    """The plain form (float64, the reference's far quadrature) on the same
    workload: the same W warm-up and K timed steps, CUDA events."""
    import torch
    from bem_b200 import engine

    tracer = engine.Tracer(wl["geometry"], device=dev, form="fp64", z_max=wl["z_max"], far_rule="reference")
    batch = engine.GroupBatch(pos, vel, tb, q, m, sizes, device=dev)
    stream = torch.cuda.current_stream(dev)
    prm = lambda: tracer.params(wl["t_max"], wl["rtol"], wl["atol"], 1e-12, cm, args.attempts)
    for _ in range(args.warmup):
        tracer.launch(batch, prm(), stream)
    torch.cuda.synchronize()
    c0 = tracer.counter_dict()
    t = 0.0
    for _ in range(args.steps):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        tracer.launch(batch, prm(), stream)
        e.record(stream)
        e.synchronize()
        t += s.elapsed_time(e) * 1e-3
    steps = tracer.counter_dict()["particle_steps"] - c0["particle_steps"]
    return dict(value=steps / t, unit=UNIT, ms_per_step=1e3 * t / args.steps, form="fp64", far_rule="reference")


def accuracy_leg(args, wl, pos, vel, tb, q, m, cm, sizes, dev):
    """Endpoint error of the chosen form against the plain form: the first
    `acc_groups` groups traced to t_end = acc_time by both (a fixed end time,
    so no endpoint depends on which step crossed z_max).  Particles alive at
    t_end: |dx| / |x| and |dv| / |v| of the plain endpoint.  Particles that
    returned to the emitter keep the state of the step that landed inside it,
    which moves with the step sequence: they are compared by death time."""
    import torch
    from bem_b200 import engine

    n = min(args.acc_groups, len(sizes))
    k = int(np.sum(sizes[:n]))
    out = {}
    for form, rule in (("fp64", "reference"), (args.form, args.far_rule)):
        tracer = engine.Tracer(wl["geometry"], device=dev, form=form, z_max=wl["z_max"], far_rule=rule)
        tracer.kappa_max = args.kappa
        batch = engine.GroupBatch(pos[:k], vel[:k], tb[:k], q[:k], m[:k], sizes[:n], device=dev)
        if (form, rule) == (args.form, args.far_rule) and getattr(args, "tuned_config", None):
            from bem_b200 import autotune
            autotune.apply(args.tuned_config, tracer, batch)  # the chosen form as timed
        tracer.run(batch, args.acc_time, wl["rtol"], wl["atol"], 1e-12, cm)
        torch.cuda.synchronize()
        c = tracer.counter_dict()
        out[form, rule] = (batch.positions().cpu().numpy(), batch.velocities().cpu().numpy(),
                           batch.t_death.cpu().numpy(), c["attempts"], c["accepted"])
    (p0, v0, d0, a0, s0), (p1, v1, d1, a1, s1) = out[("fp64", "reference")], out[(args.form, args.far_rule)]
    alive = ~np.isfinite(d0) & ~np.isfinite(d1)
    dead = np.isfinite(d0) & np.isfinite(d1)
    ex = np.linalg.norm(p1 - p0, axis=-1)[alive] / np.linalg.norm(p0, axis=-1)[alive]
    ev = np.linalg.norm(v1 - v0, axis=-1)[alive] / np.linalg.norm(v0, axis=-1)[alive]
    et = np.abs(d1[dead] - d0[dead]) / d0[dead]
    return dict(groups=n, particles=k, t_end=args.acc_time, against="plain fp64 (reference quadrature) on the GPU",
                alive=int(alive.sum()), max_rel_pos=float(ex.max()), median_rel_pos=float(np.median(ex)),
                max_rel_vel=float(ev.max()), median_rel_vel=float(np.median(ev)),
                killed=int(dead.sum()), killed_in_one_only=int((np.isfinite(d0) != np.isfinite(d1)).sum()),
                max_rel_t_death=float(et.max()) if et.size else None,
                attempts_plain=int(a0), attempts_chosen=int(a1), accepted_steps_ratio=float(s1 / s0))


def e2e_leg(args, wl, tracer, pos, vel, tb, q, m, cm, sizes, dev):
    """Same slices through the public API with the state in pinned host
    memory: H2D of the step's state, spt_trace, D2H of the new state."""
    import torch
    from bem_b200 import engine

    batch = engine.GroupBatch(pos, vel, tb, q, m, sizes, device=dev)
    if getattr(tracer, "tuned_order", None):
        batch.set_order(tracer.tuned_order)
    names = ["x", "y", "z", "vx", "vy", "vz", "t_death", "t", "h", "status", "n_accepted", "n_rejected"]
    host = {k: torch.empty_like(getattr(batch, k), device="cpu").pin_memory() for k in names}
    for k in names:
        host[k].copy_(getattr(batch, k))
    stream = torch.cuda.current_stream(dev)
    prm = lambda: tracer.params(wl["t_max"], wl["rtol"], wl["atol"], 1e-12, cm, args.attempts)
    for _ in range(args.warmup):
        tracer.launch(batch, prm(), stream)
    torch.cuda.synchronize()
    for k in names:
        host[k].copy_(getattr(batch, k))
    h2d = sum(host[k].numel() * host[k].element_size() for k in names)
    c0 = tracer.counter_dict()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for k in names:
            getattr(batch, k).copy_(host[k], non_blocking=True)
        tracer.launch(batch, prm(), stream)
        for k in names:
            host[k].copy_(getattr(batch, k), non_blocking=True)
        stream.synchronize()
    wall = time.perf_counter() - t0
    c1 = tracer.counter_dict()
    steps = c1["particle_steps"] - c0["particle_steps"]
    return dict(value=steps / wall, unit=UNIT, h2d_bytes_per_step=int(h2d), d2h_bytes_per_step=int(h2d))


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
    ap.add_argument("--attempts", type=int, default=16, help="RK45 attempts per group per step")
    ap.add_argument("--form", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--far-rule", default="adaptive", choices=["reference", "adaptive"],
                    help="far-field quadrature of the BEM sum (adaptive: whole-segment Gauss-4/2 when distant)")
    ap.add_argument("--cpu-attempts", type=int, default=16)
    ap.add_argument("--groups", type=int, default=None, help="first N emission groups only (profiling a smaller case)")
    ap.add_argument("--no-plain", action="store_true", help="skip timing the plain form beside the chosen one")
    ap.add_argument("--tune", dest="tune", action="store_true", default=True,
                    help="autotune the launch configuration first (untimed; the default)")
    ap.add_argument("--no-tune", dest="tune", action="store_false", help="time the default launch configuration")
    ap.add_argument("--kappa", type=float, default=0.0,
                    help="mixed form: conditioning bound above which float32 sums are redone in float64 (0: 16)")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the endpoint-error leg")
    ap.add_argument("--acc-groups", type=int, default=64)
    ap.add_argument("--acc-time", type=float, default=20e-12, help="end time of the endpoint-error traces [s]")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))

    if args.impl == "reference":
        return reference_arm(args, rank, world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args)

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
    plain = r["plain"]
    if plain is not None:
        plain = dict(plain, ratio=r["value"] / plain["value"])
    line = dict(
        metric=METRIC, value=r["value"], unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup,
        ms_per_step=mean_ms, higher_is_better=True, scaling="weak", vs_baseline=None,
        dtype="f64" if fp64 else "f32+f64", data="synthetic (seeded samplers, workloads.py)",
        config=dict(r["config"], form=args.form, far_rule=args.far_rule, attempts_per_step=args.attempts,
                    kappa_max=args.kappa or 16.0, autotuned=r["tuned"],
                    parallelism=f"groups x {world} GPUs",
                    l2="flushed between steps (256 MiB write); each step timed alone with CUDA events"),
        clocks=r["clocks"], gpu_launches=args.steps,
        roofline=dict(bound="fp64" if fp64 else "fp32", achieved=r["achieved"], peak=r["peak"], unit="TFLOP/s",
                      frac=(r["achieved"] / r["peak"]) if r["peak"] else None,
                      traffic=(t or {}).get("dram_bytes_per_launch"),
                      peak_source=("measured in-run: cuBLAS DGEMM 4096^3" if fp64 else
                                   "measured in-run: cuBLAS SGEMM 8192^3, TF32 off")
                      + " (the driver's peak file has HBM and BF16 figures only)",
                      flop_model=f"{FLOP_PER_RING:g} FLOP/ring eval, {FLOP_PER_PAIR:g} FLOP/pair (nominal)"),
        plain_fp64=plain,
        accuracy=r["accuracy"],
        counters=r["counters"],
        e2e=r["e2e"],
        cpu_baseline=cpu,
    )
    print(json.dumps(line))
    return 0


def cpu_baseline(args, for_reference=False):
    """The oracle port on the host cores, on a bounded sample of the same
    workload: `procs` groups (one per process) for --cpu-attempts attempts each
    from the initial state."""
    wl = build_workload_cpu_side(args.workload)
    procs = min(physical_cores(), 64)
    n_groups = len(wl["data"]["group_sizes"])
    groups = list(range(min(procs, n_groups)))
    value, steps, wall, attempts = cpu_leg(args.workload, procs, args.cpu_attempts, groups)
    return dict(value=value, unit=UNIT, cores=procs, kind="port",
                sample=f"{len(groups)} groups x {args.cpu_attempts} attempts from emission, one group per process "
                       f"({steps} accepted particle-steps in {wall:.1f} s)")


def build_workload_cpu_side(name):
    """Build the workload for the CPU leg without touching CUDA for the
    non-BEM case; BEM workloads need the device solve, done in a child
    process so this process stays CUDA-free for the spawn pool."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        path = pool.apply(_make_blob, (name,))
    os.environ["SPT_BENCH_CPU_BLOB"] = path
    return build_workload_cpu(name)


def _make_blob(name):
    wl = build_workload(name)
    return prepare_cpu_blob(name, wl)


def reference_arm(args, rank, world):
    """The reference's algorithm for this path on the host cores (the NumPy
    oracle port, float64, the reference's quadrature), on the same workload:
    each step is a bounded sample -- one group per process, --cpu-attempts
    attempts from emission.  Under torchrun only rank 0 runs."""
    if rank != 0:
        return 0
    wl = build_workload_cpu_side(args.workload)
    procs = min(physical_cores(), 64)
    groups = list(range(min(procs, len(wl["data"]["group_sizes"]))))
    total_steps, total_wall = 0, 0.0
    for _ in range(args.steps):
        value, steps, wall, _ = cpu_leg(args.workload, procs, args.cpu_attempts, groups)
        total_steps += steps
        total_wall += wall
    value = total_steps / total_wall
    cpu = dict(value=value, unit=UNIT, cores=procs, kind="port",
               sample=f"per step {len(groups)} groups x {args.cpu_attempts} attempts from emission, one group per "
                      f"process; {args.steps} steps, {total_steps} accepted particle-steps in {total_wall:.1f} s")
    line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps, warmup=0,
                ms_per_step=1e3 * total_wall / args.steps, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="f64", data="synthetic (seeded samplers, workloads.py)", impl="reference",
                config=dict(wl.get("config", {}), form="fp64 (reference algorithm, NumPy port)",
                            attempts_per_step=args.cpu_attempts),
                cpu_baseline=cpu, e2e=dict(value=value, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
