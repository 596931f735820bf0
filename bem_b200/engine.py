"""Device-resident trace driver over the C ABI (spt_trace).

``GroupBatch`` holds the structure-of-arrays particle state and per-group
integrator state in torch CUDA tensors (torch is only the allocator and
stream here; all arithmetic is in the CUDA library).  ``integrate`` is the
drop-in for batched_rk45.integrate (batched_rk45.py:55-323): it advances
every group with its own t and h until t >= t_max, with the same stopping
rule, birth checkpoints, kill-after-accept and step-size controller, but as
one persistent kernel per call instead of a Python loop with host syncs.
"""

import ctypes

import numpy as np

from . import _lib
from .constants import COULOMB_CONSTANT

DEFAULT_ATTEMPT_CHUNK = 4096  # attempts per group per launch; the host loops until every group is done
DEFAULT_BINS = ((8, 64), (64, 128), (1024, 256))  # (largest group size, CTA width) of size-binned launches


def _torch():
    import torch
    return torch


def _as_dev(a, dtype, device):
    torch = _torch()
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=device)


class GroupBatch:
    """Flat SoA particle arrays with group offsets, plus group clocks."""

    def __init__(self, pos, vel, t_birth, charge, mass, group_sizes, device="cuda", order="largest_first"):
        torch = _torch()
        f64 = torch.float64
        pos = np.asarray(pos, dtype=np.float64) if not isinstance(pos, torch.Tensor) else pos
        sizes = np.asarray(group_sizes, dtype=np.int64)
        if np.any(sizes < 1):
            raise ValueError("every group needs at least one particle")
        n = int(sizes.sum())
        if pos.shape != (n, 3):
            raise ValueError(f"pos must be ({n}, 3) for these group sizes, got {tuple(pos.shape)}")
        if sizes.max() > 1024:
            raise ValueError("groups larger than 1024 particles are not supported")
        self.device = torch.device(device)
        self.n_groups = len(sizes)
        self.n_particles = n
        self.sizes = sizes
        self.max_group_size = int(sizes.max())
        offs = np.zeros(len(sizes) + 1, dtype=np.int64)
        np.cumsum(sizes, out=offs[1:])
        self.offsets_host = offs
        d = self.device
        self.offsets = torch.as_tensor(offs, device=d)
        if order == "largest_first":
            perm = np.argsort(-sizes, kind="stable").astype(np.int32)
            self.order = torch.as_tensor(perm, device=d)
        else:
            self.order = None
        p = _as_dev(pos, f64, d)
        v = _as_dev(vel, f64, d)
        self.x, self.y, self.z = (p[:, k].contiguous() for k in range(3))
        self.vx, self.vy, self.vz = (v[:, k].contiguous() for k in range(3))
        self.t_birth = _as_dev(t_birth, f64, d).reshape(-1)
        self.charge = _as_dev(charge, f64, d).reshape(-1)
        self.mass = _as_dev(mass, f64, d).reshape(-1)
        self.live = None       # compacted processing order (enable_compaction)
        self.n_active = None
        self.t_death = torch.full((n,), float("inf"), dtype=f64, device=d)
        G = self.n_groups
        self.t = torch.zeros(G, dtype=f64, device=d)
        self.h = torch.zeros(G, dtype=f64, device=d)
        self.status = torch.zeros(G, dtype=torch.int32, device=d)
        self.n_accepted = torch.zeros(G, dtype=torch.int64, device=d)
        self.n_rejected = torch.zeros(G, dtype=torch.int64, device=d)

    STATE = ("x", "y", "z", "vx", "vy", "vz", "t_death", "t", "h", "status", "n_accepted", "n_rejected")

    def copy_state_from(self, other):
        """Copy the evolving state (positions, velocities, deaths, group
        clocks and counts) of a batch with the same groups."""
        for k in self.STATE:
            getattr(self, k).copy_(getattr(other, k))

    def set_order(self, order):
        """Processing order: "largest_first" or "given" (group index order)."""
        torch = _torch()
        if order == "largest_first":
            perm = np.argsort(-self.sizes, kind="stable").astype(np.int32)
            self.order = torch.as_tensor(perm, device=self.device)
        elif order == "given":
            self.order = None
        else:
            raise ValueError(order)
        self.live = None
        self.n_active = None

    def enable_compaction(self):
        """Process only the running groups: `compact()` (on the device, no
        host sync) rebuilds the processing order from the statuses."""
        torch = _torch()
        if self.live is None:
            base = self.order if self.order is not None else torch.arange(self.n_groups, dtype=torch.int32,
                                                                          device=self.device)
            self.live = base.clone()
            self.n_active = torch.full((1,), self.n_groups, dtype=torch.int32, device=self.device)

    def compact(self, stream=None):
        """spt_compact_groups on `stream`: live = the running groups of the
        processing order, n_active = their number."""
        torch = _torch()
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        base = self.order.data_ptr() if self.order is not None else None
        _lib.check(_lib.lib().spt_compact_groups(base, self.n_groups, self.status.data_ptr(), self.live.data_ptr(),
                                                 self.n_active.data_ptr(), ctypes.c_void_p(stream.cuda_stream)),
                   "spt_compact_groups")

    def bin_plan(self, bins=None):
        """Size-binned scheduling: the groups split by size into bins, each
        traced by its own launch with its own CTA width (Tracer.launch_binned).
        bins: ((largest group size, CTA width), ...) ascending; the default
        puts groups of 1-8 particles on 64-thread CTAs, 9-64 on 128, larger
        on 256.  Returns one entry per non-empty bin: the device order of its
        groups (largest first), their count and largest size, the CTA width,
        and the bin's share of the estimated work (partition.group_cost)."""
        torch = _torch()
        from .partition import group_cost
        bins = DEFAULT_BINS if bins is None else bins
        cost = group_cost(self.sizes)
        total = float(cost.sum())
        plan, lo = [], 0
        for hi, threads in bins:
            idx = np.nonzero((self.sizes > lo) & (self.sizes <= hi))[0]
            lo = hi
            if len(idx) == 0:
                continue
            idx = idx[np.argsort(-self.sizes[idx], kind="stable")].astype(np.int32)
            plan.append(dict(order=torch.as_tensor(idx, device=self.device), n=len(idx),
                             max_size=int(self.sizes[idx].max()), threads=int(threads),
                             share=float(cost[idx].sum()) / total))
        if sum(b["n"] for b in plan) != self.n_groups:
            raise ValueError("the bins do not cover every group size")
        return plan

    def struct(self):
        s = _lib.SptState()
        s.n_groups = self.n_groups
        s.max_group_size = self.max_group_size
        s.n_particles = self.n_particles
        P = lambda t: None if t is None else t.data_ptr()
        s.group_offset = P(self.offsets)
        s.group_order = P(self.order)
        if self.live is not None:
            s.group_order = P(self.live)
            s.n_active = P(self.n_active)
        s.x, s.y, s.z = P(self.x), P(self.y), P(self.z)
        s.vx, s.vy, s.vz = P(self.vx), P(self.vy), P(self.vz)
        s.t_birth, s.t_death = P(self.t_birth), P(self.t_death)
        s.charge, s.mass = P(self.charge), P(self.mass)
        s.t, s.h, s.status = P(self.t), P(self.h), P(self.status)
        s.n_accepted, s.n_rejected = P(self.n_accepted), P(self.n_rejected)
        return s

    def positions(self):
        torch = _torch()
        return torch.stack([self.x, self.y, self.z], dim=-1)

    def velocities(self):
        torch = _torch()
        return torch.stack([self.vx, self.vy, self.vz], dim=-1)


FORMS = {"fp64": _lib.FORM_FP64, "mixed": _lib.FORM_MIXED, "surrogate": _lib.FORM_SURROGATE}


class Tracer:
    """Persistent-kernel RK45 tracer for one geometry on one device."""

    def __init__(self, geometry, device="cuda", form="fp64", z_max=None, surrogate=None, band=5e-9, spot=0.01,
                 far_rule="reference", ratio4=None, ratio2=None, ratio_run=None):
        """form: "fp64" (plain), "mixed" (float32 + Kahan sums) or "surrogate"
        (mixed, with the learned field outside the `band` [m] around the
        surface, `spot` of the other points checked against the exact sum).
        far_rule: "reference" (every far segment on all its sub-panel nodes)
        or "adaptive" (whole-segment Gauss-4 / Gauss-2 for segments at least
        ratio4 / ratio2 lengths away, the 8-node run rule for flagged
        straight runs at least ratio_run run arclengths away)."""
        torch = _torch()
        self.geometry = geometry
        self.device = torch.device(device)
        self.form = FORMS[form] if isinstance(form, str) else int(form)
        self.z_max = z_max
        self.geom = geometry.to_struct(z_max=z_max)
        self.tables = geometry.bem_tables(self.device) if geometry.is_bem else None
        self.far_rule = far_rule
        self.round_points = 0  # far-sum points per round (0: the kernel's default, 4); see autotune
        self.cta_threads = 0   # CTA width, 32/64/128/256 (0: the library's choice by group size); see autotune
        self.kappa_max = 0.0   # mixed form's conditioning bound for float32 sums (0: the kernel's default, 16)
        self.team = _lib.TEAM_AUTO  # one group per warp where offered (TEAM_WARP), or per CTA (TEAM_CTA)
        self.bem = None
        if self.tables is not None:
            kw = {k: v for k, v in (("ratio4", ratio4), ("ratio2", ratio2), ("ratio_run", ratio_run)) if v is not None}
            self.bem = self.tables.view(far_rule, **kw)
        self._ws = None
        self.counters = torch.zeros(_lib.N_COUNTERS, dtype=torch.int64, device=self.device)
        self.surrogate = None
        if self.form == _lib.FORM_SURROGATE:
            if surrogate is None:
                raise ValueError("form='surrogate' needs a trained FieldSurrogate")
            self.surrogate = SurrogateBinding(surrogate, band, spot, self.device)

    def params(self, t_max, rtol, atol, plummer_radius, charge_to_mass, max_attempts, log=None,
               safety=0.9, min_factor=0.2, max_factor=10.0, initial_step_fraction=1e-6,
               coulomb_constant=COULOMB_CONSTANT, records=None, round_points=None, kappa_max=None, cta_threads=None,
               team=None):
        p = _lib.SptTraceParams()
        p.team = int(self.team if team is None else team)
        p.round_points = int(self.round_points if round_points is None else round_points)
        p.cta_threads = int(self.cta_threads if cta_threads is None else cta_threads)
        p.kappa_max = float(self.kappa_max if kappa_max is None else kappa_max)
        p.t_max, p.rtol, p.atol = float(t_max), float(rtol), float(atol)
        p.plummer_radius = float(plummer_radius)
        p.charge_to_mass = float(charge_to_mass)
        p.coulomb_constant = float(coulomb_constant)
        p.safety, p.min_factor, p.max_factor = float(safety), float(min_factor), float(max_factor)
        p.initial_step_fraction = float(initial_step_fraction)
        p.max_attempts = int(max_attempts)
        p.form = self.form
        if log is not None:
            p.log_capacity = log[0].shape[1]
            p.log_h = log[0].data_ptr()
            p.log_err = log[1].data_ptr()
        p.counters = self.counters.data_ptr()
        if records is not None:
            records.fill(p)
        if self.surrogate is not None:
            self.surrogate.fill(p)
        return p

    def surrogate_stats(self):
        return self.surrogate.stats()

    def workspace(self, state, params):
        torch = _torch()
        nbytes = ctypes.c_int64(0)
        bem = ctypes.byref(self.bem) if self.bem is not None else None
        _lib.check(_lib.lib().spt_trace_workspace_bytes(ctypes.byref(state), ctypes.byref(params),
                                                        ctypes.byref(self.geom), bem, ctypes.byref(nbytes)),
                   "spt_trace_workspace_bytes")
        need = max(int(nbytes.value), 256)
        if self._ws is None or self._ws.numel() < need:
            self._ws = torch.empty(need, dtype=torch.uint8, device=self.device)
        return self._ws

    def launch(self, batch, params, stream=None):
        """One spt_trace call (asynchronous on `stream`)."""
        torch = _torch()
        st = batch.struct()
        ws = self.workspace(st, params)
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        bem = ctypes.byref(self.bem) if self.bem is not None else None
        _lib.check(_lib.lib().spt_trace(ctypes.byref(st), ctypes.byref(params), ctypes.byref(self.geom), bem,
                                        ctypes.c_void_p(ws.data_ptr()), ws.numel(),
                                        ctypes.c_void_p(stream.cuda_stream)), "spt_trace")

    def launch_binned(self, batch, params, plan, stream=None):
        """One spt_trace launch per size bin of `plan` (GroupBatch.bin_plan),
        each on its own stream with its own CTA width and a persistent grid
        in proportion to its share of the work, so the bins run side by side
        and fill each other's tails.  The launches share the batch's arrays
        (disjoint groups) and are joined back into `stream`."""
        torch = _torch()
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        if not hasattr(self, "_bin_streams"):
            self._bin_streams, self._bin_ws = [], []
        while len(self._bin_streams) < len(plan):
            self._bin_streams.append(torch.cuda.Stream(self.device))
            self._bin_ws.append(None)
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        ready = torch.cuda.Event()
        ready.record(stream)
        bem = ctypes.byref(self.bem) if self.bem is not None else None
        for b, binfo in enumerate(plan):
            st = batch.struct()
            st.group_order = binfo["order"].data_ptr()
            st.n_active = None
            st.n_groups = binfo["n"]
            st.max_group_size = binfo["max_size"]
            p = _lib.SptTraceParams()
            ctypes.pointer(p)[0] = params
            p.cta_threads = binfo["threads"]
            full = sms * max(1, 65536 // (128 * binfo["threads"]))  # resident CTAs at 128 registers a thread
            p.max_ctas = max(1, int(np.ceil(full * binfo["share"])))
            nbytes = ctypes.c_int64(0)
            _lib.check(_lib.lib().spt_trace_workspace_bytes(ctypes.byref(st), ctypes.byref(p), ctypes.byref(self.geom),
                                                            bem, ctypes.byref(nbytes)), "spt_trace_workspace_bytes")
            need = max(int(nbytes.value), 256)
            if self._bin_ws[b] is None or self._bin_ws[b].numel() < need:
                self._bin_ws[b] = torch.empty(need, dtype=torch.uint8, device=self.device)
            ws = self._bin_ws[b]
            s = self._bin_streams[b]
            s.wait_event(ready)
            _lib.check(_lib.lib().spt_trace(ctypes.byref(st), ctypes.byref(p), ctypes.byref(self.geom), bem,
                                            ctypes.c_void_p(ws.data_ptr()), ws.numel(), ctypes.c_void_p(s.cuda_stream)),
                       "spt_trace")
            done = torch.cuda.Event()
            done.record(s)
            stream.wait_event(done)

    def run(self, batch, t_max, rtol, atol, plummer_radius, charge_to_mass, max_steps=10_000_000,
            attempt_chunk=DEFAULT_ATTEMPT_CHUNK, log_capacity=0, screens=None, output_times=None,
            screen_capacity=None, compact=False, graph=False, graph_launches=4, bins=None, **kw):
        """Integrate every group to t_max.  Raises RuntimeError when a group
        needs more than max_steps attempts (batched_rk45.py:320-321).

        bins: size-binned scheduling -- a GroupBatch.bin_plan (or True for the
        default bins): one launch per size bin on concurrent streams.

        With `screens` (z planes) and/or `output_times`, returns a
        TraceRecords holding every crossing and every output-time snapshot;
        otherwise returns the attempt log (or None).

        compact: before every launch, retired groups are dropped from the
        processing order on the device (spt_compact_groups).  graph (implies
        compact): `graph_launches` x [compact, spt_trace of attempt_chunk
        attempts] are captured once as a CUDA graph and replayed, the host
        checking the statuses once per replay."""
        torch = _torch()
        if graph:
            if screens or output_times is not None or log_capacity:
                raise ValueError("graph=True records neither screens, output times nor attempt logs")
            return self._run_graph(batch, t_max, rtol, atol, plummer_radius, charge_to_mass, max_steps,
                                   attempt_chunk, graph_launches, **kw)
        plan = None
        if bins is not None and bins is not False:
            if compact:
                raise ValueError("size-binned launches take their own group orders; compact=False")
            plan = batch.bin_plan() if bins is True else bins
        if compact:
            batch.enable_compaction()
        records = None
        if screens or output_times is not None:
            records = TraceRecords(batch, screens or [], output_times, self.device, screen_capacity)
            kw["records"] = records
        log = None
        if log_capacity:
            log = (torch.full((batch.n_groups, log_capacity), float("nan"), dtype=torch.float64, device=self.device),
                   torch.full((batch.n_groups, log_capacity), float("nan"), dtype=torch.float64, device=self.device))
        done_attempts = 0
        while True:
            chunk = min(attempt_chunk, max_steps - done_attempts)
            if chunk <= 0:
                raise RuntimeError(f"batched RK45 did not converge within {max_steps} steps")
            p = self.params(t_max, rtol, atol, plummer_radius, charge_to_mass, chunk, log=log, **kw)
            if compact:
                batch.compact()
            if plan is not None:
                self.launch_binned(batch, p, plan)
            else:
                self.launch(batch, p)
            done_attempts += chunk
            if records is not None:
                records.collect()
            if self._check_done(batch):
                break
        return records if records is not None else log

    @staticmethod
    def _check_done(batch):
        status = batch.status.cpu().numpy()
        bad = np.isin(status, [_lib.GROUP_NONFINITE, _lib.GROUP_TIMEOUT])
        if np.any(bad):
            g = int(np.nonzero(bad)[0][0])
            raise RuntimeError(f"group {g} stopped with status {int(status[g])} "
                               f"({'non-finite error norm' if status[g] == _lib.GROUP_NONFINITE else 'device wait timeout'})")
        return bool(np.all(status == _lib.GROUP_DONE))

    def _run_graph(self, batch, t_max, rtol, atol, plummer_radius, charge_to_mass, max_steps, attempt_chunk,
                   graph_launches, **kw):
        torch = _torch()
        batch.enable_compaction()
        chunk = min(attempt_chunk, max_steps)
        p = self.params(t_max, rtol, atol, plummer_radius, charge_to_mass, chunk, **kw)
        # one eager chunk first: sizes the workspace and sets the kernel attributes outside the capture
        batch.compact()
        self.launch(batch, p)
        done_attempts = chunk
        if self._check_done(batch):
            return None
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, capture_error_mode="thread_local"):
            for _ in range(graph_launches):
                batch.compact()
                self.launch(batch, p)
        self._graph = g  # kept alive with its parameter blocks
        while True:
            if done_attempts + graph_launches * chunk <= max_steps:
                g.replay()
                done_attempts += graph_launches * chunk
            else:
                # the last attempts before max_steps: eager launches, never past it
                rest = min(chunk, max_steps - done_attempts)
                if rest <= 0:
                    raise RuntimeError(f"batched RK45 did not converge within {max_steps} steps")
                batch.compact()
                self.launch(batch, self.params(t_max, rtol, atol, plummer_radius, charge_to_mass, rest, **kw))
                done_attempts += rest
            if self._check_done(batch):
                return None

    def counter_dict(self):
        c = self.counters.cpu().numpy().astype(np.uint64)
        return {k: int(v) for k, v in zip(_lib.COUNTERS, c)}


class TraceRecords:
    """Device buffers for screen crossings and output-time snapshots, and
    their host copies (screens.py:18-40, trajectories.py:16-41)."""

    def __init__(self, batch, screens, output_times, device, screen_capacity=None):
        torch = _torch()
        self.batch = batch
        self.screens = [float(z) for z in screens]
        n = batch.n_particles
        ns = len(self.screens)
        self.capacity = int(screen_capacity or (8 * n * max(ns, 1) + 4096))
        f64 = torch.float64
        self.screen_z = torch.as_tensor(np.asarray(self.screens, dtype=np.float64), device=device) if ns else None
        self.screen_rec = torch.empty((9, self.capacity), dtype=f64, device=device) if ns else None
        self.screen_count = torch.zeros(1, dtype=torch.int64, device=device)
        self.chunks = []
        if output_times is not None:
            self.output_times = np.sort(np.asarray(output_times, dtype=np.float64))
            no = len(self.output_times)
            self.out_t = torch.as_tensor(self.output_times, device=device)
            self.out_rec = torch.zeros((no, 7, n), dtype=f64, device=device)
            self.out_flag = torch.zeros((no, n), dtype=torch.uint8, device=device)
        else:
            self.output_times = None

    def fill(self, p):
        if self.screens:
            p.n_screens = len(self.screens)
            p.screens = self.screen_z.data_ptr()
            p.screen_rec = self.screen_rec.data_ptr()
            p.screen_capacity = self.capacity
            p.screen_count = self.screen_count.data_ptr()
        if self.output_times is not None and len(self.output_times):
            p.n_outputs = len(self.output_times)
            p.output_times = self.out_t.data_ptr()
            p.output_rec = self.out_rec.data_ptr()
            p.output_flag = self.out_flag.data_ptr()

    def collect(self):
        """Move this launch's crossings to the host and reset the counter."""
        if not self.screens:
            return
        n = int(self.screen_count.item())
        if n > self.capacity:
            raise RuntimeError(f"{n} screen crossings in one launch exceed the record buffer ({self.capacity}); "
                               "pass a larger screen_capacity")
        if n:
            self.chunks.append(self.screen_rec[:, :n].cpu().numpy())
        self.screen_count.zero_()

    def screen_records(self):
        """One dict of arrays per screen, in the order found (or None)."""
        allr = np.concatenate(self.chunks, axis=1) if self.chunks else np.zeros((9, 0))
        out = []
        for k in range(len(self.screens)):
            r = allr[:, allr[7] == k]
            if r.shape[1] == 0:
                out.append(None)
                continue
            out.append(dict(t=r[0], x=r[1], y=r[2], z=r[3], vx=r[4], vy=r[5], vz=r[6],
                            particle=r[8].astype(np.int64)))
        return out

    def output_records(self):
        """One dict of arrays per output time: every particle born by then."""
        if self.output_times is None:
            return []
        rec = self.out_rec.cpu().numpy()
        flag = self.out_flag.cpu().numpy().astype(bool)
        out = []
        for k in range(len(self.output_times)):
            idx = np.nonzero(flag[k])[0]
            if len(idx) == 0:
                out.append(None)
                continue
            r = rec[k][:, idx]
            out.append(dict(t=r[0], x=r[1], y=r[2], z=r[3], vx=r[4], vy=r[5], vz=r[6], particle=idx))
        return out


def accel(geometry, pos, active, charge, mass, group_sizes, charge_to_mass, plummer_radius, device="cuda",
          form="fp64", coulomb_constant=COULOMB_CONSTANT, far_rule="reference"):
    """One stage evaluation through spt_accel; returns acc [N, 3] (torch)."""
    torch = _torch()
    sizes = np.asarray(group_sizes, dtype=np.int64)
    offs = np.zeros(len(sizes) + 1, dtype=np.int64)
    np.cumsum(sizes, out=offs[1:])
    d = torch.device(device)
    p = _as_dev(pos, torch.float64, d)
    x, y, z = (p[:, k].contiguous() for k in range(3))
    act = _as_dev(np.asarray(active, dtype=np.uint8) if not isinstance(active, torch.Tensor) else active.to(torch.uint8),
                  torch.uint8, d)
    q = _as_dev(charge, torch.float64, d).reshape(-1)
    m = _as_dev(mass, torch.float64, d).reshape(-1)
    off_t = torch.as_tensor(offs, device=d)
    out = [torch.empty_like(x) for _ in range(3)]
    a = _lib.SptAccelArgs()
    a.n_groups = len(sizes)
    a.max_group_size = int(sizes.max())
    a.n_particles = int(offs[-1])
    a.group_offset = off_t.data_ptr()
    a.x, a.y, a.z = x.data_ptr(), y.data_ptr(), z.data_ptr()
    a.active, a.charge, a.mass = act.data_ptr(), q.data_ptr(), m.data_ptr()
    a.charge_to_mass = float(charge_to_mass)
    a.coulomb_constant = float(coulomb_constant)
    a.plummer_radius = float(plummer_radius)
    a.form = FORMS[form] if isinstance(form, str) else int(form)
    a.ax, a.ay, a.az = (o.data_ptr() for o in out)
    geom = geometry.to_struct()
    tables = geometry.bem_tables(d) if geometry.is_bem else None
    stream = torch.cuda.current_stream(d)
    _lib.check(_lib.lib().spt_accel(ctypes.byref(a), ctypes.byref(geom),
                                    ctypes.byref(tables.view(far_rule)) if tables is not None else None,
                                    ctypes.c_void_p(stream.cuda_stream)), "spt_accel")
    return torch.stack(out, dim=-1)


def bem_field(tables, points, form="fp64", far_rule="reference", **rule_kw):
    """Perturbation field of a BEM solution at points [N, 3] (spt_bem_field)."""
    view = tables.view(far_rule, **rule_kw)
    torch = _torch()
    p = _as_dev(points, torch.float64, tables.seg.device).reshape(-1, 3)
    x, y, z = (p[:, k].contiguous() for k in range(3))
    out = [torch.empty_like(x) for _ in range(3)]
    stream = torch.cuda.current_stream(tables.seg.device)
    _lib.check(_lib.lib().spt_bem_field(x.data_ptr(), y.data_ptr(), z.data_ptr(), x.numel(),
                                        ctypes.byref(view), FORMS[form] if isinstance(form, str) else form,
                                        out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(),
                                        ctypes.c_void_p(stream.cuda_stream)), "spt_bem_field")
    return torch.stack(out, dim=-1)


class SurrogateBinding:
    """Device-side parameters of a trained FieldSurrogate for the learned
    form: the sur_* fields of SptTraceParams, and the statistics buffer
    (surrogate points, band points, spot checks, max spot error).  The
    parameters are copied when the binding is made: the FP32 set the stage
    kernel reads holds the BF16-rounded weights and the FP32 biases, as the
    standalone network uses them."""

    def __init__(self, model, band=5e-9, spot=0.01, device="cuda"):
        torch = _torch()
        d = torch.device(device)
        self.model = model
        self.w = model.pr.clone()
        for name, _ in sg_param_shapes():
            if name.startswith("b"):
                model.view(self.w, name).copy_(model.view(model.p, name))
        self.w16 = model.p16.clone()
        self.band, self.spot = float(band), float(spot)
        self.s_start = torch.as_tensor(model.s_start, dtype=torch.float64, device=d)
        self.log_scale = torch.as_tensor(np.log(model.scale_table), dtype=torch.float64, device=d)
        self.stats_buf = torch.zeros(4, dtype=torch.int64, device=d)
        if self.w16.data_ptr() % 16:
            raise ValueError("surrogate BF16 parameters must be 16-byte aligned")

    def fill(self, p):
        m = self.model
        p.sur_w = self.w.data_ptr()
        p.sur_w16 = self.w16.data_ptr()
        p.sur_s_start = self.s_start.data_ptr()
        p.sur_log_scale = self.log_scale.data_ptr()
        p.sur_s_end, p.sur_sig_floor = float(m.s_end), float(m.sig_floor)
        p.sur_band, p.sur_spot = self.band, self.spot
        p.sur_d_min, p.sur_d_max = float(m.D_MIN), float(m.D_MAX)
        p.sur_stats = self.stats_buf.data_ptr()
        return p

    def reset(self):
        self.stats_buf.zero_()

    def stats(self):
        """(surrogate points, band points, spot checks, max spot error relative
        to the whole external field at the point)."""
        v = self.stats_buf.cpu().numpy()
        err = np.array([v[3] & 0xFFFFFFFF], dtype=np.uint32).view(np.float32)[0]
        return int(v[0]), int(v[1]), int(v[2]), float(err)


def sg_param_shapes():
    from .surrogate import PARAM_SHAPES
    return PARAM_SHAPES


def surrogate_field(tables, binding, points, far_rule="reference"):
    """Learned-form perturbation field at points [N, 3] (spt_surrogate_field):
    the surrogate outside the binding's band, exact inside it and for its
    spot checks."""
    torch = _torch()
    p = _as_dev(points, torch.float64, tables.seg.device).reshape(-1, 3)
    x, y, z = (p[:, k].contiguous() for k in range(3))
    out = [torch.empty_like(x) for _ in range(3)]
    prm = binding.fill(_lib.SptTraceParams())
    stream = torch.cuda.current_stream(tables.seg.device)
    _lib.check(_lib.lib().spt_surrogate_field(x.data_ptr(), y.data_ptr(), z.data_ptr(), x.numel(),
                                              ctypes.byref(tables.view(far_rule)), ctypes.byref(prm), out[0].data_ptr(),
                                              out[1].data_ptr(), out[2].data_ptr(),
                                              ctypes.c_void_p(stream.cuda_stream)), "spt_surrogate_field")
    return torch.stack(out, dim=-1)


def ring_field(rho, z, a, form="fp64", device="cuda"):
    torch = _torch()
    d = torch.device(device)
    r, zz, aa = (_as_dev(v, torch.float64, d).reshape(-1) for v in (rho, z, a))
    er, ez = torch.empty_like(r), torch.empty_like(r)
    stream = torch.cuda.current_stream(d)
    _lib.check(_lib.lib().spt_ring_field(r.data_ptr(), zz.data_ptr(), aa.data_ptr(), r.numel(),
                                         FORMS[form] if isinstance(form, str) else form, er.data_ptr(),
                                         ez.data_ptr(), ctypes.c_void_p(stream.cuda_stream)), "spt_ring_field")
    return er, ez


def ellip_ke(p, form="fp64", device="cuda"):
    torch = _torch()
    d = torch.device(device)
    pp = _as_dev(p, torch.float64, d).reshape(-1)
    K, E = torch.empty_like(pp), torch.empty_like(pp)
    stream = torch.cuda.current_stream(d)
    _lib.check(_lib.lib().spt_ellip_ke(pp.data_ptr(), pp.numel(), FORMS[form] if isinstance(form, str) else form,
                                       K.data_ptr(), E.data_ptr(), ctypes.c_void_p(stream.cuda_stream)),
               "spt_ellip_ke")
    return K, E
