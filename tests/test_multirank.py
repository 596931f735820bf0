"""The N > 1 path on the CPU: one workload split into contiguous group
ranges balanced by cost (bem_b200.partition), each rank tracing its range,
the final state all-gathered in group order -- run as two gloo ranks, each
tracing its shard with the oracle; the gathered result must equal one rank
tracing everything, bit for bit (groups never interact)."""

import os
import socket
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

from bem_b200 import partition  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _workload():
    """Seven flat-cathode groups of uneven sizes (1 to 9)."""
    from bem_b200 import workloads as w
    sizes = [3, 1, 9, 2, 5, 7, 4]
    d = w.flat_c0(n_groups=len(sizes), n_emit=9, seed=5, t_spread=0.2e-12)
    # regroup the first sum(sizes) particles into the uneven sizes
    n = sum(sizes)
    d = {k: (v[:n] if isinstance(v, np.ndarray) and v.shape[:1] == (len(sizes) * 9,) else v) for k, v in d.items()}
    d["group_sizes"] = np.asarray(sizes)
    return d


def _trace_oracle(data):
    """Oracle trace (40 attempts) of every group of `data`, one group per
    call (each group has its own size); returns the partition module's state
    arrays."""
    from oracle import geometry as ogeo
    from oracle import physics as ophys
    from oracle import rk45 as ork
    spec = dict(kind="flat", E_gun=-1e7, z0=3e-9, kill_z_below=0.0)
    m = ophys.ev_to_kg(ophys.ELECTRON_MASS_EV)
    q = -ophys.ELEMENTARY_CHARGE
    sizes = np.asarray(data["group_sizes"])
    offs = np.concatenate([[0], np.cumsum(sizes)])
    out = {k: [] for k in ("x", "y", "z", "vx", "vy", "vz", "t_death", "t", "h")}
    for g in range(len(sizes)):
        sl = slice(offs[g], offs[g + 1])
        E = int(sizes[g])
        pos = np.stack([data["x"][sl], data["y"][sl], data["z"][sl]], -1).reshape(1, E, 3)
        vel = np.stack([data[k][sl] for k in ("px", "py", "pz")], -1).reshape(1, E, 3) * (
            ophys.ELEMENTARY_CHARGE / ophys.SPEED_OF_LIGHT / m)
        tb = data["t"][sl].reshape(1, E)
        acc = ogeo.make_accel(spec, np.full((1, E), q), np.full((1, E), m), q / m, 1e-12)
        p, v, td, t, h, _ = ork.integrate(acc, pos, vel, tb, 2e-12, 1e-8, 1e-12, kill=ogeo.make_kill(spec, 1e-3),
                                          max_attempts=40)
        for k, a in zip(("x", "y", "z"), p[0].T):
            out[k].append(a)
        for k, a in zip(("vx", "vy", "vz"), v[0].T):
            out[k].append(a)
        out["t_death"].append(td[0])
        out["t"].append(np.atleast_1d(t))
        out["h"].append(np.atleast_1d(h))
    return {k: np.concatenate(v) for k, v in out.items()}


def _rank_main(rank, world, port, out):
    sys.path.insert(0, REPO)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        t, steps = bench.combine_ranks(1.0 + rank, 10 * (rank + 1), world, "cpu")
        data = _workload()
        sizes = np.asarray(data["group_sizes"])
        ranges = partition.partition(sizes, world)
        g0, g1 = ranges[rank]
        local = _trace_oracle(partition.shard(data, g0, g1))
        counts = [int(sizes[a:b].sum()) for a, b in ranges]
        gcounts = [b - a for a, b in ranges]
        got = partition.gather_state({k: torch.as_tensor(v) for k, v in local.items()}, counts, gcounts)
        out[rank] = (t, steps, ranges, {k: v.numpy() for k, v in got.items()})
    finally:
        dist.destroy_process_group()


def test_two_ranks_partition_gather_equals_one_rank():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    whole = _trace_oracle(_workload())
    for rank in range(world):
        t, steps, ranges, got = res[rank]
        assert t == 2.0 and steps == 30.0   # max of the ranks' times, sum of their particle-steps
        assert ranges[0][0] == 0 and ranges[-1][1] == 7 and ranges[0][1] == ranges[1][0]
        for k, v in whole.items():
            np.testing.assert_array_equal(got[k], v, err_msg=k)


def test_partition_is_contiguous_and_balanced():
    rng = np.random.default_rng(0)
    sizes = np.clip(np.rint(np.exp(rng.uniform(0, np.log(256), 4096))), 1, 256).astype(int)
    cost = partition.group_cost(sizes)
    for n in (1, 2, 3, 8):
        ranges = partition.partition(sizes, n)
        assert ranges[0][0] == 0 and ranges[-1][1] == len(sizes)
        assert all(a < b for a, b in ranges)
        assert all(ranges[i][1] == ranges[i + 1][0] for i in range(n - 1))
        shares = np.array([cost[a:b].sum() for a, b in ranges])
        # every boundary is within one group of its ideal position
        assert shares.max() - shares.min() <= 2 * cost.max() + 1e-9


def test_partition_more_ranks_than_groups_leaves_some_empty():
    ranges = partition.partition([5, 5], 3)
    assert ranges[0][0] == 0 and ranges[-1][1] == 2
    assert sum(b - a for a, b in ranges) == 2


def test_one_rank_needs_no_process_group():
    import bench
    assert bench.combine_ranks(1.5, 7, 1, "cpu") == (1.5, 7.0)
