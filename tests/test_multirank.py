"""The N > 1 path of bench.py on the CPU: two ranks over gloo.  Each rank
traces its own workload (seed + rank, same shapes) and the whole-job numbers
are the slowest rank's time and the sum of particle-steps."""

import os
import socket
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, REPO)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        t, steps = bench.combine_ranks(1.0 + rank, 10 * (rank + 1), world, "cpu")
        wl = bench.build_workload("c0", rank)
        out[rank] = (t, steps, float(wl["data"]["x"][0]), tuple(wl["data"]["group_sizes"]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_combine_max_time_and_summed_steps():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        t, steps, _, _ = res[rank]
        assert t == 2.0 and steps == 30.0
    # weak scaling: same shapes, different seeds per rank
    assert res[0][3] == res[1][3]
    assert res[0][2] != res[1][2]


def test_one_rank_needs_no_process_group():
    sys.path.insert(0, REPO)
    import bench
    assert bench.combine_ranks(1.5, 7, 1, "cpu") == (1.5, 7.0)
    assert np.isfinite(bench.combine_ranks(1.5, 7, 1, "cpu")[0])
