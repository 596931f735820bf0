"""Multi-GPU partition of one tracer workload (one process per GPU).

Emission groups never interact (batched_rk45.py:4-17), so a workload shards
with no collective on the data path: every rank traces a contiguous range of
groups and the results are gathered once at the end.  The reference splits
its groups into even contiguous chunks for its CPU worker processes
(parallel.py:50) and concatenates the chunks' results in order
(parallel.py:64-68); here the ranges are balanced by an estimate of each
group's cost instead of its count, since uneven group sizes (1 to 256
particles) differ in cost by four orders of magnitude:

    cost(E) = E^2 * pair_weight + E * field_weight

(pair sums grow with E^2, the BEM field with E; both per attempt, and
attempts per group are taken as equal).  The BEM tables are replicated:
every rank builds its own copy from the same profile and density.

``gather_state`` concatenates the ranks' final particle state and group
counters in group order on every rank with ``all_gather`` (NCCL on the GPU
path, gloo on the CPU), padding the shards to a common length.
"""

import numpy as np

STATE_PARTICLE = ("x", "y", "z", "vx", "vy", "vz", "t_death")
STATE_GROUP = ("t", "h", "status", "n_accepted", "n_rejected")


def group_cost(sizes, pair_weight=1.0, field_weight=64.0):
    """Estimated relative cost of each group (per attempt)."""
    e = np.asarray(sizes, dtype=np.float64)
    return e * e * pair_weight + e * field_weight


def partition(sizes, n_ranks, cost=None):
    """Contiguous group ranges [(g0, g1), ...], one per rank, whose summed
    costs are as equal as a split at group boundaries allows: rank r's range
    ends at the first group where the running cost passes (r + 1) / n of the
    total.  Every range is non-empty when there are at least n_ranks groups."""
    sizes = np.asarray(sizes)
    G = len(sizes)
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    c = group_cost(sizes) if cost is None else np.asarray(cost, dtype=np.float64)
    cum = np.cumsum(c)
    total = cum[-1] if G else 0.0
    bounds = [0]
    for r in range(1, n_ranks):
        b = int(np.searchsorted(cum, total * r / n_ranks, side="left")) + 1
        # keep at least one group for every remaining rank, and ranges ordered
        b = max(b, bounds[-1] + (1 if G - bounds[-1] > n_ranks - r else 0))
        b = min(b, G - (n_ranks - r) if G >= n_ranks else G)
        bounds.append(b)
    bounds.append(G)
    return [(bounds[r], bounds[r + 1]) for r in range(n_ranks)]


def shard(data, g0, g1):
    """The workload dict (workloads.py convention) cut to groups [g0, g1)."""
    sizes = np.asarray(data["group_sizes"])
    offs = np.concatenate([[0], np.cumsum(sizes)])
    n = int(offs[-1])
    p0, p1 = int(offs[g0]), int(offs[g1])
    out = {}
    for k, v in data.items():
        if isinstance(v, np.ndarray) and v.shape[:1] == (n,):
            out[k] = v[p0:p1]
        else:
            out[k] = v
    out["group_sizes"] = sizes[g0:g1]
    return out


def gather_state(local, counts, group_counts, device=None):
    """All-gather of per-rank results.

    local: dict of 1-D tensors -- the particle arrays of STATE_PARTICLE
    (length counts[rank]) and the group arrays of STATE_GROUP (length
    group_counts[rank]).  counts / group_counts: every rank's lengths.
    Returns the same keys concatenated in rank order (= group order)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size()
    out = {}
    for keys, lens in ((STATE_PARTICLE, counts), (STATE_GROUP, group_counts)):
        n_max = int(max(lens))
        for k in keys:
            if k not in local:
                continue
            t = local[k]
            if device is not None:
                t = t.to(device)
            pad = torch.zeros(n_max, dtype=t.dtype, device=t.device)
            pad[: t.numel()] = t
            parts = [torch.empty_like(pad) for _ in range(world)]
            dist.all_gather(parts, pad)
            out[k] = torch.cat([p[: int(n)] for p, n in zip(parts, lens)])
    return out
