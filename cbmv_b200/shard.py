"""Stereo pairs across ranks: one process per GPU.

The reference runs one rectified pair per process (main.py:53-70) and no
step inside a pair exchanges data with another pair, so pairs are the unit
of work across GPUs: a batch of pairs is split longest-processing-time
first (by H*W*D) over the ranks, every rank runs its share through the
learned path (its own CUDA-graph batch), and the only collective is the
gather of the disparity maps and per-pair timings on rank 0.  The gather is
point-to-point send/recv, so the same code runs over NCCL (device tensors)
and gloo (host tensors).  Every rank calls the same collectives in the same
order.
"""
import numpy as np


def lpt_assign(work, n_ranks):
    """Longest processing time first: pairs in order of decreasing work
    (ties: lower index first), each onto the rank with the least work so far
    (ties: lower rank).  Returns, per rank, its pair indices in run order."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(work)), key=lambda i: (-float(work[i]), i))
    load = [0.0] * n_ranks
    out = [[] for _ in range(n_ranks)]
    for i in order:
        k = min(range(n_ranks), key=lambda r: (load[r], r))
        out[k].append(i)
        load[k] += float(work[i])
    return out


def pair_work(shapes):
    """H*W*D of every (H, W, D) shape: the (pixel, d) units of the pair."""
    return [int(h) * int(w) * int(d) for h, w, d in shapes]


def _distributed(group=None):
    """(rank, world size) of this process, (0, 1) when no process group is
    initialised (a single-process run)."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def gather_maps(maps, assign, shapes, device=None, group=None):
    """Disparity maps of every pair on rank 0.

    maps: this rank's maps (float32 tensors [H,W]) for the pairs
    assign[rank], in that order; shapes: (H, W, D) of every pair.  Rank 0
    returns the list of all maps in pair order; the other ranks None."""
    import torch
    import torch.distributed as dist
    rank, ws = _distributed(group)
    if len(maps) != len(assign[rank]):
        raise ValueError("rank %d holds %d maps for %d pairs" % (rank, len(maps), len(assign[rank])))
    if rank != 0:
        for m in maps:
            dist.send(m.contiguous(), dst=0, group=group)
        return None
    out = [None] * len(shapes)
    for i, m in zip(assign[0], maps):
        out[i] = m
    for src in range(1, ws):
        for i in assign[src]:
            buf = torch.empty((int(shapes[i][0]), int(shapes[i][1])), dtype=torch.float32, device=device)
            dist.recv(buf, src=src, group=group)
            out[i] = buf
    return out


def gather_values(values, assign, n, device=None, group=None):
    """Per-pair numbers (e.g. latencies) of every pair on every rank: each
    rank fills its pairs' slots, the others stay zero, and a sum-reduction
    combines them.  values: this rank's numbers in assign[rank] order."""
    import torch
    import torch.distributed as dist
    rank, ws = _distributed(group)
    t = torch.zeros(n, dtype=torch.float64, device=device)
    for i, v in zip(assign[rank], values):
        t[i] = float(v)
    if ws > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def max_over_ranks(x, device=None, group=None):
    """The largest of every rank's x (a step time: the job is as slow as its
    slowest rank)."""
    import torch
    import torch.distributed as dist
    if _distributed(group)[1] == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def assignment_summary(assign, work):
    """Units and pairs per rank, and the imbalance max/mean of the units."""
    units = np.array([sum(work[i] for i in a) for a in assign], np.float64)
    return {"pairs": [len(a) for a in assign], "units": units.astype(np.int64).tolist(),
            "imbalance": float(units.max() / units.mean()) if units.mean() > 0 else 1.0}
