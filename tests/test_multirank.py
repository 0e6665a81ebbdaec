"""The multi-GPU form of the batched path, on CPU: cbmv_b200.shard splits a
batch of uneven pairs longest-processing-time first over the ranks, every
rank runs its own pairs, and rank 0 gathers every pair's disparity map and
per-pair numbers (world-size-2 gloo ranks here; bench.py --batch runs the
same functions over NCCL).  The per-pair work of each rank is a small
stand-in computed on the host (the census winner-take-all of the oracle),
so that the gathered maps can be checked against a single-process run."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _specs():
    rng = np.random.default_rng(3)
    return [dict(seed=100 + i, width=int(rng.integers(40, 90)), height=int(rng.integers(24, 40)),
                 ndisp=int(rng.choice([8, 12, 16])), planes=3, dmin=1, dmax=6) for i in range(9)]


def _disparity(spec):
    """A stand-in for one pair's device path: census cost, first minimum."""
    from cbmv_b200 import synth
    from oracle import cpu
    L, R, _, _ = synth.make_pair(**spec)
    return np.argmin(cpu.mtc.census(L, R, spec["ndisp"], 11), axis=2).astype(np.float32)


def _rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from cbmv_b200 import shard
    specs = _specs()
    shapes = [(s["height"], s["width"], s["ndisp"]) for s in specs]
    assign = shard.lpt_assign(shard.pair_work(shapes), world)
    mine = [torch.from_numpy(_disparity(specs[i])) for i in assign[rank]]
    maps = shard.gather_maps(mine, assign, shapes)
    lat = shard.gather_values([10.0 * i + rank for i in assign[rank]], assign, len(shapes))
    t = shard.max_over_ranks(5.0 + rank)
    q.put((rank, assign, None if maps is None else [m.numpy() for m in maps], lat.tolist(), t))
    dist.destroy_process_group()


def test_lpt_assignment_properties():
    from cbmv_b200 import shard
    work = [5, 9, 1, 9, 3, 7, 2, 8]
    a = shard.lpt_assign(work, 3)
    assert sorted(i for r in a for i in r) == list(range(len(work)))  # each pair exactly once
    assert a == shard.lpt_assign(work, 3)                             # deterministic
    loads = [sum(work[i] for i in r) for r in a]
    # LPT's bound: the largest load is within 4/3 of the best possible split
    assert max(loads) <= 4 / 3 * max(max(work), sum(work) / 3)
    assert a[0][0] == 1 and a[1][0] == 3   # the two longest pairs go first, to different ranks
    assert shard.lpt_assign(work, 1) == [sorted(range(len(work)), key=lambda i: (-work[i], i))]
    with pytest.raises(ValueError):
        shard.lpt_assign(work, 0)


def test_two_ranks_shard_gather_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=180) for _ in procs], key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, a0, maps, lat0, t0), (r1, a1, none, lat1, t1) = res
    assert a0 == a1 and len(a0[0]) and len(a1[0])      # both ranks computed the same split
    assert none is None and maps is not None
    specs = _specs()
    for i, s in enumerate(specs):                      # every map in its pair's slot
        assert np.array_equal(maps[i], _disparity(s)), i
    owner = {i: r for r in range(2) for i in a0[r]}
    assert lat0 == lat1 == [10.0 * i + owner[i] for i in range(len(specs))]
    assert t0 == t1 == 6.0                             # both see the slower rank's time


def test_shard_functions_without_a_process_group():
    """A single-process run (no torch.distributed group): the gather
    returns the maps in pair order, the values as given, the maximum the
    value itself."""
    import torch
    from cbmv_b200 import shard
    shapes = [(3, 4, 8), (2, 5, 8), (4, 4, 8)]
    assign = shard.lpt_assign(shard.pair_work(shapes), 1)
    maps = [torch.full((shapes[i][0], shapes[i][1]), float(i)) for i in assign[0]]
    out = shard.gather_maps(maps, assign, shapes)
    assert [float(m[0, 0]) for m in out] == [0.0, 1.0, 2.0]
    vals = shard.gather_values([10.0 * i for i in assign[0]], assign, 3)
    assert list(vals) == [0.0, 10.0, 20.0]
    assert shard.max_over_ranks(2.5) == 2.5
