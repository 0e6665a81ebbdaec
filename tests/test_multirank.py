"""The multi-GPU form of the benchmark, on CPU: world-size-2 gloo ranks each
take their own pair (weak scaling by independent pairs, no data-path
collective) and agree on the step time by a max-reduction, as bench.py does
over NCCL."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import numpy as np
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from cbmv_b200 import synth
    from oracle import cpu
    # each rank its own pair (seed = rank), as bench.py shards pairs
    L, R, _, _ = synth.make_pair(seed=rank, width=64, height=40, ndisp=12, planes=3, dmin=1, dmax=9)
    c = cpu.mtc.census(L, R, 12, 11)
    local_ms = float(10 + rank)  # stand-in for the rank's device time
    t = torch.tensor([local_ms], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    digest = torch.tensor([float(np.sum(c[c < 1e9]))], dtype=torch.float64)
    got = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(got, digest)
    q.put((rank, float(t.item()), [float(g.item()) for g in got]))
    dist.destroy_process_group()


def test_two_ranks_shard_pairs_and_reduce_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    # both ranks see the slower rank's time
    assert res[0][1] == res[1][1] == 11.0
    # and they processed different pairs
    digests = res[0][2]
    assert digests == res[1][2] and digests[0] != digests[1]
