"""Batches of uneven pairs as one CUDA graph launch (cbmv_batch_*), and the
autotuner that picks its launch shape."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
MLP = os.path.join(HERE, "golden", "mlp_694x554.npz")
SHAPES = [(120, 160, 32), (150, 200, 64), (96, 300, 48), (200, 180, 64), (130, 130, 24), (110, 250, 40)]


def _pairs(seed0=50):
    from cbmv_b200 import synth
    out = []
    for k, (h, w, d) in enumerate(SHAPES):
        L, R, _, _ = synth.make_pair(seed=seed0 + k, width=w, height=h, ndisp=d, planes=4, dmin=2, dmax=d - 4)
        out.append((torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()))
    return out


def test_tile_shapes_do_not_change_results(gpu):
    """The autotuner's tile shapes (CBCA tile rows, SGM prefetch depth)
    leave the disparities bit-identical."""
    from cbmv_b200 import _lib
    from cbmv_b200.mlp import GpuMlp
    from cbmv_b200.pipeline import StereoPipeline
    net = GpuMlp.load(MLP)
    (l, r), (_, _, d) = _pairs()[3], SHAPES[3]
    ref = StereoPipeline().run_mlp(net, l, r, d).cpu().numpy()
    for rows, pf in ((16, 0), (32, 1), (16, 4), (32, 2)):
        got = StereoPipeline(params=_lib.default_params(cbca_rows=rows, sgm_prefetch=pf)).run_mlp(net, l, r, d)
        assert np.array_equal(got.cpu().numpy(), ref), (rows, pf)


def test_batch_graph_matches_single_pairs(gpu):
    from cbmv_b200.batch import StereoBatch
    from cbmv_b200.mlp import GpuMlp
    from cbmv_b200.pipeline import StereoPipeline
    net = GpuMlp.load(MLP)
    pairs = _pairs()
    pipe = StereoPipeline()
    want = [pipe.run_mlp(net, l, r, d).cpu().numpy() for (l, r), (_, _, d) in zip(pairs, SHAPES)]
    b = StereoBatch(SHAPES, streams=3)
    lefts, rights = [p[0] for p in pairs], [p[1] for p in pairs]
    for rep in range(2):  # capture, then replay
        got = [t.cpu().numpy() for t in b.run_mlp(net, lefts, rights)]
        for i in range(len(SHAPES)):
            assert np.array_equal(got[i], want[i]), (rep, i)
    t = b.timings()
    assert np.all(t["pair_ms"] > 0) and np.all(t["done_ms"] <= t["total_ms"] + 1e-3)
    # new image buffers: the batch captures a new graph
    pairs2 = _pairs(seed0=80)
    want2 = [pipe.run_mlp(net, l, r, d).cpu().numpy() for (l, r), (_, _, d) in zip(pairs2, SHAPES)]
    got2 = [t.cpu().numpy() for t in b.run_mlp(net, [p[0] for p in pairs2], [p[1] for p in pairs2])]
    for i in range(len(SHAPES)):
        assert np.array_equal(got2[i], want2[i]), i
    assert net.status() == 0
    b.close()


def test_autotuner_picks_and_caches(gpu, tmp_path):
    from cbmv_b200.batch import tune_batch
    from cbmv_b200.mlp import GpuMlp
    net = GpuMlp.load(MLP)
    pairs = _pairs()
    cache = str(tmp_path / "autotune.json")
    res = tune_batch(SHAPES, net, [p[0] for p in pairs], [p[1] for p in pairs], streams=(1, 2), mlp_ctas=(0, None),
                     iters=1, cache_path=cache)
    # one context: "SMs / contexts" is every SM, the same candidate as 0, tried once;
    # then the tile search: CBCA rows 16, SGM prefetch 1 and 4
    assert not res["cached"] and res["streams"] in (1, 2) and len(res["tried"]) == 6
    assert res["cbca_rows"] in (16, 32) and res["sgm_prefetch"] in (0, 1, 4)
    assert res["ms"] == min(t["ms"] for t in res["tried"])
    again = tune_batch(SHAPES, net, [p[0] for p in pairs], [p[1] for p in pairs], cache_path=cache)
    assert again["cached"] and again["streams"] == res["streams"]
