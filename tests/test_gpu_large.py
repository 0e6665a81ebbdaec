"""The larger workloads on the device.

1482x994, D=256 (the plain path at a larger size, seed 1): census and
SAD-on-Sobel volumes of the whole image bit-exact against the oracle run on a
band of rows (every matcher is row-local within its window, so a band with a
10-row margin reproduces the whole-image rows), and the forest's leaves and
P(class 0) bit-exact on sampled (pixel, d) of that band.

2880x1988, D=400 (the full-resolution pair, seed 5; 2.29 G (pixel, d), past
2^31): the learned path's four float32 volumes checked on rows near the
bottom (linear indices beyond 2^31) against the oracle's band, then the
learned classifier end to end with the random forest as its judge: bad-2.0
(non-occluded) of the network within 0.5 percentage points of the forest's
(both trained on 694x554, D=128 pairs; neither was tuned for this size).
"""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FOREST = os.path.join(HERE, "golden", "forest_694x554.npz")
MLP = os.path.join(HERE, "golden", "mlp_694x554.npz")


def _band_costs(oracle_cpu, L, R, y0, rows, D, margin=10):
    """The oracle's four [rows,W,D] float64 volumes of image rows y0..y0+rows."""
    from oracle import glue
    a, b = max(y0 - margin, 0), min(y0 + rows + margin, L.shape[0])
    vols = glue.get_costs(oracle_cpu.mtc, oracle_cpu.fte, L[a:b].copy(), R[a:b].copy(), D)
    return [v[y0 - a:y0 - a + rows] for v in vols]


def test_1482x994_census_sad_and_forest_bitexact(gpu, oracle_cpu):
    from cbmv_b200 import libmatchers as mtc, synth
    from cbmv_b200.forest import FlatForest
    from cbmv_b200.forest_gpu import GpuForest
    from cbmv_b200.pipeline import StereoPipeline
    from oracle import glue
    L, R, _, _ = synth.pair_1482x994()
    H, W = L.shape
    D = 256
    y0, rows = 700, 4
    ref = _band_costs(oracle_cpu, L, R, y0, rows, D)
    l, r = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    census = mtc.census(l, r, D, 11)                                   # [H,W,D] float64, device
    assert torch.equal(census[y0:y0 + rows].cpu(), torch.from_numpy(ref[0]))
    del census
    sad = mtc.sadsob(mtc.sobel(l), mtc.sobel(r), D, 5)                 # [D,H,W] float64, device
    assert torch.equal(sad[:, y0:y0 + rows].permute(1, 2, 0).cpu(), torch.from_numpy(ref[2]))
    del sad
    # forest: the fused path's P(class 0) and the leaves of sampled (pixel, d)
    flat = FlatForest.load(FOREST)
    gf = GpuForest(flat)
    pipe = StereoPipeline(gf)
    prob = torch.empty((H, W, D), device="cuda")
    pipe.run_rf(l, r, D, prob_out=prob)
    X = glue.extract_features_lr(oracle_cpu.fte, *ref)                 # [rows*W*D, 20] float64
    idx = np.random.default_rng(0).choice(X.shape[0], 60000, replace=False)
    p_ref, leaves_ref = oracle_cpu.rf_predict(flat, X[idx], return_leaves=True)
    band_idx = torch.from_numpy(y0 * W * D + idx).cuda()
    feats = pipe.features_at(l, r, D, band_idx).cpu().numpy()
    assert np.array_equal(feats, X[idx].astype(np.float32))
    assert np.array_equal(gf.apply(feats), leaves_ref)
    p0 = prob.reshape(-1)[band_idx].cpu().numpy()
    assert np.mean(p0 == p_ref.astype(np.float32)) > 0.9999


def test_2880x1988_learned_path_judged_by_forest(gpu, oracle_cpu):
    from cbmv_b200 import synth
    from cbmv_b200.evaluate import bad_x
    from cbmv_b200.forest_gpu import GpuForest
    from cbmv_b200.mlp import GpuMlp
    from cbmv_b200.pipeline import StereoPipeline
    L, R, gt, nonocc = synth.pair_2880x1988()
    H, W = L.shape
    D = 400
    assert H * W * D > 2 ** 31
    l, r = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    pipe = StereoPipeline()
    # matcher volumes of the whole pair, checked on bottom rows (indices past 2^31)
    y0, rows = H - 20, 3
    assert y0 * W * D > 2 ** 31
    vols = pipe.volumes_f32(l, r, D)
    band = vols[:, y0:y0 + rows].cpu().numpy()
    del vols
    torch.cuda.empty_cache()
    ref = _band_costs(oracle_cpu, L, R, y0, rows, D)
    for m in range(3):
        assert np.array_equal(band[m], ref[m].astype(np.float32)), m
    ulp = np.abs(band[3].view(np.int32).astype(np.int64) - ref[3].astype(np.float32).view(np.int32).astype(np.int64))
    assert ulp.max() <= 1
    # the learned path end to end, then the forest's on its own context
    net = GpuMlp.load(MLP)
    disp_mlp = pipe.run_mlp(net, l, r, D).cpu().numpy()
    assert net.status() == 0
    pipe.close()
    torch.cuda.empty_cache()
    rf_pipe = StereoPipeline(GpuForest.load(FOREST))
    disp_rf = rf_pipe.run_rf(l, r, D).cpu().numpy()
    rf_pipe.close()
    b_mlp, b_rf = bad_x(disp_mlp, gt, nonocc), bad_x(disp_rf, gt, nonocc)
    print("2880x1988 D=400 bad-2.0: network %.4f forest %.4f" % (b_mlp, b_rf))
    assert np.isfinite(disp_mlp).all() and disp_mlp.min() >= 0 and disp_mlp.max() <= D
    # both classifiers were trained on 694x554, D=128 pairs: at this size
    # (coarser texture, 400 disparities) both lose accuracy (forest ~31 %,
    # network ~26 % bad-2.0 here); the bound only rules out a broken path
    assert b_rf < 0.5
    assert b_mlp <= b_rf + 0.005
