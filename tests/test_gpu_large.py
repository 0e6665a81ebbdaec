"""The larger workloads on the device.

1482x994, D=256 (the plain path at a larger size, seed 1): census and
SAD-on-Sobel volumes bit-exact against the oracle on four bands of rows (the
first rows, two interior bands and the last rows; every matcher is row-local
within its window, so a band with a 10-row margin reproduces the
whole-image rows), the forest's leaves and P(class 0) bit-exact on sampled
(pixel, d) of one band, and the disparity of the fused path against the
reference's own post.cu run on the same P(class 0) (>= 99.9 % within 0.5 px).

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
MLP = os.path.join(HERE, "golden", "mlp_gelu_694x554.npz")


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
    l, r = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    census = mtc.census(l, r, D, 11)                                   # [H,W,D] float64, device
    sad = mtc.sadsob(mtc.sobel(l), mtc.sobel(r), D, 5)                 # [D,H,W] float64, device
    bands = [(0, 4), (350, 4), (700, 4), (H - 4, 4)]
    for b0, n in bands:
        rb = _band_costs(oracle_cpu, L, R, b0, n, D)
        assert torch.equal(census[b0:b0 + n].cpu(), torch.from_numpy(rb[0])), b0
        assert torch.equal(sad[:, b0:b0 + n].permute(1, 2, 0).cpu(), torch.from_numpy(rb[2])), b0
    del census, sad
    torch.cuda.empty_cache()
    y0, rows = 700, 4
    ref = _band_costs(oracle_cpu, L, R, y0, rows, D)
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


def test_1482x994_disparity_against_reference_post(gpu):
    """The fused forest path's disparity at 1482x994, D=256 against the
    reference's post.cu (oracle/_ref, run on the GPU as shipped) driven by
    Testing.__postprocessing_mem (test.py:341-449) on the same P(class 0)
    volume (whose leaves and probabilities the test above holds to the
    reference).  The reference's kernels need W >= H (its SGM state) and
    read up to 48 pixels x D past the end of a volume in swap_axis_back when
    H*W is not a multiple of 64: here 96 KB, inside the 2 MiB rounding of
    its 3 GB allocation."""
    from cbmv_b200 import synth
    from cbmv_b200.forest_gpu import GpuForest
    from cbmv_b200.pipeline import StereoPipeline
    from oracle import glue, ref
    assert ref.post_available(), "oracle/_ref/libcbmv_ref_post.so is not built"
    L, R, _, _ = synth.pair_1482x994()
    H, W = L.shape
    D = 256
    assert W >= H
    pipe = StereoPipeline(GpuForest.load(FOREST))
    prob = torch.empty((H, W, D), device="cuda")
    disp = pipe.run_rf(L, R, D, prob_out=prob)
    cost = prob.cpu().numpy().astype(np.float64)
    del prob
    pipe.close()
    torch.cuda.empty_cache()
    ref.post.InitCUDA()
    imgl, imgr = glue.normalise_images(L, R)
    d_ref = glue.postprocessing_mem(ref.post, imgl, imgr, cost, -1)
    close = float(np.mean(np.abs(disp - d_ref) <= 0.5))
    print("1482x994 D=256: fused forest path vs reference post.cu, within 0.5 px %.5f" % close)
    assert close >= 0.999, close


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
