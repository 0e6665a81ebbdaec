"""The headline workload, 694x554 with D=128 (seed 0), whole path against
the reference's own implementation run here: its matchers and feature
assembly compiled unmodified (oracle/_ref), batched as Testing.test_model
does (test.py:597-626), scikit-learn's predict_proba on the committed
forest, then Testing.eval_prob's _mem post (test.py:143-149, 341-449)
through its post.cu on the GPU.  The fused forest path must give the same
P(class 0) (equal float32 roundings of the same leaves' averages) and the
same disparity on >= 99.9 % of pixels within 0.5 px.

The reference's post.cu needs W >= H (its SGM state, post.cu:213) and, as
H*W = 384,476 is not a multiple of 64, its swap_axis_back reads up to 48
pixels x D doubles (48 KB) past the end of its 394 MB volume, inside the
2 MiB rounding of that allocation.
"""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FOREST = os.path.join(HERE, "golden", "forest_694x554.npz")


def test_forest_path_equals_reference_path_694x554(gpu):
    from cbmv_b200 import synth
    from cbmv_b200.evaluate import bad_x
    from cbmv_b200.forest import FlatForest
    from cbmv_b200.forest_gpu import GpuForest
    from cbmv_b200.pipeline import StereoPipeline
    from oracle import glue, ref, skforest
    assert ref.cpu_available() and ref.post_available(), "oracle/_ref is not built (make -C oracle ref)"
    L, R, gt, nonocc = synth.pair_694x554(seed=0)
    H, W = L.shape
    D = 128
    assert W >= H
    cores = len(os.sched_getaffinity(0))
    ref.set_threads(cores)
    flat = FlatForest.load(FOREST)
    skl = skforest.to_sklearn(flat, n_jobs=cores)
    proba = glue.test_model(ref.mtc, ref.fte, skl.predict_proba, L, R, D)
    ref.post.InitCUDA()
    d_ref = glue.eval_prob(ref.post, ref.fte, proba, L, R, D)
    pipe = StereoPipeline(GpuForest(flat))
    prob = torch.empty((H, W, D), device="cuda")
    disp = pipe.run_rf(L, R, D, prob_out=prob)
    p0 = prob.cpu().numpy().reshape(-1)
    same = float(np.mean(p0 == proba[:, 0].astype(np.float32)))
    close = float(np.mean(np.abs(disp - d_ref) <= 0.5))
    print("694x554 D=128 forest path vs reference path: P0 equal on %.6f, disparity within 0.5 px %.5f, "
          "bad-2.0 %.4f (reference %.4f)" % (same, close, bad_x(disp, gt, nonocc), bad_x(d_ref, gt, nonocc)))
    assert same > 0.9999, same
    assert close >= 0.999, close
