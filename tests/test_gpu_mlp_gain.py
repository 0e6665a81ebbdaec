"""What the trained network gains over the method without it.

On held-out seeded 694x554, D=128 pairs, the same test path (matchers, 20
features, classifier, MC-CNN `_mem` post) is run three ways:

- with the trained GELU network (tests/golden/mlp_gelu_694x554.npz,
  trained by cbmv_b200/train_mlp.py on GPU-emitted samples of pairs
  2000..2199);
- with the same network before training (its random initialisation, same
  input transform): the learned weights alone are what differs;
- without a classifier: the post-processing applied to the normalised census
  cost, the best single matcher (test.py:341-449 driven with that volume),
  i.e. MC-CNN's pipeline on a hand-made cost.

The trained network must beat both by a clear margin on bad-2.0, and its
bf16 form of the fused inference (cbmv_mlp_set_precision) must stay within
0.5 percentage points of the f16 form it runs in by default.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
MLP = os.path.join(HERE, "golden", "mlp_gelu_694x554.npz")
SEEDS = [3000, 3001, 3002]


def _census_only(L, R, nonocc, gt):
    from cbmv_b200 import libmatchers, post
    from cbmv_b200.evaluate import bad_x
    from oracle import glue
    c = libmatchers.census(L, R, 128, 11)            # [H,W,D] f64 Hamming distances
    c = np.minimum(c, 121.0) / 121.0                  # sentinel -> 1, costs in [0,1] like P(class 0)
    imgl, imgr = glue.normalise_images(L, R)
    d = glue.postprocessing_mem(post, imgl, imgr, c, -1)
    return bad_x(np.asarray(d, np.float32), gt, nonocc)


def test_trained_mlp_beats_untrained_and_no_classifier(gpu):
    import torch
    from cbmv_b200 import synth
    from cbmv_b200.evaluate import bad_x
    from cbmv_b200.mlp import GpuMlp, MlpParams
    from cbmv_b200.pipeline import StereoPipeline
    trained = MlpParams.load(MLP)
    v = trained.views()
    untrained = MlpParams.init(0, v["cap"].copy(), v["mu"].copy(), 1.0 / v["inv_sd"], trained.activation)
    net_t, net_u, net_b = GpuMlp(trained), GpuMlp(untrained), GpuMlp(trained, "bf16")
    pipe = StereoPipeline()
    rows = []
    for s in SEEDS:
        L, R, gt, nonocc = synth.pair_694x554(s)
        l, r = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
        bt = bad_x(pipe.run_mlp(net_t, l, r, 128).cpu().numpy(), gt, nonocc)
        bu = bad_x(pipe.run_mlp(net_u, l, r, 128).cpu().numpy(), gt, nonocc)
        bb = bad_x(pipe.run_mlp(net_b, l, r, 128).cpu().numpy(), gt, nonocc)
        bc = _census_only(L, R, nonocc, gt)
        rows.append((bt, bu, bc, bb))
    assert net_t.status() == 0 and net_u.status() == 0 and net_b.status() == 0
    bt, bu, bc, bb = (float(np.mean(c)) for c in zip(*rows))
    print("bad-2.0 trained %.4f (bf16 form %.4f) untrained %.4f census-only %.4f" % (bt, bb, bu, bc))
    assert abs(bb - bt) < 0.005, (bb, bt)
    assert bt < 0.06, bt
    assert bt < bu - 0.05, (bt, bu)      # training, not the architecture, makes the classifier
    assert bt < 0.8 * bc, (bt, bc)       # the learned classifier over the best single matcher
