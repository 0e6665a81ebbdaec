"""Disparity error rates (bad-x) and the RF-vs-MLP comparison on held-out pairs.

bad-x follows the Local Expansion evaluator of the reference
(cpp/localexp/Evaluator.h:196-211): the fraction of pixels in the mask whose
|disparity - ground truth| exceeds the threshold (threshold 2.0 for bad-2.0).

    python -m cbmv_b200.evaluate --forest F.npz --mlp M.npz [--seeds 3000-3019]
"""
import argparse
import json
import time

import numpy as np

from . import synth

HELD_OUT = list(range(3000, 3020))


def bad_x(disp, gt, mask, thr=2.0):
    """1 - (pixels of the mask with |disp - gt| <= thr) / (pixels of the
    mask), as Evaluator.h:196-211 counts it (errorMap = |disp - dispGT| <=
    threshold), so a NaN disparity counts as an error; ground-truth pixels
    that are not finite are outside the mask (the reference's validMask)."""
    m = mask & np.isfinite(gt)
    return float(1.0 - np.mean(np.abs(disp[m] - gt[m]) <= thr))


def compare(forest_path, mlp_path, seeds=HELD_OUT, ndisp=128):
    from .forest_gpu import GpuForest
    from .mlp import GpuMlp
    from .pipeline import StereoPipeline
    return compare_loaded(StereoPipeline(GpuForest.load(forest_path)), GpuMlp.load(mlp_path), seeds, ndisp)


def compare_loaded(pipe, net, seeds=HELD_OUT, ndisp=128):
    """bad-2.0 (non-occluded) of the RF and MLP paths on the seeded 694x554
    pairs `seeds`, with a pipeline that holds the forest and an uploaded net."""
    import torch
    rows = []
    for s in seeds:
        L, R, gt, nonocc = synth.pair_694x554(s)
        l, r = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
        d_rf = pipe.run_rf(l, r, ndisp).cpu().numpy()
        d_mlp = pipe.run_mlp(net, l, r, ndisp).cpu().numpy()
        rows.append((s, bad_x(d_rf, gt, nonocc), bad_x(d_mlp, gt, nonocc)))
    if net.status() != 0:
        raise RuntimeError("a tensor-core wait timed out")
    rf = float(np.mean([r[1] for r in rows]))
    mlp = float(np.mean([r[2] for r in rows]))
    return {"seeds": [r[0] for r in rows], "bad2_rf": rf, "bad2_mlp": mlp,
            "per_seed": [{"seed": r[0], "rf": r[1], "mlp": r[2]} for r in rows]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--forest", required=True)
    ap.add_argument("--mlp", required=True)
    ap.add_argument("--seeds", default="3000-3019")
    a = ap.parse_args()
    lo, hi = (int(v) for v in a.seeds.split("-"))
    t0 = time.time()
    res = compare(a.forest, a.mlp, list(range(lo, hi + 1)))
    res["seconds"] = time.time() - t0
    print(json.dumps(res))


if __name__ == "__main__":
    main()
