"""The random forest's training path (train.py:100-293) with the samples
emitted on the GPU.

Training.__create_samples_mem (train.py:100-273) takes, for every valid
ground-truth pixel (finite, >= 0), one positive disparity round(gt) and two
negatives drawn at distance > 1 (featextract.cpp:154-215), the 20 features
at those (pixel, d) and labels [1, 0, 0].  Here the draws come from the
counter-based generator of `cbmv_generate_d_indices` (keyed by the pair's
seed: the reference's rand() inside OpenMP is not reproducible) and the
features from `cbmv_ctx_features_at` (the float64 features, stored as the
float32 that sklearn fits on), so the samples equal the CPU path's
(oracle.glue.create_samples_mem with the same draws) bit for bit.

    python -m cbmv_b200.train_rf --out forest.npz [--pairs 30] [--max-depth 20]

fits RandomForestClassifier(n_estimators=50, min_samples_leaf=700,
random_state=0) (train.py:287-288; max_depth 20 for the benchmark's forest)
on pairs 1000..1000+pairs-1 and writes a FlatForest .npz.
"""
import argparse
import os
import time

import numpy as np

from . import libfeatextract, synth


def emit_samples(pipe, L, R, gt, ndisp, seed):
    """(X float32 [3S, 20], y int32 [3S]) for the pair, rows 3s..3s+2 the
    positive and the two negatives of the s-th valid ground-truth pixel."""
    import torch
    g = np.asarray(gt, np.float64).reshape(-1)
    valid = ~((g == np.inf) | (g < 0))                    # train.py:105-107
    p = np.nonzero(valid)[0].astype(np.int64)
    gi = np.round(g[valid]).astype(np.int32)
    dind = np.asarray(libfeatextract.generate_d_indices(gi, ndisp, 1, seed=seed), np.int64)  # [S, 3]
    idx = (p[:, None] * ndisp + dind).reshape(-1)
    X = pipe.features_at(L, R, ndisp, torch.from_numpy(idx).cuda())
    y = np.tile(np.array([1, 0, 0], np.int32), len(p))  # featextract.cpp:490-516
    return X.cpu().numpy(), y


def train(pairs=30, max_depth=20, n_jobs=None, log=print):
    from sklearn.ensemble import RandomForestClassifier
    from .forest import FlatForest
    from .pipeline import StereoPipeline
    pipe = StereoPipeline()
    t0 = time.time()
    Xs, ys = [], []
    for seed in synth.RF_TRAIN_SEEDS[:pairs]:
        L, R, gt, _ = synth.pair_694x554(seed)
        X, y = emit_samples(pipe, L, R, gt, 128, seed)
        Xs.append(X)
        ys.append(y)
    X, y = np.concatenate(Xs), np.concatenate(ys)
    log("samples %s emitted on the GPU in %.1fs" % (X.shape, time.time() - t0))
    t0 = time.time()
    rf = RandomForestClassifier(n_estimators=50, min_samples_leaf=700, max_depth=max_depth,
                                n_jobs=n_jobs or os.cpu_count(), random_state=0)
    rf.fit(X, y)
    log("fit in %.1fs" % (time.time() - t0))
    return FlatForest.from_sklearn(rf)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--pairs", type=int, default=30)
    ap.add_argument("--max-depth", type=int, default=20)
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args()
    ff = train(a.pairs, a.max_depth, a.jobs)
    ff.save(a.out)
    print("saved %s: %d trees, %d nodes" % (a.out, ff.n_trees, ff.n_nodes), flush=True)


if __name__ == "__main__":
    main()
