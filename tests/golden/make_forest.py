"""Train the random-forest fixture used by the tests and the benchmark.

Follows the reference's training path (train.py:277-293 over
train.py:100-273): for each training pair, one positive and two negative
disparities per ground-truth pixel, the 20 CBMV features of each, label
[1, 0, 0]; then RandomForestClassifier(n_estimators=50, min_samples_leaf=700)
with max_depth=20 (the benchmark workload's forest) and a fixed random_state.
The training pairs are the seeded synthetic 694x554, D=128 pairs 1000..1029.

Features come from the oracle (oracle/oracle.c, bit-identical to the
reference's C++ — see tests/test_oracle.py), and the negative draws from the
oracle's counter-based generator keyed by the pair's seed, since the
reference's rand() inside OpenMP is not reproducible.

Usage:  python tests/golden/make_forest.py [--pairs 30] [--jobs N] [--out PATH]
Writes a FlatForest .npz (cbmv_b200.forest).  The default output,
tests/golden/forest_694x554.npz (16.6 MB), is committed: bench.py times the
forest arm with it and judges the learned classifier's bad-2.0 against it.
Training is deterministic (fixed seeds, random_state=0), so re-running this
script reproduces the file.
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cbmv_b200 import synth  # noqa: E402
from cbmv_b200.forest import FlatForest  # noqa: E402
from oracle import cpu, glue  # noqa: E402

DEFAULT_OUT = os.path.join(HERE, "forest_694x554.npz")


def samples_for_pair(seed):
    L, R, gt, _ = synth.pair_694x554(seed)
    return glue.create_samples_mem(
        cpu.mtc, cpu.fte, L, R, gt, 128,
        lambda g, nd: cpu.fte.generate_d_indices(g, nd, 1, seed=seed)).astype(np.float32)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=30)
    ap.add_argument("--jobs", type=int, default=os.cpu_count())
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--max-depth", type=int, default=20)
    a = ap.parse_args()
    from sklearn.ensemble import RandomForestClassifier
    t0 = time.time()
    S = np.concatenate([samples_for_pair(s) for s in synth.RF_TRAIN_SEEDS[:a.pairs]])
    print("samples %s in %.1fs" % (S.shape, time.time() - t0), flush=True)
    t0 = time.time()
    rf = RandomForestClassifier(n_estimators=50, min_samples_leaf=700, max_depth=a.max_depth,
                                n_jobs=a.jobs, random_state=0)
    rf.fit(S[:, :20], S[:, 20])
    print("fit in %.1fs" % (time.time() - t0), flush=True)
    ff = FlatForest.from_sklearn(rf)
    ff.save(a.out)
    sizes = ff.tree_sizes()
    print("saved %s: %d trees, %d nodes (mean %.0f, max %d per tree)"
          % (a.out, ff.n_trees, ff.n_nodes, sizes.mean(), sizes.max()), flush=True)


if __name__ == "__main__":
    main()
