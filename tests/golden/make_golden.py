"""Generates the committed golden fixtures from the reference itself.

Run in a container that has the reference sources (it builds
oracle/_ref/libcbmv_ref_cpu.so from them, see oracle/Makefile):

    python tests/golden/make_golden.py

Writes tests/golden/ref_cpu_small.npz: two seeded small stereo pairs and the
reference's own outputs of every matcher (cpp/matchers/matchers.cpp) and a
seeded subset of the rows of the feature assembly of test.py:521-595
(restated glue over the reference's compiled featextract), so the oracle can
be pinned where the reference is absent.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cbmv_b200 import synth  # noqa: E402
from oracle import glue, ref  # noqa: E402

CASES = [dict(seed=21, width=48, height=36, ndisp=12, planes=3, dmin=2, dmax=9),
         dict(seed=22, width=41, height=30, ndisp=14, planes=4, dmin=1, dmax=11)]
FEATURE_ROWS = 3000  # a seeded subset of the [H*W*D, 20] feature rows is kept


def main():
    out = {}
    for k, c in enumerate(CASES):
        L, R, gt, _ = synth.make_pair(**c)
        D = c["ndisp"]
        out["L%d" % k], out["R%d" % k] = L, R
        out["census%d" % k] = ref.mtc.census(L, R, D, 11)
        out["ncc%d" % k] = ref.mtc.nccNister(L, R, D, 3)
        sl, sr = ref.mtc.sobel(L), ref.mtc.sobel(R)
        out["sobelL%d" % k] = sl
        out["sadsob%d" % k] = ref.mtc.sadsob(sl, sr, D, 5)
        out["zsad%d" % k] = ref.mtc.zsad(L, R, D, 5)
        costs = glue.get_costs(ref.mtc, ref.fte, L, R, D)
        feats = glue.extract_features_lr(ref.fte, *costs)
        rows = np.sort(np.random.default_rng(k).choice(feats.shape[0], FEATURE_ROWS, replace=False))
        out["feature_rows%d" % k] = rows.astype(np.int64)
        out["features%d" % k] = feats[rows]
        out["D%d" % k] = np.int32(D)
    path = os.path.join(HERE, "ref_cpu_small.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
