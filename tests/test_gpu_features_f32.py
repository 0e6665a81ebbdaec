"""The learned classifier's own features: the 20 float32 values per (pixel,
d) that the fused network kernel of cbmv_run_mlp forms from its float32
cost volumes and float32 row statistics (read back through
cbmv_ctx_features_f32_at, which runs the kernel's feature code) against the
reference's float64 features (test.py:521-595, featextract.cpp:254-450),
computed by the oracle (itself bit-exact against the reference build).

Bar: |f32 - ref| <= 1e-5 |ref| + 1e-16, i.e. 1e-5 relative for every
feature above 1e-11.  The absolute floor covers likelihoods of about
exp(-25) and below only: their argument x = -(c - m)^2 / sigma is formed
from the float32 roundings of c and m (for NCC, sigma = 0.02 and costs in
[-1, 1] stored with a spacing of 6e-8, that alone moves exp() by about
9e-6 |c - m| relative) and the approximate exponential adds about |x| 6e-8,
so far from the row minimum the relative error reaches 1e-5 (measured:
1.4e-5 at 1.4e-17).  Such a feature enters the network as (x - mu) inv_sd
rounded to f16, where a relative change of 1e-4 in x is invisible.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NAMES = ["census", "ncc", "sob", "sad"]
COLUMNS = (NAMES + ["ratio_" + n for n in NAMES] + ["lik_" + n for n in NAMES] +
           ["r_ratio_" + n for n in NAMES] + ["r_lik_" + n for n in NAMES])


@pytest.mark.parametrize("shape", ["694x160_D128", "97x53_D37", "120x72_D68"])
def test_learned_features_within_1e5_relative(gpu, oracle_cpu, shape):
    """Cases: the headline width and disparity count; D = 37 (the row
    statistics' general kernels, D not a multiple of 4); D = 68 (their
    float4 kernels with part of each warp's lanes idle)."""
    from oracle import glue
    from cbmv_b200 import synth
    from cbmv_b200.pipeline import StereoPipeline
    if shape == "694x160_D128":
        L, R, _, _ = synth.pair_694x554(seed=0)
        L, R, D = L[:160].copy(), R[:160].copy(), 128
        bands = [(0, 3), (5, 7), (60, 62), (154, 160)]  # borders (sentinel rows and columns) and interior
    elif shape == "97x53_D37":
        L, R, _, _ = synth.make_pair(seed=7, width=97, height=53, ndisp=37, planes=4, dmin=2, dmax=33)
        D = 37
        bands = [(0, 53)]
    else:
        L, R, _, _ = synth.make_pair(seed=8, width=120, height=72, ndisp=68, planes=4, dmin=2, dmax=60)
        D = 68
        bands = [(0, 72)]
    H, W = L.shape
    vols = glue.get_costs(oracle_cpu.mtc, oracle_cpu.fte, L, R, D)
    pipe = StereoPipeline()
    worst = np.zeros(20)
    for a, b in bands:
        ref = glue.extract_features_lr(oracle_cpu.fte, *(v[a:b] for v in vols))
        idx = np.arange(a * W * D, b * W * D, dtype=np.int64)
        got = pipe.features_at(L, R, D, idx, learned=True).cpu().numpy().astype(np.float64)
        err = np.abs(got - ref)
        ok = err <= 1e-5 * np.abs(ref) + 1e-16
        big = np.abs(ref) >= 1e-11
        rel = np.where(big, err / np.maximum(np.abs(ref), 1e-300), 0.0)
        worst = np.maximum(worst, rel.max(axis=0))
        bad = np.argwhere(~ok)
        if len(bad):
            i, k = bad[0]
            pytest.fail("%s rows %d..%d: %d features off, first %s at sample %d: %.9g vs %.9g"
                        % (shape, a, b, len(bad), COLUMNS[k], idx[i], got[i, k], ref[i, k]))
    print("%s: max relative error per column (|ref| >= 1e-11): %s"
          % (shape, ", ".join("%s %.1e" % (c, w) for c, w in zip(COLUMNS, worst))))
