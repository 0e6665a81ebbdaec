"""CUDA feature extraction against the oracle: the reference's layout and
confidence functions (float64) and the fused 20-feature kernel (float32 of
the reference's float64 features)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def costs(oracle_cpu, small_pair):
    from oracle import glue
    L, R, gt, _ = small_pair
    return glue.get_costs(oracle_cpu.mtc, oracle_cpu.fte, L, R, 24)


def test_layout_ops_exact(gpu, oracle_cpu, costs):
    from cbmv_b200 import libfeatextract as fte
    o = oracle_cpu.fte
    v = costs[1]
    assert np.array_equal(fte.get_right_cost(v), o.get_right_cost(v))
    assert np.array_equal(fte.get_left_cost(v), o.get_left_cost(v))
    dhw = o.swap_axes_back(v)
    assert np.array_equal(fte.swap_axes_back(v), dhw)
    assert np.array_equal(fte.swap_axes(dhw), v)
    p4 = np.random.default_rng(0).random(v.shape + (2,))
    assert np.array_equal(fte.get_cost(p4), o.get_cost(p4))


def test_confidences(gpu, oracle_cpu, costs):
    from cbmv_b200 import libfeatextract as fte
    o = oracle_cpu.fte
    for v, e, s in zip(costs, (.01, 1.01, .01, .01), (128.0, 0.02, 2e4, 2e4)):
        flat = v.reshape(-1, v.shape[2])
        assert np.array_equal(fte.extract_ratio(flat, e), o.extract_ratio(flat, e))
        # the denominator's summation order may move it by an ulp of float64
        np.testing.assert_allclose(fte.extract_likelihood(flat, s), o.extract_likelihood(flat, s),
                                   rtol=1e-13, atol=1e-300)
        vr = o.get_right_cost(v).reshape(-1, v.shape[2])
        assert np.array_equal(fte.extract_ratio(vr, e), o.extract_ratio(vr, e))


def test_training_form_and_sampling(gpu, oracle_cpu, costs, small_pair):
    from cbmv_b200 import libfeatextract as fte
    o = oracle_cpu.fte
    _, _, gt, _ = small_pair
    g = np.clip(np.rint(gt.reshape(-1)), 0, 20).astype(np.int32)
    s_gpu = fte.generate_d_indices(g, 24, 1, seed=5)
    s_cpu = o.generate_d_indices(g, 24, 1, seed=5)
    assert np.array_equal(s_gpu, s_cpu)
    flat = costs[3].reshape(-1, 24)
    assert np.array_equal(fte.get_samples(flat, s_gpu), o.get_samples(flat, s_cpu))
    assert np.array_equal(fte.extract_ratio(flat, s_gpu, .01), o.extract_ratio(flat, s_cpu, .01))
    np.testing.assert_allclose(fte.extract_likelihood(flat, s_gpu, 2e4),
                               o.extract_likelihood(flat, s_cpu, 2e4), rtol=1e-13)
    assert np.array_equal(fte.generate_labels(s_gpu), o.generate_labels(s_cpu))
    from cbmv_b200._lib import CbmvError
    with pytest.raises(CbmvError):
        fte.generate_d_indices(np.array([22], np.int32), 24, 1)  # gt = maxd - 2


def test_fused_features_match_reference_assembly(gpu, oracle_cpu, costs):
    """Fused kernel == float32(test.py:521-595 features) (tolerance 1e-6 rel
    covers an occasional ulp of exp; in practice the columns are equal)."""
    from oracle import glue
    from cbmv_b200 import libfeatextract as fte
    ref = glue.extract_features_lr(oracle_cpu.fte, *costs).astype(np.float32)
    got = fte.features(*costs)
    assert got.shape == ref.shape
    np.testing.assert_allclose(got, ref, rtol=1e-6, atol=1e-30)
    exact = np.mean(np.all(got == ref, axis=1))
    assert exact > 0.9999, exact


def test_gpu_training_samples_equal_the_cpu_path(gpu, oracle_cpu):
    """Training-sample emission on the GPU (cbmv_b200.train_rf.emit_samples)
    against the reference's Training.__create_samples_mem restated over the
    oracle with the same draws: features and labels bit-exact (as the
    float32 sklearn fits on)."""
    from cbmv_b200 import synth
    from cbmv_b200.pipeline import StereoPipeline
    from cbmv_b200.train_rf import emit_samples
    from oracle import glue
    L, R, gt, _ = synth.make_pair(seed=21, width=110, height=70, ndisp=24, planes=4, dmin=2, dmax=19)
    gt = gt.copy()
    gt[3, 5:9] = np.inf   # invalid ground truth is skipped, as train.py:105-107 does
    gt[10, 2] = -1.0
    X, y = emit_samples(StereoPipeline(), L, R, gt, 24, seed=21)
    S = glue.create_samples_mem(oracle_cpu.mtc, oracle_cpu.fte, L, R, gt, 24,
                                lambda g, nd: oracle_cpu.fte.generate_d_indices(g, nd, 1, seed=21))
    assert X.shape == (S.shape[0], 20)
    assert np.array_equal(X, S[:, :20].astype(np.float32))
    assert np.array_equal(y, S[:, 20].astype(np.int32))
