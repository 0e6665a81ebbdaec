"""GPU random forest against sklearn: bit-exact leaves on identical float32
features, probabilities equal to sklearn's single-job accumulation."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rf():
    from sklearn.ensemble import RandomForestClassifier
    rng = np.random.default_rng(7)
    X = rng.normal(size=(20000, 20)).astype(np.float32)
    X[:, 2] = np.round(X[:, 2] * 50)
    y = ((X[:, 2] > 3) ^ (X[:, 11] > 0.1) | (X[:, 4] > 1.5)).astype(float)
    return RandomForestClassifier(n_estimators=13, min_samples_leaf=30, max_depth=20,
                                  random_state=0, n_jobs=1).fit(X, y)


def test_leaves_and_proba(gpu, rf):
    from cbmv_b200.forest_gpu import GpuForest
    rng = np.random.default_rng(8)
    X = rng.normal(size=(50001, 20)).astype(np.float32)
    X[:, 2] = np.round(X[:, 2] * 50)
    gf = GpuForest.from_sklearn(rf)
    assert np.array_equal(gf.apply(X), np.stack([e.apply(X) for e in rf.estimators_], 1))
    np.testing.assert_array_equal(gf.predict_proba(X), rf.predict_proba(X))


def test_float64_input_cast_like_sklearn(gpu, rf):
    from cbmv_b200.forest_gpu import GpuForest
    X = np.random.default_rng(9).normal(size=(3000, 20))
    gf = GpuForest.from_sklearn(rf)
    np.testing.assert_array_equal(gf.predict_proba(X), rf.predict_proba(X))


def test_cbmv_forest_on_cbmv_features(gpu, oracle_cpu, small_pair):
    """The forest fixture (if trained) on real CBMV features: leaves exact."""
    import os
    from conftest import FOREST_PATH
    if not os.path.exists(FOREST_PATH):
        pytest.skip("forest fixture not trained (tests/golden/make_forest.py)")
    from oracle import glue
    from cbmv_b200.forest import FlatForest
    from cbmv_b200.forest_gpu import GpuForest
    ff = FlatForest.load(FOREST_PATH)
    L, R, _, _ = small_pair
    feats = glue.extract_features_lr(oracle_cpu.fte, *glue.get_costs(oracle_cpu.mtc, oracle_cpu.fte, L, R, 24))
    X = feats[::7].astype(np.float32)
    p_cpu, leaves_cpu = oracle_cpu.rf_predict(ff, X, return_leaves=True)
    gf = GpuForest(ff)
    assert np.array_equal(gf.apply(X), leaves_cpu)
    np.testing.assert_array_equal(gf.predict_proba(X)[:, 0], p_cpu)
