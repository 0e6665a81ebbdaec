"""Flat forest packing: the device layout walked on the host equals
sklearn's own apply / predict_proba."""
import numpy as np
import pytest

from cbmv_b200.forest import FlatForest, LEAF_FLAG


def _walk(blocks, leafv, offs, X):
    """The device walk of csrc/rf.cuh restated in numpy."""
    N, T = X.shape[0], len(offs) - 1
    thr = blocks[:, 0:3].view(np.float32)
    feats = blocks[:, 3].astype(np.int64)
    child = blocks[:, 4:8].astype(np.int64)
    flag = int(LEAF_FLAG)
    rows = np.arange(N)
    p = np.zeros((N, 2))
    leaves = np.zeros((N, T), np.int64)
    for t in range(T):
        b = np.full(N, offs[t], np.int64)
        leaf = np.full(N, -1, np.int64)
        for _ in range(40):
            act = leaf < 0
            if not act.any():
                break
            bb = b[act]
            r = rows[act]
            f0 = feats[bb] & 0xFF
            is0 = f0 == 0xFF
            x0 = X[r, np.where(is0, 0, f0)]
            right = ~(x0 <= thr[bb, 0])
            n = np.where(right, 2, 1)
            fn = (feats[bb] >> (8 * n)) & 0xFF
            isn = fn == 0xFF
            tn = thr[bb, n]
            xn = X[r, np.where(isn, 0, fn)]
            right2 = ~(xn <= tn)
            slot = 2 * (n - 1) + np.where(isn, 0, right2.astype(np.int64))
            c = child[bb, slot]
            nl = np.where(is0, child[bb, 0] | flag, np.where(isn, c | flag, c))
            done = (nl & flag) != 0
            idx = np.nonzero(act)[0]
            leaf[idx[done]] = nl[done] & (flag - 1)
            b[idx[~done]] = nl[~done]
        p += leafv[leaf]
        leaves[:, t] = leaf
    return p / T, leaves


@pytest.fixture(scope="module")
def rf_and_data():
    from sklearn.ensemble import RandomForestClassifier
    rng = np.random.default_rng(1)
    X = rng.normal(size=(6000, 20)).astype(np.float32)
    X[:, 0] = np.round(X[:, 0] * 10)  # integer-valued feature: many ties at thresholds
    y = ((X[:, 0] > 2) ^ (X[:, 5] > 0.3)).astype(float)
    rf = RandomForestClassifier(n_estimators=9, min_samples_leaf=15, max_depth=12, random_state=3,
                                n_jobs=1).fit(X, y)
    return rf, rng.normal(size=(3000, 20)).astype(np.float32)


def test_pack_walk_equals_sklearn(rf_and_data):
    rf, Xt = rf_and_data
    Xt[:, 0] = np.round(Xt[:, 0] * 10)
    ff = FlatForest.from_sklearn(rf)
    blocks, leafv, offs, leaf_node = ff.pack()
    assert blocks.shape[1] == 8 and offs[-1] == blocks.shape[0]
    p, leaves = _walk(blocks, leafv, offs, Xt)
    assert np.array_equal(leaf_node[leaves], np.stack([e.apply(Xt) for e in rf.estimators_], 1))
    np.testing.assert_allclose(p, rf.predict_proba(Xt), rtol=1e-15, atol=1e-15)


def test_threshold_rounding_is_exact():
    # t32 must be the largest float32 <= the float64 threshold
    from cbmv_b200.forest import FlatForest
    thr = np.array([0.1, 1.0, -2.5e-8, 3.0000001192092896, 1e30, -1e-45])
    ff = FlatForest(roots=[0], feature=np.r_[[0] * 6, [-2] * 7], threshold=np.r_[thr, [-2.0] * 7],
                    left=np.r_[[1, 3, 5, 7, 9, 11], [-1] * 7], right=np.r_[[2, 4, 6, 8, 10, 12], [-1] * 7],
                    value0=np.linspace(0, 1, 13))
    # only the root is reachable; check the rounding rule directly on every threshold
    t32 = thr.astype(np.float32)
    over = t32.astype(np.float64) > thr
    t32[over] = np.nextafter(t32[over], np.float32(-np.inf))
    assert np.all(t32.astype(np.float64) <= thr)
    assert np.all(np.nextafter(t32, np.float32(np.inf)).astype(np.float64) > thr)
    blocks, _, _, _ = ff.pack()
    assert blocks[0, 0].view(np.float32) == t32[0]


def test_save_load_roundtrip(tmp_path, rf_and_data):
    rf, _ = rf_and_data
    ff = FlatForest.from_sklearn(rf)
    p = tmp_path / "f.npz"
    ff.save(p)
    g = FlatForest.load(p)
    for a in ("roots", "feature", "threshold", "left", "right", "value0", "value1"):
        assert np.array_equal(getattr(ff, a), getattr(g, a))
