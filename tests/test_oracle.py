"""The oracle pinned to the reference: the C restatement (oracle/oracle.c)
against the committed golden vectors made by the reference's own compiled
code (tests/golden/make_golden.py), and, where the reference build exists,
against that build directly on seeded inputs including edge cases."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, rand_pair

GOLD = os.path.join(GOLDEN, "ref_cpu_small.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.mark.parametrize("k", [0, 1])
def test_matchers_equal_reference_golden(oracle_cpu, gold, k):
    L, R, D = gold["L%d" % k], gold["R%d" % k], int(gold["D%d" % k])
    m = oracle_cpu.mtc
    assert np.array_equal(m.census(L, R, D, 11), gold["census%d" % k])
    assert np.array_equal(m.nccNister(L, R, D, 3), gold["ncc%d" % k])
    sl = m.sobel(L)
    assert np.array_equal(sl, gold["sobelL%d" % k])
    assert np.array_equal(m.sadsob(sl, m.sobel(R), D, 5), gold["sadsob%d" % k])
    assert np.array_equal(m.zsad(L, R, D, 5), gold["zsad%d" % k])


@pytest.mark.parametrize("k", [0, 1])
def test_features_equal_reference_golden(oracle_cpu, gold, k):
    from oracle import glue
    L, R, D = gold["L%d" % k], gold["R%d" % k], int(gold["D%d" % k])
    costs = glue.get_costs(oracle_cpu.mtc, oracle_cpu.fte, L, R, D)
    f = glue.extract_features_lr(oracle_cpu.fte, *costs)
    rows = gold["feature_rows%d" % k]
    assert np.array_equal(f[rows], gold["features%d" % k])


def _ref():
    from oracle import ref
    if not ref.cpu_available():
        pytest.skip("reference build oracle/_ref not present")
    return ref


@pytest.mark.parametrize("shape,D,flat", [((40, 57), 16, False), ((23, 31), 40, True),
                                          ((12, 12), 8, False), ((13, 40), 1, False)])
def test_matchers_equal_reference_build(oracle_cpu, shape, D, flat):
    ref = _ref()
    L, R = rand_pair(5, *shape, flat=flat)
    for name, w in [("census", 11), ("nccNister", 3), ("zsad", 5)]:
        a = getattr(ref.mtc, name)(L, R, D, w)
        b = getattr(oracle_cpu.mtc, name)(L, R, D, w)
        assert np.array_equal(a, b), name
    sl, sr = ref.mtc.sobel(L), ref.mtc.sobel(R)
    assert np.array_equal(sl, oracle_cpu.mtc.sobel(L))
    assert np.array_equal(ref.mtc.sadsob(sl, sr, D, 5), oracle_cpu.mtc.sadsob(sl, sr, D, 5))


def test_featextract_equal_reference_build(oracle_cpu, small_pair):
    from oracle import glue
    ref = _ref()
    L, R, gt, _ = small_pair
    cr = glue.get_costs(ref.mtc, ref.fte, L, R, 24)
    cc = glue.get_costs(oracle_cpu.mtc, oracle_cpu.fte, L, R, 24)
    for a, b in zip(cr, cc):
        assert np.array_equal(a, b)
    # whole image and two row batches, as test.py:608-623 slices them
    for lo, hi in [(0, 72), (0, 40), (40, 72)]:
        fa = glue.extract_features_lr(ref.fte, *[v[lo:hi] for v in cr])
        fb = glue.extract_features_lr(oracle_cpu.fte, *[v[lo:hi] for v in cc])
        assert np.array_equal(fa, fb)
    # layout helpers and the training-form confidences
    v = cr[1]
    assert np.array_equal(ref.fte.swap_axes_back(v), oracle_cpu.fte.swap_axes_back(v))
    gti = np.clip(np.rint(gt.reshape(-1, 1)), 0, 20).astype(np.int32)
    s = oracle_cpu.fte.generate_d_indices(gti, 24, 1, seed=3)
    flat = v.reshape(-1, 24)
    assert np.array_equal(ref.fte.get_samples(flat, s), oracle_cpu.fte.get_samples(flat, s))
    assert np.array_equal(ref.fte.extract_ratio(flat, s, 1.01), oracle_cpu.fte.extract_ratio(flat, s, 1.01))
    assert np.array_equal(ref.fte.extract_likelihood(flat, s, .02),
                          oracle_cpu.fte.extract_likelihood(flat, s, .02))
    assert np.array_equal(ref.fte.generate_labels(s), oracle_cpu.fte.generate_labels(s))


def test_training_samples_equal_reference_build(oracle_cpu, small_pair):
    from oracle import glue
    ref = _ref()
    L, R, gt, _ = small_pair
    idx = lambda g, nd: oracle_cpu.fte.generate_d_indices(g, nd, 1, seed=9)
    a = glue.create_samples_mem(ref.mtc, ref.fte, L, R, gt, 24, idx)
    b = glue.create_samples_mem(oracle_cpu.mtc, oracle_cpu.fte, L, R, gt, 24, idx)
    assert np.array_equal(a, b)


def test_d_indices_ranges(oracle_cpu):
    gt = np.arange(0, 30, dtype=np.int32)
    gt = gt[gt != 30 - 2]  # the reference divides by zero at gt = maxd - 2
    s = oracle_cpu.fte.generate_d_indices(gt, 30, 1, seed=1)
    assert np.array_equal(s[:, 0], gt)
    for col in (1, 2):
        assert np.all(np.abs(s[:, col] - gt) > 1)
        assert np.all((s[:, col] >= 0) & (s[:, col] < 30))
    with pytest.raises(ValueError):
        oracle_cpu.fte.generate_d_indices(np.array([28], np.int32), 30, 1)


def test_post_restatement_basics(oracle_cpu):
    """Hand-checked cases of the restated post kernels."""
    from oracle import glue
    H, W = 5, 9
    img = np.zeros((H, W), np.float32)
    img[:, 5:] = 1.0
    res = np.empty((4, H, W), np.float32)
    oracle_cpu.lib().orc_cross(img.ctypes.data, H, W, 6, np.float32(0.07), res.ctypes.data)
    # row 2, x=2: left arm runs off the image at -1; right arm stops at the edge x=5
    assert res[0, 2, 2] == -1 and res[1, 2, 2] == 5
    assert res[2, 2, 2] == -1 and res[3, 2, 2] == 5
    # median / wta
    d = np.arange(H * W, dtype=np.float32).reshape(H, W)
    med = np.empty_like(d)
    oracle_cpu.lib().orc_median2d(d.ctypes.data, H, W, 3, med.ctypes.data)
    assert med[2, 4] == d[2, 4]
    c = np.ones((4, H, W))
    c[2] = 0.5
    c[3] = 0.5
    assert np.all(oracle_cpu.wta(c) == 2)
    k = glue.gaussian(2.2)
    assert k.shape == (15, 15) and np.argmax(k) == np.ravel_multi_index((8, 8), (15, 15))


def test_rf_oracle_matches_sklearn(oracle_cpu):
    from sklearn.ensemble import RandomForestClassifier
    from cbmv_b200.forest import FlatForest
    rng = np.random.default_rng(0)
    X = rng.random((4000, 20)).astype(np.float32)
    y = (X[:, 3] + 0.3 * X[:, 7] > 0.6).astype(float)
    rf = RandomForestClassifier(n_estimators=7, min_samples_leaf=20, max_depth=8, random_state=0,
                                n_jobs=1).fit(X, y)
    ff = FlatForest.from_sklearn(rf)
    Xt = rng.random((2000, 20)).astype(np.float32)
    p0, leaves = oracle_cpu.rf_predict(ff, Xt, return_leaves=True)
    assert np.array_equal(leaves, np.stack([e.apply(Xt) for e in rf.estimators_], 1))
    assert np.array_equal(p0, rf.predict_proba(Xt)[:, 0])


def test_separable_cbca_model_close_to_reference_order(oracle_cpu):
    """The separable summation order (oracle/post_model.py, the fused
    pipeline's default CBCA) against the reference's single running sum:
    relative difference <= 1e-5 everywhere, most elements identical."""
    from oracle import glue, post_model
    from cbmv_b200 import synth
    L, R, _, _ = synth.make_pair(seed=7, width=90, height=60, ndisp=16, planes=4, dmin=2, dmax=14)
    imgl, imgr = glue.normalise_images(L, R)
    o = oracle_cpu.post
    a, b = o.CUDA_float_array(imgl), o.CUDA_float_array(imgr)
    lc, rc = o.CUDA_float_array(np.zeros(1)), o.CUDA_float_array(np.zeros(1))
    o.cross(a, lc, 6, .07)
    o.cross(b, rc, 6, .07)
    H, W, D = 60, 90, 16
    vol = np.random.default_rng(4).random((H, W, D)).astype(np.float32)
    for direction in (-1, 1):
        dhw64 = np.ascontiguousarray(np.transpose(vol, (2, 0, 1))).astype(np.float64)
        ref = np.empty(dhw64.shape, np.float64)
        oracle_cpu.lib().orc_cbca(lc.a.ctypes.data, rc.a.ctypes.data, dhw64.ctypes.data, D, H, W,
                                  direction, ref.ctypes.data)
        ref = np.transpose(ref.astype(np.float32), (1, 2, 0))
        got = post_model.cbca_separable(lc.a, rc.a, vol, direction, 5)
        rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-30)
        assert rel.max() <= 1e-5, rel.max()
        assert np.mean(got == ref) > 0.5


def test_support_words_reproduce_separable_model(oracle_cpu):
    """The pipeline's CBCA runs from precomputed support words (row taps,
    column taps, pixel count, copy flag); restated on the CPU, a pass from
    the words equals the separable model bit for bit, in both directions,
    and the words' counts equal the support sizes."""
    from oracle import glue, post_model
    from cbmv_b200 import synth
    L, R, _, _ = synth.make_pair(seed=9, width=70, height=40, ndisp=20, planes=4, dmin=2, dmax=16)
    imgl, imgr = glue.normalise_images(L, R)
    o = oracle_cpu.post
    a, b = o.CUDA_float_array(imgl), o.CUDA_float_array(imgr)
    lc, rc = o.CUDA_float_array(np.zeros(1)), o.CUDA_float_array(np.zeros(1))
    o.cross(a, lc, 6, .07)
    o.cross(b, rc, 6, .07)
    H, W, D = 40, 70, 20
    vol = np.random.default_rng(5).random((H, W, D)).astype(np.float32)
    for direction in (-1, 1):
        words = post_model.cbca_support_words(lc.a, rc.a, H, W, D, direction)
        copy = (words >> 31) == 1
        x = np.arange(W)[None, :, None] + np.arange(D)[None, None, :] * direction
        assert np.array_equal(copy, np.broadcast_to((x < 0) | (x >= W), copy.shape))
        cnt = (words >> 22) & 0x7F
        assert cnt[~copy].min() >= 1 and cnt.max() <= 121
        got = post_model.cbca_from_words(words, vol)
        ref = post_model.cbca_separable(lc.a, rc.a, vol, direction, 5)
        assert np.array_equal(got, ref)


def test_swap_axis_back_as_shipped_leaves_the_tail_unwritten():
    """The as-shipped restatement of the reference's swap_axis_back (its
    store condition tests Col + d with Col already the pixel,
    post.cu:645-646): disparity d keeps the destination's previous contents
    in its last 16 * floor((d mod 64) / 16) pixels, everything else is the
    transpose."""
    from oracle import cpu
    H, W, D = 3, 7, 70
    rng = np.random.default_rng(0)
    hwd = rng.random((H, W, D))
    prev = rng.random((D, H, W)) + 10  # distinguishable
    a, out = cpu.post_as_shipped.CUDA_double_array(hwd), cpu.post_as_shipped.CUDA_double_array(prev)
    cpu.post_as_shipped.swap_axis_back(a, out)
    meant = np.transpose(hwd, (2, 0, 1)).reshape(D, -1)
    got = out.a.reshape(D, -1)
    for d in range(D):
        k = min(16 * ((d % 64) // 16), H * W)
        assert np.array_equal(got[d, :H * W - k], meant[d, :H * W - k]), d
        assert np.array_equal(got[d, H * W - k:], prev.reshape(D, -1)[d, H * W - k:]), d
    b, out2 = cpu.post.CUDA_double_array(hwd), cpu.post.CUDA_double_array(prev)
    cpu.post.swap_axis_back(b, out2)
    assert np.array_equal(out2.a.reshape(D, -1), meant)
