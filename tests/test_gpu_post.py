"""CUDA post-processing kernels against the oracle's restatement of
cpp/post/post.cu.  Kernels whose reference arithmetic is float32 are
compared exactly on float32-representable inputs; SGM, whose reference sums
are float64, within a stated tolerance."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene(small_pair):
    from oracle import glue
    L, R, _, _ = small_pair
    imgl, imgr = glue.normalise_images(L, R)
    rng = np.random.default_rng(2)
    H, W = L.shape
    D = 24
    vol = rng.random((H, W, D)).astype(np.float32)  # [H,W,D], exactly representable
    return imgl, imgr, vol, D


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _crosses(oracle_cpu, imgl, imgr, L1=6):
    o = oracle_cpu.post
    a, b = o.CUDA_float_array(imgl), o.CUDA_float_array(imgr)
    lc, rc = o.CUDA_float_array(np.zeros(1)), o.CUDA_float_array(np.zeros(1))
    o.cross(a, lc, L1, .07)
    o.cross(b, rc, L1, .07)
    return lc.a, rc.a


def test_cross_exact(gpu, oracle_cpu, scene):
    from cbmv_b200 import _lib
    imgl, imgr, _, _ = scene
    lc, _ = _crosses(oracle_cpu, imgl, imgr)
    H, W = imgl.shape
    out = torch.empty((4, H, W), device="cuda")
    im = _t(imgl)
    _lib.call("cbmv_cross", im.data_ptr(), H, W, 6, 0.07, out.data_ptr(), None)
    assert np.array_equal(out.cpu().numpy(), lc)


@pytest.mark.parametrize("direction", [-1, 1])
def test_cbca_exact_both_layouts(gpu, oracle_cpu, scene, direction):
    from cbmv_b200 import _lib
    imgl, imgr, vol, D = scene
    lc, rc = _crosses(oracle_cpu, imgl, imgr)
    H, W = imgl.shape
    dhw = np.ascontiguousarray(np.transpose(vol, (2, 0, 1)))
    ref = np.empty(dhw.shape, np.float64)
    dhw64 = dhw.astype(np.float64)
    oracle_cpu.lib().orc_cbca(lc.ctypes.data, rc.ctypes.data, dhw64.ctypes.data, D, H, W,
                              direction, ref.ctypes.data)
    tl, tr = _t(lc), _t(rc)
    for layout, src in ((_lib.DHW, dhw), (_lib.HWD, vol)):
        ts = _t(src)
        out = torch.empty_like(ts)
        _lib.call("cbmv_cbca", tl.data_ptr(), tr.data_ptr(), ts.data_ptr(), H, W, D, layout,
                  direction, out.data_ptr(), None)
        got = out.cpu().numpy()
        if layout == _lib.HWD:
            got = np.transpose(got, (2, 0, 1))
        assert np.array_equal(got, ref.astype(np.float32))


def test_sgm_close(gpu, oracle_cpu, scene):
    from cbmv_b200 import _lib
    imgl, imgr, vol, D = scene
    H, W = imgl.shape
    ref = np.zeros((H, W, D))
    vol64 = vol.astype(np.float64)
    oracle_cpu.lib().orc_sgm(imgl.ctypes.data, imgr.ctypes.data, vol64.ctypes.data, H, W, D,
                             1.3, 10, .12, 1.4, 2.2, 3, -1, ref.ctypes.data)
    out = torch.zeros((H, W, D), device="cuda")
    a, b, v = _t(imgl), _t(imgr), _t(vol)
    _lib.call("cbmv_sgm", a.data_ptr(), b.data_ptr(), v.data_ptr(), H, W, D, 1.3, 10,
              .12, 1.4, 2.2, 3, -1, out.data_ptr(), None)
    # float32 path sums vs the reference's float64 sums: 4 directions x W steps
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=2e-5, atol=2e-4)


@pytest.mark.parametrize("D", [68, 128, 200, 256])
@pytest.mark.parametrize("direction", [-1, 1])
def test_sgm_consecutive_lanes_equal_strided(gpu, scene, D, direction):
    """The SGM scan with KPL consecutive disparities per lane (float4 path
    costs, taken for D % 4 == 0 in (64, 512] on 16-byte aligned volumes:
    KPL 4 and 8 here) and the strided scan (lane = d mod 32, taken
    otherwise) agree bit for bit: same per-element arithmetic in the same
    order.  An input volume 4 bytes off a 16-byte boundary selects the
    strided scan."""
    from cbmv_b200 import _lib
    imgl, imgr, _, _ = scene
    H, W = imgl.shape
    rng = np.random.default_rng(D)
    vol = rng.random((H, W, D)).astype(np.float32)
    a, b = _t(imgl), _t(imgr)
    buf = torch.zeros(H * W * D + 4, device="cuda")
    outs = []
    for off in (0, 1):  # 16-byte aligned (consecutive lanes), then 4 bytes off (strided)
        v = buf[off:off + H * W * D]
        v.copy_(torch.from_numpy(vol.reshape(-1)).cuda())
        assert (v.data_ptr() % 16 == 0) == (off == 0)
        out = torch.zeros((H, W, D), device="cuda")
        _lib.call("cbmv_sgm", a.data_ptr(), b.data_ptr(), v.data_ptr(), H, W, D, 1.3, 10,
                  .12, 1.4, 2.2, 3, direction, out.data_ptr(), None)
        outs.append(out.cpu().numpy())
    assert np.isfinite(outs[0]).all()
    assert np.array_equal(outs[0], outs[1])


def test_wta_subpixel_median_mean2d_exact(gpu, oracle_cpu, scene):
    from oracle import glue
    from cbmv_b200 import _lib
    imgl, _, vol, D = scene
    H, W = imgl.shape
    dhw = np.ascontiguousarray(np.transpose(vol, (2, 0, 1))).astype(np.float64)
    d_ref = oracle_cpu.wta(dhw)
    d = torch.empty((H, W), device="cuda")
    tv = _t(vol)
    _lib.call("cbmv_wta", tv.data_ptr(), H, W, D, _lib.HWD, d.data_ptr(), None)
    assert np.array_equal(d.cpu().numpy(), d_ref)
    sub_ref = np.empty((H, W), np.float32)
    oracle_cpu.lib().orc_subpixel(d_ref.ctypes.data, dhw.ctypes.data, H, W, D, sub_ref.ctypes.data)
    sub = torch.empty((H, W), device="cuda")
    _lib.call("cbmv_subpixel", d.data_ptr(), tv.data_ptr(), H, W, D, _lib.HWD, sub.data_ptr(), None)
    assert np.array_equal(sub.cpu().numpy(), sub_ref)
    med_ref = np.empty((H, W), np.float32)
    oracle_cpu.lib().orc_median2d(sub_ref.ctypes.data, H, W, 3, med_ref.ctypes.data)
    med = torch.empty((H, W), device="cuda")
    _lib.call("cbmv_median2d", sub.data_ptr(), H, W, 3, med.data_ptr(), None)
    assert np.array_equal(med.cpu().numpy(), med_ref)
    k = glue.gaussian(2.2)
    mean_ref = np.empty((H, W), np.float32)
    oracle_cpu.lib().orc_mean2d(med_ref.ctypes.data, H, W, k.ctypes.data, 15, np.float32(1.3),
                                mean_ref.ctypes.data)
    mean = torch.empty((H, W), device="cuda")
    tk = _t(k)
    _lib.call("cbmv_mean2d", med.data_ptr(), H, W, tk.data_ptr(), 15, 1.3, mean.data_ptr(), None)
    np.testing.assert_allclose(mean.cpu().numpy(), mean_ref, rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("D", [24, 128, 160])
def test_wta_first_minimum_ties_and_inf_rows(gpu, D):
    """Winner-take-all is np.argmin along d (test.py:408-409): the first of
    tied minima, 0 for a row of +inf, at D <= 128 (one reduction of the
    minimum and one of its first index) and above (the per-lane loop)."""
    from cbmv_b200 import _lib
    rng = np.random.default_rng(D)
    H, W = 6, 40
    vol = rng.integers(0, 5, (H, W, D)).astype(np.float32)  # many ties
    vol[0, 0, :] = np.inf
    vol[0, 1, :] = 7.0
    vol[0, 2, :] = np.inf
    vol[0, 2, D - 1] = 1.0  # the only finite value, last
    ref = np.argmin(vol, axis=2).astype(np.float32)
    d = torch.empty((H, W), device="cuda")
    _lib.call("cbmv_wta", _t(vol).data_ptr(), H, W, D, _lib.HWD, d.data_ptr(), None)
    assert np.array_equal(d.cpu().numpy(), ref)


def test_lr_check_and_interpolation_exact(gpu, oracle_cpu):
    from cbmv_b200 import _lib
    rng = np.random.default_rng(4)
    H, W, D = 30, 50, 16
    d0 = rng.integers(0, D, (H, W)).astype(np.float32)
    d1 = np.where(rng.random((H, W)) < 0.7, np.roll(d0, 3, axis=1), rng.integers(0, D, (H, W))).astype(np.float32)
    o_ref = np.empty((H, W), np.float32)
    oracle_cpu.lib().orc_outlier_detection(d0.ctypes.data, d1.ctypes.data, H, W, D, o_ref.ctypes.data)
    o = torch.empty((H, W), device="cuda")
    t0, t1, to = _t(d0), _t(d1), _t(o_ref)
    _lib.call("cbmv_outlier_detection", t0.data_ptr(), t1.data_ptr(), H, W, D, o.data_ptr(), None)
    assert np.array_equal(o.cpu().numpy(), o_ref)
    assert set(np.unique(o_ref)) <= {0.0, 1.0, 2.0} and len(np.unique(o_ref)) == 3
    for name, fn in (("cbmv_interpolate_mismatch", "orc_interpolate_mismatch"),
                     ("cbmv_interpolate_occlusion", "orc_interpolate_occlusion")):
        ref = np.empty((H, W), np.float32)
        getattr(oracle_cpu.lib(), fn)(d0.ctypes.data, o_ref.ctypes.data, H, W, ref.ctypes.data)
        out = torch.empty((H, W), device="cuda")
        _lib.call(name, t0.data_ptr(), to.data_ptr(), H, W, out.data_ptr(), None)
        assert np.array_equal(out.cpu().numpy(), ref), name


def test_dropin_post_module_runs_reference_driver(gpu, oracle_cpu, scene):
    """glue.postprocessing_mem (test.py:341-449 restated) over the drop-in
    post module vs over the oracle's post: disparity maps agree."""
    from oracle import glue
    from cbmv_b200 import post
    imgl, imgr, vol, D = scene
    cost = vol.astype(np.float64)
    ref = glue.postprocessing_mem(oracle_cpu.post, imgl, imgr, cost, -1)
    got = glue.postprocessing_mem(post, imgl, imgr, cost, -1)
    close = np.mean(np.abs(got - ref) <= 0.5)
    print("drop-in post module vs oracle post, _mem chain: within 0.5 px %.5f" % close)
    assert close >= 0.999, close
    ref_i = glue.postprocessing_mem_interp(oracle_cpu.post, oracle_cpu.fte, imgl, imgr, cost, -1)
    from cbmv_b200 import libfeatextract as fte
    got_i = glue.postprocessing_mem_interp(post, fte, imgl, imgr, cost, -1)
    close_i = np.mean(np.abs(got_i - ref_i) <= 0.5)
    print("drop-in post module vs oracle post, _interp chain: within 0.5 px %.5f" % close_i)
    assert close_i >= 0.999, close_i


@pytest.mark.parametrize("direction,L1,D70", [(-1, 6, False), (1, 6, False), (-1, 9, False), (-1, 6, True),
                                               (1, 6, True)])
def test_cbca_separable_matches_model_exactly(gpu, oracle_cpu, scene, direction, L1, D70):
    """cbmv_cbca_separable (the fused pipeline's default CBCA: with L1 <= 6
    its supports precomputed once and read by the pass; with L1 = 9 the
    arms are built with L1 = 9, reach up to 8 pixels and the pass reads the
    arms themselves) against the oracle's float32 model of its summation
    order with a halo of L1 - 1: bit-exact; against the reference-order
    cbca: relative 1e-5.  D70: 70 disparities (three 32-wide disparity
    tiles, the last one partial)."""
    from cbmv_b200 import _lib
    from oracle import post_model
    imgl, imgr, vol, D = scene
    if D70:
        D = 70
        vol = np.random.default_rng(70).random((imgl.shape[0], imgl.shape[1], D)).astype(np.float32)
    lc, rc = _crosses(oracle_cpu, imgl, imgr, L1)
    H, W = imgl.shape
    reach = max(int(np.max(np.abs(lc[0] - np.arange(W)[None, :]))), int(np.max(np.abs(lc[2] - np.arange(H)[:, None]))))
    assert reach == L1, reach  # the longest arm ends L1 pixels away (its last pixel at L1 - 1)
    tl, tr, ts = _t(lc), _t(rc), _t(vol)
    out = torch.empty_like(ts)
    _lib.call("cbmv_cbca_separable", tl.data_ptr(), tr.data_ptr(), ts.data_ptr(), H, W, D, L1,
              direction, out.data_ptr(), None)
    ref_order = torch.empty_like(ts)
    _lib.call("cbmv_cbca", tl.data_ptr(), tr.data_ptr(), ts.data_ptr(), H, W, D, _lib.HWD, direction,
              ref_order.data_ptr(), None)
    got = out.cpu().numpy()
    assert np.array_equal(got, post_model.cbca_separable(lc, rc, vol, direction, L1 - 1))
    ro = ref_order.cpu().numpy()
    assert np.max(np.abs(got - ro) / np.maximum(np.abs(ro), 1e-30)) <= 1e-5
