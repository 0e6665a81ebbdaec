"""CUDA matchers against the oracle (bit-exact in float64), through the
drop-in module and the C ABI, over layouts, output dtypes and edge sizes."""
import numpy as np
import pytest

from conftest import rand_pair

pytestmark = pytest.mark.gpu

RAND_MAX = 2147483647.0


def _cases(small_pair):
    L, R, _, _ = small_pair
    yield "synthetic", L, R, 24
    yield "noise+flat", *rand_pair(3, 41, 67, flat=True), 30
    yield "D>W", *rand_pair(4, 20, 18, flat=False), 32
    yield "tiny", *rand_pair(5, 12, 12), 4


def test_census_ncc_zsad_sobel_sadsob_bitexact(gpu, oracle_cpu, small_pair):
    from cbmv_b200 import libmatchers as mtc
    for name, L, R, D in _cases(small_pair):
        o = oracle_cpu.mtc
        assert np.array_equal(mtc.census(L, R, D, 11), o.census(L, R, D, 11)), name
        assert np.array_equal(mtc.nccNister(L, R, D, 3), o.nccNister(L, R, D, 3)), name
        assert np.array_equal(mtc.zsad(L, R, D, 5), o.zsad(L, R, D, 5)), name
        sl, sr = mtc.sobel(L), mtc.sobel(R)
        assert np.array_equal(sl, o.sobel(L)), name
        assert np.array_equal(mtc.sadsob(sl, sr, D, 5), o.sadsob(o.sobel(L), o.sobel(R), D, 5)), name


def test_layouts_and_float32(gpu, oracle_cpu, small_pair):
    from cbmv_b200 import libmatchers as mtc
    L, R, _, _ = small_pair
    D = 24
    ref = oracle_cpu.mtc.nccNister(L, R, D, 3)  # [D,H,W]
    hwd = mtc.nccNister(L, R, D, 3, layout="HWD")
    assert np.array_equal(hwd, np.transpose(ref, (1, 2, 0)))
    f32 = mtc.nccNister(L, R, D, 3, dtype=np.float32)
    assert f32.dtype == np.float32 and np.array_equal(f32, ref.astype(np.float32))
    c32 = mtc.census(L, R, D, 11, dtype=np.float32, layout="DHW")
    cref = oracle_cpu.mtc.census(L, R, D, 11)
    assert np.array_equal(c32, np.transpose(cref, (2, 0, 1)).astype(np.float32))
    assert c32.max() == np.float32(RAND_MAX)
    # the [H,W,D] float32 census (the learned path's layout, its own kernel),
    # also with more than 128 disparities (two disparity blocks)
    for d in (D, 140):
        h32 = mtc.census(L, R, d, 11, dtype=np.float32, layout="HWD")
        assert np.array_equal(h32, oracle_cpu.mtc.census(L, R, d, 11).astype(np.float32)), d


def test_device_tensors_stay_on_device(gpu, oracle_cpu, small_pair):
    import torch
    from cbmv_b200 import libmatchers as mtc
    L, R, _, _ = small_pair
    l, r = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    out = mtc.census(l, r, 16, 11)
    assert isinstance(out, torch.Tensor) and out.is_cuda
    assert np.array_equal(out.cpu().numpy(), oracle_cpu.mtc.census(L, R, 16, 11))


def test_windows(gpu, oracle_cpu):
    from cbmv_b200 import libmatchers as mtc
    L, R = rand_pair(8, 30, 50)
    for w in (1, 3, 7):
        assert np.array_equal(mtc.census(L, R, 9, w), oracle_cpu.mtc.census(L, R, 9, w))
        assert np.array_equal(mtc.zsad(L, R, 9, w), oracle_cpu.mtc.zsad(L, R, 9, w))
        assert np.array_equal(mtc.nccNister(L, R, 9, w), oracle_cpu.mtc.nccNister(L, R, 9, w))


def test_bad_arguments_raise(gpu):
    from cbmv_b200 import libmatchers as mtc
    from cbmv_b200._lib import CbmvError
    L, R = rand_pair(1, 20, 20)
    with pytest.raises(CbmvError):
        mtc.census(L, R, 8, 13)  # 169 bits > 128
    with pytest.raises(CbmvError):
        mtc.zsad(L, R, 8, 4)


@pytest.mark.parametrize("D", [24, 130])
def test_learned_path_f32_volumes(gpu, small_pair, D):
    """The learned path's float32 volumes (strip kernels for NCC, SAD-on-Sobel
    and ZSAD) against the float64 matchers rounded to float32: census, NCC
    and SAD-on-Sobel bit-exact, ZSAD within one float32 unit."""
    from cbmv_b200 import libmatchers as mtc, libfeatextract as fte
    from cbmv_b200.pipeline import StereoPipeline
    L, R, _, _ = small_pair
    vols = StereoPipeline().volumes_f32(L, R, D).cpu().numpy()
    ref = [mtc.census(L, R, D, 11), fte.swap_axes(mtc.nccNister(L, R, D, 3)),
           fte.swap_axes(mtc.sadsob(mtc.sobel(L), mtc.sobel(R), D, 5)), fte.swap_axes(mtc.zsad(L, R, D, 5))]
    for m in range(3):
        assert np.array_equal(vols[m], ref[m].astype(np.float32)), m
    z, zr = vols[3], ref[3].astype(np.float32)
    ulp = np.abs(z.view(np.int32).astype(np.int64) - zr.view(np.int32).astype(np.int64))
    assert ulp.max() <= 1
    assert np.mean(ulp == 0) > 0.999
