"""cbmv_census_static: the census matcher for callers that cannot allocate
device memory when they call it (an arena or caching allocator owning the
device heap, a graph under capture, a plugin host that only hands out input
and output buffers).  Its descriptors live in a fixed device array instead
of a per-call allocation.  Called through the C ABI, twice in a row on
different pairs, it must return exactly what cbmv_census returns (the costs
are integers, so the tolerance is zero), and reject images larger than its
fixed scratch.  This file is named to run last."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(seed, h, w):
    rng = np.random.default_rng(seed)
    L = rng.integers(0, 256, (h, w), dtype=np.uint8)
    R = np.clip(np.roll(L, -4, axis=1).astype(int) + rng.integers(-3, 4, (h, w)), 0, 255).astype(np.uint8)
    return L, R


def _census(fn, l, r, D, dtype, layout):
    import torch
    from cbmv_b200 import _lib
    H, W = l.shape
    shape = (H, W, D) if layout == _lib.HWD else (D, H, W)
    out = torch.full(shape, -7.0, dtype=torch.float64 if dtype == _lib.F64 else torch.float32,
                     device="cuda")
    rc = getattr(_lib.lib(), fn)(ctypes.c_void_p(l.data_ptr()), ctypes.c_void_p(r.data_ptr()),
                                 H, W, D, 11, ctypes.c_void_p(out.data_ptr()), dtype, layout, None)
    assert rc == 0, _lib.lib().cbmv_last_error()
    return out


def test_static_census_matches_allocating_census_twice():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cbmv_b200 import _lib
    cases = [(_pair(1, 97, 131), 40, _lib.F64, _lib.HWD),   # first call: scratch address set-up
             (_pair(2, 64, 200), 24, _lib.F32, _lib.DHW)]   # second call reuses the array
    for (L, R), D, dtype, layout in cases:
        l = torch.from_numpy(L).cuda()
        r = torch.from_numpy(R).cuda()
        want = _census("cbmv_census", l, r, D, dtype, layout)
        got = _census("cbmv_census_static", l, r, D, dtype, layout)
        torch.cuda.synchronize()
        assert torch.equal(got, want)


def test_static_census_rejects_images_beyond_its_scratch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cbmv_b200 import _lib
    L = _lib.lib()
    maxp = L.cbmv_census_static_max_pixels()
    assert maxp == 1 << 20
    buf = torch.empty(16, dtype=torch.uint8, device="cuda")
    # sizes are checked before anything touches the buffers
    rc = L.cbmv_census_static(ctypes.c_void_p(buf.data_ptr()), ctypes.c_void_p(buf.data_ptr()),
                              1025, 1024, 8, 11, ctypes.c_void_p(buf.data_ptr()), _lib.F32, _lib.HWD,
                              None)
    assert rc == -4
    assert b"exceeds its fixed scratch" in L.cbmv_last_error()
