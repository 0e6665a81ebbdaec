"""The C-ABI library: it loads, exports every entry point include/cbmv.h
declares, and rejects bad arguments on the host before any launch (these
calls need no GPU)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "cbmv.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cbmv_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from cbmv_b200 import _lib
    L = _lib.lib()
    names = _declared()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding covers every one of them
    assert not [n for n in names if n not in _lib.SIGNATURES], "unbound entry points"


def test_host_side_argument_checks():
    from cbmv_b200 import _lib
    L = _lib.lib()
    buf = ctypes.c_void_p(16)  # never dereferenced: the calls fail their checks first
    assert L.cbmv_census(None, buf, 10, 10, 4, 11, buf, 0, 0, None) == -1
    assert b"null" in L.cbmv_last_error()
    assert L.cbmv_census(buf, buf, 10, 10, 4, 4, buf, 0, 0, None) == -1  # even window
    assert L.cbmv_ncc(buf, buf, 10, 10, 4, 3, buf, 7, 0, None) == -1      # bad dtype
    assert L.cbmv_zsad(buf, buf, 10, 10, 0, 5, buf, 0, 0, None) == -1     # D = 0
    assert L.cbmv_median2d(buf, 10, 10, 4, buf, None) == -1                # even median
    assert L.cbmv_sgm(buf, buf, buf, 10, 10, 2000, 1, 1, 1, 1, 1, 1, -1, buf, None) == -4
    assert L.cbmv_cbca(buf, buf, buf, 10, 10, 4, 0, 2, buf, None) == -1    # direction
    assert L.cbmv_cbca(buf, buf, buf, 10, 10, 4, 0, 1, buf, None) == -1    # in == out
    p = _lib.default_params()
    assert (p.censw, p.nccw, p.sadw, p.sgm_i, p.cbca_i2, p.direction) == (11, 3, 5, 2, 4, -1)
    assert abs(p.pi1 - 1.3) < 1e-6 and abs(p.blur_t - 1.3) < 1e-6


def test_forest_upload_validation():
    import numpy as np
    from cbmv_b200 import _lib
    L = _lib.lib()
    leafv = np.zeros((2, 2))
    offs = np.array([0, 1], np.int32)
    h = ctypes.c_void_p()
    # a block whose root is a leaf with an index beyond the leaf array
    bad = np.zeros((1, 8), np.uint32)
    bad[0, 3] = 0xFFFFFF
    bad[0, 4] = 7
    assert L.cbmv_forest_create(bad.ctypes.data, 1, leafv.ctypes.data, 2, offs.ctypes.data, 1, 20,
                                ctypes.byref(h)) == -1
    # a child block pointing outside its tree (the walk would leave the array)
    bad = np.zeros((1, 8), np.uint32)
    bad[0, 3] = 3 | (4 << 8) | (5 << 16)
    bad[0, 4:8] = [0x80000000, 0x80000001, 5, 0x80000000]
    assert L.cbmv_forest_create(bad.ctypes.data, 1, leafv.ctypes.data, 2, offs.ctypes.data, 1, 20,
                                ctypes.byref(h)) == -1
    assert b"child" in L.cbmv_last_error()
    # a feature beyond n_features
    bad[0, 3] = 25
    assert L.cbmv_forest_create(bad.ctypes.data, 1, leafv.ctypes.data, 2, offs.ctypes.data, 1, 20,
                                ctypes.byref(h)) == -1
