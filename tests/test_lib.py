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


def test_library_exports_nothing_else():
    """Hidden visibility: the dynamic symbol table holds the C ABI of
    include/cbmv.h and no C++ internals of the library (kernel stubs,
    cbmv:: functions) that could clash with a host process's own."""
    import shutil
    import subprocess
    from cbmv_b200 import _lib
    nm = shutil.which("nm")
    if nm is None:
        pytest.skip("nm not installed")
    out = subprocess.run([nm, "-D", "--defined-only", _lib.lib()._name], capture_output=True, text=True,
                         check=True).stdout
    syms = [ln.split()[-1] for ln in out.splitlines() if ln.split() and ln.split()[-2] in "TDBR"]
    ours = sorted(s for s in syms if s.startswith("cbmv_"))
    assert ours == _declared()
    assert not [s for s in syms if "cbmv" in s and not s.startswith("cbmv_")], "C++ internals exported"


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


def test_census_entry_points_reject_alike():
    """cbmv_census_static validates its arguments with cbmv_census's own
    checks, so both return the same code for the same bad input; only its
    pixel limit is its own (checked without forming an overflowing H*W)."""
    from cbmv_b200 import _lib
    L = _lib.lib()
    buf = ctypes.c_void_p(16)  # never dereferenced
    bad = [(None, buf, 10, 10, 4, 11, 0, 0),       # null image
           (buf, buf, 10, 10, 4, 4, 0, 0),         # even window
           (buf, buf, 10, 10, 4, 13, 0, 0),        # window beyond 11
           (buf, buf, 10, 10, 0, 11, 0, 0),        # D = 0
           (buf, buf, 70000, 10, 4, 11, 0, 0),     # H beyond 65535
           (buf, buf, 10, 10, 70000, 11, 0, 0),    # D beyond 65535
           (buf, buf, 10, 10, 4, 11, 5, 0),        # dtype
           (buf, buf, 10, 10, 4, 11, 0, 9)]        # layout
    for a, b, H, W, D, w, dt, lay in bad:
        r1 = L.cbmv_census(a, b, H, W, D, w, buf, dt, lay, None)
        r2 = L.cbmv_census_static(a, b, H, W, D, w, buf, dt, lay, None)
        assert r1 == r2 != 0, (H, W, D, w, dt, lay, r1, r2)
    mx = L.cbmv_census_static_max_pixels()
    assert L.cbmv_census_static(buf, buf, 1024, mx // 1024 + 1, 4, 11, buf, 0, 0, None) == -4
    assert L.cbmv_census_static(buf, buf, 65535, 1 << 50, 4, 11, buf, 0, 0, None) == -4  # H*W > 2^63


def test_argument_checks_of_the_fused_entry_points():
    """The batch, post-only, separable CBCA and parameter checks reject bad
    arguments on the host, before any device work."""
    import numpy as np
    from cbmv_b200 import _lib
    L = _lib.lib()
    buf = ctypes.c_void_p(16)
    h = ctypes.c_void_p()
    Hs, Ws, Ds = (np.array(v, dt) for v, dt in (([64, 8], np.int64), ([64, 64], np.int64), ([32, 32], np.int32)))
    assert L.cbmv_batch_create(0, Hs.ctypes.data, Ws.ctypes.data, Ds.ctypes.data, 2, ctypes.byref(h)) == -1
    assert L.cbmv_batch_create(2, Hs.ctypes.data, Ws.ctypes.data, Ds.ctypes.data, 2, ctypes.byref(h)) == -1
    assert b"pair 1" in L.cbmv_last_error()                               # an 8-row image
    assert L.cbmv_batch_create(1, Hs.ctypes.data, Ws.ctypes.data, Ds.ctypes.data, 0, ctypes.byref(h)) == -1
    assert L.cbmv_batch_run_mlp(None, buf, None, buf, buf, buf, None) == -1
    assert L.cbmv_cbca_separable(buf, buf, buf, 10, 10, 4, 12, -1, buf, None) == -1   # L1 > 9
    assert L.cbmv_cbca_separable(buf, buf, buf, 10, 10, 4, 6, -1, buf, None) == -1    # in == out
    assert L.cbmv_run_post(None, None, buf, buf, 10, 10, 4, buf, buf) == -1
    prm = _lib.default_params(cbca_rows=24)
    assert L.cbmv_run_mlp(buf, buf, ctypes.byref(prm), buf, buf, 64, 64, 32, buf, None) != 0
    assert b"cbca_rows" in L.cbmv_last_error()
    prm = _lib.default_params(sgm_prefetch=3)
    assert L.cbmv_run_mlp(buf, buf, ctypes.byref(prm), buf, buf, 64, 64, 32, buf, None) != 0
    assert b"sgm_prefetch" in L.cbmv_last_error()
    # the host-buffer forms check their pointers and sizes before touching the context
    assert L.cbmv_run_mlp_host(None, buf, None, buf, buf, 64, 64, 32, buf) == -1
    assert L.cbmv_run_mlp_host(buf, None, None, buf, buf, 64, 64, 32, buf) == -1
    assert L.cbmv_run_rf_host(buf, buf, None, buf, None, 64, 64, 32, buf) == -1
    assert L.cbmv_run_rf_host(buf, buf, None, buf, buf, 0, 64, 32, buf) == -1
    assert L.cbmv_run_mlp_host(buf, buf, None, buf, buf, 70000, 64, 32, buf) == -4
    assert b"65535" in L.cbmv_last_error()
    prec = ctypes.c_int()
    assert L.cbmv_mlp_set_precision(None, 1) == -1
    assert L.cbmv_mlp_get_precision(None, ctypes.byref(prec)) == -1


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


def test_learned_classifier_falls_back_to_the_forest():
    """StereoPipeline.run_classified: the network's result when it ran
    cleanly, the forest's when the network call failed or reported a
    tensor-core timeout (the pipeline's calls stubbed: host logic only)."""
    import pytest
    from cbmv_b200 import _lib
    from cbmv_b200.pipeline import StereoPipeline

    class Net:
        def __init__(self, status):
            self.s = status

        def status(self):
            return self.s

    p = StereoPipeline.__new__(StereoPipeline)  # no device context needed for the stubs
    p.forest = object()
    p.run_rf = lambda *a, **k: "rf-disparity"
    p.run_mlp = lambda net, *a, **k: "mlp-disparity"
    assert p.run_classified(None, None, 8, net=Net(0)) == ("mlp-disparity", "mlp")
    assert p.run_classified(None, None, 8, net=Net(1)) == ("rf-disparity", "rf")
    assert p.run_classified(None, None, 8) == ("rf-disparity", "rf")

    def fail(*a, **k):
        raise _lib.CbmvError("cbmv_run_mlp", -2, "injected")
    p.run_mlp = fail
    assert p.run_classified(None, None, 8, net=Net(0)) == ("rf-disparity", "rf")
    p.forest = None
    with pytest.raises(RuntimeError):
        p.run_classified(None, None, 8, net=Net(0))
    p.ctx = None  # nothing to release


def test_product_never_imports_the_oracle():
    """The oracle is the checker only: no module of the package imports it,
    and the library's sources include nothing from it."""
    import ast
    pkg = os.path.join(ROOT, "cbmv_b200")
    for name in sorted(os.listdir(pkg)):
        if not name.endswith(".py"):
            continue
        tree = ast.parse(open(os.path.join(pkg, name)).read())
        for node in ast.walk(tree):
            mods = []
            if isinstance(node, ast.Import):
                mods = [a.name for a in node.names]
            elif isinstance(node, ast.ImportFrom):
                mods = [node.module or ""]
            assert not [m for m in mods if m == "oracle" or m.startswith("oracle.")], (name, mods)
    csrc = os.path.join(pkg, "csrc")
    for name in sorted(os.listdir(csrc)):
        if name.endswith((".cu", ".cuh", ".h")):
            for line in open(os.path.join(csrc, name)):
                if line.lstrip().startswith("#include"):
                    assert "oracle" not in line, (name, line)


def test_header_is_plain_c_and_links(tmp_path):
    """include/cbmv.h compiles as pedantic C99 (cgo, JNI and other FFIs bind
    it from C), and a C program links against libcbmv.so and calls it."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not installed")
    src = tmp_path / "t.c"
    src.write_text('#include "cbmv.h"\n#include <stdio.h>\n'
                   "int main(void) { cbmv_params p; cbmv_params_default(&p);\n"
                   '  printf("%d %d %s\\n", p.censw, p.sgm_i, cbmv_version()); return 0; }\n')
    exe = tmp_path / "t"
    lib_dir = os.path.join(ROOT, "cbmv_b200")
    subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe), "-L" + lib_dir, "-lcbmv", "-Wl,-rpath," + lib_dir,
                    "-Wl,--unresolved-symbols=ignore-in-shared-libs"], check=True, capture_output=True)
    env = dict(os.environ)
    try:
        import nvidia.cuda_runtime as cr  # the CUDA runtime the library was linked against
        env["LD_LIBRARY_PATH"] = os.path.join(cr.__path__[0], "lib") + ":" + env.get("LD_LIBRARY_PATH", "")
    except ImportError:
        pass
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, env=env).stdout.split()
    assert out[:2] == ["11", "2"] and out[2].startswith("cbmv-b200")
