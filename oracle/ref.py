"""ctypes bindings of the reference's own code (test infrastructure only).

oracle/_ref/libcbmv_ref_cpu.so holds cpp/matchers/matchers.cpp and
cpp/featextract/featextract.cpp compiled unmodified; oracle/_ref/
libcbmv_ref_post.so holds cpp/post/post.cu compiled unmodified for sm_100a.
Both are built by oracle/Makefile from the reference sources.  The objects
`mtc`, `fte` and `post` expose the reference's boost.python module surface
(libmatchers, libfeatextract, post) under the same names and argument orders,
so oracle.glue can drive them exactly like the reference's test.py/train.py.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
CPU_SO = os.path.join(REF_DIR, "libcbmv_ref_cpu.so")
POST_SO = os.path.join(REF_DIR, "libcbmv_ref_post.so")

_P = ctypes.py_object
_cpu = None
_post = None


def cpu_available():
    return os.path.exists(CPU_SO)


def post_available():
    return os.path.exists(POST_SO)


def _load_cpu():
    global _cpu
    if _cpu is None:
        if not cpu_available():
            raise FileNotFoundError(CPU_SO + " is not built (make -C oracle ref)")
        lib = ctypes.PyDLL(CPU_SO)
        sig = {
            "ref_nccNister": ([_P, _P, ctypes.c_int, ctypes.c_int], _P),
            "ref_census": ([_P, _P, ctypes.c_int, ctypes.c_int], _P),
            "ref_sadsob": ([_P, _P, ctypes.c_int, ctypes.c_int], _P),
            "ref_zsad": ([_P, _P, ctypes.c_int, ctypes.c_int], _P),
            "ref_sobel": ([_P], _P),
            "ref_initthreads": ([], ctypes.c_int),
            "ref_swap_axes": ([_P], _P),
            "ref_swap_axes_back": ([_P], _P),
            "ref_get_cost": ([_P], _P),
            "ref_get_right_cost": ([_P], _P),
            "ref_generate_d_indices": ([_P, ctypes.c_int, ctypes.c_int], _P),
            "ref_get_samples": ([_P, _P], _P),
            "ref_extract_ratio_samples": ([_P, _P, ctypes.c_double], _P),
            "ref_extract_ratio": ([_P, ctypes.c_double], _P),
            "ref_extract_likelihood_samples": ([_P, _P, ctypes.c_double], _P),
            "ref_extract_likelihood": ([_P, ctypes.c_double], _P),
            "ref_get_left_cost": ([_P], _P),
            "ref_generate_labels": ([_P], _P),
            "cbmv_ref_init": ([], ctypes.c_int),
            "cbmv_ref_threads": ([], ctypes.c_int),
            "cbmv_ref_set_threads": ([ctypes.c_int], None),
        }
        for name, (args, res) in sig.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        if lib.cbmv_ref_init() != 0:
            raise RuntimeError("numpy C-API initialisation of the reference build failed")
        _cpu = lib
    return _cpu


def set_threads(n):
    """Thread count used by every OpenMP region of the reference build."""
    _load_cpu().cbmv_ref_set_threads(int(n))


def threads():
    return _load_cpu().cbmv_ref_threads()


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class _Matchers:
    """The reference's libmatchers module (cpp/matchers/matchers.cpp:568-582)."""

    def census(self, l, r, ndisp, wsize):
        return _load_cpu().ref_census(_c(l, np.uint8), _c(r, np.uint8), int(ndisp), int(wsize))

    def nccNister(self, l, r, ndisp, wsize):
        return _load_cpu().ref_nccNister(_c(l, np.uint8), _c(r, np.uint8), int(ndisp), int(wsize))

    def sadsob(self, l, r, ndisp, wsize):
        return _load_cpu().ref_sadsob(_c(l, np.float64), _c(r, np.float64), int(ndisp), int(wsize))

    def zsad(self, l, r, ndisp, wsize):
        return _load_cpu().ref_zsad(_c(l, np.uint8), _c(r, np.uint8), int(ndisp), int(wsize))

    def sobel(self, img):
        return _load_cpu().ref_sobel(_c(img, np.uint8))

    def initthreads(self):
        return _load_cpu().ref_initthreads()


class _FeatExtract:
    """The reference's libfeatextract module (cpp/featextract/featextract.cpp:519-540).

    extract_ratio / extract_likelihood are arity-overloaded exactly as the
    boost.python registrations at featextract.cpp:533-536: (vol, samples, x)
    is the training form, (vol, x) the test form.
    """

    def swap_axes(self, c):
        return _load_cpu().ref_swap_axes(_c(c, np.float64))

    def swap_axes_back(self, c):
        return _load_cpu().ref_swap_axes_back(_c(c, np.float64))

    def get_cost(self, c):
        return _load_cpu().ref_get_cost(_c(c, np.float64))

    def get_right_cost(self, c):
        return _load_cpu().ref_get_right_cost(_c(c, np.float64))

    def get_left_cost(self, c):
        return _load_cpu().ref_get_left_cost(_c(c, np.float64))

    def generate_d_indices(self, gt, maxd, thr):
        return _load_cpu().ref_generate_d_indices(_c(gt, np.int32), int(maxd), int(thr))

    def get_samples(self, vol, samples):
        return _load_cpu().ref_get_samples(_c(vol, np.float64), _c(samples, np.int32))

    def extract_ratio(self, vol, *args):
        if len(args) == 2:
            return _load_cpu().ref_extract_ratio_samples(_c(vol, np.float64), _c(args[0], np.int32), float(args[1]))
        return _load_cpu().ref_extract_ratio(_c(vol, np.float64), float(args[0]))

    def extract_likelihood(self, vol, *args):
        if len(args) == 2:
            return _load_cpu().ref_extract_likelihood_samples(_c(vol, np.float64), _c(args[0], np.int32), float(args[1]))
        return _load_cpu().ref_extract_likelihood(_c(vol, np.float64), float(args[0]))

    def generate_labels(self, samples):
        return _load_cpu().ref_generate_labels(_c(samples, np.int32))


mtc = _Matchers()
fte = _FeatExtract()


def _load_post():
    global _post
    if _post is None:
        if not post_available():
            raise FileNotFoundError(POST_SO + " is not built (make -C oracle ref)")
        lib = ctypes.PyDLL(POST_SO)
        V = ctypes.c_void_p
        F = ctypes.c_float
        I = ctypes.c_int
        sig = {
            "refpost_import_numpy": ([], I),
            "refpost_InitCUDA": ([], I),
            "refpost_sync": ([], I),
            "refpost_double_new": ([_P], V),
            "refpost_double_delete": ([V], None),
            "refpost_double_zero": ([V], None),
            "refpost_double_get": ([V], _P),
            "refpost_float_new": ([_P], V),
            "refpost_float_delete": ([V], None),
            "refpost_float_zero": ([V], None),
            "refpost_float_get": ([V], _P),
            "refpost_sgm": ([V, V, V, V, V, F, F, F, F, F, F, I], None),
            "refpost_cross": ([V, V, I, F], None),
            "refpost_cbca": ([V, V, V, V, I], None),
            "refpost_subpixel": ([V, V, V], None),
            "refpost_median2d": ([V, V, I], None),
            "refpost_mean2d": ([V, V, _P, F], None),
            "refpost_swap_axis": ([V, V], None),
            "refpost_swap_axis_back": ([V, V], None),
            "refpost_copy_double": ([V, V], None),
            "refpost_copy_float": ([V, V], None),
            "refpost_divide_double": ([V, ctypes.c_double], None),
            "refpost_outlier_detection": ([V, V, V, I], None),
            "refpost_interpolate_mismatch": ([V, V, V], None),
            "refpost_interpolate_occlusion": ([V, V, V], None),
        }
        for name, (args, res) in sig.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        if lib.refpost_import_numpy() != 0:
            raise RuntimeError("numpy C-API initialisation of the reference post build failed")
        _post = lib
    return _post


class _DeviceArray:
    _kind = None

    def __init__(self, arr):
        lib = _load_post()
        dt = np.float64 if self._kind == "double" else np.float32
        self._keep = np.ascontiguousarray(arr, dtype=dt)
        self.h = getattr(lib, "refpost_%s_new" % self._kind)(self._keep)

    def set_to_zero(self):
        getattr(_load_post(), "refpost_%s_zero" % self._kind)(self.h)

    def get_array(self):
        return getattr(_load_post(), "refpost_%s_get" % self._kind)(self.h)

    def __del__(self):
        if getattr(self, "h", None) and _post is not None:
            getattr(_post, "refpost_%s_delete" % self._kind)(self.h)
            self.h = None


class CUDA_double_array(_DeviceArray):
    _kind = "double"


class CUDA_float_array(_DeviceArray):
    _kind = "float"


class _Post:
    """The reference's post module (cpp/post/post.cu:905-933)."""
    CUDA_double_array = CUDA_double_array
    CUDA_float_array = CUDA_float_array

    def InitCUDA(self):
        return bool(_load_post().refpost_InitCUDA())

    def sync(self):
        return _load_post().refpost_sync()

    def sgm(self, l, r, cin, cout, tmp, pi1, pi2, tau_so, alpha1, q1, q2, direction):
        _load_post().refpost_sgm(l.h, r.h, cin.h, cout.h, tmp.h, pi1, pi2, tau_so, alpha1, q1, q2, int(direction))

    def cross(self, im, out, L1, tau1):
        _load_post().refpost_cross(im.h, out.h, int(L1), float(tau1))

    def cbca(self, lc, rc, vol, out, direction):
        _load_post().refpost_cbca(lc.h, rc.h, vol.h, out.h, int(direction))

    def subpixel_enchancement(self, d, cost, out):
        _load_post().refpost_subpixel(d.h, cost.h, out.h)

    def median2d(self, a, out, k):
        _load_post().refpost_median2d(a.h, out.h, int(k))

    def mean2d(self, a, out, kernel, alpha2):
        _load_post().refpost_mean2d(a.h, out.h, np.ascontiguousarray(kernel, dtype=np.float32), float(alpha2))

    def swap_axis(self, a, out):
        _load_post().refpost_swap_axis(a.h, out.h)

    def swap_axis_back(self, a, out):
        _load_post().refpost_swap_axis_back(a.h, out.h)

    def CUDA_copy_double(self, a, out):
        _load_post().refpost_copy_double(a.h, out.h)

    def CUDA_copy_float(self, a, out):
        _load_post().refpost_copy_float(a.h, out.h)

    def CUDA_divide_double(self, a, v):
        _load_post().refpost_divide_double(a.h, float(v))

    def outlier_detection(self, d0, d1, out, disp_max):
        _load_post().refpost_outlier_detection(d0.h, d1.h, out.h, int(disp_max))

    def interpolate_mismatch(self, d0, outlier, out):
        _load_post().refpost_interpolate_mismatch(d0.h, outlier.h, out.h)

    def interpolate_occlusion(self, d0, outlier, out):
        _load_post().refpost_interpolate_occlusion(d0.h, outlier.h, out.h)


post = _Post()
