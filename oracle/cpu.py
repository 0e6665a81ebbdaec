"""ctypes bindings of oracle.c, the CPU restatement (test infrastructure only).

`mtc`, `fte` and `post` mirror the reference's boost.python modules
(libmatchers, libfeatextract, post) with the same names, argument orders,
array layouts and dtypes, so that oracle.glue drives them exactly like the
reference's own drivers.  `post` here is host-resident: its CUDA_double_array
/ CUDA_float_array simply hold numpy arrays and every kernel runs on the CPU.
`rf_predict` walks a flat forest (cbmv_b200.forest.FlatForest) as sklearn does.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(_HERE, "liboracle.so")
_lib = None

_i64 = ctypes.c_longlong
_int = ctypes.c_int
_dbl = ctypes.c_double
_flt = ctypes.c_float
_vp = ctypes.c_void_p


def available():
    return os.path.exists(SO)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(SO + " is not built (make -C oracle liboracle.so)")
        L = ctypes.CDLL(SO)
        sig = {
            "orc_census": [_vp, _vp, _i64, _i64, _int, _int, _vp],
            "orc_ncc": [_vp, _vp, _i64, _i64, _int, _int, _vp],
            "orc_sobel": [_vp, _i64, _i64, _vp],
            "orc_sadsob": [_vp, _vp, _i64, _i64, _int, _int, _vp],
            "orc_zsad": [_vp, _vp, _i64, _i64, _int, _int, _vp],
            "orc_swap_axes": [_vp, _i64, _i64, _i64, _vp],
            "orc_swap_axes_back": [_vp, _i64, _i64, _i64, _vp],
            "orc_get_cost": [_vp, _i64, _i64, _i64, _i64, _vp],
            "orc_get_right_cost": [_vp, _i64, _i64, _i64, _vp],
            "orc_get_left_cost": [_vp, _i64, _i64, _i64, _vp],
            "orc_extract_ratio": [_vp, _i64, _i64, _dbl, _vp],
            "orc_extract_likelihood": [_vp, _i64, _i64, _dbl, _vp],
            "orc_extract_ratio_samples": [_vp, _i64, _i64, _vp, _dbl, _vp],
            "orc_extract_likelihood_samples": [_vp, _i64, _i64, _vp, _dbl, _vp],
            "orc_get_samples": [_vp, _i64, _i64, _vp, _vp],
            "orc_generate_labels": [_i64, _vp],
            "orc_generate_d_indices": [_vp, _i64, _int, _int, ctypes.c_uint64, _vp],
            "orc_rf_predict": [_vp, _int, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _int, _vp, _vp],
            "orc_cross": [_vp, _i64, _i64, _int, _flt, _vp],
            "orc_cbca": [_vp, _vp, _vp, _i64, _i64, _i64, _int, _vp],
            "orc_sgm": [_vp, _vp, _vp, _i64, _i64, _int, _flt, _flt, _flt, _flt, _flt, _flt, _int, _vp],
            "orc_wta": [_vp, _i64, _i64, _i64, _vp],
            "orc_subpixel": [_vp, _vp, _i64, _i64, _int, _vp],
            "orc_median2d": [_vp, _i64, _i64, _int, _vp],
            "orc_mean2d": [_vp, _i64, _i64, _vp, _int, _flt, _vp],
            "orc_outlier_detection": [_vp, _vp, _i64, _i64, _int, _vp],
            "orc_interpolate_mismatch": [_vp, _vp, _i64, _i64, _vp],
            "orc_interpolate_occlusion": [_vp, _vp, _i64, _i64, _vp],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _int if name == "orc_generate_d_indices" else None
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_vp)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class _Matchers:
    """libmatchers (cpp/matchers/matchers.cpp:568-582), restated."""

    def census(self, l, r, ndisp, wsize):
        l, r = _c(l, np.uint8), _c(r, np.uint8)
        H, W = l.shape
        out = np.empty((H, W, ndisp), np.float64)
        lib().orc_census(_p(l), _p(r), H, W, ndisp, wsize, _p(out))
        return out

    def nccNister(self, l, r, ndisp, wsize):
        l, r = _c(l, np.uint8), _c(r, np.uint8)
        H, W = l.shape
        out = np.empty((ndisp, H, W), np.float64)
        lib().orc_ncc(_p(l), _p(r), H, W, ndisp, wsize, _p(out))
        return out

    def sobel(self, img):
        img = _c(img, np.uint8)
        H, W = img.shape
        out = np.empty((H, W), np.float64)
        lib().orc_sobel(_p(img), H, W, _p(out))
        return out

    def sadsob(self, l, r, ndisp, wsize):
        l, r = _c(l, np.float64), _c(r, np.float64)
        H, W = l.shape
        out = np.empty((ndisp, H, W), np.float64)
        lib().orc_sadsob(_p(l), _p(r), H, W, ndisp, wsize, _p(out))
        return out

    def zsad(self, l, r, ndisp, wsize):
        l, r = _c(l, np.uint8), _c(r, np.uint8)
        H, W = l.shape
        out = np.empty((ndisp, H, W), np.float64)
        lib().orc_zsad(_p(l), _p(r), H, W, ndisp, wsize, _p(out))
        return out

    def initthreads(self):
        return os.cpu_count()


class _FeatExtract:
    """libfeatextract (cpp/featextract/featextract.cpp:519-540), restated."""

    def swap_axes(self, c):
        c = _c(c, np.float64)
        D, H, W = c.shape
        out = np.empty((H, W, D), np.float64)
        lib().orc_swap_axes(_p(c), D, H, W, _p(out))
        return out

    def swap_axes_back(self, c):
        c = _c(c, np.float64)
        H, W, D = c.shape
        out = np.empty((D, H, W), np.float64)
        lib().orc_swap_axes_back(_p(c), H, W, D, _p(out))
        return out

    def get_cost(self, c):
        c = _c(c, np.float64)
        H, W, D, K = c.shape
        out = np.empty((H, W, D), np.float64)
        lib().orc_get_cost(_p(c), H, W, D, K, _p(out))
        return out

    def get_right_cost(self, c):
        c = _c(c, np.float64)
        H, W, D = c.shape
        out = np.empty_like(c)
        lib().orc_get_right_cost(_p(c), H, W, D, _p(out))
        return out

    def get_left_cost(self, c):
        c = _c(c, np.float64)
        H, W, D = c.shape
        out = np.empty_like(c)
        lib().orc_get_left_cost(_p(c), H, W, D, _p(out))
        return out

    def extract_ratio(self, vol, *args):
        vol = _c(vol, np.float64)
        N, D = vol.shape
        if len(args) == 2:
            s = _c(args[0], np.int32)
            out = np.empty(3 * s.shape[0], np.float64)
            lib().orc_extract_ratio_samples(_p(vol), N, D, _p(s), float(args[1]), _p(out))
            return out
        out = np.empty_like(vol)
        lib().orc_extract_ratio(_p(vol), N, D, float(args[0]), _p(out))
        return out

    def extract_likelihood(self, vol, *args):
        vol = _c(vol, np.float64)
        N, D = vol.shape
        if len(args) == 2:
            s = _c(args[0], np.int32)
            out = np.empty(3 * s.shape[0], np.float64)
            lib().orc_extract_likelihood_samples(_p(vol), N, D, _p(s), float(args[1]), _p(out))
            return out
        out = np.empty_like(vol)
        lib().orc_extract_likelihood(_p(vol), N, D, float(args[0]), _p(out))
        return out

    def get_samples(self, vol, samples):
        vol = _c(vol, np.float64)
        s = _c(samples, np.int32)
        out = np.empty(3 * s.shape[0], np.float64)
        lib().orc_get_samples(_p(vol), vol.shape[0], vol.shape[1], _p(s), _p(out))
        return out

    def generate_labels(self, samples):
        n = np.asarray(samples).shape[0]
        out = np.empty(3 * n, np.int32)
        lib().orc_generate_labels(n, _p(out))
        return out

    def generate_d_indices(self, gt, maxd, thr, seed=0):
        gt = _c(np.asarray(gt).reshape(-1), np.int32)
        out = np.empty((gt.shape[0], 3), np.int32)
        rc = lib().orc_generate_d_indices(_p(gt), gt.shape[0], int(maxd), int(thr), int(seed), _p(out))
        if rc != 0:
            raise ValueError("generate_d_indices: a ground-truth value leaves an empty sampling range")
        return out


mtc = _Matchers()
fte = _FeatExtract()


def rf_predict(forest, X, return_leaves=False):
    """P(class 0) per row of X (cast to float32), optionally the leaf per tree."""
    X = _c(X, np.float32)
    N, F = X.shape
    p0 = np.empty(N, np.float64)
    leaves = np.empty((N, forest.n_trees), np.int32) if return_leaves else None
    lib().orc_rf_predict(_p(forest.roots), forest.n_trees, _p(forest.feature), _p(forest.threshold),
                         _p(forest.left), _p(forest.right), _p(forest.value0), _p(X), N, F, _p(p0),
                         _p(leaves) if return_leaves else None)
    return (p0, leaves) if return_leaves else p0


class _HostArray:
    dtype = None

    def __init__(self, arr):
        self.a = np.array(arr, dtype=self.dtype, copy=True, order="C")

    @property
    def ins(self):
        return self.a.shape

    def set_to_zero(self):
        self.a[...] = 0

    def get_array(self):
        return self.a.copy()


class CUDA_double_array(_HostArray):
    dtype = np.float64


class CUDA_float_array(_HostArray):
    dtype = np.float32


class _Post:
    """post (cpp/post/post.cu:905-933), restated on the CPU.

    Shapes follow the reference's bookkeeping: swap_axis / swap_axis_back /
    CUDA_copy_double change the destination's shape (post.cu:612-614,
    663-665, 702-704).

    as_shipped=False (`post`): swap_axis_back is the transpose it is meant
    to be.  as_shipped=True (`post_as_shipped`): it also restates the
    reference kernel's store condition, `(Col + d) < cols*rows` with Col
    already the pixel index (post.cu:645-646): the pixel p of disparity d is
    not written when p + 16 * floor((d mod 64) / 16) >= H*W, so the last
    16..48 pixels of those disparities keep the destination's previous
    contents (in the reference's drivers, the same buffer in the [H,W,D]
    layout).  That is what the reference computes; the fused path computes
    the transpose."""
    CUDA_double_array = CUDA_double_array
    CUDA_float_array = CUDA_float_array

    def __init__(self, as_shipped=False):
        self.as_shipped = as_shipped

    def InitCUDA(self):
        return True

    def sync(self):
        return 0

    def cross(self, im, out, L1, tau1):
        H, W = im.a.shape
        res = np.empty((4, H, W), np.float32)
        lib().orc_cross(_p(im.a), H, W, int(L1), float(tau1), _p(res))
        out.a = res

    def cbca(self, lc, rc, vol, out, direction):
        D, H, W = vol.a.shape
        res = np.empty_like(vol.a)
        lib().orc_cbca(_p(lc.a), _p(rc.a), _p(vol.a), D, H, W, int(direction), _p(res))
        out.a = res

    def sgm(self, l, r, cin, cout, tmp, pi1, pi2, tau_so, alpha1, q1, q2, direction):
        H, W, D = cin.a.shape
        res = np.zeros((H, W, D), np.float64)
        lib().orc_sgm(_p(l.a), _p(r.a), _p(cin.a), H, W, D, pi1, pi2, tau_so, alpha1, q1, q2,
                      int(direction), _p(res))
        cout.a = cout.a.reshape(H, W, D)
        cout.a += res

    def swap_axis(self, a, out):
        out.a = np.ascontiguousarray(np.transpose(a.a, (1, 2, 0)))

    def swap_axis_back(self, a, out):
        res = np.ascontiguousarray(np.transpose(a.a, (2, 0, 1)))  # [D,H,W]
        if self.as_shipped:
            D = res.shape[0]
            HW = res.shape[1] * res.shape[2]
            prev = out.a.reshape(-1)
            flat = res.reshape(D, HW)
            for d in range(D):
                skip = 16 * ((d % 64) // 16)
                if skip:
                    lo = max(HW - skip, 0)
                    flat[d, lo:] = prev[d * HW + lo:(d + 1) * HW]
        out.a = res

    def CUDA_copy_double(self, a, out):
        out.a = a.a.copy()

    def CUDA_copy_float(self, a, out):
        out.a[...] = a.a.reshape(out.a.shape)

    def CUDA_divide_double(self, a, v):
        a.a /= v

    def subpixel_enchancement(self, d, cost, out):
        D, H, W = cost.a.shape
        res = np.empty((H, W), np.float32)
        lib().orc_subpixel(_p(d.a), _p(cost.a), H, W, D, _p(res))
        out.a = res

    def median2d(self, a, out, k):
        H, W = a.a.shape
        res = np.empty((H, W), np.float32)
        lib().orc_median2d(_p(a.a), H, W, int(k), _p(res))
        out.a = res

    def mean2d(self, a, out, kernel, alpha2):
        H, W = a.a.shape
        k = _c(kernel, np.float32)
        res = np.empty((H, W), np.float32)
        lib().orc_mean2d(_p(a.a), H, W, _p(k), k.shape[0], float(alpha2), _p(res))
        out.a = res

    def outlier_detection(self, d0, d1, out, disp_max):
        H, W = d0.a.shape
        res = np.empty((H, W), np.float32)
        lib().orc_outlier_detection(_p(d0.a), _p(d1.a), H, W, int(disp_max), _p(res))
        out.a = res

    def interpolate_mismatch(self, d0, outlier, out):
        H, W = d0.a.shape
        res = np.empty((H, W), np.float32)
        lib().orc_interpolate_mismatch(_p(d0.a), _p(outlier.a), H, W, _p(res))
        out.a = res

    def interpolate_occlusion(self, d0, outlier, out):
        H, W = d0.a.shape
        res = np.empty((H, W), np.float32)
        lib().orc_interpolate_occlusion(_p(d0.a), _p(outlier.a), H, W, _p(res))
        out.a = res


post = _Post()
post_as_shipped = _Post(as_shipped=True)


def wta(cost_dhw):
    """np.argmin(cost, axis=0) as float32 (test.py:408-409)."""
    c = _c(cost_dhw, np.float64)
    D, H, W = c.shape
    out = np.empty((H, W), np.float32)
    lib().orc_wta(_p(c), D, H, W, _p(out))
    return out
