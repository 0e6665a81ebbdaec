"""ctypes binding of libcbmv.so (include/cbmv.h).

The library is built in-tree by cbmv_b200.build; loading fails loudly when it
is missing: there is no CPU fallback anywhere in this package.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "libcbmv.so")

F32, F64 = 0, 1
ACT_RELU, ACT_GELU = 0, 1
HWD, DHW = 0, 1

_i64 = ctypes.c_int64
_int = ctypes.c_int
_dbl = ctypes.c_double
_flt = ctypes.c_float
_vp = ctypes.c_void_p
_u64 = ctypes.c_uint64


class CbmvError(RuntimeError):
    def __init__(self, fn, code, msg):
        super().__init__("%s failed (%d): %s" % (fn, code, msg))
        self.code = code


class cbmv_params(ctypes.Structure):
    _fields_ = [("censw", _int), ("nccw", _int), ("sadw", _int), ("sobw", _int),
                ("pi1", _flt), ("pi2", _flt), ("sgm_q1", _flt), ("sgm_q2", _flt),
                ("alpha1", _flt), ("tau_so", _flt), ("sgm_i", _int), ("L1", _int),
                ("tau1", _flt), ("cbca_i1", _int), ("cbca_i2", _int), ("median_i", _int),
                ("median_w", _int), ("blur_sigma", _flt), ("blur_t", _flt), ("direction", _int),
                ("exact_cbca", _int), ("mlp_ctas", _int), ("cbca_rows", _int), ("sgm_prefetch", _int),
                ("interpolate", _int)]


# name -> argtypes (all return int status unless listed in _RESTYPE)
SIGNATURES = {
    "cbmv_last_error": [],
    "cbmv_version": [],
    "cbmv_sync": [_vp],
    "cbmv_census": [_vp, _vp, _i64, _i64, _int, _int, _vp, _int, _int, _vp],
    "cbmv_census_static": [_vp, _vp, _i64, _i64, _int, _int, _vp, _int, _int, _vp],
    "cbmv_census_static_max_pixels": [],
    "cbmv_ncc": [_vp, _vp, _i64, _i64, _int, _int, _vp, _int, _int, _vp],
    "cbmv_sobel": [_vp, _i64, _i64, _vp, _int, _vp],
    "cbmv_sadsob": [_vp, _vp, _int, _i64, _i64, _int, _int, _vp, _int, _int, _vp],
    "cbmv_zsad": [_vp, _vp, _i64, _i64, _int, _int, _vp, _int, _int, _vp],
    "cbmv_swap_axes": [_vp, _i64, _i64, _i64, _vp, _vp],
    "cbmv_swap_axes_back": [_vp, _i64, _i64, _i64, _vp, _vp],
    "cbmv_get_cost": [_vp, _i64, _i64, _i64, _i64, _vp, _vp],
    "cbmv_get_right_cost": [_vp, _i64, _i64, _i64, _vp, _vp],
    "cbmv_get_left_cost": [_vp, _i64, _i64, _i64, _vp, _vp],
    "cbmv_extract_ratio": [_vp, _i64, _i64, _dbl, _vp, _vp],
    "cbmv_extract_likelihood": [_vp, _i64, _i64, _dbl, _vp, _vp],
    "cbmv_extract_ratio_samples": [_vp, _i64, _i64, _vp, _dbl, _vp, _vp],
    "cbmv_extract_likelihood_samples": [_vp, _i64, _i64, _vp, _dbl, _vp, _vp],
    "cbmv_get_samples": [_vp, _i64, _i64, _vp, _vp, _vp],
    "cbmv_generate_labels": [_i64, _vp, _vp],
    "cbmv_generate_d_indices": [_vp, _i64, _int, _int, _u64, _vp, _vp],
    "cbmv_features": [_vp, _vp, _vp, _vp, _i64, _i64, _int, _vp, _vp],
    "cbmv_forest_create": [_vp, _i64, _vp, _i64, _vp, _int, _int, ctypes.POINTER(_vp)],
    "cbmv_forest_info": [_vp, ctypes.POINTER(_int), ctypes.POINTER(_i64), ctypes.POINTER(_i64)],
    "cbmv_forest_destroy": [_vp],
    "cbmv_forest_predict": [_vp, _vp, _i64, _vp, _vp, _vp],
    "cbmv_gemm_bf16": [_vp, _vp, _vp, _i64, _i64, _i64, _vp, _vp],
    "cbmv_mlp_num_params": [],
    "cbmv_mlp_create": [_int, ctypes.POINTER(_vp)],
    "cbmv_mlp_destroy": [_vp],
    "cbmv_mlp_set_params": [_vp, _vp],
    "cbmv_mlp_get_params": [_vp, _vp],
    "cbmv_mlp_train_step": [_vp, _vp, _vp, _flt, _flt, _vp, _vp],
    "cbmv_mlp_gradients": [_vp, _vp, _vp, _vp, _vp, _vp],
    "cbmv_mlp_status": [_vp, ctypes.POINTER(_int)],
    "cbmv_mlp_set_activation": [_vp, _int],
    "cbmv_mlp_get_activation": [_vp, _vp],
    "cbmv_mlp_set_precision": [_vp, _int],
    "cbmv_mlp_get_precision": [_vp, _vp],
    "cbmv_cross": [_vp, _i64, _i64, _int, _flt, _vp, _vp],
    "cbmv_sgm": [_vp, _vp, _vp, _i64, _i64, _int, _flt, _flt, _flt, _flt, _flt, _flt, _int, _vp, _vp],
    "cbmv_cbca": [_vp, _vp, _vp, _i64, _i64, _int, _int, _int, _vp, _vp],
    "cbmv_cbca_separable": [_vp, _vp, _vp, _i64, _i64, _int, _int, _int, _vp, _vp],
    "cbmv_wta": [_vp, _i64, _i64, _int, _int, _vp, _vp],
    "cbmv_subpixel": [_vp, _vp, _i64, _i64, _int, _int, _vp, _vp],
    "cbmv_median2d": [_vp, _i64, _i64, _int, _vp, _vp],
    "cbmv_mean2d": [_vp, _i64, _i64, _vp, _int, _flt, _vp, _vp],
    "cbmv_outlier_detection": [_vp, _vp, _i64, _i64, _int, _vp, _vp],
    "cbmv_interpolate_mismatch": [_vp, _vp, _i64, _i64, _vp, _vp],
    "cbmv_interpolate_occlusion": [_vp, _vp, _i64, _i64, _vp, _vp],
    "cbmv_transpose_f32": [_vp, _i64, _i64, _i64, _int, _vp, _vp],
    "cbmv_scale_f32": [_vp, _i64, _flt, _vp],
    "cbmv_f64_to_f32": [_vp, _i64, _vp, _vp],
    "cbmv_f32_to_f64": [_vp, _i64, _vp, _vp],
    "cbmv_params_default": [ctypes.POINTER(cbmv_params)],
    "cbmv_ctx_create": [_vp, ctypes.POINTER(_vp)],
    "cbmv_ctx_destroy": [_vp],
    "cbmv_ctx_timings": [_vp, ctypes.POINTER(_flt)],
    "cbmv_run_rf": [_vp, _vp, ctypes.POINTER(cbmv_params), _vp, _vp, _i64, _i64, _int, _vp, _vp],
    "cbmv_run_mlp": [_vp, _vp, ctypes.POINTER(cbmv_params), _vp, _vp, _i64, _i64, _int, _vp, _vp],
    "cbmv_run_rf_host": [_vp, _vp, ctypes.POINTER(cbmv_params), _vp, _vp, _i64, _i64, _int, _vp],
    "cbmv_run_mlp_host": [_vp, _vp, ctypes.POINTER(cbmv_params), _vp, _vp, _i64, _i64, _int, _vp],
    "cbmv_ctx_features_at": [_vp, ctypes.POINTER(cbmv_params), _vp, _vp, _i64, _i64, _int, _vp, _i64, _vp],
    "cbmv_ctx_features_f32_at": [_vp, ctypes.POINTER(cbmv_params), _vp, _vp, _i64, _i64, _int, _vp, _i64, _vp],
    "cbmv_ctx_volumes_f32": [_vp, ctypes.POINTER(cbmv_params), _vp, _vp, _i64, _i64, _int, _vp],
    "cbmv_run_post": [_vp, ctypes.POINTER(cbmv_params), _vp, _vp, _i64, _i64, _int, _vp, _vp],
    "cbmv_batch_create": [_int, _vp, _vp, _vp, _int, _vp],
    "cbmv_batch_destroy": [_vp],
    "cbmv_batch_run_mlp": [_vp, _vp, ctypes.POINTER(cbmv_params), _vp, _vp, _vp, _vp],
    "cbmv_batch_timings": [_vp, _vp, _vp, _vp],
}
_RESTYPE = {"cbmv_last_error": ctypes.c_char_p, "cbmv_version": ctypes.c_char_p,
            "cbmv_params_default": None, "cbmv_census_static_max_pixels": ctypes.c_int64}

_lib = None


def lib():
    """The loaded library with argtypes/restype set (raises if not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(SO):
            raise ImportError("libcbmv.so is not built: run `python -m cbmv_b200.build` "
                              "(the CUDA extension is required; there is no CPU path)")
        L = ctypes.CDLL(SO)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPE.get(name, ctypes.c_int)
        _lib = L
    return _lib


def call(name, *args):
    """Calls a status-returning entry point; raises CbmvError on failure."""
    rc = getattr(lib(), name)(*args)
    if rc != 0:
        raise CbmvError(name, rc, lib().cbmv_last_error().decode(errors="replace"))
    return rc


def default_params(**overrides):
    p = cbmv_params()
    lib().cbmv_params_default(ctypes.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p
