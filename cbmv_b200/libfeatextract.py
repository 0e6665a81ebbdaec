"""Drop-in for the reference's libfeatextract module
(cpp/featextract/featextract.cpp:519-540), float64 like the reference.

extract_ratio / extract_likelihood keep the reference's arity overloading
(featextract.cpp:533-536): (vol, e) is the test form over an [N,D] volume,
(vol, samples, e) the training form returning [3N].  generate_d_indices takes
an extra `seed`: its negatives come from a counter-based generator (the
reference's rand() inside OpenMP is not reproducible).  `features` is the
fused replacement of Testing.__extract_features_lr (test.py:521-595).
"""
import numpy as np

from . import _dev, _lib


def _vol(a):
    return _dev.to_device(a, np.float64)


def swap_axes(cost):
    c, host = _vol(cost)
    D, H, W = c.shape
    out = _dev.empty((H, W, D), np.float64)
    _lib.call("cbmv_swap_axes", _dev.ptr(c), D, H, W, _dev.ptr(out), _dev.stream_ptr())
    return _dev.result(out, host)


def swap_axes_back(cost):
    c, host = _vol(cost)
    H, W, D = c.shape
    out = _dev.empty((D, H, W), np.float64)
    _lib.call("cbmv_swap_axes_back", _dev.ptr(c), H, W, D, _dev.ptr(out), _dev.stream_ptr())
    return _dev.result(out, host)


def get_cost(cost):
    c, host = _vol(cost)
    H, W, D, K = c.shape
    out = _dev.empty((H, W, D), np.float64)
    _lib.call("cbmv_get_cost", _dev.ptr(c), H, W, D, K, _dev.ptr(out), _dev.stream_ptr())
    return _dev.result(out, host)


def get_right_cost(cost):
    c, host = _vol(cost)
    H, W, D = c.shape
    out = _dev.empty((H, W, D), np.float64)
    _lib.call("cbmv_get_right_cost", _dev.ptr(c), H, W, D, _dev.ptr(out), _dev.stream_ptr())
    return _dev.result(out, host)


def get_left_cost(cost):
    c, host = _vol(cost)
    H, W, D = c.shape
    out = _dev.empty((H, W, D), np.float64)
    _lib.call("cbmv_get_left_cost", _dev.ptr(c), H, W, D, _dev.ptr(out), _dev.stream_ptr())
    return _dev.result(out, host)


def extract_ratio(vol, *args):
    v, host = _vol(vol)
    N, D = v.shape
    if len(args) == 2:
        s, _ = _dev.to_device(args[0], np.int32)
        out = _dev.empty((3 * s.shape[0],), np.float64)
        _lib.call("cbmv_extract_ratio_samples", _dev.ptr(v), N, D, _dev.ptr(s), float(args[1]),
                  _dev.ptr(out), _dev.stream_ptr())
    else:
        out = _dev.empty((N, D), np.float64)
        _lib.call("cbmv_extract_ratio", _dev.ptr(v), N, D, float(args[0]), _dev.ptr(out),
                  _dev.stream_ptr())
    return _dev.result(out, host)


def extract_likelihood(vol, *args):
    v, host = _vol(vol)
    N, D = v.shape
    if len(args) == 2:
        s, _ = _dev.to_device(args[0], np.int32)
        out = _dev.empty((3 * s.shape[0],), np.float64)
        _lib.call("cbmv_extract_likelihood_samples", _dev.ptr(v), N, D, _dev.ptr(s),
                  float(args[1]), _dev.ptr(out), _dev.stream_ptr())
    else:
        out = _dev.empty((N, D), np.float64)
        _lib.call("cbmv_extract_likelihood", _dev.ptr(v), N, D, float(args[0]), _dev.ptr(out),
                  _dev.stream_ptr())
    return _dev.result(out, host)


def get_samples(vol, samples):
    v, host = _vol(vol)
    s, _ = _dev.to_device(samples, np.int32)
    out = _dev.empty((3 * s.shape[0],), np.float64)
    _lib.call("cbmv_get_samples", _dev.ptr(v), v.shape[0], v.shape[1], _dev.ptr(s), _dev.ptr(out),
              _dev.stream_ptr())
    return _dev.result(out, host)


def generate_labels(samples):
    n = int(samples.shape[0])
    host = not _dev.is_device(samples)
    out = _dev.empty((3 * n,), np.int32)
    _lib.call("cbmv_generate_labels", n, _dev.ptr(out), _dev.stream_ptr())
    return _dev.result(out, host)


def generate_d_indices(gt, maxd, dispThresh, seed=0):
    g, host = _dev.to_device(np.asarray(gt).reshape(-1) if not _dev.is_device(gt) else gt.reshape(-1),
                             np.int32)
    out = _dev.empty((g.shape[0], 3), np.int32)
    _lib.call("cbmv_generate_d_indices", _dev.ptr(g), g.shape[0], int(maxd), int(dispThresh),
              int(seed), _dev.ptr(out), _dev.stream_ptr())
    return _dev.result(out, host)


def features(census, ncc, sobel, sad):
    """The 20 features per (pixel, d), float32 [H*W*D, 20], from four [H,W,D]
    float64 volumes -- what __extract_features_lr (test.py:521-595) builds in
    float64 and sklearn then casts to float32."""
    vs = [_vol(v) for v in (census, ncc, sobel, sad)]
    host = vs[0][1]
    H, W, D = vs[0][0].shape
    out = _dev.empty((H * W * D, 20), np.float32)
    _lib.call("cbmv_features", *[_dev.ptr(v) for v, _ in vs], H, W, D, _dev.ptr(out),
              _dev.stream_ptr())
    return _dev.result(out, host)
