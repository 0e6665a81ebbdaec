"""Drop-in for the reference's libmatchers module (cpp/matchers/matchers.cpp:568-582).

Same function names, argument orders, output shapes and float64 values as
the reference: census -> [H,W,D]; nccNister, sadsob, zsad -> [D,H,W];
sobel -> [H,W].  numpy inputs give numpy outputs (computed on the GPU);
torch CUDA inputs give device tensors.  `dtype=np.float32` and `layout`
("HWD" / "DHW") select other output forms.
"""
import numpy as np

from . import _dev, _lib

_LAYOUT = {"HWD": _lib.HWD, "DHW": _lib.DHW}


def _run(fn, L, R, ndisp, wsize, default_layout, dtype, layout, in_dtype=np.uint8, extra=()):
    l, host = _dev.to_device(L, in_dtype)
    r, _ = _dev.to_device(R, in_dtype)
    if l.dim() != 2 or tuple(l.shape) != tuple(r.shape):
        raise ValueError("left and right images must be 2-D with equal shapes")
    H, W = l.shape
    lay = _LAYOUT[layout or default_layout]
    shape = (H, W, ndisp) if lay == _lib.HWD else (ndisp, H, W)
    out = _dev.empty(shape, dtype)
    dt = _lib.F64 if np.dtype(dtype) == np.float64 else _lib.F32
    _lib.call(fn, _dev.ptr(l), _dev.ptr(r), *extra, H, W, int(ndisp), int(wsize), _dev.ptr(out), dt,
              lay, _dev.stream_ptr())
    return _dev.result(out, host)


def census(left, right, ndisp, wsize, dtype=np.float64, layout=None):
    """matchers.cpp:209-350: census Hamming cost, [H,W,D]."""
    return _run("cbmv_census", left, right, ndisp, wsize, "HWD", dtype, layout)


def nccNister(left, right, ndisp, wsize, dtype=np.float64, layout=None):
    """matchers.cpp:24-205: NCC cost, [D,H,W]."""
    return _run("cbmv_ncc", left, right, ndisp, wsize, "DHW", dtype, layout)


def zsad(left, right, ndisp, wsize, dtype=np.float64, layout=None):
    """matchers.cpp:440-512: zero-mean SAD cost, [D,H,W]."""
    return _run("cbmv_zsad", left, right, ndisp, wsize, "DHW", dtype, layout)


def sadsob(left, right, ndisp, wsize, dtype=np.float64, layout=None):
    """matchers.cpp:353-436: SAD of Sobel responses, [D,H,W].  Inputs are the
    float64 Sobel images from sobel()."""
    l, host = _dev.to_device(left, np.float64)
    r, _ = _dev.to_device(right, np.float64)
    H, W = l.shape
    lay = _LAYOUT[layout or "DHW"]
    shape = (H, W, ndisp) if lay == _lib.HWD else (ndisp, H, W)
    out = _dev.empty(shape, dtype)
    dt = _lib.F64 if np.dtype(dtype) == np.float64 else _lib.F32
    _lib.call("cbmv_sadsob", _dev.ptr(l), _dev.ptr(r), _lib.F64, H, W, int(ndisp), int(wsize),
              _dev.ptr(out), dt, lay, _dev.stream_ptr())
    return _dev.result(out, host)


def sobel(img, dtype=np.float64):
    """matchers.cpp:515-555: horizontal Sobel response, [H,W]."""
    t, host = _dev.to_device(img, np.uint8)
    H, W = t.shape
    out = _dev.empty((H, W), dtype)
    dt = _lib.F64 if np.dtype(dtype) == np.float64 else _lib.F32
    _lib.call("cbmv_sobel", _dev.ptr(t), H, W, _dev.ptr(out), dt, _dev.stream_ptr())
    return _dev.result(out, host)


def initthreads():
    """matchers.cpp:557-566 returns the OpenMP thread count; the GPU path has
    no host threads to start, so this reports the device's SM count."""
    import torch
    _dev.require_cuda()
    return torch.cuda.get_device_properties(0).multi_processor_count
