"""Drop-in for the reference's post module (cpp/post/post.cu:905-933).

Same function names and argument orders as the boost.python module, driven
the same way by Testing.__postprocessing_mem (test.py:341-449).  Device
buffers are CUDA_double_array / CUDA_float_array objects, as in the
reference; both hold float32 on the device (the kernels' working precision
-- the reference itself does its arithmetic in float32 over float64
storage), and get_array returns the dtype the reference returns.  Shape
bookkeeping follows the reference: swap_axis / swap_axis_back /
CUDA_copy_double rewrite the destination's shape (post.cu:612-614, 663-665,
702-704); the other kernels leave it alone.
"""
import numpy as np
import torch

from . import _dev, _lib


class _DeviceArray:
    _out_dtype = None

    def __init__(self, arr):
        a = np.asarray(arr) if not _dev.is_device(arr) else arr
        self.ins = list(a.shape)
        t, _ = _dev.to_device(a, np.float32)
        self.t = t.reshape(-1).clone()

    def _numel(self):
        n = 1
        for s in self.ins:
            n *= int(s)
        return n

    def set_to_zero(self):
        self.t.zero_()

    def get_array(self):
        return self.t[:self._numel()].reshape(self.ins).cpu().numpy().astype(self._out_dtype)

    def free_array(self):
        self.t = torch.empty(0, device="cuda")

    @property
    def ptr(self):
        return self.t.data_ptr()


class CUDA_double_array(_DeviceArray):
    """post.cu:63-116 (float64 on the host side, float32 on the device)."""
    _out_dtype = np.float64


class CUDA_float_array(_DeviceArray):
    """post.cu:118-170."""
    _out_dtype = np.float32


def _s():
    return _dev.stream_ptr()


def InitCUDA():
    """post.cu:874-901: true when a CUDA device is present."""
    ok = torch.cuda.is_available()
    if ok:
        torch.cuda.init()
    return ok


def cross(img, out, L1, tau1):
    H, W = img.ins
    _lib.call("cbmv_cross", img.ptr, H, W, int(L1), float(tau1), out.ptr, _s())


def sgm(left, right, in_cost, out_cost, tmp, pi1, pi2, tau_so, alpha1, sgm_q1, sgm_q2, direction):
    """post.cu:263-333: out_cost += the four scan directions' path costs of
    in_cost ([H,W,D]).  `tmp` is the reference's per-line scratch; the path
    values live in registers here, so it is unused."""
    H, W, D = in_cost.ins
    _lib.call("cbmv_sgm", left.ptr, right.ptr, in_cost.ptr, H, W, D, float(pi1), float(pi2),
              float(tau_so), float(alpha1), float(sgm_q1), float(sgm_q2), int(direction),
              out_cost.ptr, _s())


def cbca(leftc, rightc, vol, vol_out, direction):
    """post.cu:399-450 on a [D,H,W] volume."""
    D, H, W = vol.ins
    _lib.call("cbmv_cbca", leftc.ptr, rightc.ptr, vol.ptr, H, W, D, _lib.DHW, int(direction),
              vol_out.ptr, _s())


def subpixel_enchancement(d, cost, out):
    """post.cu:453-483; cost is [D,H,W]."""
    D, H, W = cost.ins
    _lib.call("cbmv_subpixel", d.ptr, cost.ptr, H, W, D, _lib.DHW, out.ptr, _s())


def median2d(img, out, kernel_size):
    H, W = img.ins
    _lib.call("cbmv_median2d", img.ptr, H, W, int(kernel_size), out.ptr, _s())


def mean2d(img, out, kernel, alpha2):
    H, W = img.ins
    k, _ = _dev.to_device(np.asarray(kernel, np.float32), np.float32)
    _lib.call("cbmv_mean2d", img.ptr, H, W, k.data_ptr(), int(k.shape[0]), float(alpha2), out.ptr,
              _s())


def swap_axis(a, out):
    """post.cu:569-616: [D,H,W] -> [H,W,D]."""
    D, H, W = a.ins
    _lib.call("cbmv_transpose_f32", a.ptr, H, W, D, _lib.HWD, out.ptr, _s())
    out.ins = [H, W, D]


def swap_axis_back(a, out):
    """post.cu:619-667: [H,W,D] -> [D,H,W]."""
    H, W, D = a.ins
    _lib.call("cbmv_transpose_f32", a.ptr, H, W, D, _lib.DHW, out.ptr, _s())
    out.ins = [D, H, W]


def CUDA_copy_double(a, out):
    out.t[:a.t.numel()].copy_(a.t)
    out.ins = list(a.ins)


def CUDA_copy_float(a, out):
    out.t[:a.t.numel()].copy_(a.t)


def CUDA_divide_double(a, val):
    _lib.call("cbmv_scale_f32", a.ptr, a.t.numel(), float(1.0 / val), _s())


def outlier_detection(d0, d1, outlier, disp_max):
    H, W = d0.ins
    _lib.call("cbmv_outlier_detection", d0.ptr, d1.ptr, H, W, int(disp_max), outlier.ptr, _s())


def interpolate_mismatch(d0, outlier, out):
    H, W = d0.ins
    _lib.call("cbmv_interpolate_mismatch", d0.ptr, outlier.ptr, H, W, out.ptr, _s())


def interpolate_occlusion(d0, outlier, out):
    H, W = d0.ins
    _lib.call("cbmv_interpolate_occlusion", d0.ptr, outlier.ptr, H, W, out.ptr, _s())
