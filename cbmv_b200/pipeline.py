"""The fused CBMV test path on one B200: images -> disparity.

StereoPipeline.run_rf(L, R, D) does on the device what the reference's
main.py:53-70 does on the host (matchers, features, random forest, then
eval_prob with the `_mem` post-processing) and returns the disparity map.
Inputs may be host memory -- numpy uint8 [H,W] or CPU tensors, pinned or
not -- (the host-buffer entry points cbmv_run_rf_host / cbmv_run_mlp_host
copy them in and the disparity out; the result is a numpy array, or
`disp_out` when that is a host buffer) or torch CUDA uint8 tensors (result
stays on the device).
"""
import ctypes

import numpy as np

from . import _dev, _lib


class StereoPipeline:
    def __init__(self, forest=None, params=None, stream=None):
        _dev.require_cuda()
        self.forest = forest
        self.params = params if params is not None else _lib.default_params()
        h = ctypes.c_void_p()
        self._stream = stream
        _lib.call("cbmv_ctx_create", stream if stream is not None else _dev.stream_ptr(), ctypes.byref(h))
        self.ctx = h

    def close(self):
        if getattr(self, "ctx", None):
            _lib.lib().cbmv_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _host_call(self, left, right, disp_out, prob_out):
        """True when the call goes through a host-buffer entry point: both
        images and the output (if given) in host memory, no cost volume
        requested."""
        return (prob_out is None and _dev.is_host(left) and _dev.is_host(right)
                and (disp_out is None or _dev.is_host(disp_out)))

    def _run_host(self, fn, model, left, right, ndisp, disp_out):
        l = _dev.host_array(left, np.uint8)
        r = _dev.host_array(right, np.uint8)
        if l.ndim != 2 or tuple(r.shape) != tuple(l.shape):
            raise ValueError("left and right must be [H,W] images of one shape")
        H, W = l.shape
        out = disp_out if disp_out is not None else np.empty((H, W), np.float32)
        if not _dev.host_f32_buffer(out, (H, W)):
            raise ValueError("disp_out must be a writable C-contiguous float32 [H,W] host buffer")
        _lib.call(fn, self.ctx, model, ctypes.byref(self.params), _dev.host_ptr(l), _dev.host_ptr(r), H, W,
                  int(ndisp), _dev.host_ptr(out))
        return out

    def run_rf(self, left, right, ndisp, disp_out=None, prob_out=None):
        if self._host_call(left, right, disp_out, prob_out):
            return self._run_host("cbmv_run_rf_host", self.forest.handle, left, right, ndisp, disp_out)
        l, host = _dev.to_device(left, np.uint8)
        r, _ = _dev.to_device(right, np.uint8)
        H, W = l.shape
        disp = disp_out if disp_out is not None else _dev.empty((H, W), np.float32)
        _lib.call("cbmv_run_rf", self.ctx, self.forest.handle, ctypes.byref(self.params), l.data_ptr(),
                  r.data_ptr(), H, W, int(ndisp), disp.data_ptr(),
                  prob_out.data_ptr() if prob_out is not None else None)
        return _dev.result(disp, host)

    def run_mlp(self, net, left, right, ndisp, disp_out=None, prob_out=None):
        """The same path with the learned classifier (cbmv_b200.mlp.GpuMlp)."""
        if self._host_call(left, right, disp_out, prob_out):
            return self._run_host("cbmv_run_mlp_host", net.h, left, right, ndisp, disp_out)
        l, host = _dev.to_device(left, np.uint8)
        r, _ = _dev.to_device(right, np.uint8)
        H, W = l.shape
        disp = disp_out if disp_out is not None else _dev.empty((H, W), np.float32)
        _lib.call("cbmv_run_mlp", self.ctx, net.h, ctypes.byref(self.params), l.data_ptr(), r.data_ptr(),
                  H, W, int(ndisp), disp.data_ptr(),
                  prob_out.data_ptr() if prob_out is not None else None)
        return _dev.result(disp, host)

    def run_classified(self, left, right, ndisp, net=None, disp_out=None, prob_out=None):
        """The learned classifier with the random forest as its fallback:
        runs `net` (cbmv_b200.mlp.GpuMlp) when given; if that call fails or
        the network reports a tensor-core wait timeout, the pair is run again
        with the pipeline's forest.  Returns (disparity, "mlp" or "rf")."""
        if net is not None:
            try:
                disp = self.run_mlp(net, left, right, ndisp, disp_out=disp_out, prob_out=prob_out)
                if net.status() == 0:
                    return disp, "mlp"
            except _lib.CbmvError:
                pass
        if self.forest is None:
            raise RuntimeError("the learned classifier failed and the pipeline has no forest to fall back on")
        return self.run_rf(left, right, ndisp, disp_out=disp_out, prob_out=prob_out), "rf"

    def run_post(self, left, right, cost, disp_out=None):
        """The post-processing alone on a matching cost [H,W,D] float32 (numpy
        or a CUDA tensor; low = good), e.g. a cost volume saved earlier
        (cbmv_b200.costvol).  Returns the disparity map."""
        l, host = _dev.to_device(left, np.uint8)
        r, _ = _dev.to_device(right, np.uint8)
        c, _ = _dev.to_device(cost, np.float32)
        H, W = l.shape
        if c.dim() != 3 or tuple(c.shape[:2]) != (H, W):
            raise ValueError("cost must be [H,W,D] for images of %dx%d" % (W, H))
        disp = disp_out if disp_out is not None else _dev.empty((H, W), np.float32)
        _lib.call("cbmv_run_post", self.ctx, ctypes.byref(self.params), l.data_ptr(), r.data_ptr(), H, W,
                  int(c.shape[2]), c.contiguous().data_ptr(), disp.data_ptr())
        return _dev.result(disp, host)

    def volumes_f32(self, left, right, ndisp):
        """The learned path's four float32 matcher volumes (census, NCC,
        SAD-on-Sobel, ZSAD) as a device tensor [4,H,W,D]."""
        import torch
        l, _ = _dev.to_device(left, np.uint8)
        r, _ = _dev.to_device(right, np.uint8)
        H, W = l.shape
        out = torch.empty((4, H, W, int(ndisp)), dtype=torch.float32, device="cuda")
        _lib.call("cbmv_ctx_volumes_f32", self.ctx, ctypes.byref(self.params), l.data_ptr(), r.data_ptr(),
                  H, W, int(ndisp), out.data_ptr())
        return out

    def features_at(self, left, right, ndisp, idx, learned=False):
        """20 float32 features of the samples idx = (y*W + x)*D + d (device
        tensor [n,20]): the reference's float64 features rounded to float32
        (what the random forest reads), or with learned=True the learned
        path's own float32 features (what its network reads)."""
        import torch
        l, _ = _dev.to_device(left, np.uint8)
        r, _ = _dev.to_device(right, np.uint8)
        H, W = l.shape
        ix, _ = _dev.to_device(idx, np.int64)
        if ix.numel() and (int(ix.min()) < 0 or int(ix.max()) >= H * W * int(ndisp)):
            raise ValueError("sample index outside the H*W*D volume")
        out = torch.empty((ix.numel(), 20), dtype=torch.float32, device="cuda")
        fn = "cbmv_ctx_features_f32_at" if learned else "cbmv_ctx_features_at"
        _lib.call(fn, self.ctx, ctypes.byref(self.params), l.data_ptr(), r.data_ptr(),
                  H, W, int(ndisp), ix.data_ptr(), ix.numel(), out.data_ptr())
        return out

    def timings(self):
        """Stage times of the last run in ms: matchers, feature statistics,
        features+classifier, post, total (after a synchronize)."""
        ms = (ctypes.c_float * 5)()
        _lib.call("cbmv_ctx_timings", self.ctx, ms)
        return dict(zip(["matchers", "stats", "classify", "post", "total"], list(ms)))
