"""The fused CBMV test path on one B200: images -> disparity.

StereoPipeline.run_rf(L, R, D) does on the device what the reference's
main.py:53-70 does on the host (matchers, features, random forest, then
eval_prob with the `_mem` post-processing) and returns the disparity map.
Inputs may be numpy uint8 [H,W] (copied in, result copied out) or torch
CUDA uint8 tensors (result stays on the device).
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

    def run_rf(self, left, right, ndisp, disp_out=None, prob_out=None):
        l, host = _dev.to_device(left, np.uint8)
        r, _ = _dev.to_device(right, np.uint8)
        H, W = l.shape
        disp = disp_out if disp_out is not None else _dev.empty((H, W), np.float32)
        _lib.call("cbmv_run_rf", self.ctx, self.forest.handle, ctypes.byref(self.params), l.data_ptr(),
                  r.data_ptr(), H, W, int(ndisp), disp.data_ptr(),
                  prob_out.data_ptr() if prob_out is not None else None)
        return _dev.result(disp, host)

    def timings(self):
        """Stage times of the last run in ms: matchers, feature statistics,
        features+classifier, post, total (after a synchronize)."""
        ms = (ctypes.c_float * 5)()
        _lib.call("cbmv_ctx_timings", self.ctx, ms)
        return dict(zip(["matchers", "stats", "classify", "post", "total"], list(ms)))
