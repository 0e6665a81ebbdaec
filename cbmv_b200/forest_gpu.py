"""GPU random forest: the drop-in for RandomForestClassifier.predict_proba
as the reference calls it (test.py:603-620).

    gf = GpuForest.from_sklearn(rf)          # or GpuForest.load("forest.npz")
    proba = gf.predict_proba(features)       # [N,2] float64, like sklearn
    leaves = gf.apply(features)              # [N,n_trees] sklearn node ids

Features are cast to float32 as sklearn does before its walk.
"""
import ctypes

import numpy as np

from . import _dev, _lib
from .forest import FlatForest


class GpuForest:
    def __init__(self, flat):
        self.flat = flat
        blocks, leafv, offs, leaf_node = flat.pack()
        self.n_trees = flat.n_trees
        self.n_features = flat.n_features
        self.n_blocks = int(blocks.shape[0])
        self._leaf_node = leaf_node
        h = ctypes.c_void_p()
        _dev.require_cuda()
        _lib.call("cbmv_forest_create", blocks.ctypes.data, blocks.shape[0], leafv.ctypes.data,
                  leafv.shape[0], offs.ctypes.data, flat.n_trees, flat.n_features, ctypes.byref(h))
        self.handle = h

    @classmethod
    def from_sklearn(cls, rf):
        return cls(FlatForest.from_sklearn(rf))

    @classmethod
    def load(cls, path):
        return cls(FlatForest.load(path))

    def close(self):
        if getattr(self, "handle", None):
            _lib.lib().cbmv_forest_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _run(self, X, want_leaves):
        x, host = _dev.to_device(X, np.float32)
        if x.dim() != 2 or x.shape[1] != self.n_features:
            raise ValueError("X must be [N, %d]" % self.n_features)
        N = int(x.shape[0])
        proba = _dev.empty((N, 2), np.float64)
        leaves = _dev.empty((N, self.n_trees), np.int32) if want_leaves else None
        _lib.call("cbmv_forest_predict", self.handle, _dev.ptr(x), N, _dev.ptr(proba),
                  _dev.ptr(leaves) if want_leaves else None, _dev.stream_ptr())
        return proba, leaves, host

    def predict_proba(self, X):
        proba, _, host = self._run(X, False)
        return _dev.result(proba, host)

    def apply(self, X):
        """Leaf reached in each tree, in sklearn's node numbering."""
        _, leaves, host = self._run(X, True)
        out = self._leaf_node[leaves.cpu().numpy()].astype(np.int64)
        if host:
            return out
        import torch
        return torch.from_numpy(out).cuda()
