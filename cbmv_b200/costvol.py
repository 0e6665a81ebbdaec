"""Cost-volume files: the reference's `--saveCostVolume` / `--loadCostVolume`
(main.py:56-67) for the fused pipeline.

The reference saves the random forest's `predict_proba` output, an [N, 2]
float64 array with N = H*W*D in (row, column, disparity) order, to
`<prob_save_path><test_set>.prob.npy`, and on `--loadCostVolume` feeds
column 0 (P(class 0), the matching cost) to the post-processing
(test.py:143-149).  Three layouts are written here, all from the device
volume the pipeline produces (`prob_out` of `StereoPipeline.run_rf/run_mlp`):

- "reference": [N, 2] float64, column 0 the cost and column 1 = 1 - cost,
  readable by the reference's main.py;
- "hwd": float32 [H, W, D], a quarter of the size;
- "dhw": float32 [D, H, W], the layout Local Expansion's unary cost reads
  (test.py:453-482).

`load` returns the float32 [H, W, D] cost for `StereoPipeline.run_post`.
"""
import numpy as np

FORMATS = ("reference", "hwd", "dhw")


def reference_path(prob_save_path, test_set):
    """The file name main.py:56 uses."""
    return prob_save_path + test_set + ".prob.npy"


def save(path, cost, fmt="reference"):
    """cost: [H, W, D] float32, a CUDA tensor or numpy array."""
    if fmt not in FORMATS:
        raise ValueError("fmt must be one of %s" % (FORMATS,))
    try:
        import torch
        is_tensor = isinstance(cost, torch.Tensor)
    except ImportError:
        is_tensor = False
    if cost.ndim != 3:
        raise ValueError("cost must be [H, W, D]")
    if fmt == "dhw":
        c = cost.permute(2, 0, 1).contiguous() if is_tensor else np.ascontiguousarray(np.transpose(cost, (2, 0, 1)))
    else:
        c = cost
    a = c.cpu().numpy() if is_tensor else np.asarray(c)
    a = a.astype(np.float32, copy=False)
    if fmt == "reference":
        p0 = a.reshape(-1).astype(np.float64)
        a = np.stack([p0, 1.0 - p0], axis=1)
    np.save(path, a)


def load(path, shape=None, fmt=None):
    """The float32 [H, W, D] cost in a file written by `save` or by the
    reference's main.py.  An [N, 2] file needs `shape` = (H, W, D); a 3-D
    file is [H, W, D] unless fmt == "dhw"."""
    a = np.load(path)
    if a.ndim == 2 and a.shape[1] == 2:
        if shape is None:
            raise ValueError("an [N, 2] cost file needs shape=(H, W, D)")
        H, W, D = (int(v) for v in shape)
        if a.shape[0] != H * W * D:
            raise ValueError("%d rows do not make %dx%dx%d" % (a.shape[0], H, W, D))
        return np.ascontiguousarray(a[:, 0].reshape(H, W, D), dtype=np.float32)
    if a.ndim != 3:
        raise ValueError("unrecognised cost file of shape %s" % (a.shape,))
    if fmt == "dhw":
        a = np.transpose(a, (1, 2, 0))
    out = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None and out.shape != tuple(int(v) for v in shape):
        raise ValueError("cost is %s, expected %s" % (out.shape, tuple(shape)))
    return out
