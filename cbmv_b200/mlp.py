"""The learned classifier: a 16-bit MLP (bf16 training; f16 or bf16 fused
inference) standing in for the reference's random
forest (test.py:603-620) as the per-(pixel, d) matching-probability model.

    net = MlpParams.init(seed, stats)        # fresh weights + input transform
    tr = MlpTrainer(net, batch=8192)         # device state, tcgen05 GEMMs
    loss = tr.step(X, y, lr)                 # X [B,20] float32, y [B] (1 = correct)
    net = tr.params()

Architecture 20 -> 128 -> 128 -> 64 -> 1 with GELU (or ReLU) hidden
layers and a sigmoid output P(correct); the matching cost handed to the
post-processing is 1 - P, as the reference hands it P(class 0) of the
forest.  The parameter vector layout is documented in include/cbmv.h
(cbmv_mlp_*); the activation is stored beside it ("gelu" or "relu").
"""
import ctypes

import numpy as np

from . import _dev, _lib

F = 20
LAYERS = [(128, F), (128, 128), (64, 128)]
ACTIVATIONS = {"relu": 0, "gelu": 1}  # CBMV_ACT_RELU, CBMV_ACT_GELU
PRECISIONS = {"f16": 0, "bf16": 1}  # CBMV_PREC_F16, CBMV_PREC_BF16


def num_params():
    return _lib.lib().cbmv_mlp_num_params()


class MlpParams:
    """Host-side parameter vector with named views."""

    def __init__(self, vec, activation="relu"):
        self.vec = np.ascontiguousarray(vec, np.float32)
        assert self.vec.size == num_params()
        if activation not in ACTIVATIONS:
            raise ValueError("activation must be one of %s" % sorted(ACTIVATIONS))
        self.activation = activation

    def views(self):
        v, o, out = self.vec, 0, {}
        for name, size in [("cap", F), ("mu", F), ("inv_sd", F), ("W1", 128 * F), ("b1", 128),
                           ("W2", 128 * 128), ("b2", 128), ("W3", 64 * 128), ("b3", 64),
                           ("w4", 64), ("b4", 1)]:
            out[name] = v[o:o + size]
            o += size
        out["W1"] = out["W1"].reshape(128, F)
        out["W2"] = out["W2"].reshape(128, 128)
        out["W3"] = out["W3"].reshape(64, 128)
        return out

    @classmethod
    def init(cls, seed, cap, mu, sd, activation="relu"):
        rng = np.random.default_rng(seed)
        vec = np.zeros(num_params(), np.float32)
        p = cls(vec, activation)
        v = p.views()
        v["cap"][:] = cap
        v["mu"][:] = mu
        v["inv_sd"][:] = 1.0 / np.maximum(sd, 1e-12)
        for (n, k), name in zip(LAYERS + [(1, 64)], ["W1", "W2", "W3", "w4"]):
            # He-uniform into the hidden layers, Glorot-uniform into the output
            lim = np.sqrt(6.0 / k) if n > 1 else np.sqrt(6.0 / (k + n))
            v[name][...] = rng.uniform(-lim, lim, v[name].shape).astype(np.float32)
        return p

    def save(self, path):
        np.savez(path, params=self.vec, activation=np.array(self.activation))

    @classmethod
    def load(cls, path):
        z = np.load(path)
        return cls(z["params"], str(z["activation"]) if "activation" in z.files else "relu")


def input_stats(X):
    """Input transform fitted on raw features X [N,20]: cap = largest value
    below the cost sentinel (RAND_MAX), then mean / std of min(x, cap)."""
    X = np.asarray(X, np.float64)
    sentinel = X >= 1e9
    cap = np.where(sentinel, -np.inf, X).max(axis=0)
    cap = np.where(np.isfinite(cap), cap, 1.0)
    Xc = np.minimum(X, cap[None, :])
    return cap.astype(np.float32), Xc.mean(axis=0).astype(np.float32), Xc.std(axis=0).astype(np.float32)


class MlpTrainer:
    def __init__(self, params, batch=8192):
        _dev.require_cuda()
        self.batch = int(batch)
        h = ctypes.c_void_p()
        _lib.call("cbmv_mlp_create", self.batch, ctypes.byref(h))
        self.h = h
        self.set_params(params)
        import torch
        self._loss = torch.zeros(1, device="cuda")

    def set_params(self, params):
        _lib.call("cbmv_mlp_set_params", self.h, params.vec.ctypes.data)
        _lib.call("cbmv_mlp_set_activation", self.h, ACTIVATIONS[params.activation])
        self.activation = params.activation

    def params(self):
        out = np.empty(num_params(), np.float32)
        _lib.call("cbmv_mlp_get_params", self.h, out.ctypes.data)
        return MlpParams(out, self.activation)

    def step(self, X, y, lr, weight_decay=0.0):
        """X, y: torch CUDA float32 tensors [batch,20], [batch]; returns the
        loss as a device tensor (no synchronisation)."""
        _lib.call("cbmv_mlp_train_step", self.h, X.data_ptr(), y.data_ptr(), float(lr),
                  float(weight_decay), self._loss.data_ptr(), _dev.stream_ptr())
        return self._loss

    def gradients(self, X, y):
        import torch
        g = torch.empty(num_params() - 3 * F, device="cuda")
        loss = torch.empty(1, device="cuda")
        _lib.call("cbmv_mlp_gradients", self.h, X.data_ptr(), y.data_ptr(), g.data_ptr(),
                  loss.data_ptr(), _dev.stream_ptr())
        return g, loss

    def status(self):
        s = ctypes.c_int()
        _lib.call("cbmv_mlp_status", self.h, ctypes.byref(s))
        return s.value

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().cbmv_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuMlp:
    """A trained network uploaded for inference (cbmv_run_mlp).

    precision: operand type of the fused inference, "f16" (the default:
    the faster and the more precise of the two) or "bf16"."""

    def __init__(self, params, precision="f16"):
        _dev.require_cuda()
        h = ctypes.c_void_p()
        _lib.call("cbmv_mlp_create", 128, ctypes.byref(h))
        self.h = h
        _lib.call("cbmv_mlp_set_params", self.h, params.vec.ctypes.data)
        _lib.call("cbmv_mlp_set_activation", self.h, ACTIVATIONS[params.activation])
        self.activation = params.activation
        self.set_precision(precision)

    @classmethod
    def load(cls, path, precision="f16"):
        return cls(MlpParams.load(path), precision)

    def set_precision(self, precision):
        if precision not in PRECISIONS:
            raise ValueError("precision must be one of %s" % sorted(PRECISIONS))
        _lib.call("cbmv_mlp_set_precision", self.h, PRECISIONS[precision])
        self.precision = precision

    def status(self):
        s = ctypes.c_int()
        _lib.call("cbmv_mlp_status", self.h, ctypes.byref(s))
        return s.value

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().cbmv_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
