"""Batches of stereo pairs of uneven size through the learned path, as one
CUDA graph launch (cbmv_batch_* in include/cbmv.h), and the autotuner that
picks the batch's launch shape.

    b = StereoBatch(shapes, streams=4)            # shapes: [(H, W, D), ...]
    disps = b.run_mlp(net, lefts, rights)         # device uint8 images -> device disparities
    t = b.timings()                               # per-pair latency, graph span

The reference runs one pair per process (main.py:53-70); a batch keeps the
B200 busy with many small pairs at once: the pairs are spread over `streams`
concurrent contexts, and the graph replays every pair's kernels with one
host call.
"""
import ctypes
import hashlib
import json
import os
import time

import numpy as np

from . import _dev, _lib


class StereoBatch:
    def __init__(self, shapes, streams=4):
        _dev.require_cuda()
        import torch
        self.shapes = [(int(h), int(w), int(d)) for h, w, d in shapes]
        n = len(self.shapes)
        H = np.array([s[0] for s in self.shapes], np.int64)
        W = np.array([s[1] for s in self.shapes], np.int64)
        D = np.array([s[2] for s in self.shapes], np.int32)
        h = ctypes.c_void_p()
        _lib.call("cbmv_batch_create", n, H.ctypes.data, W.ctypes.data, D.ctypes.data, int(streams),
                  ctypes.byref(h))
        self.h = h
        self.streams = int(streams)
        self.disp = [torch.empty((s[0], s[1]), dtype=torch.float32, device="cuda") for s in self.shapes]
        self._disp_ptrs = np.array([t.data_ptr() for t in self.disp], np.uint64)

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().cbmv_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run_mlp(self, net, lefts, rights, params=None):
        """lefts/rights: device uint8 tensors of the batch's shapes; returns the
        batch's device disparity maps (overwritten by the next run)."""
        prm = params if params is not None else _lib.default_params()
        for (h, w, _), l, r in zip(self.shapes, lefts, rights):
            if tuple(l.shape) != (h, w) or tuple(r.shape) != (h, w) or not l.is_cuda or not r.is_cuda:
                raise ValueError("images must be device uint8 tensors of the batch's shapes")
        lp = np.array([t.data_ptr() for t in lefts], np.uint64)
        rp = np.array([t.data_ptr() for t in rights], np.uint64)
        self._keep = (lefts, rights, lp, rp)  # the graph holds these addresses
        _lib.call("cbmv_batch_run_mlp", self.h, net.h, ctypes.byref(prm), lp.ctypes.data, rp.ctypes.data,
                  self._disp_ptrs.ctypes.data, _dev.stream_ptr())
        return self.disp

    def timings(self):
        """Per-pair ms from its first kernel to its last, ms from the graph's
        start to each pair's end, and the graph's span (after the run)."""
        n = len(self.shapes)
        pair = np.zeros(n, np.float32)
        done = np.zeros(n, np.float32)
        total = ctypes.c_float()
        _lib.call("cbmv_batch_timings", self.h, pair.ctypes.data, done.ctypes.data, ctypes.byref(total))
        return {"pair_ms": pair, "done_ms": done, "total_ms": float(total.value)}


# ----------------------------------------------------------------- autotuner
CANDIDATE_STREAMS = (1, 2, 4, 8)


def _signature(shapes):
    import torch
    key = json.dumps([torch.cuda.get_device_name(), sorted(shapes)])
    return hashlib.sha1(key.encode()).hexdigest()[:16]


def default_cache_path():
    return os.path.join(os.path.expanduser("~"), ".cache", "cbmv_b200", "autotune.json")


def tune_batch(shapes, net, lefts, rights, streams=CANDIDATE_STREAMS, mlp_ctas=(0, None), iters=2,
               cache_path=None, log=None, tile_search=True):
    """Pick the batch's launch shape by timing it: the number of concurrent
    contexts and the classifier kernel's CTA cap (0 = every SM, None = the
    SM count divided by the number of contexts), then (tile_search) the
    kernel tile shapes, one at a time from the best: rows per CBCA tile
    (32, 16) and SGM prefetch depth (default, 1, 4).  None of these change
    the results.  Each candidate is captured, run once untimed and `iters`
    times timed (graph span, CUDA events); the fastest is cached per (GPU,
    batch shapes) in a JSON file.  Returns {"streams", "mlp_ctas",
    "cbca_rows", "sgm_prefetch", "ms", "tried": [...]}."""
    import torch
    shapes = [tuple(int(v) for v in s) for s in shapes]
    cache_path = cache_path or default_cache_path()
    sig = _signature(shapes)
    cache = {}
    if os.path.exists(cache_path):
        try:
            cache = json.load(open(cache_path))
        except (OSError, ValueError):
            cache = {}
    if sig in cache:
        return dict(cache[sig], cached=True)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    tried = []

    def measure(b, cand):
        prm = _lib.default_params(mlp_ctas=cand["mlp_ctas"], cbca_rows=cand["cbca_rows"],
                                  sgm_prefetch=cand["sgm_prefetch"])
        b.run_mlp(net, lefts, rights, prm)
        torch.cuda.synchronize()
        spans = []
        for _ in range(iters):
            b.run_mlp(net, lefts, rights, prm)
            torch.cuda.synchronize()
            spans.append(b.timings()["total_ms"])
        cand = dict(cand, ms=float(np.median(spans)))
        tried.append(cand)
        if log:
            log("autotune: " + ", ".join("%s %s" % (k, v) for k, v in cand.items()))
        return cand

    for k in streams:
        if k > len(shapes):
            continue
        b = StereoBatch(shapes, streams=k)
        for cap in mlp_ctas:
            c = 0 if cap == 0 else (max(1, sms // k) if cap is None else int(cap))
            if c and c >= sms:
                continue
            measure(b, {"streams": k, "mlp_ctas": c, "cbca_rows": 32, "sgm_prefetch": 0})
        b.close()
        torch.cuda.synchronize()
    best = min(tried, key=lambda t: t["ms"])
    if tile_search:
        b = StereoBatch(shapes, streams=best["streams"])
        for key, values in (("cbca_rows", (16,)), ("sgm_prefetch", (1, 4))):
            for v in values:
                cand = measure(b, dict({k: best[k] for k in ("streams", "mlp_ctas", "cbca_rows", "sgm_prefetch")},
                                       **{key: v}))
                if cand["ms"] < best["ms"]:
                    best = cand
        b.close()
        torch.cuda.synchronize()
    res = {"streams": best["streams"], "mlp_ctas": best["mlp_ctas"], "cbca_rows": best["cbca_rows"],
           "sgm_prefetch": best["sgm_prefetch"], "ms": best["ms"], "tried": tried,
           "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
    cache[sig] = res
    try:
        os.makedirs(os.path.dirname(cache_path), exist_ok=True)
        json.dump(cache, open(cache_path, "w"), indent=1)
    except OSError:
        pass
    return dict(res, cached=False)
