"""Benchmark: pixel·disparities per second of the CBMV test path on B200.

Workload: one synthetic rectified pair at 694x554, D=128 (seeded, the
reference's README-scale Middlebury size), 49,212,928 (pixel, d) units.  A
step is the whole test path for that pair: four matchers, 20 features, the
per-(pixel,d) classifier, then the MC-CNN `_mem` post-processing to the
disparity map.  Both classifiers are timed: the random forest (50 trees,
depth <= 20, trained on 30 seeded pairs, tests/golden/make_forest.py) and
the 16-bit MLP 20-128-128-64-1 with GELU hidden layers (f16 inference)
(tests/golden/mlp_gelu_694x554.npz, cbmv_b200/train_mlp.py).  The RF judges
the MLP: both run on 20 held-out seeded pairs and the MLP is the headline
only when its bad-2.0 is within 0.5 percentage points of the RF's.  Beside
the headline: the same network with ReLU (a labelled variant), the
headline network with bf16 operands in its fused inference (a labelled
variant), and the learned path with the `_interp` post (the reference's
LR-check chain).
With N GPUs (torchrun), every rank processes its own pair (seed = rank):
weak scaling by independent pairs, no collective on the data path; with
--batch, the 64 uneven pairs are split over the ranks (strong scaling) and
gathered on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cbmv|reference]

(started directly with --gpus N > 1 it relaunches itself under torchrun, one
process per GPU; under torchrun --gpus must equal WORLD_SIZE)

`value` is device time with the images resident in HBM and L2 flushed
between steps; `e2e` is the same metric through the public call with pinned
host buffers, i.e. the C ABI's host-buffer entry point cbmv_run_mlp_host
(H2D of both images and D2H of the disparity inside the timed region).  `--impl reference` times the reference's own implementation of the
path on whole pairs: its C++ matchers and feature extraction compiled
unmodified (oracle/_ref) and batched as its test.py does, scikit-learn's
predict_proba on the same forest, and its post.cu on the GPU (as shipped;
the CPU restatement when that build is absent) on that classifier's own
P(class 0).
"""
import argparse
import contextlib
import ctypes
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FOREST = os.path.join(ROOT, "tests", "golden", "forest_694x554.npz")
MLP = os.path.join(ROOT, "tests", "golden", "mlp_gelu_694x554.npz")       # the GELU network of record
MLP_RELU = os.path.join(ROOT, "tests", "golden", "mlp_694x554.npz")      # the ReLU variant
W0, H0, D0 = 694, 554, 128
UNITS = W0 * H0 * D0
METRIC = "pixel·disparities/s end-to-end at 694×554, D=128; MLP vs RF at matched bad-2.0"
BYTES_PER_UNIT_FUSED = 4.0  # algorithmic HBM bytes of matchers+features+classifier per (p,d)
BYTES_PER_UNIT_PATH = 80.0  # algorithmic HBM bytes per (p,d) of the whole path with the _mem post
BYTES_PER_UNIT_INTERP = 156.0  # the same with the _interp post (the right view's chain added)
REF_BUDGET_S = 100  # the reference arm's timed whole-pair steps stop after this many seconds
# dense flops of the 20-128-128-64-1 network per (p,d): 2*(20*128 + 128*128 + 128*64 + 64)
FLOPS_PER_UNIT_MLP = 2.0 * (20 * 128 + 128 * 128 + 128 * 64 + 64)
# MMA work the fused kernel issues per (pixel, d): layer 1 K = 32 (20 inputs + 2 bias ones + padding),
# the K = 16 bias MMAs of layers 2 and 3, layer 4 as N = 16 (w4 high + low rows and padding)
MMA_FLOPS_PER_UNIT_MLP = 2 * (32 * 128 + 16 * 128 + 128 * 128 + 16 * 64 + 128 * 64 + 64 * 16)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def tensor_peak():
    """Dense bf16 TFLOP/s: the burst figure (the classifier kernel runs for
    milliseconds inside a step, not a seconds-long loop)."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        if "bf16_tflops" in d:
            return float(d["bf16_tflops"]), "measured (burst)"
    return 1590.0, "fallback (burst)"


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.p:
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
                self.out, _ = self.p.communicate()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def env_ranks():
    """(world size, rank, local rank) as torchrun sets them."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def dist_init():
    ws, rank, local = env_ranks()
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def reduce_max(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    import torch
    torch.cuda.synchronize()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()


def _time_path(run, a, ws, flush, st, pipe):
    """Device time of `a.steps` runs (L2 flushed before each) and the mean
    stage times; returns (ms, stage)."""
    import torch
    for _ in range(a.warmup):
        run()
    barrier(ws)
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    stage = {"matchers": 0.0, "stats": 0.0, "classify": 0.0, "post": 0.0, "total": 0.0}
    for k in range(a.steps):
        flush.fill_(float(k))
        ev0[k].record(st)
        run()
        ev1[k].record(st)
        st.synchronize()
        for kk, v in pipe.timings().items():
            stage[kk] += v
    barrier(ws)
    ms = sum(e0.elapsed_time(e1) for e0, e1 in zip(ev0, ev1)) / a.steps
    return reduce_max(ms, ws), {k: v / a.steps for k, v in stage.items()}


def _time_e2e(run_host, a, ws, flush, st):
    """Wall time of the public call with pinned host buffers, which goes
    through the C ABI's host-buffer entry point (cbmv_run_mlp_host /
    cbmv_run_rf_host: H2D of both images, the whole path, D2H of the
    disparity map and the stream synchronisation inside the timed region)."""
    for _ in range(2):
        run_host()
    barrier(ws)
    tot = 0.0
    for k in range(a.steps):
        flush.fill_(float(k))
        st.synchronize()
        t0 = time.perf_counter()
        run_host()
        tot += (time.perf_counter() - t0) * 1e3
    return reduce_max(tot / a.steps, ws)


def clk_max_mhz():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p)).get("sm_max_mhz", 1965.0))
    return 1965.0


def forest_visits_per_unit(pipe, gf, flat, l, r, n=65536):
    """Mean comparisons per (pixel, d) over all trees: the depth of the leaf
    each tree's walk reaches, for n sampled (p,d) of the pair (the forest
    path's own features and leaves)."""
    import torch
    H, W = l.shape
    rng = np.random.default_rng(0)
    idx = torch.from_numpy(rng.integers(0, H * W * D0, n, dtype=np.int64)).cuda()
    X = pipe.features_at(l, r, D0, idx)
    leaves = gf.apply(X).cpu().numpy()  # sklearn node ids [n, T]
    depth = flat.node_depths()
    return float(depth[flat.roots[None, :].astype(np.int64) + leaves].sum(axis=1).mean())


def launches_per_pair(prm, classifier="mlp"):
    """Kernel launches of one cbmv_run_mlp / cbmv_run_rf call (pipeline.cu)
    for parameters prm.  Front end: census descriptors, NCC sums and Sobel of
    both images (6) plus the ZSAD window means (2) except on the learned path
    with window 5, whose strip kernel forms them itself; 4 cost volumes; the
    row statistics (learned path 2, forest path one per volume, 4); 1
    features + classifier.  Post: image normalisation (4), cross arms (2),
    the SGM neighbour differences (2, with any SGM iteration); per cost
    chain one CBCA support build (when the passes read precomputed
    supports, L1 <= 6 and not exact_cbca) and one launch per CBCA pass, 2
    per SGM iteration; WTA + subpixel; with interpolate the right view's
    cost (1), its chain and its WTA (1), and the left-right check and fills
    (3); median per iteration; mean2d.  33 (learned) and 37 (forest) with
    the defaults, as the ncu launch lists of the headline step count them
    per pass."""
    f32 = classifier == "mlp"
    front = 6 + (0 if (f32 and prm.sadw == 5) else 2) + 4 + (2 if f32 else 4) + 1
    masked = not prm.exact_cbca and prm.L1 - 1 <= 5
    passes = prm.cbca_i1 + prm.cbca_i2
    chain = (1 if masked and passes else 0) + passes + 2 * prm.sgm_i
    post = 4 + 2 + (2 if prm.sgm_i else 0) + chain + 1 + prm.median_i + 1
    if prm.interpolate:
        post += 1 + chain + 1 + 3
    return front + post


def run_cbmv(a, ws, rank, local):
    import torch
    from cbmv_b200 import evaluate, synth
    from cbmv_b200._lib import default_params as _default_params
    from cbmv_b200.forest import FlatForest
    from cbmv_b200.forest_gpu import GpuForest
    from cbmv_b200.mlp import GpuMlp
    from cbmv_b200.pipeline import StereoPipeline

    have_forest = os.path.exists(a.forest)
    if not have_forest and a.classifier != "mlp":
        raise SystemExit("forest fixture missing: run `python tests/golden/make_forest.py` (%s)" % a.forest)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    L, R, gt, nonocc = synth.pair_694x554(seed=rank)
    if a.height != H0:
        L, R, gt, nonocc = (v[:a.height].copy() for v in (L, R, gt, nonocc))
    units = L.shape[0] * W0 * D0
    flat = FlatForest.load(a.forest) if have_forest else None
    gf = GpuForest(flat) if have_forest else None
    net = GpuMlp.load(a.mlp, a.mlp_precision) if os.path.exists(a.mlp) else None
    pipe = StereoPipeline(gf)
    l = torch.from_numpy(L).to(dev)
    r = torch.from_numpy(R).to(dev)
    disp = torch.empty(L.shape, dtype=torch.float32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # 256 MB > L2
    st = torch.cuda.current_stream()
    Lh = torch.from_numpy(L).pin_memory()
    Rh = torch.from_numpy(R).pin_memory()
    Dh = torch.empty(L.shape, dtype=torch.float32).pin_memory()

    if a.classifier == "mlp" and net is None:
        raise SystemExit("MLP parameters missing: %s (python -m cbmv_b200.train_mlp)" % a.mlp)
    paths = {}
    if a.classifier in ("both", "rf"):
        paths["rf"] = (lambda: pipe.run_rf(l, r, D0, disp_out=disp), lambda: pipe.run_rf(Lh, Rh, D0, disp_out=Dh))
    if a.classifier in ("both", "mlp") and net is not None:
        paths["mlp"] = (lambda: pipe.run_mlp(net, l, r, D0, disp_out=disp),
                        lambda: pipe.run_mlp(net, Lh, Rh, D0, disp_out=Dh))
    res = {}
    relu = bf16v = None
    with Clocks(local) as clk:
        for name, (run_dev, run_host) in paths.items():
            ms, stage = _time_path(run_dev, a, ws, flush, st, pipe)
            d = disp.cpu().numpy()
            res[name] = {"ms": ms, "stage_ms": stage, "bad2_nonocc": evaluate.bad_x(d, gt, nonocc)}
        # the same architecture with ReLU hidden layers, a labelled variant
        if a.classifier in ("both", "mlp") and os.path.exists(a.mlp_relu) and not a.device_only:
            net_r = GpuMlp.load(a.mlp_relu)
            ms_r, stage_r = _time_path(lambda: pipe.run_mlp(net_r, l, r, D0, disp_out=disp), a, ws, flush, st, pipe)
            relu = {"activation": net_r.activation, "ms_per_step": ms_r, "value": units * ws / (ms_r / 1e3),
                    "stage_ms": stage_r, "bad2_nonocc": evaluate.bad_x(disp.cpu().numpy(), gt, nonocc),
                    "classify_tflops": FLOPS_PER_UNIT_MLP * units / (stage_r["classify"] / 1e3) / 1e12}
            net_r.close()
        # the headline network with bf16 operands in the fused inference, a labelled variant
        if net is not None and a.classifier in ("both", "mlp") and not a.device_only \
                and a.mlp_precision == "f16":
            net.set_precision("bf16")
            ms_b, stage_b = _time_path(lambda: pipe.run_mlp(net, l, r, D0, disp_out=disp), a, ws, flush, st, pipe)
            bf16v = {"precision": "bf16", "activation": net.activation, "ms_per_step": ms_b,
                     "value": units * ws / (ms_b / 1e3), "stage_ms": stage_b,
                     "bad2_nonocc": evaluate.bad_x(disp.cpu().numpy(), gt, nonocc),
                     "classify_tflops": FLOPS_PER_UNIT_MLP * units / (stage_b["classify"] / 1e3) / 1e12}
            net.set_precision("f16")
    for name, (_, run_host) in paths.items():
        res[name]["e2e_ms"] = _time_e2e(run_host, a, ws, flush, st) if not a.device_only else None
    # the _interp post (test.py:153-338: the right view's chain, the left-right
    # check and its fills) as a separate variant of the learned path
    interp = None
    if net is not None and a.classifier in ("both", "mlp") and not a.device_only:
        pipe_i = StereoPipeline(gf, params=_default_params(interpolate=1))
        ms_i, stage_i = _time_path(lambda: pipe_i.run_mlp(net, l, r, D0, disp_out=disp), a, ws, flush, st, pipe_i)
        hbm_i, _ = peaks()
        interp = {"ms_per_step": ms_i, "value": units * ws / (ms_i / 1e3), "stage_ms": stage_i,
                  "bad2_nonocc": evaluate.bad_x(disp.cpu().numpy(), gt, nonocc),
                  "whole_path": {"bytes_per_unit": BYTES_PER_UNIT_INTERP,
                                 "achieved": BYTES_PER_UNIT_INTERP * units / (ms_i / 1e3) / 1e9,
                                 "frac": BYTES_PER_UNIT_INTERP * units / (ms_i / 1e3) / 1e9 / hbm_i,
                                 "unit": "GB/s"}}
        pipe_i.close()
    if net is not None and net.status() != 0:
        raise RuntimeError("a tensor-core wait of the MLP kernel timed out")

    # held-out accuracy: the RF judges the MLP (bad-2.0 on 20 seeded pairs)
    matched = None
    if net is not None and a.classifier == "both" and not a.no_eval and not a.device_only and rank == 0:
        ev = evaluate.compare_loaded(pipe, net, evaluate.HELD_OUT, D0)
        matched = {"seeds": "%d-%d" % (ev["seeds"][0], ev["seeds"][-1]), "bad2_rf": ev["bad2_rf"],
                   "bad2_mlp": ev["bad2_mlp"], "delta_pp": 100 * (ev["bad2_mlp"] - ev["bad2_rf"]),
                   "within_0.5pp": bool(ev["bad2_mlp"] - ev["bad2_rf"] <= 0.005)}
    # the headline classifier: the MLP where it matches the RF's bad-2.0, else the RF
    if a.classifier == "both":
        head = "mlp" if matched is not None and matched["within_0.5pp"] else "rf"
    else:
        head = a.classifier
    h = res[head]

    launches = launches_per_pair(pipe.params, head)

    hbm, hbm_kind = peaks()
    tc, tc_kind = tensor_peak()
    traffic = {}
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        traffic = json.load(open(tp))
    if "rf" in res:
        visits = forest_visits_per_unit(pipe, gf, flat, l, r) if not a.device_only else 0.0
        t_rf = res["rf"]["stage_ms"]["classify"] / 1e3
        rf_achieved = visits * units / t_rf
        sm_count = torch.cuda.get_device_properties(dev).multi_processor_count
        mhz = clk_max_mhz()
        # L1 sector bound of the walk: each lane's next 32-byte node block (two tree
        # levels) is a different sector; an SM's L1 returns 4 sectors (128 B) per clock
        rf_peak = sm_count * 4 * 2 * mhz * 1e6
        res["rf"]["roofline"] = {
            "bound": "l1", "kernel": "features_rf_tiled", "achieved": rf_achieved, "peak": rf_peak,
            "unit": "node-visits/s", "frac": rf_achieved / rf_peak,
            "traffic": traffic.get("features_rf_kernel"), "peak_kind": "derived (L1 sectors/clock)",
            "visits_per_unit": visits,
            "note": "node visits = comparisons per (pixel,d) summed over the 50 trees (mean over 65,536 "
                    "sampled (p,d) of this pair); peak = SMs x 4 sectors/clock x 2 levels per 32-byte "
                    "block x max SM clock; HBM: %.0f GB/s of %.0f for 4 B/(p,d)"
                    % (BYTES_PER_UNIT_FUSED * units / t_rf / 1e9, hbm)}
    if "mlp" in res:
        mlp_tflops = FLOPS_PER_UNIT_MLP * units / (res["mlp"]["stage_ms"]["classify"] / 1e3) / 1e12
        t_cls = res["mlp"]["stage_ms"]["classify"]
        mma_floor_ms = MMA_FLOPS_PER_UNIT_MLP * units / (tc * 1e12) * 1e3
        roof_mlp = {"bound": "tensor", "kernel": "features_mlp_kernel", "achieved": mlp_tflops,
                    "peak": tc, "unit": "TFLOP/s", "frac": mlp_tflops / tc,
                    "traffic": traffic.get("features_mlp_kernel"), "peak_kind": tc_kind,
                    "flops_per_unit": FLOPS_PER_UNIT_MLP,
                    "mma_issued": {"flops_per_unit": MMA_FLOPS_PER_UNIT_MLP, "floor_ms": mma_floor_ms,
                                   "frac": mma_floor_ms / t_cls,
                                   "note": "tensor time of the MMAs as issued (padding and bias MMAs "
                                           "included) at the measured peak"},
                    "note": "dense flops of 20-128-128-64-1 per (pixel,d); the kernel also builds "
                            "the 20 features from the four float32 cost volumes"}
        ipu = traffic.get("features_mlp_kernel_warp_inst_per_unit")
        if ipu:
            # the bound the kernel actually meets: instruction issue (one warp
            # instruction per clock per SM sub-partition); the GELU epilogues
            # and the features are CUDA-core work beside the MMAs
            sm_count = torch.cuda.get_device_properties(dev).multi_processor_count
            issue_peak = sm_count * 4 * clk_max_mhz() * 1e6
            issue_achieved = ipu * units / (t_cls / 1e3)
            roof_mlp["issue"] = {"warp_inst_per_unit": ipu, "achieved": issue_achieved, "peak": issue_peak,
                                 "unit": "warp instructions/s", "frac": issue_achieved / issue_peak,
                                 "note": "warp instructions per (pixel,d) from the committed ncu capture "
                                         "(profiles/traffic.json); peak = SMs x 4 sub-partitions x max SM "
                                         "clock"}
        res["mlp"]["roofline"] = roof_mlp
    roof = res[head]["roofline"]

    classifier = {"rf": "random_forest (50 trees, depth<=20)",
                  "mlp": "f16 MLP 20-128-128-64-1 (%s) on tcgen05 (RF as judge)"
                         % (net.activation.upper() if net is not None else "")}[head]
    line = {
        "metric": METRIC, "value": units * ws / (h["ms"] / 1e3), "unit": "pixel·disparities/s",
        "n_gpus": ws, "steps": a.steps, "warmup": a.warmup, "ms_per_step": h["ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": ("%s/f32" % a.mlp_precision) if head == "mlp" else "f64/f32",
        "data": "synthetic (seeded 694x554 pair per rank; L2 flushed between steps)",
        "config": {"workload": "694x554 D=128 test path: 4 matchers, 20 features, %s, MC-CNN _mem post"
                               % classifier, "width": W0, "height": int(L.shape[0]), "ndisp": D0,
                   "units_per_pair": units, "classifier": head,
                   "forest_nodes": int(flat.n_nodes) if have_forest else None,
                   "l2": "flushed (256 MB write) between steps",
                   "parallelism": "replica per GPU, one pair per rank"},
        "stage_ms": h["stage_ms"],
        "bad2_nonocc": h["bad2_nonocc"],
        "gpu_launches": launches * a.steps,
        "e2e": None if h["e2e_ms"] is None else {
            "value": units * ws / (h["e2e_ms"] / 1e3), "unit": "pixel·disparities/s",
            "ms_per_step": h["e2e_ms"], "h2d_bytes_per_step": 2 * L.size, "d2h_bytes_per_step": 4 * L.size},
        "roofline": roof,
        "whole_path": {"bound": "hbm", "bytes_per_unit": BYTES_PER_UNIT_PATH,
                       "achieved": BYTES_PER_UNIT_PATH * units / (h["ms"] / 1e3) / 1e9, "peak": hbm,
                       "unit": "GB/s", "frac": BYTES_PER_UNIT_PATH * units / (h["ms"] / 1e3) / 1e9 / hbm,
                       "peak_kind": hbm_kind,
                       "note": "compulsory HBM bytes of an ideal fused path with the _mem post (4 B cost + "
                               "SGM 2 x 20 B + CBCA 4 x 8 B + WTA 4 B per (p,d)) over the device step time; "
                               "the learned classifier's own bound is the tensor roofline above"},
        "classifiers": {k: {"value": units * ws / (v["ms"] / 1e3), "ms_per_step": v["ms"],
                            "e2e_ms": v["e2e_ms"], "stage_ms": v["stage_ms"],
                            "bad2_nonocc": v["bad2_nonocc"], "roofline": v["roofline"]}
                        for k, v in res.items()},
        "matched_bad2": matched,
        "interp_variant": interp,
        "relu_variant": relu,
        "bf16_variant": bf16v,
        "clocks": clk.summary(),
    }
    if rank == 0 and ws == 1 and not a.no_cpu_baseline and not a.device_only and have_forest:
        line["cpu_baseline"] = cpu_baseline(flat, L, R, a)
    return line


def _cpu_stage_band(ref, skl, L, R, rows, cores):
    """The reference's CPU stages (test.py:122-138, 521-595, 597-626) on the
    first `rows` image rows: the matchers run on a band with a 10-row margin
    (every matcher is row-local within +-5 rows, so the kept rows equal the
    full-image ones), then the feature assembly and predict_proba on those
    rows.  Returns seconds."""
    from oracle import glue
    ref.set_threads(cores)
    band_l, band_r = L[:rows + 10], R[:rows + 10]
    t0 = time.perf_counter()
    glue.test_model(ref.mtc, ref.fte, skl.predict_proba, band_l, band_r, D0, rows=rows)
    return time.perf_counter() - t0


def cpu_baseline(flat, L, R, a):
    """The reference's own CPU stages, timed on this host (bounded sample)."""
    from oracle import ref, skforest
    cores = len(os.sched_getaffinity(0))
    if not ref.cpu_available():
        return {"value": None, "unit": "pixel·disparities/s", "cores": cores, "kind": "reference",
                "sample": "unavailable: oracle/_ref not built"}
    skl = skforest.to_sklearn(flat, n_jobs=cores)
    rows = a.cpu_rows
    _cpu_stage_band(ref, skl, L, R, 8, cores)  # warm-up (thread pools, page-in)
    t = _cpu_stage_band(ref, skl, L, R, rows, cores)
    units = rows * W0 * D0
    return {"value": units / t, "unit": "pixel·disparities/s", "cores": cores, "kind": "reference",
            "sample": "first %d rows of the 694x554 D=128 pair: reference matchers (on a %d-row band) + "
                      "feature assembly + sklearn predict_proba (n_jobs=%d); post excluded (the "
                      "reference runs it on the GPU); %.1f s" % (rows, rows + 10, cores, t)}


def run_reference(a, ws, rank, local):
    """--impl reference: the reference's implementation of the path on one
    whole 694x554 D=128 pair per step: its compiled matchers and feature
    assembly (oracle/_ref, all host cores) batched as test.py:597-626 does
    (floor(100000/694) = 144 rows per batch, np.append of every batch's
    probabilities), scikit-learn's predict_proba on the same forest, then
    Testing.eval_prob with the _mem chain on that classifier's own P(class 0)
    through the reference's post.cu on the GPU (as shipped: its host copies
    and host argmin included).  Each step is ~30 s of host work, so the timed
    steps stop once REF_BUDGET_S has passed (at least one; the line states
    how many ran); each of the max(3, --warmup) warm-up steps is one
    16-row band, which pages in the libraries and starts the thread
    pools."""
    if rank != 0:
        return None
    import torch
    from cbmv_b200 import synth
    from cbmv_b200.forest import FlatForest
    from oracle import cpu, glue, ref, skforest

    cores = len(os.sched_getaffinity(0))
    if not ref.cpu_available():
        return {"impl": "reference", "unavailable": "oracle/_ref (the reference compiled from its sources) "
                                                  "is not built"}
    if not os.path.exists(a.forest):
        return {"impl": "reference", "unavailable": "forest fixture missing (tests/golden/make_forest.py)"}
    flat = FlatForest.load(a.forest)
    skl = skforest.to_sklearn(flat, n_jobs=cores)
    ref.set_threads(cores)
    L, R, gt, nonocc = synth.pair_694x554(seed=0)
    on_gpu = ref.post_available() and torch.cuda.is_available()
    post_kind = "reference post.cu on the GPU (as shipped)" if on_gpu else "oracle CPU restatement of post.cu"
    post_mod = ref.post if on_gpu else cpu.post
    n_warm = max(3, a.warmup)
    for _ in range(n_warm):  # warm-up steps: one 16-row band each
        glue.test_model(ref.mtc, ref.fte, skl.predict_proba, L[:26], R[:26], D0, rows=16)
    times, disp = [], None
    t_start = time.perf_counter()
    for k in range(max(1, a.steps)):
        t0 = time.perf_counter()
        proba = glue.test_model(ref.mtc, ref.fte, skl.predict_proba, L, R, D0)
        t1 = time.perf_counter()
        disp = glue.eval_prob(post_mod, ref.fte, proba, L, R, D0)
        if on_gpu:
            ref.post.sync()
        t2 = time.perf_counter()
        times.append((t1 - t0, t2 - t1))
        if time.perf_counter() - t_start > REF_BUDGET_S:
            break
    from cbmv_b200 import evaluate
    t_cpu = float(np.mean([t for t, _ in times]))
    t_post = float(np.mean([t for _, t in times]))
    t_pair = t_cpu + t_post
    value = UNITS / t_pair
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "pixel·disparities/s",
        "n_gpus": ws, "steps": len(times), "steps_requested": a.steps, "warmup": n_warm,
        "warmup_note": "each warm-up step is a 16-row band of the pair (pages in the libraries, "
                       "starts the thread pools); a whole pair is ~30 s of host work",
        "ms_per_step": t_pair * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded 694x554 pair, seed 0)",
        "config": {"workload": "694x554 D=128 test path: 4 matchers, 20 features, RF 50 trees "
                               "depth<=20, MC-CNN _mem post", "width": W0, "height": H0, "ndisp": D0},
        "step_cap": "timed whole-pair steps stop after %d s (at least one): %d of %d ran"
                    % (REF_BUDGET_S, len(times), a.steps),
        "bad2_nonocc": evaluate.bad_x(disp, gt, nonocc),
        "stage_s": {"matchers_features_rf": t_cpu, "post": t_post},
        "cpu_baseline": {"value": value, "unit": "pixel·disparities/s", "cores": cores,
                         "kind": "reference",
                         "sample": "per step one whole 694x554 D=128 pair: reference matchers + feature "
                                   "assembly in 4 row batches of 144 (test.py:597-626) + sklearn "
                                   "predict_proba (n_jobs=%d) %.2f s, then %s on that P(class 0) %.2f s"
                                   % (cores, t_cpu, post_kind, t_post)},
        "e2e": {"value": value, "unit": "pixel·disparities/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def _make_pair_spec(spec):
    from cbmv_b200 import synth
    return synth.make_pair(**spec)


def run_batch(a, ws, rank, local):
    """--batch: 64 seeded pairs of uneven size (W~U[320,1500], H~U[240,1000],
    D in {64,128,192,256}, seeds 4000..4063) through the learned path as one
    CUDA graph launch per step, launch shape from the autotuner; per-pair
    latency p50/p99 beside the aggregate throughput, and the same pairs run
    one after another (one pipeline call each) for comparison.  With N
    ranks the 64 pairs are split longest-first over the GPUs
    (cbmv_b200.shard.lpt_assign; strong scaling: the total work is fixed),
    each GPU runs its share as its own graph, and rank 0 gathers every
    pair's disparity map, latency and bad-2.0 (the only data-path
    collectives)."""
    import multiprocessing as mp
    import torch
    from cbmv_b200 import _lib, evaluate, synth
    from cbmv_b200.batch import StereoBatch, tune_batch
    from cbmv_b200.mlp import GpuMlp
    from cbmv_b200.pipeline import StereoPipeline
    from cbmv_b200 import shard
    all_specs = synth.batch_specs(a.batch_pairs, 4000)
    all_shapes = [(sp["height"], sp["width"], sp["ndisp"]) for sp in all_specs]
    assign = shard.lpt_assign(shard.pair_work(all_shapes), ws)  # this rank runs assign[rank]
    specs = [all_specs[i] for i in assign[rank]]
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        pairs = pool.map(_make_pair_spec, specs)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    shapes = [(sp["height"], sp["width"], sp["ndisp"]) for sp in specs]
    units = int(sum(h * w * d for h, w, d in all_shapes))
    lefts = [torch.from_numpy(p[0]).to(dev) for p in pairs]
    rights = [torch.from_numpy(p[1]).to(dev) for p in pairs]
    net = GpuMlp.load(a.mlp, a.mlp_precision)
    t_tune = time.perf_counter()
    tune = tune_batch(shapes, net, lefts, rights, log=lambda m: print(m, file=sys.stderr))
    t_tune = time.perf_counter() - t_tune
    b = StereoBatch(shapes, streams=tune["streams"])
    prm = _lib.default_params(mlp_ctas=tune["mlp_ctas"], cbca_rows=tune.get("cbca_rows", 32),
                              sgm_prefetch=tune.get("sgm_prefetch", 0))
    st = torch.cuda.current_stream()
    for _ in range(a.warmup):
        b.run_mlp(net, lefts, rights, prm)
    barrier(ws)
    spans, pair_ms, done_ms = [], [], []
    with Clocks(local) as clk:
        for k in range(a.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            b.run_mlp(net, lefts, rights, prm)
            e1.record(st)
            e1.synchronize()
            spans.append(e0.elapsed_time(e1))
            t = b.timings()
            pair_ms.append(t["pair_ms"])
            done_ms.append(t["done_ms"])
        barrier(ws)
    ms = shard.max_over_ranks(float(np.mean(spans)), device=dev)
    disp = [t.cpu().numpy() for t in b.disp]
    bad_local = [evaluate.bad_x(d, p[2], p[3]) for d, p in zip(disp, pairs)]
    pair_ms, done_ms = np.stack(pair_ms), np.stack(done_ms)  # [steps, this rank's pairs]
    # the same pairs one pipeline call each, back to back on one stream
    pipe = StereoPipeline()
    outs = [torch.empty(l.shape, dtype=torch.float32, device=dev) for l in lefts]
    for i in range(len(shapes)):
        pipe.run_mlp(net, lefts[i], rights[i], shapes[i][2], disp_out=outs[i])
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for i in range(len(shapes)):
        pipe.run_mlp(net, lefts[i], rights[i], shapes[i][2], disp_out=outs[i])
    e1.record(st)
    e1.synchronize()
    seq_ms = shard.max_over_ranks(e0.elapsed_time(e1), device=dev)
    same = all(np.array_equal(o.cpu().numpy(), d) for o, d in zip(outs, disp))
    same = shard.max_over_ranks(0.0 if same else 1.0, device=dev) == 0.0
    # every pair's map, latency and error on rank 0 (the only collectives of the data path)
    maps = shard.gather_maps(list(b.disp), assign, all_shapes, device=dev)
    n = len(all_shapes)
    lat = {k: shard.gather_values(v.mean(axis=0), assign, n, device=dev)
           for k, v in (("pair", pair_ms), ("done", done_ms))}
    bad = shard.gather_values(bad_local, assign, n, device=dev)
    if rank != 0:
        return None
    assert all(m is not None and tuple(m.shape) == (h, w) for m, (h, w, _) in zip(maps, all_shapes))
    return {
        "metric": "pixel·disparities/s, %d uneven pairs in one CUDA graph launch per GPU (learned classifier)" % n,
        "value": units / (ms / 1e3), "unit": "pixel·disparities/s", "n_gpus": ws, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong" if ws > 1 else "weak", "vs_baseline": None,
        "dtype": "%s/f32" % a.mlp_precision, "data": "synthetic (seeded uneven pairs, seeds 4000+)",
        "config": {"workload": "%d pairs W~U[320,1500] H~U[240,1000] D in {64,128,192,256}" % n,
                   "units": units,
                   "autotune": {k: tune.get(k) for k in ("streams", "mlp_ctas", "cbca_rows", "sgm_prefetch", "ms",
                                                         "tried")},
                   "autotune_seconds": t_tune,
                   "parallelism": "pairs split longest-first over %d GPU(s), concurrent contexts in one graph "
                                  "per GPU, disparity maps gathered on rank 0" % ws,
                   "shards": shard.assignment_summary(assign, shard.pair_work(all_shapes))},
        "latency_ms": {"pair_p50": float(np.percentile(lat["pair"], 50)), "pair_p99": float(np.percentile(lat["pair"], 99)),
                       "done_p50": float(np.percentile(lat["done"], 50)), "done_p99": float(np.percentile(lat["done"], 99)),
                       "note": "pair: a pair's first to last kernel; done: its GPU's graph start to the pair's end "
                               "(means over the timed steps)"},
        "sequential_ms": seq_ms, "sequential_value": units / (seq_ms / 1e3),
        "identical_to_sequential": bool(same), "bad2_nonocc_mean": float(np.mean(bad)),
        "gpu_launches": a.steps * len(all_shapes) * launches_per_pair(_lib.default_params(), "mlp"),
        "gpu_launches_note": "this package's kernels inside the graphs over the timed steps: %d per pair "
                             "x %d pairs per step, one graph launch per step per GPU"
                             % (launches_per_pair(_lib.default_params(), "mlp"), len(all_shapes)),
        "clocks": clk.summary(),
    }


@contextlib.contextmanager
def native_stdout_to_stderr():
    """Text that compiled code prints on file descriptor 1 (the reference's
    post module announces "CUDA initialized.") goes to stderr instead, so
    that stdout carries only the JSON line."""
    sys.stdout.flush()
    saved = os.dup(1)
    os.dup2(2, 1)
    try:
        yield
    finally:
        try:
            ctypes.CDLL(None).fflush(None)  # C stdio buffers, before fd 1 is restored
        except OSError:
            pass
        sys.stdout.flush()
        os.dup2(saved, 1)
        os.close(saved)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["cbmv", "reference"], default="cbmv")
    ap.add_argument("--forest", default=FOREST)
    ap.add_argument("--mlp", default=MLP, help="trained MLP parameters (cbmv_b200.train_mlp)")
    ap.add_argument("--mlp-relu", default=MLP_RELU, help="the ReLU network, timed as a variant")
    ap.add_argument("--mlp-precision", choices=["f16", "bf16"], default="f16",
                    help="operand type of the network's fused inference (bf16 is also timed as a "
                         "variant of the f16 default)")
    ap.add_argument("--classifier", choices=["both", "rf", "mlp"], default="both",
                    help="classifier paths to time (both: the MLP is the headline when it matches "
                         "the RF's held-out bad-2.0)")
    ap.add_argument("--batch", action="store_true",
                    help="the batched workload: uneven pairs in one graph launch (autotuned)")
    ap.add_argument("--batch-pairs", type=int, default=64)
    ap.add_argument("--no-eval", action="store_true",
                    help="skip the held-out bad-2.0 comparison (the RF stays the headline)")
    ap.add_argument("--cpu-rows", type=int, default=288,
                    help="rows of the cpu_baseline sample (288 = two of the reference's 144-row batches)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--device-only", action="store_true",
                    help="time the device path(s) only: no e2e, variants, held-out evaluation or CPU "
                         "baseline (short runs for profiler captures)")
    ap.add_argument("--height", type=int, default=H0,
                    help="rows of the pair (smaller cases for profiler captures; default 554)")
    a = ap.parse_args()
    if a.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # started directly with --gpus N: one process per GPU under torchrun
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(a.gpus),
               "--master-addr", "127.0.0.1", "--master-port", os.environ.get("MASTER_PORT", "29517"),
               os.path.abspath(__file__)] + sys.argv[1:]
        os.execv(sys.executable, cmd)
    if a.gpus != env_ranks()[0]:
        raise SystemExit("--gpus %d but WORLD_SIZE=%d: launch with torchrun --nproc-per-node %d"
                         % (a.gpus, env_ranks()[0], a.gpus))
    if a.impl == "reference":
        # rank 0 alone runs the reference and no rank exchanges anything, so
        # no process group is opened (the other ranks exit at once)
        ws, rank, local = env_ranks()
        with native_stdout_to_stderr():
            line = run_reference(a, ws, rank, local)
        if rank == 0 and line is not None:
            print(json.dumps(line))
        return
    ws, rank, local = dist_init()
    if a.batch:
        line = run_batch(a, ws, rank, local)
    else:
        line = run_cbmv(a, ws, rank, local)
    if rank == 0 and line is not None:
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
