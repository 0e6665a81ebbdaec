"""The reference's driver (main.py, with the parts of test.py and train.py it
calls) in Python 3 over this package.

    # test: one scene -> disparity PFM (main.py:50-70)
    python -m cbmv_b200.driver --data_path DATA/ --test_set Adirondack --model forest.npz \\
        [--disp_save_path ./results/disp.pfm] [--prob_save_path ./results/] \\
        [--saveCostVolume | --loadCostVolume]
    # train: scenes listed comma-separated in a file (train.py:32-47, 277-293)
    python -m cbmv_b200.driver --train --data_path DATA/ --train_set mb/train.txt --model forest.npz

A scene directory holds im0.png / im1.png (read as 8-bit grey, like
scipy.misc.imread(mode='L'), test.py:509-510), calib.txt (width, height,
ndisp, test.py:91-104) and, for training, disp0GT.pfm (train.py:103).  The
model is a forest (.npz of cbmv_b200.forest.FlatForest, or a scikit-learn
RandomForestClassifier pickle) or the learned classifier (.npz of
cbmv_b200.mlp.MlpParams): the whole test path runs fused on the GPU.
Rectification correction (`__fix_rectification` with librectification)
needs OpenCV and is not applied: the images are used as given.
"""
import argparse
import os
import pickle
import time

import numpy as np

from . import costvol, pfm


def read_calib(path):
    """(width, height, ndisp) from a Middlebury calib.txt (test.py:91-104)."""
    w = h = d = 0
    with open(path) as f:
        for line in f:
            k, _, v = line.strip("\n").partition("=")
            if k == "width":
                w = int(v)
            elif k == "height":
                h = int(v)
            elif k == "ndisp":
                d = int(v)
    return w, h, d


def read_grey(path):
    from PIL import Image
    return np.array(Image.open(path).convert("L"), dtype=np.uint8)  # a writable copy


def load_model(path):
    """('rf', GpuForest) or ('mlp', GpuMlp) from a model file."""
    if path.endswith(".npz"):
        z = np.load(path)
        if "params" in z.files:
            from .mlp import GpuMlp
            return "mlp", GpuMlp.load(path)
        from .forest_gpu import GpuForest
        return "rf", GpuForest.load(path)
    with open(path, "rb") as f:  # a scikit-learn forest, as train.py:291 writes it
        rf = pickle.load(f)
    from .forest_gpu import GpuForest
    return "rf", GpuForest.from_sklearn(rf)


def test_scene(data_path, test_set, model, disp_save_path="./results/disp.pfm", prob_save_path="./results/",
               save_cost=False, load_cost=False, iml="", imr="", calib="", w=0, h=0, d=0, log=print):
    """main.py:50-70 for one scene; returns the disparity map [H,W] float32."""
    import torch
    from .pipeline import StereoPipeline
    scene = os.path.join(data_path, test_set)
    if not (w and h and d):
        w, h, d = read_calib(os.path.join(data_path, calib) if calib else os.path.join(scene, "calib.txt"))
    L = read_grey(os.path.join(data_path, iml) if iml else os.path.join(scene, "im0.png"))
    R = read_grey(os.path.join(data_path, imr) if imr else os.path.join(scene, "im1.png"))
    if L.shape != (h, w) or R.shape != (h, w):
        raise ValueError("images are %s / %s, calibration says %dx%d" % (L.shape, R.shape, w, h))
    kind, clf = load_model(model)
    pipe = StereoPipeline(clf if kind == "rf" else None)
    cost_file = costvol.reference_path(prob_save_path, test_set)
    t0 = time.time()
    if load_cost and os.path.exists(cost_file):
        log("Loading cost volume from file : {}".format(cost_file))
        disp = pipe.run_post(L, R, costvol.load(cost_file, shape=(h, w, d)))
    else:
        prob = torch.empty((h, w, d), dtype=torch.float32, device="cuda") if save_cost else None
        run = pipe.run_rf if kind == "rf" else (lambda *a, **k: pipe.run_mlp(clf, *a, **k))
        disp = run(L, R, d, prob_out=prob)
        if save_cost:
            os.makedirs(os.path.dirname(cost_file) or ".", exist_ok=True)
            costvol.save(cost_file, prob, "reference")
            log("Saved cost volume {}".format(cost_file))
    log("%s %dx%d D=%d: %.3f s (%s)" % (test_set, w, h, d, time.time() - t0, kind))
    os.makedirs(os.path.dirname(disp_save_path) or ".", exist_ok=True)
    pfm.save(disp_save_path, np.asarray(disp, np.float32))  # test.py:503
    log("Saved {}".format(disp_save_path))
    return disp


def train(data_path, train_set, model, train_add="", n_jobs=None, max_depth=None, log=print):
    """train.py:277-293 over scene directories, samples emitted on the GPU."""
    from sklearn.ensemble import RandomForestClassifier
    from .forest import FlatForest
    from .pipeline import StereoPipeline
    from .train_rf import emit_samples
    names = open(train_set).read().rstrip().split(",")
    if train_add:
        names += open(train_add).read().rstrip().split(",")
    names = [n.strip() for n in names if n.strip()]
    if not names:
        raise ValueError("train set is empty")
    pipe = StereoPipeline()
    Xs, ys = [], []
    for k, name in enumerate(names):
        scene = os.path.join(data_path, name)
        w, h, d = read_calib(os.path.join(scene, "calib.txt"))
        L, R = read_grey(os.path.join(scene, "im0.png")), read_grey(os.path.join(scene, "im1.png"))
        gt = pfm.load(os.path.join(scene, "disp0GT.pfm"))[0]
        X, y = emit_samples(pipe, L, R, gt, d, seed=k)
        Xs.append(X)
        ys.append(y)
        log("sampling %s: %d samples" % (name, len(y)))
    X, y = np.concatenate(Xs), np.concatenate(ys)
    rf = RandomForestClassifier(n_estimators=50, min_samples_leaf=700, max_depth=max_depth,
                                n_jobs=n_jobs or os.cpu_count(), random_state=0)
    rf.fit(X, y)
    ff = FlatForest.from_sklearn(rf)
    ff.save(model)
    log("model is saved at {}".format(model))
    return ff


def main(argv=None):
    ap = argparse.ArgumentParser(description="CBMV on B200")
    ap.add_argument("--data_path", default="")
    ap.add_argument("--train_set", default="")
    ap.add_argument("--train_add", default="")
    ap.add_argument("--test_set", default="")
    ap.add_argument("--train", action="store_true")
    ap.add_argument("--model", default="")
    ap.add_argument("--prob_save_path", default="./results")
    ap.add_argument("--disp_save_path", default="./results/disp.pfm")
    ap.add_argument("--l", dest="lim", default="")
    ap.add_argument("--r", dest="rim", default="")
    ap.add_argument("--calib", default="")
    ap.add_argument("--w", type=int, default=0)
    ap.add_argument("--h", type=int, default=0)
    ap.add_argument("--d", type=int, default=0)
    ap.add_argument("--n_jobs", type=int, default=None)
    ap.add_argument("--saveCostVolume", action="store_true")
    ap.add_argument("--loadCostVolume", action="store_true")
    a = ap.parse_args(argv)
    if a.train:
        train(a.data_path, a.train_set, a.model, a.train_add, a.n_jobs)
    else:
        test_scene(a.data_path, a.test_set, a.model, a.disp_save_path, a.prob_save_path, a.saveCostVolume,
                   a.loadCostVolume, a.lim, a.rim, a.calib, a.w, a.h, a.d)


if __name__ == "__main__":
    main()
