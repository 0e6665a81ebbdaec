"""Trains the learned classifier on samples the GPU pipeline emits.

    python -m cbmv_b200.train_mlp --out mlp.npz [--pairs 200] [--per-pair 50000] [--activation gelu]

Training data (the GPU counterpart of the reference's train.py:100-273, with
the MLP's labelling): seeded synthetic 694x554, D=128 pairs (seeds 2000..),
`per-pair` non-occluded ground-truth pixels each, one positive disparity
with |d - gt| <= 1 and one negative with |d - gt| > 1 per pixel (1:1
balance; half of the negatives within 8 px of the ground truth, the rest
uniform), their 20 CBMV features computed on the device
(cbmv_ctx_features_at).  The network (cbmv_b200.mlp) is trained with the
project's tcgen05 forward/backward kernels and Adam.
"""
import argparse
import math
import time

import numpy as np

from . import synth
from .mlp import MlpParams, MlpTrainer, input_stats
from .pipeline import StereoPipeline

D = 128
TRAIN_SEED0 = 2000


def pick_samples(gt, nonocc, per_pair, seed, ndisp=D, hard_frac=0.0, hard_range=8):
    """(flat sample indices, labels) for one pair: positives |d-gt|<=1,
    negatives |d-gt|>1, one of each per chosen pixel.  A fraction
    `hard_frac` of the negatives is drawn within `hard_range` of the ground
    truth (the near-miss disparities the cost volume must rank below it),
    the rest uniformly over [0, D)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    H, W = gt.shape
    valid = nonocc & (gt >= 0) & (gt <= ndisp - 1)
    pix = np.flatnonzero(valid)
    if pix.size > per_pair:
        pix = np.sort(rng.choice(pix, per_pair, replace=False))
    g = gt.reshape(-1)[pix].astype(np.float64)
    # positive: a uniform pick among round(gt)-1 .. round(gt)+1 within 1 px of gt
    cand = np.rint(g)[:, None] + np.array([-1, 0, 1])[None, :]
    ok = (np.abs(cand - g[:, None]) <= 1) & (cand >= 0) & (cand < ndisp)
    u = rng.random(cand.shape) * ok
    dpos = cand[np.arange(len(g)), np.argmax(u, axis=1)].astype(np.int64)
    # negative: uniform over [0, D) with |d - gt| > 1 (redraw the few rejects)
    hard = rng.random(len(g)) < hard_frac

    def draw(m):
        off = rng.integers(2, hard_range + 1, m) * np.where(rng.random(m) < 0.5, -1, 1)
        return off

    dneg = rng.integers(0, ndisp, len(g))
    dneg[hard] = (np.rint(g[hard]) + draw(int(hard.sum()))).astype(np.int64)
    for _ in range(64):
        bad = (np.abs(dneg - g) <= 1) | (dneg < 0) | (dneg >= ndisp)
        if not bad.any():
            break
        dneg[bad] = rng.integers(0, ndisp, int(bad.sum()))
    keep = np.abs(dneg - g) > 1
    idx = np.concatenate([pix * ndisp + dpos, (pix * ndisp + dneg)[keep]])
    lab = np.concatenate([np.ones(len(pix), np.float32), np.zeros(int(keep.sum()), np.float32)])
    return idx, lab


def emit(pairs, per_pair, seed0=TRAIN_SEED0, log=print, hard_frac=0.5):
    import torch
    pipe = StereoPipeline()
    Xs, ys = [], []
    t0 = time.time()
    for k in range(pairs):
        L, R, gt, nonocc = synth.pair_694x554(seed0 + k)
        idx, lab = pick_samples(gt, nonocc, per_pair, seed0 + k + 7777, hard_frac=hard_frac)
        Xs.append(pipe.features_at(L, R, D, torch.from_numpy(idx).cuda()))
        ys.append(torch.from_numpy(lab).cuda())
        if (k + 1) % 25 == 0:
            log("emitted %d pairs, %d samples, %.1fs" % (k + 1, sum(x.shape[0] for x in Xs), time.time() - t0))
    return torch.cat(Xs), torch.cat(ys)


def train(X, y, epochs=4, batch=8192, lr=2e-3, wd=1e-4, seed=0, log=print, activation="gelu"):
    import torch
    n = X.shape[0]
    sub = X[torch.randperm(n, generator=torch.Generator().manual_seed(seed))[:1_000_000].cuda()]
    cap, mu, sd = input_stats(sub.cpu().numpy())
    tr = MlpTrainer(MlpParams.init(seed, cap, mu, sd, activation), batch=batch)
    steps_per_epoch = n // batch
    total = epochs * steps_per_epoch
    g = torch.Generator(device="cuda").manual_seed(seed)
    step = 0
    t0 = time.time()
    for ep in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=g)
        run = 0.0
        for s in range(steps_per_epoch):
            b = perm[s * batch:(s + 1) * batch]
            cur = lr * 0.5 * (1 + math.cos(math.pi * step / total))  # cosine schedule
            loss = tr.step(X[b].contiguous(), y[b].contiguous(), cur, wd)
            step += 1
            if s % 200 == 0:
                run = loss.item()
                log("epoch %d step %d/%d loss %.4f lr %.2e (%.1fs)" % (ep, s, steps_per_epoch, run, cur,
                                                                      time.time() - t0))
    if tr.status() != 0:
        raise RuntimeError("a tensor-core wait timed out during training")
    return tr.params()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--pairs", type=int, default=200)
    ap.add_argument("--per-pair", type=int, default=50000)
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--hard-frac", type=float, default=0.5)
    ap.add_argument("--activation", choices=["gelu", "relu"], default="gelu")
    a = ap.parse_args()
    X, y = emit(a.pairs, a.per_pair, hard_frac=a.hard_frac)
    print("samples", tuple(X.shape), "positives", float(y.mean()), flush=True)
    net = train(X, y, a.epochs, a.batch, a.lr, activation=a.activation)
    net.save(a.out)
    print("saved", a.out, flush=True)


if __name__ == "__main__":
    main()
