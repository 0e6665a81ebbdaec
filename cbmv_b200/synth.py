"""Seeded synthetic rectified stereo pairs with piecewise-planar ground truth.

There is no public benchmark data for this path in the container (the
reference's Middlebury lists, mb/*.txt, name scenes that are not shipped), so
every workload is generated here from a seed with numpy's PCG64:

  left image   4-octave value noise (lattice period W/8, halving per octave,
               amplitude halving per octave, smoothstep-weighted interpolation
               of the lattice values), rescaled to 0..255, then random flat
               axis-aligned grey patches (sides uniform in 8..64 px) until they
               cover 10% of the area; rounded to uint8
  ground truth Voronoi partition into `planes` regions, each a slanted plane
               d = d0 + b*(x-cx) + c*(y-cy), d0 uniform in [dmin, dmax],
               b, c uniform in [-0.2, 0.2]; clamped to [dmin, dmax].  Left-view
               disparity: L(x) matches R(x - d).
  right image  forward warp of the left image to x - d with a z-buffer (the
               larger disparity wins), sampled back by linear interpolation;
               pixels nothing maps to get fresh noise; then N(0, 2^2) noise,
               clipped to uint8
  nonocc mask  left pixels whose warp target is the visible (winning) one
"""
import numpy as np


def _value_noise(rng, h, w, octaves=4):
    out = np.zeros((h, w), np.float64)
    period = max(w / 8.0, 2.0)
    amp = 1.0
    ys = np.arange(h, dtype=np.float64)
    xs = np.arange(w, dtype=np.float64)
    for _ in range(octaves):
        gh = int(np.ceil(h / period)) + 2
        gw = int(np.ceil(w / period)) + 2
        lat = rng.random((gh, gw))
        fy = ys / period
        fx = xs / period
        iy = np.floor(fy).astype(np.int64)
        ix = np.floor(fx).astype(np.int64)
        ty = fy - iy
        tx = fx - ix
        sy = ty * ty * (3.0 - 2.0 * ty)
        sx = tx * tx * (3.0 - 2.0 * tx)
        v00 = lat[iy[:, None], ix[None, :]]
        v01 = lat[iy[:, None], ix[None, :] + 1]
        v10 = lat[iy[:, None] + 1, ix[None, :]]
        v11 = lat[iy[:, None] + 1, ix[None, :] + 1]
        top = v00 + (v01 - v00) * sx[None, :]
        bot = v10 + (v11 - v10) * sx[None, :]
        out += amp * (top + (bot - top) * sy[:, None])
        period = max(period / 2.0, 1.0)
        amp *= 0.5
    out -= out.min()
    mx = out.max()
    if mx > 0:
        out *= 255.0 / mx
    return out


def _flat_patches(rng, img, frac=0.10):
    h, w = img.shape
    mask = np.zeros((h, w), bool)
    target = frac * h * w
    while mask.sum() < target:
        ph = int(rng.integers(8, 65))
        pw = int(rng.integers(8, 65))
        y0 = int(rng.integers(0, max(h - ph, 0) + 1))
        x0 = int(rng.integers(0, max(w - pw, 0) + 1))
        img[y0:y0 + ph, x0:x0 + pw] = rng.uniform(0.0, 255.0)
        mask[y0:y0 + ph, x0:x0 + pw] = True
    return img


def _planes_gt(rng, h, w, planes, dmin, dmax):
    cy = rng.uniform(0, h, planes)
    cx = rng.uniform(0, w, planes)
    d0 = rng.uniform(dmin, dmax, planes)
    b = rng.uniform(-0.2, 0.2, planes)
    c = rng.uniform(-0.2, 0.2, planes)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    best = np.full((h, w), np.inf)
    label = np.zeros((h, w), np.int64)
    for k in range(planes):
        dist = (yy - cy[k]) ** 2 + (xx - cx[k]) ** 2
        sel = dist < best
        best[sel] = dist[sel]
        label[sel] = k
    gt = d0[label] + b[label] * (xx - cx[label]) + c[label] * (yy - cy[label])
    return np.clip(gt, dmin, dmax)


def make_pair(seed, width, height, ndisp, planes, dmin, dmax):
    """Return (left u8 [H,W], right u8 [H,W], gt f32 [H,W], nonocc bool [H,W])."""
    rng = np.random.Generator(np.random.PCG64(seed))
    h, w = int(height), int(width)
    dmax = min(float(dmax), float(ndisp - 3))
    left = _flat_patches(rng, _value_noise(rng, h, w))
    left_u8 = np.clip(np.rint(left), 0, 255).astype(np.uint8)
    gt = _planes_gt(rng, h, w, planes, dmin, dmax)

    # forward warp with z-buffer: each left pixel lands on round(x - d)
    yy, xx = np.mgrid[0:h, 0:w]
    tx = np.rint(xx - gt).astype(np.int64)
    inside = (tx >= 0) & (tx < w)
    zbuf = np.full((h, w), -np.inf)
    np.maximum.at(zbuf, (yy[inside], tx[inside]), gt[inside])
    filled = np.isfinite(zbuf)
    # Slanted planes leave 1-2 px gaps between forward-warped samples; a gap
    # whose two nearest filled neighbours (within 2 px) lie on the same surface
    # (disparities within 1 px) takes their interpolated disparity.  Wider
    # gaps are disocclusions and get fresh noise below.
    cols = np.broadcast_to(np.arange(w)[None, :], (h, w))
    li = np.maximum.accumulate(np.where(filled, cols, -1), axis=1)
    ri = np.flip(np.minimum.accumulate(np.flip(np.where(filled, cols, w), axis=1), axis=1), axis=1)
    ok = (~filled) & (li >= 0) & (ri < w) & (ri - li <= 3)
    zl = np.where(ok, zbuf[yy, np.clip(li, 0, w - 1)], 0.0)
    zr = np.where(ok, zbuf[yy, np.clip(ri, 0, w - 1)], 0.0)
    ok &= np.abs(zl - zr) < 1.0
    t = np.where(ok, (cols - li) / np.maximum(ri - li, 1), 0.0)
    zbuf = np.where(ok, zl + (zr - zl) * t, zbuf)
    filled = filled | ok
    src = np.where(filled, np.arange(w)[None, :] + np.where(filled, zbuf, 0.0), 0.0)
    x0 = np.clip(np.floor(src).astype(np.int64), 0, w - 1)
    x1 = np.clip(x0 + 1, 0, w - 1)
    fr = np.clip(src - np.floor(src), 0.0, 1.0)
    lf = left_u8.astype(np.float64)
    rows = np.arange(h)[:, None]
    right = lf[rows, x0] * (1.0 - fr) + lf[rows, x1] * fr
    holes = ~filled
    right[holes] = rng.uniform(0.0, 255.0, int(holes.sum()))
    right += rng.normal(0.0, 2.0, (h, w))
    right_u8 = np.clip(np.rint(right), 0, 255).astype(np.uint8)

    nonocc = np.zeros((h, w), bool)
    txc = np.clip(tx, 0, w - 1)
    nonocc[inside] = gt[inside] >= zbuf[yy[inside], txc[inside]] - 0.5
    return left_u8, right_u8, gt.astype(np.float32), nonocc


# Workload shapes (width, height, ndisp, planes, dmin, dmax, seed).
PAIR_694x554 = dict(width=694, height=554, ndisp=128, planes=12, dmin=4, dmax=120, seed=0)
PAIR_1482x994 = dict(width=1482, height=994, ndisp=256, planes=20, dmin=8, dmax=240, seed=1)
PAIR_2880x1988 = dict(width=2880, height=1988, ndisp=400, planes=30, dmin=10, dmax=390, seed=5)
RF_TRAIN_SEEDS = list(range(1000, 1030))


def pair_694x554(seed=0):
    p = dict(PAIR_694x554)
    p["seed"] = seed
    return make_pair(**p)


def pair_1482x994(seed=1):
    p = dict(PAIR_1482x994)
    p["seed"] = seed
    return make_pair(**p)


def pair_2880x1988(seed=5):
    p = dict(PAIR_2880x1988)
    p["seed"] = seed
    return make_pair(**p)


def batch_specs(n=64, seed0=4000):
    """Uneven batch: W~U[320,1500], H~U[240,1000], D in {64,128,192,256}, planes~U[6,24]."""
    out = []
    for k in range(n):
        rng = np.random.Generator(np.random.PCG64(seed0 + k))
        w = int(rng.integers(320, 1501))
        h = int(rng.integers(240, 1001))
        d = int(rng.choice([64, 128, 192, 256]))
        planes = int(rng.integers(6, 25))
        dmin = 4
        dmax = max(dmin + 1, d - 8)
        out.append(dict(width=w, height=h, ndisp=d, planes=planes, dmin=dmin, dmax=dmax, seed=seed0 + k))
    return out
