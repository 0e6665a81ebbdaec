"""Model of the fused pipeline's separable cross-based cost aggregation
(test infrastructure only).

The reference (cpp/post/post.cu:399-450) sums each support region with one
running float32 sum, rows ascending, columns ascending.  The device's
default form splits it: R(yy, x, d) = float32 sum of the support row of row
yy (columns ascending, from 0), C = its length; out(y, x, d) = float32 sum
of R over the support rows (ascending, from 0) / sum of C.  This restates
that order exactly in numpy float32, so the CUDA kernel can be compared with
it bit for bit, while tests/test_oracle.py bounds its distance from the
reference-order sum.  The pipeline runs this form from precomputed support
words (one 32-bit word per (y, x, d), shared by the passes of one post);
cbca_support_words / cbca_from_words restate that encoding.
"""
import numpy as np


def cbca_separable(lc, rc, vol, direction, halo):
    """lc, rc: float32 [4, H, W] cross arms (cpp/post/post.cu:376-396);
    vol: float32 [H, W, D].  Returns float32 [H, W, D]."""
    lc = np.asarray(lc, np.float32)
    rc = np.asarray(rc, np.float32)
    vol = np.asarray(vol, np.float32)
    H, W, D = vol.shape
    x = np.arange(W)[None, :, None]
    d = np.arange(D)[None, None, :]
    dd = d * direction
    xm = x + dd                                  # [1, W, D]
    valid = (xm >= 0) & (xm < W)
    xmc = np.clip(xm, 0, W - 1)[0]               # [W, D]
    xi = np.broadcast_to(np.arange(W)[:, None], (W, D))

    def arm(a, side):
        """arm a of the left view at (yy, x) or of the right view at (yy, xm): [H, W, D] int"""
        if side == 0:
            return np.broadcast_to(lc[a][:, :, None], (H, W, D)).astype(np.int64)
        return rc[a][:, xmc].astype(np.int64)

    xxs = np.maximum(arm(0, 0), arm(0, 1) - dd)
    xxt = np.minimum(arm(1, 0), arm(1, 1) - dd)
    R = np.zeros((H, W, D), np.float32)
    dix = np.broadcast_to(np.arange(D)[None, :], (W, D))
    for k in range(-halo, halo + 1):
        xx = xi + k
        m = (xx[None] > xxs) & (xx[None] < xxt) & valid
        vals = vol[:, np.clip(xx, 0, W - 1), dix]     # [H, W, D]
        R = R + np.where(m, vals, np.float32(0))
    C = np.where(valid, np.maximum(xxt - xxs - 1, 0), 0)
    yys = np.maximum(arm(2, 0), arm(2, 1))
    yyt = np.minimum(arm(3, 0), arm(3, 1))
    S = np.zeros((H, W, D), np.float32)
    N = np.zeros((H, W, D), np.int64)
    y = np.arange(H)[:, None, None]
    for k in range(-halo, halo + 1):
        yy = y + k
        m = (yy > yys) & (yy < yyt)
        src = np.clip(yy[:, 0, 0], 0, H - 1)
        S = S + np.where(m, R[src], np.float32(0))
        N = N + np.where(m, C[src], 0)
    out = np.where(valid, S / np.maximum(N, 1).astype(np.float32), vol)
    return out.astype(np.float32)


MASK_HALO = 5


def cbca_support_words(lc, rc, H, W, D, direction):
    """The supports of every (y, x, d) as the pipeline's 32-bit words
    (cbca_mask_build_kernel): bits 0..10 the taps k = -5..5 of the support
    row (bit k + 5), bits 11..21 the taps of the support column, bits 22..28
    the number of support pixels, bit 31 set where x + d*direction leaves
    the image (the pass copies the input there).  uint32 [H, W, D]."""
    lc = np.asarray(lc, np.float32)
    rc = np.asarray(rc, np.float32)
    h = MASK_HALO
    x = np.arange(W)[None, :, None]
    d = np.arange(D)[None, None, :]
    dd = d * direction
    xm = x + dd
    valid = np.broadcast_to((xm >= 0) & (xm < W), (H, W, D))
    xmc = np.clip(xm, 0, W - 1)[0]

    def arm(a, side):
        if side == 0:
            return np.broadcast_to(lc[a][:, :, None], (H, W, D)).astype(np.int64)
        return rc[a][:, xmc].astype(np.int64)

    ks = np.maximum(arm(0, 0), arm(0, 1) - dd) - x
    kt = np.minimum(arm(1, 0), arm(1, 1) - dd) - x
    cnt_row = np.where(valid, np.maximum(kt - ks - 1, 0), 0)
    hm = np.zeros((H, W, D), np.int64)
    for k in range(-h, h + 1):
        hm |= np.where(valid & (k > ks) & (k < kt), 1 << (k + h), 0)
    y = np.arange(H)[:, None, None]
    vs = np.maximum(arm(2, 0), arm(2, 1)) - y
    vt = np.minimum(arm(3, 0), arm(3, 1)) - y
    vm = np.zeros((H, W, D), np.int64)
    cnt = np.zeros((H, W, D), np.int64)
    for k in range(-h, h + 1):
        m = (k > vs) & (k < vt)
        vm |= np.where(m, 1 << (k + h), 0)
        yy = np.arange(H) + k
        inside = ((yy >= 0) & (yy < H))[:, None, None]
        cnt += np.where(m & inside, cnt_row[np.clip(yy, 0, H - 1)], 0)
    words = hm | (vm << 11) | ((cnt & 0x7F) << 22)
    return np.where(valid, words, 1 << 31).astype(np.uint32)


def cbca_from_words(words, vol):
    """One CBCA pass from the support words (cbca_hwd_mask_kernel): the same
    taps, in the same ascending order and float32 arithmetic, as
    cbca_separable.  float32 [H, W, D]."""
    words = np.asarray(words, np.uint32).astype(np.int64)
    vol = np.asarray(vol, np.float32)
    H, W, D = vol.shape
    h = MASK_HALO
    xi = np.arange(W)[:, None]
    dix = np.broadcast_to(np.arange(D)[None, :], (W, D))
    R = np.zeros((H, W, D), np.float32)
    for k in range(-h, h + 1):
        xx = xi + k
        m = ((words >> (k + h)) & 1).astype(bool) & ((xx >= 0) & (xx < W))[None]
        R = R + np.where(m, vol[:, np.clip(xx, 0, W - 1), dix], np.float32(0))
    S = np.zeros((H, W, D), np.float32)
    for k in range(-h, h + 1):
        yy = np.arange(H) + k
        m = ((words >> (k + h + 11)) & 1).astype(bool) & ((yy >= 0) & (yy < H))[:, None, None]
        S = S + np.where(m, R[np.clip(yy, 0, H - 1)], np.float32(0))
    cnt = ((words >> 22) & 0x7F).astype(np.float32)
    copy = ((words >> 31) & 1).astype(bool)
    return np.where(copy, vol, S / np.maximum(cnt, 1)).astype(np.float32)
