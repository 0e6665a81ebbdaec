"""Float64 restatement of the classifier network's forward and backward
pass (test infrastructure only): the checker of the tcgen05 training kernels.

It follows cbmv_b200's network (include/cbmv.h, cbmv_mlp_*) and rounds to
bfloat16 exactly where the device does -- the GEMM operands (normalised
inputs, hidden activations, back-propagated deltas and the weights) -- and
computes everything else in float64, so the device's remaining differences
are float32 accumulation only.
"""
import numpy as np

F = 20


def bf16(x):
    """Round float64/float32 values to bfloat16 (round to nearest even)."""
    a = np.asarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def relu(x):
    """ReLU and its derivative (0 at x = 0)."""
    return np.maximum(x, 0.0), (x > 0).astype(np.float64)


def bf16_rn(x):
    """Round float64 values to bfloat16 directly (round to nearest even), as
    one bf16 operation rounds its exact result; below 2^-126 onto the
    subnormal grid of 2^-133."""
    a = np.ascontiguousarray(np.asarray(x, np.float64))
    u = a.view(np.uint64)
    r = (((u + np.uint64(0xFFFFFFFFFFF) + ((u >> np.uint64(45)) & np.uint64(1))) >> np.uint64(45))
         << np.uint64(45)).view(np.float64)
    tiny = np.abs(a) < 2.0 ** -126
    return np.where(tiny, np.round(a * 2.0 ** 133) * 2.0 ** -133, r)


def f16(x):
    """Round float64/float32 values to IEEE binary16 directly (round to
    nearest even; beyond 65504 to infinity), returned as float64."""
    with np.errstate(over="ignore"):
        return np.asarray(x, np.float64).astype(np.float16).astype(np.float64)


def f16_sat(x):
    """f16 rounding saturated to the largest finite value, +-65504 (the
    device's `cvt.rn.satfinite` of its float32 accumulators)."""
    return np.clip(f16(x), -65504.0, 65504.0)


def f16_acc(x):
    """A float32 accumulator's value rounded to f16 as the device converts
    it: through float32, saturated."""
    return f16_sat(np.asarray(x, np.float32))


# the network's GELU coefficients (cbmv_b200/csrc/mlp_net.cuh, gelu_t), f16 values
G = np.array([0.37451171875, -0.042694091796875, 0.0022716522216796875])


def gelu_f16(x):
    """The network's GELU as the device evaluates it: x rounded from float32
    to f16, then u = x*x, p = G2 u + G1, p = p u + G0, q = x p + 0.5
    clamped to [0, 1], x*q, each operation rounded once to f16 (mlp_net.cuh
    gelu_t; the fused kernel's packed form is the same, its clamp folded
    into the FMA).  Every product of two f16 values, and the FMAs here, are
    exact in float64 before that one rounding."""
    xh = f16_acc(x)
    with np.errstate(over="ignore", invalid="ignore"):
        u = f16(xh * xh)
        p = f16(G[2] * u + G[1])
        p = f16(p * u + G[0])
        q = f16(xh * p + 0.5)
    q = np.where(np.isnan(q), 0.0, np.clip(q, 0.0, 1.0))
    return f16(xh * q)


def gelu(x):
    """The network's GELU (f16 evaluation) and, for the backward pass, the
    derivative of the smooth function it approximates at f16(x)."""
    g = gelu_f16(x)
    xb = f16_acc(x)
    u = xb * xb
    p = (G[2] * u + G[1]) * u + G[0]
    qr = 0.5 + xb * p
    dq = p + 2 * u * (2 * G[2] * u + G[1])
    d = np.where(qr <= 0, 0.0, np.where(qr >= 1, 1.0, qr + xb * dq))
    return g, d


# the bf16 form's GELU coefficients (cbmv_b200/csrc/mlp_net.cuh, kGB*Bits), bf16 values
GB = np.array([0.373046875, -0.04296875, 0.00238037109375])


def gelu_bf16(x):
    """The GELU of the fused kernel's bf16 form: x rounded from float32 to
    bf16, then u = x*x, p = GB2 u + GB1, p = p u + GB0, q = max(x p + 0.5,
    0) (a `.relu` FMA), q = min(q, 1), x*q, each operation rounded once to
    bf16 (mlp_infer.cuh, Op16<false>::gelu)."""
    xb = bf16(x)
    u = bf16_rn(xb * xb)
    p = bf16_rn(GB[2] * u + GB[1])
    p = bf16_rn(p * u + GB[0])
    q = np.maximum(bf16_rn(xb * p + 0.5), 0.0)
    q = np.minimum(q, 1.0)
    return bf16_rn(xb * q)


ACT = {"relu": relu, "gelu": gelu}


def unpack(vec):
    v, o, out = np.asarray(vec, np.float64), 0, {}
    for name, size in [("cap", F), ("mu", F), ("inv_sd", F), ("W1", 128 * F), ("b1", 128),
                       ("W2", 128 * 128), ("b2", 128), ("W3", 64 * 128), ("b3", 64), ("w4", 64),
                       ("b4", 1)]:
        out[name] = v[o:o + size]
        o += size
    out["W1"] = out["W1"].reshape(128, F)
    out["W2"] = out["W2"].reshape(128, 128)
    out["W3"] = out["W3"].reshape(64, 128)
    return out


def forward(vec, X, act="relu"):
    f_act = ACT[act]
    p = unpack(vec)
    # the input transform in float32, as the device computes it
    c32, m32, s32 = (np.float32(p[k]) for k in ("cap", "mu", "inv_sd"))
    X0 = bf16((np.minimum(np.asarray(X, np.float32), c32) - m32) * s32)
    S1 = X0 @ bf16(p["W1"]).T + p["b1"]
    A1, d1 = f_act(S1)
    S2 = bf16(A1) @ bf16(p["W2"]).T + p["b2"]
    A2, d2 = f_act(S2)
    S3 = bf16(A2) @ bf16(p["W3"]).T + p["b3"]
    A3, d3 = f_act(S3)
    z = A3 @ p["w4"] + p["b4"][0]
    return dict(X0=X0, S1=S1, A1=A1, d1=d1, S2=S2, A2=A2, d2=d2, S3=S3, A3=A3, d3=d3, z=z, p=p)


def loss_and_grads(vec, X, y, act="relu"):
    """Mean BCE and its gradients in parameter order (input transform excluded)."""
    f = forward(vec, X, act)
    p, z = f["p"], f["z"]
    y = np.asarray(y, np.float64)
    B = z.shape[0]
    prob = 1 / (1 + np.exp(-z))
    loss = np.mean(np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))))
    dz = (prob - y) / B
    dw4 = f["A3"].T @ dz
    db4 = dz.sum()
    dS3 = dz[:, None] * p["w4"][None, :] * f["d3"]
    db3 = dS3.sum(0)
    dW3 = bf16(dS3).T @ bf16(f["A2"])
    dA2 = bf16(dS3) @ bf16(p["W3"])
    dS2 = dA2 * f["d2"]
    db2 = dS2.sum(0)
    dW2 = bf16(dS2).T @ bf16(f["A1"])
    dA1 = bf16(dS2) @ bf16(p["W2"])
    dS1 = dA1 * f["d1"]
    db1 = dS1.sum(0)
    dW1 = bf16(dS1).T @ f["X0"]
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3, dw4, [db4]])
    return loss, g, prob


def split_f16(x):
    """f16 high part of float32 x and the f16 rounding of the rest (the
    rest formed in float32)."""
    x = np.asarray(x, np.float32)
    hi = f16_sat(x)
    return hi, f16_sat(x - np.float32(hi))


def split_bf16(x):
    """bf16 high part of float32 x and the bf16 rounding of the rest (the
    rest formed in float32)."""
    x = np.asarray(x, np.float32)
    hi = bf16(x)
    return hi, bf16(x - np.float32(hi))


def forward_fused(vec, X, act="relu", prec="f16"):
    """The network as the fused inference kernel evaluates it (test
    infrastructure), in its f16 form (prec="f16") or its bf16 form
    (prec="bf16"): 16-bit operands throughout -- the normalised inputs, the
    weights, the hidden activations (ReLU of the float32 accumulator rounded
    to the 16-bit type, or that form's GELU of it) -- every bias (and w4) as
    its 16-bit high + low parts; the output layer runs on those 16-bit
    activations.  Returns z."""
    if prec == "f16":
        r16, split, g16 = f16_sat, split_f16, gelu_f16
    elif prec == "bf16":
        r16, split, g16 = bf16, split_bf16, gelu_bf16
    else:
        raise ValueError("prec must be 'f16' or 'bf16'")
    if act == "gelu":
        h = g16
    else:
        def h(s):
            return r16(np.maximum(np.asarray(s, np.float32), 0))
    p = unpack(vec)
    c32, m32, s32 = (np.float32(p[k]) for k in ("cap", "mu", "inv_sd"))
    X0 = r16((np.minimum(np.asarray(X, np.float32), c32) - m32) * s32)
    b1h, b1l = split(p["b1"])
    b2h, b2l = split(p["b2"])
    b3h, b3l = split(p["b3"])
    wh, wl = split(p["w4"])
    A1 = h(X0 @ r16(np.float32(p["W1"])).T + (b1h + b1l))
    A2 = h(A1 @ r16(np.float32(p["W2"])).T + (b2h + b2l))
    A3 = h(A2 @ r16(np.float32(p["W3"])).T + (b3h + b3l))
    return A3 @ (wh + wl) + p["b4"][0]
