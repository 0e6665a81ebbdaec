"""The float64 network restatement (oracle/mlp_ref.py) is itself checked
against central finite differences of its own loss (no bf16 or f16
rounding in this check), so the GPU gradient test rests on a verified
backward pass."""
import numpy as np
import pytest


def test_gelu_against_erf_and_f16_emulation():
    """The network's GELU, evaluated in f16 operations, is within 8.32e-3 of
    x * Phi(x) on every finite f16 value (the clamped polynomial itself is
    within 7.7e-3), exactly x / 0 in the tails and finite up to +-65504
    (saturated input, overflowing x*x); its emulation rounds float64 to f16
    directly (ties to even); the backward pass's derivative is the smooth
    function's (central differences)."""
    from scipy.special import erf
    from oracle import mlp_ref
    xs = np.arange(65536, dtype=np.uint16).view(np.float16).astype(np.float64)
    xs = np.unique(xs[np.isfinite(xs)])
    exact = 0.5 * xs * (1 + erf(xs / np.sqrt(2)))
    g = mlp_ref.gelu_f16(xs)
    assert np.isfinite(g).all()
    assert np.max(np.abs(g - exact)) <= 8.32e-3
    assert np.all(g[xs >= 3.5] == xs[xs >= 3.5]) and np.all(g[xs <= -3.5] == 0)
    assert np.array_equal(mlp_ref.f16(g), g)                          # f16 values
    v = np.array([1 + 2.0 ** -11, 1 + 3 * 2.0 ** -11, 1 + 2.0 ** -11 + 2.0 ** -40])
    assert list(mlp_ref.f16(v)) == [1.0, 1 + 2.0 ** -9, 1 + 2.0 ** -10]   # ties to even; above a tie rounds up
    assert list(mlp_ref.f16_sat(np.array([7e4, -7e4]))) == [65504.0, -65504.0]
    assert list(mlp_ref.gelu_f16(np.array([1e6, -1e6]))) == [65504.0, 0.0]
    h = 1e-6
    xm = np.linspace(-3.2, 3.2, 1001)
    smooth = lambda x: x * np.clip(0.5 + x * ((mlp_ref.G[2] * x * x + mlp_ref.G[1]) * x * x + mlp_ref.G[0]), 0, 1)
    xb = mlp_ref.f16(xm.astype(np.float32))
    fdb = (smooth(xb + h) - smooth(xb - h)) / (2 * h)
    assert np.max(np.abs(fdb - mlp_ref.gelu(xm)[1])) < 1e-5


def test_bf16_gelu_against_erf_and_bf16_emulation():
    """The fused kernel's bf16-form GELU is within 1.21e-2 of x * Phi(x) on
    every finite bf16 value, exactly x above 2.6 and 0 below -2.63, bf16
    valued (subnormals included); the direct bf16 rounding ties to even,
    subnormals on the 2^-133 grid."""
    from scipy.special import erf
    from oracle import mlp_ref
    x32 = (np.arange(65536, dtype=np.uint32) << 16).view(np.float32)
    xs = np.unique(x32[np.isfinite(x32)].astype(np.float64))  # NaN patterns dropped before the cast
    exact = 0.5 * xs * (1 + erf(xs / np.sqrt(2)))
    g = mlp_ref.gelu_bf16(xs)
    assert np.isfinite(g).all()
    assert np.max(np.abs(g - exact)) <= 1.21e-2
    assert np.all(g[xs >= 2.6] == xs[xs >= 2.6]) and np.all(g[xs <= -2.63] == 0)
    assert np.array_equal(mlp_ref.bf16(g), g)
    q = 2.0 ** -133
    v = np.array([1 + 2.0 ** -8, 1 + 3 * 2.0 ** -8, 1 + 2.0 ** -8 + 2.0 ** -40, 1.5 * q, 2.5 * q])
    assert list(mlp_ref.bf16_rn(v)) == [1.0, 1 + 2.0 ** -6, 1 + 2.0 ** -7, 2 * q, 2 * q]


@pytest.mark.parametrize("act", ["relu", "gelu"])
def test_oracle_backward_matches_finite_differences(monkeypatch, act):
    from oracle import mlp_ref
    for name in ("bf16", "bf16_rn", "f16", "f16_sat", "f16_acc"):
        monkeypatch.setattr(mlp_ref, name, lambda x: np.asarray(x, np.float64))
    rng = np.random.default_rng(0)
    n = 37
    X = rng.normal(size=(n, 20))
    y = (rng.random(n) < 0.5).astype(np.float64)
    sizes = [20, 20, 20, 128 * 20, 128, 128 * 128, 128, 64 * 128, 64, 64, 1]
    vec = rng.normal(scale=0.1, size=sum(sizes))
    vec[:20] = 1e9      # cap
    vec[20:40] = 0.0    # mu
    vec[40:60] = 1.0    # inv_sd
    # the input transform runs in float32 even here; use exactly representable inputs
    X = X.astype(np.float32).astype(np.float64)
    _, g, _ = mlp_ref.loss_and_grads(vec, X, y, act)
    for j in rng.choice(np.arange(60, vec.size), 40, replace=False):
        e = np.zeros_like(vec)
        e[j] = 1e-6
        lp, _, _ = mlp_ref.loss_and_grads(vec + e, X, y, act)
        lm, _, _ = mlp_ref.loss_and_grads(vec - e, X, y, act)
        fd = (lp - lm) / 2e-6
        assert abs(fd - g[j - 60]) < 1e-6 + 1e-4 * abs(fd), (j, fd, g[j - 60])


@pytest.mark.parametrize("prec", ["f16", "bf16"])
@pytest.mark.parametrize("act", ["relu", "gelu"])
def test_fused_model_close_to_float64_network(act, prec):
    """The oracle's model of the fused inference kernel (16-bit inputs,
    weights and activations, biases as 16-bit high + low parts) stays within
    16-bit rounding of the float64 network, and the high + low split
    reproduces each bias to 2^-21 relative in f16 (above its subnormal
    range), 2^-16 in bf16."""
    from oracle import mlp_ref
    rng = np.random.default_rng(1)
    sizes = [20, 20, 20, 128 * 20, 128, 128 * 128, 128, 64 * 128, 64, 64, 1]
    vec = np.concatenate([np.full(20, 1e9), np.zeros(20), np.ones(20),
                          rng.normal(scale=0.2, size=sum(sizes) - 60)])
    X = rng.normal(size=(500, 20)).astype(np.float32)
    z_model = mlp_ref.forward_fused(vec, X, act, prec)
    z_exact = mlp_ref.forward(vec, X, act)["z"]
    scale = np.abs(z_exact).max()
    assert np.abs(z_model - z_exact).max() < 0.05 * scale
    assert np.abs(z_model - z_exact).mean() < 0.01 * scale
    b = mlp_ref.unpack(vec)["b2"].astype(np.float32)
    if prec == "f16":
        hi, lo = mlp_ref.split_f16(b)
        assert np.all(np.abs((hi + lo) - b) <= 2.0 ** -21 * np.abs(b) + 2.0 ** -25)
    else:
        hi, lo = mlp_ref.split_bf16(b)
        assert np.all(np.abs((hi + lo) - b) <= 2.0 ** -16 * np.abs(b))
    with pytest.raises(ValueError):
        mlp_ref.forward_fused(vec, X, act, "f32")
