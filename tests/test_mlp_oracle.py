"""The float64 network restatement (oracle/mlp_ref.py) is itself checked
against central finite differences of its own loss (no bf16 rounding in
this check), so the GPU gradient test rests on a verified backward pass."""
import numpy as np


def test_oracle_backward_matches_finite_differences(monkeypatch):
    from oracle import mlp_ref
    monkeypatch.setattr(mlp_ref, "bf16", lambda x: np.asarray(x, np.float64))
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
    _, g, _ = mlp_ref.loss_and_grads(vec, X, y)
    for j in rng.choice(np.arange(60, vec.size), 40, replace=False):
        e = np.zeros_like(vec)
        e[j] = 1e-6
        lp, _, _ = mlp_ref.loss_and_grads(vec + e, X, y)
        lm, _, _ = mlp_ref.loss_and_grads(vec - e, X, y)
        fd = (lp - lm) / 2e-6
        assert abs(fd - g[j - 60]) < 1e-6 + 1e-4 * abs(fd), (j, fd, g[j - 60])
