"""Tensor-core (tcgen05) kernels of the learned classifier against a plain
torch float32 reference of the same op."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(128, 32, 64), (256, 128, 128), (384, 64, 192), (128, 256, 64),
                                   (1024, 96, 640)])
def test_gemm_bf16_matches_fp32_reference(gpu, M, N, K):
    from cbmv_b200 import _lib
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn((M, K), generator=g, device="cuda").to(torch.bfloat16)
    B = torch.randn((N, K), generator=g, device="cuda").to(torch.bfloat16)
    C = torch.full((M, N), float("nan"), device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("cbmv_gemm_bf16", A.data_ptr(), B.data_ptr(), C.data_ptr(), M, N, K, status.data_ptr(), None)
    torch.cuda.synchronize()
    assert status.item() == 0
    ref = A.float() @ B.float().t()
    # bf16 inputs are exact in fp32; only the fp32 accumulation order differs
    torch.testing.assert_close(C, ref, rtol=1e-5, atol=1e-4 * np.sqrt(K))


def _toy(seed, n):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, 20)).astype(np.float32) * np.linspace(0.5, 40, 20).astype(np.float32)
    X[rng.random((n, 20)) < 0.02] = 2147483648.0  # cost sentinels
    y = ((X[:, 0] + 0.05 * X[:, 7] - 0.01 * X[:, 12]) > 0).astype(np.float32)
    return X, y


@pytest.mark.parametrize("act", ["relu", "gelu"])
def test_mlp_gradients_match_fp64_oracle(gpu, act):
    """Device forward+backward (tcgen05 GEMMs, float32 accumulation) vs the
    float64 restatement rounding to bf16 at the same points: rel. error of
    every gradient block below 1e-3."""
    from cbmv_b200.mlp import MlpParams, MlpTrainer, input_stats
    from oracle import mlp_ref
    X, y = _toy(0, 256)
    cap, mu, sd = input_stats(X)
    net = MlpParams.init(1, cap, mu, sd, act)
    v = net.views()
    v["b1"][:] = 0.1
    v["b2"][:] = -0.05
    v["b3"][:] = 0.02
    v["b4"][:] = 0.3
    tr = MlpTrainer(net, batch=256)
    g, loss = tr.gradients(torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda())
    torch.cuda.synchronize()
    assert tr.status() == 0
    lref, gref, _ = mlp_ref.loss_and_grads(net.vec, X, y, act)
    assert abs(loss.item() - lref) < 1e-5 * max(1.0, abs(lref))
    g = g.cpu().numpy().astype(np.float64)
    sizes = [128 * 20, 128, 128 * 128, 128, 64 * 128, 64, 64, 1]
    o = 0
    for s in sizes:
        a, b = g[o:o + s], gref[o:o + s]
        err = np.abs(a - b).max() / max(np.abs(b).max(), 1e-12)
        assert err < 1e-3, (o, s, err)
        o += s


@pytest.mark.parametrize("act", ["relu", "gelu"])
def test_mlp_training_reduces_loss(gpu, act):
    from cbmv_b200.mlp import MlpParams, MlpTrainer, input_stats
    X, y = _toy(1, 8192)
    cap, mu, sd = input_stats(X)
    tr = MlpTrainer(MlpParams.init(2, cap, mu, sd, act), batch=1024)
    Xt, yt = torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda()
    losses = []
    for it in range(60):
        s = (it * 1024) % 8192
        losses.append(tr.step(Xt[s:s + 1024], yt[s:s + 1024], 3e-3).item())
    assert tr.status() == 0
    assert np.mean(losses[-8:]) < 0.5 * np.mean(losses[:4]), losses


@pytest.mark.parametrize("prec", ["f16", "bf16"])
@pytest.mark.parametrize("act", ["relu", "gelu"])
def test_fused_inference_matches_oracle_forward(gpu, small_pair, act, prec):
    """cbmv_run_mlp's matching cost (float32 features + four tcgen05 layers
    fused on f16 or bf16 operands, 16-bit ReLU or GELU activations, biases
    as 16-bit high + low parts) against (a) the oracle's model of the same
    arithmetic: max 5e-3, mean 3e-4 on P -- the kernel's float32 features
    and accumulation order move a 16-bit rounding of an input or activation
    here and there; (b) the float64 network on the same features: max
    3e-2, mean 2e-3 -- the cost of 16-bit activations."""
    from cbmv_b200.mlp import GpuMlp, MlpParams, input_stats
    from cbmv_b200.pipeline import StereoPipeline
    from oracle import mlp_ref
    L, R, _, _ = small_pair
    H, W = L.shape
    D = 24
    pipe = StereoPipeline()
    idx = torch.arange(H * W * D, device="cuda")
    X = pipe.features_at(L, R, D, idx).cpu().numpy()
    cap, mu, sd = input_stats(X)
    net = MlpParams.init(5, cap, mu, sd, act)
    v = net.views()
    v["b1"][:] = 0.05
    v["b2"][:] = np.linspace(-0.2, 0.2, 128)
    v["b3"][:] = -0.1
    v["b4"][:] = 0.2
    g = GpuMlp(net, prec)
    prob = torch.empty((H, W, D), device="cuda")
    pipe.run_mlp(g, L, R, D, prob_out=prob)
    torch.cuda.synchronize()
    assert g.status() == 0
    got = prob.cpu().numpy().reshape(-1)
    model = 1.0 / (1.0 + np.exp(mlp_ref.forward_fused(net.vec, X, act, prec)))
    exact = 1.0 / (1.0 + np.exp(mlp_ref.forward(net.vec, X, act)["z"]))
    e_model, e_exact = np.abs(got - model), np.abs(got - exact)
    print("%s %s fused vs model: max %.2e mean %.2e; vs float64 network: max %.2e mean %.2e"
          % (act, prec, e_model.max(), e_model.mean(), e_exact.max(), e_exact.mean()))
    assert e_model.max() < 5e-3 and e_model.mean() < 3e-4, (e_model.max(), e_model.mean())
    assert e_exact.max() < 3e-2 and e_exact.mean() < 2e-3, (e_exact.max(), e_exact.mean())


def test_training_samples_follow_labels(gpu):
    from cbmv_b200 import synth
    from cbmv_b200.train_mlp import pick_samples
    L, R, gt, nonocc = synth.make_pair(seed=3, width=80, height=50, ndisp=24, planes=3, dmin=2, dmax=18)
    idx, lab = pick_samples(gt, nonocc, 500, 1, ndisp=24)
    d = idx % 24
    g = gt.reshape(-1)[idx // 24]
    assert np.all(np.abs(d[lab == 1] - g[lab == 1]) <= 1)
    assert np.all(np.abs(d[lab == 0] - g[lab == 0]) > 1)
    assert abs(lab.mean() - 0.5) < 0.02
