"""The fused pipeline (images -> disparity on the device) against the
reference's test path restated over the oracle (matchers, features, random
forest, eval_prob with the _mem post-processing)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _small_forest(oracle_cpu):
    from sklearn.ensemble import RandomForestClassifier
    from oracle import glue
    from cbmv_b200 import synth
    from cbmv_b200.forest import FlatForest
    S = []
    for seed in (31, 32):
        L, R, gt, _ = synth.make_pair(seed=seed, width=120, height=72, ndisp=24, planes=5, dmin=2, dmax=20)
        S.append(glue.create_samples_mem(oracle_cpu.mtc, oracle_cpu.fte, L, R, gt, 24,
                                         lambda g, nd: oracle_cpu.fte.generate_d_indices(g, nd, 1, seed=seed)))
    S = np.concatenate(S).astype(np.float32)
    rf = RandomForestClassifier(n_estimators=10, min_samples_leaf=50, max_depth=20, random_state=0,
                                n_jobs=4).fit(S[:, :20], S[:, 20])
    return FlatForest.from_sklearn(rf)


@pytest.fixture(scope="module")
def forest(oracle_cpu):
    return _small_forest(oracle_cpu)


def test_pipeline_matches_reference_path(gpu, oracle_cpu, small_pair, forest):
    from oracle import glue
    from cbmv_b200.forest_gpu import GpuForest
    from cbmv_b200.pipeline import StereoPipeline
    L, R, gt, nonocc = small_pair
    D = 24
    H, W = L.shape
    # reference path, restated over the oracle
    proba = glue.test_model(oracle_cpu.mtc, oracle_cpu.fte,
                            lambda X: np.stack([oracle_cpu.rf_predict(forest, X),
                                                1 - oracle_cpu.rf_predict(forest, X)], 1), L, R, D)
    p0_ref = proba[:, 0].reshape(H, W, D)
    disp_ref = glue.eval_prob(oracle_cpu.post, oracle_cpu.fte, proba, L, R, D)
    # fused GPU path
    gf = GpuForest(forest)
    pipe = StereoPipeline(gf)
    prob = torch.empty((H, W, D), device="cuda")
    disp = pipe.run_rf(L, R, D, prob_out=prob)
    torch.cuda.synchronize()
    p0 = prob.cpu().numpy()
    # identical features -> identical leaves -> P0 equal to float32 rounding
    same = np.mean(p0 == p0_ref.astype(np.float32))
    assert same > 0.9999, same
    # post: separable CBCA by default (rounding differs from the reference's
    # summation order); with exact_cbca the whole chain follows the reference
    close = np.mean(np.abs(disp - disp_ref) <= 0.5)
    print("disparity within 0.5 px: separable CBCA %.5f" % close)
    assert close >= 0.999, close
    t = pipe.timings()
    assert t["total"] > 0
    from cbmv_b200 import _lib
    prm = _lib.default_params()
    prm.exact_cbca = 1
    pipe_x = StereoPipeline(gf, params=prm)
    disp_x = pipe_x.run_rf(L, R, D)
    close_x = np.mean(np.abs(disp_x - disp_ref) <= 0.5)
    print("disparity within 0.5 px: reference-order CBCA %.5f" % close_x)
    assert close_x >= 0.999, close_x


def test_pipeline_long_arms_matches_reference_path(gpu, oracle_cpu, small_pair, forest):
    """Cross arms of up to 8 pixels (L1 = 9; the fused post then aggregates
    from the arms themselves, past the 5-pixel reach of its precomputed
    support words) against the reference path with the same L1."""
    from oracle import glue
    from cbmv_b200 import _lib
    from cbmv_b200.forest_gpu import GpuForest
    from cbmv_b200.pipeline import StereoPipeline
    L, R, _, _ = small_pair
    D = 24
    proba = glue.test_model(oracle_cpu.mtc, oracle_cpu.fte,
                            lambda X: np.stack([oracle_cpu.rf_predict(forest, X),
                                                1 - oracle_cpu.rf_predict(forest, X)], 1), L, R, D)
    disp_ref = glue.eval_prob(oracle_cpu.post, oracle_cpu.fte, proba, L, R, D, p=dict(glue.PARAMS, L1=9))
    prm = _lib.default_params()
    prm.L1 = 9
    disp = StereoPipeline(GpuForest(forest), params=prm).run_rf(L, R, D)
    close = np.mean(np.abs(disp - disp_ref) <= 0.5)
    print("L1 = 9: disparity within 0.5 px %.5f" % close)
    assert close >= 0.999, close


def test_pipeline_repeatable_and_device_io(gpu, small_pair, forest):
    from cbmv_b200.forest_gpu import GpuForest
    from cbmv_b200.pipeline import StereoPipeline
    L, R, _, _ = small_pair
    pipe = StereoPipeline(GpuForest(forest))
    a = pipe.run_rf(L, R, 24)
    l, r = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    b = pipe.run_rf(l, r, 24)
    assert isinstance(b, torch.Tensor) and b.is_cuda
    assert np.array_equal(a, b.cpu().numpy())  # deterministic


def test_host_buffer_entry_points_equal_device_ones(gpu, small_pair, forest):
    """cbmv_run_rf_host / cbmv_run_mlp_host (images in host memory, the
    disparity written to host memory; pageable numpy arrays and pinned
    tensors) give the device-pointer forms' disparity bit for bit, on
    repeated calls and after a larger pair has grown the context's device
    copies."""
    import os
    from cbmv_b200 import synth
    from cbmv_b200.forest_gpu import GpuForest
    from cbmv_b200.mlp import GpuMlp
    from cbmv_b200.pipeline import StereoPipeline
    net = GpuMlp.load(os.path.join(os.path.dirname(__file__), "golden", "mlp_gelu_694x554.npz"))
    pipe = StereoPipeline(GpuForest(forest))
    L2, R2, _, _ = synth.make_pair(seed=12, width=130, height=70, ndisp=32, planes=4, dmin=2, dmax=28)
    for (L, R), D in (((small_pair[0], small_pair[1]), 24), ((L2, R2), 32), ((small_pair[0], small_pair[1]), 24)):
        l, r = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
        Lp, Rp = torch.from_numpy(L).pin_memory(), torch.from_numpy(R).pin_memory()
        out = torch.empty(L.shape, dtype=torch.float32).pin_memory()
        for run in (lambda *a, **k: pipe.run_rf(*a, **k), lambda *a, **k: pipe.run_mlp(net, *a, **k)):
            want = run(l, r, D).cpu().numpy()
            for _ in range(2):
                got = run(L, R, D)
                assert isinstance(got, np.ndarray) and np.array_equal(got, want)
                assert run(Lp, Rp, D, disp_out=out) is out
                assert np.array_equal(out.numpy(), want)


def test_saved_cost_volume_gives_the_same_disparity(gpu, small_pair, tmp_path):
    """--saveCostVolume then --loadCostVolume (main.py:56-67): the post run on
    the reloaded cost reproduces the fused path's disparity bit for bit."""
    from cbmv_b200 import costvol
    from cbmv_b200.mlp import GpuMlp
    from cbmv_b200.pipeline import StereoPipeline
    import os
    L, R, _, _ = small_pair
    H, W = L.shape
    D = 24
    net = GpuMlp.load(os.path.join(os.path.dirname(__file__), "golden", "mlp_694x554.npz"))
    pipe = StereoPipeline()
    prob = torch.empty((H, W, D), device="cuda")
    disp = pipe.run_mlp(net, L, R, D, prob_out=prob)
    for fmt in costvol.FORMATS:
        path = str(tmp_path / ("cost_%s.npy" % fmt))
        costvol.save(path, prob, fmt)
        cost = costvol.load(path, shape=(H, W, D), fmt=fmt)
        assert np.array_equal(pipe.run_post(L, R, cost), disp), fmt


NETS = {"gelu": "mlp_gelu_694x554.npz", "relu": "mlp_694x554.npz"}


@pytest.mark.parametrize("net_kind", ["gelu", "relu"])
@pytest.mark.parametrize("W,H,D", [(97, 53, 37), (150, 64, 70), (694, 64, 128)])
def test_learned_path_matches_reference_path(gpu, oracle_cpu, W, H, D, net_kind):
    """The learned classifier's whole path at sizes off the tile grids (D not
    a multiple of 32, widths not multiples of 8 or 16) and at the headline
    width and disparity count, for the GELU network of record and the ReLU
    variant, against the reference's test path restated over the oracle
    (test_model with the network as its classifier, in batches of 8 rows,
    then eval_prob with the _mem post in the reference's summation order):
    disparities within 0.5 px on >= 99.9 % of pixels, the bar for final
    disparity maps (the device forms the features in float32 and rounds
    activations to f16; the oracle models that arithmetic from the
    float64 features)."""
    import os
    from oracle import glue, mlp_ref
    from cbmv_b200 import synth
    from cbmv_b200.mlp import GpuMlp, MlpParams
    from cbmv_b200.pipeline import StereoPipeline
    mlp = os.path.join(os.path.dirname(__file__), "golden", NETS[net_kind])
    L, R, _, _ = synth.make_pair(seed=W + H + D, width=W, height=H, ndisp=D, planes=4, dmin=2, dmax=D - 4)
    params = MlpParams.load(mlp)
    assert params.activation == net_kind

    def predict(X):
        p0 = 1.0 / (1.0 + np.exp(mlp_ref.forward_fused(params.vec, X, params.activation)))
        return np.stack([p0, 1 - p0], 1)

    proba = glue.test_model(oracle_cpu.mtc, oracle_cpu.fte, predict, L, R, D, batch=8 * W)
    disp_ref = glue.eval_prob(oracle_cpu.post, oracle_cpu.fte, proba, L, R, D)
    disp = StereoPipeline().run_mlp(GpuMlp(params), L, R, D)
    close = np.mean(np.abs(disp - disp_ref) <= 0.5)
    print("learned path (%s) %dx%d D=%d: within 0.5 px %.5f" % (net_kind, W, H, D, close))
    assert close >= 0.999, close


def test_run_classified_uses_the_network(gpu, small_pair, forest):
    """On a clean run the learned classifier answers, not its fallback."""
    import os
    from cbmv_b200.forest_gpu import GpuForest
    from cbmv_b200.mlp import GpuMlp
    from cbmv_b200.pipeline import StereoPipeline
    L, R, _, _ = small_pair
    net = GpuMlp.load(os.path.join(os.path.dirname(__file__), "golden", "mlp_694x554.npz"))
    pipe = StereoPipeline(GpuForest(forest))
    disp, which = pipe.run_classified(L, R, 24, net=net)
    assert which == "mlp" and np.array_equal(disp, pipe.run_mlp(net, L, R, 24))
    disp_rf, which_rf = pipe.run_classified(L, R, 24)
    assert which_rf == "rf" and np.array_equal(disp_rf, pipe.run_rf(L, R, 24))
