"""The Python-3 driver (main.py's flow) over scene directories in the
reference's layout, on the GPU."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
MLP = os.path.join(HERE, "golden", "mlp_694x554.npz")


def _scene(root, name, seed, w=150, h=90, d=24):
    from PIL import Image
    from cbmv_b200 import pfm, synth
    L, R, gt, _ = synth.make_pair(seed=seed, width=w, height=h, ndisp=d, planes=4, dmin=2, dmax=d - 4)
    os.makedirs(os.path.join(root, name))
    Image.fromarray(L).save(os.path.join(root, name, "im0.png"))
    Image.fromarray(R).save(os.path.join(root, name, "im1.png"))
    with open(os.path.join(root, name, "calib.txt"), "w") as f:
        f.write("width=%d\nheight=%d\nndisp=%d\n" % (w, h, d))
    pfm.save(os.path.join(root, name, "disp0GT.pfm"), gt)
    return L, R, d


def test_driver_test_and_cost_volume_flags(gpu, tmp_path):
    from cbmv_b200 import driver, pfm
    from cbmv_b200.mlp import GpuMlp
    from cbmv_b200.pipeline import StereoPipeline
    root = str(tmp_path) + "/"
    L, R, d = _scene(root, "scene", 5)
    out = str(tmp_path / "res" / "disp.pfm")
    probdir = str(tmp_path / "res") + "/"
    driver.main(["--data_path", root, "--test_set", "scene", "--model", MLP, "--disp_save_path", out,
                 "--prob_save_path", probdir, "--saveCostVolume"])
    disp, _ = pfm.load(out)
    want = StereoPipeline().run_mlp(GpuMlp.load(MLP), L, R, d)
    assert np.array_equal(disp, want)
    assert os.path.exists(probdir + "scene.prob.npy")
    out2 = str(tmp_path / "res" / "disp2.pfm")
    driver.main(["--data_path", root, "--test_set", "scene", "--model", MLP, "--disp_save_path", out2,
                 "--prob_save_path", probdir, "--loadCostVolume"])
    assert np.array_equal(pfm.load(out2)[0], want)


def test_driver_train_then_test(gpu, tmp_path):
    from cbmv_b200 import driver, pfm
    root = str(tmp_path) + "/"
    for k in range(2):
        _scene(root, "s%d" % k, 30 + k)
    with open(str(tmp_path / "train.txt"), "w") as f:
        f.write("s0,s1\n")
    model = str(tmp_path / "forest.npz")
    driver.main(["--train", "--data_path", root, "--train_set", str(tmp_path / "train.txt"), "--model", model])
    out = str(tmp_path / "d.pfm")
    driver.main(["--data_path", root, "--test_set", "s0", "--model", model, "--disp_save_path", out])
    disp, _ = pfm.load(out)
    assert disp.shape == (90, 150) and np.isfinite(disp).all()
