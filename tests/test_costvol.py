"""Cost-volume files (the reference's --saveCostVolume/--loadCostVolume,
main.py:56-67): the three layouts round-trip on the host."""
import numpy as np
import pytest


@pytest.mark.parametrize("fmt", ["reference", "hwd", "dhw"])
def test_roundtrip(tmp_path, fmt):
    from cbmv_b200 import costvol
    cost = np.random.default_rng(0).random((5, 7, 3)).astype(np.float32)
    path = str(tmp_path / ("c_" + fmt + ".npy"))
    costvol.save(path, cost, fmt)
    raw = np.load(path)
    if fmt == "reference":
        # predict_proba's layout: [N, 2] float64, rows in (y, x, d) order
        assert raw.shape == (5 * 7 * 3, 2) and raw.dtype == np.float64
        assert np.array_equal(raw[:, 0], cost.reshape(-1).astype(np.float64))
        assert np.allclose(raw[:, 0] + raw[:, 1], 1.0)
        back = costvol.load(path, shape=cost.shape)
    elif fmt == "dhw":
        assert raw.shape == (3, 5, 7)
        back = costvol.load(path, fmt="dhw")
    else:
        back = costvol.load(path)
    assert back.dtype == np.float32 and np.array_equal(back, cost)


def test_reference_name_and_errors(tmp_path):
    from cbmv_b200 import costvol
    assert costvol.reference_path("./results/", "Adirondack") == "./results/Adirondack.prob.npy"
    path = str(tmp_path / "c.npy")
    costvol.save(path, np.zeros((2, 3, 4), np.float32), "reference")
    with pytest.raises(ValueError):
        costvol.load(path)
    with pytest.raises(ValueError):
        costvol.load(path, shape=(2, 3, 5))
