"""Host parts of the Python-3 driver: PFM files as the reference's
pylibs/pfmutil.py writes them, and calib.txt."""
import struct

import numpy as np


def test_pfm_matches_the_reference_layout(tmp_path):
    from cbmv_b200 import pfm
    img = np.arange(12, dtype=np.float32).reshape(3, 4) / 7
    path = str(tmp_path / "d.pfm")
    pfm.save(path, img)
    raw = open(path, "rb").read()
    # header lines, negative scale = little-endian, rows bottom-up (pfmutil.py:44-66)
    assert raw.startswith(b"Pf\n4 3\n-1.000000\n")
    body = raw[len(b"Pf\n4 3\n-1.000000\n"):]
    assert struct.unpack("<4f", body[:16]) == tuple(img[2])
    back, scale = pfm.load(path)
    assert scale == 1.0 and np.array_equal(back, img)


def test_pfm_big_endian_and_colour(tmp_path):
    from cbmv_b200 import pfm
    img = np.random.default_rng(1).random((2, 3, 3)).astype(np.float32)
    path = str(tmp_path / "c.pfm")
    with open(path, "wb") as f:  # a big-endian colour file, as other tools write them
        f.write(b"PF\n3 2\n2.5\n")
        np.flipud(img).astype(">f4").tofile(f)
    back, scale = pfm.load(path)
    assert scale == 2.5 and np.array_equal(back, img)


def test_calib(tmp_path):
    from cbmv_b200.driver import read_calib
    p = tmp_path / "calib.txt"
    p.write_text("cam0=[1 0 0]\ndoffs=0\nbaseline=193\nwidth=694\nheight=554\nndisp=128\nvmin=1\n")
    assert read_calib(str(p)) == (694, 554, 128)


def test_bad_x_counts_as_the_reference_evaluator():
    """bad-x as Evaluator.h:196-211: 1 - |{|d - gt| <= thr} & mask| / |mask|;
    a NaN disparity is an error, an infinite ground truth is outside the
    mask, the threshold itself is not an error."""
    from cbmv_b200.evaluate import bad_x
    gt = np.array([[10.0, 10.0, 10.0], [10.0, np.inf, 10.0]], np.float32)
    disp = np.array([[12.0, 12.5, np.nan], [10.0, 99.0, 7.0]], np.float32)
    mask = np.array([[True, True, True], [True, True, False]])
    # in the mask with a finite gt: 12 (|2| <= 2, good), 12.5 (bad), NaN (bad), 10 (good)
    assert bad_x(disp, gt, mask) == 0.5
    assert bad_x(disp, gt, mask, thr=3.0) == 0.25
    assert bad_x(disp, gt, np.ones_like(mask)) == 0.6  # + 7 vs 10 (bad); the inf pixel stays out
