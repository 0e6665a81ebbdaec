import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
FOREST_PATH = os.path.join(GOLDEN, "forest_694x554.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libcbmv.so")


@pytest.fixture(scope="session")
def oracle_cpu():
    from oracle import cpu
    if not cpu.available():
        import subprocess
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True,
                       capture_output=True)
    return cpu


@pytest.fixture(scope="session")
def small_pair():
    from cbmv_b200 import synth
    return synth.make_pair(seed=11, width=120, height=72, ndisp=24, planes=5, dmin=2, dmax=20)


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cbmv_b200 import _lib
    _lib.lib()
    return torch.device("cuda")


def rand_pair(seed, h, w, flat=False):
    rng = np.random.default_rng(seed)
    L = rng.integers(0, 256, (h, w), dtype=np.uint8)
    R = np.roll(L, -3, axis=1).copy()
    R = np.clip(R.astype(int) + rng.integers(-3, 4, (h, w)), 0, 255).astype(np.uint8)
    if flat:
        L[h // 3: h // 3 + 8, w // 4: w // 4 + 10] = 77
        R[h // 3: h // 3 + 8, w // 4: w // 4 + 10] = 77
    return L, R
