"""Host-side pieces of bench.py (no GPU): the launch count it claims, the
algorithmic figures its rooflines use, and the reading of the nvidia-smi
clock samples."""
import os
import re

from conftest import ROOT


def _bench():
    import bench
    return bench


def test_launch_count_matches_the_committed_launch_list():
    """gpu_launches = launches_per_pair x steps; with the default parameters
    one pair is the 33 launches the ncu launch list of the headline step
    shows per pass."""
    from cbmv_b200 import _lib
    b = _bench()
    dp = _lib.default_params
    assert b.launches_per_pair(dp(), "mlp") == 33
    text = open(os.path.join(ROOT, "profiles", "launches_694x554_mlp.md")).read()
    m = re.search(r"Per pass: (\d+) launches", text)
    assert m and int(m.group(1)) == 33
    # the forest path: ZSAD window means and four float64 statistics launches
    assert b.launches_per_pair(dp(), "rf") == 37
    text = open(os.path.join(ROOT, "profiles", "launches_694x554_rf.md")).read()
    m = re.search(r"Per pass (\d+) launches", text)
    assert m and int(m.group(1)) == 37
    # every SGM iteration adds its scan and its combine, every CBCA pass one
    # launch; one support build per chain, none when the passes build their
    # own supports (L1 > 6 or the reference's summation order)
    assert b.launches_per_pair(dp(sgm_i=1)) == 31
    assert b.launches_per_pair(dp(cbca_i2=2)) == 31
    assert b.launches_per_pair(dp(cbca_i1=1, cbca_i2=1)) == 31
    assert b.launches_per_pair(dp(L1=9)) == 32
    assert b.launches_per_pair(dp(exact_cbca=1)) == 32
    # _interp: the right view's cost, chain and WTA, then the check and fills
    assert b.launches_per_pair(dp(interpolate=1)) == 33 + 1 + 9 + 1 + 3


def test_algorithmic_figures():
    b = _bench()
    # the dense 20-128-128-64-1 network: 2 x (20x128 + 128x128 + 128x64 + 64x1)
    assert b.FLOPS_PER_UNIT_MLP == 2 * (20 * 128 + 128 * 128 + 128 * 64 + 64)
    assert b.MMA_FLOPS_PER_UNIT_MLP == 65536
    # compulsory bytes per (p,d): 4 B cost + SGM 2 x 20 B + CBCA 4 x 8 B + WTA 4 B
    assert b.BYTES_PER_UNIT_PATH == 4 + 2 * 20 + 4 * 8 + 4
    assert b.BYTES_PER_UNIT_INTERP == b.BYTES_PER_UNIT_PATH + 76
    assert b.UNITS == 694 * 554 * 128


def test_clock_samples_and_throttle_reasons():
    b = _bench()
    c = b.Clocks(0)
    c.out = "\n".join([
        "0, 1965, 1965, 700.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1942, 1965, 990.3, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1950, 1965, 980.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, [N/A], 1965, [N/A], [N/A], [N/A], [N/A], [N/A], [N/A]",
        "garbage",
    ])
    s = c.summary()
    assert s == {"sm_mhz": 1950.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    c.out = "0, 1200, 1965, 900, 0x48, Active, Not Active, Active, Not Active"
    assert c.summary()["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]
    c.out = ""
    assert c.summary()["samples"] == 0
