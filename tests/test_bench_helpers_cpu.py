"""bench.py's measurement arithmetic on CPU: the roofline of the dominant kernel (algorithmic
bytes per launch over its average CUDA-event time, against the measured peak), the traffic
and FP64-pipe figures taken from the committed ncu summaries, per-kernel rates and the
whole-job value. No GPU: the profiles are fed in as the dicts the library returns."""

import importlib
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    sys.path.insert(0, ROOT)
    return importlib.import_module("bench")


PEAKS = {"hbm_gbs": 6500.0, "source": "test"}


def test_roofline_of_the_dominant_kernel(bench):
    # 100 launches of the split sum sweep over 8 x 1024^2 cells each, 95 us per launch
    cells = 8 * 1024 * 1024
    prof = {"sweep32_sums": (100 * 0.095, 100), "sweep32_update": (100 * 0.073, 100), "dct32_cols": (100 * 0.039, 100)}
    r = bench.roofline(prof, cells * 100, 1, PEAKS)
    assert r["kernel"] == "sweep32_sums" and r["bound"] == "hbm" and r["unit"] == "GB/s"
    assert r["alg_bytes_per_launch"] == 24 * cells
    assert r["achieved"] == pytest.approx(24 * cells / 95e-6 / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / PEAKS["hbm_gbs"])
    assert r["avg_launch_us"] == pytest.approx(95.0)
    # traffic: the committed ncu bytes per cell times the cells of one launch
    traffic = json.load(open(os.path.join(ROOT, "profiles", "traffic_per_cell.json")))["sweep32_sums"]
    assert r["traffic"] == pytest.approx(traffic * cells)
    # the FP64-pipe context of a kernel below the HBM roofline
    pipes = json.load(open(os.path.join(ROOT, "profiles", "pipe_utilisation.json")))["sweep32_sums"]
    assert r["fp64_pipe_busy"] == pipes["fp64_pipe"] and r["registers"] == pipes["registers"]


def test_roofline_without_algorithmic_bytes(bench):
    r = bench.roofline({"some_other_kernel": (5.0, 10)}, 1000, 1, PEAKS)
    assert r == {"kernel": "some_other_kernel", "launches": 10, "total_ms": 5.0, "bound": None}
    assert bench.roofline(None, 0, 1, PEAKS) is None


def test_kernel_rates(bench):
    cells = 4 * 1024 * 1024
    rates = bench.kernel_rates({"dct32_rows_fwd": (2.0, 100), "forward_mesh": (0.5, 8)}, cells * 100, PEAKS)
    fwd = rates["dct32_rows_fwd"]
    assert fwd["avg_launch_us"] == pytest.approx(20.0)
    assert fwd["achieved_gbs"] == pytest.approx(8 * cells * 100 / 2e-3 / 1e9)
    assert fwd["frac_of_hbm"] == pytest.approx(fwd["achieved_gbs"] / PEAKS["hbm_gbs"])
    assert "achieved_gbs" not in rates["forward_mesh"]


def test_job_value_and_seeds(bench):
    # whole-job throughput: every rank's instances over the slowest rank's step time
    assert bench.job_value(8, 1, 25.0) == pytest.approx(320.0)
    assert bench.job_value(8, 4, 25.0) == pytest.approx(1280.0)
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert [bench.rank_first_seed(r) for r in range(3)] == [0, 1000, 2000]


def test_algorithmic_bytes_table(bench):
    # FP64 arrays: 5 reads (sums), 4 reads + 3 writes (update), read + write per transform pass;
    # split precision: psi 8 B, the other fields 4 B
    t = bench.ALG_BYTES_PER_CELL
    assert (t["sweep_sums"], t["sweep_update"], t["dct_cols"]) == (40, 56, 16)
    assert (t["sweep32_sums"], t["sweep32_update"], t["dct32_cols"]) == (8 + 4 * 4, 8 + 3 * 4 + 8 + 4 + 4, 8)
