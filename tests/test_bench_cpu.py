"""The host-side pieces of bench.py's JSON line: algorithmic bytes per
column, the DRAM traffic and FP64-pipe figures read from the committed
summaries, and the CPU baseline's keys.  No GPU needed."""
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

import bench  # noqa: E402
from mgcm_rt import synth  # noqa: E402


def test_algorithmic_bytes_per_column():
    # 8 * (171 L + 815) with cloud (DETAU and CUMTAUV in and out); minus
    # 8 * 38 * (2L + 4) without
    for L in (24, 36, 48):
        assert bench.algorithmic_bytes_per_column(L, True) == 8 * (171 * L + 815)
        assert bench.algorithmic_bytes_per_column(L, False) == 8 * (171 * L + 815) - 8 * 38 * (2 * L + 4)
    assert bench.algorithmic_bytes_per_column(24, True) == 39352


def test_traffic_scales_with_columns():
    t1 = bench.traffic_per_step("fp64", 8192, 24)
    t2 = bench.traffic_per_step("fp64", 64800, 24)
    assert t1 and t2 and t2 == pytest.approx(t1 * 64800 / 8192)
    assert bench.traffic_per_step("fp64", 8192, 48) is None   # captured at L = 24 only


def test_fp64_pipe_figures():
    r = bench.fp64_pipe(24, 64800, 0.014)
    assert r["unit"] == "TFLOP/s" and 0.0 < r["frac"] < 1.0
    assert r["achieved"] == pytest.approx(r["flops_per_column"] * 64800 / 0.014 / 1e12)
    assert r["gather_gbs"] == pytest.approx(r["gathers_per_column"] * 8 * 64800 / 0.014 / 1e9)
    assert bench.fp64_pipe(36, 100, 1.0) is None                # no counts for that layer count


def test_cpu_baseline_keys(data_dir):
    b = synth.make_batch(64, L=24, seed=1000, cloud=True)
    r = bench.cpu_baseline(b, data_dir, budget_s=0.2)
    for k in ("value", "unit", "cores", "kind", "sample", "one_core", "cpu_model"):
        assert k in r
    assert r["kind"] == "port" and r["value"] > 0 and r["one_core"]["value"] > 0
