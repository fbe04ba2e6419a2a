"""bench.py's arithmetic, on the CPU: the roofline of each kernel kind is its
algorithmic work over its device time, DRAM traffic comes from the committed ncu
table scaled by points, and the reference arm prints nothing on ranks other than 0."""
import json
import os
import sys
import types

import pytest

from conftest import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402


def stats(**kw):
    s = {"key_bytes": 4, "n_valid": 1_000_000, "sort_passes": 4, "pipelines": 0, "union_pairs": 3_000_000,
         "count_pairs": 50_000_000, "border_pairs": 100_000, "count_pair_dims": 150_000_000,
         "union_pair_dims": 9_000_000, "border_pair_dims": 300_000}
    s.update(kw)
    return s


def test_sort_roofline_is_bytes_per_pass_over_time():
    r = bench.roofline("radix_sort", 0.5, stats(), 1_000_000, 6500.0, "measured", {})
    # per pass: upsweep reads 4-byte keys, downsweep reads and writes (key, id)
    expect = 1_000_000 * (4 + 2 * 8) * 4 / 0.5e-3 / 1e9
    assert r["achieved"] == pytest.approx(expect)
    assert r["frac"] == pytest.approx(expect / 6500.0) and r["unit"] == "GB/s" and r["bound"] == "hbm"


def test_union_roofline_counts_parent_reads_and_point_writes():
    r = bench.roofline("union_kernel", 0.25, stats(), 1_000_000, 6500.0, "measured", {})
    assert r["achieved"] == pytest.approx((8 * 3_000_000 + 12 * 1_000_000) / 0.25e-3 / 1e9)


def test_count_roofline_is_three_fp32_ops_per_pair_dimension():
    r = bench.roofline("count_kernel", 2.0, stats(), 1_000_000, 6500.0, "measured", {"sm_mhz": 1965.0})
    assert r["achieved"] == pytest.approx(150_000_000 * 3 / 2.0e-3 / 1e12)
    assert r["peak"] == pytest.approx(148 * 128 * 1965.0e6 / 1e12)
    assert r["unit"] == "TFLOP/s"


def test_traffic_table_scales_by_points():
    t12 = bench.traffic_per_launch("plain-3d-10m", "count_kernel", 12_000_000)
    t10 = bench.traffic_per_launch("plain-3d-10m", "count_kernel", 10_000_000)
    assert t12 and t10 == pytest.approx(t12 * 10 / 12)
    assert bench.traffic_per_launch("plain-3d-10m", "no_such_kernel", 10) is None


def test_peaks_read_the_measured_file():
    hbm, src = bench.peaks()
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        assert src == "measured" and hbm == pytest.approx(float(json.load(open(p))["hbm_gbs"]))
    else:
        assert (hbm, src) == (bench.HBM_PEAK_FALLBACK, "fallback")


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = types.SimpleNamespace(config=2, cpu_sample=1000, steps=1, warmup=0, gpus=2)
    assert bench.run_reference_arm(args) == 0
    assert capsys.readouterr().out == ""


def test_reference_arm_line_on_rank_zero(monkeypatch, capsys):
    monkeypatch.setenv("RANK", "0")
    monkeypatch.setenv("WORLD_SIZE", "1")
    args = types.SimpleNamespace(config=2, cpu_sample=2000, steps=1, warmup=0, gpus=1)
    assert bench.run_reference_arm(args) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_cpu_baseline_extrapolates_quadratically():
    import importlib
    pkg = importlib.import_module("nextdbscan-exa_b200")
    cb = bench.cpu_reference(pkg, 3, 2000, 2)
    assert cb["full_n"] == 2_000_000
    assert cb["extrapolated_value_at_full_n"] == pytest.approx(cb["value"] * 2000 / 2_000_000)
