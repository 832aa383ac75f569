"""Host-side pieces of bench.py (CPU): the clock/throttle summary of nvidia-smi samples, the
roofline denominator, and the algorithmic bytes of the block SpMV."""

import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def test_clock_summary_flags_throttle_reasons():
    import bench

    c = bench.Clocks(0)
    c.lines = ["1965, 1965, 820.1, Not Active, Not Active, Not Active, Not Active",
               "1950, 1965, 990.0, Not Active, Not Active, Not Active, Active",
               "1965, 1965, 1000.3, Not Active, Active, Not Active, Not Active",
               "garbage"]
    s = c.summary()
    assert s["samples"] == 3 and s["sm_max_mhz"] == 1965.0 and s["sm_mhz"] == 1965.0
    assert s["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]


def test_roofline_denominator_is_the_measured_copy_bandwidth():
    import bench

    peak, kind = bench.peaks()
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        assert kind == "measured" and peak == float(json.loads(p.read_text())["hbm_gbs"])
    else:
        assert kind == "fallback" and peak == 6650.0


def test_algorithmic_byte_formulas():
    import bench

    n, nnz = 400_686, 9_896_216
    # the FP64 block SpMV: 132 B per block, 72 B per row and 8 (the last row pointer)
    assert bench.spmv_bytes(n, nnz) == 132 * nnz + 72 * n + 8
    # FP32 values, FP32 vectors: 68 B per block
    assert bench.spmv_bytes(n, nnz, 4, 4) == 68 * nnz + 8 * (n + 1) + 32 * n
    # a Gauss-Seidel pass adds the inverse (128 B per row in FP64) and one more vector pass
    assert bench.gs_pass_bytes(n, nnz) == bench.spmv_bytes(n, nnz) + 128 * n + 32 * n
    stats = {"levels": [n, 120_000, 24_000, 20], "blocks": [nnz, 4_000_000, 900_000, 400]}
    v64, v32 = bench.vcycle_bytes(stats, 8), bench.vcycle_bytes(stats, 4)
    # six passes on the finest level dominate; FP32 values take a bit more than half the bytes
    assert 6 * bench.gs_pass_bytes(n, nnz) < v64 < 12 * bench.gs_pass_bytes(n, nnz)
    assert 0.45 * v64 < v32 < 0.6 * v64


def test_reference_arm_times_measured_full_size_iterations(monkeypatch, capsys):
    """The reference arm reports the outer iterations it timed, at the size it ran, without
    scaling: at most REFERENCE_MAX_STEPS after one untimed iteration."""
    import types

    import bench

    calls = []

    class Fake:
        n_nodes = 400_686
        linear_iterations = [3, 2, 2]

        def __init__(self, n_axial):
            calls.append(n_axial)

        def step(self):
            return 2.0

    monkeypatch.setattr(bench, "CpuCase", Fake)
    args = types.SimpleNamespace(axial=285, steps=20, warmup=5)
    bench.reference_arm(args, 0, 1)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert calls == [285]
    assert line["impl"] == "reference" and line["steps"] == bench.REFERENCE_MAX_STEPS
    assert line["steps_requested"] == 20 and line["warmup"] == 1
    assert line["value"] == 0.5 and line["ms_per_step"] == 2000.0
    assert line["e2e"]["value"] == line["value"] and line["config"]["nodes"] == 400_686
    assert line["cpu_baseline"]["cores"] == 1 and "nproc" in line["cpu_baseline"]["host"]
    bench.reference_arm(args, 1, 2)          # other ranks print nothing
    assert capsys.readouterr().out == ""
