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


def test_spmv_traffic_ratio_is_the_profiled_one():
    import bench

    # the ratio comes from the ncu capture summarised in the profiles: within 1 % of 1
    assert abs(bench.SPMV_TRAFFIC_PER_ALGORITHMIC_BYTE - 1.0) < 0.01
