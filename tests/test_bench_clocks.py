"""bench.Clocks.summary reads the nvidia-smi samples taken during a timed
region: the median SM clock of the benchmarked GPU, its maximum, and every
throttle reason seen active in any sample (a run with hw_slowdown or a thermal
slowdown is rejected, sw_power_cap is kept and noted)."""
import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(__file__), ".."))

import bench  # noqa: E402

ROWS = [
    # index, sm, max sm, power, active mask, hw_slowdown, hw_thermal, sw_thermal, sw_power_cap
    "0, 1965, 1965, 640.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
    "1, 1200, 1965, 300.0, 0x0000000000000008, Active, Not Active, Not Active, Not Active",
    "0, 1890, 1965, 998.7, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
    "0, 1950, 1965, 990.2, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
]


def _clocks(tmp_path, rows):
    p = tmp_path / "clocks.csv"
    p.write_text("\n".join(rows) + "\n")
    return bench.Clocks(str(p))


def test_summary_takes_the_median_and_reasons_of_one_gpu(tmp_path):
    s = _clocks(tmp_path, ROWS).summary(0)
    assert s["samples"] == 3
    assert s["sm_mhz"] == 1950.0
    assert s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]


def test_summary_reports_a_hardware_slowdown_on_its_gpu(tmp_path):
    s = _clocks(tmp_path, ROWS).summary(1)
    assert s["samples"] == 1 and s["sm_mhz"] == 1200.0
    assert s["reasons"] == ["hw_slowdown"]


def test_summary_of_no_samples(tmp_path):
    s = _clocks(tmp_path, []).summary(0)
    assert s["samples"] == 0 and s["sm_mhz"] is None and s["reasons"] == []
