"""bench.py's host-side helpers on the CPU: the clock record taken during the timed region
(median SM clock, max clock, throttle reasons that decide whether a run is kept), the DRAM
traffic read from the committed ncu summary, and the whole-job throughput."""
import io

import bench


class _Running:
    """Stands in for the nvidia-smi process."""


def _summary(text):
    c = bench.ClockSampler(0)
    c.proc = _Running()
    c.out = io.StringIO(text)
    return c.summary()


def test_clock_summary_median_max_and_reasons():
    lines = [
        "0, 1965, 1965, 612.40, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 998.10, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1920, 1965, 1001.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, [N/A], 1965, [N/A], [N/A], [N/A], [N/A], [N/A], [N/A]",     # a sample without readings
        "garbage",
    ]
    s = _summary("\n".join(lines) + "\n")
    assert s["sm_mhz"] == 1950.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 3
    assert s["reasons"] == ["sw_power_cap"]


def test_clock_summary_reports_slowdowns():
    lines = ["0, 1500, 1965, 700, 0x8, Active, Not Active, Active, Not Active"]
    assert _summary("\n".join(lines))["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]


def test_clock_summary_without_nvidia_smi():
    c = bench.ClockSampler(0)
    assert c.summary()["reasons"] == ["nvidia-smi unavailable"]


def test_traffic_of_the_committed_profile():
    # tile_pass2 on the 2001 x 1001 RCM wedge: 938.5 + 115.6 MB per launch (profiles/)
    assert bench.traffic_from_profiles("pass2", "fp64_rcm_2001x1001") == 1054147072.0
    assert bench.traffic_from_profiles("pass2", "no_such_workload") is None


def test_aggregate_is_whole_job_throughput():
    # 4 ranks, 1e9 units each, slowest rank 500 ms
    assert bench.aggregate(1e9, 4, 500.0) == 8e9
