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
    # tile_pass2 on the 2001 x 1001 RCM wedge: 855.5 + 117.4 MB per launch (profiles/)
    assert bench.traffic_from_profiles("pass2", "fp64_rcm_2001x1001") == 972516352.0
    assert bench.traffic_from_profiles("pass2", "no_such_workload") is None


def test_aggregate_is_whole_job_throughput():
    # 4 ranks, 1e9 units each, slowest rank 500 ms
    assert bench.aggregate(1e9, 4, 500.0) == 8e9


def test_reference_arm_runs_the_reference_without_the_product_library():
    """bench.py --impl reference on a small wedge: one JSON line from the reference compiled
    unchanged, K timed steps after W warm-up steps, and no product library in the process."""
    import json
    import subprocess
    import sys
    import oracle as O
    if not O.RefSolver.available():
        import pytest
        pytest.skip("the reference library was not built here")
    code = ("import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--mesh', '41x21', '--steps', '3', "
            "'--warmup', '4']; import bench; bench.main(); maps = open('/proc/self/maps').read(); "
            "print(json.dumps({'product_loaded': 'libhcfd_gpu' in maps, 'ref_loaded': 'libhcfd_ref' in maps}))")
    out = subprocess.run([sys.executable, "-c", code], cwd=bench.ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    line, probe = (json.loads(x) for x in out.stdout.strip().splitlines()[-2:])
    assert probe == {"product_loaded": False, "ref_loaded": True}
    assert line["impl"] == "reference" and line["steps"] == 3 and line["warmup"] == 4
    assert "Barth-Jespersen, fixed dt" in line["config"]["workload"]
    assert line["value"] > 0 and line["e2e"]["h2d_bytes_per_step"] == 0
