"""bench.py's host-side pieces on the CPU: the clock-sample summary that
decides whether a run is valid, the measured peak and ncu traffic lookups,
and the argument defaults the driver relies on."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _sampler(rows):
    s = bench.ClockSampler(0)
    s.out.write("".join(r + "\n" for r in rows))
    return s


def test_clock_summary_median_under_load_and_reasons():
    rows = ["0, 1965, 1965, 700.1, 98, Not Active, Not Active, Not Active, Not Active",
            "0, 1950, 1965, 900.0, 100, Not Active, Not Active, Not Active, Active",
            "0, 345, 1965, 90.0, 0, Not Active, Not Active, Not Active, Not Active",
            "0, 1965, 1965, 800.0, 100, Not Active, Not Active, Not Active, Not Active"]
    s = _sampler(rows).summary()
    assert s["sm_mhz"] == 1965.0          # idle sample (utilisation 0) left out
    assert s["sm_max_mhz"] == 1965.0 and s["samples"] == 4
    assert s["reasons"] == ["sw_power_cap"]


def test_clock_summary_flags_thermal_slowdown_and_empty_log():
    rows = ["0, 1500, 1965, 990.0, 100, Not Active, Active, Not Active, Active"]
    s = _sampler(rows).summary()
    assert s["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
    assert _sampler([]).summary() is None


def test_peak_and_traffic_lookups():
    peak, kind = bench.measured_peak()
    assert peak > 1000 and kind in ("measured", "fallback")
    t = bench.ncu_traffic("sssp_plain_kernel", "c2")
    assert t is None or t > 0
    assert bench.ncu_traffic("no_such_kernel", "c2") is None


def test_default_arguments(monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse()
    assert a.gpus == 1 and a.workload == "all" and a.impl != "reference"
    assert a.warmup >= 3 and a.steps >= 1 and a.skip == ""


def test_both_arms_print_the_same_workload_config():
    """The headline config holds workload keys only (solver settings go to
    "solver"), so the reference arm, which never tunes, prints the same dict."""
    from mlmq_tpds_withl3_b200 import HostGraph
    g = HostGraph.grid(16, 16, seed=2)
    a = bench.workload_config("c2", g, [0, 5], False)
    b = bench.workload_config("c2", g, [0, 5], False)
    assert a == b and set(a) == {"workload", "n", "m", "sources", "graph_sha256_16"}
    assert bench.workload_config("c2", g, [0, 5], True)["workload"].endswith("[scaled down: --small]")


def test_host_cpu_is_reported():
    h = bench.host_cpu()
    assert h["nproc"] >= 1 and isinstance(h["model"], str)
