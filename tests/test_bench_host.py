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
    t, _ = bench.ncu_traffic("sssp_plain_kernel", "c2")
    assert t is None or t > 0
    assert bench.ncu_traffic("no_such_kernel", "c2") == (None, None)


def test_traffic_lookup_takes_the_capture_at_the_nearest_delta(tmp_path, monkeypatch):
    (tmp_path / "profiles").mkdir()
    (tmp_path / "profiles" / "ncu_traffic.txt").write_text(
        "# comment\n"
        "k w 100 delta=50000\n"
        "k w 300 delta=200000\n"
        "k2 w 7\n")
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.ncu_traffic("k", "w", 55389) == (100.0, 50000)
    assert bench.ncu_traffic("k", "w", 221558) == (300.0, 200000)
    assert bench.ncu_traffic("k", "w") == (100.0, 50000)
    assert bench.ncu_traffic("k2", "w", 12345) == (7.0, None)


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


@pytest.mark.parametrize("name", ["c1", "c2", "c3"])
def test_reference_arm_builds_the_same_workload_without_the_product(name, monkeypatch):
    """The reference arm's graph (oracle/workload.c) and sources equal the GPU
    arm's (mlmq_tpds_withl3_b200.workloads), on the scaled-down workloads."""
    from mlmq_tpds_withl3_b200 import workloads
    args = bench.parse(["--workload", name, "--small"])
    rname, rg, rsrcs = bench.reference_workload(args)
    gname, gg, gsrcs = bench.headline_workload(args)
    assert rname == gname == name
    assert bench.workload_config(name, rg, rsrcs, True) == bench.workload_config(name, gg, gsrcs, True)


def test_reference_arm_does_not_load_the_product_library():
    """bench.py --impl reference in a fresh process maps oracle libraries
    only (checked through /proc/self/maps at the end of a tiny run)."""
    import subprocess
    code = ("import sys, runpy; sys.argv=['bench.py','--impl','reference','--workload','c1',"
            "'--steps','1','--warmup','0'];"
            "import bench; bench.main();"
            "maps=open('/proc/self/maps').read();"
            "print('PRODUCT' if 'libmlmq_b200' in maps else 'CLEAN')")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip().splitlines()[-1] == "CLEAN"
    line = __import__("json").loads(out.stdout.strip().splitlines()[0])
    assert line["impl"] == "reference" and line["config"]["n"] == 512 * 512
