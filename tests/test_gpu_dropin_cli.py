"""Drop-in proof: the reference's own CLI (SS/SSSP/main.cu and csr_graph.cu,
compiled unchanged by oracle/Makefile into oracle/_ref/mlmq_dropin) linked
against libmlmq_b200.so instead of the reference's sssp_run.cu.  The CLI
computes its own CPU Dijkstra, calls sssp_init / sssp_re_init /
sssp_run_adaptive / sssp_cp_data from this library, compares every vertex
and prints "mlmq sssp correct!" (exit 0) or exits 2 on a mismatch
(SS/SSSP/main.cu:236-238)."""
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CLI = os.path.join(HERE, "..", "oracle", "_ref", "mlmq_dropin")
GOLDEN = os.path.join(HERE, "golden")


def _cases():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        man = json.load(f)
    for name in ("supplement2052", "star2000", "grid64", "rmat11"):
        for src in sorted(man[name]["sources"], key=int):
            yield name, man[name]["file"], int(src)


@pytest.mark.skipif(not os.path.exists(CLI), reason="reference CLI not built (no reference tree)")
@pytest.mark.parametrize("name,gr,src", list(_cases()))
def test_reference_cli_reports_correct(name, gr, src):
    env = dict(os.environ, BENCH_SOURCE=str(src), BENCH_WARMUPS="0", BENCH_REPEATS="1")
    r = subprocess.run([CLI, "-i", os.path.join(GOLDEN, gr)], env=env, capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, (name, src, r.stdout[-2000:], r.stderr[-2000:])
    assert "mlmq sssp correct!" in r.stdout, (name, src, r.stdout[-2000:])
