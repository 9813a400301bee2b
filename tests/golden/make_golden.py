#!/usr/bin/env python3
"""Regenerates the golden fixtures in this directory FROM THE REFERENCE'S OWN
CODE, compiled by oracle/Makefile into oracle/_ref/:

  * <name>.gr                 the fixture graph (.gr v1, written by this
                              library's writer; byte layout of the reference's
                              SSSP/csr_graph.cu:302-418)
  * <name>.s<src>.i32         n int32 distances from the reference's int64
                              oracle, scripts/multigpu/supplement_graph.cpp
                              (oracle/_ref/supplement_graph, which also reads
                              the .gr back with its own validating reader)
  * manifest.json             per graph and source: the reference
                              sssp_sequential's total_work (SS/SSSP/main.cu:71),
                              reached count, max distance, sha256 of each file

The distances of the reference's int32 sssp_sequential
(oracle/_ref/libref_sssp.so) must equal the int64 oracle's; the script
stops otherwise.

Run from the repository root after `make -C oracle`:
    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from fixtures import golden_graphs  # noqa: E402
import oracle_lib  # noqa: E402

EXPORTER = os.path.join(ROOT, "oracle", "_ref", "supplement_graph")


def sha(path):
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def main():
    if not os.path.exists(EXPORTER) or oracle_lib.reference() is None:
        sys.exit("build the reference checkers first: make -C oracle")
    manifest = {}
    for name, (g, sources) in golden_graphs().items():
        gr = os.path.join(HERE, f"{name}.gr")
        g.write_gr(gr)
        entry = {"file": f"{name}.gr", "sha256": sha(gr), "n": g.n, "m": g.m, "sources": {}}
        for src in sources:
            out = os.path.join(HERE, f"{name}.s{src}.i32")
            with tempfile.TemporaryDirectory() as td:
                res = subprocess.run([EXPORTER, gr, str(src), str(g.n // 2),
                                      os.path.join(td, "gplus.gr"), out],
                                     capture_output=True, text=True)
            if res.returncode != 0:
                sys.exit(f"supplement_graph failed on {name} src {src}: {res.stderr}")
            d64 = np.fromfile(out, dtype=np.int32)
            d32, work = oracle_lib.ref_sequential(g, src)
            if not np.array_equal(d64, d32):
                sys.exit(f"{name} src {src}: reference int32 and int64 oracles disagree")
            finite = d64[d64 != oracle_lib.INT_MAX]
            entry["sources"][str(src)] = {
                "file": os.path.basename(out), "sha256": sha(out), "total_work": int(work),
                "reached": int(finite.size), "max_distance": int(finite.max()),
                "exporter": res.stdout.strip().splitlines(),
            }
            print(name, src, "reached", finite.size, "work", work)
        manifest[name] = entry
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
