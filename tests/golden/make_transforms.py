#!/usr/bin/env python3
"""Regenerates tests/golden/transforms.json FROM THE REFERENCE'S OWN CODE,
compiled by oracle/Makefile into oracle/_ref/:

  * BFS reordering: the reference's graph_transform/reorder_gr tool run on
    each fixture .gr from root 0 and from the fixture's last source; the
    digest covers the reordered CSR (read back with this library's .gr
    reader) and the perm / invperm sidecars.
  * Chain shortcuts G+: the reference's SSSP/l3/l3_chain_shortcuts.h builder
    (oracle/_ref/libref_chain.so) on each fixture with source = the fixture's
    first source, for cut = n (no partition) and cut = n / 2; the digest
    covers the augmented CSR, and the builder's counters are kept.

Digests are sha256 over the little-endian int32 bytes of row, col, w (and
perm, invperm), concatenated in that order.

Run from the repository root after `make -C oracle`:
    python tests/golden/make_transforms.py
"""
import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from fixtures import golden_graphs  # noqa: E402
import oracle_lib  # noqa: E402
from mlmq_tpds_withl3_b200 import HostGraph  # noqa: E402


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype="<i4").tobytes())
    return h.hexdigest()


def main():
    if not os.path.exists(oracle_lib.REORDER_BIN) or not os.path.exists(oracle_lib.CHAIN_SO):
        sys.exit("build the reference checkers first: make -C oracle")
    out = {}
    for name, (g, sources) in golden_graphs().items():
        gr = os.path.join(HERE, f"{name}.gr")
        entry = {"reorder": {}, "chain": {}}
        for root in sorted({0, int(sources[-1])}):
            with tempfile.TemporaryDirectory() as td:
                path, perm, inv = oracle_lib.ref_reorder_bfs(gr, root, td)
                r = HostGraph.read_gr(path)
                entry["reorder"][str(root)] = {
                    "sha256": digest(r.row, r.col, r.w, perm, inv), "m": int(r.m)}
        src = int(sources[0])
        for label, cut in (("n", g.n), ("half", g.n // 2)):
            row, col, w, st = oracle_lib.ref_chain_shortcuts(g, src, cut)
            entry["chain"][label] = {
                "source": src, "cut": int(cut), "sha256": digest(row, col, w), "m": int(len(col)),
                "stats": [int(x) for x in st]}
        out[name] = entry
        print(name, {k: v["m"] for k, v in entry["chain"].items()})
    with open(os.path.join(HERE, "transforms.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
