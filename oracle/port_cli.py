"""Command-line driver of the C restatement (oracle/liboracle_port.so), with
the same arguments and JSON lines as oracle/_ref/fap_ref.  TEST
INFRASTRUCTURE ONLY: the CPU baseline when the reference binary is absent.

The graph's CSR, partition and renumbering come from the host half of the
drop-in fapGraph (MatrixMarket reader, METIS, sort_and_encode -- no GPU);
stages 1-3 are the restatement's.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from oracle import oracle as O  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dir", default=".")
    ap.add_argument("-f", required=True)
    ap.add_argument("-k", type=int, required=True)
    ap.add_argument("-direct", type=int, default=0)
    ap.add_argument("-weight", type=int, default=0)
    ap.add_argument("--parts", default="all")
    a = ap.parse_args()
    from fastapsp_b200.graph import fapGraph
    g = fapGraph(a.f, bool(a.direct), bool(a.weight), a.k, root=a.dir)
    g.preCondition()
    ro, col, w = g.csr()
    gid = g.getGraphId()
    st2ed = g.getMapping()
    ed2st = np.argsort(st2ed).astype(np.int32)
    vn, vo, bn = g.partInfo()
    n = g.num_vertexs
    parts = range(1, a.k + 1) if a.parts == "all" else [int(x) for x in a.parts.split(",")]
    for p in parts:
        t0 = time.perf_counter()
        O.port_run_part(ro, col, w, gid, st2ed, ed2st, int(vo[p]), int(vn[p]), int(bn[p]))
        t1 = time.perf_counter()
        print(json.dumps({"event": "part", "part": p, "rows": int(vn[p]), "bdy": int(bn[p]),
                          "entries": int(vn[p]) * n, "seconds": t1 - t0}), flush=True)


if __name__ == "__main__":
    main()
