"""Generates the mid-size golden fixtures in tests/golden/mid/ from the
reference itself (oracle/_ref/fap_ref, built from the reference sources by
`make -C oracle ref`):

    python tests/golden/make_golden_mid.py [name ...]

The graphs are the seeded benchmark workloads of fastapsp_b200.generators,
large enough that the automatic rules of the B200 path pick the forms the
small fixtures reach only when forced:
  road20k  (20,000 vertices, K=24, int32)   boundary graph closed by Floyd,
                                            thin min-plus (<= 16 boundary
                                            vertices per part)
  grid256  (65,536 vertices, K=64, int32)   boundary graph over 8,192
                                            boundary vertices: Bellman-Ford
                                            closure and tiled expansion;
                                            min-plus tiles (b > 16)
  rmat14   (16,384 vertices, K=16, float32) tiled multi-source Bellman-Ford
                                            SSSP (m >= 6n), directed
The partition is the one this library's host code computes (the reference's
METIS call on the same input for undirected graphs; for directed ones the
reference's METIS input is misaligned, so the same partition is given to
both); the reference binary runs with it (FAP_PARTITION_FILE) and the
fixture records it with the reference's renumbering (st2ed).  int32 cases
store the per-row checksums of every row (sum_j uint32(d[r][j]) * (2j+1)
mod 2^64, rows in st2ed order); the float32 case stores sampled rows whole
(the first and the last row of every part: a boundary and an inner row).
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

OUT = os.path.join(HERE, "mid")
CASES = ("road20k", "grid256", "rmat14")


def _run_part(job):
    root, name, directed, weighted, K, part, pfile, out_f, kind = job
    kw = {"rowsum_out": out_f} if kind == "rowsum" else {"dist_out": out_f}
    O.run_ref(root, name, directed, weighted, K, parts=[part], threads=1, partition_file=pfile, **kw)
    return part


def make(name, procs):
    from fastapsp_b200 import workloads
    wl = workloads.load(name)
    n, K = wl.n, wl.K
    gid = wl.graph.getGraphId()
    st2ed = wl.graph.getMapping()
    vn, vo, bn = wl.ver_num, wl.ver_offset, wl.bdy_num
    integral = bool(wl.edges.integral)
    with tempfile.TemporaryDirectory() as tmp:
        pfile = os.path.join(tmp, "partition.bin")
        (np.asarray(gid, np.int64) - 1).astype(np.int32).tofile(pfile)
        meta_f = os.path.join(tmp, "meta.bin")
        O.run_ref(wl.root, name, wl.edges.directed, wl.edges.weighted, K, parts="none",
                  meta_out=meta_f, partition_file=pfile)
        meta = O.read_meta(meta_f)
        assert np.array_equal(meta.st2ed, st2ed), "renumbering differs from the reference's"
        assert np.array_equal(meta.graph_id, gid)
        kind = "rowsum" if integral else "dist"
        jobs = [(wl.root, name, wl.edges.directed, wl.edges.weighted, K, p, pfile,
                 os.path.join(tmp, f"{kind}_{p}.bin"), kind) for p in range(1, K + 1)]
        with mp.get_context("spawn").Pool(procs) as pool:
            pool.map(_run_part, jobs, chunksize=1)
        out = dict(name=np.array(name), K=K, n=n, integral=integral, graph_id=gid, st2ed=st2ed,
                   ver_num=vn, ver_offset=vo, bdy_num=bn)
        if integral:
            out["row_checksums"] = np.concatenate(
                [np.fromfile(os.path.join(tmp, f"rowsum_{p}.bin"), np.uint64) for p in range(1, K + 1)])
        else:
            rows, dist = [], []
            for p in range(1, K + 1):
                blk = np.fromfile(os.path.join(tmp, f"dist_{p}.bin"), np.float32).reshape(-1, n)
                for r in (0, blk.shape[0] - 1):
                    rows.append(int(vo[p]) + r)
                    dist.append(blk[r])
            out["sample_rows"] = np.array(rows, np.int64)
            out["sample_dist"] = np.stack(dist)
    os.makedirs(OUT, exist_ok=True)
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **out)
    print(f"{name}: n={n} K={K} boundary={int(bn.sum())} integral={integral}")


if __name__ == "__main__":
    procs = max(1, min(os.cpu_count() or 1, 16))
    for name in sys.argv[1:] or CASES:
        make(name, procs)
