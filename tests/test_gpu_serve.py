"""Serving loop (fap_server_*): every request's result is the same whether it
runs alone on a fresh server or mixed with other graphs' and other kinds of
requests, submitted from several threads, under a roomy or a tiny memory
budget (the tiny one leaves the largest graph without its resident cache, so
its requests take the uncached path); results also match the reference's
outputs (golden fixtures: rows of its solved blocks).  Tolerances as in the parity tests: int32 bit-exact,
float32 |d - ref| <= 1e-5 |ref| with reachability exact.
"""
import threading

import numpy as np
import pytest

from conftest import load_golden
from fastapsp_b200 import FapError
from fastapsp_b200 import _lib as L
from fastapsp_b200.serve import DONE, FAILED, REQ_SUBGRAPH, Server
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = ["grid64_k8", "road300_k6", "rmat8_f32_k4", "rmat8_int_k4"]


def _add(srv, case):
    return srv.add_csr(case["row_offset"], case["col_val"], case["weight"], int(case["K"]),
                       case["graph_id"], case["st2ed"], case["ver_num"], case["ver_offset"],
                       case["bdy_num"])


def _submit(srv, gi, req):
    kind, ids = req
    if kind == REQ_SUBGRAPH:
        return srv.submit_subgraph(gi, ids[0])
    return srv.submit_rows(gi, ids)


def _requests(cases, seed=5):
    rng = np.random.default_rng(seed)
    reqs = []
    for ci, c in enumerate(cases):
        for p in range(1, int(c["K"]) + 1):
            reqs += [(ci, (REQ_SUBGRAPH, (p,)))] * 2   # every part, twice
        for _ in range(3):
            k = int(rng.integers(1, 6))
            reqs.append((ci, (1, tuple(int(x) for x in rng.integers(0, int(c["n"]), k)))))
    return [reqs[i] for i in rng.permutation(len(reqs))]


def _alone(cases, reqs):
    out = {}
    for key in sorted(set(reqs)):
        ci, req = key
        with Server(0) as srv:
            gi = _add(srv, cases[ci])
            out[key] = np.array(_submit(srv, gi, req).result(timeout=120))
    return out


def _same(a, b):
    assert a.shape == b.shape
    np.testing.assert_array_equal(a.view(np.int32), b.view(np.int32))


def _check_against_reference(case, req, got):
    """Sub-graph blocks and distance rows against the reference's own output
    (rows of its solved blocks: full distances, or per-row checksums)."""
    kind, ids = req
    n = int(case["n"])
    integral = bool(case["integral"])
    if kind == REQ_SUBGRAPH:
        p = ids[0]
        off, rows = int(case["ver_offset"][p]), int(case["ver_num"][p])
        pos = np.arange(off, off + rows)
    else:
        ed2st = np.empty(n, np.int64)
        ed2st[case["st2ed"]] = np.arange(n)
        pos = ed2st[np.asarray(ids)]
    assert got.shape == (len(pos), n)
    if "dist" not in case:
        np.testing.assert_array_equal(O.row_checksums(O.to_i32(got)), case["row_checksums"][pos])
        return
    ref = np.asarray(case["dist"][pos], np.float32)
    if integral:
        _same(got, ref)
    else:
        reach = ref < 1e8
        assert np.array_equal(reach, got < 1e8)
        rel = np.abs(got[reach] - ref[reach]) / np.maximum(np.abs(ref[reach]), 1e-30)
        assert rel.max(initial=0.0) <= 1e-5


@pytest.fixture(scope="module")
def served():
    cases = [load_golden(n) for n in CASES]
    reqs = _requests(cases)
    return cases, reqs, _alone(cases, reqs)


def test_alone_results_match_reference(cuda_ok, served):
    cases, _, alone = served
    for (ci, req), got in alone.items():
        _check_against_reference(cases[ci], req, got)


@pytest.mark.parametrize("budget_mb,batch_bytes", [(0, 0), (24, 0), (0, 1)])
def test_same_alone_and_in_mix(cuda_ok, served, budget_mb, batch_bytes):
    """Requests of four graphs, both kinds, submitted in a shuffled order from
    three threads; budget 0 = default (roomy), 24 MB = room for about one
    part of the largest graph at a time (forces eviction and re-solves);
    batch_bytes 1 = one request per batch, 0 = the default cap."""
    cases, reqs, alone = served
    with Server(0, budget_bytes=budget_mb * 2**20) as srv:
        if batch_bytes:
            srv.set_option("max_batch_bytes", batch_bytes)
        gis = [_add(srv, c) for c in cases]
        handles = [None] * len(reqs)

        def client(idx):
            for i in idx:
                ci, req = reqs[i]
                handles[i] = _submit(srv, gis[ci], req)

        ths = [threading.Thread(target=client, args=(range(t, len(reqs), 3),)) for t in range(3)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        for i, h in enumerate(handles):
            _same(np.asarray(h.result(timeout=120)), alone[reqs[i]])
            info = h.info()
            assert info["status"] == L.FAP_OK and info["latency_ms"] >= 0
        srv.drain()
        st = srv.stats()
        assert st.completed == len(reqs) and st.failed == 0
        assert st.batches + st.resident_hits <= len(reqs)
        assert st.busy_ms > 0
        assert st.p99_ms >= st.p50_ms > 0
        if budget_mb:
            assert st.peak_bytes <= budget_mb * 2**20


def test_repeat_of_resident_block_is_not_recomputed(cuda_ok, served):
    cases, _, alone = served
    with Server(0) as srv:
        gi = _add(srv, cases[0])
        a = srv.submit_subgraph(gi, 3).result(timeout=120)
        b = srv.submit_subgraph(gi, 3).result(timeout=120)
        _same(a, b)
        _same(a, alone[(0, (REQ_SUBGRAPH, (3,)))])
        st = srv.stats()
        assert st.batches == 1 and st.resident_hits == 1 and st.cache_builds == 1


def test_invalid_requests_fail_cleanly(cuda_ok, served):
    cases, _, alone = served
    c = cases[1]
    with Server(0, budget_bytes=2 * 2**20) as srv:
        gi = _add(srv, c)
        with pytest.raises(FapError):
            srv.submit_subgraph(gi, 0)                      # parts are 1..K
        with pytest.raises(FapError):
            srv.submit_subgraph(gi, int(c["K"]) + 1)
        with pytest.raises(FapError):
            srv.submit_rows(gi, [int(c["n"])])              # vertex out of range
        with pytest.raises(FapError):
            srv.submit_subgraph(gi + 5, 1)                  # no such graph
        # a request larger than the whole budget fails, the server carries on
        big = srv.submit_rows(gi, list(range(int(c["n"]))) * 8)   # 5.8 MB > 2 MB
        assert big.wait(120) == FAILED
        assert big.info()["status"] == L.FAP_ERR_NOMEM
        ok = srv.submit_subgraph(gi, 2)
        assert ok.wait(120) == DONE
        _same(ok.out, alone[(1, (REQ_SUBGRAPH, (2,)))])
