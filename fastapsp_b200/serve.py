"""Serving loop over resident graphs (libfap_b200's fap_server_*).

A Server owns one device.  Graphs are added once; requests are submitted
from any thread and answered asynchronously by the native worker, which
batches each graph's pending sub-graph requests into one batched solve
(continuous batching), answers repeats of resident blocks without
recomputing, admits a batch only when its estimated device footprint fits
the memory budget, and runs each graph on its own stream.

    srv = Server(device=0)
    gi = srv.add_graph(g)                       # a preconditioned fapGraph
    req = srv.submit_subgraph(gi, part)         # what solveSubGraph computes
    dist = req.result()                         # (ver_num[part], n) float32

The reference answers one solveSubGraph call at a time on the caller's
thread (fap/fap.cpp:197-207); this loop has no counterpart there.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib as L
from ._lib import check, lib, ptr

REQ_SUBGRAPH = 0
REQ_ROWS = 1
PENDING, RUNNING, DONE, FAILED = 0, 1, 2, 3


@dataclass
class ServerStats:
    completed: int
    entries: int
    p50_ms: float
    p99_ms: float
    mean_ms: float
    peak_bytes: int
    batches: int
    resident_hits: int
    failed: int
    cache_builds: int
    busy_ms: float
    # longest single host call of the worker thread by kind, ms (HOST_STEPS)
    host_max_ms: dict = None


# Kinds of worker host calls timed by the server (fap_server_stats 11-18).
HOST_STEPS = ("launch", "complete", "cache_build", "admission", "reserve", "solve", "rows", "tail")


class Request:
    """One submitted request; keeps its host buffers alive until done."""

    def __init__(self, server: "Server", rid: int, ids: np.ndarray, out: Optional[np.ndarray],
                 checksums: Optional[np.ndarray]):
        self.server = server
        self.id = rid
        self._ids = ids
        self.out = out
        self.checksums = checksums

    def wait(self, timeout: float = -1.0) -> int:
        st = ctypes.c_int()
        check(lib().fap_server_wait(self.server._h, self.id, float(timeout), ctypes.byref(st)),
              "fap_server_wait")
        return int(st.value)

    def info(self) -> dict:
        v = np.zeros(4, np.float64)
        check(lib().fap_server_request_info(self.server._h, self.id, ptr(v)), "request_info")
        return {"latency_ms": float(v[0]), "queue_ms": float(v[1]), "entries": int(v[2]),
                "status": int(v[3])}

    def result(self, timeout: float = -1.0):
        """Waits, raises FapError if the request failed, returns the host
        distances (or the checksums when no distances were asked for)."""
        st = self.wait(timeout)
        if st == FAILED:
            code = self.info()["status"]
            raise L.FapError(code, f"request {self.id} failed with status {code}")
        if st != DONE:
            raise TimeoutError(f"request {self.id} not done after {timeout} s")
        return self.out if self.out is not None else self.checksums

    def forget(self) -> None:
        check(lib().fap_server_forget(self.server._h, self.id), "fap_server_forget")


class Server:
    def __init__(self, device: int = 0, budget_bytes: float = 0.0, max_batch_rows: int = 0):
        h = ctypes.c_void_p()
        check(lib().fap_server_create(int(device), float(budget_bytes), int(max_batch_rows),
                                      ctypes.byref(h)), "fap_server_create")
        self._h = h
        self._graphs = []  # (n, ver_num) per graph index

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and L._lib is not None:
            L._lib.fap_server_destroy(self._h)
        self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add_graph(self, g, dtype: Optional[int] = None) -> int:
        """Adds a preconditioned fapGraph (CSR + partition); returns its index."""
        ro, cv, w = g.csr()
        vn, vo, bn = g.partInfo()
        return self.add_csr(ro, cv, w, int(vn.shape[0] - 1), g.getGraphId(), g.getMapping(),
                            vn, vo, bn, g.dtype() if dtype is None else dtype)

    def add_csr(self, row_offset, col_val, weight, K: int, graph_id, st2ed, ver_num, ver_offset,
                bdy_num, dtype: int = L.FAP_DTYPE_AUTO) -> int:
        """Adds a graph from its CSR and partition arrays (fap_graph_set_parts'
        conventions); returns its index."""
        ro = L_i32(row_offset)
        m = int(ro[-1])
        cv = L_i32(col_val)[:m]
        w = np.ascontiguousarray(weight, np.float32)[:m]
        vn, vo, bn, gid, s2e = (L_i32(x) for x in (ver_num, ver_offset, bdy_num, graph_id, st2ed))
        n = int(ro.shape[0] - 1)
        idx = ctypes.c_int32()
        check(lib().fap_server_add_graph(self._h, n, m, ptr(ro), ptr(cv), ptr(w), int(dtype),
                                         int(K), ptr(gid), ptr(s2e), ptr(vn), ptr(vo), ptr(bn),
                                         ctypes.byref(idx)), "fap_server_add_graph")
        self._graphs.append((n, vn))
        return int(idx.value)

    def _meta(self, graph: int):
        if 0 <= graph < len(self._graphs):
            return self._graphs[graph]
        return 0, np.zeros(1, np.int32)   # unknown index: the library rejects the request

    def _submit(self, graph: int, kind: int, ids: np.ndarray, rows: int, distances: bool,
                checksums: bool) -> Request:
        n = self._meta(graph)[0]
        out = np.empty((rows, n), np.float32) if distances else None
        cs = np.empty(rows, np.uint64) if checksums else None
        rid = ctypes.c_int64()
        check(lib().fap_server_submit(self._h, int(graph), kind, ptr(ids), int(ids.shape[0]),
                                      ptr(out), ptr(cs), ctypes.byref(rid)), "fap_server_submit")
        return Request(self, int(rid.value), ids, out, cs)

    def submit_subgraph(self, graph: int, part: int, distances: bool = True,
                        checksums: bool = False) -> Request:
        """The ver_num[part] x n block of one part (rows in st2ed order)."""
        vn = self._meta(graph)[1]
        rows = int(vn[part]) if 1 <= part < vn.shape[0] else 0
        return self._submit(graph, REQ_SUBGRAPH, L_i32([part]), rows, distances, checksums)

    def submit_rows(self, graph: int, sources: Sequence[int], distances: bool = True,
                    checksums: bool = False) -> Request:
        """Shortest-distance rows from the given source vertices."""
        s = L_i32(np.asarray(sources).ravel())
        return self._submit(graph, REQ_ROWS, s, int(s.shape[0]), distances, checksums)

    def set_option(self, key: str, value: float) -> None:
        """"max_batch_bytes", "max_batch_rows" or "budget_bytes"."""
        check(lib().fap_server_set_option(self._h, key.encode(), float(value)), "set_option")

    def drain(self) -> None:
        check(lib().fap_server_drain(self._h), "fap_server_drain")

    def stats(self) -> ServerStats:
        v = np.zeros(19, np.float64)
        check(lib().fap_server_stats(self._h, ptr(v), 19), "fap_server_stats")
        host = dict(zip(HOST_STEPS, (float(x) for x in v[11:19])))
        return ServerStats(int(v[0]), int(v[1]), float(v[2]), float(v[3]), float(v[4]), int(v[5]),
                           int(v[6]), int(v[7]), int(v[8]), int(v[9]), float(v[10]), host)

    def reset_stats(self) -> None:
        check(lib().fap_server_reset_stats(self._h), "fap_server_reset_stats")


def L_i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a), dtype=np.int32)
