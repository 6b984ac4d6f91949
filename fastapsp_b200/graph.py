"""Python mirror of the reference's fap::fapGraph (fap/fap.h:79-124) over the
C ABI of libfap_b200.so, plus thin handles for the device-resident graph and
the three stage operators.

    g = fapGraph("luxembourg_osm", directed=False, weighted=False, K=128, root=".")
    g.preCondition()
    if g.isSplit():
        g.solveSubGraph(1)
        block = g.getSubGraphDistance(1)      # ver_num[1] x n float32
    else:
        g.solve()
        dist = g.getAllDistance()             # n x n float32 (rows in st2ed order)

Names, argument meaning and error behaviour follow the reference; errors
raise FapError instead of exiting.
"""
from __future__ import annotations

import contextlib
import ctypes
import os
import threading
from typing import Iterable, Optional, Sequence

import numpy as np

from . import _lib as L
from ._lib import FapError, check, lib, ptr

_cwd_lock = threading.Lock()


@contextlib.contextmanager
def _in_dir(root: Optional[str]):
    if root is None:
        yield
        return
    with _cwd_lock:
        old = os.getcwd()
        os.chdir(root)
        try:
            yield
        finally:
            os.chdir(old)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


class fapGraph:
    """Drop-in mirror of fap::fapGraph.

    fapGraph(input_graph, directed, weighted, K, root=None) reads
    <root or cwd>/graph/<kind>/<input_graph>.mtx like the reference
    (fap/utils/readMatFile.h:43-51) and partitions it with METIS.
    fapGraph.from_csr(...) is the metadata constructor."""

    def __init__(self, input_graph: Optional[str] = None, directed: bool = False,
                 weighted: bool = False, K: int = 1, *, root: Optional[str] = None,
                 _handle=None):
        self._h = None
        if _handle is not None:
            self._h = _handle
        else:
            if input_graph is None:
                raise FapError(L.FAP_ERR_INVALID, "input_graph is required")
            h = ctypes.c_void_p()
            with _in_dir(root):
                rc = lib().fap_host_from_mtx(input_graph.encode(), int(directed), int(weighted),
                                             int(K), ctypes.byref(h))
            check(rc, "fapGraph")
            self._h = h
        self.directed = bool(directed)
        self.weighted = bool(weighted)
        self._mode = L.FAP_MODE_BATCHED
        self._dtype = L.FAP_DTYPE_AUTO
        self._device = 0

    def save(self, path: str) -> None:
        """Writes the graph and its partition to a binary file (fap_host_save)."""
        check(lib().fap_host_save(self._h, str(path).encode()), "fapGraph.save")

    @classmethod
    def load(cls, path: str) -> "fapGraph":
        """Rebuilds a graph saved by save() without text parsing or METIS;
        call preCondition() next (fap_host_load)."""
        h = ctypes.c_void_p()
        check(lib().fap_host_load(str(path).encode(), ctypes.byref(h)), "fapGraph.load")
        d, w = ctypes.c_int(), ctypes.c_int()
        check(lib().fap_host_flags(h, ctypes.byref(d), ctypes.byref(w)), "fapGraph.load")
        return cls(_handle=h, directed=bool(d.value), weighted=bool(w.value))

    @classmethod
    def from_csr(cls, num_vertexs: int, num_edges: int, row_offset, col_val, weight, K: int,
                 directed: bool = False) -> "fapGraph":
        ro = _i32(row_offset)
        cv = _i32(col_val)
        w = np.ascontiguousarray(weight, dtype=np.float32)
        h = ctypes.c_void_p()
        check(lib().fap_host_from_csr(int(num_vertexs), int(num_edges), ptr(ro), ptr(cv), ptr(w),
                                      int(K), int(directed), ctypes.byref(h)), "fapGraph.from_csr")
        g = cls(_handle=h, directed=directed, weighted=True)
        return g

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and L._lib is not None:
            L._lib.fap_host_destroy(h)
            self._h = None

    def close(self):
        self.__del__()

    # ---- options (not in the reference) ----
    def setPartition(self, graph_id_1based) -> None:
        gid = _i32(graph_id_1based)
        if gid.shape[0] != self.num_vertexs:
            raise FapError(L.FAP_ERR_PARTITION, "partition size != n")
        check(lib().fap_host_set_partition(self._h, ptr(gid)), "setPartition")

    def setOptions(self, *, device: Optional[int] = None, dtype: Optional[int] = None,
                   mode: Optional[int] = None) -> None:
        if device is not None:
            self._device = int(device)
        if dtype is not None:
            self._dtype = int(dtype)
        if mode is not None:
            self._mode = int(mode)
        check(lib().fap_host_set_options(self._h, self._device, self._dtype, self._mode),
              "setOptions")

    def setMode(self, mode: str) -> None:
        self.setOptions(mode=L.FAP_MODE_PLAIN if mode == "plain" else L.FAP_MODE_BATCHED)

    def setMaxResidentRows(self, rows: int) -> None:
        """At most `rows` output rows on the device (0 = no bound): solve and
        solveSubGraph then run the parts in groups whose rows fit, as they do
        when HBM cannot hold all n rows."""
        check(lib().fap_host_set_max_resident_rows(self._h, int(rows)), "setMaxResidentRows")

    # ---- sizes / CSR ----
    def _sizes(self):
        out = np.zeros(4, np.int64)
        check(lib().fap_host_sizes(self._h, ptr(out)))
        return out

    @property
    def num_vertexs(self) -> int:
        return int(self._sizes()[0])

    @property
    def num_edges(self) -> int:
        return int(self._sizes()[1])

    @property
    def K(self) -> int:
        return int(self._sizes()[2])

    def csr(self):
        n, _, _, used = (int(x) for x in self._sizes())
        ro = np.empty(n + 1, np.int32)
        col = np.empty(max(used, 1), np.int32)
        w = np.empty(max(used, 1), np.float32)
        check(lib().fap_host_csr(self._h, ptr(ro), ptr(col), ptr(w)))
        return ro, col[:used], w[:used]

    @property
    def row_offset(self):
        return self.csr()[0]

    @property
    def col_val(self):
        return self.csr()[1]

    @property
    def weight(self):
        return self.csr()[2]

    @property
    def adj_size(self):
        return np.diff(self.csr()[0]).astype(np.int32)

    # ---- reference API ----
    def preCondition(self) -> None:
        check(lib().fap_host_precondition(self._h), "preCondition")

    def isSplit(self) -> bool:
        return bool(lib().fap_host_is_split(self._h))

    def getGraphId(self) -> np.ndarray:
        out = np.empty(self.num_vertexs, np.int32)
        check(lib().fap_host_graph_id(self._h, ptr(out)))
        return out

    def getMapping(self) -> np.ndarray:
        out = np.empty(self.num_vertexs, np.int32)
        check(lib().fap_host_mapping(self._h, ptr(out)))
        return out

    def partInfo(self):
        """(ver_num, ver_offset, bdy_num), each K+1 entries, index 1..K."""
        K = self.K
        vn, vo, bn = (np.zeros(K + 1, np.int32) for _ in range(3))
        check(lib().fap_host_parts(self._h, ptr(vn), ptr(vo), ptr(bn)))
        return vn, vo, bn

    def dtype(self) -> int:
        rc = lib().fap_host_dtype(self._h)
        if rc < 0:
            check(rc, "dtype")
        return rc

    def solve(self, is_path_needed: bool = False) -> int:
        check(lib().fap_host_solve(self._h, int(is_path_needed)), "solve")
        return 0

    def solveSubGraph(self, sub_graph_id: int, is_path_needed: bool = False) -> int:
        check(lib().fap_host_solve_subgraph(self._h, int(sub_graph_id), int(is_path_needed)),
              "solveSubGraph")
        return 0

    def getAllDistance(self) -> np.ndarray:
        n = self.num_vertexs
        out = np.empty((n, n), np.float32)
        check(lib().fap_host_all_distance(self._h, ptr(out)), "getAllDistance")
        return out

    def getCurrentSubGraphId(self) -> int:
        return int(lib().fap_host_current_subgraph(self._h))

    def getSubGraphIndex(self, sub_graph_id: int) -> np.ndarray:
        vn, vo, _ = self.partInfo()
        m = self.getMapping()
        return m[vo[sub_graph_id]:vo[sub_graph_id] + vn[sub_graph_id]].copy()

    def getSubGraphDistance(self, sub_graph_id: int) -> np.ndarray:
        vn, _, _ = self.partInfo()
        out = np.empty((int(vn[sub_graph_id]), self.num_vertexs), np.float32)
        check(lib().fap_host_subgraph_distance(self._h, int(sub_graph_id), ptr(out)),
              "getSubGraphDistance")
        return out

    def getDistanceFromOnePoint(self, vertex_id: int) -> np.ndarray:
        out = np.empty(self.num_vertexs, np.float32)
        check(lib().fap_host_distance_from_one_point(self._h, int(vertex_id), ptr(out)),
              "getDistanceFromOnePoint")
        return out

    def getDistanceP2P(self, u: int, v: int) -> float:
        x = ctypes.c_float()
        check(lib().fap_host_distance_p2p(self._h, int(u), int(v), ctypes.byref(x)),
              "getDistanceP2P")
        return float(x.value)

    # ---- predecessor (path) matrices: solve(..., is_path_needed=True) ----
    def getAllPath(self) -> np.ndarray:
        n = self.num_vertexs
        out = np.empty((n, n), np.int32)
        check(lib().fap_host_all_path(self._h, ptr(out)), "getAllPath")
        return out

    def getSubGraphPath(self, sub_graph_id: int) -> np.ndarray:
        vn, _, _ = self.partInfo()
        out = np.empty((int(vn[sub_graph_id]), self.num_vertexs), np.int32)
        check(lib().fap_host_subgraph_path(self._h, int(sub_graph_id), ptr(out)), "getSubGraphPath")
        return out

    def getPathFromOnePoint(self, vertex_id: int) -> np.ndarray:
        out = np.empty(self.num_vertexs, np.int32)
        check(lib().fap_host_path_from_one_point(self._h, int(vertex_id), ptr(out)),
              "getPathFromOnePoint")
        return out

    def getPathP2P(self, u: int, v: int) -> list:
        """Vertices of a shortest path u .. v (inclusive); [] if unreachable."""
        out = np.empty(self.num_vertexs + 1, np.int32)
        ln = ctypes.c_int32()
        check(lib().fap_host_path_p2p(self._h, int(u), int(v), ptr(out), int(out.shape[0]),
                                      ctypes.byref(ln)), "getPathP2P")
        return out[:ln.value].tolist()

    def check_result(self, sub_graph_id: Optional[int] = None) -> bool:
        """Sampled self-check of the current part (fap/utils/checkResult.h:38-82)."""
        pid = self.getCurrentSubGraphId() if sub_graph_id is None else int(sub_graph_id)
        ok = ctypes.c_int()
        check(lib().fap_host_check_result(self._h, pid, ctypes.byref(ok)), "check_result")
        return bool(ok.value)

    def device_graph(self) -> "DeviceGraph":
        """The device-resident graph behind this object (after the first solve)."""
        p = lib().fap_host_device_graph(self._h)
        if not p:
            raise FapError(L.FAP_ERR_STATE, "no device graph before the first solve")
        return DeviceGraph._borrow(p, self)


class Context:
    """One CUDA device + stream (fap_ctx)."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        check(lib().fap_ctx_create(int(device), ctypes.byref(h)), "fap_ctx_create")
        self._h = h
        self.device = device

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and L._lib is not None:
            L._lib.fap_ctx_destroy(h)
            self._h = None

    def set_stream(self, stream_handle: int) -> None:
        check(lib().fap_ctx_set_stream(self._h, ctypes.c_void_p(stream_handle)))

    def use_torch_stream(self) -> None:
        """Run on torch's current stream, switching torch to a dedicated
        stream first when the current one is the legacy default stream (the
        library's calls and torch's events must share one stream)."""
        import torch
        s = torch.cuda.current_stream(self.device)
        if s.cuda_stream == 0:
            s = torch.cuda.Stream(self.device)
            torch.cuda.set_stream(s)
        self._torch_stream = s
        self.set_stream(s.cuda_stream)

    def sync(self) -> None:
        check(lib().fap_ctx_sync(self._h))

    def relax_peak(self, dtype: int = L.FAP_DTYPE_I32) -> float:
        x = ctypes.c_double()
        check(lib().fap_measure_relax_peak(self._h, int(dtype), ctypes.byref(x)), "relax_peak")
        return float(x.value)

    # ---- stage operators on device tensors (torch) ----
    def sssp(self, row_offset, col_val, weight, sources, out, dtype: int) -> None:
        n = int(row_offset.shape[0]) - 1
        m = int(col_val.shape[0])
        check(lib().fap_op_sssp(self._h, dtype, n, m, ptr(row_offset), ptr(col_val), ptr(weight),
                                ptr(sources), int(sources.shape[0]), ptr(out), int(out.stride(0))),
              "fap_op_sssp")

    def floyd(self, mat, dtype: int) -> None:
        check(lib().fap_op_floyd(self._h, dtype, int(mat.shape[0]), ptr(mat), int(mat.stride(0))),
              "fap_op_floyd")

    def minplus(self, A, B, C, dtype: int) -> None:
        M, K = int(A.shape[0]), int(A.shape[1])
        N = int(B.shape[1])
        check(lib().fap_op_minplus(self._h, dtype, M, N, K, ptr(A), int(A.stride(0)), ptr(B),
                                   int(B.stride(0)), ptr(C), int(C.stride(0))), "fap_op_minplus")


class DeviceGraph:
    """Device-resident CSR + partition + output (fap_dgraph)."""

    def __init__(self, ctx: Context, row_offset, col_val, weight, dtype: int = L.FAP_DTYPE_AUTO):
        self.ctx = ctx
        ro = _i32(row_offset)
        cv = _i32(col_val)
        w = np.ascontiguousarray(weight, dtype=np.float32)
        n = ro.shape[0] - 1
        h = ctypes.c_void_p()
        check(lib().fap_graph_create(ctx._h, int(n), int(ro[-1]), ptr(ro), ptr(cv), ptr(w),
                                     int(dtype), ctypes.byref(h)), "fap_graph_create")
        self._h = h
        self._owned = True
        self.n = int(n)
        self._vn = None

    @classmethod
    def _borrow(cls, handle, owner) -> "DeviceGraph":
        self = cls.__new__(cls)
        self._h = ctypes.c_void_p(handle)
        self._owned = False
        self._owner = owner
        self.ctx = None
        self.n = owner.num_vertexs
        vn, _, _ = owner.partInfo()
        self._vn = vn
        return self

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and getattr(self, "_owned", False) and L._lib is not None:
            L._lib.fap_graph_destroy(h)
            self._h = None

    @property
    def dtype(self) -> int:
        return int(lib().fap_graph_dtype(self._h))

    def set_parts(self, K: int, graph_id, st2ed, ver_num, ver_offset, bdy_num) -> None:
        args = [_i32(x) for x in (graph_id, st2ed, ver_num, ver_offset, bdy_num)]
        check(lib().fap_graph_set_parts(self._h, int(K), *[ptr(a) for a in args]),
              "fap_graph_set_parts")
        self._vn = args[2]

    def set_param(self, key: str, value: float) -> None:
        check(lib().fap_graph_set_param(self._h, key.encode(), float(value)), "set_param")

    def mean_weight(self) -> float:
        return float(lib().fap_graph_mean_weight(self._h))

    def tune_sssp(self, deltas: Sequence[float], sample: int = 0):
        """Times the SSSP stage for each candidate bucket width and keeps the
        fastest; returns (best_delta, ms per candidate)."""
        d = np.ascontiguousarray(deltas, dtype=np.float64)
        ms = np.zeros(d.shape[0], np.float32)
        best = ctypes.c_double()
        check(lib().fap_graph_tune_sssp(self._h, ptr(d), int(d.shape[0]), int(sample),
                                        ctypes.byref(best), ptr(ms)), "tune_sssp")
        return float(best.value), ms

    def reserve(self, max_rows: int = 0) -> None:
        check(lib().fap_graph_reserve(self._h, int(max_rows)), "fap_graph_reserve")

    def solve(self, parts: Optional[Iterable[int]] = None, mode: int = L.FAP_MODE_BATCHED,
              check_errors: bool = True) -> None:
        if parts is None:
            rc = lib().fap_solve(self._h, None, 0, int(mode))
        else:
            ids = _i32(list(parts))
            rc = lib().fap_solve(self._h, ptr(ids), int(ids.shape[0]), int(mode))
        check(rc, "fap_solve")
        if check_errors:
            self.check()

    def check(self) -> None:
        check(lib().fap_graph_check(self._h), "fap_graph_check")

    def block_info(self, part: int):
        p = ctypes.c_void_p()
        rows = ctypes.c_int64()
        ld = ctypes.c_int64()
        check(lib().fap_graph_block(self._h, int(part), ctypes.byref(p), ctypes.byref(rows),
                                    ctypes.byref(ld)), "fap_graph_block")
        return int(p.value or 0), int(rows.value), int(ld.value)

    def copy_block(self, part: int, out_dtype: Optional[int] = None, out=None) -> np.ndarray:
        dt = self.dtype if out_dtype is None else out_dtype
        _, rows, _ = self.block_info(part)
        if out is None:
            out = np.empty((rows, self.n), np.int32 if dt == L.FAP_DTYPE_I32 else np.float32)
        check(lib().fap_graph_copy_block(self._h, int(part), ptr(out), int(dt)),
              "fap_graph_copy_block")
        return out

    def copy_block_async(self, part: int, out, slot: int, out_dtype: Optional[int] = None) -> None:
        """Queues the copy of part's block into `out` (rows x n, contiguous;
        pinned for the full rate) on copy slot 0 or 1 without waiting for
        it; `out` must stay alive until copy_wait(slot) or the slot's next
        copy (fap_graph_copy_block_async)."""
        dt = self.dtype if out_dtype is None else out_dtype
        _, rows, _ = self.block_info(part)
        want = np.int32 if dt == L.FAP_DTYPE_I32 else np.float32
        if out.dtype != want or out.shape != (rows, self.n) or not out.flags.c_contiguous:
            raise ValueError(f"out must be a contiguous {rows} x {self.n} {np.dtype(want).name} array")
        check(lib().fap_graph_copy_block_async(self._h, int(part), ptr(out), int(dt), int(slot)),
              "fap_graph_copy_block_async")

    def copy_wait(self, slot: int) -> None:
        check(lib().fap_graph_copy_wait(self._h, int(slot)), "fap_graph_copy_wait")

    def copy_path_block(self, part: int) -> np.ndarray:
        """rows x n int32 predecessors of a part solved with set_param("paths", 1)."""
        _, rows, _ = self.block_info(part)
        out = np.empty((rows, self.n), np.int32)
        check(lib().fap_graph_copy_path_block(self._h, int(part), ptr(out)), "copy_path_block")
        return out

    def block_checksums(self, part: int) -> np.ndarray:
        _, rows, _ = self.block_info(part)
        out = np.empty(rows, np.uint64)
        check(lib().fap_graph_block_checksums(self._h, int(part), ptr(out)), "checksums")
        return out

    def cache_build(self, rebuild: bool = False) -> None:
        """Builds the resident cache (every part's boundary rows and closed
        Floyd matrix); later batched solves and rows() use it.  rebuild:
        compute it again in the same buffers even when it exists."""
        if rebuild:
            check(lib().fap_graph_cache_rebuild(self._h), "fap_graph_cache_rebuild")
        else:
            check(lib().fap_graph_cache_build(self._h), "fap_graph_cache_build")

    def cache_timing(self) -> list:
        """Device ms of the last cache build's four phases (fap_graph_cache_timing)."""
        out = np.zeros(4, np.float32)
        check(lib().fap_graph_cache_timing(self._h, ptr(out)), "fap_graph_cache_timing")
        return [float(x) for x in out]

    def cache_release(self) -> None:
        check(lib().fap_graph_cache_release(self._h), "fap_graph_cache_release")

    def cache_bytes(self):
        """(bytes, built): what the cache holds, or would need if not built."""
        b = ctypes.c_int64()
        built = ctypes.c_int()
        check(lib().fap_graph_cache_bytes(self._h, ctypes.byref(b), ctypes.byref(built)),
              "fap_graph_cache_bytes")
        return int(b.value), bool(built.value)

    def device_bytes(self) -> int:
        b = ctypes.c_int64()
        check(lib().fap_graph_device_bytes(self._h, ctypes.byref(b)), "fap_graph_device_bytes")
        return int(b.value)

    def release(self) -> None:
        check(lib().fap_graph_release(self._h), "fap_graph_release")

    def rows(self, sources: Sequence[int]) -> np.ndarray:
        """Distance rows (float32) through fap_graph_rows_async: from the
        resident cache when it is built, else by SSSP."""
        import torch
        s = _i32(list(sources))
        out = torch.empty((s.shape[0], self.n), dtype=torch.float32, device="cuda")
        check(lib().fap_graph_rows_async(self._h, ptr(s), int(s.shape[0]), ptr(out)),
              "fap_graph_rows_async")
        self.check()
        return out.cpu().numpy()

    def sssp_rows(self, sources: Sequence[int]) -> np.ndarray:
        s = _i32(list(sources))
        out = np.empty((s.shape[0], self.n), np.float32)
        check(lib().fap_graph_sssp_rows(self._h, ptr(s), int(s.shape[0]), ptr(out)), "sssp_rows")
        return out

    def last_timing(self) -> np.ndarray:
        t = np.zeros(5, np.float32)
        check(lib().fap_graph_last_timing(self._h, ptr(t)), "last_timing")
        return t

    def last_stage1(self) -> int:
        """1 SSSP, 2 boundary graph, 3 resident cache (see fap_graph_last_stage1)."""
        return int(lib().fap_graph_last_stage1(self._h))

    def pack16_tiles(self):
        """(min-plus tiles run in the packed 16-bit form, tiles run) over
        every solve of this graph so far."""
        a, b = ctypes.c_int64(), ctypes.c_int64()
        check(lib().fap_graph_pack16_tiles(self._h, ctypes.byref(a), ctypes.byref(b)), "pack16_tiles")
        return int(a.value), int(b.value)

    def shard_begin(self, own_parts, send_ptr: int, send_cap: int) -> int:
        """Sharded boundary-graph form, step 1 (fap_graph_shard_begin): local
        closures of this rank's parts; their boundary rows packed into the
        device buffer at send_ptr (send_cap elements of the graph's dtype).
        Returns the element count written."""
        ids = _i32(list(own_parts))
        out = ctypes.c_int64()
        check(lib().fap_graph_shard_begin(self._h, ptr(ids), int(ids.shape[0]), ctypes.c_void_p(send_ptr),
                                          int(send_cap), ctypes.byref(out)), "fap_graph_shard_begin")
        return int(out.value)

    def shard_finish(self, recv_ptr: int, world: int, owner, stride: int) -> None:
        """Step 2 (fap_graph_shard_finish): every rank's packed rows at
        recv_ptr (rank r's at r * stride elements), owner[p] = rank of part p
        (index 0 unused).  Leaves this rank's parts in the resident cache."""
        own = _i32(owner)
        check(lib().fap_graph_shard_finish(self._h, ctypes.c_void_p(recv_ptr), int(world), ptr(own),
                                           int(stride)), "fap_graph_shard_finish")

    def expand16_tiles(self):
        """(tiles of the boundary graph's tiled expansion run in the packed
        16-bit form, tiles run) over every solve and cache build so far."""
        a, b = ctypes.c_int64(), ctypes.c_int64()
        check(lib().fap_graph_expand16_tiles(self._h, ctypes.byref(a), ctypes.byref(b)), "expand16_tiles")
        return int(a.value), int(b.value)

    def stage1_name(self) -> str:
        """How stage 1 of the last solve ran, in words (fap_graph_stage1_name)."""
        return (lib().fap_graph_stage1_name(self._h) or b"").decode()

    def last_launches(self) -> int:
        x = ctypes.c_int64()
        check(lib().fap_graph_last_launches(self._h, ctypes.byref(x)))
        return int(x.value)
