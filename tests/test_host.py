"""Host half of the drop-in fapGraph (no GPU needed): MatrixMarket reading,
METIS partition, boundary detection and renumbering must reproduce the
reference's CSR, graph_id and st2ed exactly (golden fixtures made by the
reference itself)."""
import ctypes
import os
import tempfile

import numpy as np
import pytest

from conftest import golden_names, load_golden, write_golden_mtx
from fastapsp_b200 import FapError, fapGraph
from fastapsp_b200 import _lib as L


def _host_graph(case, tmp):
    write_golden_mtx(case, tmp)
    g = fapGraph(case["name"], bool(case["directed"]), bool(case["weighted"]), int(case["K"]),
                 root=tmp)
    if case["injected_partition"]:
        gid0 = (np.arange(case["n"], dtype=np.int64) * case["K"] // case["n"]).astype(np.int32)
        g.setPartition(gid0 + 1)
    g.preCondition()
    return g


@pytest.mark.parametrize("name", golden_names())
def test_csr_partition_renumbering_match_reference(name):
    case = load_golden(name)
    with tempfile.TemporaryDirectory() as tmp:
        g = _host_graph(case, tmp)
        ro, col, w = g.csr()
        assert g.num_vertexs == case["n"]
        assert g.num_edges == case["m"]
        np.testing.assert_array_equal(ro, case["row_offset"])
        used = case["row_offset"][-1]
        np.testing.assert_array_equal(col, case["col_val"][:used])
        np.testing.assert_array_equal(w, case["weight"][:used])
        np.testing.assert_array_equal(g.getGraphId(), case["graph_id"])
        np.testing.assert_array_equal(g.getMapping(), case["st2ed"])
        vn, vo, bn = g.partInfo()
        np.testing.assert_array_equal(vn[1:], case["ver_num"][1:])
        np.testing.assert_array_equal(vo[1:], case["ver_offset"][1:])
        np.testing.assert_array_equal(bn[1:], case["bdy_num"][1:])
        assert g.isSplit() == (case["n"] > 20000)
        for p in range(1, case["K"] + 1):
            idx = g.getSubGraphIndex(p)
            np.testing.assert_array_equal(idx, case["st2ed"][vo[p]:vo[p] + vn[p]])


def test_metadata_constructor_matches_file_constructor():
    case = load_golden("road300_k6")
    with tempfile.TemporaryDirectory() as tmp:
        a = _host_graph(case, tmp)
    ro, col, w = a.csr()
    b = fapGraph.from_csr(case["n"], case["m"], ro, col, w, int(case["K"]))
    b.preCondition()
    np.testing.assert_array_equal(a.getGraphId(), b.getGraphId())
    np.testing.assert_array_equal(a.getMapping(), b.getMapping())


def test_missing_file_raises_io_error():
    with tempfile.TemporaryDirectory() as tmp:
        with pytest.raises(FapError) as e:
            fapGraph("nope", False, False, 4, root=tmp)
        assert e.value.code == L.FAP_ERR_IO


def test_bad_k_and_bad_partition():
    case = load_golden("grid12_k4")
    with tempfile.TemporaryDirectory() as tmp:
        write_golden_mtx(case, tmp)
        with pytest.raises(FapError):
            fapGraph(case["name"], False, False, 0, root=tmp)
        g = fapGraph(case["name"], False, False, 4, root=tmp)
        with pytest.raises(FapError):
            g.setPartition(np.zeros(case["n"], np.int32))      # ids must be 1..K
        with pytest.raises(FapError):
            g.setPartition(np.ones(case["n"] - 1, np.int32))   # wrong length


def test_malformed_mtx():
    with tempfile.TemporaryDirectory() as tmp:
        d = os.path.join(tmp, "graph", "unweight-undirected")
        os.makedirs(d)
        with open(os.path.join(d, "bad.mtx"), "w") as f:
            f.write("3 3 2\n1 2\n2 9\n")   # vertex 9 out of range
        with pytest.raises(FapError) as e:
            fapGraph("bad", False, False, 2, root=tmp)
        assert e.value.code == L.FAP_ERR_IO


def test_solve_before_precondition_is_an_error():
    case = load_golden("grid12_k4")
    with tempfile.TemporaryDirectory() as tmp:
        write_golden_mtx(case, tmp)
        g = fapGraph(case["name"], False, False, 4, root=tmp)
        with pytest.raises(FapError) as e:
            g.solveSubGraph(1)
        assert e.value.code == L.FAP_ERR_STATE


@pytest.mark.parametrize("name", ["grid12_k4", "road300_k6", "rmat8_f32_k4", "disconnected_k3"])
def test_binary_file_round_trip(name):
    """save() then load(): the same CSR, partition and, after preCondition,
    the same renumbering and part counts as the reference's, without text
    parsing or METIS; flags and sizes kept."""
    case = load_golden(name)
    with tempfile.TemporaryDirectory() as tmp:
        g = _host_graph(case, tmp)
        path = os.path.join(tmp, "g.fapb")
        g.save(path)
        h = fapGraph.load(path)
        assert (h.directed, h.weighted) == (bool(case["directed"]), bool(case["weighted"]))
        assert (h.num_vertexs, h.num_edges) == (g.num_vertexs, g.num_edges)
        h.preCondition()
        for a, b in zip(h.csr(), g.csr()):
            np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(h.getGraphId(), case["graph_id"])
        np.testing.assert_array_equal(h.getMapping(), case["st2ed"])
        for a, b in zip(h.partInfo(), g.partInfo()):
            np.testing.assert_array_equal(a, b)


def test_binary_file_damage_is_an_io_error():
    case = load_golden("grid12_k4")
    with tempfile.TemporaryDirectory() as tmp:
        g = _host_graph(case, tmp)
        path = os.path.join(tmp, "g.fapb")
        g.save(path)
        raw = bytearray(open(path, "rb").read())
        for damaged in (raw[:-9], raw[:40] + bytes([raw[40] ^ 1]) + raw[41:], b"NOTAFAPB" + raw[8:]):
            with open(path, "wb") as f:
                f.write(bytes(damaged))
            with pytest.raises(FapError) as e:
                fapGraph.load(path)
            assert e.value.code == L.FAP_ERR_IO
        with pytest.raises(FapError) as e:
            fapGraph.load(os.path.join(tmp, "missing.fapb"))
        assert e.value.code == L.FAP_ERR_IO


def _fnv1a64(data):
    h = 14695981039346656037
    for b in data:
        h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def test_binary_file_with_valid_checksum_but_bad_contents_is_an_io_error():
    """Files that pass the checksum are still checked: a declared edge
    count beyond int32 (no huge allocation), a column id past n, a part id
    past K."""
    case = load_golden("grid12_k4")
    with tempfile.TemporaryDirectory() as tmp:
        g = _host_graph(case, tmp)
        path = os.path.join(tmp, "g.fapb")
        g.save(path)
        raw = bytearray(open(path, "rb").read())
        n = int.from_bytes(raw[8:12], "little")
        nnz = int.from_bytes(raw[24:32], "little")
        cv_at = 40 + (n + 1) * 4
        gid_at = cv_at + 2 * nnz * 4
        edits = [(16, (1 << 40).to_bytes(8, "little")),        # m_decl
                 (cv_at, n.to_bytes(4, "little")),             # col_val[0] = n
                 (gid_at, (1000).to_bytes(4, "little"))]       # graph_id[0] > K
        for at, val in edits:
            body = bytearray(raw[:-8])
            body[at:at + len(val)] = val
            with open(path, "wb") as f:
                f.write(bytes(body) + _fnv1a64(body).to_bytes(8, "little"))
            with pytest.raises(FapError) as e:
                fapGraph.load(path)
            assert e.value.code == L.FAP_ERR_IO
        # the unedited body with its recomputed checksum still loads
        body = bytes(raw[:-8])
        with open(path, "wb") as f:
            f.write(body + _fnv1a64(body).to_bytes(8, "little"))
        assert fapGraph.load(path).num_vertexs == n


def test_host_wrappers_refuse_null_arguments():
    """Every C wrapper of fapGraph checks its pointers: NULL is
    FAP_ERR_INVALID with a message, never a crash (no GPU needed)."""
    lib = L.lib()
    calls = [
        lambda: lib.fap_host_sizes(None, None),
        lambda: lib.fap_host_csr(None, None, None, None),
        lambda: lib.fap_host_graph_id(None, None),
        lambda: lib.fap_host_mapping(None, None),
        lambda: lib.fap_host_parts(None, None, None, None),
        lambda: lib.fap_host_precondition(None),
        lambda: lib.fap_host_is_split(None),
        lambda: lib.fap_host_dtype(None),
        lambda: lib.fap_host_set_partition(None, None),
        lambda: lib.fap_host_set_options(None, 0, 0, 0),
        lambda: lib.fap_host_set_max_resident_rows(None, 0),
        lambda: lib.fap_host_solve(None, 0),
        lambda: lib.fap_host_solve_subgraph(None, 1, 0),
        lambda: lib.fap_host_current_subgraph(None),
        lambda: lib.fap_host_subgraph_distance(None, 1, None),
        lambda: lib.fap_host_all_distance(None, None),
        lambda: lib.fap_host_distance_from_one_point(None, 0, None),
        lambda: lib.fap_host_distance_p2p(None, 0, 0, None),
        lambda: lib.fap_host_subgraph_path(None, 1, None),
        lambda: lib.fap_host_all_path(None, None),
        lambda: lib.fap_host_path_from_one_point(None, 0, None),
        lambda: lib.fap_host_path_p2p(None, 0, 0, None, 0, None),
        lambda: lib.fap_host_check_result(None, 1, None),
        lambda: lib.fap_host_flags(None, None, None),
        lambda: lib.fap_host_save(None, None),
        lambda: lib.fap_host_load(None, None),
        lambda: lib.fap_host_from_mtx(None, 0, 0, 2, None),
        lambda: lib.fap_host_from_csr(4, 0, None, None, None, 2, 0, None),
    ]
    for i, call in enumerate(calls):
        assert call() == L.FAP_ERR_INVALID, i
        assert lib.fap_host_last_error()
    assert lib.fap_host_device_graph(None) is None
    out = ctypes.c_void_p()
    ro = np.zeros(1, np.int32)
    assert lib.fap_host_from_csr(0, 0, L.ptr(ro), None, None, 1, 0, ctypes.byref(out)) == L.FAP_ERR_INVALID
