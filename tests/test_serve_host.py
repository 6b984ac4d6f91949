"""Host side of the serving stream (no GPU): the seeded graph specs, the
CSR builder, and the partitions the server receives."""
import numpy as np

from fastapsp_b200 import generators as G
from fastapsp_b200.graph import fapGraph


def test_serve_specs_are_seeded_and_in_range():
    a, b = G.serve_specs(), G.serve_specs()
    assert a == b and len(a) == 32
    for s in a:
        assert 16000 <= s["n"] <= 200000
        assert s["K"] in (16, 32, 64, 128, 256)
        assert 2.0 <= s["avg_degree"] <= 4.0
    assert G.serve_specs(seed=1) != a


def test_edges_to_csr_matches_dense_adjacency():
    el = G.random_geometric_graph(500, 3.0, seed=3)
    ro, col, w = G.edges_to_csr(el)
    assert ro[0] == 0 and ro[-1] == 2 * el.edges.shape[0] and np.all(np.diff(ro) >= 0)
    A = np.zeros((500, 500), np.float32)
    for (u, v), x in zip(el.edges.tolist(), el.weights.tolist()):
        A[u, v] = A[v, u] = x
    B = np.zeros_like(A)
    for u in range(500):
        for k in range(ro[u], ro[u + 1]):
            B[u, col[k]] = w[k]
    np.testing.assert_array_equal(A, B)


def test_serve_graph_partitions():
    spec = dict(name="t", n=3000, K=16, avg_degree=2.5, seed=5)
    spec2, ro, col, w = G.serve_graph_csr(spec)
    g = fapGraph.from_csr(spec["n"], int(ro[-1]), ro, col, w, spec["K"])
    g.preCondition()
    vn, vo, bn = g.partInfo()
    assert vn.shape[0] == 17 and vn[1:].sum() == 3000
    assert np.all(vo[1:] == np.concatenate([[0], np.cumsum(vn[1:])[:-1]]))
    assert np.all(bn[1:] <= vn[1:]) and bn[1:].sum() > 0
    assert sorted(g.getMapping().tolist()) == list(range(3000))
