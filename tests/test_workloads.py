"""The benchmark workloads and their profiling stand-ins (no GPU needed):
seeded, with the shapes the stand-ins are meant to share with the full
configurations (part sizes, boundary sets above or below the 8,192 vertices
where the boundary graph switches from Floyd to Bellman-Ford, degrees)."""
import numpy as np
import pytest

from fastapsp_b200 import workloads
from fastapsp_b200 import generators as G


def _shape(name):
    wl = workloads.load(name)
    d = wl.describe()
    return wl, d


@pytest.mark.parametrize("name", ["grid64", "grid128", "grid256", "road20k", "rmat14"])
def test_small_workloads_have_their_documented_shape(name):
    wl, d = _shape(name)
    assert d["n"] == wl.n and d["K"] == wl.K
    vn, bn = wl.ver_num[1:], wl.bdy_num[1:]
    assert int(vn.sum()) == wl.n and np.all(bn <= vn)
    if name in ("grid128", "grid256", "rmat14"):
        # about 1,024 vertices per part, like grid512 and rmat16
        assert 900 <= int(np.median(vn)) <= 1100
    if name == "grid256":
        assert int(bn.sum()) > 8192      # the Bellman-Ford closure of the boundary graph
    if name == "grid128":
        assert 16 < int(np.median(bn)) and int(bn.sum()) <= 8192   # thick parts, Floyd closure
    if name == "rmat14":
        assert d["arcs"] >= 6 * d["n"]   # the tiled SSSP form


def test_workloads_are_seeded():
    a = G.WORKLOADS["grid128"]["make"]()
    b = G.WORKLOADS["grid128"]["make"]()
    for x, y in zip(G.edges_to_csr(a), G.edges_to_csr(b)):
        np.testing.assert_array_equal(x, y)
