"""The Floyd work queue's item list (built on the host, no GPU): the
persistent launch's CTAs claim items in list order and wait, bounded, for
an item's dependencies (per part: the diagonal closure of pivot block kb
after every remainder item of block kb - 1, the panels after the diagonal
closure, the remainder after every panel), so every dependency must come
earlier in the list and every item must be listed once.  Checked by the
library itself (fap_queue_order_check) for mixed part sizes, one-block
parts, partial last blocks, empty parts, symmetric and full items."""
import numpy as np
import pytest

from fastapsp_b200 import _lib as L
from fastapsp_b200._lib import ptr


def _check(sizes, sym):
    a = np.ascontiguousarray(sizes, dtype=np.int32)
    return L.lib().fap_queue_order_check(ptr(a), int(a.size), int(sym))


@pytest.mark.parametrize("sym", [0, 1])
def test_queue_order_keeps_dependencies(sym):
    rng = np.random.default_rng(3 + sym)
    cases = [
        [1], [128], [129], [900], [1024] * 3,
        [858, 895, 922, 900, 870],                     # road-shaped parts
        list(rng.integers(858, 923, 128)),             # the road114k batch
        list(rng.integers(1, 2500, 40)),               # mixed, partial last blocks
        list(rng.integers(1, 300, 200)),               # many one- and two-block parts
        [0, 500, 0, 129],                              # empty parts
    ]
    for sizes in cases:
        assert _check(sizes, sym) == L.FAP_OK, sizes


def test_queue_order_check_rejects_bad_arguments():
    assert _check([], 0) == L.FAP_OK
    assert L.lib().fap_queue_order_check(None, 1, 0) != L.FAP_OK
    assert _check([-1], 0) != L.FAP_OK
