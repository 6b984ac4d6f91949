"""Predecessor outputs of the reference's kernel ABI (fap/kernel/cuda/
cuda_kernel.h:21-42) as this library implements it (include/
fap_legacy_kernel.h).

CPU: the oracle's restatements of the reference's CPU kernels with
predecessors (floyd_CPU_path, min_plus_path_CPU_advanced, floyd_min_plus_CPU,
floyd_path_A_CPU, floyd_path_B_CPU) are pinned against those kernels compiled
from the reference sources (oracle/_ref/fap_kernels_ref), on inputs with many
ties.  The panels are computed out of place on the GPU (each entry from its
current value and predecessor, then the first strictly shorter candidate);
on the GPU test's inputs that rule gives what the reference's in-place CPU
panels give, which is checked here too.

GPU: every path-carrying legacy entry point against the restatement, bit for
bit (values and predecessors), including ties for the three entry points
whose order of candidates equals the reference's."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import oracle as O

INF = np.float32(1e8)
KREF = os.path.join(O.HERE, "_ref", "fap_kernels_ref")


def _kref(op, ints, arrays, outs):
    """Runs the reference's kernel `op` through oracle/_ref/fap_kernels_ref."""
    with tempfile.TemporaryDirectory() as tmp:
        fin, fout = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
        with open(fin, "wb") as f:
            f.write(np.asarray(ints, np.int32).tobytes())
            for a in arrays:
                f.write(np.ascontiguousarray(a).tobytes())
        subprocess.run([KREF, op, fin, fout], check=True)
        raw = np.fromfile(fout, np.uint8)
    res, o = [], 0
    for shape, dt in outs:
        nb = int(np.prod(shape)) * 4
        res.append(raw[o:o + nb].view(dt).reshape(shape))
        o += nb
    return res


def _dist(rng, r, c, p_inf, lo, hi):
    x = rng.integers(lo, hi, (r, c)).astype(np.float32)
    x[rng.random((r, c)) < p_inf] = INF
    return x


def _arc_and_path(rng, s, p_inf, lo, hi):
    """A sub-graph matrix the way the reference builds one
    (fap/utils/util_Myalgorithm.h:30-73): edge weights, diagonal 0, path =
    the row's vertex on edges and the diagonal, -1 elsewhere."""
    arc = _dist(rng, s, s, p_inf, lo, hi)
    np.fill_diagonal(arc, 0)
    path = np.where(arc < INF, np.arange(s, dtype=np.int32)[:, None], -1).astype(np.int32)
    return arc, path


def gpu_cases(seed=5):
    """Inputs of the GPU test: integer weights over a wide range, so that
    distinct paths have distinct lengths."""
    rng = np.random.default_rng(seed)
    lo, hi = 1, 100000
    c = {}
    c["floyd"] = _arc_and_path(rng, 90, 0.85, lo, hi)
    m, n, k = 45, 70, 19
    c["minplus"] = (_dist(rng, m, k, 0.3, lo, hi), _dist(rng, k, n, 0.3, lo, hi),
                    rng.integers(0, 1000, (k, n)).astype(np.int32))
    c["fmp"] = c["minplus"] + (_dist(rng, m, n, 0.3, lo, 3 * hi),
                               rng.integers(0, 1000, (m, n)).astype(np.int32))
    row, col = 37, 23
    dA, dpA = O.port_floyd_path(*_arc_and_path(rng, col, 0.6, lo, hi))
    c["path_A"] = (_dist(rng, row, col, 0.4, lo, hi), rng.integers(0, 1000, (row, col)).astype(np.int32),
                   dA, dpA)
    dB, dpB = O.port_floyd_path(*_arc_and_path(rng, row, 0.6, lo, hi))
    c["path_B"] = (_dist(rng, row, col, 0.4, lo, hi), rng.integers(0, 1000, (row, col)).astype(np.int32),
                   dB, dpB)
    return c


def panel_rule(which, x, xp, diag, diag_path):
    """The GPU's panel rule: out of place, each entry from its current value
    and predecessor, then the first strictly shorter candidate."""
    if which == "A":
        return O.port_minplus_path(x, diag, diag_path, x, xp)
    return O.port_minplus_path(diag, x, xp, x, xp)


needs_ref = pytest.mark.skipif(not os.path.exists(KREF), reason="reference kernels not built here")


@needs_ref
@pytest.mark.parametrize("seed", [1, 2])
def test_restated_path_kernels_match_the_reference(seed):
    """Small integer weights (many equal-length paths): the restatements give
    the reference kernels' values and predecessors exactly."""
    rng = np.random.default_rng(seed)
    arc, path = _arc_and_path(rng, 60, 0.8, 1, 6)
    want = _kref("floyd_path", [60], [arc, path], [((60, 60), np.float32), ((60, 60), np.int32)])
    got = O.port_floyd_path(arc, path)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    m, n, k = 23, 31, 17
    a, b = _dist(rng, m, k, 0.3, 0, 5), _dist(rng, k, n, 0.3, 0, 5)
    bp = rng.integers(0, 99, (k, n)).astype(np.int32)
    want = _kref("minplus_path", [m, n, k], [a, b, bp], [((m, n), np.float32), ((m, n), np.int32)])
    got = O.port_minplus_path(a, b, bp)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    c0, p0 = _dist(rng, m, n, 0.3, 0, 12), rng.integers(0, 99, (m, n)).astype(np.int32)
    want = _kref("floyd_min_plus", [m, n, k], [a, b, bp, c0, p0],
                 [((m, n), np.float32), ((m, n), np.int32)])
    got = O.port_minplus_path(a, b, bp, c0, p0)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    row, col = 19, 13
    for which, dn in (("A", col), ("B", row)):
        diag, dpath = O.port_floyd_path(*_arc_and_path(rng, dn, 0.5, 1, 6))
        x, xp = _dist(rng, row, col, 0.4, 0, 9), rng.integers(0, 99, (row, col)).astype(np.int32)
        want = _kref("path_" + which, [row, col], [x, xp, diag, dpath],
                     [((row, col), np.float32), ((row, col), np.int32)])
        got = O.port_floyd_path_panel(which, x, xp, diag, dpath)
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
        # values of the out-of-place rule equal the in-place reference's
        # even with ties (the diagonal block is closed)
        assert np.array_equal(panel_rule(which, x, xp, diag, dpath)[0], want[0])


def test_panel_rule_equals_the_reference_panels_on_the_gpu_inputs():
    """On the GPU test's inputs (distinct path lengths) the out-of-place
    panel rule gives the in-place reference panels' values and predecessors."""
    c = gpu_cases()
    for which in ("A", "B"):
        x, xp, diag, dpath = c["path_" + which]
        ref = O.port_floyd_path_panel(which, x, xp, diag, dpath)
        got = panel_rule(which, x, xp, diag, dpath)
        assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])


@pytest.mark.gpu
def test_legacy_abi_writes_the_reference_predecessors(cuda_ok):
    """floyd_GPU_Nvidia_path, minplus_NVIDIA_path, floyd_min_plus_Nvidia and
    the two panels with real path arrays, against the restatement of the
    reference's CPU kernels: values and predecessors bit for bit."""
    from fastapsp_b200 import _lib as L
    lib = L.lib()
    f = {k: getattr(lib, L.LEGACY_SYMBOLS[k]) for k in
         ("floyd_GPU_Nvidia_path", "minplus_NVIDIA_path", "floyd_min_plus_Nvidia", "floyd_path_A_Nvidia",
          "floyd_path_B_Nvidia")}
    c = gpu_cases()
    for lo_hi_seed in (None, 9):
        if lo_hi_seed is not None:
            # small weights: many ties, still exact for the Floyd pivots and
            # the two min-plus forms (same candidate order as the reference)
            rng = np.random.default_rng(lo_hi_seed)
            c["floyd"] = _arc_and_path(rng, 70, 0.7, 1, 4)
            m, n, k = 33, 57, 21
            c["minplus"] = (_dist(rng, m, k, 0.3, 0, 4), _dist(rng, k, n, 0.3, 0, 4),
                            rng.integers(0, 99, (k, n)).astype(np.int32))
            c["fmp"] = c["minplus"] + (_dist(rng, m, n, 0.3, 0, 8),
                                       rng.integers(0, 99, (m, n)).astype(np.int32))
        arc, path = (x.copy() for x in c["floyd"])
        want = O.port_floyd_path(arc, path)
        f["floyd_GPU_Nvidia_path"](arc.shape[0], L.ptr(arc), L.ptr(path))
        assert lib.fap_legacy_last_status() == 0
        assert np.array_equal(arc, want[0]) and np.array_equal(path, want[1])
        a, b, bp = c["minplus"]
        m, k = a.shape
        n = b.shape[1]
        res, rp = np.zeros((m, n), np.float32), np.zeros((m, n), np.int32)
        f["minplus_NVIDIA_path"](L.ptr(a), L.ptr(b), L.ptr(bp), L.ptr(res), L.ptr(rp), m, n, k)
        assert lib.fap_legacy_last_status() == 0
        want = O.port_minplus_path(a, b, bp)
        assert np.array_equal(res, want[0]) and np.array_equal(rp, want[1])
        a, b, bp, c0, p0 = c["fmp"]
        res, rp = c0.copy(), p0.copy()
        f["floyd_min_plus_Nvidia"](L.ptr(a), L.ptr(b), L.ptr(bp), L.ptr(res), L.ptr(rp), m, n, k)
        assert lib.fap_legacy_last_status() == 0
        want = O.port_minplus_path(a, b, bp, c0, p0)
        assert np.array_equal(res, want[0]) and np.array_equal(rp, want[1])
    for which in ("A", "B"):
        x, xp, diag, dpath = (v.copy() for v in c["path_" + which])
        row, col = x.shape
        want = O.port_floyd_path_panel(which, x, xp, diag, dpath)
        f["floyd_path_" + which + "_Nvidia"](L.ptr(x), L.ptr(xp), row, col, L.ptr(diag), L.ptr(dpath))
        assert lib.fap_legacy_last_status() == 0
        assert np.array_equal(x, want[0]) and np.array_equal(xp, want[1])
