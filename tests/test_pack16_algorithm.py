"""CPU restatement of the packed 16-bit min-plus (the int32 min-plus tiles
that run two relaxations per DPX instruction): columns of the boundary rows
are shifted by their least finite entry, every entry is clamped to 16383, the
halves are added and minimised as signed 16-bit values, and a result below
16383 is shifted back (16383 or more: no finite path).  When the part's
largest finite A plus the tile's largest shifted B is below 16383 this equals
the int32 min-plus exactly; the tests check that on random tiles at and just
under the bound, with unreachable entries, and that the bound is what the
bounds kernels compute."""
import numpy as np

INF = 100000000
CAP = 16383


def minplus_i32(A, B):
    s = A[:, :, None].astype(np.int64) + B[None, :, :].astype(np.int64)
    return np.minimum(s.min(axis=1), INF).astype(np.int32)


def bounds(A, B):
    fin_b = B < INF
    off = np.where(fin_b.any(0), np.where(fin_b, B, np.iinfo(np.int32).max).min(0), 0).astype(np.int32)
    hi = np.where(fin_b, B, 0).max(0)
    rng = np.where(fin_b.any(0), hi - off, 0)
    maxa = int(np.where(A < INF, A, 0).max(initial=0))
    return off, int(rng.max(initial=0)), maxa


def minplus_packed(A, B, off):
    """The packed form, element for element as the GPU computes it: wrapping
    16-bit adds of the clamped halves, signed 16-bit minimum from 32766."""
    a16 = np.minimum(A, CAP).astype(np.int16)
    b16 = np.where(B >= INF, CAP, np.minimum(B - off[None, :], CAP)).astype(np.int16)
    with np.errstate(over="ignore"):
        s = a16[:, :, None] + b16[None, :, :]          # int16 arithmetic (would wrap on overflow)
    r = np.minimum(s.min(axis=1), np.int16(32766)).astype(np.int32)
    return np.where(r < CAP, r + off[None, :], INF).astype(np.int32)


def _tile(rng, m, k, n, amax, brange, boff, p_inf):
    A = rng.integers(0, amax + 1, (m, k)).astype(np.int32)
    A[rng.random((m, k)) < p_inf] = INF
    base = rng.integers(0, boff + 1, n)
    B = (base[None, :] + rng.integers(0, brange + 1, (k, n))).astype(np.int32)
    B[rng.random((k, n)) < p_inf] = INF
    return A, B


def test_packed_equals_int32_when_the_bound_holds():
    rng = np.random.default_rng(3)
    for trial in range(40):
        m, k, n = rng.integers(1, 40), rng.integers(1, 70), rng.integers(1, 60)
        amax = int(rng.integers(0, 9000))
        brange = int(rng.integers(0, CAP - 1 - amax))
        A, B = _tile(rng, m, k, n, amax, brange, 10 ** 6, float(rng.choice([0.0, 0.2, 0.9, 1.0])))
        off, rg, maxa = bounds(A, B)
        assert maxa + rg < CAP
        np.testing.assert_array_equal(minplus_packed(A, B, off), minplus_i32(A, B))


def test_packed_at_the_edge_of_the_bound():
    """maxA + range = 16382: the largest finite sum sits right below the
    clamp of an unreachable entry."""
    rng = np.random.default_rng(4)
    m, k, n = 8, 5, 9
    A = np.full((m, k), 8000, np.int32)
    B = np.full((k, n), 500, np.int32)
    B[1, :] = 500 + (CAP - 1 - 8000)       # range 8382 in every column
    A[2, 3] = INF
    B[4, 2] = INF
    off, rg, maxa = bounds(A, B)
    assert maxa + rg == CAP - 1
    np.testing.assert_array_equal(minplus_packed(A, B, off), minplus_i32(A, B))
    # one more unit would break the proof: the bounds reject the tile
    B[1, 0] += 1
    off, rg, maxa = bounds(A, B)
    assert maxa + rg >= CAP


def test_columns_without_finite_entries():
    A = np.array([[0, 5], [INF, 7]], np.int32)
    B = np.array([[INF, 3], [INF, INF]], np.int32)
    off, rg, maxa = bounds(A, B)
    assert off[0] == 0 and rg == 0
    np.testing.assert_array_equal(minplus_packed(A, B, off), minplus_i32(A, B))
