"""The tiled multi-source Bellman-Ford of stage 1 (msbf_seed_kernel /
msbf_iter_kernel), restated on the CPU and checked against exact shortest
distances on random graphs (no GPU needed).

Per iteration every vertex pulls over its in-arcs from the tails that
changed in the previous iteration (act_cur) and lowers its own row in place;
a vertex that improved joins act_next.  The work items run in a random
order and a tail row may be read as it was when the iteration began or as
another item has already lowered it (the GPU's concurrent warps may see
either); the host repeats iterations until one changes nothing.  Integer
weights, so every comparison is exact."""
import numpy as np
import pytest

INF = 10**8


def _msbf(n, u, v, w, sources, rng, max_iters=10_000):
    ins = [[] for _ in range(n)]                  # transposed CSR: in-arcs of every vertex
    for a, b, c in zip(u, v, w):
        ins[b].append((a, int(c)))
    S = len(sources)
    Dt = np.full((n, S), INF, np.int64)            # vertex-major tile
    act = np.zeros(n, bool)
    for s, x in enumerate(sources):                # seed
        Dt[x, s] = 0
        act[x] = True
    for _ in range(max_iters):
        nxt = np.zeros(n, bool)
        snap = Dt.copy()
        for x in rng.permutation(n):
            pull = [(a, c) for a, c in ins[x] if act[a]]
            if not pull:
                continue
            acc = np.full(S, INF, np.int64)
            for a, c in pull:
                src = snap if rng.random() < 0.5 else Dt
                acc = np.minimum(acc, np.minimum(src[a] + c, INF))
            if (acc < Dt[x]).any():                # atomic minima
                Dt[x] = np.minimum(Dt[x], acc)
                nxt[x] = True
        if not nxt.any():
            return Dt.T
        act = nxt
    raise AssertionError("did not converge")


@pytest.mark.parametrize("seed", range(10))
def test_tiled_bellman_ford_gives_the_exact_distances(seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(20, 80))
    m = int(rng.integers(n, 4 * n))
    u, v, w = rng.integers(0, n, m), rng.integers(0, n, m), rng.integers(0, 30, m)   # zero weights too
    keep = u != v
    u, v, w = u[keep], v[keep], w[keep]
    if seed % 2 == 0:
        u, v, w = np.concatenate([u, v]), np.concatenate([v, u]), np.concatenate([w, w])
    sources = rng.choice(n, size=min(n, 16), replace=False)
    got = _msbf(n, u, v, w, sources, rng)
    d = np.full((n, n), np.inf)
    for a, b, c in zip(u, v, w):
        d[a, b] = min(d[a, b], c)
    np.fill_diagonal(d, 0)
    # dense Dijkstra (a sparse matrix would drop the zero-weight arcs)
    want = np.full((len(sources), n), INF, np.int64)
    for i, s in enumerate(sources):
        dist = np.full(n, np.inf)
        dist[s] = 0
        done = np.zeros(n, bool)
        for _ in range(n):
            cand = np.where(done, np.inf, dist)
            x = int(np.argmin(cand))
            if not np.isfinite(cand[x]):
                break
            done[x] = True
            dist = np.minimum(dist, dist[x] + d[x])
        want[i] = np.where(np.isfinite(dist), dist, INF).astype(np.int64)
    np.testing.assert_array_equal(got, want)
