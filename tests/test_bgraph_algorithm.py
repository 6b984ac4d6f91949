"""The boundary-graph form of stage 1, restated step by step on the CPU and
checked against plain all-pairs shortest paths on random graphs (no GPU
needed).  This pins the algorithm the GPU kernels follow:

  local closures F_p (Floyd over each part's own arcs);
  the boundary graph closed by alternating steps (bgraph_lstep_kernel /
  bgraph_xstep_kernel): a local step over the rows the last cross step
  changed, a cross step over the heads whose tails changed, repeated until a
  cross step changes nothing, with updates applied in a random order and
  reads that may see values from before the step (as the GPU's concurrent
  CTAs may);
  expansion D[g][v] = min_b' dB[g][b'] + F_q[b'][v] (bdy_expand_*);
  fix-up of the inner rows (local_fixup_*).

Integer weights, so every comparison is exact."""
import numpy as np
import pytest
from scipy.sparse import csr_matrix
from scipy.sparse.csgraph import shortest_path

INF = 10**8


def _random_graph(rng, n, m, directed):
    u = rng.integers(0, n, m)
    v = rng.integers(0, n, m)
    w = rng.integers(1, 50, m)
    keep = u != v
    u, v, w = u[keep], v[keep], w[keep]
    if not directed:
        u, v, w = np.concatenate([u, v]), np.concatenate([v, u]), np.concatenate([w, w])
    return u, v, w


def _apsp(n, u, v, w):
    d = np.full((n, n), np.inf)
    np.fill_diagonal(d, 0)
    for a, b, c in zip(u, v, w):
        d[a, b] = min(d[a, b], c)
    g = csr_matrix(np.where(np.isinf(d), 0, d))
    out = shortest_path(g, method="D", directed=True)
    out[np.isinf(out)] = INF
    return out.astype(np.int64)


def _boundary_form(n, u, v, w, gid, K, rng):
    # boundary flags as the reference defines them (both ends of a cross arc)
    bdy = np.zeros(n, bool)
    cross = gid[u] != gid[v]
    bdy[u[cross]] = True
    bdy[v[cross]] = True
    parts = [np.concatenate([np.flatnonzero((gid == p) & bdy), np.flatnonzero((gid == p) & ~bdy)])
             for p in range(K)]
    b = [int(((gid == p) & bdy).sum()) for p in range(K)]
    # local closures over each part's own arcs
    F = []
    for p in range(K):
        vs = parts[p]
        loc = {x: i for i, x in enumerate(vs)}
        m = np.full((len(vs), len(vs)), INF, np.int64)
        np.fill_diagonal(m, 0)
        for a, c, ww in zip(u, v, w):
            if gid[a] == p and gid[c] == p:
                m[loc[a], loc[c]] = min(m[loc[a], loc[c]], ww)
        for k in range(len(vs)):
            m = np.minimum(m, m[:, k:k + 1] + m[k:k + 1, :])
        F.append(np.minimum(m, INF))
    # boundary indices
    boff = np.concatenate([[0], np.cumsum(b)])
    nb = int(boff[-1])
    gof = {}
    for p in range(K):
        for c in range(b[p]):
            gof[parts[p][c]] = boff[p] + c
    part_of_g = np.concatenate([[p] * b[p] for p in range(K)]).astype(int) if nb else np.zeros(0, int)
    xin = [[] for _ in range(nb)]      # cross in-arcs of every boundary vertex
    xout = [[] for _ in range(nb)]
    for a, c, ww in zip(u, v, w):
        if gid[a] != gid[c]:
            xin[gof[c]].append((gof[a], ww))
            xout[gof[a]].append(gof[c])
    # closure from every boundary vertex (one "tile" of all sources at once)
    dB = np.full((nb, nb), INF, np.int64)
    for s in range(nb):
        D = np.full(nb, INF, np.int64)
        D[s] = 0
        lrows = {part_of_g[s]: {s}}          # rows a changed by the cross step (or the seed)
        while True:
            changed = set()
            # local step: parts in a random order, reads possibly stale
            snap = D.copy()
            for p in rng.permutation(list(lrows.keys())):
                rows = list(lrows[p])
                for c in rng.permutation(b[p]):
                    g = boff[p] + c
                    src = snap if rng.random() < 0.5 else D
                    cand = min(int(src[boff[p] + a] + F[p][a, c]) for a in (g2 - boff[p] for g2 in rows))
                    if cand < D[g]:
                        D[g] = cand
                        changed.add(g)
            changed |= {g for rows in lrows.values() for g in rows}   # (their own arcs, too)
            # cross step: heads of arcs leaving changed rows, in a random order
            heads = sorted({h for g in changed for h in xout[g]})
            lrows = {}
            improved = False
            snap = D.copy()
            for h in rng.permutation(heads) if heads else []:
                src = snap if rng.random() < 0.5 else D
                cand = min(int(src[t] + ww) for t, ww in xin[h])
                if cand < D[h]:
                    D[h] = cand
                    improved = True
                    lrows.setdefault(part_of_g[h], set()).add(h)
            if not improved:
                break
        dB[s] = np.minimum(D, INF)
    # expansion and fix-up into the full matrix (rows and columns: vertex ids)
    out = np.full((n, n), INF, np.int64)
    FB = {}
    for g_vertex, g in gof.items():
        for q in range(K):
            vs = parts[q]
            if b[q] == 0:
                row = np.full(len(vs), INF, np.int64)
            else:
                row = np.min(dB[g, boff[q]:boff[q] + b[q]][:, None] + F[q][:b[q], :], axis=0)
            if q == gid[g_vertex]:
                FB[g] = np.minimum(row, INF)
            out[g_vertex, vs] = np.minimum(row, INF)
    for p in range(K):
        vs = parts[p]
        exact = F[p].copy()
        for i in range(b[p], len(vs)):
            best = exact[i].copy()
            for k in range(b[p]):
                best = np.minimum(best, F[p][i, k] + FB[boff[p] + k])
            exact[i] = best
        for i in range(b[p]):
            exact[i] = FB[boff[p] + i]
        for i in range(b[p], len(vs)):
            # inner rows: the part's own columns from the exact closure, the
            # other columns through the part's boundary rows (the min-plus merge)
            row = np.full(n, INF, np.int64)
            for k in range(b[p]):
                row = np.minimum(row, exact[i, k] + out[vs[k]])
            row[vs] = exact[i]
            out[vs[i]] = np.minimum(row, INF)
    return out


@pytest.mark.parametrize("seed", range(12))
def test_boundary_graph_form_gives_the_exact_distances(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(20, 60))
    K = int(rng.integers(2, 6))
    directed = bool(seed % 2)
    u, v, w = _random_graph(rng, n, int(rng.integers(n, 4 * n)), directed)
    gid = rng.integers(0, K, n)
    got = _boundary_form(n, u, v, w, gid, K, rng)
    want = _apsp(n, u, v, w)
    np.testing.assert_array_equal(got, want)
