"""Part sharding across ranks (one process per GPU).

Parts are independent units of the per-subgraph solve path: rank r solves
its own subset of parts into its own GPU's memory and nothing crosses
between ranks on the data path.  This is the single-node equivalent of the
reference's MPI task split (fap/fap_more_task_mpi.cpp:34-53, a shuffle and
a contiguous split); here the split is a greedy longest-processing-time
assignment by estimated cost, which keeps ranks balanced when boundary
counts differ.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def part_cost(s: int, b: int, n: int) -> float:
    """Relative cost of one part: Floyd s^3 + min-plus (s-b) b n relaxations
    + output writes s n + SSSP b (n + m) ~ b n."""
    inner = s - b
    return float(s) ** 3 + float(inner) * b * n + 4.0 * s * n + 8.0 * b * n


def shard_parts(ver_num: Sequence[int], bdy_num: Sequence[int], n: int, world: int) -> List[List[int]]:
    """Assign parts 1..K (ver_num/bdy_num indexed 1..K) to `world` ranks.
    Deterministic; every part appears exactly once; each rank's list is in
    ascending part order."""
    K = len(ver_num) - 1
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(1, K + 1), key=lambda p: (-part_cost(ver_num[p], bdy_num[p], n), p))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out: List[List[int]] = [[] for _ in range(world)]
    for p in order:
        load, r = heapq.heappop(heap)
        out[r].append(p)
        heapq.heappush(heap, (load + part_cost(ver_num[p], bdy_num[p], n), r))
    return [sorted(x) for x in out]


def rows_of(parts: Sequence[int], ver_num: Sequence[int]) -> int:
    return int(sum(int(ver_num[p]) for p in parts))


def reduce_over_ranks(x: float, op: str = "max", device=None) -> float:
    """Max or sum of a scalar over all ranks of the default process group
    (identity without one).  `device` is where the reduction tensor lives
    (a CUDA device for NCCL, None/CPU for gloo)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def group_parts_by_rows(parts: Sequence[int], ver_num: Sequence[int], max_rows: int) -> List[List[int]]:
    """Split `parts` (in order) into consecutive groups whose row counts fit
    in max_rows -- the output of a graph too large for device memory is
    produced group by group into one reserved row budget."""
    groups: List[List[int]] = []
    cur: List[int] = []
    rows = 0
    for p in parts:
        r = int(ver_num[p])
        if r > max_rows:
            raise ValueError(f"part {p} has {r} rows, more than the budget of {max_rows}")
        if cur and rows + r > max_rows:
            groups.append(cur)
            cur, rows = [], 0
        cur.append(p)
        rows += r
    if cur:
        groups.append(cur)
    return groups


def shard_layout(ver_num: Sequence[int], bdy_num: Sequence[int], shards: Sequence[Sequence[int]]):
    """Layout of the boundary-row exchange of the sharded boundary-graph form
    (fap_graph_shard_begin / _finish): owner[p] = rank of part p (index 0
    unused), elems[r] = elements rank r sends (its parts ascending, b_p x s_p
    each), stride = the largest of them (every rank's send buffer is padded
    to it for the all-gather), offset[p] = where part p's rows start inside
    its owner's segment."""
    K = len(ver_num) - 1
    owner = [0] * (K + 1)
    for r, parts in enumerate(shards):
        for p in parts:
            owner[p] = r
    elems = [0] * len(shards)
    offset = [0] * (K + 1)
    for p in range(1, K + 1):
        r = owner[p]
        offset[p] = elems[r]
        elems[r] += int(bdy_num[p]) * int(ver_num[p])
    return owner, elems, max(elems) if elems else 0, offset
