"""Multi-rank logic on CPU (gloo, world size 2): part sharding covers every
part exactly once with balanced cost, rows/entries add up over ranks, the
timing reduction takes the maximum, and a rank that fails before a
collective makes the other rank's collective fail instead of hang."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from fastapsp_b200.sharding import part_cost, reduce_over_ranks, rows_of, shard_parts


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, vn, bn, n, out_q, fail_rank):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=10))
    try:
        if rank == fail_rank:
            raise RuntimeError("injected host-side failure before the collective")
        mine = shard_parts(vn, bn, n, world)[rank]
        entries = rows_of(mine, vn) * n
        total = reduce_over_ranks(entries, "sum")
        slowest = reduce_over_ranks(10.0 + rank, "max")
        out_q.put(("ok", rank, mine, total, slowest))
    except Exception as e:  # reported to the parent
        out_q.put(("err", rank, repr(e)))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(world, fail_rank=-1):
    rng = np.random.default_rng(0)
    K, n = 37, 5000
    vn = np.concatenate([[0], rng.integers(100, 200, K)]).astype(np.int64)
    vn[1:] = vn[1:] * n // vn[1:].sum() + 1
    bn = np.concatenate([[0], rng.integers(0, 90, K)])
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, vn, bn, n, q, fail_rank))
          for r in range(world)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in ps:
        p.join(timeout=60)
    return vn, bn, n, res


def test_shard_parts_single_process_properties():
    vn = [0, 900, 880, 910, 870, 905, 899]
    bn = [0, 5, 9, 2, 30, 7, 1]
    for world in (1, 2, 3, 4, 8):
        sh = shard_parts(vn, bn, 114599, world)
        flat = sorted(p for s in sh for p in s)
        assert flat == list(range(1, 7))
        assert all(s == sorted(s) for s in sh)
    loads = [sum(part_cost(vn[p], bn[p], 114599) for p in s) for s in shard_parts(vn, bn, 114599, 2)]
    assert max(loads) / min(loads) < 1.6


def test_two_gloo_ranks_cover_all_parts():
    vn, bn, n, res = _run(2)
    assert all(r[0] == "ok" for r in res), res
    parts = sorted(p for r in res for p in r[2])
    assert parts == list(range(1, len(vn)))
    totals = {r[3] for r in res}
    assert totals == {float(int(vn[1:].sum()) * n)}
    assert {r[4] for r in res} == {11.0}


def test_failing_rank_does_not_hang_the_other():
    vn, bn, n, res = _run(2, fail_rank=1)
    kinds = {r[1]: r[0] for r in res}
    assert kinds[1] == "err"
    assert kinds[0] == "err"   # its collective ends with an error (peer gone / timeout)
