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


def _exchange_worker(rank, world, port, vn, bn, out_q):
    """One gloo rank of the boundary-row exchange: pack its parts' rows at
    the layout's offsets, all-gather, and read every other rank's parts back
    the way fap_graph_shard_finish does (owner segment + offset)."""
    import torch
    import torch.distributed as dist

    from fastapsp_b200.sharding import shard_layout
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    try:
        shards = shard_parts(vn, bn, 1000, world)
        owner, elems, stride, offset = shard_layout(vn, bn, shards)

        def block(p):
            r = np.arange(int(bn[p]))[:, None]
            c = np.arange(int(vn[p]))[None, :]
            return (p * 1000000 + r * 1000 + c).astype(np.int32)

        send = np.full(stride, -1, np.int32)
        pos = 0
        for p in sorted(shards[rank]):          # the library's packing order
            assert offset[p] == pos
            blk = block(p).ravel()
            send[pos:pos + blk.size] = blk
            pos += blk.size
        assert pos == elems[rank]
        got = [torch.empty(stride, dtype=torch.int32) for _ in range(world)]
        dist.all_gather(got, torch.from_numpy(send))
        recv = torch.cat(got).numpy()
        bad = []
        for p in range(1, len(vn)):
            n_el = int(bn[p]) * int(vn[p])
            seg = recv[owner[p] * stride + offset[p]: owner[p] * stride + offset[p] + n_el]
            if not np.array_equal(seg.reshape(int(bn[p]), int(vn[p])), block(p)):
                bad.append(p)
        out_q.put(("ok", rank, bad, elems, stride))
    except Exception as e:  # reported to the parent
        out_q.put(("err", rank, repr(e)))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def test_boundary_row_exchange_layout_over_two_gloo_ranks():
    """The sharded boundary-graph form's exchange: every rank packs its own
    parts' boundary rows (ascending, b x s each) at the offsets of
    shard_layout, and after an all-gather every rank finds every part's rows
    at owner * stride + offset."""
    rng = np.random.default_rng(5)
    K = 11
    vn = np.concatenate([[0], rng.integers(20, 40, K)]).astype(np.int64)
    bn = np.concatenate([[0], rng.integers(0, 6, K)]).astype(np.int64)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_exchange_worker, args=(r, 2, port, vn, bn, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in ps:
        p.join(timeout=60)
    assert all(r[0] == "ok" for r in res), res
    assert all(r[2] == [] for r in res), res
    elems, stride = res[0][3], res[0][4]
    assert stride == max(elems) and sum(elems) == int((vn * bn).sum())
