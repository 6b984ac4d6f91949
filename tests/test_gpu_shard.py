"""The sharded boundary-graph form on one GPU: two "ranks" (two device
graphs of the same CSR and partition) each close their own parts locally,
a device copy stands in for the all-gather of their boundary rows, and each
closes the boundary graph, expands and fixes up its own parts; every block
must equal the one-GPU full batch bit for bit.  The ranks run one after the
other (no rank waits on another's kernels)."""
import numpy as np
import pytest

from fastapsp_b200 import FAP_MODE_BATCHED, Context, DeviceGraph, FapError, workloads
from fastapsp_b200 import _lib as L
from fastapsp_b200.sharding import rows_of, shard_layout, shard_parts

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,world", [("road20k", 2), ("grid128", 3), ("grid256", 2)])
def test_emulated_ranks_equal_the_one_gpu_batch(cuda_ok, name, world):
    import torch
    wl = workloads.load(name)
    ro, col, w = wl.csr()
    vn, vo, bn = wl.ver_num, wl.ver_offset, wl.bdy_num
    gid, st2ed = wl.graph.getGraphId(), wl.graph.getMapping()
    ctx = Context(0)

    def graph():
        dg = DeviceGraph(ctx, ro, col, w)
        dg.set_parts(wl.K, gid, st2ed, vn, vo, bn)
        return dg

    ref = graph()
    ref.solve(None, FAP_MODE_BATCHED)
    want = {p: ref.copy_block(p) for p in range(1, wl.K + 1)}
    del ref
    shards = shard_parts(vn, bn, wl.n, world)
    owner, elems, stride, offset = shard_layout(vn, bn, shards)
    tdt = torch.int32
    ranks = [graph() for _ in range(world)]
    sends = [torch.full((max(stride, 1),), -7, dtype=tdt, device="cuda") for _ in range(world)]
    for r in range(world):
        got = ranks[r].shard_begin(shards[r], sends[r].data_ptr(), stride)
        assert got == elems[r]
    torch.cuda.synchronize()
    recv = torch.cat(sends)          # stands in for the all-gather
    torch.cuda.synchronize()
    for r in range(world):
        dg = ranks[r]
        dg.shard_finish(recv.data_ptr(), world, owner, stride)
        dg.reserve(rows_of(shards[r], vn))
        dg.solve(shards[r], FAP_MODE_BATCHED)
        assert "sharded" in dg.stage1_name()
        for p in shards[r]:
            assert np.array_equal(dg.copy_block(p), want[p]), f"rank {r} part {p}"
        other = next(p for p in range(1, wl.K + 1) if owner[p] != r)
        with pytest.raises(FapError) as ei:
            dg.solve([other], FAP_MODE_BATCHED)
        assert ei.value.code == L.FAP_ERR_STATE
