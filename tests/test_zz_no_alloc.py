"""The allocation-free closure, fap_floyd_noalloc, against the allocating
fap_op_floyd.

fap_floyd_noalloc exists for callers that may not allocate device memory
when they run a closure -- a host framework that owns all GPU memory through
its own pool, or a latency-sensitive path where cudaMalloc/cudaFree would
synchronise the device.  It keeps its working copy in one device array built
into the library, so this test checks that two calls in a row (the second
on a smaller matrix, over whatever the first left in that array) both give
exactly what the allocating entry point gives.  This file is named to be
collected last.
"""
import ctypes

import numpy as np
import pytest

from fastapsp_b200 import FAP_DTYPE_F32, FAP_DTYPE_I32, Context
from fastapsp_b200 import _lib as L

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5


def _matrix(s, dtype, seed):
    rng = np.random.default_rng(seed)
    if dtype == FAP_DTYPE_I32:
        M = rng.integers(1, 1000, (s, s)).astype(np.int32)
        M[rng.random((s, s)) < 0.9] = L.FAP_INF_I32
    else:
        M = np.exp(rng.uniform(np.log(0.01), np.log(100), (s, s))).astype(np.float32)
        M[rng.random((s, s)) < 0.9] = np.float32(1e8)
    np.fill_diagonal(M, 0)
    return M


def _compare(got, ref, dtype):
    if dtype == FAP_DTYPE_I32:
        assert np.array_equal(got, ref)
    else:
        reach = ref < 1e8
        assert np.array_equal(reach, got < 1e8)
        rel = np.abs(got[reach] - ref[reach]) / np.maximum(np.abs(ref[reach]), 1e-30)
        assert rel.max(initial=0.0) <= REL_TOL


@pytest.mark.parametrize("dtype", [FAP_DTYPE_I32, FAP_DTYPE_F32])
def test_noalloc_matches_allocating_floyd_twice(cuda_ok, dtype):
    import torch
    lib = L.lib()
    ctx = Context(0)
    ctx.use_torch_stream()
    stream = torch.cuda.current_stream().cuda_stream
    tdt = torch.int32 if dtype == FAP_DTYPE_I32 else torch.float32
    for call, (s, seed) in enumerate([(700, 1), (300, 2)]):
        M = _matrix(s, dtype, seed + 10 * dtype)
        # a strided view (ld > s) exercises the leading dimension too
        buf_a = torch.full((s, s + 5), -1, dtype=tdt, device="cuda")
        buf_b = buf_a.clone()
        a = buf_a[:, :s]
        b = buf_b[:, :s]
        a.copy_(torch.from_numpy(M))
        b.copy_(torch.from_numpy(M))
        ctx.floyd(a, dtype)                     # allocating entry point
        rc = lib.fap_floyd_noalloc(dtype, s, ctypes.c_void_p(b.data_ptr()), b.stride(0),
                                   ctypes.c_void_p(stream))
        assert rc == L.FAP_OK, lib.fap_floyd_noalloc_last_error()
        torch.cuda.synchronize()
        assert lib.fap_floyd_noalloc_status() == L.FAP_OK, lib.fap_floyd_noalloc_last_error()
        _compare(b.cpu().numpy(), a.cpu().numpy(), dtype)
        # the padding columns of the caller's buffer are untouched
        assert torch.all(buf_b[:, s:] == -1).item(), f"call {call} wrote past column s"


@pytest.mark.parametrize("dtype", [FAP_DTYPE_I32, FAP_DTYPE_F32])
def test_noalloc_matches_the_oracle_at_edge_sizes(cuda_ok, dtype):
    """One element, exactly one tile, a ragged size, and the largest size the
    built-in array holds (its last tile row and column), each against the
    oracle's Floyd-Warshall (the reference's k-i-j loop with strict >)."""
    import torch

    from oracle import oracle as O
    lib = L.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for s, seed in [(1, 5), (128, 6), (700, 7), (L.FAP_NOALLOC_FLOYD_MAX, 8)]:
        M = _matrix(s, dtype, seed + 10 * dtype)
        if dtype == FAP_DTYPE_I32:
            M[M == L.FAP_INF_I32] = 100000000
        ref = O.port_floyd(M.astype(np.float32))
        if dtype == FAP_DTYPE_I32:
            ref = O.to_i32(ref)
        b = torch.from_numpy(M).to("cuda")
        rc = lib.fap_floyd_noalloc(dtype, s, ctypes.c_void_p(b.data_ptr()), s, ctypes.c_void_p(stream))
        assert rc == L.FAP_OK, lib.fap_floyd_noalloc_last_error()
        torch.cuda.synchronize()
        assert lib.fap_floyd_noalloc_status() == L.FAP_OK, lib.fap_floyd_noalloc_last_error()
        _compare(b.cpu().numpy(), ref, dtype)


def test_noalloc_rejects_oversize_before_gpu_work(cuda_ok):
    import torch
    lib = L.lib()
    s = L.FAP_NOALLOC_FLOYD_MAX + 1
    small = torch.zeros(4, dtype=torch.int32, device="cuda")  # never touched
    rc = lib.fap_floyd_noalloc(FAP_DTYPE_I32, s, ctypes.c_void_p(small.data_ptr()), s,
                               ctypes.c_void_p(0))
    assert rc == L.FAP_ERR_RANGE
    assert b"FAP_NOALLOC_FLOYD_MAX" in lib.fap_floyd_noalloc_last_error()
