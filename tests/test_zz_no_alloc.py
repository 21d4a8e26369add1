"""The allocation-free row-id entry point (wahgpu_rids_noalloc).

It serves callers that cannot allocate device memory while they run: GPU
pipelines driven from host callbacks (a callback may not call cudaMalloc),
runtimes that own all device memory through their own pool, and paths that
cannot take the synchronisation an allocation may bring.  It computes into
caller-provided device buffers with a fixed scratch area compiled into the
library.  These tests check its row ids against the oracle's restatement of
the reference's indexSet walk and against the regular entry point
(wahgpu_bv_rids), on two calls in a row (the shared scratch area keeps the
previous call's contents and must not leak them into the next), with a
capacity below the count, and at the largest input the scratch area takes.
Collected last on purpose; it passes alone and after the other tests.
"""
import ctypes

import numpy as np
import pytest

import oracle
from oracle import wahgen as G

pytestmark = pytest.mark.gpu

MAX_WORDS = 1 << 24  # whole words the fixed scratch area takes


def _lib():
    import libfastlib_b200 as L
    lib = L.load_library()
    lib.wahgpu_rids_noalloc.restype = ctypes.c_int
    lib.wahgpu_rids_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64,
                                        ctypes.c_void_p, ctypes.c_void_p]
    return lib


def _noalloc(lib, ser, cap, stream):
    """One call through the C ABI; returns (ids written, count)."""
    import torch
    d_ser = torch.from_numpy(np.ascontiguousarray(ser, dtype=np.uint32).view(np.int32)).cuda()
    d_out = torch.full((max(cap, 1),), -1, dtype=torch.int32, device="cuda")
    d_cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    rc = lib.wahgpu_rids_noalloc(ctypes.c_void_p(d_ser.data_ptr()), ctypes.c_uint64(len(ser)),
                                 ctypes.c_void_p(d_out.data_ptr()), ctypes.c_uint64(cap),
                                 ctypes.c_void_p(d_cnt.data_ptr()), ctypes.c_void_p(stream))
    assert rc == 0, lib.wahgpu_last_error(None)
    torch.cuda.synchronize()
    n = int(d_cnt.item())
    got = d_out[:min(n, cap)].cpu().numpy().view(np.uint32).copy()
    return got, n


def test_noalloc_rids_match_regular_entry_point(gpu_ctx):
    import torch
    lib = _lib()
    stream = torch.cuda.current_stream().cuda_stream
    cases = [
        oracle.build_runs(G.geometric_runs(21, 1 << 22, 0.05)),
        oracle.build_runs(G.geometric_runs(22, (1 << 20) + 13, 0.5)),
        G.serialize([0xC0000002] * 5000 + [0x7FFFFFFF, 0x80000004, 0x1234], 7, 0x55),
    ]
    for ser in cases:
        want = oracle.rids(ser)
        regular = gpu_ctx.bitvector(ser).rids()
        assert np.array_equal(regular, want)
        cap = int(want.size) + 8
        for _ in range(2):  # two calls in a row share the scratch area
            got, n = _noalloc(lib, ser, cap, stream)
            assert n == want.size
            assert np.array_equal(got, want)
            assert np.array_equal(got, regular)


def test_noalloc_capacity_below_count(gpu_ctx):
    """ids past cap are dropped; the count is still the full count."""
    import torch
    lib = _lib()
    stream = torch.cuda.current_stream().cuda_stream
    ser = oracle.build_runs(G.geometric_runs(23, 1 << 21, 0.2))
    want = oracle.rids(ser)
    for cap in (want.size // 2, 1, 0):
        got, n = _noalloc(lib, ser, cap, stream)
        assert n == want.size
        assert np.array_equal(got, want[:cap])


def test_noalloc_largest_input(gpu_ctx):
    """2^24 + 1 whole words and no active word (2^24 + 2 serialized words):
    the most the fixed scratch area takes, against the oracle and the
    regular entry point."""
    import torch
    lib = _lib()
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(24)
    body = np.zeros(MAX_WORDS + 1, dtype=np.uint32)
    pick = rng.choice(body.size, size=20000, replace=False)
    body[pick] = rng.integers(1, 0x7FFFFFFF, size=pick.size, dtype=np.uint32)
    body[-1] = 0xC0000003  # a 1-fill as the last whole word
    ser = np.concatenate([body, np.zeros(1, np.uint32)])
    assert ser.size == MAX_WORDS + 2
    want = oracle.rids(ser)
    regular = gpu_ctx.bitvector(ser).rids()
    assert np.array_equal(regular, want)
    for _ in range(2):
        got, n = _noalloc(lib, ser, int(want.size), stream)
        assert n == want.size
        assert np.array_equal(got, want)


def test_noalloc_rejects_oversize(gpu_ctx):
    lib = _lib()
    fake = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.wahgpu_rids_noalloc(fake, ctypes.c_uint64((1 << 24) + 3), fake, ctypes.c_uint64(1), fake, None)
    assert rc == -8
    assert b"16,777,216" in lib.wahgpu_last_error(None)
