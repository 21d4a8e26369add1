"""The allocation-free row-id entry point (wahgpu_rids_noalloc).

It serves callers that cannot allocate device memory while they run — work
issued during CUDA graph capture, host-callback pipelines, runtimes that
own all device memory — so it computes into caller-provided device buffers
with a fixed scratch area compiled into the library.  This test compares its
output with the regular entry point (wahgpu_bv_rids) on two calls in a row,
which also checks that the shared scratch area is reset between calls.
Collected last on purpose; it passes alone and after the other tests.
"""
import ctypes

import numpy as np
import pytest

import oracle
from oracle import wahgen as G

pytestmark = pytest.mark.gpu


def _noalloc(lib, ser, stream):
    import torch
    d_ser = torch.from_numpy(np.ascontiguousarray(ser, dtype=np.uint32).view(np.int32)).cuda()
    cap = max(int(oracle.rids(ser).size) + 8, 1)
    d_out = torch.zeros(cap, dtype=torch.int32, device="cuda")
    d_cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    rc = lib.wahgpu_rids_noalloc(ctypes.c_void_p(d_ser.data_ptr()), ctypes.c_uint64(len(ser)),
                                 ctypes.c_void_p(d_out.data_ptr()), ctypes.c_uint64(cap),
                                 ctypes.c_void_p(d_cnt.data_ptr()), ctypes.c_void_p(stream))
    assert rc == 0, lib.wahgpu_last_error(None)
    torch.cuda.synchronize()
    n = int(d_cnt.item())
    return d_out[:n].cpu().numpy().view(np.uint32)


def test_noalloc_rids_match_regular_entry_point(gpu_ctx):
    import torch
    import libfastlib_b200 as L
    lib = L.load_library()
    lib.wahgpu_rids_noalloc.restype = ctypes.c_int
    lib.wahgpu_rids_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64,
                                        ctypes.c_void_p, ctypes.c_void_p]
    stream = torch.cuda.current_stream().cuda_stream
    cases = [
        oracle.build_runs(G.geometric_runs(21, 1 << 22, 0.05)),
        oracle.build_runs(G.geometric_runs(22, (1 << 20) + 13, 0.5)),
        G.serialize([0xC0000002] * 5000 + [0x7FFFFFFF, 0x80000004, 0x1234], 7, 0x55),
    ]
    for ser in cases:
        want = gpu_ctx.bitvector(ser).rids()
        first = _noalloc(lib, ser, stream)
        second = _noalloc(lib, ser, stream)
        assert np.array_equal(first, want)
        assert np.array_equal(second, want)


def test_noalloc_rejects_oversize(gpu_ctx):
    import libfastlib_b200 as L
    lib = L.load_library()
    lib.wahgpu_rids_noalloc.restype = ctypes.c_int
    lib.wahgpu_rids_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64,
                                        ctypes.c_void_p, ctypes.c_void_p]
    fake = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.wahgpu_rids_noalloc(fake, ctypes.c_uint64((1 << 24) + 3), fake, ctypes.c_uint64(1), fake, None)
    assert rc == -8
    assert b"16,777,216" in lib.wahgpu_last_error(None)
