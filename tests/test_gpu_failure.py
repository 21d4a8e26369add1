"""Failure paths on the GPU, made without faulting it: every device-side
wait is bounded and every error comes back as a status the host reads.

* A tile that never publishes its look-back record (a flag nothing sets,
  WAHGPU_TEST_WITHHOLD_TILE): the tiles waiting on it give up after their
  bounded wait and the call reports WAHGPU_ETIMEOUT; the context stays
  usable and the next call is exact.
* A serialized bitvector holding a fill word of count 0 (which no valid
  bitvector has): the upload scan reports WAHGPU_EFORMAT.
* A device allocation that fails (WAHGPU_TEST_FAIL_ALLOC): WAHGPU_ENOMEM,
  and the next call succeeds."""
import numpy as np
import pytest

import oracle
from oracle import wahgen as G

pytestmark = pytest.mark.gpu


def _pair():
    a = oracle.build_runs(G.geometric_runs(41, 6 * 2048 * 31, 0.3))
    b = oracle.build_runs(G.geometric_runs(42, 6 * 2048 * 31, 0.3))
    return a, b


@pytest.mark.parametrize("engine", [4, 5])
def test_withheld_record_times_out(gpu_ctx, engine):
    import libfastlib_b200 as L
    a, b = _pair()
    A, B = gpu_ctx.bitvector(a), gpu_ctx.bitvector(b)
    old = gpu_ctx.get_tuning(L.TUNE_DENSE_ENGINE)
    gpu_ctx.set_tuning(L.TUNE_DENSE_ENGINE, engine)
    try:
        gpu_ctx.set_tuning(L.TEST_WITHHOLD_TILE, 1)
        with pytest.raises(L.WahError) as e:
            A._binop(1, B, False).write()
        assert e.value.code == -7  # WAHGPU_ETIMEOUT
        # the hook cleared itself; the context is still usable
        ref, cnt = oracle.binop(1, a, b)
        r = A._binop(1, B, False)
        assert np.array_equal(r.write(), ref) and r.cnt() == cnt
    finally:
        gpu_ctx.set_tuning(L.TUNE_DENSE_ENGINE, old)


def test_corrupt_serialized_bitvector(gpu_ctx):
    import libfastlib_b200 as L
    bad = np.asarray(G.serialize([0x12345, 0x80000000, 0x7FFFFFFF]), np.uint32)  # a 0-fill of count 0
    with pytest.raises(L.WahError) as e:
        gpu_ctx.bitvector(bad).size()
    assert e.value.code == -5  # WAHGPU_EFORMAT


def test_allocation_failure(gpu_ctx):
    import libfastlib_b200 as L
    a, b = _pair()
    gpu_ctx.set_tuning(L.TEST_FAIL_ALLOC, 1)
    with pytest.raises(L.WahError) as e:
        gpu_ctx.bitvector(a)
    assert e.value.code == -4  # WAHGPU_ENOMEM
    A, B = gpu_ctx.bitvector(a), gpu_ctx.bitvector(b)
    ref, cnt = oracle.binop(0, a, b)
    r = A._binop(0, B, False)
    assert np.array_equal(r.write(), ref) and r.cnt() == cnt
