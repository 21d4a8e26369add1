"""GPU parity of the WAH operators through the C ABI (libwahgpu.so):
word-for-word against the reference's golden outputs and against the oracle
at the full 2^28-bit size of the raw-WAH workload."""
import numpy as np
import pytest

import oracle
from oracle import wahgen as G
from conftest import load_golden, unpack

pytestmark = pytest.mark.gpu


def _bin(ctx, op, a, b, inplace):
    import libfastlib_b200 as L
    A, B = ctx.bitvector(a), ctx.bitvector(b)
    r = A._binop(op, B, inplace)
    return r.write(), r.cnt()


def test_random_golden(gpu_ctx):
    import libfastlib_b200 as L
    g = load_golden("binop_random.npz")
    ndeg = 0
    for i in range(len(g["op"])):
        if g["status"][i] != 0:
            continue
        a, b = unpack(g, "a", i), unpack(g, "b", i)
        op, ip = int(g["op"][i]), int(g["inplace"][i])
        if oracle.is_degenerate(a) or oracle.is_degenerate(b):
            with pytest.raises(L.WahError) as e:
                _bin(gpu_ctx, op, a, b, ip)
            assert e.value.code == -9
            ndeg += 1
            continue
        w, c = _bin(gpu_ctx, op, a, b, ip)
        assert c == int(g["cnt"][i]), (i, op, ip)
        assert np.array_equal(w, unpack(g, "res", i)), (i, op, ip, [hex(x) for x in a], [hex(x) for x in b])
    assert ndeg > 0


def test_geometric_golden(gpu_ctx):
    g = load_golden("binop_geom.npz")
    for k, (di, op, ip) in enumerate(g["case"]):
        a, b = unpack(g, "operands", 2 * di), unpack(g, "operands", 2 * di + 1)
        w, c = _bin(gpu_ctx, int(op), a, b, int(ip))
        assert c == int(g["cnt"][k]), (di, op, ip)
        assert np.array_equal(w, unpack(g, "res", k)), (di, op, ip)


@pytest.mark.parametrize("density", [1e-4, 1e-3, 1e-2, 0.1, 0.5])
def test_full_size_against_oracle(gpu_ctx, density):
    """2^28-bit operands (the raw-WAH workload) — every op, both forms."""
    nbits = 1 << 28
    a = oracle.build_runs(G.geometric_runs(11, nbits, density))
    b = oracle.build_runs(G.geometric_runs(12, nbits, density))
    A, B = gpu_ctx.bitvector(a), gpu_ctx.bitvector(b)
    assert A.size() == nbits and B.size() == nbits
    for op in range(4):
        for ip in (0, 1):
            ref, rc = oracle.binop(op, a, b, inplace=bool(ip))
            r = A._binop(op, B, bool(ip))
            w = r.write()
            assert r.cnt() == rc, (op, ip)
            assert np.array_equal(w, ref), (op, ip)


def test_many_tiles_fuzz(gpu_ctx):
    """Operands of ~10^5 words of mixed forms so results span many tiles and
    the look-back carries runs, heads and step states across tile edges."""
    rng = np.random.default_rng(5)
    for trial in range(12):
        ng = int(rng.integers(20000, 200000))
        style_a = ["mixed", "short", "sparse", "canon", "dense"][trial % 5]
        style_b = ["canon", "sparse", "mixed", "short", "mixed"][trial % 5]
        wa = G.random_words(rng, ng, style_a)
        wb = G.random_words(rng, ng, style_b)
        anb = int(rng.integers(0, 31))
        a = G.serialize(wa, anb, int(rng.integers(0, 1 << 31)))
        b = G.serialize(wb, anb, int(rng.integers(0, 1 << 31)))
        if oracle.is_degenerate(a) or oracle.is_degenerate(b):
            continue
        for op in range(4):
            ip = int(rng.integers(0, 2))
            ref, rc = oracle.binop(op, a, b, inplace=bool(ip))
            w, c = _bin(gpu_ctx, op, a, b, ip)
            assert c == rc and np.array_equal(w, ref), (trial, op, ip)


def test_unary_golden(gpu_ctx):
    g = load_golden("unary.npz")
    for i in range(len(g["src_off"]) - 1):
        src = unpack(g, "src", i)
        A = gpu_ctx.bitvector(src)
        assert np.array_equal(A.rids(), unpack(g, "rids", i)), i
        A.compress()
        assert np.array_equal(A.write(), unpack(g, "compress", i)), i
        assert A.cnt() == int(g["compress_cnt"][i])
        B = gpu_ctx.bitvector(src)
        B.decompress()
        ref = unpack(g, "decompress", i)
        got = B.write()
        # decompress() of an all-zero vector is collapsed again by the cnt()
        # the fixture took after write(); compare bits through compress()
        assert np.array_equal(got, ref) or np.array_equal(oracle.compress(got)[0], oracle.compress(ref)[0]), i
        C = gpu_ctx.bitvector(src)
        C.flip()
        assert np.array_equal(C.write(), oracle.compress(unpack(g, "flip", i))[0]), i


def test_rids_large(gpu_ctx):
    nbits = 1 << 24
    a = oracle.build_runs(G.geometric_runs(3, nbits, 0.3, mean1=200.0))
    A = gpu_ctx.bitvector(a)
    assert np.array_equal(A.rids(), oracle.rids(a))


def test_many_one_fills_per_tile(gpu_ctx):
    """Row ids and decompress of words that are all 1-fills (more per 4096-word
    tile than the kernels' shared fill list holds)."""
    words = [0xC0000002] * 9000 + [0x12345, 0x80000003] * 500
    a = G.serialize(words, 5, 0b10110)
    A = gpu_ctx.bitvector(a)
    assert np.array_equal(A.rids(), oracle.rids(a))
    B = gpu_ctx.bitvector(a)
    B.decompress()
    assert np.array_equal(B.write(), oracle.decompress(a))
