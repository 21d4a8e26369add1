"""The C oracle against the reference library's own outputs (tests/golden/,
made by tests/golden/make_golden.py from FastBit built from source)."""
import numpy as np
import pytest

import oracle
from conftest import load_golden, unpack


def test_binop_random_word_exact():
    g = load_golden("binop_random.npz")
    n = len(g["op"])
    bad = 0
    for i in range(n):
        if g["status"][i] != 0:
            continue
        w, c = oracle.binop(int(g["op"][i]), unpack(g, "a", i), unpack(g, "b", i), inplace=bool(g["inplace"][i]))
        ref = unpack(g, "res", i)
        if c != int(g["cnt"][i]) or not np.array_equal(w, ref):
            bad += 1
    assert bad == 0


def test_binop_unequal_sizes_word_exact():
    """Operands of different sizes: the padding inside the reference's
    operators (adjustSize) restated by the oracle."""
    g = load_golden("binop_unequal.npz")
    assert len(g["op"]) == 400
    for i in range(len(g["op"])):
        assert g["status"][i] == 0
        w, c = oracle.binop(int(g["op"][i]), unpack(g, "a", i), unpack(g, "b", i), inplace=bool(g["inplace"][i]))
        assert c == int(g["cnt"][i]) and np.array_equal(w, unpack(g, "res", i)), i


def test_binop_geometric_word_exact():
    g = load_golden("binop_geom.npz")
    for k, (di, op, ip) in enumerate(g["case"]):
        a = unpack(g, "operands", 2 * di)
        b = unpack(g, "operands", 2 * di + 1)
        w, c = oracle.binop(int(op), a, b, inplace=bool(ip))
        assert c == int(g["cnt"][k])
        assert np.array_equal(w, unpack(g, "res", k)), (di, op, ip)


def test_appendfill_construction_matches_reference():
    g = load_golden("binop_geom.npz")
    offs = np.zeros(1, np.int64)
    ro = g["runs_off"]
    for k in range(len(ro) - 1):
        runs = g["runs"][ro[k]:ro[k + 1]].astype(np.uint64)
        assert np.array_equal(oracle.build_runs(runs), unpack(g, "operands", k))


def test_unary_ops():
    g = load_golden("unary.npz")
    for i in range(len(g["src_off"]) - 1):
        src = unpack(g, "src", i)
        w, c = oracle.compress(src)
        assert np.array_equal(w, unpack(g, "compress", i))
        assert c == int(g["compress_cnt"][i])
        assert np.array_equal(oracle.decompress(src), unpack(g, "decompress", i))
        assert np.array_equal(oracle.flip(src), unpack(g, "flip", i))
        assert np.array_equal(oracle.rids(src), unpack(g, "rids", i))


def test_relic_small_hits_match_scan():
    import ctypes
    g = load_golden("relic_small.npz")
    lib = oracle.lib()
    vals = np.ascontiguousarray(g["vals"], dtype=np.uint32)
    for q, (lo, hi) in enumerate(g["queries"]):
        out = np.empty(len(vals), np.uint32)
        lib.ro_range_u32.restype = ctypes.c_long
        n = lib.ro_range_u32(vals.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), ctypes.c_uint64(len(vals)),
                             ctypes.c_double(lo), ctypes.c_double(hi),
                             out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), ctypes.c_uint64(len(vals)))
        assert n == int(g["counts"][q])
        assert np.array_equal(out[:n], unpack(g, "rids", q))


def test_bin_small_hits_match_scan():
    g = load_golden("bin_small.npz")
    v = g["vals"].astype(np.float64)
    for q, (lo, hi) in enumerate(g["queries"]):
        e = np.flatnonzero((v >= lo) & (v < hi))
        assert len(e) == int(g["counts"][q])
        assert np.array_equal(e, unpack(g, "rids", q))
