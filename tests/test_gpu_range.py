"""GPU parity of relic / bin range evaluation and of conjunctive queries,
through the C ABI: hit counts and row ids against the reference's own
answers (golden fixtures, and the reference library run through
oracle/refdrv at the relic workload's full size) and against brute-force
scans of the raw values."""
import ctypes
import struct
import tempfile

import numpy as np
import pytest

import oracle
from oracle import wahgen as G
from conftest import load_golden, unpack

pytestmark = pytest.mark.gpu


def _scan(vals, lo, hi):
    v = vals.astype(np.float64)
    return np.flatnonzero((v >= lo) & (v < hi)).astype(np.uint32)


def _relic_ref(vals, queries):
    """Reference relic over vals: triple, counts, row ids."""
    with tempfile.TemporaryDirectory() as td:
        R = G.run_refdrv(oracle.REFDRV, [G.req_relic(vals, queries)], td)
        nk = R.u32(); keys = np.frombuffer(R.d, np.float64, nk, R.p).copy(); R.p += 8 * nk
        no = R.u32(); offs = np.frombuffer(R.d, np.int64, no, R.p).copy(); R.p += 8 * no
        bms = R.vec()
        res = []
        for _ in queries:
            st = R.u32(); c = R.u32(); r = R.vec()
            res.append((c, r))
    return keys, offs, bms, res


def _bin_ref(vals, nbins, queries):
    req = (struct.pack("<II", 9, len(vals)) + np.ascontiguousarray(vals, np.float32).tobytes()
           + struct.pack("<II", nbins, len(queries)) + np.asarray(queries, np.float64).reshape(-1, 2).tobytes())
    with tempfile.TemporaryDirectory() as td:
        R = G.run_refdrv(oracle.REFDRV, [req], td)
        nk = R.u32(); keys = np.frombuffer(R.d, np.float64, nk, R.p).copy(); R.p += 8 * nk
        no = R.u32(); offs = np.frombuffer(R.d, np.int64, no, R.p).copy(); R.p += 8 * no
        bms = R.vec()
        res = []
        for _ in range(len(queries)):
            st = R.u32(); c = R.u32(); r = R.vec()
            res.append((c, r))
    return keys, offs, bms, res


def test_relic_small_golden(gpu_ctx):
    import libfastlib_b200 as L
    g = load_golden("relic_small.npz")
    idx = L.Index(gpu_ctx, L.RELIC, len(g["vals"]), g["keys"], g["offsets"], g["bitmaps"], values=g["vals"])
    for q, (lo, hi) in enumerate(g["queries"]):
        n, rids, _ = L.evaluate(gpu_ctx, [idx.term(lo, hi)])
        assert n == int(g["counts"][q])
        assert np.array_equal(rids, unpack(g, "rids", q)), q


def test_bin_small_golden(gpu_ctx):
    import libfastlib_b200 as L
    g = load_golden("bin_small.npz")
    idx = L.Index(gpu_ctx, L.BIN, len(g["vals"]), g["keys"], g["offsets"], g["bitmaps"], values=g["vals"])
    for q, (lo, hi) in enumerate(g["queries"]):
        n, rids, _ = L.evaluate(gpu_ctx, [idx.term(lo, hi)])
        assert n == int(g["counts"][q]), q
        assert np.array_equal(rids, unpack(g, "rids", q)), q


def test_relic_full_size_against_reference(gpu_ctx):
    """1M-row uint32 column in [0,100), 100 seeded ranges lo <= x < hi, one
    batch: counts and row ids equal the reference's relic::evaluate."""
    import libfastlib_b200 as L
    rng = np.random.default_rng(42)
    vals = rng.integers(0, 100, size=1 << 20).astype(np.uint32)
    qs = []
    qrng = np.random.default_rng(7)
    while len(qs) < 100:
        lo, hi = (int(v) for v in qrng.integers(0, 101, size=2))
        if lo < hi:
            qs.append((float(lo), float(hi)))
    keys, offs, bms, ref = _relic_ref(vals, qs)
    idx = L.Index(gpu_ctx, L.RELIC, len(vals), keys, offs, bms, values=vals)
    total = sum(c for c, _ in ref)
    B = L.Batch(gpu_ctx, [[idx.term(lo, hi)] for lo, hi in qs], rid_cap=total)
    B.run()
    counts = B.counts()
    for q, (c, r) in enumerate(ref):
        assert int(counts[q]) == c, q
        assert np.array_equal(B.rids(q, c), r), q


def test_bin_reduced_against_reference(gpu_ctx):
    """Binned index (1000 equal-weight bins) over a 2M-row float32 mixture
    column; ranges spanning 1..500 bins with both edges inside bins."""
    import libfastlib_b200 as L
    rng = np.random.default_rng(3)
    n = 2 << 20
    z = rng.zipf(1.2, size=n) % 100000
    vals = np.where(rng.random(n) < 0.7, rng.normal(size=n), z).astype(np.float32)
    sv = np.sort(vals.astype(np.float64))
    qs = []
    for _ in range(40):
        span = int(rng.integers(1, 501)) / 1000.0
        a = float(rng.random()) * (1.0 - span)
        lo = sv[int(a * (n - 1))] + 1e-4
        hi = sv[int((a + span) * (n - 1))] - 1e-4
        if lo < hi:
            qs.append((lo, hi))
    keys, offs, bms, ref = _bin_ref(vals, 1000, qs)
    idx = L.Index(gpu_ctx, L.BIN, n, keys, offs, bms, values=vals)
    for q, (lo, hi) in enumerate(qs):
        cnt, rids, _ = L.evaluate(gpu_ctx, [idx.term(lo, hi)])
        assert cnt == ref[q][0], q
        assert np.array_equal(rids, ref[q][1]), q
        assert np.array_equal(rids, _scan(vals, lo, hi)), q


def test_conjunctions_and_batch_equal_scan(gpu_ctx):
    """AND of 1-4 range terms over four 1M-row columns (two relic, two
    bin), as one batch and one query at a time."""
    import libfastlib_b200 as L
    rng = np.random.default_rng(11)
    n = 1 << 20
    c0 = rng.integers(0, 1000, size=n).astype(np.uint32)
    c1 = (rng.zipf(1.1, size=n) % 5000).astype(np.uint32)
    c2 = rng.normal(size=n).astype(np.float32)
    c3 = np.where(rng.random(n) < 0.7, rng.normal(size=n), rng.zipf(1.2, size=n) % 100000).astype(np.float32)
    k0 = _relic_ref(c0, [])[:3]
    k1 = _relic_ref(c1, [])[:3]
    k2 = _bin_ref(c2, 512, [])[:3]
    k3 = _bin_ref(c3, 256, [])[:3]
    cols = [(c0, L.RELIC, k0), (c1, L.RELIC, k1), (c2, L.BIN, k2), (c3, L.BIN, k3)]
    idxs = [L.Index(gpu_ctx, kind, n, *k, values=c) for c, kind, k in cols]
    queries, specs = [], []
    for _ in range(60):
        cs = rng.choice(4, size=int(rng.integers(1, 5)), replace=False)
        terms, spec = [], []
        for ci in cs:
            v = cols[ci][0].astype(np.float64)
            lo, hi = np.sort(rng.choice(v, size=2))
            if lo == hi:
                hi = lo + 1
            terms.append(idxs[ci].term(lo, hi))
            spec.append((ci, lo, hi))
        queries.append(terms)
        specs.append(spec)
    expect = []
    for spec in specs:
        m = np.ones(n, dtype=bool)
        for ci, lo, hi in spec:
            v = cols[ci][0].astype(np.float64)
            m &= (v >= lo) & (v < hi)
        expect.append(np.flatnonzero(m).astype(np.uint32))
    B = L.Batch(gpu_ctx, queries, rid_cap=sum(len(e) for e in expect))
    B.run()
    counts = B.counts()
    for q, e in enumerate(expect):
        assert int(counts[q]) == len(e), q
        assert np.array_equal(B.rids(q, len(e)), e), q
    for q in range(0, 60, 7):
        cnt, rids, _ = L.evaluate(gpu_ctx, queries[q])
        assert cnt == len(expect[q]) and np.array_equal(rids, expect[q])


def test_hit_bitvector_is_compressed_result(gpu_ctx):
    """The hit bitvector of an evaluation holds the hit rows, in the words
    compress() gives for them."""
    import libfastlib_b200 as L
    g = load_golden("relic_small.npz")
    idx = L.Index(gpu_ctx, L.RELIC, len(g["vals"]), g["keys"], g["offsets"], g["bitmaps"], values=g["vals"])
    n, rids, hits = L.evaluate(gpu_ctx, [idx.term(10, 60)], want_hits=True)
    assert hits.size() == len(g["vals"])
    assert hits.cnt() == n
    assert np.array_equal(hits.rids(), rids)
    dense = oracle.decompress(hits.write())
    assert np.array_equal(oracle.compress(dense)[0], hits.write())


def test_relic_all_comparisons_and_orders(gpu_ctx):
    """Every operator pair on a relic index (binary-search locate) and both
    batch work orders give the scan's counts."""
    import libfastlib_b200 as L
    rng = np.random.default_rng(21)
    n = 200_003
    vals = rng.integers(0, 5000, n).astype(np.uint32)
    idx = L.Index.build(gpu_ctx, L.RELIC, vals)
    bidx = L.Index.build(gpu_ctx, L.BIN, rng.normal(0, 1, n).astype(np.float32), nbins=64)
    f = vals.astype(np.float64)
    ops = [(L.CMP_NONE, L.CMP_LT), (L.CMP_LT, L.CMP_LE), (L.CMP_LE, L.CMP_NONE), (L.CMP_LE, L.CMP_LE), (L.CMP_LT, L.CMP_LT)]
    queries, want = [], []
    for i in range(60):
        lo, hi = sorted(rng.integers(-5, 5005, 2).astype(float) + rng.choice([0.0, 0.5]))
        lop, rop = ops[i % len(ops)]
        m = np.ones(n, bool)
        if lop == L.CMP_LT: m &= lo < f
        if lop == L.CMP_LE: m &= lo <= f
        if rop == L.CMP_LT: m &= f < hi
        if rop == L.CMP_LE: m &= f <= hi
        t = idx.term(lo if lop else None, hi if rop else None, lop=lop or L.CMP_LE, rop=rop or L.CMP_LT)
        c, rids, _ = L.evaluate(gpu_ctx, [t])
        assert c == m.sum() and np.array_equal(rids, np.flatnonzero(m)), (i, lo, hi, lop, rop)
        queries.append([t, bidx.term(-0.5, 0.7)] if i % 2 else [t])
        want.append(c if i % 2 == 0 else None)
    B = L.Batch(gpu_ctx, queries, 0)
    try:
        for order in (0, 1):
            gpu_ctx.set_tuning(L.TUNE_RANGE_ORDER, order)
            for ctas in (0, 1):
                gpu_ctx.set_tuning(L.TUNE_RANGE_CTAS, ctas)
                B.run()
                got = B.counts()
                if order == 0 and ctas == 0:
                    ref = got.copy()
                assert np.array_equal(got, ref), (order, ctas)
        assert all(int(ref[i]) == w for i, w in enumerate(want) if w is not None)
    finally:
        gpu_ctx.set_tuning(L.TUNE_RANGE_ORDER, 1)
        gpu_ctx.set_tuning(L.TUNE_RANGE_CTAS, 0)


def test_cumulative_rows_any_stride(gpu_ctx):
    """Indexes built with cumulative rows of several strides (and none)
    give the scan's row ids: relic over a random and over a sorted column,
    bin over a mixture, with ragged last groups."""
    import libfastlib_b200 as L
    rng = np.random.default_rng(5)
    n = 300_007
    cols = [
        (L.RELIC, rng.integers(0, 3000, n).astype(np.uint32), {}),
        (L.RELIC, np.sort(rng.integers(0, 700, n)).astype(np.uint32), {}),
        (L.BIN, np.where(rng.random(n) < 0.6, rng.normal(size=n), rng.zipf(1.3, size=n) % 5000).astype(np.float32),
         {"nbins": 400}),
    ]
    try:
        for kind, vals, kw in cols:
            f = vals.astype(np.float64)
            sv = np.sort(f)
            spans = []
            for i in range(24):
                a, b = sorted(rng.integers(0, n, 2))
                lo, hi = sv[a], sv[b]
                if i % 3 == 0:
                    lo, hi = sv[0] - 1, sv[b]  # from below the smallest key
                if i % 5 == 0:
                    hi = sv[-1] + 1           # to above the largest
                spans.append((float(lo), float(hi) + (0.5 if i % 2 else 0.0)))
            want = [np.flatnonzero((f >= lo) & (f < hi)) for lo, hi in spans]
            # 40 and 300: edge spans wider than the direct walk, taken from
            # the tile lists
            for stride in (1, 2, 3, 8, 40, 300, 0):
                gpu_ctx.set_tuning(L.TUNE_CUM_STRIDE, stride)
                idx = L.Index.build(gpu_ctx, kind, vals, **kw)
                B = L.Batch(gpu_ctx, [[idx.term(lo, hi)] for lo, hi in spans], rid_cap=sum(len(w) for w in want))
                B.run()
                counts = B.counts()
                for q, w in enumerate(want):
                    assert int(counts[q]) == len(w), (kind, stride, q)
                    assert np.array_equal(B.rids(q, len(w)), w), (kind, stride, q)
                del B, idx
    finally:
        gpu_ctx.set_tuning(L.TUNE_CUM_STRIDE, 0)


def test_row_id_orders_agree(gpu_ctx):
    """A batch with row ids gives the same counts, ids and per-query starts
    query by query (look-back) and in two tile-by-tile passes around a scan,
    at every resident-CTA setting; ids equal the scan's."""
    import libfastlib_b200 as L
    rng = np.random.default_rng(17)
    n = 1_000_003
    c0 = rng.integers(0, 800, n).astype(np.uint32)
    c1 = rng.normal(size=n).astype(np.float32)
    i0 = L.Index.build(gpu_ctx, L.RELIC, c0)
    i1 = L.Index.build(gpu_ctx, L.BIN, c1, nbins=300)
    queries, want = [], []
    for q in range(70):
        a, b = sorted(rng.integers(0, 801, 2))
        lo, hi = sorted(rng.normal(size=2))
        if q % 10 == 3:
            a, b = 900, 901  # no hits
        terms = [i0.term(float(a), float(b) + 0.5)] + ([i1.term(float(lo), float(hi))] if q % 3 else [])
        m = (c0 >= a) & (c0 < b + 0.5)
        if q % 3:
            m &= (c1.astype(np.float64) >= lo) & (c1.astype(np.float64) < hi)
        queries.append(terms)
        want.append(np.flatnonzero(m).astype(np.uint32))
    B = L.Batch(gpu_ctx, queries, rid_cap=sum(len(w) for w in want))
    try:
        for order in (0, 2):
            gpu_ctx.set_tuning(L.TUNE_RANGE_ORDER, order)
            for ctas in (0, 1, 3):
                gpu_ctx.set_tuning(L.TUNE_RANGE_CTAS, ctas)
                B.run()
                counts = B.counts()
                for q, w in enumerate(want):
                    assert int(counts[q]) == len(w), (order, ctas, q)
                    assert np.array_equal(B.rids(q, len(w)), w), (order, ctas, q)
    finally:
        gpu_ctx.set_tuning(L.TUNE_RANGE_ORDER, 1)
        gpu_ctx.set_tuning(L.TUNE_RANGE_CTAS, 0)
