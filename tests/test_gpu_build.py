"""Indexes built on the device (wahgpu_index_build): every bitmap holds
exactly the rows of its value (relic) or bin, in compress() form, and range
queries over them return the reference library's answers."""
import numpy as np
import pytest

import oracle
from conftest import load_golden
from test_gpu_range import _bin_ref, _relic_ref, _scan

pytestmark = pytest.mark.gpu

ALL = 0x7FFFFFFF


def canonical_words(rows, nrows):
    """Serialized compress()-form bitvector of the given ascending rows."""
    G, anb = nrows // 31, nrows % 31
    pats = np.zeros(G, dtype=np.int64)
    aval = 0
    for r in rows:
        g, k = divmod(int(r), 31)
        if g < G:
            pats[g] |= 1 << (30 - k)
        else:
            aval |= 1 << (anb - 1 - k)
    out, i = [], 0
    while i < G:
        v = int(pats[i])
        if v in (0, ALL):
            j = i
            while j < G and pats[j] == v:
                j += 1
            n = j - i
            out.append(((0xC0000000 if v else 0x80000000) | n) if n >= 2 else v)
            i = j
        else:
            out.append(v)
            i += 1
    if anb:
        out.append(aval)
    out.append(anb)
    return np.array(out, dtype=np.uint32)


def unpacked_words(words, nrows):
    """index::optionalUnpack's default rule (src/index.cpp:8838-8853) on a
    serialized bitvector of nrows rows: when m_vec's bytes plus
    sizeof(ibis::bitvector) (40) exceed max(nrows / 9, 52), every fill
    becomes its literals."""
    w = np.asarray(words, np.uint32)
    tail = w[-2:] if 0 < w[-1] < 31 else w[-1:]
    body = w[: len(w) - len(tail)]
    G = nrows // 31
    if len(body) * 4 + 40 <= max(nrows // 9, 52) or len(body) == G:
        return w
    out = []
    for x in body:
        x = int(x)
        if x > ALL:
            out.extend([ALL if x >= 0xC0000000 else 0] * (x & 0x3FFFFFFF))
        else:
            out.append(x)
    return np.concatenate([np.asarray(out, np.uint32), tail])


@pytest.mark.parametrize("nrows", [1, 30, 31, 62, 1000, 100003])
def test_relic_build_bitmaps(gpu_ctx, nrows):
    import libfastlib_b200 as L
    rng = np.random.default_rng(nrows)
    card = max(1, min(50, nrows // 3))
    vals = rng.integers(0, card, nrows).astype(np.uint32)
    # a long run of one value: all-1 groups and their fills
    if nrows > 200:
        vals[40:200] = 7
    idx = L.Index.build(gpu_ctx, L.RELIC, vals)
    keys = idx.keys()
    uniq = np.unique(vals)
    assert np.array_equal(keys, uniq.astype(np.float64))
    for j, v in enumerate(uniq):
        rows = np.flatnonzero(vals == v).astype(np.uint32)
        bv = idx.bitmap(j)
        assert np.array_equal(bv.rids(), rows), v
        assert np.array_equal(bv.write(), unpacked_words(canonical_words(rows, nrows), nrows)), v
        assert bv.cnt() == len(rows)


def test_bin_build_partition(gpu_ctx):
    import libfastlib_b200 as L
    rng = np.random.default_rng(3)
    n = 500_000
    vals = np.where(rng.random(n) < 0.7, rng.normal(0, 1, n),
                    (rng.zipf(1.2, n) % 1000).astype(np.float64)).astype(np.float32)
    nbins = 100
    idx = L.Index.build(gpu_ctx, L.BIN, vals, nbins=nbins)
    nb = idx.nbitmaps()
    keys = idx.keys()
    lo, hi = keys[:nb], keys[nb:]
    assert nb <= nbins + 1 and np.all(lo <= hi) and np.all(hi[:-1] < lo[1:])
    seen = 0
    for j in range(nb):
        rows = np.flatnonzero((vals >= lo[j]) & (vals <= hi[j])).astype(np.uint32)
        assert np.array_equal(idx.bitmap(j).rids(), rows), j
        seen += len(rows)
        # equal weight: a bin exceeds its share only when one value does
        if len(rows) > 2 * n / nbins:
            assert lo[j] == hi[j]
    assert seen == n


def test_built_indexes_answer_like_reference(gpu_ctx):
    """Relic over the small golden column and a bin index over a float32
    mixture: counts and row ids equal the reference library's evaluate()."""
    import libfastlib_b200 as L
    g = load_golden("relic_small.npz")
    vals = g["vals"].astype(np.uint32)
    idx = L.Index.build(gpu_ctx, L.RELIC, vals)
    for q, (lo, hi) in enumerate(g["queries"]):
        n, rids, _ = L.evaluate(gpu_ctx, [idx.term(lo, hi)])
        assert n == int(g["counts"][q]) and np.array_equal(rids, _scan(vals, lo, hi))

    rng = np.random.default_rng(11)
    n = 300_000
    fv = np.where(rng.random(n) < 0.7, rng.normal(0, 1, n),
                  (rng.zipf(1.2, n) % 10_000).astype(np.float64)).astype(np.float32)
    queries = []
    srt = np.sort(fv)
    for _ in range(40):
        a, b = sorted(rng.integers(0, n, 2))
        queries.append((float(srt[a]) + 1e-3, float(srt[b]) + 1e-3))
    _k, _o, _b, ref = _bin_ref(fv, 200, queries)
    bidx = L.Index.build(gpu_ctx, L.BIN, fv, nbins=200)
    for q, (lo, hi) in enumerate(queries):
        c, rids, _ = L.evaluate(gpu_ctx, [bidx.term(lo, hi)])
        assert c == ref[q][0] and np.array_equal(rids, ref[q][1]), q


@pytest.mark.parametrize("card,nrows", [(100, 1_000_000), (7, 99_999), (1000, 200_000), (3, 310_001)])
def test_relic_build_equals_relic_construct(gpu_ctx, card, nrows):
    """The device-built relic index is word for word the reference's
    relic::construct (src/irelic.cpp:879-925: mapValues, then
    optionalUnpack's default decompression of heavy bitmaps): the same
    keys, offsets and serialized bitmaps as relic::write(keys, offs, bms)."""
    import libfastlib_b200 as L
    from oracle import reference as R
    if not R.available():
        pytest.skip("reference build (oracle/_ref) absent")
    rng = np.random.default_rng(card)
    vals = rng.integers(0, card, size=nrows).astype(np.uint32)
    keys, offs, bms = R.relic_triple(vals)
    idx = L.Index.build(gpu_ctx, L.RELIC, vals)
    k, o, b = idx.deconstruct()
    assert np.array_equal(k, keys)
    assert np.array_equal(o, offs)
    assert np.array_equal(b, bms)
