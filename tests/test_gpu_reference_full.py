"""Parity at the workloads' full sizes, against the reference library
itself where that is feasible and a double-precision scan of the raw values
elsewhere.

* Raw WAH: for every density both 2^28-bit operands are built by the
  reference's own appendFill (src/bitvector.h:800) from the seeded run
  lengths, and the reference computes a OP b and a OP= b for & | ^ -
  followed by compress() (src/bitvector.cpp:1194-1838, 378-469).  The GPU's
  words and cnt() equal the reference's, and the operands equal the ones
  the benchmark builds on the device.
* Binned range: 100M float32 rows on the reference's own 1000-bin index.
* Batched and served conjunctions: 8 x 50M and 16 x 200M rows, counts of
  every query from one batch, a sample checked row by row.
The reference runs through oracle/_ref/refdrv (compiled from its sources).
"""
import os

import numpy as np
import pytest

import oracle
from oracle import reference as R

pytestmark = pytest.mark.gpu

NBITS = 1 << 28
needs_ref = pytest.mark.skipif(not os.path.exists(oracle.REFDRV), reason="reference build (oracle/_ref) absent")


@needs_ref
@pytest.mark.parametrize("density", [1e-4, 1e-3, 1e-2, 0.1, 0.5])
def test_raw_wah_full_size_against_reference(gpu_ctx, density):
    from libfastlib_b200 import workloads as W
    from libfastlib_b200.replicas import operand_seeds
    k = [1e-4, 1e-3, 1e-2, 0.1, 0.5].index(density)
    sa, sb = operand_seeds(0, 5)[k]
    runs_a = W.geometric_runs(sa, NBITS, density)
    runs_b = W.geometric_runs(sb, NBITS, density)
    a, b, res = R.runs_pair_all_ops(runs_a, runs_b)
    # the benchmark's operands (built on the device) are the reference's
    assert np.array_equal(W.raw_wah_operand(sa, NBITS, density, "cuda"), a)
    assert np.array_equal(W.raw_wah_operand(sb, NBITS, density, "cuda"), b)
    A, B = gpu_ctx.bitvector(a), gpu_ctx.bitvector(b)
    for op in range(4):
        for ip in (0, 1):
            st, cnt, words = res[2 * op + ip]
            assert st == 0
            r = A._binop(op, B, bool(ip))
            assert r.cnt() == cnt, (density, op, ip)
            assert np.array_equal(r.write(), words), (density, op, ip)


def _sorted_counts(sv, qs):
    """Exact hit counts of lo <= x < hi from the column sorted in double."""
    lo = np.array([q[0] for q in qs])
    hi = np.array([q[1] for q in qs])
    return np.searchsorted(sv, hi, side="left") - np.searchsorted(sv, lo, side="left")


@needs_ref
def test_binned_range_full_size_on_reference_index(gpu_ctx):
    """The binned range workload at full size on the reference's own index:
    100M float32 rows (70% Normal(0,1), 30% Zipf(1.2) over 1e5 ranks), the
    index built by the reference (fastbit_iapi_build_index with
    <binning nbins=1000 equal_weight/>, exported by
    fastbit_iapi_deconstruct_index) and attached on the GPU; the 1000
    ranges of 1-500 bins with both ends inside edge bins.  All 1000 counts
    equal exact counts from the sorted column; for a sample of queries the
    counts and row ids equal the reference's own answers (its in-memory C
    API on that same triple)."""
    import libfastlib_b200 as L
    from libfastlib_b200 import workloads as W
    n = 100_000_000
    vals = W.mixture_column(3, n).cpu().numpy()
    (keys, offs, bms), _ = R.bin_index(vals, 1000)
    nobs = len(offs) - 1
    assert len(keys) == 2 * nobs
    idx = L.Index(gpu_ctx, L.BIN, n, keys, offs, bms, values=vals)
    qs = W.binned_range_queries(5, keys, nobs, 1000, 500)
    B = L.Batch(gpu_ctx, [[idx.term(lo, hi)] for lo, hi in qs], 0)
    B.run()
    counts = [int(c) for c in B.counts()]
    B.close()
    sv = np.sort(vals.astype(np.float64))
    assert counts == [int(c) for c in _sorted_counts(sv, qs)]
    sample = list(range(0, 1000, 50))
    _s, ref_counts, ref_ids = R.iapi_queries([(vals, (keys, offs, bms))], [[(0, *qs[q])] for q in sample],
                                             rids=True)
    for k, q in enumerate(sample):
        assert ref_counts[k] == counts[q], q
        cnt, rids, _ = L.evaluate(gpu_ctx, [idx.term(*qs[q])])
        assert cnt == counts[q]
        assert np.array_equal(rids, ref_ids[k]), q
    idx.close()


def _conjunction_check(gpu_ctx, cols, host, queries, sample, with_reference):
    """Counts of every query from one batch; for the sample, counts and row
    ids against a double-precision scan of the raw columns and, when asked,
    counts against the reference's in-memory C API on the GPU-built indexes'
    triples."""
    import libfastlib_b200 as L
    B = L.Batch(gpu_ctx, [[cols[c].term(lo, hi) for c, lo, hi in q] for q in queries], 0)
    B.run()
    counts = [int(c) for c in B.counts()]
    B.close()
    for q in sample:
        m = np.ones(len(host[0]), bool)
        for c, lo, hi in queries[q]:
            v = host[c].astype(np.float64)
            m &= (v >= lo) & (v < hi)
        want = np.flatnonzero(m).astype(np.uint32)
        assert counts[q] == len(want), q
        cnt, rids, _ = L.evaluate(gpu_ctx, [cols[c].term(lo, hi) for c, lo, hi in queries[q]])
        assert cnt == len(want) and np.array_equal(rids, want), q
    if with_reference:
        used = sorted({c for q in sample for c, _, _ in queries[q]})
        pos = {c: k for k, c in enumerate(used)}
        triples = [(host[c], cols[c].deconstruct()) for c in used]
        _s, ref_counts, _ = R.iapi_queries(triples, [[(pos[c], lo, hi) for c, lo, hi in queries[q]] for q in sample])
        assert ref_counts == [counts[q] for q in sample]
    return counts


@needs_ref
def test_batched_conjunctions_full_size(gpu_ctx):
    """The batched workload at full size: 8 columns x 50M rows (3 uint32
    U{0..999} relic, 3 uint32 Zipf(1.1) over 1e6 relic, 2 float32 Normal
    with 512 equal-weight bins), 4096 WHERE clauses of 1-4 column ranges.
    All counts come from one fused batch; 24 queries are checked against a
    double-precision scan (counts and row ids) and against the reference's
    in-memory C API on the same indexes (counts)."""
    import torch
    import libfastlib_b200 as L
    from libfastlib_b200 import workloads as W
    n = 50_000_000
    cols, metas, host = [], [], []
    for c in range(3):
        v = W.uniform_int_column(40 + c, n, 1000)
        cols.append(L.Index.build(gpu_ctx, L.RELIC, v))
        metas.append({"kind": "relic", "card": 1000})
        host.append(v.cpu().numpy())
    for c in range(3):
        v = W.zipf_column(50 + c, n, 1.1, 1_000_000).to(torch.int32)
        cols.append(L.Index.build(gpu_ctx, L.RELIC, v))
        metas.append({"kind": "relic", "card": 1_000_000})
        host.append(v.cpu().numpy())
    for c in range(2):
        v = W.normal_column(60 + c, n)
        ix = L.Index.build(gpu_ctx, L.BIN, v, nbins=512)
        cols.append(ix)
        metas.append({"kind": "bin", "keys": ix.keys(), "nobs": ix.nbitmaps(), "max_span": 256})
        host.append(v.cpu().numpy())
    qs = W.conjunctive_queries(4, metas, 4096, max_terms=4)
    _conjunction_check(gpu_ctx, cols, host, qs, list(range(0, 4096, 171)), True)
    for ix in cols:
        ix.close()


def test_served_conjunctions_full_size(gpu_ctx):
    """The served workload's indexes at full size: 16 columns x 200M rows
    (4 int32 U{0..999} relic, 4 int32 Zipf(1.1) over 1e5 relic, 4 float32
    Normal and 4 float32 Normal/Zipf mixture with 1024 bins), 1-6-term
    conjunctions.  Counts of 2000 queries from one batch; 12 checked
    against a double-precision scan of the 200M-row columns (counts and row
    ids)."""
    import torch
    import libfastlib_b200 as L
    from libfastlib_b200 import workloads as W
    n = 200_000_000
    cols, metas, host = [], [], []
    for c in range(16):
        seed = 5 + c
        if c < 4:
            v = W.uniform_int_column(seed, n, 1000)
            ix = L.Index.build(gpu_ctx, L.RELIC, v)
            metas.append({"kind": "relic", "card": 1000})
        elif c < 8:
            v = W.zipf_column(seed, n, 1.1, 100_000).to(torch.int32)
            ix = L.Index.build(gpu_ctx, L.RELIC, v)
            metas.append({"kind": "relic", "card": 100_000})
        else:
            v = W.normal_column(seed, n) if c < 12 else W.mixture_column(seed, n)
            ix = L.Index.build(gpu_ctx, L.BIN, v, nbins=1024)
            metas.append({"kind": "bin", "keys": ix.keys(), "nobs": ix.nbitmaps(), "max_span": 512})
        cols.append(ix)
        host.append(v.cpu().numpy())
        del v
    qs = W.conjunctive_queries(1600, metas, 2000, max_terms=6)
    _conjunction_check(gpu_ctx, cols, host, qs, list(range(0, 2000, 167)), False)
    for ix in cols:
        ix.close()
