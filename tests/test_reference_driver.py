"""The reference driver's query requests (oracle/reference.py), on the CPU:
the in-memory C API on attached index triples (request 12), relic
evaluation (requests 13 and 14) and the appendFill-built operator pairs
(request 11) give the answers of a double-precision scan or of the C
oracle, with one thread and with several.  These requests time the
reference in bench.py and pin the GPU's answers at full size, so they are
checked here first.  Needs the reference built from source (oracle/_ref)."""
import numpy as np
import pytest

import oracle
from oracle import reference as R
from oracle import wahgen as G

pytestmark = pytest.mark.skipif(not R.available(), reason="reference build (oracle/_ref) absent")


def _scan(cols, q):
    m = np.ones(len(cols[0]), bool)
    for c, lo, hi in q:
        v = cols[c].astype(np.float64)
        m &= (v >= lo) & (v < hi)
    return np.flatnonzero(m).astype(np.uint32)


def test_iapi_conjunctions_on_attached_triples():
    rng = np.random.default_rng(12)
    n = 200_000
    c0 = rng.integers(0, 100, size=n).astype(np.uint32)
    c1 = np.where(rng.random(n) < 0.7, rng.normal(size=n), rng.zipf(1.2, size=n) % 1000).astype(np.float32)
    t0 = R.relic_triple(c0)
    t1, _ = R.bin_index(c1, 64)
    qs = []
    for _ in range(60):
        q = []
        if rng.random() < 0.7:
            lo = int(rng.integers(0, 90))
            q.append((0, float(lo), float(lo + rng.integers(1, 10))))
        if rng.random() < 0.7 or not q:
            a = float(rng.normal())
            q.append((1, a, a + float(rng.random())))
        qs.append(q)
    for nth in (1, 4):
        secs, counts, ids = R.iapi_queries([(c0, t0), (c1, t1)], qs, nthreads=nth, reps=1, rids=True)
        assert secs > 0 and len(R.latencies()) == len(qs)
        for i, q in enumerate(qs):
            want = _scan([c0, c1], q)
            assert counts[i] == len(want)
            assert np.array_equal(ids[i], want)


def test_relic_timed_counts():
    rng = np.random.default_rng(13)
    v = rng.integers(0, 100, size=100_000).astype(np.uint32)
    qs = [(10.0, 20.0), (0.0, 100.0), (50.0, 51.0), (99.0, 100.0)]
    for nth in (1, 3):
        secs, counts = R.relic_timed(v, qs, nthreads=nth, reps=2)
        assert secs > 0
        assert counts == [int(np.sum((v >= lo) & (v < hi))) for lo, hi in qs]


def test_relic_every_comparison_pair_equals_the_scan():
    """Request 14: the reference's relic::evaluate for every operator pair
    the GPU tests use (x < b, a < x <= b, a <= x, a <= x <= b, a < x < b),
    with bounds below, inside and above the values, whole and halfway
    between keys, negative strict lower bounds among them, gives exactly
    the double-precision scan that the GPU's range results are compared
    with (count and row ids)."""
    rng = np.random.default_rng(14)
    n = 50_003
    v = rng.integers(0, 500, size=n).astype(np.uint32)
    v[:10] = 0  # the value 0 is present, for the negative strict bounds
    f = v.astype(np.float64)
    pairs = [(0, 1), (1, 2), (2, 0), (2, 2), (1, 1)]
    qs = [(-3.0, 1, 99.0, 1), (-0.5, 1, 0.5, 2), (0.0, 1, 10.0, 1), (-5.0, 2, 0.0, 2)]
    for k in range(80):
        lo, hi = sorted(rng.integers(-5, 505, 2).astype(float) + rng.choice([0.0, 0.5]))
        lop, rop = pairs[k % len(pairs)]
        qs.append((lo, lop, hi, rop))
    got = R.relic_compare(v, qs)
    for (lo, lop, hi, rop), (cnt, rids) in zip(qs, got):
        m = np.ones(n, bool)
        if lop == 1: m &= lo < f
        if lop == 2: m &= lo <= f
        if rop == 1: m &= f < hi
        if rop == 2: m &= f <= hi
        assert cnt == int(m.sum()), (lo, lop, hi, rop)
        assert np.array_equal(rids, np.flatnonzero(m).astype(np.uint32)), (lo, lop, hi, rop)


@pytest.mark.parametrize("density", [1e-3, 0.1, 0.5])
def test_runs_pair_all_ops_equal_oracle(density):
    from libfastlib_b200 import workloads as W
    ra = W.geometric_runs(1, 1 << 20, density)
    rb = W.geometric_runs(2, 1 << 20, density)
    a, b, res = R.runs_pair_all_ops(ra, rb)
    assert np.array_equal(a, oracle.build_runs(ra))
    assert np.array_equal(b, W.raw_wah_operand(2, 1 << 20, density))
    for op in range(4):
        for ip in range(2):
            w, c = oracle.binop(op, a, b, inplace=bool(ip))
            st, cnt, words = res[2 * op + ip]
            assert st == 0 and cnt == c and np.array_equal(words, w), (op, ip)
