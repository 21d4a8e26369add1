"""The serving loop (wahgpu_server_*): every query's answer in a continuous
batching mix — several batches in flight, admission held back by a small
scratch budget, requests arriving while others run — equals its answer
evaluated alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _columns(ctx, n):
    import torch
    import libfastlib_b200 as L
    from libfastlib_b200 import workloads as W
    cols = [
        (L.Index.build(ctx, L.RELIC, W.uniform_int_column(1, n, 1000)), {"kind": "relic", "card": 1000}),
        (L.Index.build(ctx, L.RELIC, W.zipf_column(2, n, 1.1, 100_000).to(torch.int32)), {"kind": "relic", "card": 100_000}),
        (L.Index.build(ctx, L.BIN, W.normal_column(3, n), nbins=256), None),
        (L.Index.build(ctx, L.BIN, W.mixture_column(4, n), nbins=256), None),
    ]
    out = []
    for idx, meta in cols:
        if meta is None:
            meta = {"kind": "bin", "keys": idx.keys(), "nobs": idx.nbitmaps(), "max_span": 128}
        out.append((idx, meta))
    return out


def test_server_results_equal_alone(gpu_ctx):
    import libfastlib_b200 as L
    from libfastlib_b200 import workloads as W
    n = 2_000_003
    cols = _columns(gpu_ctx, n)
    qs = W.conjunctive_queries(6, [m for _, m in cols], 240, max_terms=4)
    queries = [[cols[c][0].term(lo, hi) for c, lo, hi in q] for q in qs]
    alone = [L.evaluate(gpu_ctx, q, want_rids=(i % 3 == 0)) for i, q in enumerate(queries)]
    # tiny budget: a few queries per batch, the rest wait for scratch
    S = L.Server(gpu_ctx, nslots=3, max_batch=8, scratch_budget=8 * (n // 31 // 4096 + 1) * 48 + 64 * n)
    try:
        ids = [S.submit(q, rid_cap=(n if i % 3 == 0 else 0)) for i, q in enumerate(queries)]
        for i, rid in enumerate(ids):
            c, rids, lat = S.wait(rid, rid_cap=(n if i % 3 == 0 else 0))
            assert c == alone[i][0], i
            if i % 3 == 0:
                assert np.array_equal(rids, alone[i][1]), i
            assert lat > 0
        batches, served = S.stats()
        assert served == len(queries) and batches >= len(queries) // 8
        # open loop: Poisson arrivals while earlier batches run
        rng = np.random.default_rng(7)
        arrival = np.cumsum(rng.exponential(1 / 20_000, len(queries)))
        counts, lat, wall, _ = S.replay(queries, arrival)
        assert [int(c) for c in counts] == [a[0] for a in alone]
        assert np.all(lat > 0) and wall > 0
        # with the first 500 row ids of every query (each query its own
        # region, so queries with many hits leave the others theirs)
        counts, lat, wall, ids = S.replay(queries, arrival, rid_cap=500)
        assert [int(c) for c in counts] == [a[0] for a in alone]
        for i, q in enumerate(queries):
            want = alone[i][1] if alone[i][1] is not None else L.evaluate(gpu_ctx, q)[1]
            assert np.array_equal(ids[i], want[:500]), i
    finally:
        S.close()


def test_server_refuses_oversized_request(gpu_ctx):
    import libfastlib_b200 as L
    idx = L.Index.build(gpu_ctx, L.RELIC, np.arange(100_000, dtype=np.uint32) % 10)
    S = L.Server(gpu_ctx, nslots=1, max_batch=4, scratch_budget=1 << 16)
    try:
        with pytest.raises(L.WahError) as e:
            S.submit([idx.term(0, 5)], rid_cap=1 << 20)
        assert e.value.code == -10
        c, _, _ = S.wait(S.submit([idx.term(0, 5)]))
        assert c == 50_000
    finally:
        S.close()


@pytest.mark.parametrize("order", [0, 2])
def test_capped_batch_row_ids(gpu_ctx, order):
    """wahgpu_batch_create_capped: every query keeps its first caps[q] row
    ids in a region of its own; counts stay complete (query by query with
    the segmented look-back, and tile by tile with a count pass, a scan and
    an id pass that revisits only the items under each query's limit)."""
    import libfastlib_b200 as L
    from libfastlib_b200 import workloads as W
    n = 1_000_003
    cols = _columns(gpu_ctx, n)
    qs = W.conjunctive_queries(9, [m for _, m in cols], 64, max_terms=3)
    queries = [[cols[c][0].term(lo, hi) for c, lo, hi in q] for q in qs]
    caps = [0 if i % 5 == 0 else (1 + 97 * i) for i in range(len(queries))]
    old = gpu_ctx.get_tuning(L.TUNE_RANGE_ORDER)
    gpu_ctx.set_tuning(L.TUNE_RANGE_ORDER, order)
    try:
        B = L.Batch(gpu_ctx, queries, caps=caps)
        B.run()
        counts = B.counts()
        for i, q in enumerate(queries):
            c, rids, _ = L.evaluate(gpu_ctx, q)
            assert int(counts[i]) == c, i
            got = B.rids(i, min(c, caps[i]))
            assert np.array_equal(got, rids[:caps[i]]), i
        B.close()
    finally:
        gpu_ctx.set_tuning(L.TUNE_RANGE_ORDER, old)
