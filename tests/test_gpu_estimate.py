"""index::estimate on the GPU (wahgpu_estimate, wahgpu_estimate_count):
for relic the lower bound is the exact hit set and upper is empty
(src/irelic.h:58-62); for bin the lower bound is the OR of the bins whose
values all pass, the upper bound adds the edge bins (src/ibin.cpp:6722-6829)
and the count bound is the 1 bits of those bins (6832-6889).  Checked
against the golden indexes' keys and a scan of the raw values."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def test_relic_estimate_is_exact(gpu_ctx):
    import libfastlib_b200 as L
    g = load_golden("relic_small.npz")
    idx = L.Index(gpu_ctx, L.RELIC, len(g["vals"]), g["keys"], g["offsets"], g["bitmaps"])
    v = g["vals"].astype(np.float64)
    for lo, hi in g["queries"]:
        want = np.flatnonzero((v >= lo) & (v < hi)).astype(np.uint32)
        lower, upper = L.estimate(gpu_ctx, idx.term(lo, hi))
        assert np.array_equal(lower.rids(), want)
        assert upper.size() == 0
        assert L.estimate_count(gpu_ctx, idx.term(lo, hi)) == len(want)


def test_bin_estimate_bounds(gpu_ctx):
    import libfastlib_b200 as L
    g = load_golden("bin_small.npz")
    keys = g["keys"]
    nobs = len(keys) // 2
    mn, mx = keys[:nobs], keys[nobs:]
    idx = L.Index(gpu_ctx, L.BIN, len(g["vals"]), keys, g["offsets"], g["bitmaps"])  # no raw values needed
    v = g["vals"].astype(np.float64)
    binof = np.full(len(v), -1)  # the bin of every row, from the bitmaps
    for j in range(nobs):
        binof[idx.bitmap(j).rids()] = j
    assert (binof >= 0).all()
    for lo, hi in g["queries"]:
        hits = np.flatnonzero((v >= lo) & (v < hi)).astype(np.uint32)
        ones = [j for j in range(nobs) if np.any(binof == j)]
        inside = [j for j in ones if lo <= mn[j] and mx[j] < hi]
        some = [j for j in ones if j not in inside and not (mx[j] < lo or mn[j] >= hi)]
        want_lower = np.flatnonzero(np.isin(binof, inside)).astype(np.uint32)
        lower, upper = L.estimate(gpu_ctx, idx.term(lo, hi))
        assert np.array_equal(lower.rids(), want_lower)
        bound = L.estimate_count(gpu_ctx, idx.term(lo, hi))
        if some:
            want_upper = np.flatnonzero(np.isin(binof, inside + some)).astype(np.uint32)
            assert np.array_equal(upper.rids(), want_upper)
            assert bound == len(want_upper)
        else:
            assert upper.size() == 0
            assert np.array_equal(lower.rids(), hits)
            assert bound == len(hits)
        assert set(want_lower.tolist()) <= set(hits.tolist()) and bound >= len(hits)
