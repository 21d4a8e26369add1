"""Indexes read from FastBit .idx files (written by the reference's own
relic::write / bin::write, tests/golden/make_idx_files.py) answer ranges
like a scan of the column they were built from, whichever way the file
reaches the library (path or image, 4- or 8-byte offsets)."""
import os

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _ranges(vals, n, seed):
    rng = np.random.default_rng(seed)
    sv = np.sort(vals.astype(np.float64))
    out = []
    for _ in range(n):
        a, b = sorted(rng.integers(0, len(sv), 2))
        out.append((float(sv[a]) + (0.5 if a % 3 == 0 else 0.0), float(sv[b]) + (0.25 if b % 2 else 0.0)))
    out.append((float(sv[0]) - 1.0, float(sv[-1]) + 1.0))  # every row
    out.append((float(sv[-1]) + 1.0, float(sv[-1]) + 2.0))  # none
    return out


@pytest.mark.parametrize("name,kind", [("relic_3001", "relic"), ("bin_5000", "bin")])
@pytest.mark.parametrize("suffix", ["", "_o64"])
@pytest.mark.parametrize("how", ["path", "image"])
def test_index_file_ranges_equal_scan(gpu_ctx, name, kind, suffix, how):
    import libfastlib_b200 as L
    g = load_golden("idxfile_inputs.npz")
    vals = g[f"{kind}_vals"]
    path = os.path.join(GOLD, f"{name}{suffix}.idx")
    if how == "path":
        idx = L.Index.read(gpu_ctx, path, values=vals)
    else:
        with open(path, "rb") as f:
            idx = L.Index.from_file_image(gpu_ctx, f.read(), values=vals)
    assert idx.nrows == len(vals)
    f64 = vals.astype(np.float64)
    qs = _ranges(vals, 30, 7)
    want = [np.flatnonzero((f64 >= lo) & (f64 < hi)).astype(np.uint32) for lo, hi in qs]
    B = L.Batch(gpu_ctx, [[idx.term(lo, hi)] for lo, hi in qs], rid_cap=sum(len(w) for w in want))
    B.run()
    counts = B.counts()
    for q, w in enumerate(want):
        assert int(counts[q]) == len(w), q
        assert np.array_equal(B.rids(q, len(w)), w), q
    n, rids, _ = L.evaluate(gpu_ctx, [idx.term(*qs[3])])
    assert n == len(want[3]) and np.array_equal(rids, want[3])
    idx.close()


def test_missing_and_malformed_files(gpu_ctx, tmp_path):
    import libfastlib_b200 as L
    with pytest.raises(L.WahError) as e:
        L.Index.read(gpu_ctx, str(tmp_path / "absent.idx"))
    assert e.value.code == -1
    bad = tmp_path / "bad.idx"
    bad.write_bytes(b"#IBIS\x03\x04\x00" + b"\0" * 64)
    with pytest.raises(L.WahError) as e:
        L.Index.read(gpu_ctx, str(bad))
    assert e.value.code == -5
