"""WHERE clauses through libfastlib_b200.query.where on device-built
indexes: counts and row ids equal numpy scans of the columns, for AND-only
clauses (one fused evaluation) and for OR / NOT trees."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_where_equals_scan(gpu_ctx):
    import libfastlib_b200 as L
    from libfastlib_b200.query import QueryError, where
    rng = np.random.default_rng(31)
    n = 200_003
    ca = rng.integers(0, 100, n).astype(np.uint32)
    cb = rng.normal(0, 1, n).astype(np.float32)
    cols = {"a": L.Index.build(gpu_ctx, L.RELIC, ca), "b": L.Index.build(gpu_ctx, L.BIN, cb, nbins=64)}
    fa, fb = ca.astype(np.float64), cb.astype(np.float64)
    cases = [
        ("a >= 10 and a < 20", (fa >= 10) & (fa < 20)),
        ("a between 5 and 7 and b < 0.5", (fa >= 5) & (fa <= 7) & (fb < 0.5)),
        ("a < 5 or b < -1", (fa < 5) | (fb < -1)),
        ("not a < 50", ~(fa < 50)),
        ("a != 42 and b < 0", (fa != 42) & (fb < 0)),
        ("(a < 10 or a >= 90) and not (b between -0.5 and 0.5)",
         ((fa < 10) | (fa >= 90)) & ~((fb >= -0.5) & (fb <= 0.5))),
        ("!(a >= 3) || b > 2", ~(fa >= 3) | (fb > 2)),
        ("a < 20 and (b < -1 or b > 1) and a >= 10", (fa < 20) & ((fb < -1) | (fb > 1)) & (fa >= 10)),
        ("90 <= a", fa >= 90),
        ("a in (3, 17, 42) and b > 0", np.isin(fa, [3, 17, 42]) & (fb > 0)),
    ]
    for clause, m in cases:
        cnt, rows = where(gpu_ctx, clause, cols)
        assert cnt == int(m.sum()), clause
        assert np.array_equal(rows, np.flatnonzero(m)), clause
    with pytest.raises(QueryError):
        where(gpu_ctx, "c < 3", cols)
