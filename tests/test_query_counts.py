"""The WHERE-clause grammar and range semantics against the reference's own
known answers: the hit counts of its tests/scripts/query-count.list over
tests/test0.csv and tests/test1.csv (fixture: tests/golden/query_counts.json,
made by tests/golden/make_query_counts.py).

Each clause goes through libfastlib_b200.query.parse with stand-in columns
whose term() records (lo, lop, hi, rop) as Index.term does, and the parsed
tree is evaluated by a numpy scan in double precision; a NULL field
satisfies no condition.  Clauses with arithmetic on columns (sqrt, log,
exp, **, *) are outside the grammar (the path takes range conditions) and
must be refused with QueryError.  No device is involved.
"""
import json
import os

import numpy as np
import pytest

from libfastlib_b200 import CMP_LE, CMP_LT, CMP_NONE
from libfastlib_b200.query import QueryError, parse

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "query_counts.json")

# Strict lower bounds below zero: the reference's count leaves out the row
# whose value is 0 (98 of the 99 values 0..98 in each case); a
# qContinuousRange "-3 < x < 99" holds for 0, and so does every evaluation
# here.  Where the reference loses that row was not traced; it is not
# reproduced.
REFERENCE_DROPS_ZERO = {"-3 < i0 < 99", "-4 < i1 < 99", "-5 < i2 < 99"}


class _Col:
    def __init__(self, values):
        self.v = np.array([np.nan if x is None else x for x in values], dtype=np.float64)

    def term(self, lo=None, hi=None, lop=CMP_LE, rop=CMP_LT):
        return (self.v, CMP_NONE if lo is None else lop, lo, CMP_NONE if hi is None else rop, hi)


def _mask(node):
    kind = node[0]
    if kind == "leaf":
        v, lop, lo, rop, hi = node[1]
        m = ~np.isnan(v)
        if lop == CMP_LT:
            m &= lo < v
        elif lop == CMP_LE:
            m &= lo <= v
        if rop == CMP_LT:
            m &= v < hi
        elif rop == CMP_LE:
            m &= v <= hi
        return m
    if kind == "not":
        return ~_mask(node[1])
    parts = [_mask(k) for k in node[1]]
    out = parts[0].copy()
    for p in parts[1:]:
        out = (out & p) if kind == "and" else (out | p)
    return out


def _load():
    with open(FIXTURE) as f:
        d = json.load(f)
    tables = {name: {c: _Col(vals) for c, vals in zip(t["columns"], t["values"])}
              for name, t in d["tables"].items()}
    return tables, d["queries"]


def test_fixture_shape():
    tables, queries = _load()
    assert len(tables["test0"]["i0"].v) == 100 and len(tables["test1"]["c2z0"].v) == 1000
    assert len(queries) == 40


def test_counts_equal_the_reference():
    tables, queries = _load()
    checked = refused = 0
    for q in queries:
        clause, want = q["where"], q["count"]
        try:
            node = parse(clause, tables[q["table"]])
        except QueryError:
            assert any(f in clause for f in ("sqrt", "log", "exp", "**", "*")), clause
            refused += 1
            continue
        got = int(_mask(node).sum())
        if clause in REFERENCE_DROPS_ZERO:
            assert got == want + 1, clause
        else:
            assert got == want, (clause, got, want)
        checked += 1
    assert checked >= 30 and checked + refused == len(queries)


@pytest.mark.parametrize("clause", ["i0 in (3 5 7)", "i0 in (3, 5, 7)"])
def test_in_lists_with_or_without_commas(clause):
    tables, _ = _load()
    node = parse(clause, tables["test0"])
    assert int(_mask(node).sum()) == 3
