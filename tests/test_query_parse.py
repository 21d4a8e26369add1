"""WHERE-clause parsing of libfastlib_b200.query on the host (no device):
the trees countQuery would evaluate, and the clauses it refuses."""
import pytest

from libfastlib_b200 import CMP_LE, CMP_LT, CMP_NONE
from libfastlib_b200.query import QueryError, parse


class _Col:
    def __init__(self, name):
        self.name = name

    def term(self, lo=None, hi=None, lop=CMP_LE, rop=CMP_LT):
        return (self.name, CMP_NONE if lo is None else lop, lo, CMP_NONE if hi is None else rop, hi)


COLS = {"a": _Col("a"), "B": _Col("b")}


def leaf(*t):
    return ("leaf", t)


@pytest.mark.parametrize("clause,tree", [
    ("a >= 3", leaf("a", CMP_LE, 3.0, CMP_NONE, None)),
    ("2.5 <= b < 7", leaf("b", CMP_LE, 2.5, CMP_LT, 7.0)),
    ("a between 1 and 4", leaf("a", CMP_LE, 1.0, CMP_LE, 4.0)),
    ("a = 5", leaf("a", CMP_LE, 5.0, CMP_LE, 5.0)),
    ("a != 5", ("not", leaf("a", CMP_LE, 5.0, CMP_LE, 5.0))),
    ("5 > a", leaf("a", CMP_NONE, None, CMP_LT, 5.0)),
    ("a < 1 or b > -0.5 and not a <= 9",
     ("or", [leaf("a", CMP_NONE, None, CMP_LT, 1.0),
             ("and", [leaf("b", CMP_LT, -0.5, CMP_NONE, None), ("not", leaf("a", CMP_NONE, None, CMP_LE, 9.0))])])),
    ("a in (3, 5.5, 7)", ("or", [leaf("a", CMP_LE, 3.0, CMP_LE, 3.0), leaf("a", CMP_LE, 5.5, CMP_LE, 5.5),
                                  leaf("a", CMP_LE, 7.0, CMP_LE, 7.0)])),
    ("b in (2) and not a in (1, 2)",
     ("and", [leaf("b", CMP_LE, 2.0, CMP_LE, 2.0),
              ("not", ("or", [leaf("a", CMP_LE, 1.0, CMP_LE, 1.0), leaf("a", CMP_LE, 2.0, CMP_LE, 2.0)]))])),
    # the reference's own test queries write IN lists without commas
    ("a in (1 2)", ("or", [leaf("a", CMP_LE, 1.0, CMP_LE, 1.0), leaf("a", CMP_LE, 2.0, CMP_LE, 2.0)])),
    ("!(a >= 3) || (b < 1 && a > 2)",
     ("or", [("not", leaf("a", CMP_LE, 3.0, CMP_NONE, None)),
             ("and", [leaf("b", CMP_NONE, None, CMP_LT, 1.0), leaf("a", CMP_LT, 2.0, CMP_NONE, None)])])),
])
def test_trees(clause, tree):
    assert parse(clause, COLS) == tree


@pytest.mark.parametrize("clause", ["c < 3", "a < 5 or", "(a < 3", "a between 1 4", "a <", "a < 3 b < 4", "a @ 3",
                                    "a in (1, 2", "a in ()", "a in (1 2", "a in (1 , , 2)"])
def test_refused(clause):
    with pytest.raises(QueryError):
        parse(clause, COLS)
