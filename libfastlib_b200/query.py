"""WHERE clauses over named columns (the Python face of ibis::countQuery,
src/countQuery.cpp:81-410): range conditions — ``a >= 3``, ``2.5 <= b < 7``,
``c between 1 and 4``, ``d = 5``, ``d != 5``, ``e in (1, 4, 9)`` (a
qDiscreteRange, evaluated as an OR of equalities) — combined with AND, OR, NOT
(also ``&&``, ``||``, ``!``) and parentheses, as countQuery::doEvaluate
combines qContinuousRange leaves (src/countQuery.cpp:929-1036).

An AND of ranges is one fused evaluation on the device; other nodes combine
the hit bitvectors of their parts with the device operators (OR ``|``, NOT
``flip()``, AND ``&``).

    n, rows = where(ctx, "age between 30 and 40 or not price < 99.5",
                    {"age": age_index, "price": price_index})
"""
from __future__ import annotations

import re

from . import AND, CMP_LE, CMP_LT, OR, evaluate

_TOKEN = re.compile(r"\s*(?:(?P<num>[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?)"
                    r"|(?P<name>[A-Za-z_][A-Za-z0-9_.]*)"
                    r"|(?P<op><=|>=|==|!=|&&|\|\||[<>=()!,]))")


class QueryError(ValueError):
    """The clause does not parse or names an unknown column."""


def _tokens(text):
    out, pos = [], 0
    text = text.rstrip()
    while pos < len(text):
        m = _TOKEN.match(text, pos)
        if not m or m.end() == pos:
            raise QueryError(f"cannot read the clause at {text[pos:pos + 10]!r}")
        pos = m.end()
        if m.group("num") is not None:
            out.append(("num", float(m.group("num"))))
        elif m.group("name") is not None:
            out.append(("name", m.group("name")))
        else:
            out.append(("op", m.group("op")))
    return out


class _Parser:
    # node forms: ("leaf", term) | ("and", [kids]) | ("or", [kids]) | ("not", kid)
    def __init__(self, tokens, columns):
        self.t, self.i = tokens, 0
        self.cols = {k.lower(): v for k, v in columns.items()}

    def _word(self, *words):
        if self.i < len(self.t):
            kind, v = self.t[self.i]
            if (kind == "name" and v.lower() in words) or (kind == "op" and v in words):
                return True
        return False

    def _col(self, name):
        try:
            return self.cols[name.lower()]
        except KeyError:
            raise QueryError(f"unknown column {name}") from None

    def parse(self):
        node = self._or()
        if self.i != len(self.t):
            raise QueryError(f"unexpected {self.t[self.i][1]!r}")
        return node

    def _or(self):
        kids = [self._and()]
        while self._word("or", "||"):
            self.i += 1
            kids.append(self._and())
        return kids[0] if len(kids) == 1 else ("or", kids)

    def _and(self):
        kids = [self._unary()]
        while self._word("and", "&&"):
            self.i += 1
            kids.append(self._unary())
        return kids[0] if len(kids) == 1 else ("and", kids)

    def _unary(self):
        if self._word("not", "!"):
            self.i += 1
            return ("not", self._unary())
        if self._word("("):
            self.i += 1
            node = self._or()
            if not self._word(")"):
                raise QueryError("missing ')'")
            self.i += 1
            return node
        return self._condition()

    def _condition(self):
        t, i = self.t, self.i
        cmp_ops = ("<", "<=", ">", ">=", "=", "==", "!=")

        def kind(k):
            return t[k][0] if k < len(t) else None

        def val(k):
            return t[k][1] if k < len(t) else None

        if (kind(i) == "name" and kind(i + 1) == "name" and str(val(i + 1)).lower() == "in"
                and kind(i + 2) == "op" and val(i + 2) == "("):
            # x in (v1, v2, ...) or x in (v1 v2 ...): qDiscreteRange as an
            # OR of equalities
            idx, k, vals = self._col(val(i)), i + 3, []
            while True:
                if kind(k) != "num":
                    raise QueryError("bad IN list")
                vals.append(val(k))
                if kind(k + 1) == "op" and val(k + 1) == ",":
                    k += 2
                    continue
                if kind(k + 1) == "num":
                    k += 1
                    continue
                if kind(k + 1) == "op" and val(k + 1) == ")":
                    break
                raise QueryError("bad IN list")
            self.i = k + 2
            leaves = [("leaf", idx.term(v, v, lop=CMP_LE, rop=CMP_LE)) for v in vals]
            return leaves[0] if len(leaves) == 1 else ("or", leaves)
        if kind(i) == "name" and kind(i + 1) == "name" and str(val(i + 1)).lower() == "between":
            if kind(i + 2) != "num" or str(val(i + 3)).lower() != "and" or kind(i + 4) != "num":
                raise QueryError("bad BETWEEN")
            self.i = i + 5
            return ("leaf", self._col(val(i)).term(val(i + 2), val(i + 4), lop=CMP_LE, rop=CMP_LE))
        if kind(i) == "name" and kind(i + 1) == "op" and val(i + 1) in cmp_ops and kind(i + 2) == "num":
            idx, op, v = self._col(val(i)), val(i + 1), val(i + 2)
            self.i = i + 3
            if op == "<":
                return ("leaf", idx.term(None, v, rop=CMP_LT))
            if op == "<=":
                return ("leaf", idx.term(None, v, rop=CMP_LE))
            if op == ">":
                return ("leaf", idx.term(v, None, lop=CMP_LT))
            if op == ">=":
                return ("leaf", idx.term(v, None, lop=CMP_LE))
            eq = ("leaf", idx.term(v, v, lop=CMP_LE, rop=CMP_LE))
            return ("not", eq) if op == "!=" else eq
        if kind(i) == "num" and kind(i + 1) == "op" and val(i + 1) in cmp_ops[:-1] and kind(i + 2) == "name":
            v, op, idx = val(i), val(i + 1), self._col(val(i + 2))
            self.i = i + 3
            if op in ("<", "<="):
                lop = CMP_LT if op == "<" else CMP_LE
                if kind(self.i) == "op" and val(self.i) in ("<", "<=") and kind(self.i + 1) == "num":
                    rop = CMP_LT if val(self.i) == "<" else CMP_LE
                    hi = val(self.i + 1)
                    self.i += 2
                    return ("leaf", idx.term(v, hi, lop=lop, rop=rop))
                return ("leaf", idx.term(v, None, lop=lop))
            if op == ">":
                return ("leaf", idx.term(None, v, rop=CMP_LT))
            if op == ">=":
                return ("leaf", idx.term(None, v, rop=CMP_LE))
            return ("leaf", idx.term(v, v, lop=CMP_LE, rop=CMP_LE))
        raise QueryError(f"not a range condition near {val(i)!r}")


def parse(clause: str, columns) -> tuple:
    """The clause as a tree of ("leaf", term) / ("and"|"or", kids) /
    ("not", kid) nodes over the columns' indexes."""
    return _Parser(_tokens(clause), columns).parse()


def _hits(ctx, node):
    kind = node[0]
    if kind == "leaf":
        return evaluate(ctx, [node[1]], want_rids=False, want_hits=True)[2]
    if kind == "not":
        return _hits(ctx, node[1]).flip()
    if kind == "and":
        leaves = [k[1] for k in node[1] if k[0] == "leaf"]
        parts = [evaluate(ctx, leaves, want_rids=False, want_hits=True)[2]] if leaves else []
        parts += [_hits(ctx, k) for k in node[1] if k[0] != "leaf"]
        acc = parts[0]
        for p in parts[1:]:
            acc = acc._binop(AND, p, False)
        return acc
    acc = _hits(ctx, node[1][0])
    for k in node[1][1:]:
        acc = acc._binop(OR, _hits(ctx, k), False)
    return acc


def where(ctx, clause: str, columns):
    """countQuery::evaluate + getNumHits + getHitRows: (count, row ids)."""
    node = parse(clause, columns)
    if node[0] == "leaf" or (node[0] == "and" and all(k[0] == "leaf" for k in node[1])):
        terms = [node[1]] if node[0] == "leaf" else [k[1] for k in node[1]]
        n, rows, _ = evaluate(ctx, terms)
        return n, rows
    h = _hits(ctx, node)
    return h.cnt(), h.rids()
