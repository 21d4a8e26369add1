"""Known-answer fixture from the reference's own test suite: the hit counts of
tests/scripts/query-count.list over tests/test0.csv and tests/test1.csv
(the `match-counts` target of tests/Makefile.am:343-373 runs these queries
for every encoding and binning and compares the counts).

    python tests/golden/make_query_counts.py [REFERENCE_ROOT]

REFERENCE_ROOT defaults to $FASTBIT_REFERENCE, else ../reference beside the
repository.  Writes tests/golden/query_counts.json: the two tables (column
names and values as the CSV files hold them; test0 is loaded as i0:ubyte,
i1:float, i2:short, tests/Makefile.am:454) and every query with its count.
"""
from __future__ import annotations

import csv
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def read_table(path):
    """Columns as lists of numbers; an empty field (a NULL, which satisfies
    no range condition) is None."""
    with open(path) as f:
        lines = f.read().splitlines()
    names = [c.strip().strip('"') for c in lines[0].lstrip("#").split(",")]
    rows = [r for r in csv.reader(lines[1:]) if r and not r[0].startswith("#")]
    cols = [[float(r[k]) if r[k].strip() else None for r in rows] for k in range(len(names))]
    return {"columns": names, "values": cols}


def read_queries(path):
    out = []
    with open(path) as f:
        for line in f:
            line = line.strip()
            if not line or line.startswith("#"):
                continue
            text, count = line.rsplit(";", 1)
            words = text.split()
            assert words[0].lower() == "from" and words[2].lower() == "where", line
            out.append({"table": words[1], "where": " ".join(words[3:]), "count": int(count)})
    return out


def main(argv):
    root = argv[1] if len(argv) > 1 else (os.environ.get("FASTBIT_REFERENCE")
                                          or os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(HERE))),
                                                          "reference"))
    t = os.path.join(root, "tests")
    data = {"source": "tests/scripts/query-count.list, tests/test0.csv, tests/test1.csv of the reference",
            "tables": {"test0": read_table(os.path.join(t, "test0.csv")),
                       "test1": read_table(os.path.join(t, "test1.csv"))},
            "queries": read_queries(os.path.join(t, "scripts", "query-count.list"))}
    with open(os.path.join(HERE, "query_counts.json"), "w") as f:
        json.dump(data, f, separators=(",", ":"))
    print(len(data["queries"]), "queries")


if __name__ == "__main__":
    main(sys.argv)
