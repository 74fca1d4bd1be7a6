"""Generate tests/golden/filter_fixtures.json from the reference's SQL filter
conformance fixtures (wasm/tests/conformance/fixtures/*.expected.json, made
by PyLance over a 10-row table with NULLs, see
wasm/tests/conformance/generate_sql_fixtures.py:28-47).

Only fixtures expressible on the GPU path are kept: comparisons of numeric
columns with numeric literals, BETWEEN / NOT BETWEEN, IS [NOT] NULL, and
AND / OR with parentheses (no NOT, IN, LIKE, NULL literals or
column-vs-column tests).  Each WHERE clause is rewritten in disjunctive normal
form, the shape QueryDescriptor takes (filters AND-ed, filterGroups OR-ed).
The string column `c` becomes int32 dictionary codes carrying its NULLs.
Expected rows are turned into row indices of the source table.

Run from the repository root, naming the reference's checkout (the output
is committed; tests never read the reference):

    python tests/golden/make_golden.py <path to the reference checkout>
"""
from __future__ import annotations

import glob
import json
import os
import re

FIXTURES = os.path.join("wasm", "tests", "conformance", "fixtures")  # inside the reference checkout
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "filter_fixtures.json")

# The fixture table, restated from generate_sql_fixtures.py:33-46.
TABLE = {
    "a": [1, 2, 3, None, 5, None, 7, 0, -1, 10],
    "b": [10, None, 30, 40, None, 60, 70, 0, -10, 100],
    "c": ["foo", "bar", None, "baz", "qux", None, "quux", "foo%bar", "f_o", ""],
    "d": [1.5, 2.0, 3.0, None, 5.5, 6.0, 7.7, 0.0, -1.5, 10.0],
}
NUMERIC = {"a": "int64", "b": "int64", "c": "int32", "d": "float64"}

class Unsupported(Exception):
    pass


TOKEN = re.compile(r"\s*(>=|<=|!=|<>|=|<|>|\(|\)|-?\d+\.\d+|-?\d+|[A-Za-z_]\w*)")


def tokenize(s: str) -> list[str]:
    out, pos = [], 0
    while pos < len(s):
        m = TOKEN.match(s, pos)
        if not m:
            if s[pos:].strip() == "":
                break
            raise Unsupported(f"cannot tokenize {s!r} at {pos}")
        out.append(m.group(1))
        pos = m.end()
    return out


def literal(tok: str):
    if re.fullmatch(r"-?\d+", tok):
        return int(tok)
    if re.fullmatch(r"-?\d+\.\d+", tok):
        return float(tok)
    raise Unsupported(tok)


def parse(tokens: list[str]):
    """expr := term (OR term)*; term := factor (AND factor)*;
    factor := '(' expr ')' | predicate.  Returns DNF: list of AND lists."""
    pos = 0

    def peek():
        return tokens[pos] if pos < len(tokens) else None

    def take():
        nonlocal pos
        t = tokens[pos]
        pos += 1
        return t

    def expr():
        d = term()
        while peek() and peek().upper() == "OR":
            take()
            d = d + term()
        return d

    def term():
        d = factor()
        while peek() and peek().upper() == "AND":
            take()
            r = factor()
            d = [x + y for x in d for y in r]
        return d

    def factor():
        if peek() == "(":
            take()
            d = expr()
            if take() != ")":
                raise Unsupported("paren")
            return d
        return [[predicate()]]

    def predicate():
        col = take()
        if col.upper() == "NOT" or col not in NUMERIC:
            raise Unsupported(col)
        t = take()
        if t.upper() == "IS":
            if peek().upper() == "NOT":
                take()
                take()  # NULL
                return {"column": col, "op": "is_not_null"}
            take()
            return {"column": col, "op": "is_null"}
        if t.upper() in ("BETWEEN", "NOT"):
            op = "between"
            if t.upper() == "NOT":
                if take().upper() != "BETWEEN":
                    raise Unsupported("NOT")
                op = "not_between"
            lo = literal(take())
            if take().upper() != "AND":
                raise Unsupported("between")
            hi = literal(take())
            return {"column": col, "op": op, "value": [lo, hi]}
        ops = {"=": "eq", "!=": "neq", "<>": "neq", "<": "lt", "<=": "lte", ">": "gt", ">=": "gte"}
        if t not in ops:
            raise Unsupported(t)
        nxt = take()
        if nxt in NUMERIC or nxt.upper() == "NULL":
            raise Unsupported(nxt)
        return {"column": col, "op": ops[t], "value": literal(nxt)}

    d = expr()
    if pos != len(tokens):
        raise Unsupported("trailing")
    return d


def row_index(data: dict, i: int) -> int:
    key = (data["a"][i], data["b"][i], data["d"][i])
    for r in range(10):
        if (TABLE["a"][r], TABLE["b"][r], TABLE["d"][r]) == key:
            return r
    raise KeyError(key)


def main(reference: str) -> None:
    cases = []
    for f in sorted(glob.glob(os.path.join(reference, FIXTURES, "*.expected.json"))):
        fx = json.load(open(f))
        res = fx["result"]
        if not res.get("success"):
            continue
        try:
            dnf = parse(tokenize(fx["query"]))
        except (Unsupported, IndexError):
            continue
        rows = sorted(row_index(res["data"], i) for i in range(res["row_count"]))
        case = {"name": fx["name"], "query": fx["query"], "expected_rows": rows}
        if len(dnf) == 1:
            case["filters"], case["filter_groups"] = dnf[0], None
        else:
            case["filters"], case["filter_groups"] = [], dnf
        cases.append(case)
    codes = {}
    c_codes = []
    for v in TABLE["c"]:
        if v is None:
            c_codes.append(None)
        else:
            c_codes.append(codes.setdefault(v, len(codes)))
    table = dict(TABLE)
    table["c"] = c_codes
    out = {
        "source": "wasm/tests/conformance/fixtures/*.expected.json (PyLance)",
        "dtypes": NUMERIC,
        "table": table,
        "cases": cases,
    }
    with open(OUT, "w") as fh:
        json.dump(out, fh, indent=1)
    print(f"wrote {len(cases)} cases to {OUT}")


if __name__ == "__main__":
    import sys
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the reference checkout>")
    main(sys.argv[1])
