#!/usr/bin/env python3
"""Extract the reference's GoogleTest golden vectors into a JSON fixture.

TimThuering/Heterogeneous-Solvers (MIT) tests every kernel of its blocked SPD
path against hard-coded packed arrays computed from a 20x20 SPD fixture
(tests/testData/testMatrixSymmetric20x20.txt, tests/testData/testVector_20.txt).
This script reads those files as text and records, per TEST_F, the ordered
steps the test performs (configuration assignments, fixture parsing, vector
set-up, kernel calls with their literal argument expressions, expectations)
together with the literal golden arrays.  tests/reference_cases.py replays
the steps against the oracle (CPU suite) and against the CUDA library (GPU
suite).

Usage (needs the reference checkout; the JSON it writes is committed):
    python tests/golden/extract_reference_tests.py <reference checkout>
or with the checkout in the environment variable HS_REFERENCE_ROOT.
"""
import json
import math
import os
import re
import sys
from pathlib import Path

TEST_FILES = [
    "tests/testSymmetricMatrix.cpp",
    "tests/testMatrixOperations.cpp",
    "tests/testMatrixMatrixOperations.cpp",
    "tests/testMatrixVectorBlock.cpp",
    "tests/testVectorOperations.cpp",
]

NUM = r"[-+]?(?:\d+\.?\d*(?:[eE][-+]?\d+)?|\.\d+(?:[eE][-+]?\d+)?)"


def strip_comments(text):
    text = re.sub(r"/\*.*?\*/", lambda m: "\n" * m.group(0).count("\n"), text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def match_brace(text, open_idx):
    depth = 0
    for i in range(open_idx, len(text)):
        if text[i] == "{":
            depth += 1
        elif text[i] == "}":
            depth -= 1
            if depth == 0:
                return i
    raise ValueError("unbalanced braces")


def parse_number_list(body):
    vals = re.findall(NUM, body)
    return [float(v) for v in vals]


ARRAY_RE = re.compile(r"std::vector<conf::fp_type>\s+(\w+)\s*=\s*\{")


def extract_arrays(text):
    arrays = {}
    for m in ARRAY_RE.finditer(text):
        end = match_brace(text, m.end() - 1)
        arrays[m.group(1)] = parse_number_list(text[m.end():end])
    return arrays


def norm(s):
    return re.sub(r"\s+", " ", s).strip()


def split_args(s):
    args, depth, cur = [], 0, ""
    for ch in s:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == "," and depth == 0:
            args.append(norm(cur))
            cur = ""
        else:
            cur += ch
    if cur.strip():
        args.append(norm(cur))
    return args


STEP_PATTERNS = [
    ("conf", re.compile(r"conf::(\w+)\s*=\s*([^;]+);")),
    ("parse_matrix", re.compile(r"SymmetricMatrix\s+(\w+)\s*=\s*MatrixParser::parseSymmetricMatrix\(")),
    ("parse_rhs", re.compile(r"RightHandSide\s+(\w+)\s*=\s*MatrixParser::parseRightHandSide\(")),
    ("resize", re.compile(r"(\w+)\.resize\(([^;]*)\);")),
    ("sqrt_accumulate", re.compile(
        r"for\s*\(\s*unsigned int i\s*=\s*0;\s*i\s*<\s*(\d+);\s*\+\+i\)\s*\{\s*"
        r"(?:if\s*\(\s*i\s*>=\s*(\d+)\s*\)\s*\{\s*)?(\w+)\s*\+=\s*std::sqrt\(i\)\s*\*\s*std::sqrt\(i\);\s*\}?\s*"
        r"(\w+)\[i\]\s*=\s*std::sqrt\(i\);\s*\}", re.S)),
    ("fill", re.compile(
        r"for\s*\(\s*(?:size_t|unsigned int|int)\s+i\s*=\s*(\w+);\s*i\s*<\s*([\w.()]+);\s*(?:\+\+i|i\+\+)\)\s*"
        r"\{\s*(\w+)\[i\]\s*=\s*([^;]+);\s*\}", re.S)),
    ("expect_loop", re.compile(
        r"for\s*\(\s*size_t\s+i\s*=\s*0;\s*i\s*<\s*([\w.()]+);\s*i\+\+\)\s*\{\s*"
        r"EXPECT_NEAR\(([^,]+),\s*([^,]+),\s*([^)]+)\);\s*\}", re.S)),
    ("call", re.compile(
        r"(?:unsigned int\s+(\w+)\s*=\s*)?(MatrixOperations|MatrixMatrixOperations|MatrixVectorOperations|"
        r"VectorOperations)::(\w+)\((.*?)\);", re.S)),
    ("expect_near", re.compile(r"EXPECT_NEAR\(([^,]+),\s*([^,]+),\s*([^)]+)\);")),
    ("expect_double_eq", re.compile(r"EXPECT_DOUBLE_EQ\(([^,]+),\s*([^)]+)\);")),
    ("expect_eq", re.compile(r"EXPECT_EQ\(([^,]+),\s*([^)]+)\);")),
]


def extract_steps(body):
    """Return the body's recognised statements in source order."""
    claimed = []  # (start, end) spans already taken by a longer pattern
    found = []
    for kind, pat in STEP_PATTERNS:
        for m in pat.finditer(body):
            s, e = m.span()
            if any(s < ce and e > cs for cs, ce in claimed):
                continue
            claimed.append((s, e))
            found.append((s, kind, m))
    found.sort(key=lambda t: t[0])
    scalars = {}
    steps = []
    for _, kind, m in found:
        if kind == "conf":
            steps.append({"op": "conf", "key": m.group(1), "value": norm(m.group(2))})
        elif kind in ("parse_matrix", "parse_rhs"):
            steps.append({"op": kind, "var": m.group(1)})
        elif kind == "resize":
            args = split_args(m.group(2))
            step = {"op": "resize", "var": m.group(1), "size": args[0]}
            if len(args) > 1:
                step["fill"] = float(args[1])
            steps.append(step)
        elif kind == "sqrt_accumulate":
            n, lo, acc, vec = int(m.group(1)), m.group(2), m.group(3), m.group(4)
            lo = int(lo) if lo else 0
            total = 0.0
            for i in range(n):
                if i >= lo:
                    total += math.sqrt(i) * math.sqrt(i)
            scalars[acc] = total
            steps.append({"op": "fill", "var": vec, "lo": "0", "hi": str(n), "expr": "std::sqrt(i)"})
        elif kind == "fill":
            steps.append({"op": "fill", "var": m.group(3), "lo": m.group(1), "hi": m.group(2),
                          "expr": norm(m.group(4))})
        elif kind == "call":
            steps.append({"op": "call", "cls": m.group(2), "fn": m.group(3), "args": split_args(m.group(4)),
                          "ret": m.group(1)})
        elif kind == "expect_loop":
            steps.append({"op": "expect_loop", "count": m.group(1), "actual": norm(m.group(2)),
                          "expected": norm(m.group(3)), "tol": float(m.group(4))})
        elif kind == "expect_near":
            exp = norm(m.group(2))
            exp = scalars.get(exp, exp)
            steps.append({"op": "expect_near", "actual": norm(m.group(1)), "expected": exp,
                          "tol": float(m.group(3))})
        elif kind == "expect_double_eq":
            steps.append({"op": "expect_double_eq", "actual": norm(m.group(1)), "expected": norm(m.group(2))})
        elif kind == "expect_eq":
            steps.append({"op": "expect_eq", "actual": norm(m.group(1)), "expected": norm(m.group(2))})
    return steps


def parse_matrix_file(path):
    lines = Path(path).read_text().strip().splitlines()
    n = int(lines[0][2:])
    rows = [[float(v) for v in line.split(";")] for line in lines[1:]]
    assert len(rows) == n and all(len(r) == i + 1 for i, r in enumerate(rows))
    return {"N": n, "rows": rows}


def parse_vector_file(path):
    lines = Path(path).read_text().strip().splitlines()
    n = int(lines[0][2:])
    vals = [float(v) for v in lines[1].split(";")]
    return {"N": n, "values": vals[:n]}


def main(ref_root):
    ref = Path(ref_root)
    out = {
        "source": "TimThuering/Heterogeneous-Solvers tests (MIT licence), extracted by "
                  "tests/golden/extract_reference_tests.py",
        "fixtures": {
            "matrix": parse_matrix_file(ref / "tests/testData/testMatrixSymmetric20x20.txt"),
            "vector": parse_vector_file(ref / "tests/testData/testVector_20.txt"),
        },
        "suite_arrays": {},
        "cases": [],
    }
    for rel in TEST_FILES:
        raw = (ref / rel).read_text()
        text = strip_comments(raw)
        # fixture-level arrays: inside `class X : public ::testing::Test { ... };`
        for cm in re.finditer(r"class\s+(\w+)\s*:\s*public\s+::testing::Test\s*\{", text):
            end = match_brace(text, cm.end() - 1)
            out["suite_arrays"][f"{rel}::{cm.group(1)}"] = extract_arrays(text[cm.end():end])
        for tm in re.finditer(r"TEST_F\(\s*(\w+)\s*,\s*(\w+)\s*\)\s*\{", text):
            end = match_brace(text, tm.end() - 1)
            body = text[tm.end():end]
            line = text.count("\n", 0, tm.start()) + 1
            out["cases"].append({
                "file": rel, "line": line, "suite": tm.group(1), "name": tm.group(2),
                "arrays": extract_arrays(body), "steps": extract_steps(body),
            })
    dst = Path(__file__).resolve().parent / "reference_cases.json"
    dst.write_text(json.dumps(out, indent=None, separators=(",", ":")))
    print(f"wrote {dst} with {len(out['cases'])} cases")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HS_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: extract_reference_tests.py <reference checkout> (or set HS_REFERENCE_ROOT)")
    main(root)
