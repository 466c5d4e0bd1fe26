"""Extract the reference's known-answer vectors into ``reference_kats.json``.

Reads the reference's own C++ test sources as TEXT (nothing of the reference
is compiled or run) and records, per test case, the literal inputs and the
expected outputs:

* ``tests/boundaries.cpp``  contractExpectationBoundaries / SOS / VS known
  answers (the ``non_trivial`` and small trivial cases),
* ``tests/chain.cpp``       TFIM sweepUntilConverged / optimizeChain energies,
* ``tests/stress.cpp``      TFIM four-lowest-level energies,
* ``tests/optimizer.cpp``   one-site optimizer mode cases.

Usage:  python tests/golden/make_golden.py <reference_root>
        (or set NUTCRACKER_REFERENCE to the reference checkout)
The committed JSON is what the tests read; the reference tree is not needed
at test time.
"""
from __future__ import annotations

import json
import os
import re
import sys

ROOT = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NUTCRACKER_REFERENCE", "")
if __name__ == "__main__" and not ROOT:
    sys.exit("usage: make_golden.py <reference_root>  (or set NUTCRACKER_REFERENCE)")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")


def read(rel):
    with open(os.path.join(ROOT, rel)) as f:
        return f.read()


def block(text, suite, case):
    """Source text of TEST_CASE(case) inside TEST_SUITE(suite)."""
    s = text.index("TEST_SUITE(%s)" % suite)
    c = text.index("TEST_CASE(%s)" % case, s)
    depth, i, started = 0, text.index("{", c), False
    j = i
    while True:
        if text[j] == "{":
            depth += 1
        elif text[j] == "}":
            depth -= 1
            if depth == 0:
                return text[c:j + 1]
        j += 1


NUM = r"[-+]?\s*[0-9.]+(?:e[-+]?[0-9]+)?"


def parse_value(tok):
    tok = tok.strip()
    m = re.fullmatch(r"(?:c|complex<double>)\(\s*(%s)\s*,\s*(%s)\s*\)" % (NUM, NUM), tok)
    if m:
        return [float(m.group(1).replace(" ", "")), float(m.group(2).replace(" ", ""))]
    m = re.fullmatch(r"complex<double>\(\s*(%s)\s*\)" % NUM, tok)
    if m:
        return [float(m.group(1).replace(" ", "")), 0.0]
    return float(tok.replace(" ", ""))


def list_of_chains(src):
    """All ``list_of(a)(b)...`` chains, in order, as lists of values."""
    out = []
    for m in re.finditer(r"list_of", src):
        i = m.end()
        vals = []
        while True:
            while i < len(src) and src[i] in " \t\r\n":
                i += 1
            if i >= len(src) or src[i] != "(":
                break
            depth, j = 0, i
            while True:
                if src[j] == "(":
                    depth += 1
                elif src[j] == ")":
                    depth -= 1
                    if depth == 0:
                        break
                j += 1
            vals.append(parse_value(src[i + 1:j]))
            i = j + 1
        out.append(vals)
    return out


def expected_array(src):
    m = re.search(r"expected_boundary\[\]\s*=\s*\{(.*?)\}", src, re.S)
    return [parse_value(t) for t in re.findall(r"c\([^)]*\)", m.group(1))]


def dims(src, name):
    return [int(x) for x in re.findall(r"%s\((\d+)\)" % name, src)]


def main():
    kats = {}
    b = read("tests/boundaries.cpp")

    src = block(b, "contractExpectationBoundaries", "non_trivial")
    ch = list_of_chains(src)
    kats["contract_expectation_boundaries"] = {
        "source": "tests/boundaries.cpp:96-129",
        "c": dims(src, "OperatorDimension")[0],
        "left": ch[0], "right": ch[1],
        "expected": parse_value(re.search(r"expected_value\s*=\s*(c\([^)]*\))", src).group(1)),
    }

    src = block(b, "computeSOSLeft", "non_trivial")
    ch = list_of_chains(src)
    kats["contract_sos_left"] = {
        "source": "tests/boundaries.cpp:164-215",
        "c_left": dims(src, "OperatorDimension")[0],
        "state_left": dims(src, "LeftDimension")[0], "state_right": dims(src, "RightDimension")[0],
        "op_left": dims(src, "LeftDimension")[1], "op_right": dims(src, "RightDimension")[1],
        "boundary": ch[0], "state": ch[1], "indices": ch[2], "matrices": ch[3],
        "expected": expected_array(src),
    }

    src = block(b, "computeSOSRight", "non_trivial")
    ch = list_of_chains(src)
    kats["contract_sos_right"] = {
        "source": "tests/boundaries.cpp:250-303",
        "c_right": dims(src, "OperatorDimension")[0],
        "state_left": dims(src, "LeftDimension")[0], "state_right": dims(src, "RightDimension")[0],
        "op_left": dims(src, "LeftDimension")[1], "op_right": dims(src, "RightDimension")[1],
        "boundary": ch[0], "state": ch[1], "indices": ch[2], "matrices": ch[3],
        "expected": expected_array(src),
    }

    for suite, key, src_lines in (("computeSSLeft", "contract_vs_left", "tests/boundaries.cpp:342-383"),
                                  ("computeSSRight", "contract_vs_right", "tests/boundaries.cpp:422-465")):
        src = block(b, suite, "non_trivial")
        ch = list_of_chains(src)
        kats[key] = {
            "source": src_lines,
            "overlap_dim": dims(src, "OverlapDimension")[0],
            "overlap_right": dims(src, "RightDimension")[0], "overlap_left": dims(src, "LeftDimension")[0],
            "state_left": dims(src, "LeftDimension")[1], "state_right": dims(src, "RightDimension")[1],
            "boundary": ch[0], "overlap_site": ch[1], "state": ch[2],
            "expected": expected_array(src),
        }
        src = block(b, suite, "trivial_with_physical_dimension_2")
        ch = list_of_chains(src)
        kats[key + "_d2"] = {"overlap_site": ch[0], "state": ch[1], "expected": ch[2][0]}

    src = block(b, "computeExpectationValueAtSite", "trivial_with_all_dimensions_1_and_imaginary_component")
    kats["expectation_imaginary"] = {"source": "tests/boundaries.cpp:30-49", "matrix": [0.0, 1.0],
                                     "expected": [0.0, 1.0]}
    d2 = re.findall(r"TEST_CASE\((_\w+)\)\s*\{\s*runTest\(([^;]*)\);", b)
    kats["expectation_d2"] = {"source": "tests/boundaries.cpp:52-83",
                              "cases": [[c[0], c[1]] for c in d2]}

    # chain energies
    c = read("tests/chain.cpp")
    suc = re.findall(r"TEST_CASE\((\w+)\)\s*\{\s*runTest\(\s*(\d+)\s*,\s*(%s)\s*,\s*(\d+)\s*,\s*(%s)\s*\);" % (NUM, NUM), c)
    kats["sweep_until_converged"] = {
        "source": "tests/chain.cpp:286-307",
        "cases": [{"name": n, "sites": int(s), "lambda": float(l), "chi": int(x),
                   "energy": float(e.replace(" ", ""))} for n, s, l, x, e in suc],
    }
    oc = re.findall(r"TEST_CASE\((10_sites_\w+)\)\s*\{\s*runTest\(\s*10\s*,\s*(%s)\s*,\s*(%s)\s*,\s*mode\s*\);" % (NUM, NUM), c)
    seen = {}
    for n, l, e in oc:
        seen[n] = {"name": n, "sites": 10, "lambda": float(l), "abs_energy": float(e)}
    kats["optimize_chain"] = {"source": "tests/chain.cpp:390-432", "tolerance": 1e-10,
                              "cases": list(seen.values())}

    s = read("tests/stress.cpp")
    st = []
    for m in re.finditer(r"TEST_SUITE\((least_value|greatest_value|largest_magnitude)\)", s):
        mode = m.group(1)
        end = s.find("TEST_SUITE(", m.end())
        body = s[m.end(): end if end > 0 else len(s)]
        for cm in re.finditer(r"TEST_CASE\(\s*(\d+)_sites_(\w+)\)\s*\{\s*runTest\(\s*(\d+)\s*,\s*(%s)\s*,\s*mode\s*,\s*list_of(.*?)\);\s*\}" % NUM, body, re.S):
            vals = [float(v.replace(" ", "")) for v in re.findall(r"\((%s)\)" % NUM, cm.group(5))]
            sanity = re.search(r",\s*(1e-\d+)\s*$", cm.group(5).strip())
            st.append({"mode": mode, "sites": int(cm.group(3)), "lambda": float(cm.group(4)),
                       "energies": vals})
    kats["stress_levels"] = {"source": "tests/stress.cpp:80-187", "tolerance": 1e-7, "cases": st}

    o = read("tests/optimizer.cpp")
    om = re.findall(r'TEST_CASE\(\w+\)\s*\{\s*runTests\("([<>][vm])"\s*,\s*(%s)\s*,\s*(%s)\s*,\s*(%s)\s*,\s*(%s)\s*,\s*(%s)\s*\);' % ((NUM,) * 5), o)
    kats["optimizer_modes"] = {"source": "tests/optimizer.cpp:71-138",
                               "cases": [{"mode": m[0], "value": float(m[1]),
                                          "diagonal": [float(x) for x in m[2:]]} for m in om]}
    with open(OUT, "w") as f:
        json.dump(kats, f, indent=1)
    print("wrote", OUT, {k: (len(v["cases"]) if "cases" in v else 1) for k, v in kats.items()})


if __name__ == "__main__":
    main()
