"""Regenerates the golden fixtures in this directory from the LADDS source tree.

Run with the path of an esa/LADDS source tree, given as ``--reference DIR``
or in the environment variable ``LADDS_REFERENCE``::

    python tests/golden/make_golden.py --reference path/to/LADDS

It reads, as text:
  * tests/testladds/CollisionFunctorTest.cpp -- the parametrised
    LinearInterpolationTest cases (x1, x2, v1, v2, dt, expected dl^2, expected
    collision point), lines 323-354 of that file;
  * data/pos_test.csv, data/v_test.csv, data/pos_test_10s.csv,
    data/v_test_10s.csv -- 10 LEO objects before and after 10 s.
Nothing is executed from the reference.  The outputs are small JSON files that
the tests read; the reference tree is never read at test time.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import sys

REF = None  # the LADDS source tree, set by main()
OUT = os.path.dirname(os.path.abspath(__file__))


def _floats(s: str):
    return [float(v) for v in re.findall(r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?", s)]


def interpolation_cases():
    path = os.path.join(REF, "tests/testladds/CollisionFunctorTest.cpp")
    src = open(path).read()
    block = src[src.index("INSTANTIATE_TEST_SUITE_P"):]
    cases = []
    for m in re.finditer(r"std::make_tuple\((.*?)\)\s*[,}]", block, re.S):
        body = m.group(1)
        arrays = re.findall(r"std::array<double,\s*3>\{([^}]*)\}", body)
        # scalars are what remains after removing the arrays
        rest = re.sub(r"std::array<double,\s*3>\{[^}]*\}", "#", body)
        scalars = [v for part in rest.split("#") for v in _floats(part)]
        if len(arrays) != 5 or len(scalars) != 2:
            continue
        vecs = [_floats(a) for a in arrays]
        cases.append({"x1": vecs[0], "x2": vecs[1], "v1": vecs[2], "v2": vecs[3], "dt": scalars[0],
                      "expected_dl2": scalars[1], "expected_point": vecs[4]})
    assert len(cases) == 4, f"expected 4 interpolation cases, found {len(cases)}"
    return {"source": "tests/testladds/CollisionFunctorTest.cpp:323-354", "cases": cases}


def two_body_fixture():
    def rd(name):
        rows = []
        for line in open(os.path.join(REF, "data", name)):
            line = line.strip()
            if line:
                rows.append([float(v) for v in line.split(",")])
        return rows

    return {"source": "data/pos_test.csv, data/v_test.csv -> data/pos_test_10s.csv, data/v_test_10s.csv",
            "dt_total": 10.0, "r0": rd("pos_test.csv"), "v0": rd("v_test.csv"), "r1": rd("pos_test_10s.csv"),
            "v1": rd("v_test_10s.csv")}


def main():
    global REF
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default=os.environ.get("LADDS_REFERENCE"),
                    help="esa/LADDS source tree (default: $LADDS_REFERENCE)")
    args = ap.parse_args()
    if not args.reference or not os.path.isfile(
            os.path.join(args.reference, "tests", "testladds", "CollisionFunctorTest.cpp")):
        sys.exit("make_golden.py: give the esa/LADDS source tree with --reference DIR or LADDS_REFERENCE "
                 f"(got {args.reference!r})")
    REF = args.reference
    with open(os.path.join(OUT, "interpolation_cases.json"), "w") as f:
        json.dump(interpolation_cases(), f, indent=1)
    with open(os.path.join(OUT, "two_body_10s.json"), "w") as f:
        json.dump(two_body_fixture(), f, indent=1)
    print("wrote", os.listdir(OUT))


if __name__ == "__main__":
    main()
