"""Extracts the reference's own golden vectors for the structured mesh
generator into tests/golden/meshstructgen_golden.json.

    python tests/golden/make_golden.py [path/to/reference]

Source: tests/geometry/mesh/implementation/source/MeshStructGenSourceTests.cpp
of the reference (Boost.Test). The file is read as text; for every test case
this records the generator's constructor arguments, the generator method the
case calls, its integer/boolean/point array initialisers, the expected
status and any scalar BOOST_CHECK_EQUAL values. The oracle tests replay each
case against the plain-C restatement of MeshStructGenSource.
"""
from __future__ import annotations

import json
import os
import re
import sys

REL = "tests/geometry/mesh/implementation/source/MeshStructGenSourceTests.cpp"


def parse(text):
    cases = []
    for m in re.finditer(r"BOOST_AUTO_TEST_CASE\((\w+)\)\s*\{(.*?)\n\}", text, re.S):
        name, body = m.group(1), m.group(2)
        body_nc = re.sub(r"//[^\n]*", "", body)
        ctor = re.search(r"MeshStructGenSource<int,\s*double>\s+source\(([^)]*)\)", body_nc)
        call = re.search(r"status\s*=\s*source\.(\w+)\(([^;]*)\);", body_nc)
        if not ctor or not call:
            continue
        case = {"name": name, "ctor": [float(x) for x in ctor.group(1).split(",")], "method": call.group(1),
                "call_args": [a.strip() for a in call.group(2).split(",")], "arrays": {}, "points": {}, "scalars": {}}
        for am in re.finditer(r"\b(int|bool)\s+(\w+)\[(\d+)\]\s*=\s*\{(.*?)\};", body_nc, re.S):
            typ, an, n, init = am.group(1), am.group(2), int(am.group(3)), am.group(4)
            vals = [v.strip() for v in init.split(",") if v.strip()]
            vals = [int(v == "true") if typ == "bool" else int(v) for v in vals]
            assert len(vals) == n, (name, an, len(vals), n)
            case["arrays"][an] = vals
        for pm in re.finditer(r"EuclideanPoint<double,\s*3>\s+(\w+)\[(\d+)\]\s*=\s*\{(.*?)\};", body_nc, re.S):
            pts = re.findall(r"EuclideanPoint<double,\s*3>\(([^)]*)\)", pm.group(3))
            case["points"][pm.group(1)] = [[float(x) for x in p.split(",")] for p in pts]
            assert len(pts) == int(pm.group(2))
        st = re.search(r"BOOST_CHECK_EQUAL\(status,\s*cupcfd::error::(\w+)\)", body_nc)
        case["expect_status"] = st.group(1) if st else None
        for sm in re.finditer(r"BOOST_CHECK_EQUAL\((\w+),\s*(-?\d+)\)", body_nc):
            case["scalars"][sm.group(1)] = int(sm.group(2))
        cases.append(case)
    return cases


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CUPCFD_REFERENCE")
    if not ref:
        sys.exit("usage: %s REFERENCE_CHECKOUT (or set CUPCFD_REFERENCE)" % sys.argv[0])
    src = os.path.join(ref, REL)
    with open(src) as fh:
        cases = parse(fh.read())
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "meshstructgen_golden.json")
    with open(out, "w") as fh:
        json.dump({"source": REL, "cases": cases}, fh, indent=1)
    print(f"{len(cases)} cases -> {out}")


if __name__ == "__main__":
    main()
