"""Extracts the reference's expectations for its HDF5 mesh fixture into
tests/golden/meshhdf5source_golden.json.

    python tests/golden/make_hdf5_golden.py [path/to/reference]

Source: tests/geometry/mesh/implementation/source/MeshHDF5SourceTests.cpp of
the reference (Boost.Test), read as text. For every test case (including the
ones the reference has commented out, marked ``active: false``), this
records the label arrays it passes in, the int / bool / double arrays it
expects and the scalar counts it checks. tests/test_hdf5.py replays them
against this library's reader on the fixture
tests/geometry/mesh/data/MeshHDF5.hdf5 (read from the reference tree, so
those checks run where the reference is present).
"""
from __future__ import annotations

import json
import os
import re
import sys

REL = "tests/geometry/mesh/implementation/source/MeshHDF5SourceTests.cpp"
FIXTURE = "tests/geometry/mesh/data/MeshHDF5.hdf5"


def _num(v, typ):
    if typ == "bool":
        return int(v == "true")
    return int(v) if typ == "int" else float(v)


def parse(text):
    cases = []
    for m in re.finditer(r"BOOST_AUTO_TEST_CASE\((\w+)\)\s*\{(.*?)\n\}", text, re.S):
        name, body = m.group(1), m.group(2)
        active = "/*" not in body
        body_nc = re.sub(r"//[^\n]*", "", body).replace("/*", "").replace("*/", "")
        call = re.search(r"status\s*=\s*file\.(\w+)\(", body_nc) or re.search(r"file\.(\w+)\(", body_nc)
        case = {"name": name, "active": active, "method": call.group(1) if call else None, "arrays": {},
                "scalars": {}}
        for am in re.finditer(r"\b(int|bool|double)\s+(\w+)\[(\d+)\]\s*=\s*\{(.*?)\};", body_nc, re.S):
            typ, an, n, init = am.group(1), am.group(2), int(am.group(3)), am.group(4)
            vals = [_num(v.strip(), typ) for v in init.split(",") if v.strip()]
            case["arrays"][an] = {"type": typ, "n": n, "values": vals}
        for sm in re.finditer(r"BOOST_CHECK_EQUAL\((\w+),\s*(-?\d+)\)", body_nc):
            case["scalars"][sm.group(1)] = int(sm.group(2))
        cases.append(case)
    return cases


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CUPCFD_REFERENCE")
    if not ref:
        sys.exit("usage: %s REFERENCE_CHECKOUT (or set CUPCFD_REFERENCE)" % sys.argv[0])
    with open(os.path.join(ref, REL)) as fh:
        cases = parse(fh.read())
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "meshhdf5source_golden.json")
    with open(out, "w") as fh:
        json.dump({"source": REL, "fixture": FIXTURE, "cases": cases}, fh, indent=1)
    print(f"{len(cases)} cases -> {out}")


if __name__ == "__main__":
    main()
