"""Extract the known-answer data of the reference's cubic-sampling unit tests.

Reads TestCase/MPhysics/DataStructure/UnitTest-ScalarGrid/
UnitTest-CellCenteredScalarField.cu of a junwei-jiang/Hybrid-Fluid-Simulation
checkout and writes sampling_golden.json beside this
script.  Every case that samples a cell-centred scalar field with
ESamplingAlgorithm::CATMULLROM / MONOCATMULLROM / CUBICBRIDSON /
CLAMPCUBICBRIDSON is recorded with:

* the source resolution, origin and spacing, and the formula that fills it;
* the sample-point resolution and the three position formulas;
* every expectation EXPECT_LT(abs(DstFieldResultData[i] -/+ v), ...), or,
  for the cases checked in a loop, the formula the loop compares against.

Formulas are kept as the C++ text of the test (in terms of i, j, k and
Res.x / Res.y); tests/test_oracle_golden.py evaluates them.

    python tests/golden/extract_sampling_golden.py <reference root>
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REL = "TestCase/MPhysics/DataStructure/UnitTest-ScalarGrid/UnitTest-CellCenteredScalarField.cu"

NUM = r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?"
RE_RES = re.compile(r"Vector3i\s+(Res2?)\s*=\s*Vector3i\(\s*(\d+)\s*,\s*(\d+)\s*,\s*(\d+)\s*\)")
RE_SRC = re.compile(r"SrcScalarFieldData\[i \* Res\.x \* Res\.y \+ j \* Res\.x \+ k\]\s*=\s*(.+);")
RE_POS = re.compile(r"PosVectorFieldData([XYZ])\[i \* (Res2?)\.x \* Res2?\.y \+ j \* Res2?\.x \+ k\]\s*=\s*(.+);")
RE_FIELD = re.compile(r"CCSSrcField\(Res,\s*Vector3\(([^)]*)\),\s*Vector3\(([^)]*)\)")
RE_SAMPLE = re.compile(r"CCSSrcField\.sampleField\(CCVPosField,\s*CCSDstField,\s*ESamplingAlgorithm::(\w+)\)")
RE_EXPECT = re.compile(r"EXPECT_LT\(abs\(DstFieldResultData\[(\d+)\]\s*([-+])\s*(" + NUM + r")\),")
RE_LOOP = re.compile(r"EXPECT_LT\(abs\(DstFieldResultData\[i \* Res2?\.x \* Res2?\.y \+ j \* Res2?\.x \+ k\]\s*-\s*(.+)\),"
                     r"\s*GRID_SOLVER_EPSILON\)")


def parse(path):
    with open(path, encoding="latin-1") as f:
        lines = f.read().splitlines()
    cases, cur = [], None
    for ln, line in enumerate(lines, 1):
        m = RE_RES.search(line)
        if m and m.group(1) == "Res":
            cur = {"line": ln, "res": [int(m.group(2)), int(m.group(3)), int(m.group(4))], "pos": {}, "expect": []}
            cases.append(cur)
            continue
        if cur is None:
            continue
        if m and m.group(1) == "Res2":
            cur["res2"] = [int(m.group(2)), int(m.group(3)), int(m.group(4))]
        m = RE_SRC.search(line)
        if m:
            cur["src"] = m.group(1).strip()
        m = RE_POS.search(line)
        if m:
            cur["pos"][m.group(1)] = m.group(3).strip()
        m = RE_FIELD.search(line)
        if m:
            cur["origin"] = [float(v) for v in m.group(1).split(",")]
            cur["spacing"] = [float(v) for v in m.group(2).split(",")]
        m = RE_SAMPLE.search(line)
        if m and "alg" not in cur:
            cur["alg"] = m.group(1)
            cur["sample_line"] = ln
        m = RE_EXPECT.search(line)
        if m:
            v = float(m.group(3))
            cur["expect"].append({"index": int(m.group(1)), "value": v if m.group(2) == "-" else -v, "line": ln})
        m = RE_LOOP.search(line)
        if m:
            cur["expect_formula"] = m.group(1).strip()
            cur["expect_line"] = ln
    keep = [c for c in cases if c.get("alg") in ("CATMULLROM", "MONOCATMULLROM", "CUBICBRIDSON", "CLAMPCUBICBRIDSON")
            and "src" in c and len(c["pos"]) == 3 and (c["expect"] or "expect_formula" in c)]
    return keep


def main():
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    base = sys.argv[1]
    cases = parse(os.path.join(base, REL))
    out = {"source": "junwei-jiang/Hybrid-Fluid-Simulation " + REL, "cases": cases}
    dst = os.path.join(HERE, "sampling_golden.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)
    n = sum(len(c["expect"]) + ("expect_formula" in c) for c in cases)
    print(f"wrote {dst}: {len(cases)} cases, {n} expectations")


if __name__ == "__main__":
    main()
