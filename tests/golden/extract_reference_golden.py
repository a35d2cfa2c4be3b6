"""Extract the known-answer data of the reference's own unit tests.

Reads the gtest sources of junwei-jiang/Hybrid-Fluid-Simulation (the
TestCase/MPhysics/Euler directory of a checkout) and writes reference_golden.json
beside this script: for every TEST block its resolutions, explicit input
assignments (NAME[i] = v), vector fills, scalar parameters, and every
expectation of the form EXPECT_LT(abs(VAR[i] -/+ value), GRID_SOLVER_EPSILON),
plus the "every other entry is UNKNOWN" loops (if (i != a && i != b ...)).
Each record keeps its source line so a test can cite it.

Only data is extracted; the tests in tests/test_oracle_golden.py restate how
each reference test wires that data (which arrays are inputs, which stage
runs) and check the oracle against the expectations.

    python tests/golden/extract_reference_golden.py <reference root>/TestCase/MPhysics/Euler

The particle, semi-Lagrangian, boundary and external-force suites are not
extracted here: their tests are replayed whole on the oracle
(oracle/reftests, tests/test_reference_replay.py).
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = {
    "Extrapolation": "UnitTest-Extrapolation/UnitTest-Extrapolation.cu",
    "PressureSolver": "UnitTest-PressureSolver/UnitTest-PressureSolver.cu",
    "GridFluidSolver": "IntegrationTest-GridFluidSolver/IntegrationTest-GridFluidSolver.cpp",
}

NUM = r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?"
RE_TEST = re.compile(r"^TEST\((\w+),\s*(\w+)\)")
RE_RES = re.compile(r"Vector3i\s+(\w+)\s*=\s*Vector3i\(\s*(\d+)\s*,\s*(\d+)\s*,\s*(\d+)\s*\)")
RE_FILL = re.compile(r"vector<Real>\s+(\w+)\(([^;]*?)(?:,\s*(UNKNOWN|" + NUM + r"))?\);")
RE_ASSIGN = re.compile(r"^\s*(\w+)\[([0-9 +*\-]+)\]\s*=\s*(" + NUM + r"|UNKNOWN)\s*;")
RE_EXPECT = re.compile(r"EXPECT_LT\(abs\((\w+)\[([0-9 +*\-]+)\]\s*([-+])\s*(UNKNOWN|" + NUM + r")\),\s*GRID_SOLVER_EPSILON\)")
RE_REAL = re.compile(r"^\s*Real\s+(\w+)\s*=\s*(" + NUM + r")\s*;")
RE_EXCEPT = re.compile(r"if\s*\(((?:\s*i\s*!=\s*\d+\s*&&?)*\s*i\s*!=\s*\d+\s*)\)")
RE_LOOP_UNKNOWN = re.compile(r"EXPECT_LT\(abs\((\w+)\[i\]\s*-\s*UNKNOWN\)")

UNKNOWN = 3.4028234663852886e38


def num(tok):
    return UNKNOWN if tok == "UNKNOWN" else float(tok)


def parse(path):
    tests = {}
    cur = None
    pending_except = None
    with open(path, encoding="latin-1") as f:
        lines = f.read().splitlines()
    for ln, line in enumerate(lines, 1):
        m = RE_TEST.match(line)
        if m:
            cur = {"line": ln, "res": {}, "fills": {}, "assign": [], "expect": [], "real": {}, "unknown_except": [],
                   "calls": []}
            tests[m.group(2)] = cur
            pending_except = None
            continue
        if cur is None:
            continue
        for m in RE_RES.finditer(line):
            cur["res"][m.group(1)] = [int(m.group(2)), int(m.group(3)), int(m.group(4))]
        m = RE_FILL.search(line)
        if m:
            cur["fills"][m.group(1)] = num(m.group(3)) if m.group(3) else 0.0
        m = RE_ASSIGN.match(line)
        if m:
            cur["assign"].append({"name": m.group(1), "index": int(eval(m.group(2))), "value": num(m.group(3)),
                                  "line": ln})
        m = RE_REAL.match(line)
        if m:
            cur["real"][m.group(1)] = float(m.group(2))
        for m in RE_EXPECT.finditer(line):
            v = num(m.group(4))
            exp = v if m.group(3) == "-" else -v
            cur["expect"].append({"var": m.group(1), "index": int(eval(m.group(2))), "value": exp, "line": ln})
        m = RE_EXCEPT.search(line)
        if m:
            pending_except = ([int(x) for x in re.findall(r"\d+", m.group(1))], ln)
        m = RE_LOOP_UNKNOWN.search(line)
        if m and pending_except is not None:
            cur["unknown_except"].append({"var": m.group(1), "except": pending_except[0], "line": pending_except[1]})
            pending_except = None
        if "Invoker(" in line or ".solvePressure(" in line or ".update(" in line or "advect(" in line:
            cur["calls"].append({"text": line.strip(), "line": ln})
    return tests


def main():
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    base = sys.argv[1]
    out = {"source": "junwei-jiang/Hybrid-Fluid-Simulation TestCase/MPhysics/Euler", "suites": {}}
    for suite, rel in FILES.items():
        p = os.path.join(base, rel)
        if not os.path.exists(p):
            continue
        out["suites"][suite] = {"file": "TestCase/MPhysics/Euler/" + rel, "tests": parse(p)}
    dst = os.path.join(HERE, "reference_golden.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)
    n = sum(len(t["expect"]) for s in out["suites"].values() for t in s["tests"].values())
    print(f"wrote {dst}: {n} expectations")


if __name__ == "__main__":
    main()
