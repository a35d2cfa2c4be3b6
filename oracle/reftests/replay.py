"""Replay the reference's own unit tests against the CPU oracle.

build.sh compiles the reference's gtest sources (read in place from the
reference checkout) against shim/refapi.h, which restates the reference's
C++ API over oracle/hfg_oracle.cpp.  Running the binaries evaluates every
EXPECT_* of those sources on the oracle's results.  This script builds,
runs and summarises them; with --write it stores the summary as
tests/golden/reference_replay.json, the record the CPU tests check.

Test infrastructure only.

    python oracle/reftests/replay.py <reference root> [--planted] [--write]
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
ROOT = os.path.dirname(ORACLE)
RECORD = os.path.join(ROOT, "tests", "golden", "reference_replay.json")

# The reference file each suite comes from, relative to its checkout.
SOURCES = {
    "ParticlesAdvection": "TestCase/MPhysics/Euler/UnitTest-ParticlesAdvection/UnitTest-ParticlesAdvection.cu",
    "SemiLagrangian": "TestCase/MPhysics/Euler/UnitTest-SemiLagrangian/UnitTest-SemiLagrangian.cu",
    "BoundarySDF": "TestCase/MPhysics/Euler/UnitTest-BoundarySDF/UnitTest-BoundarySDF.cu",
    "ExternalForces": "TestCase/MPhysics/Euler/UnitTest-ExternalForces/UnitTest-ExternalForces.cu",
    "Extrapolation": "TestCase/MPhysics/Euler/UnitTest-Extrapolation/UnitTest-Extrapolation.cu",
    "PressureSolver": "TestCase/MPhysics/Euler/UnitTest-PressureSolver/UnitTest-PressureSolver.cu",
    "HybridHelper": "TestCase/MPhysics/Hybrid/UnitTest-HybridHelper/UnitTest-HybridHelper.cu",
    "GridFluidSolver": "TestCase/MPhysics/Euler/IntegrationTest-GridFluidSolver/IntegrationTest-GridFluidSolver.cpp",
    "CellCenteredScalarField": "TestCase/MPhysics/DataStructure/UnitTest-ScalarGrid/UnitTest-CellCenteredScalarField.cu",
    "CellCenteredVectorField":
        "TestCase/MPhysics/DataStructure/UnitTest-CellCenteredVectorGrid/UnitTest-CellCenteredVectorField.cu",
    "FaceCenteredVectorField":
        "TestCase/MPhysics/DataStructure/UnitTest-FaceCenteredVectorGrid/UnitTest-FaceCenteredVectorField.cu",
}


def build(ref, planted=False):
    cmd = ["bash", os.path.join(HERE, "build.sh"), ref] + (["planted"] if planted else [])
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
    return os.path.join(ORACLE, "_ref", "reftests_planted" if planted else "reftests")


def run(bindir):
    """Runs every suite; returns {suite: {"file": ..., "tests": [...]}}."""
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for suite in sorted(SOURCES):
            dst = os.path.join(tmp, suite + ".json")
            subprocess.run([os.path.join(bindir, suite), dst], check=True, cwd=tmp, stdout=subprocess.DEVNULL,
                           timeout=600)
            with open(dst) as f:
                tests = json.load(f)["tests"]
            for t in tests:
                # keep the lines that failed; count the rest
                t["lines_evaluated"] = len(t["lines"])
                t["lines"] = [ln for ln in t["lines"] if ln["failed"]]
            out[suite] = {"file": SOURCES[suite], "tests": tests}
    return out


def checked(t):
    """A test whose expectations were evaluated on results of the oracle."""
    return t["status"] == "ran" and t["oracle_calls"] > 0


def summary(res):
    """Per suite: tests checked against the oracle, tests that only touch
    the containers of shim/refapi.h (field constructors, assignment), tests
    not restated, and the expectations evaluated / failed in the checked ones."""
    rows = []
    for suite, s in res.items():
        chk = [t for t in s["tests"] if checked(t)]
        plumbing = [t for t in s["tests"] if t["status"] == "ran" and not checked(t)]
        rows.append((suite, len(chk), len(plumbing), len(s["tests"]) - len(chk) - len(plumbing),
                     sum(t["evaluated"] for t in chk), sum(t["failed"] for t in s["tests"] if t["status"] == "ran")))
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("reference", help="root of the reference checkout")
    ap.add_argument("--planted", action="store_true", help="replay against the oracle with a planted mistake")
    ap.add_argument("--write", action="store_true", help="store the summary as " + RECORD)
    a = ap.parse_args()
    res = run(build(a.reference, a.planted))
    for suite, chk, plumbing, skipped, ev, fail in summary(res):
        print(f"{suite:24s} checked {chk:3d}  containers only {plumbing:2d}  not restated {skipped:2d}  "
              f"expectations {ev:8d}  failed {fail:6d}")
    if a.write and not a.planted:
        with open(RECORD, "w") as f:
            json.dump({"source": "junwei-jiang/Hybrid-Fluid-Simulation unit tests replayed on the CPU oracle "
                                 "(oracle/reftests/replay.py)", "suites": res}, f, indent=1, sort_keys=True)
        print("wrote", RECORD)
    return 0


if __name__ == "__main__":
    sys.exit(main())
