"""The reference's own unit tests, replayed on the CPU oracle (CPU only).

oracle/reftests/build.sh compiles the reference's gtest sources, unchanged
and read in place from a reference checkout, against
oracle/reftests/shim/refapi.h: the reference's C++ API (fields, particles,
semi-Lagrangian solver, boundaries, external forces, pressure solver, the
particle/grid invokers) restated over oracle/hfg_oracle.cpp.  Running them
evaluates every EXPECT_* of those sources on the oracle's results, with the
tests' own tolerance (GRID_SOLVER_EPSILON = 1e-4, MPhysics/Common.h:103).
oracle/reftests/replay.py stores the outcome as
tests/golden/reference_replay.json.

This pins the oracle -- the checker of every GPU parity test -- for the
particle and advection half of the step (P2G, G2P, CFL particle advection,
markers, binning, back-trace and semi-Lagrangian advection, trilinear and
cubic sampling, boundaries) as well as the pressure and extrapolation half,
and the hybrid coupler's helpers that follow the step (field mixing, fluid
density, inside / outside distance fields).

test_replay_record checks the committed record; the live tests rebuild and
rerun the replay when HFG_REFERENCE_ROOT names a reference checkout.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RECORD_PATH = os.path.join(ROOT, "tests", "golden", "reference_replay.json")
with open(RECORD_PATH) as f:
    RECORD = json.load(f)["suites"]
REF = os.environ.get("HFG_REFERENCE_ROOT")
sys.path.insert(0, os.path.join(ROOT, "oracle", "reftests"))
import replay  # noqa: E402

# Every suite of the grid step, with the least number of expectations the
# record must show evaluated on oracle results (ParticlesAdvection.cu:112-4196
# et al.; the counts include the loops over whole grids).
FLOORS = {
    "ParticlesAdvection": 2000, "SemiLagrangian": 70000, "BoundarySDF": 14000, "ExternalForces": 190000,
    "Extrapolation": 1000, "PressureSolver": 1300, "GridFluidSolver": 800, "CellCenteredScalarField": 9000,
    "CellCenteredVectorField": 20000, "FaceCenteredVectorField": 9000,
    # the hybrid coupler's helpers (UnitTest-HybridHelper.cu: field mixing,
    # the fluid domain from a box, fluid density and the inside / outside
    # distance fields)
    "HybridHelper": 850,
}

# Tests of those sources that are not replayed, and why.
NOT_RESTATED = {
    ("BoundarySDF", "ReSamplingBoundarySDF"): "generateSDF: mesh voxelisation through D3D11",
    ("CellCenteredScalarField", "CellCenteredScalarField_PlusAndScale"): "field arithmetic",
    ("CellCenteredScalarField", "CellCenteredScalarField_FieldGradient"): "gradient, off the step",
    ("CellCenteredScalarField", "CellCenteredScalarField_FieldLaplacian"): "laplacian, off the step",
    ("CellCenteredVectorField", "CellCenteredVectorField_PlusAndScale"): "field arithmetic",
    ("CellCenteredVectorField", "CellCenteredVectorField_FieldDivergence"): "cell-centred divergence, off the step",
    ("CellCenteredVectorField", "CellCenteredVectorField_FieldCurl"): "curl, off the step",
    ("FaceCenteredVectorField", "FaceCenteredVectorField_PlusAndScale"): "field arithmetic",
    ("FaceCenteredVectorField", "FaceCenteredVectorField_FieldCurl"): "curl, off the step",
    ("GridFluidSolver", "GridFluidSolver3"): "frame test on data files from the author's own drive",
    ("GridFluidSolver", "GridFluidSolver4"): "frame test on data files from the author's own drive",
    ("GridFluidSolver", "GridFluidSolver5"): "frame test on data files from the author's own drive",
    ("GridFluidSolver", "GridFluidSolver7"): "frame test on data files from the author's own drive",
}


def _check(res):
    for suite, checked, _plumbing, _skipped, evaluated, failed in replay.summary(res):
        assert failed == 0, f"{suite}: {failed} expectations of the reference's tests fail on the oracle"
        assert evaluated >= FLOORS[suite], f"{suite}: only {evaluated} expectations evaluated"
        assert checked > 0
    skipped = {(s, t["test"]) for s, v in res.items() for t in v["tests"] if t["status"] != "ran"}
    assert skipped == set(NOT_RESTATED), skipped ^ set(NOT_RESTATED)
    # the frame tests stop at their first call into the solver; nothing else
    # stops early
    for (s, name), why in NOT_RESTATED.items():
        t = next(t for t in res[s]["tests"] if t["test"] == name)
        assert t["why"], name


def test_replay_record():
    """Every expectation of the replayed reference tests held on the oracle
    when the record was made, in every suite of the step."""
    assert set(RECORD) == set(FLOORS)
    _check(RECORD)


def test_replay_covers_the_particle_chain():
    """The suites that pin the particle/advection half: every test in them
    reached the oracle and none failed."""
    for suite in ("ParticlesAdvection", "SemiLagrangian", "BoundarySDF"):
        for t in RECORD[suite]["tests"]:
            if (suite, t["test"]) in NOT_RESTATED:
                continue
            assert t["oracle_calls"] > 0 and t["evaluated"] > 0 and t["failed"] == 0, (suite, t["test"])


@pytest.mark.skipif(not REF or not os.path.isdir(REF or ""), reason="HFG_REFERENCE_ROOT names no reference checkout")
def test_replay_live():
    """Rebuild and rerun the replay on the current oracle: it passes and
    evaluates what the record says."""
    res = replay.run(replay.build(REF))
    _check(res)
    for suite, s in res.items():
        got = {t["test"]: t["evaluated"] for t in s["tests"]}
        want = {t["test"]: t["evaluated"] for t in RECORD[suite]["tests"]}
        assert got == want, suite


@pytest.mark.skipif(not REF or not os.path.isdir(REF or ""), reason="HFG_REFERENCE_ROOT names no reference checkout")
def test_replay_catches_a_planted_mistake():
    """An oracle built with a deliberate 1 % error in the linear transfer
    kernel and in trilinear sampling fails the replayed tests of P2G/G2P,
    particle advection, the semi-Lagrangian solver and sampling."""
    res = replay.run(replay.build(REF, planted=True))
    failed = {suite: failed for suite, _c, _p, _s, _e, failed in replay.summary(res)}
    for suite in ("ParticlesAdvection", "SemiLagrangian", "CellCenteredScalarField", "FaceCenteredVectorField"):
        assert failed[suite] > 0, suite
