"""The oracle against the reference's own known-answer tests (CPU only).

tests/golden/reference_golden.json holds the data of the reference's gtest
suites (extracted by tests/golden/extract_reference_golden.py): explicit
inputs and every `EXPECT_LT(abs(v[i] -/+ c), GRID_SOLVER_EPSILON)` with its
source line.  Each test below restates how the reference test wires that
data and checks the oracle -- the CPU restatement of the grid step that the
GPU parity tests compare against -- to the reference's own tolerance
GRID_SOLVER_EPSILON = 1e-4 (MPhysics/Common.h:103).  This pins the oracle.
"""
import json
import os

import numpy as np
import pytest

import oracle

EPS = 1e-4
UNKNOWN = float(np.finfo(np.float32).max)
with open(os.path.join(os.path.dirname(__file__), "golden", "reference_golden.json")) as f:
    GOLDEN = json.load(f)["suites"]


def case(suite, name):
    return GOLDEN[suite]["tests"][name]


def check(results, expects, label):
    """results: var name -> flat array.  Every expectation must hold to EPS
    (UNKNOWN entries must be exactly the sentinel)."""
    assert expects, f"{label}: no expectations extracted"
    bad = []
    for e in expects:
        if e["var"] not in results:
            continue
        got = float(results[e["var"]][e["index"]])
        want = e["value"]
        ok = (got == UNKNOWN) if want >= UNKNOWN else abs(got - want) < EPS
        if not ok:
            bad.append((e["var"], e["index"], want, got, e["line"]))
    assert not bad, f"{label}: {len(bad)} mismatches, first {bad[:5]}"
    return sum(1 for e in expects if e["var"] in results)


# ---------------------------------------------------------------- extrapolation
# UnitTest-Extrapolation.cu: inputs filled with UNKNOWN plus listed values,
# extrapolatingDataInvoker(src, markers, depth) on a cell-centred scalar
# (1-3), a face-centred vector (4) or a cell-centred vector (5) field.
EXTRAP = {
    "Extrapolation_buildDisMarkers1": ("cc", 3), "Extrapolation_buildDisMarkers3": ("cc", 200),
    "Extrapolation_buildDisMarkers4": ("fc", 3), "Extrapolation_buildDisMarkers5": ("ccv", 3),
    "Extrapolation_extrapolationData1": ("cc", 3), "Extrapolation_extrapolationData2": ("cc", 2),
    "Extrapolation_extrapolationData3": ("cc", 200), "Extrapolation_extrapolationData4": ("fc", 3),
    "Extrapolation_extrapolationData5": ("ccv", 3),
}


@pytest.mark.parametrize("name", sorted(EXTRAP))
def test_extrapolation_golden(name):
    kind, depth = EXTRAP[name]
    t = case("Extrapolation", name)
    res = t["res"]["Res"]
    if kind == "cc":
        grids = {"": res}
        arrays = {"": np.full(res[::-1], UNKNOWN, np.float32).reshape(-1)}
        names = {"ScalarFieldData": ""}
    else:
        if kind == "fc":
            grids = {"X": [res[0] + 1, res[1], res[2]], "Y": [res[0], res[1] + 1, res[2]],
                     "Z": [res[0], res[1], res[2] + 1]}
        else:
            grids = {"X": res, "Y": res, "Z": res}
        arrays = {a: np.full(g[::-1], UNKNOWN, np.float32).reshape(-1) for a, g in grids.items()}
        names = {"VectorFieldData" + a: a for a in grids}
    for a in t["assign"]:
        arrays[names[a["name"]]][a["index"]] = a["value"]
    results = {}
    for a, g in grids.items():
        vals, mk = oracle.extrapolate(tuple(g), arrays[a], depth, with_markers=True)
        results[f"MarkersResult{a}Vector"] = mk.reshape(-1)
        results[f"ExtrapolationResult{a}Vector"] = vals.reshape(-1)
    n = check(results, t["expect"], name)
    for u in t["unknown_except"]:
        arr = results[u["var"]]
        keep = np.ones(arr.size, bool)
        keep[u["except"]] = False
        assert np.all(arr[keep] == UNKNOWN), f"{name}: line {u['line']}"
    assert n > 0


# -------------------------------------------------------------- pressure solver
# UnitTest-PressureSolver.cu: spacing (10,20,30) (tests 3 and 4: unit), fluid
# SDF j - c, solid SDF -0.5 with the listed cells +0.5, face velocities and
# solid velocities from index formulas; markers from the SDFs
# (buildFluidMarkersInvoker SDF form) and the reference CG (identity
# preconditioner, sqrt(||r||) < 1e-3, N iterations).
PRESSURE = {
    # name: (fluid offset, vel formulas, solid vel formulas, spacing, dt)
    "PressureSolver_buildMarkers1": (1.5, ("k", "j", "i"), ("1", "0", "0"), (10, 20, 30), 1),
    "PressureSolver_buildVectorb2": (2.5, ("k", "j", "i"), ("1", "0", "0"), (10, 20, 30), 1),
    "PressureSolver_buildFdmMatrixA2": (2.5, ("k", "j", "i"), ("1", "0", "0"), (10, 20, 30), 2),
    "PressureSolver_MatrixFreePCG1": (2.5, ("k", "j", "i"), ("1", "0", "0"), (10, 20, 30), 2),
    "PressureSolver_PressureSolver1": (2.5, ("k", "j", "i"), ("k + 1", "j + 1", "i + 1"), (10, 20, 30), 2),
    "PressureSolver_PressureSolver2": (2.5, ("k", "j", "i"), ("1", "0", "0"), (10, 20, 30), 2),
    "PressureSolver_PressureSolver3": (2.5, ("4 - k", "0", "0"), ("1", "0", "0"), (1, 1, 1), 1),
    "PressureSolver_PressureSolver4": (2.5, ("0", "-9.8", "0"), ("0", "0", "0"), (1, 1, 1), 1),
}


def face_field(res, axis, formula):
    shape = [res[2], res[1], res[0]]
    shape[2 - axis] += 1
    i, j, k = np.meshgrid(np.arange(shape[0]), np.arange(shape[1]), np.arange(shape[2]), indexing="ij")
    return np.asarray(eval(formula, {"i": i, "j": j, "k": k}) + 0 * i, np.float32)


@pytest.mark.parametrize("name", sorted(PRESSURE))
def test_pressure_golden(name):
    off, vf, sf, h, dt = PRESSURE[name]
    t = case("PressureSolver", name)
    res = tuple(t["res"]["Res"])
    j = np.arange(res[1])[None, :, None]
    fluid = np.broadcast_to(j - off, res[::-1]).astype(np.float32).copy().reshape(-1)
    solid = np.full(res[::-1], -0.5, np.float32).reshape(-1)
    for a in t["assign"]:
        {"SolidSDFScalarFieldData": solid, "FluidSDFScalarFieldData": fluid}[a["name"]][a["index"]] = a["value"]
    vel = [face_field(res, a, vf[a]) for a in range(3)]
    svel = [face_field(res, a, sf[a]) for a in range(3)]
    mk = oracle.markers_from_sdf(res, solid, fluid)
    A = oracle.build_matrix_a(res, h, dt, mk)
    b = oracle.build_rhs(res, h, vel, svel, mk)
    v_out, p, st = oracle.project(res, h, dt, mk, vel, svel, precond=0, tol_mode=0, tol=1e-3, max_iter=-1)
    results = {"MarkersResultVector": mk.reshape(-1).astype(np.float32), "FdmMatrixAGPUResult": A,
               "VectorbResult": b.reshape(-1), "VectorxResult": p.reshape(-1),
               "FieldResultDataX": v_out[0].reshape(-1), "FieldResultDataY": v_out[1].reshape(-1),
               "FieldResultDataZ": v_out[2].reshape(-1)}
    assert check(results, t["expect"], name) > 0


def test_pressure_fp32_matches_fp64_on_golden_case():
    """The FP32 oracle (each operation rounded to FP32) and the FP64 oracle
    agree on the 4^3 PCG known answer (MatrixFreePCG1)."""
    off, vf, sf, h, dt = PRESSURE["PressureSolver_MatrixFreePCG1"]
    t = case("PressureSolver", "PressureSolver_MatrixFreePCG1")
    res = tuple(t["res"]["Res"])
    j = np.arange(res[1])[None, :, None]
    fluid = np.broadcast_to(j - off, res[::-1]).astype(np.float32).copy().reshape(-1)
    solid = np.full(res[::-1], -0.5, np.float32).reshape(-1)
    for a in t["assign"]:
        {"SolidSDFScalarFieldData": solid, "FluidSDFScalarFieldData": fluid}[a["name"]][a["index"]] = a["value"]
    vel = [face_field(res, a, vf[a]) for a in range(3)]
    svel = [face_field(res, a, sf[a]) for a in range(3)]
    mk = oracle.markers_from_sdf(res, solid, fluid)
    _, p32, _ = oracle.project(res, h, dt, mk, vel, svel, 0, 0, 1e-3, -1, dbl=0)
    _, p64, _ = oracle.project(res, h, dt, mk, vel, svel, 0, 0, 1e-3, -1, dbl=1)
    np.testing.assert_allclose(p32, p64, rtol=1e-5, atol=1e-4)


# ---------------------------------------------------------- integration tests
def _integration_case(kind):
    """IntegrationTest-GridFluidSolver.cpp:228-402 inputs (4^3, unit spacing)."""
    res = (4, 4, 4)
    g = case("GridFluidSolver", "GridFluidSolver1" if kind == 1 else "GridFluidSolver2")
    fluid = np.zeros(res[::-1], np.float32)
    for jj in range(4):
        fluid[:, jj, :] = jj - 2.5
    solid = np.full(res[::-1], -0.5, np.float32)
    for a in g["assign"]:
        {"SolidSDFScalarFieldData": solid, "FluidSDFScalarFieldData": fluid}[a["name"]].reshape(-1)[a["index"]] = \
            a["value"]
    return res, solid, fluid


@pytest.mark.parametrize("dbl", [0, 1])
def test_integration_rest_and_free_fall(dbl):
    # GridFluidSolver1 (:228-311): closed water column stays at rest, dt = 1
    res, solid, fluid = _integration_case(1)
    o = oracle.Solver(1.0, res, dbl=dbl)
    o.set_fluid_domain_field(fluid)
    o.add_solid_boundary(solid)
    for _ in range(3):
        o.update()
        assert max(np.abs(c).max() for c in o.velocity_field()) < EPS
    # GridFluidSolver2 (:313-402): free fall u_y = -9.8 dt (k + 1), dt = 0.01
    res, solid, fluid = _integration_case(2)
    dt = 0.01
    o = oracle.Solver(dt, res, dbl=dbl)
    o.set_fluid_domain_field(fluid)
    o.add_solid_boundary(solid)
    for k in range(10):
        o.update()
        vy = o.velocity_field()[1].reshape(-1)
        for f in (25, 26, 29, 30, 33, 34, 45, 46, 49, 50, 53, 54):
            assert abs(vy[f] + 9.8 * dt * (k + 1)) < EPS


def test_golden_fixture_coverage():
    """The expectations the tests above evaluate on the oracle (not merely
    extracted): every one of the extrapolation and pressure cases.  The other
    suites of the step are replayed whole (tests/test_reference_replay.py)."""
    n = {}
    for suite, names in (("Extrapolation", EXTRAP), ("PressureSolver", PRESSURE)):
        n[suite] = sum(len(case(suite, name)["expect"]) for name in names)
    assert n["Extrapolation"] >= 250 and n["PressureSolver"] >= 200, n


# ------------------------------------------------- cubic samplers (DataStructure)
SAMPLING = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "sampling_golden.json")))
SAMPLING_ALG = {"CATMULLROM": 1, "MONOCATMULLROM": 2, "CUBICBRIDSON": 3, "CLAMPCUBICBRIDSON": 4}


class _Res:
    def __init__(self, r):
        self.x, self.y, self.z = r


def _grid_eval(expr, res, dtype=np.float32):
    """Evaluate a formula of the reference test in i (z), j (y), k (x) over a
    grid, with the test's C++ int division ((Int)(k / 2)) as truncation."""
    py = expr.replace("(Int)", "int")
    out = np.empty((res[2], res[1], res[0]), dtype)
    env = {"Res": _Res(res), "Res2": _Res(res), "int": int}
    for i in range(res[2]):
        for j in range(res[1]):
            for k in range(res[0]):
                out[i, j, k] = eval(py, env, {"i": i, "j": j, "k": k})
    return out


@pytest.mark.parametrize("case", SAMPLING["cases"], ids=lambda c: f"{c['alg']}@{c['line']}")
def test_cubic_sampling_golden(case):
    """UnitTest-CellCenteredScalarField.cu: the oracle's Catmull-Rom,
    monotonic Catmull-Rom, Bridson and clamped Bridson samplers reproduce
    every expectation of the reference's own tests (tolerance 1e-4, the
    tests' GRID_SOLVER_EPSILON), in FP32 and FP64."""
    res = case["res"]
    dres = case.get("res2", res)
    src = _grid_eval(case["src"], res)
    pos = np.stack([_grid_eval(case["pos"][a], dres) for a in "XYZ"], axis=-1).reshape(-1, 3)
    for dbl in (0, 1):
        out = oracle.sample_cc(res, case["origin"], case["spacing"], src, pos, alg=SAMPLING_ALG[case["alg"]], dbl=dbl)
        for e in case["expect"]:
            assert abs(out[e["index"]] - e["value"]) < 1e-4, (e, out[e["index"]])
        if "expect_formula" in case:
            ref = _grid_eval(case["expect_formula"], dres).reshape(-1)
            assert np.abs(out - ref).max() < 1e-4


def test_sampling_fixture_coverage():
    algs = {c["alg"] for c in SAMPLING["cases"]}
    assert algs == set(SAMPLING_ALG)
    assert sum(len(c["expect"]) + ("expect_formula" in c) for c in SAMPLING["cases"]) >= 70
