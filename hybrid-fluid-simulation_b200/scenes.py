"""Seeded synthetic dam-break scenes for the grid step.

A scene is the input set of one CGridFluidSolver run (the object the
reference's integration tests build by hand, e.g. TestCase/MPhysics/Euler/
IntegrationTest-GridFluidSolver/IntegrationTest-GridFluidSolver.cpp:490-560):

* an nx x ny x nz grid on the unit cube, spacing (1/nx, 1/ny, 1/nz), origin 0;
* boundary 0: the walls -- the outermost cell layer on all six sides; its
  SDF is the signed distance to the inner box, negative inside the wall;
* further static or moving solids (spheres, boxes) as extra boundaries;
* the fluid domain: cells whose centre has x < fx and y < fy (all z), via
  generateFluidDomainFromBBox (EulerSolverTool.cu:581-608);
* particles seeded per fluid, non-solid cell by the counter-based stream.

All SDFs are evaluated at cell centres in float64 and stored as float32.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Tuple

import numpy as np


@dataclasses.dataclass
class Solid:
    kind: str                 # "sphere" | "box" | "walls"
    center: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    size: Tuple[float, float, float] = (0.0, 0.0, 0.0)   # radius in size[0] for spheres, full side lengths for boxes
    velocity: Tuple[float, float, float] = (0.0, 0.0, 0.0)


@dataclasses.dataclass
class Scene:
    res: Tuple[int, int, int]
    dt: float = 1.0 / 60.0
    fluid_max: Tuple[float, float, float] = (0.4, 0.6, 1.0)
    solids: List[Solid] = dataclasses.field(default_factory=list)
    per_cell: int = 8
    seed: int = 0
    mixing: float = 0.05       # MixingCoefficient m: FLIP weight 1 - m = 0.95
    cfl: float = 1.0
    name: str = "dam-break"

    @property
    def spacing(self) -> Tuple[float, float, float]:
        return tuple(1.0 / n for n in self.res)

    @property
    def origin(self) -> Tuple[float, float, float]:
        return (0.0, 0.0, 0.0)

    @property
    def n_cells(self) -> int:
        return int(self.res[0]) * int(self.res[1]) * int(self.res[2])


def cell_centres(res, spacing, origin=(0.0, 0.0, 0.0)):
    nx, ny, nz = res
    x = origin[0] + (np.arange(nx) + 0.5) * spacing[0]
    y = origin[1] + (np.arange(ny) + 0.5) * spacing[1]
    z = origin[2] + (np.arange(nz) + 0.5) * spacing[2]
    return np.meshgrid(z, y, x, indexing="ij")[::-1]  # X, Y, Z each (nz, ny, nx)


def sdf_walls(res, spacing):
    """Positive inside the inner box [h, 1-h]^3, negative in the wall layer."""
    X, Y, Z = cell_centres(res, spacing)
    lo = np.array(spacing)
    hi = 1.0 - lo
    d = [np.minimum(P - l, u - P) for P, l, u in zip((X, Y, Z), lo, hi)]
    inside = np.minimum(np.minimum(d[0], d[1]), d[2])
    out = np.sqrt(sum(np.minimum(di, 0.0) ** 2 for di in d))
    return np.where(inside >= 0, inside, -out).astype(np.float32)


def sdf_sphere(res, spacing, c, r):
    X, Y, Z = cell_centres(res, spacing)
    return (np.sqrt((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) - r).astype(np.float32)


def sdf_box(res, spacing, c, size):
    X, Y, Z = cell_centres(res, spacing)
    q = [np.abs(P - ci) - si / 2 for P, ci, si in zip((X, Y, Z), c, size)]
    outside = np.sqrt(sum(np.maximum(qi, 0.0) ** 2 for qi in q))
    inside = np.minimum(np.maximum(np.maximum(q[0], q[1]), q[2]), 0.0)
    return (outside + inside).astype(np.float32)


def solid_sdf(scene: Scene, s: Solid) -> np.ndarray:
    if s.kind == "walls":
        return sdf_walls(scene.res, scene.spacing)
    if s.kind == "sphere":
        return sdf_sphere(scene.res, scene.spacing, s.center, s.size[0])
    if s.kind == "box":
        return sdf_box(scene.res, scene.spacing, s.center, s.size)
    raise ValueError(s.kind)


def boundaries(scene: Scene):
    """(sdf, velocity) of every boundary, walls first."""
    out = [(sdf_walls(scene.res, scene.spacing), (0.0, 0.0, 0.0))]
    for s in scene.solids:
        out.append((solid_sdf(scene, s), tuple(s.velocity)))
    return out


def total_solid(scene: Scene) -> np.ndarray:
    """The reference's total boundary field for static solids: -(first solid
    index) inside, FLT_MAX outside (BoundaryTool.cu:3-26)."""
    out = np.full(scene.res[::-1], np.finfo(np.float32).max, np.float32)
    for i, (sdf, _) in enumerate(boundaries(scene)):
        m = (sdf < 0) & (out == np.finfo(np.float32).max)
        out[m] = -(i + 1)
    return out


def fluid_bbox(scene: Scene):
    return (0.0, 0.0, 0.0), tuple(scene.fluid_max)


def dam_break_64(seed: int = 0) -> Scene:
    """64^3, static sphere r=0.15 at (0.5, 0.15, 0.5)."""
    return Scene(res=(64, 64, 64), solids=[Solid("sphere", (0.5, 0.15, 0.5), (0.15, 0, 0))], seed=seed,
                 name="dam-break 64^3, sphere")


def dam_break_256(seed: int = 0, n: int = 256) -> Scene:
    """256^3 (or n^3), two static boxes of side 0.2 resting on the floor."""
    h = 1.0 / n
    boxes = [Solid("box", (0.7, 0.1 + h, 0.3), (0.2, 0.2, 0.2)), Solid("box", (0.7, 0.1 + h, 0.7), (0.2, 0.2, 0.2))]
    return Scene(res=(n, n, n), solids=boxes, seed=seed, name=f"dam-break {n}^3, two boxes")


@dataclasses.dataclass
class SinePath:
    """centre(t) = c + amp * sin(2 pi t / period + phase) * axis."""
    c: Tuple[float, float, float]
    phase: float
    axis: Tuple[float, float, float]
    amp: float = 0.1
    period: float = 2.0

    def centre(self, t: float):
        s = self.amp * math.sin(2 * math.pi * t / self.period + self.phase)
        return tuple(ci + s * ai for ci, ai in zip(self.c, self.axis))

    def velocity(self, t: float):
        w = 2 * math.pi / self.period
        s = self.amp * w * math.cos(w * t + self.phase)
        return tuple(s * ai for ai in self.axis)


def moving_boxes(res=(512, 256, 512), seed: int = 0, n_boxes: int = 3):
    """The moving-solid dam break: walls, the usual fluid block, and `n_boxes`
    boxes of side 0.2 on the floor moving on seeded sinusoidal paths
    (amplitude 0.1, period 2 s, axis x or z, phase U[0, 2 pi)).  Returns the
    scene (boxes at their t = 0 positions) and the paths."""
    rng = np.random.default_rng(seed)
    h = 1.0 / res[1]
    paths, solids = [], []
    for _ in range(n_boxes):
        c = (float(rng.uniform(0.6, 0.8)), 0.1 + h, float(rng.uniform(0.25, 0.75)))
        axis = (1.0, 0.0, 0.0) if rng.random() < 0.5 else (0.0, 0.0, 1.0)
        path = SinePath(c, float(rng.uniform(0.0, 2 * math.pi)), axis)
        paths.append(path)
        solids.append(Solid("box", path.centre(0.0), (0.2, 0.2, 0.2), path.velocity(0.0)))
    sc = Scene(res=tuple(res), solids=solids, seed=seed, name=f"moving boxes {res[0]}x{res[1]}x{res[2]}")
    return sc, paths


def gpu_solver(scene: Scene, precond: int = 1, tol_mode: int = 1, tol: float = 1e-6, max_iter: int = 200,
               advect_scalars: bool = False, clamp_mode: int = 1, kind: int = 3, **extra):
    """Build the scene in an hfgrid.Solver: walls + solids, bbox fluid domain,
    PIC/FLIP mix (MixingCoefficient scene.mixing, CFL scene.cfl, linear
    transfers, RK3) and seeded particles."""
    import hfgrid
    s = hfgrid.Solver(scene.dt, scene.res, scene.origin, scene.spacing)
    for sdf, vel in boundaries(scene):
        s.add_solid_boundary(sdf, vel)
    mn, mx = fluid_bbox(scene)
    s.generate_fluid_domain_from_bbox(mn, mx)
    s.set_advection(kind, hfgrid.RK3, hfgrid.LINEAR, scene.cfl, scene.mixing)
    s.set_options(precond=precond, tol_mode=tol_mode, tol=tol, max_iter=max_iter, advect_scalars=int(advect_scalars),
                  clamp_mode=clamp_mode, **extra)
    if kind != hfgrid.ADV_SEMI_LAGRANGIAN:
        s.seed_particles(scene.per_cell, scene.seed)
    return s
