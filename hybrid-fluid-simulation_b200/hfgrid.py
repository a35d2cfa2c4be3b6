"""ctypes binding of libhfgrid.so (include/hfgrid.h) for Python callers.

The library is the product: C++ host code and sm_100a CUDA kernels behind a
C ABI.  This module only marshals arguments.  `Solver` mirrors the reference's
CGridFluidSolver (MPhysics/GridFluidSolver.h:17-137) with numpy arrays in and
out; the `op_*` functions mirror the reference's per-stage Invoker functions
and take CUDA device pointers (torch tensors are accepted) plus a stream.

There is no fallback: if libhfgrid.so cannot be loaded or a call fails, an
exception is raised.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhfgrid.so")

# enums (include/hfgrid.h)
ADV_SEMI_LAGRANGIAN, ADV_PIC, ADV_FLIP, ADV_MIX_PIC_FLIP = 0, 1, 2, 3
RK1, RK2, RK3 = 0, 1, 2
P2GSUM, G2PNEAREST, LINEAR, QUADRATIC, CUBIC = 0, 1, 2, 3, 4
PRECOND_IDENTITY, PRECOND_JACOBI, PRECOND_MG = 0, 1, 2
TOL_REFERENCE, TOL_RELATIVE = 0, 1
HFG_OK, HFG_ERR_NOT_CONVERGED = 0, -5
SOLID_WALLS, SOLID_SPHERE, SOLID_BOX = 0, 1, 2
SAMPLE_TRILINEAR, SAMPLE_CATMULLROM, SAMPLE_MONOCATMULLROM, SAMPLE_CUBICBRIDSON, SAMPLE_CLAMPCUBICBRIDSON = 0, 1, 2, 3, 4


class HfgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"hfgrid error {code}: {msg}")
        self.code = code


class Options(C.Structure):
    _fields_ = [
        ("precond", C.c_int), ("tol_mode", C.c_int), ("tol", C.c_double), ("max_iter", C.c_longlong),
        ("clamp_mode", C.c_int), ("advect_scalars", C.c_int), ("extrapolation_layers", C.c_int),
        ("mg_levels", C.c_int), ("mg_smooth", C.c_int), ("mg_half", C.c_int), ("report_divergence", C.c_int),
        ("sampling", C.c_int), ("pressure_fp64", C.c_int), ("autotune", C.c_int), ("sort_interval", C.c_int),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("cg_iterations", C.c_longlong), ("cg_residual", C.c_double), ("cg_rhs_norm", C.c_double),
        ("cg_converged", C.c_int), ("substeps", C.c_int), ("extrapolation_layers", C.c_int),
        ("sim_time", C.c_double), ("num_particles", C.c_longlong), ("fluid_cells", C.c_longlong),
        ("stage_ms", C.c_float * 8), ("divergence_l2", C.c_double), ("divergence_max", C.c_double),
        ("cg_true_residual", C.c_double), ("particle_ms", C.c_float * 3),
    ]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("stage_ms", "particle_ms")}
        d["stage_ms"] = list(self.stage_ms)
        d["particle_ms"] = list(self.particle_ms)
        return d


class SceneDesc(C.Structure):
    """hfg_scene_desc_t: a seeded dam break on the unit cube."""
    _fields_ = [
        ("res", C.c_int * 3), ("dt", C.c_float), ("fluid_max", C.c_float * 3), ("n_spheres", C.c_int),
        ("spheres", (C.c_float * 4) * 4), ("per_cell", C.c_int), ("seed", C.c_ulonglong), ("cfl", C.c_float),
        ("mixing", C.c_float), ("steps", C.c_int), ("keep_particles", C.c_int), ("options", Options),
    ]


class RequestInfo(C.Structure):
    _fields_ = [
        ("status", C.c_int), ("steps_done", C.c_int), ("cells", C.c_longlong), ("particles", C.c_longlong),
        ("footprint_bytes", C.c_longlong), ("queue_ms", C.c_double), ("run_ms", C.c_double),
        ("step_ms_p50", C.c_double), ("step_ms_max", C.c_double), ("last", Stats),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_longlong), ("completed", C.c_longlong), ("failed", C.c_longlong),
        ("rejected", C.c_longlong), ("step_ms_p50", C.c_double), ("step_ms_p99", C.c_double),
        ("request_ms_p50", C.c_double), ("request_ms_p99", C.c_double), ("cell_steps", C.c_double),
        ("wall_s", C.c_double), ("peak_bytes", C.c_longlong), ("budget_bytes", C.c_longlong),
        ("peak_running", C.c_int), ("slots", C.c_int),
    ]


def _struct_dict(st) -> dict:
    out = {}
    for k, _ in st._fields_:
        v = getattr(st, k)
        out[k] = v.as_dict() if isinstance(v, Stats) else v
    return out


_lib = None

I3 = C.c_int * 3
F3 = C.c_float * 3
PF = C.POINTER(C.c_float)
PU8 = C.POINTER(C.c_uint8)
VP = C.c_void_p


def _signatures(lib):
    S = C.c_void_p  # hfg_solver_t
    sig = {
        "hfg_init": (C.c_int, [C.c_int]),
        "hfg_last_error": (C.c_char_p, []),
        "hfg_version": (C.c_char_p, []),
        "hfg_default_options": (None, [C.POINTER(Options)]),
        "hfg_solver_create": (C.c_int, [C.c_float, I3, F3, F3, C.POINTER(S)]),
        "hfg_solver_destroy": (C.c_int, [S]),
        "hfg_solver_add_solid_boundary": (C.c_int, [S, PF, F3]),
        "hfg_solver_add_external_force": (C.c_int, [S, F3]),
        "hfg_solver_set_boundary_velocity": (C.c_int, [S, C.c_int, F3]),
        "hfg_solver_set_velocity_field": (C.c_int, [S, PF, PF, PF]),
        "hfg_solver_set_fluid_domain_field": (C.c_int, [S, PF]),
        "hfg_solver_set_color_field": (C.c_int, [S, PF, PF, PF]),
        "hfg_solver_generate_fluid_domain_from_bbox": (C.c_int, [S, F3, F3]),
        "hfg_solver_set_advection": (C.c_int, [S, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float]),
        "hfg_solver_seed_particles": (C.c_int, [S, C.c_int, C.c_ulonglong]),
        "hfg_solver_set_particles": (C.c_int, [S, PF, PF, C.c_longlong]),
        "hfg_solver_set_options": (C.c_int, [S, C.POINTER(Options)]),
        "hfg_solver_enable_timing": (C.c_int, [S, C.c_int]),
        "hfg_solver_update": (C.c_int, [S]),
        "hfg_solver_update_steps": (C.c_int, [S, C.c_int]),
        "hfg_solver_update_without_pressure": (C.c_int, [S]),
        "hfg_solver_solve_pressure": (C.c_int, [S]),
        "hfg_solver_get_velocity_field": (C.c_int, [S, C.c_int, PF, PF, PF]),
        "hfg_solver_get_fluid_domain_field": (C.c_int, [S, PF]),
        "hfg_solver_get_color_field": (C.c_int, [S, PF, PF, PF]),
        "hfg_solver_get_markers": (C.c_int, [S, PU8]),
        "hfg_solver_get_pressure": (C.c_int, [S, PF]),
        "hfg_solver_get_solid_sdf": (C.c_int, [S, PF]),
        "hfg_solver_get_solid_vel_field": (C.c_int, [S, PF, PF, PF]),
        "hfg_solver_get_fluid_sdf": (C.c_int, [S, PF]),
        "hfg_solver_get_fluid_density": (C.c_int, [S, PF]),
        "hfg_solver_mix_vel_field_with_others": (C.c_int, [S, VP, VP, VP, VP, VP]),
        "hfg_solver_transfer_vel_to_particles": (C.c_int, [S, VP, C.c_longlong, C.c_int, VP]),
        "hfg_solver_num_particles": (C.c_longlong, [S]),
        "hfg_solver_get_particles": (C.c_int, [S, PF, PF]),
        "hfg_solver_sort_particles": (C.c_int, [S]),
        "hfg_solver_set_particle_mirror": (C.c_int, [S, PF, PF, C.c_longlong]),
        "hfg_solver_get_stats": (C.c_int, [S, C.POINTER(Stats)]),
        "hfg_solver_get_grid": (C.c_int, [S, I3, F3, F3]),
        "hfg_solver_stream": (C.c_void_p, [S]),
        "hfg_solver_launch_count": (C.c_longlong, [S]),
        "hfg_solver_synchronize": (C.c_int, [S]),
        "hfg_solver_time_cg": (C.c_int, [S, C.c_int, C.POINTER(C.c_float)]),
        "hfg_op_markers_from_particles": (C.c_int, [I3, F3, F3, VP, VP, C.c_longlong, VP, VP]),
        "hfg_op_bin_counts": (C.c_int, [I3, F3, F3, VP, C.c_longlong, VP, VP]),
        "hfg_op_markers_from_sdf": (C.c_int, [I3, VP, VP, VP, VP]),
        "hfg_op_build_matrix_a": (C.c_int, [I3, F3, C.c_float, VP, VP, VP]),
        "hfg_op_apply_a": (C.c_int, [I3, F3, C.c_float, VP, VP, VP, VP]),
        "hfg_op_build_rhs": (C.c_int, [I3, F3, VP, VP, VP, VP, VP, VP, VP, VP, VP]),
        "hfg_op_project": (C.c_int, [I3, F3, C.c_float, VP, VP, VP, VP, VP, VP, VP, C.c_int, C.c_int, C.c_double,
                                     C.c_longlong, VP, C.POINTER(C.c_double), VP]),
        "hfg_op_extrapolate_fc": (C.c_int, [I3, VP, VP, VP, C.c_int, VP]),
        "hfg_op_extrapolate_cc": (C.c_int, [I3, VP, C.c_int, VP]),
        "hfg_op_sample_fc": (C.c_int, [I3, F3, F3, VP, VP, VP, VP, C.c_longlong, VP, VP]),
        "hfg_op_sample_cc": (C.c_int, [I3, F3, F3, VP, VP, C.c_longlong, VP, VP]),
        "hfg_op_sample_cc_ex": (C.c_int, [I3, F3, F3, VP, VP, C.c_longlong, C.c_int, VP, VP]),
        "hfg_op_sample_fc_ex": (C.c_int, [I3, F3, F3, VP, VP, VP, VP, C.c_longlong, C.c_int, VP, VP]),
        "hfg_op_sl_advect_fc_ex": (C.c_int, [I3, F3, F3, VP, VP, VP, VP, VP, VP, C.c_float, C.c_int, C.c_int, VP, VP,
                                             VP, VP]),
        "hfg_op_sl_advect_cc_ex": (C.c_int, [I3, F3, F3, VP, VP, VP, VP, C.c_float, C.c_int, C.c_int, VP, VP]),
        "hfg_op_g2p_fc": (C.c_int, [I3, F3, F3, VP, VP, VP, VP, C.c_longlong, C.c_int, VP, VP]),
        "hfg_op_g2p_cc": (C.c_int, [I3, F3, F3, VP, VP, C.c_longlong, C.c_int, VP, VP]),
        "hfg_op_p2g_fc": (C.c_int, [I3, F3, F3, VP, VP, C.c_longlong, C.c_int, VP, VP, VP, VP, VP, VP, VP]),
        "hfg_op_p2g_fc_static": (C.c_int, [I3, F3, F3, VP, VP, C.c_longlong, C.c_int, VP, VP, VP, VP, VP, VP, VP]),
        "hfg_op_p2g_cc": (C.c_int, [I3, F3, F3, VP, VP, C.c_longlong, C.c_int, C.c_int, VP, VP, VP]),
        "hfg_op_advect_particles": (C.c_int, [I3, F3, F3, VP, VP, VP, VP, C.c_longlong, C.c_float, C.c_float,
                                              C.c_int, C.c_int, C.POINTER(C.c_int), VP]),
        "hfg_op_sl_advect_fc": (C.c_int, [I3, F3, F3, VP, VP, VP, VP, VP, VP, C.c_float, C.c_int, VP, VP, VP, VP]),
        "hfg_op_sl_advect_cc": (C.c_int, [I3, F3, F3, VP, VP, VP, VP, C.c_float, C.c_int, VP, VP]),
        "hfg_op_fluid_domain_from_bbox": (C.c_int, [I3, F3, F3, F3, F3, VP, VP]),
        "hfg_op_build_fluid_sdf": (C.c_int, [I3, VP, VP, C.c_int, VP]),
        "hfg_op_build_fluid_outside_sdf": (C.c_int, [I3, VP, VP, VP, C.c_int, VP]),
        "hfg_op_build_fluid_inside_sdf": (C.c_int, [I3, VP, VP, VP, C.c_int, VP]),
        "hfg_op_build_mixed_fluid_outside_sdf": (C.c_int, [I3, VP, VP, VP, VP, VP]),
        "hfg_op_build_fluid_density": (C.c_int, [I3, VP, VP, VP, VP]),
        "hfg_op_mix_field_with_density_cc": (C.c_int, [C.c_longlong, VP, VP, VP, VP, VP]),
        "hfg_op_mix_field_with_density_fc": (C.c_int, [I3, VP, VP, VP, VP, VP, VP, VP, VP, VP]),
        "hfg_op_mix_particle_vel_pic_flip": (C.c_int, [VP, VP, VP, C.c_longlong, C.c_float, C.c_float, C.c_float,
                                                       C.c_float, C.c_float, VP, VP]),
        "hfg_solver_add_analytic_solid": (C.c_int, [S, C.c_int, C.POINTER(C.c_double), F3]),
        "hfg_scene_bytes": (C.c_int, [I3, C.c_longlong, C.c_int, C.c_int, C.POINTER(C.c_longlong)]),
        "hfg_scene_particles_bound": (C.c_int, [C.POINTER(SceneDesc), C.POINTER(C.c_longlong)]),
        "hfg_server_create": (C.c_int, [C.c_int, C.c_int, C.c_longlong, C.POINTER(C.c_void_p)]),
        "hfg_server_submit": (C.c_int, [VP, C.POINTER(SceneDesc), C.POINTER(C.c_longlong)]),
        "hfg_server_info": (C.c_int, [VP, C.c_longlong, C.POINTER(RequestInfo)]),
        "hfg_server_wait": (C.c_int, [VP, C.c_longlong, C.POINTER(RequestInfo)]),
        "hfg_server_step_times": (C.c_int, [VP, C.c_longlong, C.POINTER(C.c_double), C.c_int]),
        "hfg_server_particles": (C.c_int, [VP, C.c_longlong, PF, C.c_longlong]),
        "hfg_server_drain": (C.c_int, [VP]),
        "hfg_server_stats": (C.c_int, [VP, C.POINTER(ServerStats)]),
        "hfg_server_destroy": (C.c_int, [VP]),
        "hfg_op_seed_particles": (C.c_int, [I3, F3, F3, VP, VP, C.c_int, C.c_ulonglong, VP, C.c_longlong,
                                            C.POINTER(C.c_longlong), VP]),
        "hfg_selftest_bounded_waits": (C.c_int, [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "hfg_test_inject_alloc_failure": (C.c_int, [C.c_int]),
        "hfg_tune_save": (C.c_int, [C.c_char_p]),
        "hfg_batch_create": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
        "hfg_batch_step": (C.c_int, [VP, C.c_int, C.c_void_p]),
        "hfg_batch_scene_stats": (C.c_int, [VP, C.c_int, C.POINTER(Stats)]),
        "hfg_batch_particles": (C.c_int, [VP, C.c_int, PF, C.c_longlong]),
        "hfg_batch_destroy": (C.c_int, [VP]),
        "hfg_tune_load": (C.c_int, [C.c_char_p, C.POINTER(C.c_int)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


def lib():
    """Load libhfgrid.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} not built; run `python {os.path.join(HERE, 'build.py')}`")
        _lib = _signatures(C.CDLL(LIB_PATH))
    return _lib


def _check(code: int):
    if code != HFG_OK:
        raise HfgError(code, lib().hfg_last_error().decode())


def init(device: int = 0):
    _check(lib().hfg_init(device))


def selftest_bounded_waits(wait_ms: int = 20):
    """(mbarrier wait timed out, grid barrier timed out) of the wait self-test."""
    a, b = C.c_int(), C.c_int()
    _check(lib().hfg_selftest_bounded_waits(wait_ms, C.byref(a), C.byref(b)))
    return a.value, b.value


def tune_save(path: str):
    """Write the autotuner's launch shapes to `path`."""
    _check(lib().hfg_tune_save(path.encode()))


def tune_load(path: str) -> int:
    """Add the launch shapes in `path` to the table; returns the entries read."""
    n = C.c_int()
    _check(lib().hfg_tune_load(path.encode(), C.byref(n)))
    return n.value


def inject_alloc_failure(after: int):
    """Make the after-th device allocation from now on fail (0 disarms)."""
    _check(lib().hfg_test_inject_alloc_failure(after))


def default_options() -> Options:
    o = Options()
    lib().hfg_default_options(C.byref(o))
    return o


def _f3(v) -> F3:
    return F3(*[float(x) for x in v])


def _i3(v) -> I3:
    return I3(*[int(x) for x in v])


def _fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(PF)


def face_shapes(res):
    nx, ny, nz = res
    return ((nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx))


class Solver:
    """CGridFluidSolver on the GPU (GridFluidSolver.cpp:32-41)."""

    def __init__(self, dt: float, res, origin=(0.0, 0.0, 0.0), spacing=(1.0, 1.0, 1.0)):
        self.res = tuple(int(r) for r in res)
        self.origin = tuple(float(o) for o in origin)
        self.spacing = tuple(float(h) for h in spacing)
        self.dt = float(dt)
        h = C.c_void_p()
        _check(lib().hfg_solver_create(C.c_float(dt), _i3(self.res), _f3(origin), _f3(spacing), C.byref(h)))
        self._h = h
        self._owned = True

    @classmethod
    def attach(cls, handle: int, dt: float, res, origin, spacing) -> "Solver":
        """Wrap a solver owned elsewhere (e.g. one a loaded MPhysics scene
        holds, from mphysics_grid_solver); closing the wrapper leaves it alive."""
        self = cls.__new__(cls)
        self.res = tuple(int(r) for r in res)
        self.origin = tuple(float(o) for o in origin)
        self.spacing = tuple(float(h) for h in spacing)
        self.dt = float(dt)
        self._h = C.c_void_p(handle)
        self._owned = False
        return self

    def close(self):
        if getattr(self, "_h", None):
            if self._owned:
                lib().hfg_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n_cells(self) -> int:
        return self.res[0] * self.res[1] * self.res[2]

    # ---- setters ----
    def add_solid_boundary(self, sdf: np.ndarray, vel=(0.0, 0.0, 0.0)):
        a = np.ascontiguousarray(sdf, dtype=np.float32).reshape(-1)
        assert a.size == self.n_cells
        _check(lib().hfg_solver_add_solid_boundary(self._h, _fptr(a), _f3(vel)))

    def add_analytic_solid(self, kind: int, params=(0.0,) * 6, vel=(0.0, 0.0, 0.0)):
        """SOLID_WALLS / SOLID_SPHERE (cx, cy, cz, r) / SOLID_BOX (cx, cy, cz,
        sx, sy, sz): the SDF is evaluated on the device."""
        p = (C.c_double * 6)(*(list(params) + [0.0] * (6 - len(params))))
        _check(lib().hfg_solver_add_analytic_solid(self._h, kind, p, _f3(vel)))

    def set_boundary_velocity(self, index: int, vel):
        _check(lib().hfg_solver_set_boundary_velocity(self._h, index, _f3(vel)))

    def add_external_force(self, f):
        _check(lib().hfg_solver_add_external_force(self._h, _f3(f)))

    def set_velocity_field(self, x, y, z):
        xs = [np.ascontiguousarray(v, dtype=np.float32).reshape(-1) for v in (x, y, z)]
        _check(lib().hfg_solver_set_velocity_field(self._h, *[_fptr(v) for v in xs]))

    def set_fluid_domain_field(self, d):
        a = np.ascontiguousarray(d, dtype=np.float32).reshape(-1)
        _check(lib().hfg_solver_set_fluid_domain_field(self._h, _fptr(a)))

    def set_color_field(self, x, y, z):
        xs = [np.ascontiguousarray(v, dtype=np.float32).reshape(-1) for v in (x, y, z)]
        _check(lib().hfg_solver_set_color_field(self._h, *[_fptr(v) for v in xs]))

    def generate_fluid_domain_from_bbox(self, mn, mx):
        _check(lib().hfg_solver_generate_fluid_domain_from_bbox(self._h, _f3(mn), _f3(mx)))

    def set_advection(self, kind: int, accuracy: int = RK3, alg: int = LINEAR, cfl: float = 1.0, mixing: float = 0.1):
        _check(lib().hfg_solver_set_advection(self._h, kind, accuracy, alg, C.c_float(cfl), C.c_float(mixing)))

    def seed_particles(self, per_cell: int, seed: int):
        _check(lib().hfg_solver_seed_particles(self._h, per_cell, seed))

    def set_particles(self, pos: np.ndarray, vel: Optional[np.ndarray] = None):
        p = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1)
        v = None if vel is None else np.ascontiguousarray(vel, dtype=np.float32).reshape(-1)
        _check(lib().hfg_solver_set_particles(self._h, _fptr(p), None if v is None else _fptr(v), p.size // 3))

    def set_options(self, **kw):
        o = default_options()
        for k, v in kw.items():
            setattr(o, k, v)
        _check(lib().hfg_solver_set_options(self._h, C.byref(o)))

    def enable_timing(self, on=True):
        _check(lib().hfg_solver_enable_timing(self._h, int(on)))

    # ---- step ----
    def update(self, steps: int = 1):
        if steps == 1:
            _check(lib().hfg_solver_update(self._h))
        else:
            _check(lib().hfg_solver_update_steps(self._h, steps))

    def update_without_pressure(self):
        _check(lib().hfg_solver_update_without_pressure(self._h))

    def solve_pressure(self):
        _check(lib().hfg_solver_solve_pressure(self._h))

    def synchronize(self):
        _check(lib().hfg_solver_synchronize(self._h))

    def time_cg(self, iters: int = 50) -> float:
        """Mean ms per CG iteration (both kernels) on the last system."""
        ms = C.c_float(0)
        _check(lib().hfg_solver_time_cg(self._h, iters, C.byref(ms)))
        return ms.value

    # ---- getters ----
    def velocity_field(self, which: int = 0):
        out = [np.empty(s, np.float32) for s in face_shapes(self.res)]
        _check(lib().hfg_solver_get_velocity_field(self._h, which, *[_fptr(o) for o in out]))
        return out

    def fluid_domain_field(self):
        out = np.empty(self.res[::-1], np.float32)
        _check(lib().hfg_solver_get_fluid_domain_field(self._h, _fptr(out)))
        return out

    def color_field(self):
        out = [np.empty(self.res[::-1], np.float32) for _ in range(3)]
        _check(lib().hfg_solver_get_color_field(self._h, *[_fptr(o) for o in out]))
        return out

    def markers(self):
        out = np.empty(self.res[::-1], np.uint8)
        _check(lib().hfg_solver_get_markers(self._h, out.ctypes.data_as(PU8)))
        return out

    def pressure(self):
        out = np.empty(self.res[::-1], np.float32)
        _check(lib().hfg_solver_get_pressure(self._h, _fptr(out)))
        return out

    def solid_sdf(self):
        out = np.empty(self.res[::-1], np.float32)
        _check(lib().hfg_solver_get_solid_sdf(self._h, _fptr(out)))
        return out

    def solid_vel_field(self):
        out = [np.empty(s, np.float32) for s in face_shapes(self.res)]
        _check(lib().hfg_solver_get_solid_vel_field(self._h, *[_fptr(o) for o in out]))
        return out

    def fluid_sdf(self):
        out = np.empty(self.res[::-1], np.float32)
        _check(lib().hfg_solver_get_fluid_sdf(self._h, _fptr(out)))
        return out

    def mix_vel_field_with_others(self, other, w_other, w_fluid):
        """torch CUDA tensors: the other face field (3), both cell densities."""
        _check(lib().hfg_solver_mix_vel_field_with_others(self._h, *[_ptr(v) for v in other], _ptr(w_other),
                                                          _ptr(w_fluid)))

    def transfer_vel_to_particles(self, pos, alg, out):
        _check(lib().hfg_solver_transfer_vel_to_particles(self._h, _ptr(pos), pos.numel() // 3, alg, _ptr(out)))

    def fluid_density(self):
        out = np.empty(self.res[::-1], np.float32)
        _check(lib().hfg_solver_get_fluid_density(self._h, _fptr(out)))
        return out

    @property
    def num_particles(self) -> int:
        return int(lib().hfg_solver_num_particles(self._h))

    def particles(self):
        n = self.num_particles
        pos = np.empty((n, 3), np.float32)
        vel = np.empty((n, 3), np.float32)
        _check(lib().hfg_solver_get_particles(self._h, _fptr(pos), _fptr(vel)))
        return pos, vel

    def sort_particles(self):
        """Reorder the particles by cell now (stable; no reference counterpart)."""
        _check(lib().hfg_solver_sort_particles(self._h))

    def copy_particles_into(self, pos: np.ndarray, vel: Optional[np.ndarray] = None):
        _check(lib().hfg_solver_get_particles(self._h, _fptr(pos), None if vel is None else _fptr(vel)))

    def set_particle_mirror(self, pos: Optional[np.ndarray], vel: Optional[np.ndarray] = None):
        """hfg_solver_set_particle_mirror: every update() also fills pos / vel
        ((capacity, 3) float32 host arrays, pinned for overlap) with the
        particles; None, None removes the mirror."""
        arrays = [a for a in (pos, vel) if a is not None]
        cap = min(a.shape[0] for a in arrays) if arrays else 0
        for a in arrays:
            assert a.ndim == 2 and a.shape[1] == 3
        _check(lib().hfg_solver_set_particle_mirror(self._h, None if pos is None else _fptr(pos),
                                                    None if vel is None else _fptr(vel), cap))
        self._mirror = (pos, vel)  # the library writes into them: keep them alive

    def stats(self) -> dict:
        s = Stats()
        _check(lib().hfg_solver_get_stats(self._h, C.byref(s)))
        return s.as_dict()

    @property
    def stream(self) -> int:
        return int(lib().hfg_solver_stream(self._h) or 0)

    @property
    def launch_count(self) -> int:
        return int(lib().hfg_solver_launch_count(self._h))


# ---------------------------------------------------------------- operators --
def _ptr(t) -> Optional[int]:
    """Device pointer of a torch tensor (or an int address / None)."""
    if t is None:
        return None
    if isinstance(t, int):
        return t
    return int(t.data_ptr())


def _stream(stream) -> Optional[int]:
    if stream is None:
        import torch
        return int(torch.cuda.current_stream().cuda_stream)
    return int(stream)


def op_markers_from_particles(res, origin, spacing, solid_sdf, pos, markers, stream=None):
    n = pos.numel() // 3
    _check(lib().hfg_op_markers_from_particles(_i3(res), _f3(origin), _f3(spacing), _ptr(solid_sdf), _ptr(pos), n,
                                               _ptr(markers), _stream(stream)))


def op_bin_counts(res, origin, spacing, pos, counts, stream=None):
    _check(lib().hfg_op_bin_counts(_i3(res), _f3(origin), _f3(spacing), _ptr(pos), pos.numel() // 3, _ptr(counts),
                                   _stream(stream)))


def op_markers_from_sdf(res, solid_sdf, fluid_sdf, markers, stream=None):
    _check(lib().hfg_op_markers_from_sdf(_i3(res), _ptr(solid_sdf), _ptr(fluid_sdf), _ptr(markers), _stream(stream)))


def op_build_matrix_a(res, spacing, dt, markers, A, stream=None):
    _check(lib().hfg_op_build_matrix_a(_i3(res), _f3(spacing), C.c_float(dt), _ptr(markers), _ptr(A), _stream(stream)))


def op_apply_a(res, spacing, dt, markers, x, y, stream=None):
    _check(lib().hfg_op_apply_a(_i3(res), _f3(spacing), C.c_float(dt), _ptr(markers), _ptr(x), _ptr(y),
                                _stream(stream)))


def op_build_rhs(res, spacing, vel, solid_vel, markers, b, stream=None):
    _check(lib().hfg_op_build_rhs(_i3(res), _f3(spacing), *[_ptr(v) for v in vel], *[_ptr(v) for v in solid_vel],
                                  _ptr(markers), _ptr(b), _stream(stream)))


def op_project(res, spacing, dt, markers, vel, solid_vel, precond=PRECOND_IDENTITY, tol_mode=TOL_REFERENCE,
               tol=1e-3, max_iter=-1, p_out=None, stream=None):
    stats = (C.c_double * 3)()
    code = lib().hfg_op_project(_i3(res), _f3(spacing), C.c_float(dt), _ptr(markers), *[_ptr(v) for v in vel],
                                *[_ptr(v) for v in solid_vel], precond, tol_mode, C.c_double(tol), max_iter,
                                _ptr(p_out), stats, _stream(stream))
    if code not in (HFG_OK, HFG_ERR_NOT_CONVERGED):
        _check(code)
    return {"iterations": int(stats[0]), "residual": stats[1], "rhs_norm": stats[2], "converged": code == HFG_OK}


def op_extrapolate_fc(res, vel, layers=1000, stream=None):
    _check(lib().hfg_op_extrapolate_fc(_i3(res), *[_ptr(v) for v in vel], layers, _stream(stream)))


def op_extrapolate_cc(res, f, layers=1000, stream=None):
    _check(lib().hfg_op_extrapolate_cc(_i3(res), _ptr(f), layers, _stream(stream)))


def op_sample_fc(res, origin, spacing, vel, pos, out, stream=None):
    _check(lib().hfg_op_sample_fc(_i3(res), _f3(origin), _f3(spacing), *[_ptr(v) for v in vel], _ptr(pos),
                                  pos.numel() // 3, _ptr(out), _stream(stream)))


def op_sample_cc(res, origin, spacing, f, pos, out, stream=None):
    _check(lib().hfg_op_sample_cc(_i3(res), _f3(origin), _f3(spacing), _ptr(f), _ptr(pos), pos.numel() // 3,
                                  _ptr(out), _stream(stream)))


def op_sample_cc_ex(res, origin, spacing, f, pos, sampling, out, stream=None):
    _check(lib().hfg_op_sample_cc_ex(_i3(res), _f3(origin), _f3(spacing), _ptr(f), _ptr(pos), pos.numel() // 3,
                                     sampling, _ptr(out), _stream(stream)))


def op_sample_fc_ex(res, origin, spacing, vel, pos, sampling, out, stream=None):
    _check(lib().hfg_op_sample_fc_ex(_i3(res), _f3(origin), _f3(spacing), *[_ptr(v) for v in vel], _ptr(pos),
                                     pos.numel() // 3, sampling, _ptr(out), _stream(stream)))


def op_g2p_fc(res, origin, spacing, vel, pos, alg, out, stream=None):
    _check(lib().hfg_op_g2p_fc(_i3(res), _f3(origin), _f3(spacing), *[_ptr(v) for v in vel], _ptr(pos),
                               pos.numel() // 3, alg, _ptr(out), _stream(stream)))


def op_g2p_cc(res, origin, spacing, f, pos, alg, out, stream=None):
    _check(lib().hfg_op_g2p_cc(_i3(res), _f3(origin), _f3(spacing), _ptr(f), _ptr(pos), pos.numel() // 3, alg,
                               _ptr(out), _stream(stream)))


def op_p2g_fc(res, origin, spacing, pos, vel, alg, out, weights=(None, None, None), stream=None):
    _check(lib().hfg_op_p2g_fc(_i3(res), _f3(origin), _f3(spacing), _ptr(pos), _ptr(vel), pos.numel() // 3, alg,
                               *[_ptr(v) for v in out], *[_ptr(w) for w in weights], _stream(stream)))


def op_p2g_fc_static(res, origin, spacing, pos, vel, alg, out, weights=(None, None, None), stream=None):
    """op_p2g_fc with the accumulators in the library's fixed 8 MiB array
    instead of freshly allocated device memory: at most 2**20 faces in total;
    calls overlapping in time on one device race (hfgrid.h)."""
    _check(lib().hfg_op_p2g_fc_static(_i3(res), _f3(origin), _f3(spacing), _ptr(pos), _ptr(vel), pos.numel() // 3,
                                      alg, *[_ptr(v) for v in out], *[_ptr(w) for w in weights], _stream(stream)))


def op_p2g_cc(res, origin, spacing, pos, val, alg, out, weights=None, normalize=True, stream=None):
    _check(lib().hfg_op_p2g_cc(_i3(res), _f3(origin), _f3(spacing), _ptr(pos), _ptr(val), pos.numel() // 3, alg,
                               int(normalize), _ptr(out), _ptr(weights), _stream(stream)))


def op_advect_particles(res, origin, spacing, vel, pos, dt, cfl=1.0, accuracy=RK3, clamp_mode=1, stream=None):
    n = C.c_int(0)
    _check(lib().hfg_op_advect_particles(_i3(res), _f3(origin), _f3(spacing), *[_ptr(v) for v in vel], _ptr(pos),
                                         pos.numel() // 3, C.c_float(dt), C.c_float(cfl), accuracy, clamp_mode,
                                         C.byref(n), _stream(stream)))
    return n.value


def op_sl_advect_fc(res, origin, spacing, field, vel, dt, accuracy, out, stream=None, sampling=SAMPLE_TRILINEAR):
    if sampling != SAMPLE_TRILINEAR:
        _check(lib().hfg_op_sl_advect_fc_ex(_i3(res), _f3(origin), _f3(spacing), *[_ptr(v) for v in field],
                                            *[_ptr(v) for v in vel], C.c_float(dt), accuracy, sampling,
                                            *[_ptr(v) for v in out], _stream(stream)))
        return
    _check(lib().hfg_op_sl_advect_fc(_i3(res), _f3(origin), _f3(spacing), *[_ptr(v) for v in field],
                                     *[_ptr(v) for v in vel], C.c_float(dt), accuracy, *[_ptr(v) for v in out],
                                     _stream(stream)))


def op_sl_advect_cc(res, origin, spacing, field, vel, dt, accuracy, out, stream=None, sampling=SAMPLE_TRILINEAR):
    if sampling != SAMPLE_TRILINEAR:
        _check(lib().hfg_op_sl_advect_cc_ex(_i3(res), _f3(origin), _f3(spacing), _ptr(field),
                                            *[_ptr(v) for v in vel], C.c_float(dt), accuracy, sampling, _ptr(out),
                                            _stream(stream)))
        return
    _check(lib().hfg_op_sl_advect_cc(_i3(res), _f3(origin), _f3(spacing), _ptr(field), *[_ptr(v) for v in vel],
                                     C.c_float(dt), accuracy, _ptr(out), _stream(stream)))


def op_fluid_domain_from_bbox(res, origin, spacing, mn, mx, out, stream=None):
    _check(lib().hfg_op_fluid_domain_from_bbox(_i3(res), _f3(origin), _f3(spacing), _f3(mn), _f3(mx), _ptr(out),
                                               _stream(stream)))


def op_mix_field_with_density_cc(a, b, wa, wb, stream=None):
    _check(lib().hfg_op_mix_field_with_density_cc(b.numel(), _ptr(a), _ptr(b), _ptr(wa), _ptr(wb), _stream(stream)))


def op_mix_field_with_density_fc(res, a, b, wa, wb, stream=None):
    _check(lib().hfg_op_mix_field_with_density_fc(_i3(res), *[_ptr(v) for v in a], *[_ptr(v) for v in b], _ptr(wa),
                                                  _ptr(wb), _stream(stream)))


def op_mix_particle_vel_pic_flip(pic, flip, dist, cell, g_rate, gf_rate, f_rate, p_rate, predict, stream=None):
    _check(lib().hfg_op_mix_particle_vel_pic_flip(_ptr(pic), _ptr(flip), _ptr(dist), dist.numel(), C.c_float(cell),
                                                  C.c_float(g_rate), C.c_float(gf_rate), C.c_float(f_rate),
                                                  C.c_float(p_rate), _ptr(predict), _stream(stream)))


def op_build_fluid_density(res, domain, solid_sdf, out, stream=None):
    _check(lib().hfg_op_build_fluid_density(_i3(res), _ptr(domain), _ptr(solid_sdf), _ptr(out), _stream(stream)))


def op_build_fluid_sdf(res, domain, sdf, layers=1000, stream=None):
    _check(lib().hfg_op_build_fluid_sdf(_i3(res), _ptr(domain), _ptr(sdf), layers, _stream(stream)))


def op_build_fluid_outside_sdf(res, density, solid_sdf, out, distance=1000, stream=None):
    """buildFluidOutsideSDFInvoker (HybridSimulatorBuildSDF.cu:177-207)."""
    _check(lib().hfg_op_build_fluid_outside_sdf(_i3(res), _ptr(density), _ptr(solid_sdf), _ptr(out), distance,
                                                _stream(stream)))


def op_build_fluid_inside_sdf(res, density, solid_sdf, out, distance=1000, stream=None):
    """buildFluidInsideSDFInvoker (HybridSimulatorBuildSDF.cu:209-238)."""
    _check(lib().hfg_op_build_fluid_inside_sdf(_i3(res), _ptr(density), _ptr(solid_sdf), _ptr(out), distance,
                                               _stream(stream)))


def op_build_mixed_fluid_outside_sdf(res, grid_density, mixed_density, grid_outside_sdf, out, stream=None):
    """buildMixedFluidOutsideSDFInvoker (HybridSimulatorBuildSDF.cu:240-266)."""
    _check(lib().hfg_op_build_mixed_fluid_outside_sdf(_i3(res), _ptr(grid_density), _ptr(mixed_density),
                                                      _ptr(grid_outside_sdf), _ptr(out), _stream(stream)))


def op_seed_particles(res, origin, spacing, fluid_sdf, solid_sdf, per_cell, seed, pos=None, capacity=0, stream=None):
    n = C.c_longlong(0)
    _check(lib().hfg_op_seed_particles(_i3(res), _f3(origin), _f3(spacing), _ptr(fluid_sdf), _ptr(solid_sdf),
                                       per_cell, seed, _ptr(pos), capacity, C.byref(n), _stream(stream)))
    return n.value


# ---------------------------------------------------------------- server --
def scene_desc(res, steps=10, spheres=(), fluid_max=(0.4, 0.6, 1.0), per_cell=8, seed=0, dt=1.0 / 60.0,
               cfl=1.0, mixing=0.05, keep_particles=False, **options) -> SceneDesc:
    """A dam-break request: walls, up to 4 static spheres (cx, cy, cz, r),
    fluid below fluid_max; `options` fill hfg_options_t (precond, tol, ...)."""
    d = SceneDesc()
    d.res[:] = [int(r) for r in res]
    d.dt = dt
    d.fluid_max[:] = [float(f) for f in fluid_max]
    d.n_spheres = len(spheres)
    for i, sp in enumerate(spheres):
        d.spheres[i][:] = [float(v) for v in sp]
    d.per_cell, d.seed, d.cfl, d.mixing, d.steps = per_cell, seed, cfl, mixing, steps
    d.keep_particles = int(keep_particles)
    o = default_options()
    for k, v in options.items():
        setattr(o, k, v)
    d.options = o
    return d


def scene_bytes(res, particles, boundaries=1, precond=PRECOND_JACOBI) -> int:
    out = C.c_longlong()
    _check(lib().hfg_scene_bytes(_i3(res), particles, boundaries, precond, C.byref(out)))
    return out.value


class Batch:
    """hfg_batch_*: many resident dam-break scenes stepped together, the CFL
    substeps of all of them in one launch per substep."""

    def __init__(self, descs, threads: int = 16, device: int = 0):
        arr = (SceneDesc * len(descs))(*descs)
        h = C.c_void_p()
        _check(lib().hfg_batch_create(device, C.cast(arr, C.c_void_p), len(descs), threads, C.byref(h)))
        self._h = h
        self.n = len(descs)

    def step(self, steps: int = 1):
        """Advances every scene `steps` steps; returns each step's wall ms."""
        ms = (C.c_double * max(steps, 1))()
        _check(lib().hfg_batch_step(self._h, steps, C.cast(ms, C.c_void_p)))
        return list(ms[:steps])

    def stats(self, scene: int) -> dict:
        st = Stats()
        _check(lib().hfg_batch_scene_stats(self._h, scene, C.byref(st)))
        return st.as_dict()

    def particles(self, scene: int, n: int) -> np.ndarray:
        out = np.empty((n, 3), np.float32)
        _check(lib().hfg_batch_particles(self._h, scene, _fptr(out), 3 * n))
        return out

    def close(self):
        if getattr(self, "_h", None):
            _check(lib().hfg_batch_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """hfg_server_*: continuous batching of dam-break requests on one GPU."""

    def __init__(self, slots: int = 8, budget_bytes: int = 150 * 10**9, device: int = 0):
        h = C.c_void_p()
        _check(lib().hfg_server_create(device, slots, budget_bytes, C.byref(h)))
        self._h = h

    def submit(self, desc: SceneDesc) -> int:
        rid = C.c_longlong()
        _check(lib().hfg_server_submit(self._h, C.byref(desc), C.byref(rid)))
        return rid.value

    def info(self, rid: int, wait: bool = False) -> dict:
        inf = RequestInfo()
        f = lib().hfg_server_wait if wait else lib().hfg_server_info
        _check(f(self._h, rid, C.byref(inf)))
        return _struct_dict(inf)

    def wait(self, rid: int) -> dict:
        return self.info(rid, wait=True)

    def step_times(self, rid: int, cap: int = 4096):
        buf = (C.c_double * cap)()
        n = lib().hfg_server_step_times(self._h, rid, buf, cap)
        if n < 0:
            _check(n)
        return list(buf[:n])

    def particles(self, rid: int, n: int) -> np.ndarray:
        out = np.empty((n, 3), np.float32)
        _check(lib().hfg_server_particles(self._h, rid, _fptr(out), 3 * n))
        return out

    def drain(self):
        _check(lib().hfg_server_drain(self._h))

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().hfg_server_stats(self._h, C.byref(st)))
        return _struct_dict(st)

    def close(self):
        if getattr(self, "_h", None):
            _check(lib().hfg_server_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
