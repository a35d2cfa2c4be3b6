"""ctypes binding of the CPU oracle (oracle/hfg_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product.  The oracle restates the
reference's grid step on the CPU (FP32 with every operation rounded separately, in
the reference's order, or FP64).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libhfg_oracle.so")

I3 = C.c_int * 3
F3 = C.c_float * 3
PF = C.POINTER(C.c_float)
PD = C.POINTER(C.c_double)
PU8 = C.POINTER(C.c_uint8)
PU32 = C.POINTER(C.c_uint32)

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "hfg_oracle.cpp")
        if not os.path.exists(LIB_PATH) or (os.path.exists(src) and os.path.getmtime(src) > os.path.getmtime(LIB_PATH)):
            build()
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        sig = {
            "orc_num_threads": (C.c_int, []),
            "orc_set_num_threads": (None, [C.c_int]),
            "orc_philox": (None, [PU32, C.c_uint32, C.c_uint32, PU32]),
            "orc_seed_particles": (C.c_longlong, [I3, F3, F3, PF, PF, C.c_int, C.c_ulonglong, PF]),
            "orc_fluid_domain_from_bbox": (None, [I3, F3, F3, F3, F3, PF]),
            "orc_build_fluid_sdf": (None, [I3, PF, C.c_int, PF]),
            "orc_build_fluid_density": (None, [I3, PF, PF, PF]),
            "orc_build_fluid_side_sdf": (None, [I3, PF, PF, C.c_int, C.c_int, PF]),
            "orc_build_mixed_fluid_outside_sdf": (None, [I3, PF, PF, PF, PF]),
            "orc_mix_field_with_density_cc": (None, [C.c_longlong, PF, PF, PF, PF]),
            "orc_mix_field_with_density_fc": (None, [I3, PF, PF, PF, PF, PF, PF, PF, PF]),
            "orc_mix_particle_vel": (None, [PF, PF, PF, C.c_longlong, C.c_float, C.c_float, C.c_float, C.c_float,
                                            C.c_float, PF]),
            "orc_solver_mix_vel": (None, [vp, PF, PF, PF, PF, PF]),
            "orc_markers_from_particles": (None, [I3, F3, F3, PF, PF, C.c_longlong, PU8, PU32]),
            "orc_markers_from_sdf": (None, [I3, PF, PF, PU8]),
            "orc_build_matrix_a": (None, [C.c_int, I3, F3, C.c_float, PU8, PF]),
            "orc_build_rhs": (None, [C.c_int, I3, F3, PF, PF, PF, PF, PF, PF, PU8, PF]),
            "orc_apply_a": (None, [C.c_int, I3, F3, C.c_float, PU8, PF, PF]),
            "orc_project": (C.c_longlong, [C.c_int, I3, F3, C.c_float, PU8, PF, PF, PF, PF, PF, PF, C.c_int, C.c_int,
                                           C.c_double, C.c_longlong, PF, PD]),
            "orc_extrapolate": (None, [I3, PF, C.c_int, PF]),
            "orc_sample_fc": (None, [C.c_int, I3, F3, F3, PF, PF, PF, PF, C.c_longlong, PF]),
            "orc_sample_cc_alg": (None, [C.c_int, I3, F3, F3, PF, PF, C.c_longlong, C.c_int, PF]),
            "orc_sample_fc_alg": (None, [I3, F3, F3, PF, PF, PF, PF, C.c_longlong, C.c_int, PF]),
            "orc_sl_advect_fc_alg": (None, [I3, F3, F3, PF, PF, PF, PF, PF, PF, C.c_float, C.c_int, C.c_int, PF, PF, PF]),
            "orc_sl_advect_cc_alg": (None, [I3, F3, F3, PF, PF, PF, PF, C.c_float, C.c_int, C.c_int, PF]),
            "orc_solver_set_sampling": (None, [vp, C.c_int]),
            "orc_sample_cc": (None, [I3, F3, F3, PF, PF, C.c_longlong, PF]),
            "orc_g2p_fc": (None, [I3, F3, F3, PF, PF, PF, PF, C.c_longlong, C.c_int, PF]),
            "orc_g2p_cc": (None, [I3, F3, F3, PF, PF, C.c_longlong, C.c_int, PF]),
            "orc_p2g_fc": (None, [C.c_int, I3, F3, F3, PF, PF, C.c_longlong, C.c_int, PF, PF, PF, PF, PF, PF]),
            "orc_p2g_cc": (None, [I3, F3, F3, PF, PF, C.c_longlong, C.c_int, C.c_int, PF, PF]),
            "orc_advect_particles": (C.c_int, [C.c_int, I3, F3, F3, PF, PF, PF, PF, C.c_longlong, C.c_float,
                                               C.c_float, C.c_int, C.c_int]),
            "orc_sl_advect_fc": (None, [C.c_int, I3, F3, F3, PF, PF, PF, PF, PF, PF, C.c_float, C.c_int, PF, PF, PF]),
            "orc_sl_advect_cc": (None, [I3, F3, F3, PF, PF, PF, PF, C.c_float, C.c_int, PF]),
            "orc_solver_create": (vp, [C.c_int, C.c_float, I3, F3, F3]),
            "orc_solver_destroy": (None, [vp]),
            "orc_solver_add_boundary": (None, [vp, PF, C.c_float, C.c_float, C.c_float]),
            "orc_solver_set_boundary_velocity": (None, [vp, C.c_int, C.c_float, C.c_float, C.c_float]),
            "orc_solver_set_velocity": (None, [vp, PF, PF, PF]),
            "orc_solver_set_fluid_domain": (None, [vp, PF]),
            "orc_solver_set_color": (None, [vp, PF, PF, PF]),
            "orc_solver_set_advection": (None, [vp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int]),
            "orc_solver_set_particles": (None, [vp, PF, PF, C.c_longlong]),
            "orc_solver_set_pcg": (None, [vp, C.c_int, C.c_int, C.c_double, C.c_longlong]),
            "orc_solver_add_external_force": (None, [vp, C.c_float, C.c_float, C.c_float]),
            "orc_solver_update": (C.c_int, [vp]),
            "orc_solver_update_without_pressure": (C.c_int, [vp]),
            "orc_solver_solve_pressure": (C.c_int, [vp]),
            "orc_solver_get_velocity": (None, [vp, C.c_int, PF, PF, PF]),
            "orc_solver_get_velocity_f64": (None, [vp, PD, PD, PD]),
            "orc_solver_get_particles_f64": (None, [vp, PD, PD]),
            "orc_solver_get_fluid_domain": (None, [vp, PF]),
            "orc_solver_get_color": (None, [vp, PF, PF, PF]),
            "orc_solver_get_markers": (None, [vp, PU8]),
            "orc_solver_get_pressure": (None, [vp, PF]),
            "orc_solver_get_solid_sdf": (None, [vp, PF]),
            "orc_solver_get_solid_vel": (None, [vp, PF, PF, PF]),
            "orc_solver_num_particles": (C.c_longlong, [vp]),
            "orc_solver_get_particles": (None, [vp, PF, PF]),
            "orc_solver_stats": (None, [vp, PD]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


def f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def fp(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(PF)


def u8p(a: np.ndarray):
    assert a.dtype == np.uint8 and a.flags.c_contiguous
    return a.ctypes.data_as(PU8)


def face_shapes(res):
    nx, ny, nz = res
    return ((nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx))


def i3(v):
    return I3(*[int(x) for x in v])


def f3(v):
    return F3(*[float(x) for x in v])


# ------------------------------------------------------------------ operators
def seed_particles(res, origin, spacing, fluid_sdf, solid_sdf, per_cell, seed):
    fs, ss = f32(fluid_sdf).reshape(-1), f32(solid_sdf).reshape(-1)
    n = lib().orc_seed_particles(i3(res), f3(origin), f3(spacing), fp(fs), fp(ss), per_cell, seed, None)
    pos = np.empty((n, 3), np.float32)
    lib().orc_seed_particles(i3(res), f3(origin), f3(spacing), fp(fs), fp(ss), per_cell, seed, fp(pos))
    return pos


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    out = (C.c_uint32 * 4)()
    lib().orc_philox(c, key & 0xFFFFFFFF, key >> 32, out)
    return list(out)


def fluid_domain_from_bbox(res, origin, spacing, mn, mx):
    out = np.empty(res[::-1], np.float32)
    lib().orc_fluid_domain_from_bbox(i3(res), f3(origin), f3(spacing), f3(mn), f3(mx), fp(out))
    return out


def build_fluid_sdf(res, domain, layers=1000):
    out = np.empty(res[::-1], np.float32)
    lib().orc_build_fluid_sdf(i3(res), fp(f32(domain).reshape(-1)), layers, fp(out))
    return out


def build_fluid_density(res, domain, solid_sdf):
    out = np.empty(res[::-1], np.float32)
    lib().orc_build_fluid_density(i3(res), fp(f32(domain).reshape(-1)), fp(f32(solid_sdf).reshape(-1)), fp(out))
    return out


def build_fluid_side_sdf(res, density, solid_sdf, outside, distance=1000, out=None):
    """buildFluidOutsideSDF (outside) / buildFluidInsideSDF with their
    invokers' `distance` sweeps (HybridSimulatorBuildSDF.cu:4-146,177-238).
    `out` is the field the sweeps start from (read only when distance is 0)."""
    out = np.zeros(res[::-1], np.float32) if out is None else f32(out).reshape(res[::-1]).copy()
    lib().orc_build_fluid_side_sdf(i3(res), fp(f32(density).reshape(-1)), fp(f32(solid_sdf).reshape(-1)),
                                   int(bool(outside)), int(distance), fp(out))
    return out


def build_mixed_fluid_outside_sdf(res, grid_density, mixed_density, grid_outside):
    """buildMixedFluidOutsideSDF (HybridSimulatorBuildSDF.cu:139-175,240-266)."""
    out = np.empty(res[::-1], np.float32)
    lib().orc_build_mixed_fluid_outside_sdf(i3(res), fp(f32(grid_density).reshape(-1)),
                                            fp(f32(mixed_density).reshape(-1)), fp(f32(grid_outside).reshape(-1)),
                                            fp(out))
    return out


def mix_field_with_density_cc(a, b, wa, wb):
    out = f32(b).copy()
    lib().orc_mix_field_with_density_cc(out.size, fp(f32(a)), fp(out), fp(f32(wa)), fp(f32(wb)))
    return out


def mix_field_with_density_fc(res, a, b, wa, wb):
    out = [f32(x).copy() for x in b]
    lib().orc_mix_field_with_density_fc(i3(res), *[fp(f32(x)) for x in a], *[fp(x) for x in out],
                                        fp(f32(wa).reshape(-1)), fp(f32(wb).reshape(-1)))
    return out


def mix_particle_vel(pic, flip, dist, cell, g, gf, f, pr, predict):
    out = f32(predict).copy()
    lib().orc_mix_particle_vel(fp(f32(pic)), fp(f32(flip)), fp(f32(dist)), f32(dist).size, cell, g, gf, f, pr, fp(out))
    return out


def markers_from_particles(res, origin, spacing, solid_sdf, pos):
    ss = f32(solid_sdf).reshape(-1)
    p = f32(pos).reshape(-1)
    mk = np.empty(res[::-1], np.uint8)
    cnt = np.empty(res[::-1], np.uint32)
    lib().orc_markers_from_particles(i3(res), f3(origin), f3(spacing), fp(ss), fp(p), p.size // 3, u8p(mk),
                                     cnt.ctypes.data_as(PU32))
    return mk, cnt


def markers_from_sdf(res, solid_sdf, fluid_sdf):
    mk = np.empty(res[::-1], np.uint8)
    lib().orc_markers_from_sdf(i3(res), fp(f32(solid_sdf).reshape(-1)), fp(f32(fluid_sdf).reshape(-1)), u8p(mk))
    return mk


def build_matrix_a(res, spacing, dt, markers, dbl=0):
    A = np.empty(4 * res[0] * res[1] * res[2], np.float32)
    lib().orc_build_matrix_a(dbl, i3(res), f3(spacing), dt, u8p(np.ascontiguousarray(markers, np.uint8).reshape(-1)),
                             fp(A))
    return A


def build_rhs(res, spacing, vel, solid_vel, markers, dbl=0):
    b = np.empty(res[::-1], np.float32)
    v = [f32(a).reshape(-1) for a in vel]
    s = [f32(a).reshape(-1) for a in solid_vel]
    lib().orc_build_rhs(dbl, i3(res), f3(spacing), *[fp(a) for a in v], *[fp(a) for a in s],
                        u8p(np.ascontiguousarray(markers, np.uint8).reshape(-1)), fp(b))
    return b


def apply_a(res, spacing, dt, markers, x, dbl=0):
    y = np.empty(res[::-1], np.float32)
    xx = f32(x).reshape(-1)
    lib().orc_apply_a(dbl, i3(res), f3(spacing), dt, u8p(np.ascontiguousarray(markers, np.uint8).reshape(-1)), fp(xx),
                      fp(y))
    return y


def project(res, spacing, dt, markers, vel, solid_vel, precond=0, tol_mode=0, tol=1e-3, max_iter=-1, dbl=0):
    v = [f32(a).copy().reshape(s) for a, s in zip(vel, face_shapes(res))]
    s = [f32(a).reshape(-1) for a in solid_vel]
    p = np.empty(res[::-1], np.float32)
    st = (C.c_double * 2)()
    it = lib().orc_project(dbl, i3(res), f3(spacing), dt, u8p(np.ascontiguousarray(markers, np.uint8).reshape(-1)),
                           *[fp(a) for a in v], *[fp(a) for a in s], precond, tol_mode, tol, max_iter, fp(p), st)
    return v, p, {"iterations": int(it), "residual": st[0], "rhs_norm": st[1]}


def extrapolate(res, field, layers=1000, with_markers=False):
    f = f32(field).copy()
    mk = np.empty_like(f) if with_markers else None
    lib().orc_extrapolate(i3(res), fp(f), layers, fp(mk) if with_markers else None)
    return (f, mk) if with_markers else f


def extrapolate_fc(res, vel, layers=1000):
    out = []
    for a, s in zip(vel, face_shapes(res)):
        r = (s[2], s[1], s[0])
        out.append(extrapolate(r, f32(a).reshape(s), layers))
    return out


def sample_fc(res, origin, spacing, vel, pos, dbl=0):
    p = f32(pos).reshape(-1)
    out = np.empty(p.size, np.float32)
    v = [f32(a).reshape(-1) for a in vel]
    lib().orc_sample_fc(dbl, i3(res), f3(origin), f3(spacing), *[fp(a) for a in v], fp(p), p.size // 3, fp(out))
    return out.reshape(-1, 3)


def sample_cc(res, origin, spacing, f, pos, alg=0, dbl=0):
    """alg: ESamplingAlgorithm (0 trilinear, 1 Catmull-Rom, 2 monotonic
    Catmull-Rom, 3 Bridson cubic, 4 clamped Bridson cubic)."""
    p = f32(pos).reshape(-1)
    out = np.empty(p.size // 3, np.float32)
    if alg == 0 and not dbl:
        lib().orc_sample_cc(i3(res), f3(origin), f3(spacing), fp(f32(f).reshape(-1)), fp(p), p.size // 3, fp(out))
    else:
        lib().orc_sample_cc_alg(dbl, i3(res), f3(origin), f3(spacing), fp(f32(f).reshape(-1)), fp(p), p.size // 3,
                                alg, fp(out))
    return out


def sample_fc_alg(res, origin, spacing, vel, pos, alg):
    p = f32(pos).reshape(-1)
    out = np.empty(p.size, np.float32)
    v = [f32(a).reshape(-1) for a in vel]
    lib().orc_sample_fc_alg(i3(res), f3(origin), f3(spacing), *[fp(a) for a in v], fp(p), p.size // 3, alg, fp(out))
    return out.reshape(-1, 3)


def g2p_fc(res, origin, spacing, vel, pos, alg):
    p = f32(pos).reshape(-1)
    out = np.empty(p.size, np.float32)
    v = [f32(a).reshape(-1) for a in vel]
    lib().orc_g2p_fc(i3(res), f3(origin), f3(spacing), *[fp(a) for a in v], fp(p), p.size // 3, alg, fp(out))
    return out.reshape(-1, 3)


def g2p_cc(res, origin, spacing, f, pos, alg):
    p = f32(pos).reshape(-1)
    out = np.empty(p.size // 3, np.float32)
    lib().orc_g2p_cc(i3(res), f3(origin), f3(spacing), fp(f32(f).reshape(-1)), fp(p), p.size // 3, alg, fp(out))
    return out


def p2g_fc(res, origin, spacing, pos, vel, alg, dbl=0):
    p = f32(pos).reshape(-1)
    v = f32(vel).reshape(-1)
    outs = [np.empty(s, np.float32) for s in face_shapes(res)]
    ws = [np.empty(s, np.float32) for s in face_shapes(res)]
    lib().orc_p2g_fc(dbl, i3(res), f3(origin), f3(spacing), fp(p), fp(v), p.size // 3, alg, *[fp(a) for a in outs],
                     *[fp(a) for a in ws])
    return outs, ws


def p2g_cc(res, origin, spacing, pos, val, alg, normalize=True):
    p = f32(pos).reshape(-1)
    out = np.empty(res[::-1], np.float32)
    w = np.empty(res[::-1], np.float32)
    lib().orc_p2g_cc(i3(res), f3(origin), f3(spacing), fp(p), fp(f32(val).reshape(-1)), p.size // 3, alg,
                     int(normalize), fp(out), fp(w))
    return out, w


def advect_particles(res, origin, spacing, vel, pos, dt, cfl=1.0, accuracy=2, clamp_mode=1, dbl=0):
    p = f32(pos).copy().reshape(-1)
    v = [f32(a).reshape(-1) for a in vel]
    n = lib().orc_advect_particles(dbl, i3(res), f3(origin), f3(spacing), *[fp(a) for a in v], fp(p), p.size // 3,
                                   dt, cfl, accuracy, clamp_mode)
    return p.reshape(-1, 3), n


def sl_advect_fc(res, origin, spacing, field, vel, dt, accuracy, dbl=0, sampling=0):
    f = [f32(a).reshape(-1) for a in field]
    v = [f32(a).reshape(-1) for a in vel]
    out = [np.empty(s, np.float32) for s in face_shapes(res)]
    if sampling:
        lib().orc_sl_advect_fc_alg(i3(res), f3(origin), f3(spacing), *[fp(a) for a in f], *[fp(a) for a in v], dt,
                                   accuracy, sampling, *[fp(a) for a in out])
        return out
    lib().orc_sl_advect_fc(dbl, i3(res), f3(origin), f3(spacing), *[fp(a) for a in f], *[fp(a) for a in v], dt,
                           accuracy, *[fp(a) for a in out])
    return out


def sl_advect_cc(res, origin, spacing, field, vel, dt, accuracy, sampling=0):
    v = [f32(a).reshape(-1) for a in vel]
    out = np.empty(res[::-1], np.float32)
    if sampling:
        lib().orc_sl_advect_cc_alg(i3(res), f3(origin), f3(spacing), fp(f32(field).reshape(-1)),
                                   *[fp(a) for a in v], dt, accuracy, sampling, fp(out))
        return out
    lib().orc_sl_advect_cc(i3(res), f3(origin), f3(spacing), fp(f32(field).reshape(-1)), *[fp(a) for a in v], dt,
                           accuracy, fp(out))
    return out


class Solver:
    """Oracle CGridFluidSolver (GridFluidSolver.cpp), FP32 (dbl=0) or FP64 (dbl=1)."""

    def __init__(self, dt, res, origin=(0, 0, 0), spacing=(1, 1, 1), dbl=0):
        self.res = tuple(int(r) for r in res)
        self._h = lib().orc_solver_create(dbl, dt, i3(res), f3(origin), f3(spacing))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_solver_destroy(self._h)
            self._h = None

    def add_solid_boundary(self, sdf, vel=(0, 0, 0)):
        lib().orc_solver_add_boundary(self._h, fp(f32(sdf).reshape(-1)), *[float(v) for v in vel])

    def mix_vel_field_with_others(self, other, w_other, w_fluid):
        lib().orc_solver_mix_vel(self._h, *[fp(f32(a).reshape(-1)) for a in other], fp(f32(w_other).reshape(-1)),
                                 fp(f32(w_fluid).reshape(-1)))

    def set_sampling(self, alg):
        lib().orc_solver_set_sampling(self._h, int(alg))

    def set_boundary_velocity(self, index, vel):
        lib().orc_solver_set_boundary_velocity(self._h, int(index), *[float(v) for v in vel])

    def set_velocity_field(self, x, y, z):
        lib().orc_solver_set_velocity(self._h, *[fp(f32(a).reshape(-1)) for a in (x, y, z)])

    def set_fluid_domain_field(self, d):
        lib().orc_solver_set_fluid_domain(self._h, fp(f32(d).reshape(-1)))

    def set_color_field(self, x, y, z):
        lib().orc_solver_set_color(self._h, *[fp(f32(a).reshape(-1)) for a in (x, y, z)])

    def set_advection(self, kind, accuracy=2, alg=2, cfl=1.0, mixing=0.1, clamp_mode=1, advect_scalars=1):
        lib().orc_solver_set_advection(self._h, kind, accuracy, alg, cfl, mixing, clamp_mode, advect_scalars)

    def set_particles(self, pos, vel=None):
        p = f32(pos).reshape(-1)
        v = None if vel is None else f32(vel).reshape(-1)
        lib().orc_solver_set_particles(self._h, fp(p), None if v is None else fp(v), p.size // 3)

    def set_pcg(self, precond=0, tol_mode=0, tol=1e-3, max_iter=-1):
        lib().orc_solver_set_pcg(self._h, precond, tol_mode, tol, max_iter)

    def add_external_force(self, f):
        lib().orc_solver_add_external_force(self._h, *[float(x) for x in f])

    def update(self, steps=1):
        for _ in range(steps):
            lib().orc_solver_update(self._h)

    def update_without_pressure(self):
        lib().orc_solver_update_without_pressure(self._h)

    def solve_pressure(self):
        lib().orc_solver_solve_pressure(self._h)

    def velocity_field(self, which=0):
        out = [np.empty(s, np.float32) for s in face_shapes(self.res)]
        lib().orc_solver_get_velocity(self._h, which, *[fp(a) for a in out])
        return out

    def velocity_field_f64(self):
        out = [np.empty(s, np.float64) for s in face_shapes(self.res)]
        lib().orc_solver_get_velocity_f64(self._h, *[a.ctypes.data_as(PD) for a in out])
        return out

    def fluid_domain_field(self):
        out = np.empty(self.res[::-1], np.float32)
        lib().orc_solver_get_fluid_domain(self._h, fp(out))
        return out

    def color_field(self):
        out = [np.empty(self.res[::-1], np.float32) for _ in range(3)]
        lib().orc_solver_get_color(self._h, *[fp(a) for a in out])
        return out

    def markers(self):
        out = np.empty(self.res[::-1], np.uint8)
        lib().orc_solver_get_markers(self._h, u8p(out))
        return out

    def pressure(self):
        out = np.empty(self.res[::-1], np.float32)
        lib().orc_solver_get_pressure(self._h, fp(out))
        return out

    def solid_sdf(self):
        out = np.empty(self.res[::-1], np.float32)
        lib().orc_solver_get_solid_sdf(self._h, fp(out))
        return out

    def solid_vel_field(self):
        out = [np.empty(s, np.float32) for s in face_shapes(self.res)]
        lib().orc_solver_get_solid_vel(self._h, *[fp(a) for a in out])
        return out

    @property
    def num_particles(self):
        return int(lib().orc_solver_num_particles(self._h))

    def particles(self):
        n = self.num_particles
        pos = np.empty((n, 3), np.float32)
        vel = np.empty((n, 3), np.float32)
        lib().orc_solver_get_particles(self._h, fp(pos), fp(vel))
        return pos, vel

    def particles_f64(self):
        """Positions and velocities at the solver's own precision (FP64 for dbl=1)."""
        n = self.num_particles
        pos = np.empty((n, 3), np.float64)
        vel = np.empty((n, 3), np.float64)
        lib().orc_solver_get_particles_f64(self._h, pos.ctypes.data_as(PD), vel.ctypes.data_as(PD))
        return pos, vel

    def stats(self):
        st = (C.c_double * 6)()
        lib().orc_solver_stats(self._h, st)
        return {"cg_iterations": int(st[0]), "cg_residual": st[1], "cg_rhs_norm": st[2], "sim_time": st[3],
                "substeps": int(st[4]), "buffer_flag": int(st[5])}
