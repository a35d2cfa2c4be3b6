"""ctypes binding of oracle/_ref/refgpu/libhfg_refgpu.so: the reference's own
CGridFluidSolver (GridFluidSolver.cpp) compiled for sm_100a from its
unmodified CUDA sources by oracle/refgpu/build.sh, behind the small C ABI of
oracle/refgpu/driver.cu.  libhfg_refgpu64.so is the same step built with the
reference's own FP64 switch (DOUBLE_REAL, Common.h:82-104); RefSolver(...,
fp64=True) drives it, with float64 arrays.

Test infrastructure: the GPU parity tests step it beside libhfgrid on the
same seeded particles, and the reference arm of bench.py times it.  The
library is built where a reference checkout exists and travels with the
tree as a built file; `available()` says whether it is there.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "refgpu", "libhfg_refgpu.so")
LIB64 = os.path.join(HERE, "_ref", "refgpu", "libhfg_refgpu64.so")

PF = C.POINTER(C.c_float)
PI = C.POINTER(C.c_int)
_libs = {}


def available(fp64: bool = False) -> bool:
    return os.path.exists(LIB64 if fp64 else LIB)


def _f3(v):
    return (C.c_float * 3)(*[float(x) for x in v])


def lib(fp64: bool = False):
    if fp64 not in _libs:
        path = LIB64 if fp64 else LIB
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is not built (oracle/refgpu/build.sh <reference checkout>)")
        L = C.CDLL(path)
        PR = C.POINTER(C.c_double if fp64 else C.c_float)
        L.rg_last_error.restype = C.c_char_p
        L.rg_init.restype = C.c_int
        L.rg_create.restype = C.c_void_p
        L.rg_create.argtypes = [C.c_float, PI, PF, PF]
        L.rg_destroy.argtypes = [C.c_void_p]
        L.rg_real_size.restype = C.c_int
        assert L.rg_real_size() == (8 if fp64 else 4)
        for name in ("rg_add_solid", "rg_set_fluid_domain", "rg_markers", "rg_pressure"):
            getattr(L, name).restype = C.c_int
            getattr(L, name).argtypes = [C.c_void_p, PR]
        L.rg_add_moving_solid.restype = C.c_int
        L.rg_add_moving_solid.argtypes = [C.c_void_p, PR, PF]
        L.rg_fluid_domain_bbox.restype = C.c_int
        L.rg_fluid_domain_bbox.argtypes = [C.c_void_p, PF, PF]
        L.rg_update_boundaries.restype = C.c_int
        L.rg_update_boundaries.argtypes = [C.c_void_p]
        L.rg_set_mix_pic_flip.restype = C.c_longlong
        L.rg_set_mix_pic_flip.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_float, PR, C.c_longlong]
        L.rg_set_cg_iteration_cap.restype = C.c_int
        L.rg_set_cg_iteration_cap.argtypes = [C.c_void_p, C.c_uint]
        L.rg_update.restype = C.c_int
        L.rg_update.argtypes = [C.c_void_p]
        L.rg_take_ax_calls.restype = C.c_ulonglong
        L.rg_velocity.restype = C.c_int
        L.rg_velocity.argtypes = [C.c_void_p, PR, PR, PR]
        L.rg_num_particles.restype = C.c_longlong
        L.rg_num_particles.argtypes = [C.c_void_p]
        L.rg_particles.restype = C.c_int
        L.rg_particles.argtypes = [C.c_void_p, PR, PR]
        L.rg_synchronize.restype = C.c_int
        L.rg_last_error.restype = C.c_char_p
        rc = L.rg_init()
        if rc != 0:
            raise RuntimeError(f"reference solver: {L.rg_last_error().decode()}")
        _libs[fp64] = L
    return _libs[fp64]


def face_shapes(res):
    nx, ny, nz = res
    return [(nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx)]


class RefSolver:
    """CGridFluidSolver(dt, res, origin, spacing) of the reference; fp64
    selects its FP64 build (arrays in and out are then float64)."""

    def __init__(self, dt, res, origin, spacing, fp64: bool = False):
        self.res = tuple(int(r) for r in res)
        self.fp64 = bool(fp64)
        self.dtype = np.float64 if self.fp64 else np.float32
        self._L = lib(self.fp64)
        h = self._L.rg_create(float(dt), (C.c_int * 3)(*self.res), _f3(origin), _f3(spacing))
        if not h:
            raise RuntimeError(f"reference solver: {self._L.rg_last_error().decode()}")
        self._h = h

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(f"reference solver: {self._L.rg_last_error().decode()}")

    def _p(self, a):
        return a.ctypes.data_as(C.POINTER(C.c_double if self.fp64 else C.c_float))

    def close(self):
        if getattr(self, "_h", None):
            self._L.rg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _cell(self, a):
        a = np.ascontiguousarray(a, self.dtype)
        assert a.shape == self.res[::-1]
        return a

    def add_solid_boundary(self, sdf, vel=None):
        """addSolidBoundary(sdf); with a nonzero velocity, the boundary moves
        at it (CBoundarys::addBoundary(sdf, vel))."""
        if vel is None or not any(vel):
            self._check(self._L.rg_add_solid(self._h, self._p(self._cell(sdf))))
        else:
            self._check(self._L.rg_add_moving_solid(self._h, self._p(self._cell(sdf)), _f3(vel)))

    def set_fluid_domain_field(self, dom):
        self._check(self._L.rg_set_fluid_domain(self._h, self._p(self._cell(dom))))

    def generate_fluid_domain_from_bbox(self, mn, mx):
        self._check(self._L.rg_fluid_domain_bbox(self._h, _f3(mn), _f3(mx)))

    def update_boundaries(self):
        """Assemble the total boundary fields now (no motion), so that the
        seeding of set_mix_pic_flip skips cells inside solids."""
        self._check(self._L.rg_update_boundaries(self._h))

    def set_mix_pic_flip(self, per_cell, cfl, mixing, pos=None) -> int:
        """The PIC/FLIP mix (linear transfers); `pos` (n, 3) replaces the
        reference's own random seeding and must have its count."""
        if pos is not None:
            pos = np.ascontiguousarray(pos, self.dtype)
            n = self._L.rg_set_mix_pic_flip(self._h, int(per_cell), float(cfl), float(mixing), self._p(pos),
                                            pos.shape[0])
        else:
            n = self._L.rg_set_mix_pic_flip(self._h, int(per_cell), float(cfl), float(mixing), None, 0)
        if n < 0:
            raise RuntimeError(f"reference solver: {self._L.rg_last_error().decode()}")
        return int(n)

    def set_cg_iteration_cap(self, cap: int):
        self._check(self._L.rg_set_cg_iteration_cap(self._h, int(cap)))

    def update(self):
        self._check(self._L.rg_update(self._h))

    def take_ax_calls(self) -> int:
        """A*x products of the pressure solves of this build since the last
        call: one for the initial residual plus one per CG iteration, per solve."""
        return int(self._L.rg_take_ax_calls())

    def velocity_field(self):
        out = [np.empty(s, self.dtype) for s in face_shapes(self.res)]
        self._check(self._L.rg_velocity(self._h, *[self._p(o) for o in out]))
        return out

    @property
    def num_particles(self) -> int:
        return int(self._L.rg_num_particles(self._h))

    def particles(self):
        n = self.num_particles
        pos = np.empty((n, 3), self.dtype)
        vel = np.empty((n, 3), self.dtype)
        self._check(self._L.rg_particles(self._h, self._p(pos), self._p(vel)))
        return pos, vel

    def markers(self):
        """The pressure solver's marker field (0 air, 1 fluid, 2 solid, as floats)."""
        out = np.empty(self.res[::-1], self.dtype)
        self._check(self._L.rg_markers(self._h, self._p(out)))
        return out

    def pressure(self):
        out = np.empty(self.res[::-1], self.dtype)
        self._check(self._L.rg_pressure(self._h, self._p(out)))
        return out

    def synchronize(self):
        self._check(self._L.rg_synchronize())
