// hfg_device.cuh -- device-side conventions shared by every sm_100a kernel of
// the grid step.
//
// Index conventions follow the reference engine (MPhysics/Common.h:250,
// MPhysics/EulerMathTool.cu:63-73): cell-centred linear index
// z*nx*ny + y*nx + x, clamp-to-edge for every neighbour and interpolation
// corner.  Face-centred components live on (nx+1,ny,nz), (nx,ny+1,nz) and
// (nx,ny,nz+1) grids whose origin is shifted by -h/2 on their own axis
// (MPhysics/FieldMathTool.cu:800-808).
#pragma once
#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

namespace hfg {

// Unknown-face sentinel (MPhysics/MMathExtra.h:58 UNKNOWN = FLT_MAX).
constexpr float kUnknown = FLT_MAX;

// Cell marker values (MPhysics/EulerParticlesTool.cu:61-75): air, fluid, solid.
constexpr uint8_t kAir = 0, kFluid = 1, kSolid = 2;

// Particle/grid transfer kernels (MPhysics/EnumType.h:19-26).
enum TransferAlg : int { P2GSUM = 0, G2PNEAREST = 1, LINEAR = 2, QUADRATIC = 3, CUBIC = 4 };

struct Dim3i {
  int x, y, z;
  __host__ __device__ long long size() const { return (long long)x * y * z; }
};

// Geometry of one scalar grid (cell-centred, or one face component).
struct Geom {
  Dim3i r;
  float ox, oy, oz;
  float hx, hy, hz;
};

__host__ __device__ inline Geom faceGeom(const Geom& cc, int axis) {
  Geom g = cc;
  if (axis == 0) { g.r.x += 1; g.ox = cc.ox - cc.hx / 2; }
  if (axis == 1) { g.r.y += 1; g.oy = cc.oy - cc.hy / 2; }
  if (axis == 2) { g.r.z += 1; g.oz = cc.oz - cc.hz / 2; }
  return g;
}

__host__ __device__ inline int clampi(int i, int n) { return i < 0 ? 0 : (i > n - 1 ? n - 1 : i); }

// clamp-to-edge linear index (transIndex2LinearWithOffset)
__host__ __device__ inline long long linc(int x, int y, int z, const Dim3i& r) {
  x = clampi(x, r.x); y = clampi(y, r.y); z = clampi(z, r.z);
  return ((long long)z * r.y + y) * r.x + x;
}

// floorCUDA (MPhysics/EulerMathTool.cu:93-103); floorCUDA(-1.0f) == -2.
__host__ __device__ inline int floorRef(float v) { return v >= 0.f ? (int)v : (int)v - 1; }

// Exact-rounding helpers: the listed expressions must round like the
// reference's separate float operations (no contraction into FMA).
__device__ inline float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ inline float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ inline float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ inline float fdiv(float a, float b) { return __fdiv_rn(a, b); }

// Particle -> cell binning (transPos2Index, MPhysics/EulerMathTool.cu:29-40):
// truncation toward zero, then clamp.  Bit-exact with the FP32 reference.
__device__ inline long long binCell(const Geom& g, float px, float py, float pz) {
  float rx = fdiv(fsub(px, g.ox), g.hx);
  float ry = fdiv(fsub(py, g.oy), g.hy);
  float rz = fdiv(fsub(pz, g.oz), g.hz);
  int ix = clampi((int)rx, g.r.x), iy = clampi((int)ry, g.r.y), iz = clampi((int)rz, g.r.z);
  return ((long long)iz * g.r.y + iy) * g.r.x + ix;
}

// Trilinear sample with clamp-to-edge corners, the formula of
// sampleCellCenteredScalarFieldTrilerp (MPhysics/FieldMathTool.cu:52-104).
__device__ inline float trilerp(const float* __restrict__ f, const Geom& g, float px, float py, float pz) {
  float rx = px - g.ox - g.hx / 2, ry = py - g.oy - g.hy / 2, rz = pz - g.oz - g.hz / 2;
  int ix = floorRef(rx / g.hx), iy = floorRef(ry / g.hy), iz = floorRef(rz / g.hz);
  float ox = (rx - (float)ix * g.hx) / g.hx;
  float oy = (ry - (float)iy * g.hy) / g.hy;
  float oz = (rz - (float)iz * g.hz) / g.hz;
  int x0 = clampi(ix, g.r.x), x1 = clampi(ix + 1, g.r.x);
  int y0 = clampi(iy, g.r.y), y1 = clampi(iy + 1, g.r.y);
  int z0 = clampi(iz, g.r.z), z1 = clampi(iz + 1, g.r.z);
  long long sy = g.r.x, sz = (long long)g.r.x * g.r.y;
  const float* b00 = f + z0 * sz + y0 * sy;
  const float* b10 = f + z0 * sz + y1 * sy;
  const float* b01 = f + z1 * sz + y0 * sy;
  const float* b11 = f + z1 * sz + y1 * sy;
  float DBL = __ldg(b00 + x0), DBR = __ldg(b00 + x1);
  float UBL = __ldg(b10 + x0), UBR = __ldg(b10 + x1);
  float DFL = __ldg(b01 + x0), DFR = __ldg(b01 + x1);
  float UFL = __ldg(b11 + x0), UFR = __ldg(b11 + x1);
  float mx = 1 - ox, my = 1 - oy, mz = 1 - oz;
  return DBL * mx * my * mz + DBR * ox * my * mz + UBL * mx * oy * mz + UBR * ox * oy * mz +
         DFL * mx * my * oz + DFR * ox * my * oz + UFL * mx * oy * oz + UFR * ox * oy * oz;
}

struct FaceField {
  float* c[3];
};
struct ConstFaceField {
  const float* c[3];
};

__device__ inline void sampleFace(const ConstFaceField& v, const Geom& cc, float px, float py, float pz, float out[3]) {
#pragma unroll
  for (int a = 0; a < 3; ++a) out[a] = trilerp(v.c[a], faceGeom(cc, a), px, py, pz);
}

// Transfer-kernel weights (MPhysics/EulerMathTool.cu:268-294).
__device__ inline float kLinear(float o) {
  float a = fabsf(o);
  return a < 1.f ? 1.f - a : 0.f;
}
__device__ inline float kQuadratic(float o) {
  float a = fabsf(o);
  if (a < 0.5f) return 0.75f - a * a;
  if (a < 1.5f) return 0.5f * (1.5f - a) * (1.5f - a);
  return 0.f;
}
__device__ inline float kCubic(float o) {
  float a = fabsf(o);
  if (a < 1.f) return 0.5f * a * a * a - a * a + (float)(2.0 / 3.0);
  if (a < 2.f) return (float)(1.0 / 6.0) * (2.f - a) * (2.f - a) * (2.f - a);
  return 0.f;
}

// Per-axis stencil base + weights (MPhysics/EulerParticlesTool.cu:99-103,
// :113-115, :140-142, :167-169).
struct Taps {
  int base[3];
  float w[3][4];
};

template <int ALG>
__device__ inline void taps(const Geom& g, float px, float py, float pz, Taps& t) {
  float rel[3] = {px - g.ox - g.hx * 0.5f, py - g.oy - g.hy * 0.5f, pz - g.oz - g.hz * 0.5f};
  float h[3] = {g.hx, g.hy, g.hz};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int b = floorRef(rel[a] / h[a]);
    float off = (rel[a] - (float)b * h[a]) / h[a];
    t.base[a] = b;
    if (ALG == LINEAR) {
      t.w[a][0] = kLinear(off);
      t.w[a][1] = kLinear(off - 1.f);
    } else if (ALG == QUADRATIC) {
      t.w[a][0] = kQuadratic(off + 1.f); t.w[a][1] = kQuadratic(off);
      t.w[a][2] = kQuadratic(off - 1.f); t.w[a][3] = kQuadratic(off - 2.f);
    } else {
      t.w[a][0] = kCubic(off + 1.f); t.w[a][1] = kCubic(off);
      t.w[a][2] = kCubic(off - 1.f); t.w[a][3] = kCubic(off - 2.f);
    }
  }
}

template <int ALG> struct TapsN { static constexpr int n = (ALG == LINEAR) ? 2 : 4; static constexpr int shift = (ALG == LINEAR) ? 0 : -1; };

// G2P of one component (accumulateCCSField2Particles, EulerParticlesTool.cu:198-288)
template <int ALG>
__device__ inline float g2p(const float* __restrict__ f, const Geom& g, float px, float py, float pz) {
  if (ALG == G2PNEAREST) return __ldg(f + binCell(g, px, py, pz));
  Taps t;
  taps<ALG>(g, px, py, pz, t);
  constexpr int n = TapsN<ALG>::n, s = TapsN<ALG>::shift;
  float acc = 0.f;
#pragma unroll
  for (int z = 0; z < n; ++z)
#pragma unroll
    for (int y = 0; y < n; ++y)
#pragma unroll
      for (int x = 0; x < n; ++x) {
        float w = t.w[0][x] * t.w[1][y] * t.w[2][z];
        acc += w * __ldg(f + linc(t.base[0] + x + s, t.base[1] + y + s, t.base[2] + z + s, g.r));
      }
  return acc;
}

// Deterministic block-level reduction helpers.
__device__ inline double warpSumD(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ inline float warpMaxF(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

}  // namespace hfg
