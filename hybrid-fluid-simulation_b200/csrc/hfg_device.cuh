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
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>
#include <utility>

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

// floorCUDA (MPhysics/EulerMathTool.cu:93-103); floorCUDA(-1.0f) == -2.  The
// argument is clamped to +-2^30 first: a point far outside the grid (a
// back-trace through UNKNOWN = FLT_MAX velocities lands ~1e36 away) would
// otherwise convert to INT_MIN and the "- 1", or the caller's "+ 1" of a
// stencil offset, would overflow; signed overflow is undefined, and the
// compiler may then fold one comparison of a clamp and not the other and
// leave an index outside the grid.  Every grid index lies far inside
// +-2^30, so the clamped result selects the same cells; a NaN (which fmaxf
// drops) still yields NaN weights.
__host__ __device__ inline int floorRef(float v) {
  v = fminf(fmaxf(v, -1073741824.f), 1073741824.f);
  return v >= 0.f ? (int)v : (int)v - 1;
}

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

// Trilinear sampling of a face-centred field, restated for speed: the cell
// coordinate u = (p - o) / h of each axis is formed once (with a reciprocal),
// and the per-axis base index and weight serve all three components (the
// component's own axis uses the face grid, shifted by h/2; the other two the
// cell-centred one).  Mathematically the reference's trilinear formula
// (FieldMathTool.cu:52-104) and its LINEAR transfer weights
// (EulerParticlesTool.cu:113-115); rounding differs in the last bits.
struct AxisW {
  int i0, i1;
  int j;  // corner-table entry less one: the floor index clamped to [-1, n - 1]
  float w1;
};

__device__ __forceinline__ void axisWeights(float t, int n, AxisW& a) {
  float f = floorf(t);
  a.w1 = t - f;
  int i = (int)f;  // saturates far outside the grid
  a.i0 = clampi(i, n);
  // clamp(i + 1) without forming i + 1 first (it overflows at i = INT_MAX)
  a.i1 = min(max(i, -1), n - 2) + 1;
  a.j = min(max(i, -1), n - 1);
}

// axisWeights with the coordinate clamped first to [-1, hi], hi the float
// below n: the floor index is then in [-1, n - 1] with no integer clamp.  A
// coordinate outside that range selects the same edge corners as the integer
// clamp does, which hold equal values (the table's x differences and the y
// and z corner pairs there are exact zeros), so every finite coordinate
// samples the same value as with axisWeights; a NaN coordinate samples the
// edge instead of returning NaN.
__device__ __forceinline__ void clampedAxis(float t, float hi, int jmax, AxisW& a) {
  const float c = fminf(fmaxf(t, -1.0f), hi);
  const float f = floorf(c);
  a.w1 = c - f;
  const int i = (int)f;
  a.i0 = max(i, 0);
  a.i1 = min(i + 1, jmax);
  a.j = i;
}

// Corner table of a face grid of nx x ny x nz values: (nx + 1) x (ny + 1) x
// (nz + 2) float4, entry (L, jy, jx) = (f[z][y0][x0], f[z][y0][x1] -
// f[z][y0][x0], f[z][y1][x0], f[z][y1][x1] - f[z][y1][x0]) with
// z = clamp(L - 1), x0 = clamp(jx - 1), x1 = clamp(jx), y0 = clamp(jy - 1),
// y1 = clamp(jy).  Entry (AxisW::j + 1 of y, AxisW::j + 1 of x) of a sample
// holds the four corners of one z layer of its trilinear stencil, so one
// 16-byte load serves four corners; layers AxisW::j + 1 and AxisW::j + 2 of z
// are the stencil's clamp(i) and clamp(i + 1), because the padding layers 0
// and nz + 1 repeat the end layers.  The two x differences are the FP32
// subtractions the x lerps of every sample would otherwise repeat: stored
// once, they give the same values.
struct FaceQuads {
  // entry (1, 1, 1) of each component's table: AxisW::j is the entry index
  // less one, so a sample's entry is c[a] + (jz * ly + jy) * lx + jx, at
  // least c[a] - (pl + lx + 1), the table's first entry
  const float4* c[3];
  // Sampling constants of the grid, formed once on the host (makeFaceQuads)
  // so that a kernel reads them as launch parameters: the coordinate of a
  // point on axis k is p * inv + offF on the face grid of that axis and
  // p * inv + offC (offF - 1/2) on the cell-centred one; hiF and hiC, the
  // float below n + 1 and n for n cells, bound the coordinate on those two
  // grids, and jF and jC (n and n - 1) are the largest floor index there;
  // lx, ly and pl are the row length, the rows per layer and the layer size
  // of component a's table.
  float inv[3], offF[3], offC[3], hiF[3], hiC[3];
  int jF[3], jC[3];
  unsigned lx[3], ly[3], pl[3];
};

inline FaceQuads makeFaceQuads(const Geom& g, const float4* q0, const float4* q1, const float4* q2) {
  FaceQuads q;
  const float4* base[3] = {q0, q1, q2};
  const float h[3] = {g.hx, g.hy, g.hz}, o[3] = {g.ox, g.oy, g.oz};
  const int n[3] = {g.r.x, g.r.y, g.r.z};
  for (int k = 0; k < 3; ++k) {
    q.inv[k] = 1.0f / h[k];
    q.offF[k] = -(o[k] * q.inv[k]);
    q.offC[k] = q.offF[k] - 0.5f;
    q.jF[k] = n[k];
    q.jC[k] = n[k] - 1;
    q.hiF[k] = std::nextafter((float)(n[k] + 1), 0.0f);
    q.hiC[k] = std::nextafter((float)n[k], 0.0f);
  }
  for (int a = 0; a < 3; ++a) {
    q.lx[a] = (unsigned)(n[0] + (a == 0) + 1);
    q.ly[a] = (unsigned)(n[1] + (a == 1) + 1);
    q.pl[a] = q.lx[a] * q.ly[a];
    q.c[a] = base[a] + (q.pl[a] + q.lx[a] + 1);
  }
  return q;
}

// The corner-table entries of the last sample of each component, kept in
// registers across the RK stages of one substep: a particle moves a fraction
// of a cell per substep, so the next sample mostly falls in the same stencil
// cell, and its two 16-byte loads are not repeated (the values are the same
// ones, the tables do not change during the substeps).
struct QuadCache {
  int e[3];
  float4 lo[3], hi[3];
};

struct FaceSampler {
  AxisW cc[3], fc[3];
  __device__ __forceinline__ FaceSampler(const Geom& g, float px, float py, float pz) {
    float ux = (px - g.ox) * (1.0f / g.hx), uy = (py - g.oy) * (1.0f / g.hy), uz = (pz - g.oz) * (1.0f / g.hz);
    axisWeights(ux - 0.5f, g.r.x, cc[0]);
    axisWeights(uy - 0.5f, g.r.y, cc[1]);
    axisWeights(uz - 0.5f, g.r.z, cc[2]);
    axisWeights(ux, g.r.x + 1, fc[0]);
    axisWeights(uy, g.r.y + 1, fc[1]);
    axisWeights(uz, g.r.z + 1, fc[2]);
  }
  // the same sampler from the constants of a corner-table set: one FMA per
  // coordinate (the two forms round alike up to the last bit), and the
  // coordinate clamped to [-1, n) before the floor (clampedAxis)
  // The same with the integer index clamps of axisWeights (same corners and
  // weights at every finite point): in the G2P kernel, which also forms the
  // corner indices of the FLIP difference, this form is the faster one
  // (1.03 against 1.19 ms per 256^3 step).
  struct IndexClamp {};
  __device__ __forceinline__ FaceSampler(const FaceQuads& q, float px, float py, float pz, IndexClamp) {
    const float p[3] = {px, py, pz};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      axisWeights(fmaf(p[k], q.inv[k], q.offC[k]), q.jC[k] + 1, cc[k]);
      axisWeights(fmaf(p[k], q.inv[k], q.offF[k]), q.jF[k] + 1, fc[k]);
    }
  }
  __device__ __forceinline__ FaceSampler(const FaceQuads& q, float px, float py, float pz) {
    const float p[3] = {px, py, pz};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      clampedAxis(fmaf(p[k], q.inv[k], q.offC[k]), q.hiC[k], q.jC[k], cc[k]);
      clampedAxis(fmaf(p[k], q.inv[k], q.offF[k]), q.hiF[k], q.jF[k], fc[k]);
    }
  }
  // weights and 8 linear indices of component `a` (corner order z, y, x);
  // 32-bit index arithmetic (every grid holds fewer than 2^31 entries)
  __device__ __forceinline__ void corners(const Geom& g, int a, unsigned idx[8], float w[8]) const {
    const AxisW& X = a == 0 ? fc[0] : cc[0];
    const AxisW& Y = a == 1 ? fc[1] : cc[1];
    const AxisW& Z = a == 2 ? fc[2] : cc[2];
    unsigned nx = (unsigned)(g.r.x + (a == 0)), ny = (unsigned)(g.r.y + (a == 1));
    unsigned r0 = (unsigned)Z.i0 * ny, r1 = (unsigned)Z.i1 * ny;
    unsigned b00 = (r0 + Y.i0) * nx, b01 = (r0 + Y.i1) * nx, b10 = (r1 + Y.i0) * nx, b11 = (r1 + Y.i1) * nx;
    idx[0] = b00 + X.i0; idx[1] = b00 + X.i1; idx[2] = b01 + X.i0; idx[3] = b01 + X.i1;
    idx[4] = b10 + X.i0; idx[5] = b10 + X.i1; idx[6] = b11 + X.i0; idx[7] = b11 + X.i1;
    float x0 = 1.f - X.w1, x1 = X.w1, y0 = 1.f - Y.w1, y1 = Y.w1, z0 = 1.f - Z.w1, z1 = Z.w1;
    w[0] = x0 * y0 * z0; w[1] = x1 * y0 * z0; w[2] = x0 * y1 * z0; w[3] = x1 * y1 * z0;
    w[4] = x0 * y0 * z1; w[5] = x1 * y0 * z1; w[6] = x0 * y1 * z1; w[7] = x1 * y1 * z1;
  }
  __device__ __forceinline__ float sample(const Geom& g, int a, const float* __restrict__ f) const {
    unsigned idx[8];
    float w[8];
    corners(g, a, idx, w);
    float v = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) v = fmaf(w[k], __ldg(f + idx[k]), v);
    return v;
  }
  // the same trilinear sample from the corner table of the component: two
  // 16-byte loads instead of eight 4-byte ones, reduced by lerps along x,
  // then y, then z (seven FMAs; rounding differs from the weighted sum in the
  // last bits, and equal corners return their value exactly)
  __device__ __forceinline__ float sampleQuads(const FaceQuads& T, int a) const {
    const AxisW& X = a == 0 ? fc[0] : cc[0];
    const AxisW& Y = a == 1 ? fc[1] : cc[1];
    const AxisW& Z = a == 2 ? fc[2] : cc[2];
    const float4* q = T.c[a] + (Z.j * (int)T.ly[a] + Y.j) * (int)T.lx[a] + X.j;
    const float4 q0 = __ldg(q), q1 = __ldg(q + T.pl[a]);
    const float wx = X.w1, wy = Y.w1, wz = Z.w1;
    const float a00 = fmaf(wx, q0.y, q0.x), a01 = fmaf(wx, q0.w, q0.z);  // .y, .w: the x differences
    const float a10 = fmaf(wx, q1.y, q1.x), a11 = fmaf(wx, q1.w, q1.z);
    const float b0 = fmaf(wy, a01 - a00, a00), b1 = fmaf(wy, a11 - a10, a10);
    return fmaf(wz, b1 - b0, b0);
  }
  // sampleQuads through the cache: the loads only when the entry differs
  // from the cached one (or fresh)
  __device__ __forceinline__ float sampleQuadsCached(const FaceQuads& T, int a, QuadCache& c, bool fresh) const {
    const AxisW& X = a == 0 ? fc[0] : cc[0];
    const AxisW& Y = a == 1 ? fc[1] : cc[1];
    const AxisW& Z = a == 2 ? fc[2] : cc[2];
    const int e = (Z.j * (int)T.ly[a] + Y.j) * (int)T.lx[a] + X.j;
    if (fresh || e != c.e[a]) {
      c.lo[a] = __ldg(T.c[a] + e);
      c.hi[a] = __ldg(T.c[a] + e + T.pl[a]);
      c.e[a] = e;
    }
    const float4 q0 = c.lo[a], q1 = c.hi[a];
    const float wx = X.w1, wy = Y.w1, wz = Z.w1;
    const float a00 = fmaf(wx, q0.y, q0.x), a01 = fmaf(wx, q0.w, q0.z);  // .y, .w: the x differences
    const float a10 = fmaf(wx, q1.y, q1.x), a11 = fmaf(wx, q1.w, q1.z);
    const float b0 = fmaf(wy, a01 - a00, a00), b1 = fmaf(wy, a11 - a10, a10);
    return fmaf(wz, b1 - b0, b0);
  }
  // sample of the difference field f - h at the same point
  __device__ __forceinline__ float sampleDiff(const Geom& g, int a, const float* __restrict__ f,
                                              const float* __restrict__ h) const {
    unsigned idx[8];
    float w[8];
    corners(g, a, idx, w);
    float v = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) v = fmaf(w[k], __fsub_rn(__ldg(f + idx[k]), __ldg(h + idx[k])), v);
    return v;
  }
};

__device__ __forceinline__ void sampleFaceFast(const ConstFaceField& v, const Geom& g, float px, float py, float pz,
                                               float out[3]) {
  FaceSampler s(g, px, py, pz);
#pragma unroll
  for (int a = 0; a < 3; ++a) out[a] = s.sample(g, a, v.c[a]);
}
__device__ __forceinline__ void sampleFaceQuads(const FaceQuads& v, float px, float py, float pz, float out[3]) {
  FaceSampler s(v, px, py, pz);
#pragma unroll
  for (int a = 0; a < 3; ++a) out[a] = s.sampleQuads(v, a);
}
__device__ __forceinline__ void sampleFaceQuadsCached(const FaceQuads& v, float px, float py, float pz, float out[3],
                                                      QuadCache& c, bool fresh) {
  FaceSampler s(v, px, py, pz);
#pragma unroll
  for (int a = 0; a < 3; ++a) out[a] = s.sampleQuadsCached(v, a, c, fresh);
}

// Cubic samplers (MPhysics/EulerMathTool.cu:134-240, FieldMathTool.cu:106-173).
// SAMP follows ESamplingAlgorithm (EnumType.h:3-10): 1 Catmull-Rom,
// 2 monotonic Catmull-Rom, 3 Bridson cubic, 4 Bridson cubic clamped to the
// two middle values.  The Bridson weights carry double literals in the
// reference, so they are formed in FP64 (products of t alone in FP32) and the
// sum is rounded to FP32 once; every operation is written out so that no
// contraction changes the rounding.
__device__ __forceinline__ float cubicBridson1(const float v[4], float t) {
  const double td = (double)t;
  const float t2 = __fmul_rn(t, t), t3 = __fmul_rn(t2, t);
  double c0 = __dsub_rn(__dadd_rn(__dmul_rn(-1.0 / 3.0, td), __dmul_rn(__dmul_rn(0.5, td), td)),
                        __dmul_rn(__dmul_rn(__dmul_rn(1.0 / 6.0, td), td), td));
  double c1 = __dadd_rn(__dsub_rn(1.0, (double)t2), __dmul_rn(0.5, (double)__fsub_rn(t3, t)));
  double c2 = __dadd_rn(td, __dmul_rn(0.5, (double)__fsub_rn(t2, t3)));
  double c3 = __dmul_rn(1.0 / 6.0, (double)__fsub_rn(t3, t));
  double s = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(c0, (double)v[0]), __dmul_rn(c1, (double)v[1])),
                                 __dmul_rn(c2, (double)v[2])),
                       __dmul_rn(c3, (double)v[3]));
  return __double2float_rn(s);
}
__device__ __forceinline__ float catmullRom1(const float v[4], float t, bool monotonic) {
  float d1 = __fdiv_rn(__fsub_rn(v[2], v[0]), 2.f), d2 = __fdiv_rn(__fsub_rn(v[3], v[1]), 2.f);
  const float delta = __fsub_rn(v[2], v[1]);
  if (monotonic) {
    if (fabsf(delta) < FLT_EPSILON) { d1 = 0.f; d2 = 0.f; }
    if (__fmul_rn(delta, d1) < 0.f) d1 = 0.f;
    if (__fmul_rn(delta, d2) < 0.f) d2 = 0.f;
  }
  const float a3 = __fsub_rn(__fadd_rn(d1, d2), __fmul_rn(2.f, delta));
  const float a2 = __fsub_rn(__fsub_rn(__fmul_rn(3.f, delta), __fmul_rn(2.f, d1)), d2);
  float r = __fmul_rn(__fmul_rn(__fmul_rn(a3, t), t), t);
  r = __fadd_rn(r, __fmul_rn(__fmul_rn(a2, t), t));
  r = __fadd_rn(r, __fmul_rn(d1, t));
  return __fadd_rn(r, v[1]);
}
template <int SAMP> __device__ __forceinline__ float cubic1(const float v[4], float t) {
  if (SAMP == 1) return catmullRom1(v, t, false);
  if (SAMP == 2) return catmullRom1(v, t, true);
  if (SAMP == 3) return cubicBridson1(v, t);
  float c = cubicBridson1(v, t);  // clampCUDA (EulerMathTool.cu:121-127)
  return fmaxf(fminf(v[1], v[2]), fminf(c, fmaxf(v[1], v[2])));
}
// 4^3 clamp-to-edge neighbourhood, reduced along x, then y, then z.
template <int SAMP>
__device__ inline float cubicSample(const float* __restrict__ f, const Geom& g, float px, float py, float pz) {
  const float rx = __fsub_rn(__fsub_rn(px, g.ox), __fdiv_rn(g.hx, 2.f));
  const float ry = __fsub_rn(__fsub_rn(py, g.oy), __fdiv_rn(g.hy, 2.f));
  const float rz = __fsub_rn(__fsub_rn(pz, g.oz), __fdiv_rn(g.hz, 2.f));
  const int ix = floorRef(__fdiv_rn(rx, g.hx)), iy = floorRef(__fdiv_rn(ry, g.hy)), iz = floorRef(__fdiv_rn(rz, g.hz));
  const float tx = __fdiv_rn(__fsub_rn(rx, __fmul_rn((float)ix, g.hx)), g.hx);
  const float ty = __fdiv_rn(__fsub_rn(ry, __fmul_rn((float)iy, g.hy)), g.hy);
  const float tz = __fdiv_rn(__fsub_rn(rz, __fmul_rn((float)iz, g.hz)), g.hz);
  int xs[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) xs[k] = clampi(ix + k - 1, g.r.x);
  float vz[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const long long zo = (long long)clampi(iz + i - 1, g.r.z) * g.r.y;
    float vy[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float* row = f + (zo + clampi(iy + j - 1, g.r.y)) * g.r.x;
      const float vx[4] = {__ldg(row + xs[0]), __ldg(row + xs[1]), __ldg(row + xs[2]), __ldg(row + xs[3])};
      vy[j] = cubic1<SAMP>(vx, tx);
    }
    vz[i] = cubic1<SAMP>(vy, ty);
  }
  return cubic1<SAMP>(vz, tz);
}
// trilinear (SAMP 0) or cubic sample of one scalar grid
template <int SAMP>
__device__ __forceinline__ float sampleAlg(const float* __restrict__ f, const Geom& g, float px, float py, float pz) {
  if (SAMP == 0) return trilerp(f, g, px, py, pz);
  return cubicSample<SAMP>(f, g, px, py, pz);
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

__device__ inline unsigned int flatTid() { return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z); }
__device__ inline unsigned int flatBlock() { return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z); }
__device__ inline unsigned int numBlocks() { return gridDim.x * gridDim.y * gridDim.z; }
__device__ inline unsigned int blockThreads() { return blockDim.x * blockDim.y * blockDim.z; }

// Sum two doubles over the block (fixed tree => deterministic).  Result valid
// in thread 0.  Works for 1-D, 2-D and 3-D blocks of a multiple of 32 threads.
__device__ inline void blockSum2(double& a, double& b) {
  __shared__ double sa[32], sb[32];
  unsigned int t = flatTid();
  a = warpSumD(a);
  b = warpSumD(b);
  unsigned int lane = t & 31, w = t >> 5;
  if (lane == 0) { sa[w] = a; sb[w] = b; }
  __syncthreads();
  unsigned int nw = blockThreads() >> 5;
  if (w == 0) {
    a = lane < nw ? sa[lane] : 0.0;
    b = lane < nw ? sb[lane] : 0.0;
    a = warpSumD(a);
    b = warpSumD(b);
  }
  __syncthreads();
}

// Publish this block's two partial sums; returns true in the one block that
// finishes last, after which `a`, `b` (thread 0) hold the grid totals summed
// in a fixed order (independent of block scheduling).
__device__ inline bool gridSum2(double& a, double& b, double* partials, unsigned int* ticket) {
  __shared__ bool isLast;
  blockSum2(a, b);
  unsigned int t = flatTid(), blk = flatBlock(), nb = numBlocks();
  if (t == 0) {
    partials[2 * blk] = a;
    partials[2 * blk + 1] = b;
    __threadfence();
    unsigned int k = atomicAdd(ticket, 1u);
    isLast = (k == nb - 1);
  }
  __syncthreads();
  if (!isLast) return false;
  __threadfence();
  double sa = 0.0, sb = 0.0;
  for (unsigned int i = t; i < nb; i += blockThreads()) {
    sa += __ldcg(partials + 2 * i);
    sb += __ldcg(partials + 2 * i + 1);
  }
  blockSum2(sa, sb);
  a = sa;
  b = sb;
  return true;
}

// Device clock in ns (globaltimer), for bounded waits.
__device__ __forceinline__ unsigned long long globalNs() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned ldAcquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// ---------------------------------------------------------------------------
// mbarrier plumbing of the TMA-fed kernels.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smemAddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbarInit(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbarFenceInit() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbarExpectTx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbarTryWait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smemAddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: false once the deadline has passed (the caller records an
// error and drains what it issued).
__device__ __forceinline__ bool mbarWait(uint64_t* bar, unsigned parity, unsigned long long deadline) {
  while (!mbarTryWait(bar, parity))
    if (globalNs() > deadline) return false;
  return true;
}
// Grid barrier of a cooperative launch (generation counting).  The wait is
// bounded: past the deadline, or once another block has given up, the error
// word is set and false returned, and the caller stops.
__device__ inline bool gridBarrier(unsigned* count, unsigned* gen, unsigned* err, unsigned nblocks) {
  __shared__ int okS;
  __syncthreads();
  if (flatTid() == 0) {
    int ok = 1;
    const unsigned g = ldAcquire(gen);
    __threadfence();  // this block's writes before its arrival
    if (atomicAdd(count, 1u) == nblocks - 1) {
      atomicExch(count, 0u);
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      const unsigned long long deadline = globalNs() + 1000000000ull;  // 1 s
      while (ldAcquire(gen) == g) {
        if (ldAcquire(err) != 0u || globalNs() > deadline) {
          atomicExch(err, 1u);
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    okS = ok;
  }
  __syncthreads();
  return okS != 0;
}

// Asks L2 for the line holding *p ahead of its load (no register is held
// while the line is fetched); p must lie inside an allocation.
__device__ __forceinline__ void prefetchL2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// Programmatic dependent launch.  A kernel launched with launchPdl may start
// while the kernel before it in the stream finishes: waitPrevGrid
// (griddepcontrol.wait) returns once that kernel has completed and its writes
// are visible, and must come before the first read of anything earlier work
// wrote.  allowNextGrid lets the next such kernel be scheduled once every
// block of this one has issued it.
__device__ __forceinline__ void waitPrevGrid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void allowNextGrid() { asm volatile("griddepcontrol.launch_dependents;" :::); }

template <class... KP, class... A>
inline cudaError_t launchPdl(void (*kernel)(KP...), dim3 grid, dim3 block, cudaStream_t s, A&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

}  // namespace hfg
