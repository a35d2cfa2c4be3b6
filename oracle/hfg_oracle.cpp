// hfg_oracle.cpp -- CPU restatement of the reference grid time step.
//
// TEST INFRASTRUCTURE ONLY.  This file is the oracle: a plain C++17 (+OpenMP)
// restatement of junwei-jiang/Hybrid-Fluid-Simulation's CGridFluidSolver step,
// used by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline
// leg as the checker.  The product library never links or calls it.
//
// Every routine below cites the reference file:line it follows (paths are
// relative to the reference project root).  Arithmetic is templated on the
// scalar type T: T=float mirrors the reference's FP32 `Real` operation by
// operation (compiled with -ffp-contract=off, so no FMA contraction), T=double
// is the FP64 oracle used for accuracy statements.
//
// Conventions (MPhysics/Common.h:250, EulerMathTool.cu:63-73):
//   cell-centred linear index  = z*nx*ny + y*nx + x
//   face grids: X (nx+1,ny,nz), Y (nx,ny+1,nz), Z (nx,ny,nz+1), each with the
//   component's origin shifted by -spacing/2 on its own axis
//   (FieldMathTool.cu:800-808)
//   every neighbour / corner index is clamped to the grid (clamp-to-edge).

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

typedef long long i64;

template <class T> struct V3 { T x, y, z; };

struct Res { int x, y, z; i64 size() const { return (i64)x * y * z; } };

template <class T> static inline T unknownv() { return std::numeric_limits<T>::max(); }

// EulerMathTool.cu:16-27 limitIndex (integer clamp-to-edge)
static inline int limitIndex(int i, int n) { return i < 0 ? 0 : (i > n - 1 ? n - 1 : i); }

// EulerMathTool.cu:63-73 transIndex2LinearWithOffset
static inline i64 lin(int x, int y, int z, const Res& r) {
  x = limitIndex(x, r.x); y = limitIndex(y, r.y); z = limitIndex(z, r.z);
  return (i64)z * r.x * r.y + (i64)y * r.x + x;
}

// EulerMathTool.cu:93-103 floorCUDA: note floorCUDA(-1.0) == -2 (quirk kept)
template <class T> static inline int floorCUDA(T v) { return v >= 0 ? (int)v : (int)v - 1; }

// EulerMathTool.cu:129-132
template <class T> static inline bool isInsideSDF(T v) { return v < 0; }

// EulerMathTool.cu:268-294 particle/grid transfer kernels
template <class T> static inline T linearKernelFunc(T o) {
  T a = std::fabs(o);
#ifdef ORC_PLANTED_MISTAKE  // a deliberate error, only in the build that checks the replay catches it
  a = a * (T)1.01;
#endif
  return a < 1 ? (T)1.0 - a : (T)0.0;
}
template <class T> static inline T quadraticKernelFunc(T o) {
  T a = std::fabs(o);
  if (a < (T)0.5) return (T)0.75 - a * a;
  if (a >= (T)0.5 && a < (T)1.5) return (T)0.5 * ((T)1.5 - a) * ((T)1.5 - a);
  return 0;
}
template <class T> static inline T cubicKernelFunc(T o) {
  T a = std::fabs(o);
  if (a < (T)1.0) return (T)0.5 * a * a * a - a * a + (T)(2.0 / 3.0);
  if (a >= (T)1.0 && a < (T)2.0) return (T)(1.0 / 6.0) * ((T)2.0 - a) * ((T)2.0 - a) * ((T)2.0 - a);
  return 0;
}

enum Alg { P2GSUM = 0, G2PNEAREST = 1, LINEAR = 2, QUADRATIC = 3, CUBIC = 4 };  // EnumType.h:19-26

// A scalar grid with its geometry: what CCellCenteredScalarField carries.
template <class T> struct GridGeom {
  Res r; V3<T> o, h;
};

// FaceCenteredVectorField component geometry (FieldMathTool.cu:800-808).
template <class T> static GridGeom<T> faceGeom(const GridGeom<T>& cc, int axis) {
  GridGeom<T> g = cc;
  if (axis == 0) { g.r.x += 1; g.o.x = cc.o.x - cc.h.x / 2; }
  if (axis == 1) { g.r.y += 1; g.o.y = cc.o.y - cc.h.y / 2; }
  if (axis == 2) { g.r.z += 1; g.o.z = cc.o.z - cc.h.z / 2; }
  return g;
}

// FieldMathTool.cu:52-104 sampleCellCenteredScalarFieldTrilerp
template <class T> static inline T trilerp(const T* f, const GridGeom<T>& g, T px, T py, T pz) {
  T rx = px - g.o.x - g.h.x / 2;
  T ry = py - g.o.y - g.h.y / 2;
  T rz = pz - g.o.z - g.h.z / 2;
  int ix = floorCUDA<T>(rx / g.h.x), iy = floorCUDA<T>(ry / g.h.y), iz = floorCUDA<T>(rz / g.h.z);
  T ox = (rx - ((T)ix * g.h.x)) / g.h.x;
  T oy = (ry - ((T)iy * g.h.y)) / g.h.y;
  T oz = (rz - ((T)iz * g.h.z)) / g.h.z;
#ifdef ORC_PLANTED_MISTAKE
  ox = ox * (T)1.01;
#endif
  T UBL = f[lin(ix, iy + 1, iz, g.r)], UBR = f[lin(ix + 1, iy + 1, iz, g.r)];
  T UFL = f[lin(ix, iy + 1, iz + 1, g.r)], UFR = f[lin(ix + 1, iy + 1, iz + 1, g.r)];
  T DBL = f[lin(ix, iy, iz, g.r)], DBR = f[lin(ix + 1, iy, iz, g.r)];
  T DFL = f[lin(ix, iy, iz + 1, g.r)], DFR = f[lin(ix + 1, iy, iz + 1, g.r)];
  return DBL * (1 - ox) * (1 - oy) * (1 - oz) + DBR * ox * (1 - oy) * (1 - oz) +
         UBL * (1 - ox) * oy * (1 - oz) + UBR * ox * oy * (1 - oz) +
         DFL * (1 - ox) * (1 - oy) * oz + DFR * ox * (1 - oy) * oz +
         UFL * (1 - ox) * oy * oz + UFR * ox * oy * oz;
}

// A face-centred vector field (three component arrays) on a cell grid.
template <class T> struct FC {
  std::vector<T> c[3];
  void resize(const Res& r) {
    c[0].assign((i64)(r.x + 1) * r.y * r.z, 0);
    c[1].assign((i64)r.x * (r.y + 1) * r.z, 0);
    c[2].assign((i64)r.x * r.y * (r.z + 1), 0);
  }
};

// FieldMathTool.cu:783-892 sampleFaceCenteredVectorFieldInvoker (trilinear):
// every component is sampled on its own shifted grid.
template <class T> static inline void sampleFC(const FC<T>& v, const GridGeom<T>& cc, T px, T py, T pz, T out[3]) {
  for (int a = 0; a < 3; ++a) out[a] = trilerp(v.c[a].data(), faceGeom(cc, a), px, py, pz);
}

// ---------------------------------------------------------------------------
// Cubic samplers (EulerMathTool.cu:134-240, FieldMathTool.cu:106-173).
// ESamplingAlgorithm order (EnumType.h:3-10): 0 trilinear, 1 Catmull-Rom,
// 2 monotonic Catmull-Rom, 3 Bridson cubic, 4 clamped Bridson cubic.  The
// reference writes the Bridson weights with double literals, so for a float
// Real they are evaluated in double (products of t alone stay in Real) and
// the sum is rounded to Real; Catmull-Rom is all Real.
// ---------------------------------------------------------------------------
template <class T> static inline T cubicBridson1(const T* v, T t) {
  double c0 = -1.0 / 3.0 * (double)t + 1.0 / 2.0 * (double)t * (double)t - 1.0 / 6.0 * (double)t * (double)t * (double)t;
  double c1 = 1.0 - (double)(t * t) + 1.0 / 2.0 * (double)(t * t * t - t);
  double c2 = (double)t + 1.0 / 2.0 * (double)(t * t - t * t * t);
  double c3 = 1.0 / 6.0 * (double)(t * t * t - t);
  return (T)(c0 * (double)v[0] + c1 * (double)v[1] + c2 * (double)v[2] + c3 * (double)v[3]);
}
template <class T> static inline T clampCUDA(T x, T a, T b) {  // EulerMathTool.cu:121-127
  T mx = std::max(a, b), mn = std::min(a, b);
  return std::max(mn, std::min(x, mx));
}
template <class T> static inline T catmullRom1(const T* v, T t, bool monotonic) {
  T d1 = (v[2] - v[0]) / (T)2, d2 = (v[3] - v[1]) / (T)2, delta = v[2] - v[1];
  if (monotonic) {
    const T eps = std::numeric_limits<T>::epsilon();  // EPSILON (MMathExtra.h:43,55)
    if (std::abs(delta) < eps) { d1 = 0; d2 = 0; }
    if (delta * d1 < 0) d1 = 0;
    if (delta * d2 < 0) d2 = 0;
  }
  T a3 = d1 + d2 - (T)2 * delta;
  T a2 = (T)3 * delta - (T)2 * d1 - d2;
  T a1 = d1, a0 = v[1];
  return a3 * t * t * t + a2 * t * t + a1 * t + a0;
}
template <class T> static inline T cubic1(const T* v, T t, int alg) {
  if (alg == 1) return catmullRom1(v, t, false);
  if (alg == 2) return catmullRom1(v, t, true);
  if (alg == 3) return cubicBridson1(v, t);
  return clampCUDA(cubicBridson1(v, t), v[1], v[2]);
}
// sampleCellCenteredScalarFieldCubic (FieldMathTool.cu:106-173): the 4^3
// clamp-to-edge neighbourhood around floor((p - o - h/2) / h), reduced along
// x, then y, then z.
template <class T> static inline T cubicSample(const T* f, const GridGeom<T>& g, T px, T py, T pz, int alg) {
  T rx = px - g.o.x - g.h.x / 2;
  T ry = py - g.o.y - g.h.y / 2;
  T rz = pz - g.o.z - g.h.z / 2;
  int ix = floorCUDA<T>(rx / g.h.x), iy = floorCUDA<T>(ry / g.h.y), iz = floorCUDA<T>(rz / g.h.z);
  T tx = (rx - ((T)ix * g.h.x)) / g.h.x;
  T ty = (ry - ((T)iy * g.h.y)) / g.h.y;
  T tz = (rz - ((T)iz * g.h.z)) / g.h.z;
  T vz[4];
  for (int i = 0; i < 4; ++i) {
    T vy[4];
    for (int j = 0; j < 4; ++j) {
      T vx[4];
      for (int k = 0; k < 4; ++k) vx[k] = f[lin(ix + k - 1, iy + j - 1, iz + i - 1, g.r)];
      vy[j] = cubic1(vx, tx, alg);
    }
    vz[i] = cubic1(vy, ty, alg);
  }
  return cubic1(vz, tz, alg);
}
template <class T> static inline T sampleAlg(const T* f, const GridGeom<T>& g, T px, T py, T pz, int alg) {
  return alg == 0 ? trilerp(f, g, px, py, pz) : cubicSample(f, g, px, py, pz, alg);
}
template <class T>
static inline void sampleFCAlg(const FC<T>& v, const GridGeom<T>& cc, T px, T py, T pz, int alg, T out[3]) {
  for (int a = 0; a < 3; ++a) out[a] = sampleAlg(v.c[a].data(), faceGeom(cc, a), px, py, pz, alg);
}

// ---------------------------------------------------------------------------
// Particle <-> grid transfers (EulerParticlesTool.cu:79-308)
// ---------------------------------------------------------------------------

// EulerMathTool.cu:29-40 transPos2Index (truncation, then clamp)
template <class T> static inline i64 binIndex(const GridGeom<T>& g, T px, T py, T pz) {
  T rx = (px - g.o.x) / g.h.x, ry = (py - g.o.y) / g.h.y, rz = (pz - g.o.z) / g.h.z;
  return lin(limitIndex((int)rx, g.r.x), limitIndex((int)ry, g.r.y), limitIndex((int)rz, g.r.z), g.r);
}

template <class T> struct Stencil {
  int base[3];
  int n;        // 1, 2 or 4 taps per axis
  int shift;    // 0 for linear, -1 for quadratic/cubic
  T w[3][4];
};

// EulerParticlesTool.cu:99-103 + :113-115 / :140-142 / :167-169 weights
template <class T> static inline void stencil(const GridGeom<T>& g, T px, T py, T pz, int alg, Stencil<T>& s) {
  T rel[3] = {px - g.o.x - g.h.x * (T)0.5, py - g.o.y - g.h.y * (T)0.5, pz - g.o.z - g.h.z * (T)0.5};
  T h[3] = {g.h.x, g.h.y, g.h.z};
  for (int a = 0; a < 3; ++a) {
    T ri = rel[a] / h[a];
    int b = floorCUDA<T>(ri);
    T off = (rel[a] - (T)b * h[a]) / h[a];
    s.base[a] = b;
    if (alg == LINEAR) {
      s.w[a][0] = linearKernelFunc<T>(off);
      s.w[a][1] = linearKernelFunc<T>(off - (T)1.0);
    } else if (alg == QUADRATIC) {
      s.w[a][0] = quadraticKernelFunc<T>(off + (T)1.0);
      s.w[a][1] = quadraticKernelFunc<T>(off);
      s.w[a][2] = quadraticKernelFunc<T>(off - (T)1.0);
      s.w[a][3] = quadraticKernelFunc<T>(off - (T)2.0);
    } else if (alg == CUBIC) {
      s.w[a][0] = cubicKernelFunc<T>(off + (T)1.0);
      s.w[a][1] = cubicKernelFunc<T>(off);
      s.w[a][2] = cubicKernelFunc<T>(off - (T)1.0);
      s.w[a][3] = cubicKernelFunc<T>(off - (T)2.0);
    }
  }
  s.n = (alg == LINEAR) ? 2 : 4;
  s.shift = (alg == LINEAR) ? 0 : -1;
}

// EulerParticlesTool.cu:198-288 accumulateCCSField2Particles (one component)
template <class T> static inline T g2pOne(const T* f, const GridGeom<T>& g, T px, T py, T pz, int alg) {
  if (alg == G2PNEAREST) return f[binIndex(g, px, py, pz)];
  if (alg != LINEAR && alg != QUADRATIC && alg != CUBIC) return 0;
  Stencil<T> s;
  stencil(g, px, py, pz, alg, s);
  T acc = 0;
  for (int z = 0; z < s.n; ++z)
    for (int y = 0; y < s.n; ++y)
      for (int x = 0; x < s.n; ++x) {
        T w = s.w[0][x] * s.w[1][y] * s.w[2][z];
        acc += w * f[lin(s.base[0] + x + s.shift, s.base[1] + y + s.shift, s.base[2] + z + s.shift, g.r)];
      }
  return acc;
}

// EulerParticlesTool.cu:79-196 accumulateParticles2CCSField + :290-308
// normalizeCCSField.  Accumulation is sequential in particle order (the
// reference uses unordered float atomics; any order is one of its outcomes).
template <class T>
static void p2gOne(const GridGeom<T>& g, const T* pos, const T* val, int span, int off, i64 P, int alg,
                   std::vector<T>& out, std::vector<T>& wout, bool normalize) {
  std::fill(out.begin(), out.end(), (T)0);
  std::fill(wout.begin(), wout.end(), (T)0);
  for (i64 p = 0; p < P; ++p) {
    T px = pos[3 * p], py = pos[3 * p + 1], pz = pos[3 * p + 2];
    T v = val[span * p + off];
    if (alg == P2GSUM) {
      out[binIndex(g, px, py, pz)] += v;
      continue;
    }
    if (alg != LINEAR && alg != QUADRATIC && alg != CUBIC) continue;
    Stencil<T> s;
    stencil(g, px, py, pz, alg, s);
    for (int z = 0; z < s.n; ++z)
      for (int y = 0; y < s.n; ++y)
        for (int x = 0; x < s.n; ++x) {
          T w = s.w[0][x] * s.w[1][y] * s.w[2][z];
          i64 li = lin(s.base[0] + x + s.shift, s.base[1] + y + s.shift, s.base[2] + z + s.shift, g.r);
          out[li] += w * v;
          wout[li] += w;
        }
  }
  if (normalize)
    for (size_t i = 0; i < out.size(); ++i)
      if (wout[i] > (T)0.0) out[i] /= wout[i];
}

// ---------------------------------------------------------------------------
// Pressure projection (EulerSolverTool.cu, PressureSolver.cpp, CuMatrixFreePCG.cpp)
// ---------------------------------------------------------------------------

// EulerParticlesTool.cu:27-77 + :366-411: truncating binning, then
// 2 = inside solid, 1 = at least one particle, 0 = air.
template <class T>
static void markersFromParticles(const GridGeom<T>& g, const T* solidSDF, const T* pos, i64 P, uint8_t* mk,
                                 uint32_t* counts) {
  i64 N = g.r.size();
  std::vector<uint32_t> cnt(N, 0);
  for (i64 p = 0; p < P; ++p) cnt[binIndex(g, pos[3 * p], pos[3 * p + 1], pos[3 * p + 2])] += 1;
  for (i64 i = 0; i < N; ++i) {
    if (isInsideSDF(solidSDF[i])) mk[i] = 2;
    else mk[i] = cnt[i] > 0 ? 1 : 0;
    if (counts) counts[i] = cnt[i];
  }
}

// EulerSolverTool.cu:30-56 buildFluidMarkers (SDF form)
template <class T> static void markersFromSDF(i64 N, const T* solidSDF, const T* fluidSDF, uint8_t* mk) {
  for (i64 i = 0; i < N; ++i) mk[i] = isInsideSDF(solidSDF[i]) ? 2 : (isInsideSDF(fluidSDF[i]) ? 1 : 0);
}

// EulerSolverTool.cu:58-126 buildPressureMatrixA: [diag, +x, +y, +z] per cell
template <class T> static void buildMatrixA(const Res& r, V3<T> sc, const uint8_t* mk, T* A) {
  for (int z = 0; z < r.z; ++z)
    for (int y = 0; y < r.y; ++y)
      for (int x = 0; x < r.x; ++x) {
        i64 c = lin(x, y, z, r);
        T* a = A + 4 * c;
        a[0] = a[1] = a[2] = a[3] = 0;
        if (mk[c] == 1) {
          uint8_t L = mk[lin(x - 1, y, z, r)], R = mk[lin(x + 1, y, z, r)];
          uint8_t D = mk[lin(x, y - 1, z, r)], U = mk[lin(x, y + 1, z, r)];
          uint8_t B = mk[lin(x, y, z - 1, r)], F = mk[lin(x, y, z + 1, r)];
          if (x > 0 && L != 2) a[0] += sc.x;
          if (x + 1 < r.x && R != 2) { a[0] += sc.x; if (R == 1) a[1] -= sc.x; }
          if (y > 0 && D != 2) a[0] += sc.y;
          if (y + 1 < r.y && U != 2) { a[0] += sc.y; if (U == 1) a[2] -= sc.y; }
          if (z > 0 && B != 2) a[0] += sc.z;
          if (z + 1 < r.z && F != 2) { a[0] += sc.z; if (F == 1) a[3] -= sc.z; }
        } else {
          a[0] = 1.0;
        }
      }
}

// EulerSolverTool.cu:199-227 fdmMatrixVectorMul
template <class T> static void matVec(const Res& r, const T* A, const T* x, T* y) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < r.z; ++z)
    for (int yy = 0; yy < r.y; ++yy)
      for (int xx = 0; xx < r.x; ++xx) {
        i64 c = lin(xx, yy, z, r);
        // the ternaries' `: 0.0` make the reference sum in double (products in T)
        double v = (double)(T)(A[4 * c] * x[c]);
        v += (xx > 0) ? (double)(T)(A[4 * lin(xx - 1, yy, z, r) + 1] * x[lin(xx - 1, yy, z, r)]) : 0.0;
        v += (xx + 1 < r.x) ? (double)(T)(A[4 * c + 1] * x[lin(xx + 1, yy, z, r)]) : 0.0;
        v += (yy > 0) ? (double)(T)(A[4 * lin(xx, yy - 1, z, r) + 2] * x[lin(xx, yy - 1, z, r)]) : 0.0;
        v += (yy + 1 < r.y) ? (double)(T)(A[4 * c + 2] * x[lin(xx, yy + 1, z, r)]) : 0.0;
        v += (z > 0) ? (double)(T)(A[4 * lin(xx, yy, z - 1, r) + 3] * x[lin(xx, yy, z - 1, r)]) : 0.0;
        v += (z + 1 < r.z) ? (double)(T)(A[4 * c + 3] * x[lin(xx, yy, z + 1, r)]) : 0.0;
        y[c] = (T)v;
      }
}

// FieldMathTool.cu:370-395 CUDADivergence (face-centred)
template <class T> static void divergenceFC(const Res& r, V3<T> h, const FC<T>& v, T* div) {
  Res rx{r.x + 1, r.y, r.z}, ry{r.x, r.y + 1, r.z}, rz{r.x, r.y, r.z + 1};
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < r.z; ++z)
    for (int y = 0; y < r.y; ++y)
      for (int x = 0; x < r.x; ++x) {
        T L = v.c[0][lin(x, y, z, rx)], R = v.c[0][lin(x + 1, y, z, rx)];
        T D = v.c[1][lin(x, y, z, ry)], U = v.c[1][lin(x, y + 1, z, ry)];
        T B = v.c[2][lin(x, y, z, rz)], F = v.c[2][lin(x, y, z + 1, rz)];
        div[lin(x, y, z, r)] = (R - L) / h.x + (U - D) / h.y + (F - B) / h.z;
      }
}

// EulerSolverTool.cu:128-197 buildPressureVectorb (scale = 1/spacing, :682)
template <class T>
static void buildRHS(const Res& r, V3<T> h, const FC<T>& v, const FC<T>& sv, const uint8_t* mk, T* b) {
  std::vector<T> div(r.size());
  divergenceFC(r, h, v, div.data());
  V3<T> s{(T)1.0 / h.x, (T)1.0 / h.y, (T)1.0 / h.z};
  Res rx{r.x + 1, r.y, r.z}, ry{r.x, r.y + 1, r.z}, rz{r.x, r.y, r.z + 1};
  for (int z = 0; z < r.z; ++z)
    for (int y = 0; y < r.y; ++y)
      for (int x = 0; x < r.x; ++x) {
        i64 c = lin(x, y, z, r);
        if (mk[c] != 1) { b[c] = 0.0; continue; }
        T val = -div[c];
        i64 uL = lin(x, y, z, rx), uR = lin(x + 1, y, z, rx);
        i64 vD = lin(x, y, z, ry), vU = lin(x, y + 1, z, ry);
        i64 wB = lin(x, y, z, rz), wF = lin(x, y, z + 1, rz);
        if (mk[lin(x - 1, y, z, r)] == 2) val -= s.x * (v.c[0][uL] - sv.c[0][uL]);
        if (mk[lin(x + 1, y, z, r)] == 2) val += s.x * (v.c[0][uR] - sv.c[0][uR]);
        if (mk[lin(x, y - 1, z, r)] == 2) val -= s.y * (v.c[1][vD] - sv.c[1][vD]);
        if (mk[lin(x, y + 1, z, r)] == 2) val += s.y * (v.c[1][vU] - sv.c[1][vU]);
        if (mk[lin(x, y, z - 1, r)] == 2) val -= s.z * (v.c[2][wB] - sv.c[2][wB]);
        if (mk[lin(x, y, z + 1, r)] == 2) val += s.z * (v.c[2][wF] - sv.c[2][wF]);
        b[c] = val;
      }
}

// EulerSolverTool.cu:229-322 applyPressureGradient
template <class T>
static void applyGradient(const Res& r, V3<T> sc, const uint8_t* mk, const T* p, FC<T>& v, const FC<T>& sv) {
  Res rx{r.x + 1, r.y, r.z}, ry{r.x, r.y + 1, r.z}, rz{r.x, r.y, r.z + 1};
  const T U = unknownv<T>();
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < r.z; ++z)
    for (int y = 0; y < r.y; ++y)
      for (int x = 0; x < r.x; ++x) {
        i64 c = lin(x, y, z, r);
        i64 l = lin(x - 1, y, z, r), d = lin(x, y - 1, z, r), bk = lin(x, y, z - 1, r);
        i64 uL = lin(x, y, z, rx), vD = lin(x, y, z, ry), wB = lin(x, y, z, rz);
        if (mk[l] == 1 || mk[c] == 1) {
          if (mk[l] == 2 || mk[c] == 2) v.c[0][uL] = sv.c[0][uL];
          else v.c[0][uL] -= sc.x * (p[c] - p[l]);
        } else v.c[0][uL] = U;
        if (mk[d] == 1 || mk[c] == 1) {
          if (mk[d] == 2 || mk[c] == 2) v.c[1][vD] = sv.c[1][vD];
          else v.c[1][vD] -= sc.y * (p[c] - p[d]);
        } else v.c[1][vD] = U;
        if (mk[bk] == 1 || mk[c] == 1) {
          if (mk[bk] == 2 || mk[c] == 2) v.c[2][wB] = sv.c[2][wB];
          else v.c[2][wB] -= sc.z * (p[c] - p[bk]);
        } else v.c[2][wB] = U;
        if (x == r.x - 1) v.c[0][lin(x + 1, y, z, rx)] = U;
        if (y == r.y - 1) v.c[1][lin(x, y + 1, z, ry)] = U;
        if (z == r.z - 1) v.c[2][lin(x, y, z + 1, rz)] = U;
      }
}

// Dot / norm in the working precision, accumulated in double (the reference
// calls cublasSdot/Snrm2 whose reduction order is unspecified).
template <class T> static double dotp(const std::vector<T>& a, const std::vector<T>& b) {
  double s = 0;
  i64 n = (i64)a.size();
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (i64 i = 0; i < n; ++i) s += (double)a[i] * (double)b[i];
  return s;
}

struct PcgOpts {
  int precond = 0;      // 0 identity (PressureSolver.cpp:12-15), 1 Jacobi (diag of A)
  int tolMode = 0;      // 0: reference rule sqrt(||r||) < tol (CuMatrixFreePCG.cpp:28,51)
                        // 1: relative ||r|| / ||b|| < tol
  double tol = 1e-3;    // CuMatrixFreePCG.h:28
  i64 maxIter = -1;     // -1: N iterations (PressureSolver.cpp:82)
};

// CuMatrixFreePCG.cpp:22-65 solvePCGInvDia, with x0 = 0 (PressureSolver.cpp:147).
// Returns the number of iterations taken and the final ||r||_2.
template <class T>
static i64 pcgSolve(const Res& r, const T* A, const std::vector<T>& b, std::vector<T>& x, const PcgOpts& o,
                    double* residOut, double* bnormOut) {
  i64 N = r.size();
  x.assign(N, 0);
  std::vector<T> R(b), Z(N), Pv(N), AP(N);
  const T eps = std::numeric_limits<float>::epsilon();  // plusAlphaX skip (CuDenseVector.cpp:178)
  double bnorm = std::sqrt(dotp(b, b));
  if (bnormOut) *bnormOut = bnorm;
  auto stop = [&](double rn) {
    if (o.tolMode == 0) return std::sqrt(rn) < o.tol;
    return bnorm == 0.0 || rn / bnorm < o.tol;
  };
  auto precond = [&](const std::vector<T>& in, std::vector<T>& out) {
    if (o.precond == 1) {
      for (i64 i = 0; i < N; ++i) out[i] = in[i] / A[4 * i];
    } else {
      out = in;
    }
  };
  double rn = std::sqrt(dotp(R, R));
  if (residOut) *residOut = rn;
  if (stop(rn)) { std::fill(x.begin(), x.end(), (T)0); return 0; }
  // r = -(A x) + b with x = 0 -> r = b
  precond(R, Z);
  Pv = Z;
  i64 maxIt = o.maxIter < 0 ? N : o.maxIter;
  i64 it = 0;
  for (i64 i = 0; i < maxIt; ++i) {
    double rz = dotp(R, Z);
    matVec(r, A, Pv.data(), AP.data());
    double pAp = dotp(Pv, AP);
    T alpha = (T)(rz / pAp);
    it = i + 1;
    if (!(std::fabs(alpha) < eps)) {
#pragma omp parallel for schedule(static)
      for (i64 k = 0; k < N; ++k) { x[k] += alpha * Pv[k]; R[k] += (-alpha) * AP[k]; }
    }
    rn = std::sqrt(dotp(R, R));
    if (residOut) *residOut = rn;
    if (stop(rn)) break;
    precond(R, Z);
    double rz2 = dotp(R, Z);
    T beta = (T)(rz2 / rz);
#pragma omp parallel for schedule(static)
    for (i64 k = 0; k < N; ++k) { Pv[k] = Pv[k] * beta; Pv[k] = Pv[k] + Z[k]; }
  }
  return it;
}

// ---------------------------------------------------------------------------
// Velocity extrapolation (EulerSolverTool.cu:450-557, :904-969)
// ---------------------------------------------------------------------------

// Layer 0 marks known values 0 and UNKNOWN values UNKNOWN; layer d marks an
// UNKNOWN entry d when a clamped 6-neighbour carries d-1 (buildExtrapolation
// Markers); then, for d = 1..nums-1, an entry of layer d becomes the plain mean
// of its neighbours with a smaller layer, summed in the fixed order
// left, right, down, up, back, front (extrapolatingData).  Restated with
// frontier lists: each layer only visits neighbours of the previous layer,
// which yields the same layers as the reference's full-grid sweeps.
template <class T> static void extrapolate(const Res& r, T* f, int nums, std::vector<T>* markersOut = nullptr) {
  i64 N = r.size();
  const T U = unknownv<T>();
  std::vector<T> mk(N);
  std::vector<i64> cur, nxt;
  for (i64 i = 0; i < N; ++i) {
    if (f[i] == U) mk[i] = U;
    else { mk[i] = 0; cur.push_back(i); }
  }
  std::vector<std::vector<i64>> layers;
  layers.push_back(cur);
  const int dx[6] = {-1, 1, 0, 0, 0, 0}, dy[6] = {0, 0, -1, 1, 0, 0}, dz[6] = {0, 0, 0, 0, -1, 1};
  for (int d = 1; d < nums; ++d) {
    nxt.clear();
    for (i64 c : layers.back()) {
      int x = (int)(c % r.x), y = (int)((c / r.x) % r.y), z = (int)(c / ((i64)r.x * r.y));
      for (int k = 0; k < 6; ++k) {
        i64 n = lin(x + dx[k], y + dy[k], z + dz[k], r);
        if (mk[n] == U) { mk[n] = (T)d; nxt.push_back(n); }
      }
    }
    if (nxt.empty()) break;
    layers.push_back(nxt);
  }
  for (size_t d = 1; d < layers.size(); ++d) {
    T dv = (T)d;
    for (i64 c : layers[d]) {
      int x = (int)(c % r.x), y = (int)((c / r.x) % r.y), z = (int)(c / ((i64)r.x * r.y));
      T acc = 0.0, cnt = 0.0;
      for (int k = 0; k < 6; ++k) {
        i64 n = lin(x + dx[k], y + dy[k], z + dz[k], r);
        if (mk[n] < dv) { acc += f[n]; cnt += (T)1.0; }
      }
      if (cnt != (T)0.0) acc /= cnt;
      f[c] = acc;
    }
  }
  if (markersOut) *markersOut = mk;
}

// ---------------------------------------------------------------------------
// Particles: CFL-substepped advection (EulerParticles.cpp:231-325) and the
// box clamp (EulerParticlesTool.cu:310-333, launched over N cells: :870-888).
// ---------------------------------------------------------------------------
template <class T>
static int advectParticles(const GridGeom<T>& cc, const FC<T>& vel, std::vector<T>& pos, T dt, T cfl, int acc,
                           int clampMode) {
  i64 P = (i64)pos.size() / 3;
  std::vector<T> v0(3 * P), v1(3 * P), v2(3 * P), mid(3 * P), tf(3 * P);
  T sub = 0.0;
  bool done = false;
  T minH = std::min(std::min(cc.h.x, cc.h.y), cc.h.z);
  int nsub = 0;
  while (!done) {
    T dsub = 0.0;
#pragma omp parallel for schedule(static)
    for (i64 p = 0; p < P; ++p) sampleFC(vel, cc, pos[3 * p], pos[3 * p + 1], pos[3 * p + 2], &v0[3 * p]);
    T amax = 0;
    for (i64 i = 0; i < 3 * P; ++i) amax = std::max(amax, (T)std::fabs(v0[i]));
    if (amax != (T)0.0) dsub = cfl * minH / amax;
    else dsub = dt;
    if (sub + dsub >= dt) { dsub = dt - sub; done = true; }
    else if (sub + 2 * dsub >= dt) { dsub = (T)(0.5 * (double)(dt - sub)); }
    if (acc == 0) {
      for (i64 i = 0; i < 3 * P; ++i) pos[i] = dsub * v0[i] + pos[i];
    } else if (acc == 1) {
      T half = (T)(0.5 * (double)dsub);
#pragma omp parallel for schedule(static)
      for (i64 p = 0; p < P; ++p) {
        for (int a = 0; a < 3; ++a) mid[3 * p + a] = half * v0[3 * p + a] + pos[3 * p + a];
        sampleFC(vel, cc, mid[3 * p], mid[3 * p + 1], mid[3 * p + 2], &v1[3 * p]);
        for (int a = 0; a < 3; ++a) pos[3 * p + a] = dsub * v1[3 * p + a] + pos[3 * p + a];
      }
    } else {
      T half = (T)(0.5 * (double)dsub), tq = (T)(0.75 * (double)dsub);
      T a29 = (T)(2.0 / 9.0 * (double)dsub), a39 = (T)(3.0 / 9.0 * (double)dsub), a49 = (T)(4.0 / 9.0 * (double)dsub);
#pragma omp parallel for schedule(static)
      for (i64 p = 0; p < P; ++p) {
        for (int a = 0; a < 3; ++a) mid[3 * p + a] = half * v0[3 * p + a] + pos[3 * p + a];
        sampleFC(vel, cc, mid[3 * p], mid[3 * p + 1], mid[3 * p + 2], &v1[3 * p]);
        for (int a = 0; a < 3; ++a) tf[3 * p + a] = tq * v1[3 * p + a] + pos[3 * p + a];
        sampleFC(vel, cc, tf[3 * p], tf[3 * p + 1], tf[3 * p + 2], &v2[3 * p]);
        for (int a = 0; a < 3; ++a) {
          T q = pos[3 * p + a];
          q = a29 * v0[3 * p + a] + q;
          q = a39 * v1[3 * p + a] + q;
          q = a49 * v2[3 * p + a] + q;
          pos[3 * p + a] = q;
        }
      }
    }
    sub += dsub;
    ++nsub;
  }
  // fixParticlesPosWithBoundarys: clampMode 0 = all particles,
  // 1 = the reference launch shape (the first min(N, P) particles),
  // 2 = none (EulerParticles.cpp:319-322: no boundary SDF of the grid's size).
  i64 nclamp = P;
  if (clampMode == 1) nclamp = std::min<i64>(P, cc.r.size());
  if (clampMode == 2) nclamp = 0;
  T mn[3] = {cc.o.x, cc.o.y, cc.o.z};
  T mx[3] = {cc.o.x + (T)cc.r.x * cc.h.x, cc.o.y + (T)cc.r.y * cc.h.y, cc.o.z + (T)cc.r.z * cc.h.z};
  for (i64 p = 0; p < nclamp; ++p)
    for (int a = 0; a < 3; ++a) {
      T v = pos[3 * p + a];
      pos[3 * p + a] = std::max(mn[a], std::min(v, mx[a]));
    }
  return nsub;
}

// ---------------------------------------------------------------------------
// Semi-Lagrangian back-trace (SemiLagrangian.cpp:23-133, :188-347)
// ---------------------------------------------------------------------------
template <class T> static inline void axpy3(T a, const T v[3], T p[3]) {
  if (std::fabs(a) < std::numeric_limits<float>::epsilon()) return;  // plusAlphaX skip
  for (int k = 0; k < 3; ++k) p[k] = a * v[k] + p[k];
}

template <class T>
static inline void backTrace(const FC<T>& vel, const GridGeom<T>& cc, T dt, int acc, const T in[3], T out[3],
                             int samp = 0) {
  T v0[3], v1[3], v2[3], mid[3], tf[3];
  out[0] = in[0]; out[1] = in[1]; out[2] = in[2];
  auto sampleFC = [&](const FC<T>& v, const GridGeom<T>& g, T x, T y, T z, T o[3]) { sampleFCAlg(v, g, x, y, z, samp, o); };
  sampleFC(vel, cc, in[0], in[1], in[2], v0);
  if (acc == 0) {
    axpy3(-dt, v0, out);
  } else if (acc == 1) {
    mid[0] = in[0]; mid[1] = in[1]; mid[2] = in[2];
    axpy3((T)(-0.5) * dt, v0, mid);
    sampleFC(vel, cc, mid[0], mid[1], mid[2], v1);
    axpy3(-dt, v1, out);
  } else {
    mid[0] = in[0]; mid[1] = in[1]; mid[2] = in[2];
    axpy3((T)(-0.5) * dt, v0, mid);
    sampleFC(vel, cc, mid[0], mid[1], mid[2], v1);
    tf[0] = in[0]; tf[1] = in[1]; tf[2] = in[2];
    axpy3((T)(-0.75) * dt, v1, tf);
    sampleFC(vel, cc, tf[0], tf[1], tf[2], v2);
    axpy3(-(T)(2.0 / 9.0) * dt, v0, out);
    axpy3(-(T)(3.0 / 9.0) * dt, v1, out);
    axpy3(-(T)(4.0 / 9.0) * dt, v2, out);
  }
}

// Sample points of SemiLagrangian.cpp:47-97 (cell centres / face centres).
template <class T> static inline void ccPoint(const GridGeom<T>& g, int x, int y, int z, T p[3]) {
  p[0] = ((T)x + (T)0.5) * g.h.x + g.o.x;
  p[1] = ((T)y + (T)0.5) * g.h.y + g.o.y;
  p[2] = ((T)z + (T)0.5) * g.h.z + g.o.z;
}
template <class T> static inline void fcPoint(const GridGeom<T>& g, int axis, int x, int y, int z, T p[3]) {
  ccPoint(g, x, y, z, p);
  if (axis == 0) p[0] = (T)x * g.h.x + g.o.x;
  if (axis == 1) p[1] = (T)y * g.h.y + g.o.y;
  if (axis == 2) p[2] = (T)z * g.h.z + g.o.z;
}

// CSemiLagrangian::advect (FC) SemiLagrangian.cpp:169-186
template <class T>
static void slAdvectFC(const GridGeom<T>& cc, const FC<T>& in, const FC<T>& vel, T dt, int acc, FC<T>& out,
                       int samp = 0) {
  for (int a = 0; a < 3; ++a) {
    GridGeom<T> fg = faceGeom(cc, a);
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < fg.r.z; ++z)
      for (int y = 0; y < fg.r.y; ++y)
        for (int x = 0; x < fg.r.x; ++x) {
          T p[3], q[3];
          fcPoint(cc, a, x, y, z, p);
          backTrace(vel, cc, dt, acc, p, q, samp);
          out.c[a][lin(x, y, z, fg.r)] = sampleAlg(in.c[a].data(), fg, q[0], q[1], q[2], samp);
        }
  }
}

// CSemiLagrangian::advect (CC scalar / vector) SemiLagrangian.cpp:135-167
template <class T>
static void slAdvectCC(const GridGeom<T>& cc, const std::vector<const T*>& in, const FC<T>& vel, T dt, int acc,
                       const std::vector<T*>& out, int samp = 0) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < cc.r.z; ++z)
    for (int y = 0; y < cc.r.y; ++y)
      for (int x = 0; x < cc.r.x; ++x) {
        T p[3], q[3];
        ccPoint(cc, x, y, z, p);
        backTrace(vel, cc, dt, acc, p, q, samp);
        for (size_t k = 0; k < in.size(); ++k) out[k][lin(x, y, z, cc.r)] = sampleAlg(in[k], cc, q[0], q[1], q[2], samp);
      }
}

// ---------------------------------------------------------------------------
// Solid boundaries (Boundary.cpp:115-150, BoundaryTool.cu:3-113)
// ---------------------------------------------------------------------------
template <class T> struct Boundary {
  std::vector<T> sdf0, sdf;  // original and current (resampled) SDF
  V3<T> vel{0, 0, 0}, trans{0, 0, 0};
};

// Philox4x32-10 (Salmon et al., "Parallel random numbers: as easy as 1, 2, 3",
// SC'11): the counter-based generator the particle seeding uses, so that host
// and device streams match.  Restated here independently of the library.
static inline void philox4x32_10(uint32_t ctr[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * ctr[0];
    uint64_t p1 = (uint64_t)0xCD9E8D57u * ctr[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ ctr[1] ^ k0, n2 = hi0 ^ ctr[3] ^ k1;
    ctr[0] = n0; ctr[1] = lo1; ctr[2] = n2; ctr[3] = lo0;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
}
static inline float u01(uint32_t v) { return (float)(v >> 8) * (1.0f / 16777216.0f); }

// ---------------------------------------------------------------------------
// The solver (GridFluidSolver.cpp:161-537)
// ---------------------------------------------------------------------------
enum AdvKind { ADV_SL = 0, ADV_PIC = 1, ADV_FLIP = 2, ADV_MIX = 3 };

template <class T> struct Solver {
  GridGeom<T> g;
  T dt = 0, time = 0;
  bool bufferFlag = true;
  int extrapNums = 1000;  // GridFluidSolver.cpp:176
  std::vector<Boundary<T>> bnd;
  std::vector<T> totalSDF;  // -(first solid index) inside, UNKNOWN outside; 0 with no solids
  FC<T> solidVel;
  std::vector<T> color1[3], color2[3], dom1, dom2;
  FC<T> vel1, vel2;
  V3<T> ext{0, 0, 0};
  V3<T> gravity{0, (T)-9.8, 0};  // ExternalForcesSolver.h:25
  // advection
  int adv = ADV_SL, acc = 2, alg = LINEAR, clampMode = 1;
  int sampling = 0;  // ESamplingAlgorithm of the semi-Lagrangian samples (AdvectionSolver.h:50)
  T cfl = 1, mixing = 0.1f;
  bool sFlag = false, vFlag = false, velFlag = false;
  std::vector<T> ppos, pvel, pscalar, pvector;
  FC<T> deltaGrid;
  bool advectScalars = true;
  // pressure
  std::vector<uint8_t> markers;
  std::vector<T> px, pb;
  PcgOpts pcg;
  i64 lastIters = 0;
  double lastResid = 0, lastBnorm = 0;
  T rho = 1.0;  // PressureSolver.h:61
  int lastSubsteps = 0;

  void create(T dt_, Res r, V3<T> o, V3<T> h) {
    dt = dt_; g.r = r; g.o = o; g.h = h;
    i64 N = r.size();
    totalSDF.assign(N, 0);
    solidVel.resize(r);
    for (int a = 0; a < 3; ++a) { color1[a].assign(N, 0); color2[a].assign(N, 0); }
    dom1.assign(N, 0); dom2.assign(N, 0);
    vel1.resize(r); vel2.resize(r);
    markers.assign(N, 0);
    px.assign(N, 0); pb.assign(N, 0);
    pcg = PcgOpts();
  }
  FC<T>& velCur() { return bufferFlag ? vel2 : vel1; }
  FC<T>& velOut() { return bufferFlag ? vel1 : vel2; }

  // Boundary.cpp:115-150
  void updateBoundarys() {
    i64 N = g.r.size();
    for (auto& b : bnd) {
      // Boundary.cpp:124-127: translation += (-dt) * velocity (cuBLAS axpy)
      b.trans.x = (-dt) * b.vel.x + b.trans.x;
      b.trans.y = (-dt) * b.vel.y + b.trans.y;
      b.trans.z = (-dt) * b.vel.z + b.trans.z;
#pragma omp parallel for collapse(2) schedule(static)
      for (int z = 0; z < g.r.z; ++z)
        for (int y = 0; y < g.r.y; ++y)
          for (int x = 0; x < g.r.x; ++x) {
            // BoundaryTool.cu:105-112 transformField
            T cx = g.o.x + (T)0.5 * g.h.x + g.h.x * (T)x;
            T cy = g.o.y + (T)0.5 * g.h.y + g.h.y * (T)y;
            T cz = g.o.z + (T)0.5 * g.h.z + g.h.z * (T)z;
            cx = cx + b.trans.x; cy = cy + b.trans.y; cz = cz + b.trans.z;
            b.sdf[lin(x, y, z, g.r)] = trilerp(b.sdf0.data(), g, cx, cy, cz);
          }
    }
    // BoundaryTool.cu:3-26 + :115-144 buildSolidsMarker
    std::fill(totalSDF.begin(), totalSDF.end(), (T)0);
    for (size_t i = 0; i < bnd.size(); ++i) {
      int idx = (int)i + 1;
      for (i64 c = 0; c < N; ++c) {
        if (idx == 1) totalSDF[c] = unknownv<T>();
        if (isInsideSDF(bnd[i].sdf[c]) && totalSDF[c] == unknownv<T>()) totalSDF[c] = (T)(-idx);
      }
    }
    // BoundaryTool.cu:28-83 buildSolidsVel: the six faces of a solid cell take
    // that solid's velocity.  Where two different solids share a face the
    // reference races (atomicExch); here the cell with the larger linear index
    // wins (cells visited in increasing order).
    for (int a = 0; a < 3; ++a) std::fill(solidVel.c[a].begin(), solidVel.c[a].end(), (T)0);
    Res rx{g.r.x + 1, g.r.y, g.r.z}, ry{g.r.x, g.r.y + 1, g.r.z}, rz{g.r.x, g.r.y, g.r.z + 1};
    for (int z = 0; z < g.r.z; ++z)
      for (int y = 0; y < g.r.y; ++y)
        for (int x = 0; x < g.r.x; ++x) {
          T m = totalSDF[lin(x, y, z, g.r)];
          if (!(m < 0)) continue;
          int si = -(1 + (int)m);
          if (si >= (int)bnd.size()) continue;
          V3<T> bv = bnd[si].vel;
          solidVel.c[0][lin(x, y, z, rx)] = bv.x; solidVel.c[0][lin(x + 1, y, z, rx)] = bv.x;
          solidVel.c[1][lin(x, y, z, ry)] = bv.y; solidVel.c[1][lin(x, y + 1, z, ry)] = bv.y;
          solidVel.c[2][lin(x, y, z, rz)] = bv.z; solidVel.c[2][lin(x, y, z + 1, rz)] = bv.z;
        }
  }

  // ExternalForcesSolver.cpp:50-58 (unit-field axpy on every face)
  void applyForces(FC<T>& v) {
    T gv[3] = {gravity.x * dt, gravity.y * dt, gravity.z * dt};
    T ev[3] = {ext.x * dt, ext.y * dt, ext.z * dt};
    const T e = std::numeric_limits<float>::epsilon();
    for (T* a : {gv, ev}) {
      if (std::fabs(a[0]) < e && std::fabs(a[1]) < e && std::fabs(a[2]) < e) continue;
      for (int k = 0; k < 3; ++k)
        for (auto& q : v.c[k]) q = a[k] * (T)1 + q;
    }
  }

  void g2pFC(const FC<T>& f, std::vector<T>& out) {
    i64 P = (i64)ppos.size() / 3;
    out.assign(3 * P, 0);
    for (int a = 0; a < 3; ++a) {
      GridGeom<T> fg = faceGeom(g, a);
#pragma omp parallel for schedule(static)
      for (i64 p = 0; p < P; ++p) out[3 * p + a] = g2pOne(f.c[a].data(), fg, ppos[3 * p], ppos[3 * p + 1], ppos[3 * p + 2], alg);
    }
  }
  void p2gFC(const std::vector<T>& val, FC<T>& out) {
    i64 P = (i64)ppos.size() / 3;
    for (int a = 0; a < 3; ++a) {
      GridGeom<T> fg = faceGeom(g, a);
      std::vector<T> w(out.c[a].size());
      p2gOne(fg, ppos.data(), val.data(), 3, a, P, alg, out.c[a], w, true);
    }
  }

  // GridFluidSolver.cpp:399-416 + the advection solvers
  void computeAdvection() {
    FC<T>& vin = velCur();
    FC<T>& vout = velOut();
    std::vector<T>* cIn = bufferFlag ? color2 : color1;
    std::vector<T>* cOut = bufferFlag ? color1 : color2;
    std::vector<T>& dIn = bufferFlag ? dom2 : dom1;
    std::vector<T>& dOut = bufferFlag ? dom1 : dom2;
    i64 N = g.r.size();
    if (adv == ADV_SL) {
      // SemiLagrangian.cpp:135-186
      slAdvectFC(g, vin, vin, dt, acc, vout, sampling);
      if (advectScalars) {
        slAdvectCC<T>(g, {cIn[0].data(), cIn[1].data(), cIn[2].data(), dIn.data()}, vin, dt, acc,
                      {cOut[0].data(), cOut[1].data(), cOut[2].data(), dOut.data()}, sampling);
      }
      return;
    }
    i64 P = (i64)ppos.size() / 3;
    std::vector<T> pic;
    if (adv == ADV_PIC) {
      // ParticleInCell.cpp:93-108
      g2pFC(vin, pvel);
    } else {
      // FluidImplicitParticle.cpp:98-127 / MixPICAndFLIP.cpp:102-136
      if (adv == ADV_MIX) g2pFC(vin, pic);
      if (!velFlag) {
        deltaGrid = vin;
        velFlag = true;
      } else {
        for (int a = 0; a < 3; ++a)
          for (size_t i = 0; i < vin.c[a].size(); ++i) {
            T q = (T)(-1.0) * vin.c[a][i] + deltaGrid.c[a][i];
            deltaGrid.c[a][i] = q * (T)(-1.0);
          }
      }
      std::vector<T> dp;
      g2pFC(deltaGrid, dp);
      for (i64 i = 0; i < 3 * P; ++i) pvel[i] = (T)1.0 * dp[i] + pvel[i];
      if (adv == ADV_MIX) {
        T s = (T)(1.0 - (double)mixing);
        for (i64 i = 0; i < 3 * P; ++i) pvel[i] = pvel[i] * s;
        for (i64 i = 0; i < 3 * P; ++i) pvel[i] = mixing * pic[i] + pvel[i];
      }
    }
    lastSubsteps = advectParticles(g, vin, ppos, dt, cfl, acc, clampMode);
    p2gFC(pvel, vout);
    if (adv != ADV_PIC) deltaGrid = vout;
    if (advectScalars) {
      // colour: CC vector (MixPICAndFLIP.cpp:83-100); domain: CC scalar (:64-81)
      if (!vFlag) {
        pvector.assign(3 * P, 0);
        for (int a = 0; a < 3; ++a)
          for (i64 p = 0; p < P; ++p)
            pvector[3 * p + a] = g2pOne(cIn[a].data(), g, ppos[3 * p], ppos[3 * p + 1], ppos[3 * p + 2], alg);
        vFlag = true;
      }
      for (int a = 0; a < 3; ++a) {
        std::vector<T> w(N);
        p2gOne(g, ppos.data(), pvector.data(), 3, a, P, alg, cOut[a], w, true);
      }
      if (!sFlag) {
        pscalar.assign(P, 0);
        for (i64 p = 0; p < P; ++p) pscalar[p] = g2pOne(dIn.data(), g, ppos[3 * p], ppos[3 * p + 1], ppos[3 * p + 2], alg);
        sFlag = true;
      }
      std::vector<T> w(N);
      p2gOne(g, ppos.data(), pscalar.data(), 1, 0, P, alg, dOut, w, true);
    }
  }

  // GridFluidSolver.cpp:435-525 + PressureSolver.cpp:154-233
  void computePressure() {
    FC<T>& v = velOut();
    i64 N = g.r.size();
    if (adv == ADV_SL) {
      std::vector<T>& dOut = bufferFlag ? dom1 : dom2;
      markersFromSDF(N, totalSDF.data(), dOut.data(), markers.data());
    } else {
      markersFromParticles(g, totalSDF.data(), ppos.data(), (i64)ppos.size() / 3, markers.data(), nullptr);
    }
    V3<T> sA{dt / (rho * g.h.x * g.h.x), dt / (rho * g.h.y * g.h.y), dt / (rho * g.h.z * g.h.z)};
    std::vector<T> A(4 * N);
    buildMatrixA(g.r, sA, markers.data(), A.data());
    buildRHS(g.r, g.h, v, solidVel, markers.data(), pb.data());
    lastIters = pcgSolve(g.r, A.data(), pb, px, pcg, &lastResid, &lastBnorm);
    V3<T> sG{dt / (rho * g.h.x), dt / (rho * g.h.y), dt / (rho * g.h.z)};
    applyGradient(g.r, sG, markers.data(), px.data(), v, solidVel);
  }

  void extrapolateVel() {
    FC<T>& v = velOut();
    Res rx{g.r.x + 1, g.r.y, g.r.z}, ry{g.r.x, g.r.y + 1, g.r.z}, rz{g.r.x, g.r.y, g.r.z + 1};
    extrapolate(rx, v.c[0].data(), extrapNums);
    extrapolate(ry, v.c[1].data(), extrapNums);
    extrapolate(rz, v.c[2].data(), extrapNums);
  }

  void updateWithoutPressure() {
    updateBoundarys();
    computeAdvection();
    applyForces(velOut());
  }
  void solvePressure() {
    computePressure();
    extrapolateVel();
    bufferFlag = !bufferFlag;
    time += dt;
  }
  void update() { updateWithoutPressure(); solvePressure(); }
};

}  // namespace orc

// ===========================================================================
// C ABI for the test harness (ctypes).  All buffers are caller-owned host
// arrays of float unless stated; `dbl` selects the FP64 (1) or FP32 (0) oracle.
// ===========================================================================
using namespace orc;

namespace {
template <class T> Res mkRes(const int* r) { return Res{r[0], r[1], r[2]}; }
template <class T> GridGeom<T> mkGeom(const int* r, const float* o, const float* h) {
  GridGeom<T> g;
  g.r = Res{r[0], r[1], r[2]};
  g.o = V3<T>{(T)o[0], (T)o[1], (T)o[2]};
  g.h = V3<T>{(T)h[0], (T)h[1], (T)h[2]};
  return g;
}
template <class T> std::vector<T> up(const float* p, i64 n) {
  std::vector<T> v(n);
  for (i64 i = 0; i < n; ++i) v[i] = (T)p[i];
  return v;
}
// FLT_MAX-preserving down-conversion (UNKNOWN in FP64 is DBL_MAX).
template <class T> void down(const std::vector<T>& v, float* p) {
  for (size_t i = 0; i < v.size(); ++i) p[i] = (v[i] == unknownv<T>()) ? FLT_MAX : (float)v[i];
}
template <class T> FC<T> upFC(const Res& r, const float* x, const float* y, const float* z) {
  FC<T> f;
  f.resize(r);
  const float* s[3] = {x, y, z};
  for (int a = 0; a < 3; ++a)
    for (size_t i = 0; i < f.c[a].size(); ++i) f.c[a][i] = (s[a][i] == FLT_MAX) ? unknownv<T>() : (T)s[a][i];
  return f;
}
template <class T> void downFC(const FC<T>& f, float* x, float* y, float* z) {
  down(f.c[0], x); down(f.c[1], y); down(f.c[2], z);
}
}  // namespace

extern "C" {

int orc_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// Philox4x32-10 block for (counter, key); used to check the seeding stream.
void orc_philox(const uint32_t* ctr_in, uint32_t k0, uint32_t k1, uint32_t* out) {
  uint32_t c[4] = {ctr_in[0], ctr_in[1], ctr_in[2], ctr_in[3]};
  philox4x32_10(c, k0, k1);
  for (int i = 0; i < 4; ++i) out[i] = c[i];
}

// EulerParticles.cpp:140-179 with the counter-based stream replacing rand():
// particle k of the f-th fluid cell (cells in linear order) sits at
// (x + u) * h + o with u from Philox(counter = {cell, cell>>32, k, 0}, key = seed).
long long orc_seed_particles(const int* res, const float* o, const float* h, const float* fluidSDF,
                             const float* solidSDF, int ppc, unsigned long long seed, float* posOut) {
  Res r{res[0], res[1], res[2]};
  long long n = 0;
  for (int z = 0; z < r.z; ++z)
    for (int y = 0; y < r.y; ++y)
      for (int x = 0; x < r.x; ++x) {
        i64 c = lin(x, y, z, r);
        if (!(fluidSDF[c] < 0 && !(solidSDF[c] < 0))) continue;
        for (int k = 0; k < ppc; ++k) {
          if (posOut) {
            uint32_t ctr[4] = {(uint32_t)c, (uint32_t)((uint64_t)c >> 32), (uint32_t)k, 0u};
            philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32));
            float* q = posOut + 3 * n;
            q[0] = ((float)x + u01(ctr[0])) * h[0] + o[0];
            q[1] = ((float)y + u01(ctr[1])) * h[1] + o[1];
            q[2] = ((float)z + u01(ctr[2])) * h[2] + o[2];
          }
          ++n;
        }
      }
  return n;
}

// EulerSolverTool.cu:324-406 buildFluidSDF, driven as buildFluidSDFInvoker
// (:760-785): `layers` full-grid sweeps; layer d only reads values written by
// layer d-1 (the reference's in-launch reads see either the old or the new
// value of a cell, and a new value never equals the tested one).
void orc_build_fluid_sdf(const int* res, const float* dom, int layers, float* sdf) {
  Res r{res[0], res[1], res[2]};
  const double FS = 0.2;  // FluidSurfaceDensity (Common.h:244)
  const float U = FLT_MAX;
  i64 N = r.size();
  auto inside = [&](i64 c) { return dom[c] < 0; };
  const int dx[6] = {-1, 1, 0, 0, 0, 0}, dy[6] = {0, 0, -1, 1, 0, 0}, dz[6] = {0, 0, 0, 0, -1, 1};
  for (int z = 0; z < r.z; ++z)
    for (int y = 0; y < r.y; ++y)
      for (int x = 0; x < r.x; ++x) {
        i64 c = lin(x, y, z, r);
        bool in = inside(c), mixed = false;
        for (int k = 0; k < 6; ++k) mixed |= inside(lin(x + dx[k], y + dy[k], z + dz[k], r)) != in;
        sdf[c] = in ? (mixed ? (float)(0.5 - FS) : -U) : (mixed ? (float)(1.5 - FS) : U);
      }
  std::vector<float> prev(N);
  for (int d = 1; d < layers; ++d) {
    std::memcpy(prev.data(), sdf, N * sizeof(float));
    float outT = (float)((double)d + (1.5 - FS) - 1), inT = (float)(-((double)d + FS - 1.5));
    float outV = (float)((double)d + (1.5 - FS)), inV = (float)(-((double)d - (0.5 - FS)));
    bool any = false;
    for (int z = 0; z < r.z; ++z)
      for (int y = 0; y < r.y; ++y)
        for (int x = 0; x < r.x; ++x) {
          i64 c = lin(x, y, z, r);
          if (prev[c] == U) {
            for (int k = 0; k < 6; ++k)
              if (std::fabs(prev[lin(x + dx[k], y + dy[k], z + dz[k], r)] - outT) < FLT_MIN) { sdf[c] = outV; any = true; break; }
          } else if (prev[c] == -U) {
            for (int k = 0; k < 6; ++k)
              if (std::fabs(prev[lin(x + dx[k], y + dy[k], z + dz[k], r)] - inT) < FLT_MIN) { sdf[c] = inV; any = true; break; }
          }
        }
    if (!any) break;
  }
}

// EulerSolverTool.cu:408-448 buildFluidDensity: 1 in the fluid, the surface
// density 0.2 where a clamp-to-edge 6-neighbour is air (fluid domain and
// solid both >= 0, isInsideAir EulerMathTool.cu:344-348), 0 elsewhere.
void orc_build_fluid_density(const int* res, const float* dom, const float* solid, float* out) {
  Res r{res[0], res[1], res[2]};
  const int dx[6] = {-1, 1, 0, 0, 0, 0}, dy[6] = {0, 0, -1, 1, 0, 0}, dz[6] = {0, 0, 0, 0, -1, 1};
  for (int z = 0; z < r.z; ++z)
    for (int y = 0; y < r.y; ++y)
      for (int x = 0; x < r.x; ++x) {
        i64 c = lin(x, y, z, r);
        float v = 0.f;
        if (dom[c] < 0 && !(solid[c] < 0)) {
          bool air = false;
          for (int k = 0; k < 6; ++k) {
            i64 nb = lin(x + dx[k], y + dy[k], z + dz[k], r);
            air = air || (dom[nb] >= 0 && solid[nb] >= 0);
          }
          v = air ? (float)0.2 : 1.0f;
        }
        out[c] = v;
      }
}

// HybridSimulatorBuildSDF.cu:4-146,177-238 buildFluidInsideSDF /
// buildFluidOutsideSDF, driven as their invokers: sweep 0 sets solids (solid
// SDF < 0) to 0, cells of the surface density 0.2 to the seed value (0.2 -
// 0.5 inside, 0.5 - 0.2 outside), cells of density 0 (inside) or 1
// (outside) to 0 and the rest to UNKNOWN; sweep i (1 .. distance - 1) gives
// an UNKNOWN cell the value i + seed when a clamp-to-edge 6-neighbour holds
// i - 1 + seed (equality as isRealEQ, |a - b| < FLT_MIN); finally negative
// values become 0 (buildFluidSDFPostProcess, :122-137).  Every shell value is
// formed in double and rounded to float once, as the reference's mixed
// UInt/double expressions are.  A cell written in sweep i never holds the
// value sweep i tests for, so reading the previous sweep's copy is the
// reference's in-place sweep.
void orc_build_fluid_side_sdf(const int* res, const float* density, const float* solid, int outside, int distance,
                              float* out) {
  Res r{res[0], res[1], res[2]};
  const double FS = 0.2;  // FluidSurfaceDensity (Common.h:244)
  const double seed = outside ? 0.5 - FS : FS - 0.5;
  const float zeroDensity = outside ? 1.0f : 0.0f;
  const float U = FLT_MAX;
  auto eq = [](float a, float b) { return std::fabs(a - b) < FLT_MIN; };
  i64 N = r.size();
  if (distance > 0)
    for (i64 c = 0; c < N; ++c) {
      if (solid[c] < 0) out[c] = 0.f;
      else if (eq(density[c], (float)FS)) out[c] = (float)seed;
      else if (eq(density[c], zeroDensity)) out[c] = 0.f;
      else out[c] = U;
    }
  const int dx[6] = {-1, 1, 0, 0, 0, 0}, dy[6] = {0, 0, -1, 1, 0, 0}, dz[6] = {0, 0, 0, 0, -1, 1};
  std::vector<float> prev(N);
  for (int i = 1; i < distance; ++i) {
    std::memcpy(prev.data(), out, N * sizeof(float));
    const float target = (float)((double)i + seed - 1), value = (float)((double)i + seed);
    bool any = false;
    for (int z = 0; z < r.z; ++z)
      for (int y = 0; y < r.y; ++y)
        for (int x = 0; x < r.x; ++x) {
          i64 c = lin(x, y, z, r);
          if (prev[c] != U) continue;
          for (int k = 0; k < 6; ++k)
            if (eq(prev[lin(x + dx[k], y + dy[k], z + dz[k], r)], target)) { out[c] = value; any = true; break; }
        }
    if (!any) break;
  }
  for (i64 c = 0; c < N; ++c)
    if (out[c] < 0) out[c] = 0.f;
}

// HybridSimulatorBuildSDF.cu:139-175,240-266 buildMixedFluidOutsideSDF: at a
// cell of grid density 0.2, 0.5 minus the mixed density (negative -> 0);
// elsewhere the grid fluid's outside SDF.
void orc_build_mixed_fluid_outside_sdf(const int* res, const float* gridDensity, const float* mixedDensity,
                                       const float* gridOutside, float* out) {
  Res r{res[0], res[1], res[2]};
  for (i64 c = 0; c < r.size(); ++c) {
    if (std::fabs(gridDensity[c] - (float)0.2) < FLT_MIN) {
      float v = (float)(0.5 - (double)mixedDensity[c]);
      out[c] = v < 0 ? 0.f : v;
    } else {
      out[c] = gridOutside[c];
    }
  }
}

// HybridSimulatorMixFieldWithDensity.cu:6-265 mixFieldWithDensity: B := (wA A +
// wB B) / (wA + wB) where wA + wB > FLT_EPSILON (B kept elsewhere).  On a
// face grid the weights are the means of the two adjacent cells (clamp to
// edge); the reference scales that sum by the double literal 0.5.
static inline void mixOne(float a, float& b, float wa, float wb) {
  if (wa + wb > std::numeric_limits<float>::epsilon()) b = (wa * a + wb * b) / (wa + wb);
}
void orc_mix_field_with_density_cc(long long n, const float* a, float* b, const float* wa, const float* wb) {
  for (i64 i = 0; i < n; ++i) mixOne(a[i], b[i], wa[i], wb[i]);
}
void orc_mix_field_with_density_fc(const int* res, const float* ax, const float* ay, const float* az, float* bx,
                                   float* by, float* bz, const float* wa, const float* wb) {
  Res r{res[0], res[1], res[2]};
  const float* A[3] = {ax, ay, az};
  float* B[3] = {bx, by, bz};
  for (int axis = 0; axis < 3; ++axis) {
    Res f = r;
    if (axis == 0) f.x += 1;
    if (axis == 1) f.y += 1;
    if (axis == 2) f.z += 1;
    for (int z = 0; z < f.z; ++z)
      for (int y = 0; y < f.y; ++y)
        for (int x = 0; x < f.x; ++x) {
          i64 lo = lin(x - (axis == 0), y - (axis == 1), z - (axis == 2), r), hi = lin(x, y, z, r);
          float wA = (float)((double)(wa[lo] + wa[hi]) * 0.5), wB = (float)((double)(wb[lo] + wb[hi]) * 0.5);
          i64 c = lin(x, y, z, f);
          mixOne(A[axis][c], B[axis][c], wA, wB);
        }
  }
}
// HybridSimulatorMixParitcleVelWithPICAndFLIP.cu:5-57: blend by the particle's
// distance (in cells) into PIC, then FLIP, then the predicted velocity.
void orc_mix_particle_vel(const float* pic, const float* flip, const float* dist, long long n, float cell, float g,
                          float gf, float f, float pr, float* predict) {
  const float dg = g * cell, dgf = gf * cell, df = f * cell, dp = pr * cell;
  for (i64 i = 0; i < n; ++i) {
    float d = dist[i];
    for (int a = 0; a < 3; ++a) {
      float P = pic[3 * i + a], F = flip[3 * i + a], Q = predict[3 * i + a], m;
      if (d <= dg) m = P;
      else if (d <= dgf) m = P + ((d - dg) / (dgf - dg)) * (Q - P);
      else if (d <= df) m = F;
      else if (d <= dp) m = F + ((d - df) / (dp - df)) * (Q - F);
      else m = Q;
      predict[3 * i + a] = m;
    }
  }
}

// EulerSolverTool.cu:581-608 generateFluidDomainFromBBox (strict inequalities)
void orc_fluid_domain_from_bbox(const int* res, const float* o, const float* h, const float* mn, const float* mx,
                                float* out) {
  Res r{res[0], res[1], res[2]};
  for (int z = 0; z < r.z; ++z)
    for (int y = 0; y < r.y; ++y)
      for (int x = 0; x < r.x; ++x) {
        float cx = o[0] + 0.5f * h[0] + h[0] * (float)x;
        float cy = o[1] + 0.5f * h[1] + h[1] * (float)y;
        float cz = o[2] + 0.5f * h[2] + h[2] * (float)z;
        bool in = cx > mn[0] && cy > mn[1] && cz > mn[2] && cx < mx[0] && cy < mx[1] && cz < mx[2];
        out[lin(x, y, z, r)] = in ? -500.0f : 500.0f;  // FluidDomainValue, Common.h:245
      }
}

void orc_markers_from_particles(const int* res, const float* o, const float* h, const float* solidSDF,
                                const float* pos, long long P, uint8_t* markers, uint32_t* counts) {
  GridGeom<float> g = mkGeom<float>(res, o, h);
  markersFromParticles<float>(g, solidSDF, pos, P, markers, counts);
}

void orc_markers_from_sdf(const int* res, const float* solidSDF, const float* fluidSDF, uint8_t* markers) {
  Res r{res[0], res[1], res[2]};
  markersFromSDF<float>(r.size(), solidSDF, fluidSDF, markers);
}

void orc_build_matrix_a(int dbl, const int* res, const float* h, float dt, const uint8_t* mk, float* A) {
  Res r{res[0], res[1], res[2]};
  if (dbl) {
    V3<double> s{(double)dt / ((double)h[0] * h[0]), (double)dt / ((double)h[1] * h[1]), (double)dt / ((double)h[2] * h[2])};
    std::vector<double> a(4 * r.size());
    buildMatrixA(r, s, mk, a.data());
    down(a, A);
  } else {
    V3<float> s{dt / (1.0f * h[0] * h[0]), dt / (1.0f * h[1] * h[1]), dt / (1.0f * h[2] * h[2])};
    buildMatrixA(r, s, mk, A);
  }
}

}  // extern "C"
template <class T>
static void rhsT(const int* res, const float* h, const float* vx, const float* vy, const float* vz, const float* sx,
                 const float* sy, const float* sz, const uint8_t* mk, float* b) {
  Res r{res[0], res[1], res[2]};
  FC<T> v = upFC<T>(r, vx, vy, vz), s = upFC<T>(r, sx, sy, sz);
  std::vector<T> bb(r.size());
  buildRHS(r, V3<T>{(T)h[0], (T)h[1], (T)h[2]}, v, s, mk, bb.data());
  down(bb, b);
}
extern "C" {
void orc_build_rhs(int dbl, const int* res, const float* h, const float* vx, const float* vy, const float* vz,
                   const float* sx, const float* sy, const float* sz, const uint8_t* mk, float* b) {
  if (dbl) rhsT<double>(res, h, vx, vy, vz, sx, sy, sz, mk, b);
  else rhsT<float>(res, h, vx, vy, vz, sx, sy, sz, mk, b);
}

}  // extern "C"
template <class T>
static void applyAT(const int* res, const float* h, float dt, const uint8_t* mk, const float* x, float* y) {
  Res r{res[0], res[1], res[2]};
  V3<T> s{(T)dt / ((T)h[0] * (T)h[0]), (T)dt / ((T)h[1] * (T)h[1]), (T)dt / ((T)h[2] * (T)h[2])};
  std::vector<T> A(4 * r.size()), xx = up<T>(x, r.size()), yy(r.size());
  buildMatrixA(r, s, mk, A.data());
  matVec(r, A.data(), xx.data(), yy.data());
  down(yy, y);
}
extern "C" {
void orc_apply_a(int dbl, const int* res, const float* h, float dt, const uint8_t* mk, const float* x, float* y) {
  if (dbl) applyAT<double>(res, h, dt, mk, x, y);
  else applyAT<float>(res, h, dt, mk, x, y);
}

// Full pressure projection on given inputs (PressureSolver.cpp:154-198):
// markers are inputs here; the RHS, CG and gradient follow.  Outputs the
// pressure, the projected velocity (in place) and the solve statistics.
}  // extern "C"
template <class T>
static long long projectT(const int* res, const float* h, float dt, const uint8_t* mk, float* vx, float* vy,
                          float* vz, const float* sx, const float* sy, const float* sz, int precond, int tolMode,
                          double tol, long long maxIter, float* pOut, double* stats) {
  Res r{res[0], res[1], res[2]};
  i64 N = r.size();
  V3<T> hh{(T)h[0], (T)h[1], (T)h[2]};
  FC<T> v = upFC<T>(r, vx, vy, vz), s = upFC<T>(r, sx, sy, sz);
  V3<T> sA{(T)dt / ((T)1.0 * hh.x * hh.x), (T)dt / ((T)1.0 * hh.y * hh.y), (T)dt / ((T)1.0 * hh.z * hh.z)};
  std::vector<T> A(4 * N), b(N), x;
  buildMatrixA(r, sA, mk, A.data());
  buildRHS(r, hh, v, s, mk, b.data());
  PcgOpts o;
  o.precond = precond; o.tolMode = tolMode; o.tol = tol; o.maxIter = maxIter;
  double rn = 0, bn = 0;
  i64 it = pcgSolve(r, A.data(), b, x, o, &rn, &bn);
  V3<T> sG{(T)dt / ((T)1.0 * hh.x), (T)dt / ((T)1.0 * hh.y), (T)dt / ((T)1.0 * hh.z)};
  applyGradient(r, sG, mk, x.data(), v, s);
  if (pOut) down(x, pOut);
  downFC(v, vx, vy, vz);
  if (stats) { stats[0] = rn; stats[1] = bn; }
  return it;
}
extern "C" {
long long orc_project(int dbl, const int* res, const float* h, float dt, const uint8_t* mk, float* vx, float* vy,
                      float* vz, const float* sx, const float* sy, const float* sz, int precond, int tolMode,
                      double tol, long long maxIter, float* pOut, double* stats) {
  if (dbl) return projectT<double>(res, h, dt, mk, vx, vy, vz, sx, sy, sz, precond, tolMode, tol, maxIter, pOut, stats);
  return projectT<float>(res, h, dt, mk, vx, vy, vz, sx, sy, sz, precond, tolMode, tol, maxIter, pOut, stats);
}

// Extrapolation of one scalar grid in place; markersOut (optional) receives
// the layer index of every entry (FLT_MAX where unreachable).
void orc_extrapolate(const int* res, float* f, int nums, float* markersOut) {
  Res r{res[0], res[1], res[2]};
  std::vector<float> mk;
  extrapolate<float>(r, f, nums, markersOut ? &mk : nullptr);
  if (markersOut) std::memcpy(markersOut, mk.data(), mk.size() * sizeof(float));
}

// Trilinear sampling of a face-centred field at M positions (AoS xyz).
void orc_sample_fc(int dbl, const int* res, const float* o, const float* h, const float* vx, const float* vy,
                   const float* vz, const float* pos, long long M, float* out) {
  if (dbl) {
    GridGeom<double> g = mkGeom<double>(res, o, h);
    FC<double> v = upFC<double>(g.r, vx, vy, vz);
    for (i64 i = 0; i < M; ++i) {
      double q[3];
      sampleFC(v, g, (double)pos[3 * i], (double)pos[3 * i + 1], (double)pos[3 * i + 2], q);
      for (int a = 0; a < 3; ++a) out[3 * i + a] = (float)q[a];
    }
  } else {
    GridGeom<float> g = mkGeom<float>(res, o, h);
    FC<float> v = upFC<float>(g.r, vx, vy, vz);
    for (i64 i = 0; i < M; ++i) sampleFC(v, g, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], out + 3 * i);
  }
}

// Sampling of a cell-centred scalar field with an ESamplingAlgorithm
// (FieldMathTool.cu:470-573), FP32 or FP64.
void orc_sample_cc_alg(int dbl, const int* res, const float* o, const float* h, const float* f, const float* pos,
                       long long M, int alg, float* out) {
  if (dbl) {
    GridGeom<double> g = mkGeom<double>(res, o, h);
    std::vector<double> fd = up<double>(f, g.r.size());
    for (i64 i = 0; i < M; ++i)
      out[i] = (float)sampleAlg(fd.data(), g, (double)pos[3 * i], (double)pos[3 * i + 1], (double)pos[3 * i + 2], alg);
  } else {
    GridGeom<float> g = mkGeom<float>(res, o, h);
    for (i64 i = 0; i < M; ++i) out[i] = sampleAlg(f, g, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], alg);
  }
}

// Sampling of a face-centred field with an ESamplingAlgorithm
// (FieldMathTool.cu:783-1128): out is 3 floats per point.
void orc_sample_fc_alg(const int* res, const float* o, const float* h, const float* vx, const float* vy,
                       const float* vz, const float* pos, long long M, int alg, float* out) {
  GridGeom<float> g = mkGeom<float>(res, o, h);
  FC<float> v = upFC<float>(g.r, vx, vy, vz);
  for (i64 i = 0; i < M; ++i) sampleFCAlg(v, g, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], alg, &out[3 * i]);
}

// Trilinear sampling of a cell-centred scalar field.
void orc_sample_cc(const int* res, const float* o, const float* h, const float* f, const float* pos, long long M,
                   float* out) {
  GridGeom<float> g = mkGeom<float>(res, o, h);
  for (i64 i = 0; i < M; ++i) out[i] = trilerp(f, g, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
}

// G2P from a face-centred field (EulerParticlesTool.cu:805-868)
void orc_g2p_fc(const int* res, const float* o, const float* h, const float* vx, const float* vy, const float* vz,
                const float* pos, long long P, int alg, float* out) {
  GridGeom<float> g = mkGeom<float>(res, o, h);
  const float* c[3] = {vx, vy, vz};
  for (int a = 0; a < 3; ++a) {
    GridGeom<float> fg = faceGeom(g, a);
    for (i64 p = 0; p < P; ++p) out[3 * p + a] = g2pOne(c[a], fg, pos[3 * p], pos[3 * p + 1], pos[3 * p + 2], alg);
  }
}

// G2P from a cell-centred scalar field (EulerParticlesTool.cu:713-741)
void orc_g2p_cc(const int* res, const float* o, const float* h, const float* f, const float* pos, long long P,
                int alg, float* out) {
  GridGeom<float> g = mkGeom<float>(res, o, h);
  for (i64 p = 0; p < P; ++p) out[p] = g2pOne(f, g, pos[3 * p], pos[3 * p + 1], pos[3 * p + 2], alg);
}

// P2G to a face-centred field with weights, normalised (EulerParticlesTool.cu:601-711)
void orc_p2g_fc(int dbl, const int* res, const float* o, const float* h, const float* pos, const float* val,
                long long P, int alg, float* ox, float* oy, float* oz, float* wx, float* wy, float* wz) {
  float* outs[3] = {ox, oy, oz};
  float* ws[3] = {wx, wy, wz};
  if (dbl) {
    GridGeom<double> g = mkGeom<double>(res, o, h);
    std::vector<double> pp = up<double>(pos, 3 * P), vv = up<double>(val, 3 * P);
    for (int a = 0; a < 3; ++a) {
      GridGeom<double> fg = faceGeom(g, a);
      std::vector<double> out(fg.r.size()), w(fg.r.size());
      p2gOne(fg, pp.data(), vv.data(), 3, a, P, alg, out, w, true);
      down(out, outs[a]);
      if (ws[a]) down(w, ws[a]);
    }
  } else {
    GridGeom<float> g = mkGeom<float>(res, o, h);
    for (int a = 0; a < 3; ++a) {
      GridGeom<float> fg = faceGeom(g, a);
      std::vector<float> out(fg.r.size()), w(fg.r.size());
      p2gOne(fg, pos, val, 3, a, P, alg, out, w, true);
      std::memcpy(outs[a], out.data(), out.size() * 4);
      if (ws[a]) std::memcpy(ws[a], w.data(), w.size() * 4);
    }
  }
}

// P2G to a cell-centred scalar field (EulerParticlesTool.cu:443-496)
void orc_p2g_cc(const int* res, const float* o, const float* h, const float* pos, const float* val, long long P,
                int alg, int normalize, float* out, float* w) {
  GridGeom<float> g = mkGeom<float>(res, o, h);
  std::vector<float> oo(g.r.size()), ww(g.r.size());
  p2gOne(g, pos, val, 1, 0, P, alg, oo, ww, normalize != 0);
  std::memcpy(out, oo.data(), oo.size() * 4);
  if (w) std::memcpy(w, ww.data(), ww.size() * 4);
}

// CFL-substepped particle advection; returns the number of substeps.
int orc_advect_particles(int dbl, const int* res, const float* o, const float* h, const float* vx, const float* vy,
                         const float* vz, float* pos, long long P, float dt, float cfl, int acc, int clampMode) {
  if (dbl) {
    GridGeom<double> g = mkGeom<double>(res, o, h);
    FC<double> v = upFC<double>(g.r, vx, vy, vz);
    std::vector<double> pp = up<double>(pos, 3 * P);
    int n = advectParticles<double>(g, v, pp, (double)dt, (double)cfl, acc, clampMode);
    down(pp, pos);
    return n;
  }
  GridGeom<float> g = mkGeom<float>(res, o, h);
  FC<float> v = upFC<float>(g.r, vx, vy, vz);
  std::vector<float> pp(pos, pos + 3 * P);
  int n = advectParticles<float>(g, v, pp, dt, cfl, acc, clampMode);
  std::memcpy(pos, pp.data(), pp.size() * 4);
  return n;
}

// Semi-Lagrangian advection of a face-centred field through `vel`.
void orc_sl_advect_fc(int dbl, const int* res, const float* o, const float* h, const float* ix, const float* iy,
                      const float* iz, const float* vx, const float* vy, const float* vz, float dt, int acc,
                      float* ox, float* oy, float* oz) {
  if (dbl) {
    GridGeom<double> g = mkGeom<double>(res, o, h);
    FC<double> in = upFC<double>(g.r, ix, iy, iz), v = upFC<double>(g.r, vx, vy, vz), out;
    out.resize(g.r);
    slAdvectFC<double>(g, in, v, (double)dt, acc, out);
    downFC(out, ox, oy, oz);
  } else {
    GridGeom<float> g = mkGeom<float>(res, o, h);
    FC<float> in = upFC<float>(g.r, ix, iy, iz), v = upFC<float>(g.r, vx, vy, vz), out;
    out.resize(g.r);
    slAdvectFC<float>(g, in, v, dt, acc, out);
    downFC(out, ox, oy, oz);
  }
}

// Semi-Lagrangian advection with an ESamplingAlgorithm for every sample.
void orc_sl_advect_fc_alg(const int* res, const float* o, const float* h, const float* ix, const float* iy,
                          const float* iz, const float* vx, const float* vy, const float* vz, float dt, int acc,
                          int samp, float* ox, float* oy, float* oz) {
  GridGeom<float> g = mkGeom<float>(res, o, h);
  FC<float> in = upFC<float>(g.r, ix, iy, iz), v = upFC<float>(g.r, vx, vy, vz), out;
  out.resize(g.r);
  slAdvectFC<float>(g, in, v, dt, acc, out, samp);
  downFC(out, ox, oy, oz);
}
void orc_sl_advect_cc_alg(const int* res, const float* o, const float* h, const float* in, const float* vx,
                          const float* vy, const float* vz, float dt, int acc, int samp, float* out) {
  GridGeom<float> g = mkGeom<float>(res, o, h);
  FC<float> v = upFC<float>(g.r, vx, vy, vz);
  slAdvectCC<float>(g, {in}, v, dt, acc, {out}, samp);
}

// Semi-Lagrangian advection of a cell-centred scalar field.
void orc_sl_advect_cc(const int* res, const float* o, const float* h, const float* in, const float* vx,
                      const float* vy, const float* vz, float dt, int acc, float* out) {
  GridGeom<float> g = mkGeom<float>(res, o, h);
  FC<float> v = upFC<float>(g.r, vx, vy, vz);
  slAdvectCC<float>(g, {in}, v, dt, acc, {out});
}

}  // extern "C"

// --------------------------- solver object ---------------------------------
// Mirrors CGridFluidSolver (GridFluidSolver.h:17-137) for multi-step parity.
struct OrcSolver {
  int dbl;
  Solver<float> f;
  Solver<double> d;
};

template <class T> static Solver<T>& pick(OrcSolver* S);
template <> Solver<float>& pick<float>(OrcSolver* S) { return S->f; }
template <> Solver<double>& pick<double>(OrcSolver* S) { return S->d; }

#define ORC_CALL(S, fn, ...) ((S)->dbl ? fn<double>(S, ##__VA_ARGS__) : fn<float>(S, ##__VA_ARGS__))

template <class T> static void sAddBoundary(OrcSolver* S, const float* sdf, float vx, float vy, float vz) {
  Solver<T>& s = pick<T>(S);
  Boundary<T> b;
  b.sdf0 = up<T>(sdf, s.g.r.size());
  b.sdf = b.sdf0;
  b.vel = V3<T>{(T)vx, (T)vy, (T)vz};
  s.bnd.push_back(b);
}
// The per-frame rigid-boundary update of the viewer loop: boundary `i` moves
// with `v` from the next step on (Boundary.cpp:124-127 uses it as -dt * v).
template <class T> static void sSetBoundaryVel(OrcSolver* S, int i, float vx, float vy, float vz) {
  Solver<T>& s = pick<T>(S);
  if (i < 0 || i >= (int)s.bnd.size()) return;
  s.bnd[i].vel = V3<T>{(T)vx, (T)vy, (T)vz};
}
template <class T> static void sSetVel(OrcSolver* S, const float* x, const float* y, const float* z) {
  Solver<T>& s = pick<T>(S);
  s.vel1 = upFC<T>(s.g.r, x, y, z);
  s.vel2 = s.vel1;
}
template <class T> static void sSetDomain(OrcSolver* S, const float* d) {
  Solver<T>& s = pick<T>(S);
  s.dom1 = up<T>(d, s.g.r.size());
  s.dom2 = s.dom1;
}
template <class T> static void sSetColor(OrcSolver* S, const float* x, const float* y, const float* z) {
  Solver<T>& s = pick<T>(S);
  i64 N = s.g.r.size();
  const float* c[3] = {x, y, z};
  for (int a = 0; a < 3; ++a) { s.color1[a] = up<T>(c[a], N); s.color2[a] = s.color1[a]; }
}
template <class T>
static void sSetAdvection(OrcSolver* S, int kind, int acc, int alg, float cfl, float mixing, int clampMode,
                          int advectScalars) {
  Solver<T>& s = pick<T>(S);
  s.adv = kind; s.acc = acc; s.alg = alg; s.cfl = (T)cfl; s.mixing = (T)mixing; s.clampMode = clampMode;
  s.advectScalars = advectScalars != 0;
  s.sFlag = s.vFlag = s.velFlag = false;
}
template <class T> static void sSetSampling(OrcSolver* S, int samp) { pick<T>(S).sampling = samp; }
// GridFluidSolver.cpp:615-642 mixVelFieldWithOthers: into the buffer the step
// in progress writes (Field1 while the flag is set, else Field2).
template <class T>
static void sMixVel(OrcSolver* S, const float* ox, const float* oy, const float* oz, const float* wo, const float* wf) {
  Solver<T>& s = pick<T>(S);
  FC<T>& b = s.velOut();
  const float* O[3] = {ox, oy, oz};
  const Res r = s.g.r;
  for (int axis = 0; axis < 3; ++axis) {
    Res f = r;
    if (axis == 0) f.x += 1;
    if (axis == 1) f.y += 1;
    if (axis == 2) f.z += 1;
    for (int z = 0; z < f.z; ++z)
      for (int y = 0; y < f.y; ++y)
        for (int x = 0; x < f.x; ++x) {
          i64 lo = lin(x - (axis == 0), y - (axis == 1), z - (axis == 2), r), hi = lin(x, y, z, r);
          T wA = (T)((double)((T)wo[lo] + (T)wo[hi]) * 0.5), wB = (T)((double)((T)wf[lo] + (T)wf[hi]) * 0.5);
          i64 c = lin(x, y, z, f);
          T& v = b.c[axis][c];
          if (wA + wB > (T)std::numeric_limits<float>::epsilon()) v = (wA * (T)O[axis][c] + wB * v) / (wA + wB);
        }
  }
}
template <class T> static void sSetParticles(OrcSolver* S, const float* pos, const float* vel, long long P) {
  Solver<T>& s = pick<T>(S);
  s.ppos = up<T>(pos, 3 * P);
  if (vel) s.pvel = up<T>(vel, 3 * P);
  else s.pvel.assign(3 * P, 0);
  s.pscalar.assign(P, 0);
  s.pvector.assign(3 * P, 0);
}
template <class T> static void sSetPcg(OrcSolver* S, int precond, int tolMode, double tol, long long maxIter) {
  Solver<T>& s = pick<T>(S);
  s.pcg.precond = precond; s.pcg.tolMode = tolMode; s.pcg.tol = tol; s.pcg.maxIter = maxIter;
}
template <class T> static void sExt(OrcSolver* S, float x, float y, float z) {
  Solver<T>& s = pick<T>(S);
  s.ext.x += (T)x; s.ext.y += (T)y; s.ext.z += (T)z;  // ExternalForcesSolver.cpp:45-48
}
template <class T> static int sStep(OrcSolver* S, int what) {
  Solver<T>& s = pick<T>(S);
  if (what == 0) s.update();
  else if (what == 1) s.updateWithoutPressure();
  else s.solvePressure();
  return 0;
}
template <class T> static void sGetVel(OrcSolver* S, int which, float* x, float* y, float* z) {
  Solver<T>& s = pick<T>(S);
  // GridFluidSolver.cpp:302-324: current = V2 if flag else V1
  const FC<T>& v = which == 0 ? s.velCur() : s.velOut();
  downFC(v, x, y, z);
}
template <class T> static void sGetVel64(OrcSolver* S, double* x, double* y, double* z) {
  Solver<T>& s = pick<T>(S);
  const FC<T>& v = s.velCur();
  double* o[3] = {x, y, z};
  for (int a = 0; a < 3; ++a)
    for (size_t i = 0; i < v.c[a].size(); ++i) o[a][i] = (v.c[a][i] == unknownv<T>()) ? (double)FLT_MAX : (double)v.c[a][i];
}
template <class T> static void sGetDomain(OrcSolver* S, float* d) {
  Solver<T>& s = pick<T>(S);
  down(s.bufferFlag ? s.dom2 : s.dom1, d);
}
template <class T> static void sGetColor(OrcSolver* S, float* x, float* y, float* z) {
  Solver<T>& s = pick<T>(S);
  std::vector<T>* c = s.bufferFlag ? s.color2 : s.color1;
  down(c[0], x); down(c[1], y); down(c[2], z);
}
template <class T> static void sGetMarkers(OrcSolver* S, uint8_t* m) {
  Solver<T>& s = pick<T>(S);
  std::memcpy(m, s.markers.data(), s.markers.size());
}
template <class T> static void sGetPressure(OrcSolver* S, float* p) { down(pick<T>(S).px, p); }
template <class T> static void sGetSolidSDF(OrcSolver* S, float* p) { down(pick<T>(S).totalSDF, p); }
template <class T> static void sGetSolidVel(OrcSolver* S, float* x, float* y, float* z) {
  downFC(pick<T>(S).solidVel, x, y, z);
}
template <class T> static long long sNumParticles(OrcSolver* S) { return (long long)pick<T>(S).ppos.size() / 3; }
template <class T> static void sGetParticles(OrcSolver* S, float* pos, float* vel) {
  Solver<T>& s = pick<T>(S);
  if (pos) down(s.ppos, pos);
  if (vel) down(s.pvel, vel);
}
template <class T> static void sGetParticles64(OrcSolver* S, double* pos, double* vel) {
  Solver<T>& s = pick<T>(S);
  if (pos) for (size_t i = 0; i < s.ppos.size(); ++i) pos[i] = (double)s.ppos[i];
  if (vel) for (size_t i = 0; i < s.pvel.size(); ++i) vel[i] = (double)s.pvel[i];
}
template <class T> static void sStats(OrcSolver* S, double* out) {
  Solver<T>& s = pick<T>(S);
  out[0] = (double)s.lastIters; out[1] = s.lastResid; out[2] = s.lastBnorm;
  out[3] = (double)s.time; out[4] = (double)s.lastSubsteps; out[5] = s.bufferFlag ? 1.0 : 0.0;
}

extern "C" {

void* orc_solver_create(int dbl, float dt, const int* res, const float* o, const float* h) {
  OrcSolver* S = new OrcSolver();
  S->dbl = dbl;
  Res r{res[0], res[1], res[2]};
  if (dbl) S->d.create((double)dt, r, V3<double>{o[0], o[1], o[2]}, V3<double>{h[0], h[1], h[2]});
  else S->f.create(dt, r, V3<float>{o[0], o[1], o[2]}, V3<float>{h[0], h[1], h[2]});
  return S;
}
void orc_solver_destroy(void* p) { delete (OrcSolver*)p; }
void orc_solver_add_boundary(void* p, const float* sdf, float vx, float vy, float vz) {
  ORC_CALL((OrcSolver*)p, sAddBoundary, sdf, vx, vy, vz);
}
void orc_solver_set_boundary_velocity(void* p, int i, float vx, float vy, float vz) {
  ORC_CALL((OrcSolver*)p, sSetBoundaryVel, i, vx, vy, vz);
}
void orc_solver_set_velocity(void* p, const float* x, const float* y, const float* z) { ORC_CALL((OrcSolver*)p, sSetVel, x, y, z); }
void orc_solver_set_fluid_domain(void* p, const float* d) { ORC_CALL((OrcSolver*)p, sSetDomain, d); }
void orc_solver_set_color(void* p, const float* x, const float* y, const float* z) { ORC_CALL((OrcSolver*)p, sSetColor, x, y, z); }
void orc_solver_set_advection(void* p, int kind, int acc, int alg, float cfl, float mixing, int clampMode,
                              int advectScalars) {
  ORC_CALL((OrcSolver*)p, sSetAdvection, kind, acc, alg, cfl, mixing, clampMode, advectScalars);
}
void orc_solver_set_sampling(void* p, int samp) { ORC_CALL((OrcSolver*)p, sSetSampling, samp); }
void orc_solver_mix_vel(void* p, const float* ox, const float* oy, const float* oz, const float* wo, const float* wf) {
  ORC_CALL((OrcSolver*)p, sMixVel, ox, oy, oz, wo, wf);
}
void orc_solver_set_particles(void* p, const float* pos, const float* vel, long long P) {
  ORC_CALL((OrcSolver*)p, sSetParticles, pos, vel, P);
}
void orc_solver_set_pcg(void* p, int precond, int tolMode, double tol, long long maxIter) {
  ORC_CALL((OrcSolver*)p, sSetPcg, precond, tolMode, tol, maxIter);
}
void orc_solver_add_external_force(void* p, float x, float y, float z) { ORC_CALL((OrcSolver*)p, sExt, x, y, z); }
int orc_solver_update(void* p) { return ORC_CALL((OrcSolver*)p, sStep, 0); }
int orc_solver_update_without_pressure(void* p) { return ORC_CALL((OrcSolver*)p, sStep, 1); }
int orc_solver_solve_pressure(void* p) { return ORC_CALL((OrcSolver*)p, sStep, 2); }
void orc_solver_get_velocity(void* p, int which, float* x, float* y, float* z) { ORC_CALL((OrcSolver*)p, sGetVel, which, x, y, z); }
void orc_solver_get_velocity_f64(void* p, double* x, double* y, double* z) { ORC_CALL((OrcSolver*)p, sGetVel64, x, y, z); }
void orc_solver_get_fluid_domain(void* p, float* d) { ORC_CALL((OrcSolver*)p, sGetDomain, d); }
void orc_solver_get_color(void* p, float* x, float* y, float* z) { ORC_CALL((OrcSolver*)p, sGetColor, x, y, z); }
void orc_solver_get_markers(void* p, uint8_t* m) { ORC_CALL((OrcSolver*)p, sGetMarkers, m); }
void orc_solver_get_pressure(void* p, float* x) { ORC_CALL((OrcSolver*)p, sGetPressure, x); }
void orc_solver_get_solid_sdf(void* p, float* x) { ORC_CALL((OrcSolver*)p, sGetSolidSDF, x); }
void orc_solver_get_solid_vel(void* p, float* x, float* y, float* z) { ORC_CALL((OrcSolver*)p, sGetSolidVel, x, y, z); }
long long orc_solver_num_particles(void* p) { return ORC_CALL((OrcSolver*)p, sNumParticles); }
void orc_solver_get_particles(void* p, float* pos, float* vel) { ORC_CALL((OrcSolver*)p, sGetParticles, pos, vel); }
void orc_solver_get_particles_f64(void* p, double* pos, double* vel) {
  ORC_CALL((OrcSolver*)p, sGetParticles64, pos, vel);
}
// stats: [cg iterations, final ||r||, ||b||, time, substeps, buffer flag]
void orc_solver_stats(void* p, double* out) { ORC_CALL((OrcSolver*)p, sStats, out); }

}  // extern "C"

// ===========================================================================
// Single stages for the replay of the reference's own unit tests
// (oracle/reftests): each is one piece of the step above, exported alone.
// ===========================================================================
extern "C" {

// SemiLagrangian.cpp:188-347 backTrace of M points (AoS xyz) through the
// face-centred velocity on the grid (res, o, h); `samp` is the
// ESamplingAlgorithm of the velocity samples.
void orc_back_trace(int dbl, const int* res, const float* o, const float* h, const float* vx, const float* vy,
                    const float* vz, const float* pos, long long M, float dt, int acc, int samp, float* out) {
  if (dbl) {
    GridGeom<double> g = mkGeom<double>(res, o, h);
    FC<double> v = upFC<double>(g.r, vx, vy, vz);
    for (i64 i = 0; i < M; ++i) {
      double in[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]}, q[3];
      backTrace<double>(v, g, (double)dt, acc, in, q, samp);
      for (int a = 0; a < 3; ++a) out[3 * i + a] = (float)q[a];
    }
  } else {
    GridGeom<float> g = mkGeom<float>(res, o, h);
    FC<float> v = upFC<float>(g.r, vx, vy, vz);
    for (i64 i = 0; i < M; ++i) backTrace<float>(v, g, dt, acc, pos + 3 * i, out + 3 * i, samp);
  }
}

// EulerParticlesTool.cu:27-46 statisticalFluidDensity: particles per cell
// (truncating binning of transPos2Index), as Real.
void orc_particle_counts(const int* res, const float* o, const float* h, const float* pos, long long P, float* out) {
  GridGeom<float> g = mkGeom<float>(res, o, h);
  std::vector<float> cnt(g.r.size(), 0.0f);
  for (i64 p = 0; p < P; ++p) cnt[binIndex(g, pos[3 * p], pos[3 * p + 1], pos[3 * p + 2])] += 1.0f;
  std::memcpy(out, cnt.data(), cnt.size() * sizeof(float));
}

// FieldMathTool.cu:370-395 divergence of a face-centred field.
void orc_divergence_fc(int dbl, const int* res, const float* h, const float* vx, const float* vy, const float* vz,
                       float* out) {
  Res r{res[0], res[1], res[2]};
  if (dbl) {
    FC<double> v = upFC<double>(r, vx, vy, vz);
    std::vector<double> d(r.size());
    divergenceFC<double>(r, V3<double>{h[0], h[1], h[2]}, v, d.data());
    down(d, out);
  } else {
    FC<float> v = upFC<float>(r, vx, vy, vz);
    divergenceFC<float>(r, V3<float>{h[0], h[1], h[2]}, v, out);
  }
}

// ExternalForcesSolver.cpp:50-58: gravity (0, -9.8, 0) plus the user force,
// times dt, added to every face of (vx, vy, vz) in place.
void orc_apply_external_forces(const int* res, float* vx, float* vy, float* vz, float dt, float fx, float fy,
                               float fz) {
  Solver<float> s;
  s.dt = dt;
  s.ext = V3<float>{fx, fy, fz};
  Res r{res[0], res[1], res[2]};
  FC<float> v = upFC<float>(r, vx, vy, vz);
  s.applyForces(v);
  downFC(v, vx, vy, vz);
}

// Boundary.cpp:115-150 updateBoundarys on nb solids: translation -= dt * vel,
// each SDF resampled at the translated cell centres, the total marker
// (-(first solid index) inside, UNKNOWN outside) and the solid face
// velocities.  sdf0/sdfCur hold nb grids back to back; vel and trans 3 per
// solid (trans is updated in place).
void orc_boundarys_update(const int* res, const float* o, const float* h, int nb, const float* sdf0,
                          const float* vel, float* trans, float dt, float* sdfCur, float* marker, float* svx,
                          float* svy, float* svz) {
  Solver<float> s;
  s.create(dt, Res{res[0], res[1], res[2]}, V3<float>{o[0], o[1], o[2]}, V3<float>{h[0], h[1], h[2]});
  i64 N = s.g.r.size();
  for (int i = 0; i < nb; ++i) {
    Boundary<float> b;
    b.sdf0.assign(sdf0 + i * N, sdf0 + (i + 1) * N);
    b.sdf = b.sdf0;
    b.vel = V3<float>{vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]};
    b.trans = V3<float>{trans[3 * i], trans[3 * i + 1], trans[3 * i + 2]};
    s.bnd.push_back(b);
  }
  s.updateBoundarys();
  for (int i = 0; i < nb; ++i) {
    trans[3 * i] = s.bnd[i].trans.x;
    trans[3 * i + 1] = s.bnd[i].trans.y;
    trans[3 * i + 2] = s.bnd[i].trans.z;
    if (sdfCur) std::memcpy(sdfCur + i * N, s.bnd[i].sdf.data(), N * sizeof(float));
  }
  if (marker) down(s.totalSDF, marker);
  if (svx) downFC(s.solidVel, svx, svy, svz);
}

}  // extern "C"
