// hfg_kernels.cu -- sm_100a kernels of the grid half of the hybrid fluid step.
//
// Every kernel restates one stage of the reference engine's CUDA code
// (junwei-jiang/Hybrid-Fluid-Simulation, MPhysics/) in a B200-first shape:
// grid-stride launches sized to the SM count, fused stages, uint8 cell
// markers, FP64 deterministic reductions and device-resident solver scalars.
// The reference line each kernel follows is cited beside it.
#include <algorithm>
#include <atomic>
#include <cstdio>

#include "hfg_kernels.h"

namespace hfg {

namespace {
int g_numSMs = 0;
constexpr int kThreads = 256;

inline int gridFor(long long n, int threads = kThreads, int perSM = 16) {
  long long b = (n + threads - 1) / threads;
  long long cap = (long long)numSMs() * perSM;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

// Grid-stride loop over [0, n).
#define HFG_FOR(i, n) \
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

// The same loop with an index of type I.  The particle kernels take I = int
// when 3 n and n + the grid's thread count stay below 2^31, which saves the
// 64-bit index and address arithmetic of every iteration.
#define HFG_FOR_T(I, i, n) \
  for (I i = (I)blockIdx.x * blockDim.x + threadIdx.x; i < (I)(n); i += (I)gridDim.x * blockDim.x)


// True when a particle kernel over n particles may index in 32 bits.
inline bool index32(long long n) { return 3 * n + (long long)numSMs() * 16 * kThreads < (1ll << 31); }

__device__ inline void cellCoord(long long c, const Dim3i& r, int& x, int& y, int& z) {
  x = (int)(c % r.x);
  long long t = c / r.x;
  y = (int)(t % r.y);
  z = (int)(t / r.y);
}

}  // namespace

int numSMs() {
  if (g_numSMs == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&g_numSMs, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || g_numSMs <= 0)
      g_numSMs = 148;
  }
  return g_numSMs;
}


// ===========================================================================
// Boundaries and classification
// ===========================================================================

// Boundary.cpp:129-146 + BoundaryTool.cu:3-26,85-113: re-sample every solid
// SDF at (cell centre + translation) and keep the first solid that contains
// the cell.  solidIdx = 0 outside every solid, i+1 inside solid i.
__global__ void kSolidClassify(Geom g, BoundarySet b, uint8_t* __restrict__ solidIdx, float* const* curSDF) {
  long long n = g.r.size();
  HFG_FOR(c, n) {
    int x, y, z;
    cellCoord(c, g.r, x, y, z);
    float cx = __fadd_rn(__fadd_rn(g.ox, 0.5f * g.hx), __fmul_rn(g.hx, (float)x));
    float cy = __fadd_rn(__fadd_rn(g.oy, 0.5f * g.hy), __fmul_rn(g.hy, (float)y));
    float cz = __fadd_rn(__fadd_rn(g.oz, 0.5f * g.hz), __fmul_rn(g.hz, (float)z));
    uint8_t idx = 0;
    for (int i = 0; i < b.n; ++i) {
      float v = trilerp(b.sdf[i], g, __fadd_rn(cx, b.tx[i]), __fadd_rn(cy, b.ty[i]), __fadd_rn(cz, b.tz[i]));
      if (curSDF && curSDF[i]) curSDF[i][c] = v;
      if (idx == 0 && v < 0.f) idx = (uint8_t)(i + 1);
    }
    solidIdx[c] = idx;
  }
}

cudaError_t launchSolidClassify(const Geom& g, const BoundarySet& b, uint8_t* solidIdx, float* const* curSDF,
                                cudaStream_t s) {
  kSolidClassify<<<gridFor(g.r.size()), kThreads, 0, s>>>(g, b, solidIdx, curSDF);
  return cudaGetLastError();
}

__global__ void kSolidFromSDF(long long n, const float* __restrict__ sdf, uint8_t* __restrict__ idx) {
  HFG_FOR(c, n) idx[c] = sdf[c] < 0.f ? 1 : 0;
}
__global__ void kAnalyticSdf(Geom g, int type, double p0, double p1, double p2, double p3, double p4, double p5,
                             float* __restrict__ sdf) {
  const Dim3i R = g.r;
  HFG_FOR(c, R.size()) {
    int x, y, z;
    cellCoord(c, R, x, y, z);
    const double P[3] = {(double)g.ox + (x + 0.5) * (double)g.hx, (double)g.oy + (y + 0.5) * (double)g.hy,
                         (double)g.oz + (z + 0.5) * (double)g.hz};
    double d;
    if (type == 0) {
      const double lo[3] = {(double)g.ox + g.hx, (double)g.oy + g.hy, (double)g.oz + g.hz};
      const double hi[3] = {(double)g.ox + (R.x - 1) * (double)g.hx, (double)g.oy + (R.y - 1) * (double)g.hy,
                            (double)g.oz + (R.z - 1) * (double)g.hz};
      double in = 1e300, outsq = 0.0;
      for (int a = 0; a < 3; ++a) {
        double da = fmin(P[a] - lo[a], hi[a] - P[a]);
        in = fmin(in, da);
        if (da < 0.0) outsq += da * da;
      }
      d = in >= 0.0 ? in : -sqrt(outsq);
    } else if (type == 1) {
      const double dx = P[0] - p0, dy = P[1] - p1, dz = P[2] - p2;
      d = sqrt(dx * dx + dy * dy + dz * dz) - p3;
    } else {
      const double c3[3] = {p0, p1, p2}, s3[3] = {p3, p4, p5};
      double outsq = 0.0, mx = -1e300;
      for (int a = 0; a < 3; ++a) {
        double q = fabs(P[a] - c3[a]) - 0.5 * s3[a];
        if (q > 0.0) outsq += q * q;
        mx = fmax(mx, q);
      }
      d = sqrt(outsq) + fmin(mx, 0.0);
    }
    sdf[c] = (float)d;
  }
}
cudaError_t launchAnalyticSdf(const Geom& g, int type, const double* p, float* sdf, cudaStream_t s) {
  kAnalyticSdf<<<gridFor(g.r.size()), kThreads, 0, s>>>(g, type, p[0], p[1], p[2], p[3], p[4], p[5], sdf);
  return cudaGetLastError();
}

cudaError_t launchSolidFromSDF(long long n, const float* solidSDF, uint8_t* solidIdx, cudaStream_t s) {
  kSolidFromSDF<<<gridFor(n), kThreads, 0, s>>>(n, solidSDF, solidIdx);
  return cudaGetLastError();
}

// The reference's "total boundary SDF" (BoundaryTool.cu:3-26): 0 everywhere
// with no solid, else -(first solid index) inside and UNKNOWN outside.
__global__ void kTotalSolidSDF(long long n, int nb, const uint8_t* __restrict__ idx, float* __restrict__ out) {
  HFG_FOR(c, n) {
    uint8_t i = idx[c];
    out[c] = nb == 0 ? 0.f : (i ? -(float)i : kUnknown);
  }
}
cudaError_t launchTotalSolidSDF(long long n, int nb, const uint8_t* solidIdx, float* out, cudaStream_t s) {
  kTotalSolidSDF<<<gridFor(n), kThreads, 0, s>>>(n, nb, solidIdx, out);
  return cudaGetLastError();
}

__global__ void kSolidVelField(Geom g, SolidVelTable t, FaceField out) {
  for (int a = 0; a < 3; ++a) {
    Dim3i fr = g.r;
    if (a == 0) fr.x += 1;
    if (a == 1) fr.y += 1;
    if (a == 2) fr.z += 1;
    long long n = fr.size();
    HFG_FOR(f, n) {
      int x, y, z;
      cellCoord(f, fr, x, y, z);
      int hx = x, hy = y, hz = z, lx = x, ly = y, lz = z;
      if (a == 0) lx = x - 1;
      if (a == 1) ly = y - 1;
      if (a == 2) lz = z - 1;
      bool hiIn = (a == 0 ? hx < g.r.x : (a == 1 ? hy < g.r.y : hz < g.r.z));
      bool loIn = (a == 0 ? lx >= 0 : (a == 1 ? ly >= 0 : lz >= 0));
      uint8_t hi = hiIn ? t.solidIdx[((long long)hz * g.r.y + hy) * g.r.x + hx] : 0;
      uint8_t lo = loIn ? t.solidIdx[((long long)lz * g.r.y + ly) * g.r.x + lx] : 0;
      out.c[a][f] = solidFaceVel(t, lo, hi, a);
    }
  }
}
cudaError_t launchSolidVelField(const Geom& g, const SolidVelTable& t, FaceField out, cudaStream_t s) {
  kSolidVelField<<<gridFor(g.r.size()), kThreads, 0, s>>>(g, t, out);
  return cudaGetLastError();
}

__global__ void kMarkersInit(long long n, const uint8_t* __restrict__ idx, uint8_t* __restrict__ mk) {
  HFG_FOR(c, n) mk[c] = idx[c] ? kSolid : kAir;
}
cudaError_t launchMarkersInit(long long n, const uint8_t* solidIdx, uint8_t* markers, cudaStream_t s) {
  kMarkersInit<<<gridFor(n), kThreads, 0, s>>>(n, solidIdx, markers);
  return cudaGetLastError();
}

// EulerParticlesTool.cu:27-77: a non-solid cell holding at least one particle
// (truncating binning) is fluid.  Only "count > 0" matters, so the count is
// replaced by an idempotent store; cells stay bit-exact.
__global__ void kMarkersFromParticles(Geom g, const float* __restrict__ pos, long long P, uint8_t* __restrict__ mk) {
  HFG_FOR(p, P) {
    long long c = binCell(g, pos[3 * p], pos[3 * p + 1], pos[3 * p + 2]);
    if (mk[c] == kAir) mk[c] = kFluid;
  }
}
cudaError_t launchMarkersFromParticles(const Geom& g, const float* pos, long long P, uint8_t* markers, cudaStream_t s) {
  if (P <= 0) return cudaSuccess;
  kMarkersFromParticles<<<gridFor(P), kThreads, 0, s>>>(g, pos, P, markers);
  return cudaGetLastError();
}

// statisticalFluidDensity (EulerParticlesTool.cu:27-46) with warp-aggregated
// integer atomics: lanes that hit the same cell add once.
__global__ void kBinCounts(Geom g, const float* __restrict__ pos, long long P, unsigned int* __restrict__ counts) {
  for (long long base = (long long)blockIdx.x * blockDim.x; base < P; base += (long long)gridDim.x * blockDim.x) {
    long long p = base + threadIdx.x;
    bool valid = p < P;
    unsigned int active = __ballot_sync(0xffffffffu, valid);
    if (!valid) continue;
    long long c = binCell(g, pos[3 * p], pos[3 * p + 1], pos[3 * p + 2]);
    unsigned int peers = __match_any_sync(active, c);
    int leader = __ffs(peers) - 1;
    if ((int)(threadIdx.x & 31) == leader) atomicAdd(counts + c, (unsigned int)__popc(peers));
  }
}
cudaError_t launchBinCounts(const Geom& g, const float* pos, long long P, unsigned int* counts, cudaStream_t s) {
  if (P <= 0) return cudaSuccess;
  kBinCounts<<<gridFor(P), kThreads, 0, s>>>(g, pos, P, counts);
  return cudaGetLastError();
}

// EulerSolverTool.cu:30-56 buildFluidMarkers (SDF form)
__global__ void kMarkersFromSDF(long long n, const uint8_t* __restrict__ idx, const float* __restrict__ fsdf,
                                uint8_t* __restrict__ mk) {
  HFG_FOR(c, n) mk[c] = idx[c] ? kSolid : (fsdf[c] < 0.f ? kFluid : kAir);
}
cudaError_t launchMarkersFromSDF(long long n, const uint8_t* solidIdx, const float* fluidSDF, uint8_t* markers,
                                 cudaStream_t s) {
  kMarkersFromSDF<<<gridFor(n), kThreads, 0, s>>>(n, solidIdx, fluidSDF, markers);
  return cudaGetLastError();
}

// EulerSolverTool.cu:581-608 generateFluidDomainFromBBox (strict inequalities,
// every cell rewritten).
__global__ void kFluidDomainFromBBox(Geom g, float mnx, float mny, float mnz, float mxx, float mxy, float mxz,
                                     float* __restrict__ out) {
  HFG_FOR(c, g.r.size()) {
    int x, y, z;
    cellCoord(c, g.r, x, y, z);
    float cx = __fadd_rn(__fadd_rn(g.ox, 0.5f * g.hx), __fmul_rn(g.hx, (float)x));
    float cy = __fadd_rn(__fadd_rn(g.oy, 0.5f * g.hy), __fmul_rn(g.hy, (float)y));
    float cz = __fadd_rn(__fadd_rn(g.oz, 0.5f * g.hz), __fmul_rn(g.hz, (float)z));
    bool in = cx > mnx && cy > mny && cz > mnz && cx < mxx && cy < mxy && cz < mxz;
    out[c] = in ? -500.f : 500.f;  // FluidDomainValue (Common.h:245)
  }
}
cudaError_t launchFluidDomainFromBBox(const Geom& g, const float mn[3], const float mx[3], float* out, cudaStream_t s) {
  kFluidDomainFromBBox<<<gridFor(g.r.size()), kThreads, 0, s>>>(g, mn[0], mn[1], mn[2], mx[0], mx[1], mx[2], out);
  return cudaGetLastError();
}

// EulerSolverTool.cu:229-322 applyPressureGradient: faces with a fluid side
// and a solid side take the solid velocity, fluid-fluid/fluid-air faces get
// -dt/(rho h) * dp, all others and the far boundary faces become UNKNOWN.
template <class TP>
__global__ void kGradient(Geom g, float gx, float gy, float gz, const uint8_t* __restrict__ mk,
                          const TP* __restrict__ p, FaceField v, ConstFaceField svArr, SolidVelTable svTab) {
  const Dim3i R = g.r;
  const Dim3i rx{R.x + 1, R.y, R.z}, ry{R.x, R.y + 1, R.z}, rz{R.x, R.y, R.z + 1};
  HFG_FOR(c, R.size()) {
    int x, y, z;
    cellCoord(c, R, x, y, z);
    long long sy = R.x, sz = (long long)R.x * R.y;
    long long cl = x > 0 ? c - 1 : c, cd = y > 0 ? c - sy : c, cb = z > 0 ? c - sz : c;
    const long long px = cgPitch(R.x);
    const long long pc = ((long long)z * R.y + y) * px + x;  // pressure is pitched
    const long long po[3] = {x > 0 ? pc - 1 : pc, y > 0 ? pc - px : pc, z > 0 ? pc - px * R.y : pc};
    uint8_t mc = mk[c];
    long long fx = ((long long)z * rx.y + y) * rx.x + x;
    long long fy = ((long long)z * ry.y + y) * ry.x + x;
    long long fz = ((long long)z * rz.y + y) * rz.x + x;
    const long long fo[3] = {fx, fy, fz};
    const long long co[3] = {cl, cd, cb};
    const float gs[3] = {gx, gy, gz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      uint8_t ml = mk[co[a]];
      float* vv = v.c[a];
      if (ml == kFluid || mc == kFluid) {
        if (ml == kSolid || mc == kSolid) {
          float s;
          if (svArr.c[0]) s = svArr.c[a][fo[a]];
          else s = solidFaceVel(svTab, co[a] == c ? 0 : svTab.solidIdx[co[a]], svTab.solidIdx[c], a);
          vv[fo[a]] = s;
        } else {
          const float dp = sizeof(TP) == 8 ? __double2float_rn(__dsub_rn((double)p[pc], (double)p[po[a]]))
                                           : __fsub_rn((float)p[pc], (float)p[po[a]]);
          vv[fo[a]] = __fsub_rn(vv[fo[a]], __fmul_rn(gs[a], dp));
        }
      } else {
        vv[fo[a]] = kUnknown;
      }
    }
    if (x == R.x - 1) v.c[0][fx + 1] = kUnknown;
    if (y == R.y - 1) v.c[1][fy + ry.x] = kUnknown;
    if (z == R.z - 1) v.c[2][fz + (long long)rz.x * rz.y] = kUnknown;
  }
}
cudaError_t launchGradient(const Geom& g, float gx, float gy, float gz, const uint8_t* markers, const void* p,
                           bool pDouble, FaceField v, ConstFaceField svArr, const SolidVelTable& svTab,
                           cudaStream_t s) {
  if (pDouble)
    kGradient<double><<<gridFor(g.r.size()), kThreads, 0, s>>>(g, gx, gy, gz, markers, (const double*)p, v, svArr,
                                                               svTab);
  else
    kGradient<float><<<gridFor(g.r.size()), kThreads, 0, s>>>(g, gx, gy, gz, markers, (const float*)p, v, svArr,
                                                              svTab);
  return cudaGetLastError();
}

// ===========================================================================
// Extrapolation (EulerSolverTool.cu:450-557, :904-969)
// ===========================================================================
//
// The reference grows UNKNOWN entries layer by layer from the known ones with
// 6-neighbour clamp-to-edge steps, 999 layers at most, then sets every layer-d
// entry to the mean of its neighbours of smaller layer.  Without obstacles the
// layer of an entry equals its L1 distance to the nearest known entry, so the
// layers come from a separable exact L1 distance transform (three 1-D min-plus
// passes); entries are then bucketed by layer and each layer is one launch.

constexpr uint16_t kFar = 0xFFFF;

__global__ void kDistInit(long long n, const float* __restrict__ v, uint16_t* __restrict__ d) {
  HFG_FOR(i, n) d[i] = (v[i] == kUnknown) ? kFar : 0;
}

__device__ inline uint16_t satInc(uint16_t a) { return a >= kFar - 1 ? kFar : (uint16_t)(a + 1); }

// 1-D pass along x: one warp per row, 32 entries at a time.  The forward
// sweep f[i] = min(d[i], f[i-1] + 1) is a warp prefix-min of d[j] - j plus the
// carry from the previous chunk; the backward sweep mirrors it.
__global__ void kDistRows(Dim3i r, uint16_t* __restrict__ d) {
  constexpr int BIG = 1 << 20;
  const int lane = threadIdx.x & 31;
  long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  long long rows = (long long)r.y * r.z;
  for (long long row = wid; row < rows; row += nw) {
    uint16_t* q = d + row * r.x;
    int carry = BIG;
    for (int s0 = 0; s0 < r.x; s0 += 32) {
      int i = s0 + lane;
      int v = i < r.x ? (q[i] == kFar ? BIG : (int)q[i]) : BIG;
      int a = v - lane;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, a, o);
        if (lane >= o) a = min(a, t);
      }
      int f = min(a + lane, carry + lane + 1);
      if (i < r.x) q[i] = (uint16_t)min(f, (int)kFar);
      carry = __shfl_sync(0xffffffffu, f, 31);
    }
    carry = BIG;
    int last = ((r.x - 1) / 32) * 32;
    for (int s0 = last; s0 >= 0; s0 -= 32) {
      int i = s0 + lane;
      int v = i < r.x ? (q[i] == kFar ? BIG : (int)q[i]) : BIG;
      int b = v + lane;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_down_sync(0xffffffffu, b, o);
        if (lane + o < 32) b = min(b, t);
      }
      int g = min(b - lane, carry + (32 - lane));
      if (i < r.x) q[i] = (uint16_t)min(g, (int)kFar);
      carry = __shfl_sync(0xffffffffu, g, 0);
    }
  }
}

// 1-D pass along y or z: threads walk columns, coalesced across x.
__global__ void kDistCols(Dim3i r, int axis, uint16_t* __restrict__ d) {
  long long stride = axis == 1 ? r.x : (long long)r.x * r.y;
  int len = axis == 1 ? r.y : r.z;
  long long lines = axis == 1 ? (long long)r.x * r.z : (long long)r.x * r.y;
  HFG_FOR(l, lines) {
    long long base;
    if (axis == 1) {
      long long x = l % r.x, z = l / r.x;
      base = z * r.x * (long long)r.y + x;
    } else {
      base = l;
    }
    // the column in batches of B: the B loads of a batch are in flight
    // together, then the batch is relaxed in order
    constexpr int B = 8;
    uint16_t* col = d + base;
    uint16_t prev = kFar;
    for (int i0 = 0; i0 < len; i0 += B) {
      uint16_t v[B];
#pragma unroll
      for (int k = 0; k < B; ++k) v[k] = i0 + k < len ? col[(long long)(i0 + k) * stride] : kFar;
#pragma unroll
      for (int k = 0; k < B; ++k) {
        if (i0 + k < len) {
          const uint16_t cand = satInc(prev);
          if (cand < v[k]) {
            v[k] = cand;
            col[(long long)(i0 + k) * stride] = cand;
          }
          prev = v[k];
        }
      }
    }
    prev = kFar;
    for (int i0 = len - 1; i0 >= 0; i0 -= B) {
      uint16_t v[B];
#pragma unroll
      for (int k = 0; k < B; ++k) v[k] = i0 - k >= 0 ? col[(long long)(i0 - k) * stride] : kFar;
#pragma unroll
      for (int k = 0; k < B; ++k) {
        if (i0 - k >= 0) {
          const uint16_t cand = satInc(prev);
          if (cand < v[k]) {
            v[k] = cand;
            col[(long long)(i0 - k) * stride] = cand;
          }
          prev = v[k];
        }
      }
    }
  }
}

// Histogram of layers 1..nums-1 (layers >= nums stay UNKNOWN).
__global__ void kDistHist(long long n, const uint16_t* __restrict__ d, int nums, unsigned int* __restrict__ hist) {
  __shared__ unsigned int sh[kMaxLayers + 1];
  for (int i = threadIdx.x; i <= kMaxLayers; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  HFG_FOR(i, n) {
    uint16_t v = d[i];
    if (v >= 1 && v < nums) atomicAdd(&sh[v], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i <= kMaxLayers; i += blockDim.x)
    if (sh[i]) atomicAdd(hist + i, sh[i]);
}

__global__ void kExclusiveScanSmall(const unsigned int* __restrict__ hist, unsigned int* __restrict__ off,
                                    unsigned int* __restrict__ cursor, int n) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    unsigned int s = 0;
    for (int i = 0; i < n; ++i) { off[i] = s; cursor[i] = s; s += hist[i]; }
    off[n] = s;
  }
}

// Neighbours of entry i of grid r in the order left, right, down, up, back,
// front, clamped to the grid (an edge entry is its own neighbour there).
__device__ __forceinline__ void extrapNeighbours(const Dim3i& r, unsigned i, unsigned nb[6]) {
  const unsigned nx = (unsigned)r.x, ny = (unsigned)r.y, t = i / nx;
  const int x = (int)(i - t * nx), y = (int)(t % ny), z = (int)(t / ny);
  const unsigned plane = nx * ny;
  nb[0] = x > 0 ? i - 1 : i;
  nb[1] = x + 1 < r.x ? i + 1 : i;
  nb[2] = y > 0 ? i - nx : i;
  nb[3] = y + 1 < r.y ? i + nx : i;
  nb[4] = z > 0 ? i - plane : i;
  nb[5] = z + 1 < r.z ? i + plane : i;
}

// Bucket the entries by layer: a block counts its chunk per layer in shared
// memory, reserves one global range per (block, layer) and hands out slots
// with shared-memory atomics.  Each entry also gets the mask of its
// neighbours in earlier layers, so that the layer pass reads no distances.
constexpr int kScatterChunk = 4096;
__global__ void kDistScatter(Dim3i r, long long base, const uint16_t* __restrict__ d, int nums,
                             unsigned int* __restrict__ cursor, unsigned int* __restrict__ list,
                             uint8_t* __restrict__ mask) {
  const long long n = r.size();
  __shared__ unsigned int cnt[kMaxLayers + 1], start[kMaxLayers + 1];
  for (long long c0 = (long long)blockIdx.x * kScatterChunk; c0 < n; c0 += (long long)gridDim.x * kScatterChunk) {
    long long c1 = c0 + kScatterChunk < n ? c0 + kScatterChunk : n;
    for (int i = threadIdx.x; i <= kMaxLayers; i += blockDim.x) cnt[i] = 0;
    __syncthreads();
    for (long long i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
      unsigned int v = d[i];
      if (v >= 1 && (int)v < nums) atomicAdd(&cnt[v], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= kMaxLayers; i += blockDim.x) {
      unsigned int k = cnt[i];
      start[i] = k ? atomicAdd(cursor + i, k) : 0u;
      cnt[i] = 0;
    }
    __syncthreads();
    for (long long i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
      unsigned int v = d[i];
      if (v >= 1 && (int)v < nums) {
        unsigned nb[6];
        extrapNeighbours(r, (unsigned)i, nb);
        unsigned m = 0;
#pragma unroll
        for (int q = 0; q < 6; ++q) m |= (unsigned)(d[nb[q]] < v) << q;
        const unsigned slot = start[v] + atomicAdd(&cnt[v], 1u);
        list[slot] = (unsigned int)(base + i);
        mask[slot] = (uint8_t)m;
      }
    }
    __syncthreads();
  }
}

cudaError_t launchExtrapDistance(const Dim3i rc[3], float* const vals[3], long long off[3], int nums,
                                 ExtrapScratch sc, cudaStream_t s) {
  if (nums > kMaxLayers) nums = kMaxLayers;
  for (int a = 0; a < 3; ++a) {
    long long n = rc[a].size();
    uint16_t* d = sc.dist + off[a];
    kDistInit<<<gridFor(n), kThreads, 0, s>>>(n, vals[a], d);
    kDistRows<<<gridFor((long long)rc[a].y * rc[a].z * 32), kThreads, 0, s>>>(rc[a], d);
    kDistCols<<<gridFor((long long)rc[a].x * rc[a].z), kThreads, 0, s>>>(rc[a], 1, d);
    kDistCols<<<gridFor((long long)rc[a].x * rc[a].y), kThreads, 0, s>>>(rc[a], 2, d);
  }
  cudaError_t e = cudaMemsetAsync(sc.hist, 0, sizeof(unsigned int) * kExtrapHistWords, s);
  if (e != cudaSuccess) return e;
  for (int a = 0; a < 3; ++a) {
    long long n = rc[a].size();
    kDistHist<<<gridFor(n, kThreads, 4), kThreads, 0, s>>>(n, sc.dist + off[a], nums, sc.hist);
  }
  kExclusiveScanSmall<<<1, 1, 0, s>>>(sc.hist, sc.offsets, sc.cursor, kMaxLayers + 1);
  for (int a = 0; a < 3; ++a) {
    long long n = rc[a].size();
    int blocks = (int)std::min<long long>((n + kScatterChunk - 1) / kScatterChunk, (long long)numSMs() * 8);
    if (blocks < 1) blocks = 1;
    kDistScatter<<<blocks, kThreads, 0, s>>>(rc[a], off[a], sc.dist + off[a], nums, sc.cursor, sc.list, sc.mask);
  }
  return cudaGetLastError();
}

// One entry of layer d: mean of the neighbours with a smaller layer (mask m),
// summed in the fixed order left, right, down, up, back, front
// (extrapolatingData).
// The values of earlier layers were written by other blocks of the same
// launch, so they are read from L2 (ld.cg), never from a stale L1 line.
// 32-bit index arithmetic: every face grid holds fewer than 2^31 entries.
__device__ __forceinline__ void extrapEntry(const Dim3i& r0, const Dim3i& r1, const Dim3i& r2, float* v0, float* v1,
                                            float* v2, unsigned off1, unsigned off2, unsigned id, unsigned m) {
  const int a = id >= off2 ? 2 : (id >= off1 ? 1 : 0);
  const unsigned base = a == 2 ? off2 : (a == 1 ? off1 : 0u);
  const unsigned i = id - base;
  const Dim3i r = a == 2 ? r2 : (a == 1 ? r1 : r0);
  float* v = a == 2 ? v2 : (a == 1 ? v1 : v0);
  unsigned nb[6];
  extrapNeighbours(r, i, nb);
  float acc = 0.f, cnt = 0.f;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    if ((m >> q) & 1u) {
      acc = __fadd_rn(acc, __ldcg(v + nb[q]));
      cnt = __fadd_rn(cnt, 1.f);
    }
  }
  if (cnt != 0.f) acc = __fdiv_rn(acc, cnt);
  v[i] = acc;
}

// Block shape of the layer pass: 512 threads, at most two blocks per SM
// (fewer, larger blocks than 256 x 4 meet at the grid barriers sooner).
constexpr int kExtrapThreads = 512, kExtrapPerSM = 2;

// Layers 1 .. nums-1, persistent: a layer with more than kExtrapSmallLayer
// faces is spread over the grid; a run of smaller consecutive layers is filled
// by block 0 alone with block barriers between them.  Every block walks the
// same layer bounds (sc.offsets), so all meet at the same grid barriers.
// barWords: count, generation, error, deepest layer filled.
__global__ void __launch_bounds__(kExtrapThreads)
    kExtrapLayers(Dim3i r0, Dim3i r1, Dim3i r2, float* v0, float* v1, float* v2, unsigned off1, unsigned off2,
                  const uint8_t* __restrict__ mask, const unsigned int* __restrict__ list,
                  const unsigned int* __restrict__ offsets, int nums, unsigned* barWords) {
  unsigned* count = barWords;
  unsigned* gen = barWords + 1;
  unsigned* err = barWords + 2;
  const unsigned stride = gridDim.x * blockDim.x, gtid = blockIdx.x * blockDim.x + threadIdx.x;
  int d = 1;
  while (d < nums && d <= kMaxLayers) {
    if (blockIdx.x == 0 && threadIdx.x == 0) barWords[3] = (unsigned)(d - 1);
    const unsigned b = __ldg(offsets + d), e = __ldg(offsets + d + 1);
    if (e <= b) break;
    if (e - b > kExtrapSmallLayer) {
      for (unsigned k = b + gtid; k < e; k += stride) extrapEntry(r0, r1, r2, v0, v1, v2, off1, off2, list[k], mask[k]);
      ++d;
    } else {
      int last = d;
      while (last + 1 < nums && last + 1 <= kMaxLayers) {
        const unsigned nb = __ldg(offsets + last + 1), ne = __ldg(offsets + last + 2);
        if (ne <= nb || ne - nb > kExtrapSmallLayer) break;
        ++last;
      }
      if (blockIdx.x == 0) {
        for (int l = d; l <= last; ++l) {
          const unsigned lb = __ldg(offsets + l), le = __ldg(offsets + l + 1);
          for (unsigned k = lb + threadIdx.x; k < le; k += blockDim.x)
            extrapEntry(r0, r1, r2, v0, v1, v2, off1, off2, list[k], mask[k]);
          __syncthreads();
        }
      }
      d = last + 1;
    }
    if (gridDim.x > 1 && !gridBarrier(count, gen, err, gridDim.x)) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) barWords[3] = (unsigned)(d - 1);
}

namespace {
std::atomic<int> g_extrapUsers{0};
}
void extrapUsers(int delta) { g_extrapUsers.fetch_add(delta); }

// Layers 1 .. nums-1 in one cooperative launch: about one block per 8192
// faces of the grids, at most kExtrapPerSM per SM, and at most an equal
// share of the GPU's resident slots for this kernel among the registered
// users, so that the grids of concurrent scenes always fit on the GPU
// together.
cudaError_t launchExtrapLayers(const Dim3i rc[3], float* const vals[3], const long long off[3], ExtrapScratch sc,
                               int nums, cudaStream_t s, long long* launches) {
  if (nums <= 1) return cudaSuccess;
  static std::atomic<int> perSM{0};
  if (perSM.load() == 0) {
    int v = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kExtrapLayers, kExtrapThreads, 0);
    if (e != cudaSuccess) return e;
    perSM.store(std::max(1, v));
  }
  const long long slots = (long long)numSMs() * perSM.load();
  const long long share = std::max(1LL, slots / std::max(1, g_extrapUsers.load()));
  const long long faces = rc[0].size() + rc[1].size() + rc[2].size();
  const int blocks = (int)std::max(
      1LL,
      std::min({(faces + 8191) / 8192, (long long)numSMs() * std::min(perSM.load(), kExtrapPerSM), share}));
  Dim3i r0 = rc[0], r1 = rc[1], r2 = rc[2];
  float *v0 = vals[0], *v1 = vals[1], *v2 = vals[2];
  unsigned o1 = (unsigned)off[1], o2 = (unsigned)off[2];
  const uint8_t* mask = sc.mask;
  const unsigned int* list = sc.list;
  const unsigned int* offs = sc.offsets;
  unsigned* bar = extrapBarWords(sc);
  void* args[] = {&r0, &r1, &r2, &v0, &v1, &v2, &o1, &o2, &mask, &list, &offs, &nums, &bar};
  cudaError_t e =
      cudaLaunchCooperativeKernel((const void*)kExtrapLayers, dim3(blocks), dim3(kExtrapThreads), args, 0, s);
  if (e == cudaSuccess && launches) ++*launches;
  return e;
}

// One warp copies `words` 32-bit words (small state read-backs into mapped
// host memory).
__global__ void kCopyWords(const unsigned* __restrict__ src, unsigned* __restrict__ dst, int words) {
  for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
}
cudaError_t launchCopyWords(const unsigned* src, unsigned* dst, int words, cudaStream_t s) {
  kCopyWords<<<1, 32, 0, s>>>(src, dst, words);
  return cudaGetLastError();
}

// ===========================================================================
// Fluid SDF of the fluid-domain field (buildFluidSDF, EulerSolverTool.cu:324-406,
// :760-785; GridFluidSolver.cpp:571-591).  Layer 0 marks the cells on both
// sides of the fluid surface (0.5 - 0.2 inside, 1.5 - 0.2 outside, +/-UNKNOWN
// elsewhere); layer d then takes every still-UNKNOWN neighbour of a layer d-1
// cell of the same side.  The reference sweeps the whole grid 1000 times;
// here each layer visits only the previous layer's cells (frontier lists).
// ===========================================================================
namespace {
constexpr double kSurf = 0.2;  // FluidSurfaceDensity (Common.h:244)
__device__ __forceinline__ float outsideValue(int d) { return (float)((double)d + (1.5 - kSurf)); }
__device__ __forceinline__ float insideValue(int d) { return d == 0 ? (float)(0.5 - kSurf) : (float)(-((double)d - (0.5 - kSurf))); }
}  // namespace

__global__ void kFluidSdfInit(Dim3i r, const float* __restrict__ dom, float* __restrict__ sdf,
                              unsigned int* __restrict__ front, unsigned int* __restrict__ count) {
  HFG_FOR(c, r.size()) {
    int x, y, z;
    cellCoord(c, r, x, y, z);
    bool in = dom[c] < 0.f;
    bool mixed = false;
    const int dx[6] = {-1, 1, 0, 0, 0, 0}, dy[6] = {0, 0, -1, 1, 0, 0}, dz[6] = {0, 0, 0, 0, -1, 1};
#pragma unroll
    for (int k = 0; k < 6; ++k) mixed |= ((dom[linc(x + dx[k], y + dy[k], z + dz[k], r)] < 0.f) != in);
    float v = in ? (mixed ? insideValue(0) : -kUnknown) : (mixed ? outsideValue(0) : kUnknown);
    sdf[c] = v;
    if (mixed) front[atomicAdd(count, 1u)] = (unsigned int)c;
  }
}

__global__ void kFluidSdfLayer(Dim3i r, float* __restrict__ sdf, const unsigned int* __restrict__ front,
                               unsigned int n, unsigned int* __restrict__ next, unsigned int* __restrict__ count, int d) {
  HFG_FOR(i, (long long)n) {
    long long c = front[i];
    int x, y, z;
    cellCoord(c, r, x, y, z);
    bool inside = sdf[c] < 1.0f;  // inner values are <= 0.3, outer >= 1.3
    float sentinel = inside ? -kUnknown : kUnknown;
    float v = inside ? insideValue(d) : outsideValue(d);
    const int dx[6] = {-1, 1, 0, 0, 0, 0}, dy[6] = {0, 0, -1, 1, 0, 0}, dz[6] = {0, 0, 0, 0, -1, 1};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      long long nb = linc(x + dx[k], y + dy[k], z + dz[k], r);
      int old = atomicCAS((int*)(sdf + nb), __float_as_int(sentinel), __float_as_int(v));
      if (old == __float_as_int(sentinel)) next[atomicAdd(count, 1u)] = (unsigned int)nb;
    }
  }
}

// buildFluidDensity (EulerSolverTool.cu:408-448): 1 inside the fluid, the
// surface density 0.2 where a 6-neighbour (clamp-to-edge) is air, 0 outside
// the fluid or inside a solid.  A cell is air when neither the fluid domain
// nor the solid is negative there (isInsideAir, EulerMathTool.cu:344-348).
__global__ void kFluidDensity(Dim3i r, const float* __restrict__ dom, const float* __restrict__ solidSdf,
                              const uint8_t* __restrict__ solidIdx, float* __restrict__ out) {
  HFG_FOR(c, r.size()) {
    int x, y, z;
    cellCoord(c, r, x, y, z);
    auto solidAt = [&](long long i) { return solidSdf ? solidSdf[i] < 0.f : solidIdx[i] != 0; };
    float v = 0.f;
    if (dom[c] < 0.f && !solidAt(c)) {
      const int dx[6] = {-1, 1, 0, 0, 0, 0}, dy[6] = {0, 0, -1, 1, 0, 0}, dz[6] = {0, 0, 0, 0, -1, 1};
      bool air = false;
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        long long nb = linc(x + dx[k], y + dy[k], z + dz[k], r);
        air |= dom[nb] >= 0.f && !solidAt(nb);
      }
      v = air ? (float)0.2 : 1.f;  // FluidSurfaceDensity (Common.h:244)
    }
    out[c] = v;
  }
}
cudaError_t launchFluidDensity(const Dim3i& r, const float* dom, const float* solidSdf, const uint8_t* solidIdx,
                               float* out, cudaStream_t s) {
  kFluidDensity<<<gridFor(r.size()), kThreads, 0, s>>>(r, dom, solidSdf, solidIdx, out);
  return cudaGetLastError();
}

// Grid <-> particle mixing of the hybrid coupler.
// HybridSimulatorMixFieldWithDensity.cu:6-265: B := (wA A + wB B) / (wA + wB)
// where wA + wB > FLT_EPSILON; on a face grid the weights are the means of the
// two adjacent cells (clamp to edge), scaled by the reference's double 0.5.
__device__ __forceinline__ void mixOne(float a, float& b, float wa, float wb) {
  float s = __fadd_rn(wa, wb);
  if (s > FLT_EPSILON) b = __fdiv_rn(__fadd_rn(__fmul_rn(wa, a), __fmul_rn(wb, b)), s);
}
__global__ void kMixCell(long long n, const float* __restrict__ a, float* __restrict__ b, const float* __restrict__ wa,
                         const float* __restrict__ wb) {
  HFG_FOR(i, n) {
    float v = b[i];
    mixOne(a[i], v, wa[i], wb[i]);
    b[i] = v;
  }
}
__global__ void kMixFace(Dim3i r, int axis, const float* __restrict__ a, float* __restrict__ b,
                         const float* __restrict__ wa, const float* __restrict__ wb) {
  const Dim3i f{r.x + (axis == 0), r.y + (axis == 1), r.z + (axis == 2)};
  HFG_FOR(c, f.size()) {
    int x, y, z;
    cellCoord(c, f, x, y, z);
    long long lo = linc(x - (axis == 0), y - (axis == 1), z - (axis == 2), r), hi = linc(x, y, z, r);
    float wA = __double2float_rn(__dmul_rn((double)__fadd_rn(wa[lo], wa[hi]), 0.5));
    float wB = __double2float_rn(__dmul_rn((double)__fadd_rn(wb[lo], wb[hi]), 0.5));
    float v = b[c];
    mixOne(a[c], v, wA, wB);
    b[c] = v;
  }
}
cudaError_t launchMixFieldWithDensity(const Dim3i& r, int face, const float* const a[3], float* const b[3],
                                      const float* wa, const float* wb, cudaStream_t s) {
  if (!face) {
    kMixCell<<<gridFor(r.size()), kThreads, 0, s>>>(r.size(), a[0], b[0], wa, wb);
    return cudaGetLastError();
  }
  for (int axis = 0; axis < 3; ++axis) {
    kMixFace<<<gridFor(r.size()), kThreads, 0, s>>>(r, axis, a[axis], b[axis], wa, wb);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}
// HybridSimulatorMixParitcleVelWithPICAndFLIP.cu:5-57: by the particle's
// distance d: PIC up to g cells, PIC -> predicted up to gf, FLIP up to f,
// FLIP -> predicted up to p, predicted beyond (lerp(a, b, t) = a + t (b - a)).
__global__ void kMixParticleVel(const float* __restrict__ pic, const float* __restrict__ flip,
                                const float* __restrict__ dist, long long n, float cell, float g, float gf, float fr,
                                float pr, float* __restrict__ predict) {
  const float dg = __fmul_rn(g, cell), dgf = __fmul_rn(gf, cell), df = __fmul_rn(fr, cell), dp = __fmul_rn(pr, cell);
  HFG_FOR(i, n) {
    const float d = dist[i];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float P = pic[3 * i + a], F = flip[3 * i + a], Q = predict[3 * i + a];
      float m;
      if (d <= dg) m = P;
      else if (d <= dgf) m = __fadd_rn(P, __fmul_rn(__fdiv_rn(__fsub_rn(d, dg), __fsub_rn(dgf, dg)), __fsub_rn(Q, P)));
      else if (d <= df) m = F;
      else if (d <= dp) m = __fadd_rn(F, __fmul_rn(__fdiv_rn(__fsub_rn(d, df), __fsub_rn(dp, df)), __fsub_rn(Q, F)));
      else m = Q;
      predict[3 * i + a] = m;
    }
  }
}
cudaError_t launchMixParticleVel(const float* pic, const float* flip, const float* dist, long long n, float cell,
                                 float g, float gf, float f, float p, float* predict, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  kMixParticleVel<<<gridFor(n), kThreads, 0, s>>>(pic, flip, dist, n, cell, g, gf, f, p, predict);
  return cudaGetLastError();
}

cudaError_t launchFluidSdf(const Dim3i& r, const float* dom, float* sdf, int layers, unsigned int* frontA,
                           unsigned int* frontB, unsigned int* counts, unsigned int* hostCount, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(unsigned int) * 2, s);
  if (e != cudaSuccess) return e;
  kFluidSdfInit<<<gridFor(r.size()), kThreads, 0, s>>>(r, dom, sdf, frontA, counts);
  unsigned int* cur = frontA;
  unsigned int* nxt = frontB;
  int slot = 0;
  for (int d = 1; d < layers; ++d) {
    e = cudaMemcpyAsync(hostCount, counts + slot, sizeof(unsigned int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    unsigned int n = *hostCount;
    if (n == 0) break;
    e = cudaMemsetAsync(counts + (slot ^ 1), 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    kFluidSdfLayer<<<gridFor(n), kThreads, 0, s>>>(r, sdf, cur, n, nxt, counts + (slot ^ 1), d);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    unsigned int* t = cur;
    cur = nxt;
    nxt = t;
    slot ^= 1;
  }
  return cudaGetLastError();
}

// ===========================================================================
// Inside / outside distance fields of the fluid density (the hybrid
// coupler's buildFluidInsideSDF / buildFluidOutsideSDF,
// HybridSimulatorBuildSDF.cu:4-146,177-238).  Sweep 0 gives solids 0,
// surface cells (density 0.2) the seed value s (0.2 - 0.5 inside, 0.5 - 0.2
// outside), cells of density 0 (inside) or 1 (outside) 0 and the rest
// UNKNOWN; sweep d then gives every UNKNOWN 6-neighbour of a cell holding
// d - 1 + s the value d + s, and negative values end as 0.  The reference
// sweeps the whole grid `distance` times; here each sweep visits the
// previous shell only (frontier lists, as launchFluidSdf).
// ===========================================================================
namespace {
__device__ __forceinline__ bool realEq(float a, float b) { return fabsf(__fsub_rn(a, b)) < FLT_MIN; }  // isRealEQ
}  // namespace

__global__ void kSideSdfInit(Dim3i r, const float* __restrict__ density, const float* __restrict__ solid,
                             float seed, float zero, float* __restrict__ out, unsigned int* __restrict__ front,
                             unsigned int* __restrict__ count) {
  HFG_FOR(c, r.size()) {
    const float rho = density[c];
    float v = kUnknown;
    bool surface = false;
    if (solid[c] < 0.f) {
      v = 0.f;
    } else if (realEq(rho, (float)kSurf)) {
      v = seed;
      surface = true;
    } else if (realEq(rho, zero)) {
      v = 0.f;
    }
    out[c] = v;
    if (surface) front[atomicAdd(count, 1u)] = (unsigned int)c;
  }
}

__global__ void kSideSdfLayer(Dim3i r, float* __restrict__ out, const unsigned int* __restrict__ front, unsigned int n,
                              unsigned int* __restrict__ next, unsigned int* __restrict__ count, float v) {
  HFG_FOR(i, (long long)n) {
    const long long c = front[i];
    int x, y, z;
    cellCoord(c, r, x, y, z);
    const int dx[6] = {-1, 1, 0, 0, 0, 0}, dy[6] = {0, 0, -1, 1, 0, 0}, dz[6] = {0, 0, 0, 0, -1, 1};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const long long nb = linc(x + dx[k], y + dy[k], z + dz[k], r);
      const int old = atomicCAS((int*)(out + nb), __float_as_int(kUnknown), __float_as_int(v));
      if (old == __float_as_int(kUnknown)) next[atomicAdd(count, 1u)] = (unsigned int)nb;
    }
  }
}

// buildFluidSDFPostProcess (HybridSimulatorBuildSDF.cu:122-137)
__global__ void kNegativeToZero(long long n, float* __restrict__ out) {
  HFG_FOR(i, n) {
    if (out[i] < 0.f) out[i] = 0.f;
  }
}

cudaError_t launchFluidSideSdf(const Dim3i& r, const float* density, const float* solid, bool outside, int distance,
                               float* out, unsigned int* frontA, unsigned int* frontB, unsigned int* counts,
                               unsigned int* hostCount, cudaStream_t s) {
  // the reference's UInt + double expressions, rounded to Real once
  const double seed = outside ? 0.5 - kSurf : kSurf - 0.5;
  if (distance > 0) {
    cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(unsigned int) * 2, s);
    if (e != cudaSuccess) return e;
    kSideSdfInit<<<gridFor(r.size()), kThreads, 0, s>>>(r, density, solid, (float)seed, outside ? 1.f : 0.f, out,
                                                         frontA, counts);
    unsigned int* cur = frontA;
    unsigned int* nxt = frontB;
    int slot = 0;
    for (int d = 1; d < distance; ++d) {
      // sweep d looks for (d + s) - 1; where that is not the value sweep
      // d - 1 wrote, the reference's shell stops growing
      if ((float)((double)d + seed - 1) != (float)((double)(d - 1) + seed)) break;
      e = cudaMemcpyAsync(hostCount, counts + slot, sizeof(unsigned int), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) return e;
      const unsigned int n = *hostCount;
      if (n == 0) break;
      e = cudaMemsetAsync(counts + (slot ^ 1), 0, sizeof(unsigned int), s);
      if (e != cudaSuccess) return e;
      kSideSdfLayer<<<gridFor(n), kThreads, 0, s>>>(r, out, cur, n, nxt, counts + (slot ^ 1),
                                                   (float)((double)d + seed));
      e = cudaGetLastError();
      if (e != cudaSuccess) return e;
      std::swap(cur, nxt);
      slot ^= 1;
    }
  }
  kNegativeToZero<<<gridFor(r.size()), kThreads, 0, s>>>(r.size(), out);
  return cudaGetLastError();
}

// buildMixedFluidOutsideSDF (HybridSimulatorBuildSDF.cu:139-175): at a cell of
// grid density 0.2, 0.5 minus the mixed density (negative -> 0); elsewhere
// the grid fluid's outside distance.
__global__ void kMixedOutsideSdf(long long n, const float* __restrict__ gridDensity,
                                 const float* __restrict__ mixedDensity, const float* __restrict__ gridOutside,
                                 float* __restrict__ out) {
  HFG_FOR(c, n) {
    float v;
    if (realEq(gridDensity[c], (float)kSurf)) {
      v = __double2float_rn(0.5 - (double)mixedDensity[c]);
      if (v < 0.f) v = 0.f;
    } else {
      v = gridOutside[c];
    }
    out[c] = v;
  }
}
cudaError_t launchMixedOutsideSdf(const Dim3i& r, const float* gridDensity, const float* mixedDensity,
                                  const float* gridOutside, float* out, cudaStream_t s) {
  kMixedOutsideSdf<<<gridFor(r.size()), kThreads, 0, s>>>(r.size(), gridDensity, mixedDensity, gridOutside, out);
  return cudaGetLastError();
}

// ===========================================================================
// Particles
// ===========================================================================

// Philox4x32-10 (Salmon et al., SC'11): counter-based stream shared with the
// host so the seeding is reproducible anywhere.
__host__ __device__ inline void philox10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
    c[1] = (uint32_t)p1;
    c[3] = (uint32_t)p0;
    c[0] = n0;
    c[2] = n2;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}
__device__ inline float unit24(uint32_t v) { return (float)(v >> 8) * (1.0f / 16777216.0f); }

// EulerParticlesTool.cu:5-25 findFluidGrid: fluid SDF < 0 and not solid.
__device__ inline bool seedCell(const float* fsdf, const uint8_t* sidx, long long c) {
  return fsdf[c] < 0.f && !(sidx && sidx[c]);
}

__global__ void kSeedCount(long long n, const float* __restrict__ fsdf, const uint8_t* __restrict__ sidx,
                           unsigned int* __restrict__ blockCounts, int cellsPerBlock) {
  long long b0 = (long long)blockIdx.x * cellsPerBlock;
  unsigned int cnt = 0;
  for (long long c = b0 + threadIdx.x; c < b0 + cellsPerBlock && c < n; c += blockDim.x) cnt += seedCell(fsdf, sidx, c);
  cnt = __reduce_add_sync(0xffffffffu, cnt);
  __shared__ unsigned int s[32];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int t = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += s[i];
    blockCounts[blockIdx.x] = t;
  }
}
cudaError_t launchSeedCount(const Dim3i& r, const float* fluidSDF, const uint8_t* solidIdx, unsigned int* blockCounts,
                            int cellsPerBlock, cudaStream_t s) {
  long long n = r.size();
  int nb = (int)((n + cellsPerBlock - 1) / cellsPerBlock);
  kSeedCount<<<nb, kThreads, 0, s>>>(n, fluidSDF, solidIdx, blockCounts, cellsPerBlock);
  return cudaGetLastError();
}

__global__ void kSeedScan(unsigned int* counts, int n, unsigned long long* total) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    unsigned long long s = 0;
    for (int i = 0; i < n; ++i) { unsigned int c = counts[i]; counts[i] = (unsigned int)s; s += c; }
    *total = s;
  }
}
cudaError_t launchSeedScan(unsigned int* blockCounts, int nBlocks, unsigned long long* total, cudaStream_t s) {
  kSeedScan<<<1, 1, 0, s>>>(blockCounts, nBlocks, total);
  return cudaGetLastError();
}

// EulerParticles.cpp:156-176: particle k of the f-th fluid cell (cells in
// linear order) at ((x + u) h + o) with u from Philox(cell, k; seed).
__global__ void kSeedWrite(Geom g, const float* __restrict__ fsdf, const uint8_t* __restrict__ sidx,
                           const unsigned int* __restrict__ blockOff, int cellsPerBlock, int ppc,
                           unsigned long long seed, float* __restrict__ pos) {
  long long n = g.r.size();
  long long b0 = (long long)blockIdx.x * cellsPerBlock;
  __shared__ unsigned int warpBase[32];
  __shared__ unsigned int runBase;
  if (threadIdx.x == 0) runBase = blockOff[blockIdx.x];
  __syncthreads();
  for (long long c0 = b0; c0 < b0 + cellsPerBlock && c0 < n; c0 += blockDim.x) {
    long long c = c0 + threadIdx.x;
    bool f = c < b0 + cellsPerBlock && c < n && seedCell(fsdf, sidx, c);
    unsigned int ball = __ballot_sync(0xffffffffu, f);
    unsigned int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) warpBase[w] = __popc(ball);
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned int s = runBase;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) { unsigned int t = warpBase[i]; warpBase[i] = s; s += t; }
      runBase = s;
    }
    __syncthreads();
    if (f) {
      unsigned long long rank = warpBase[w] + __popc(ball & ((1u << lane) - 1u));
      int x, y, z;
      cellCoord(c, g.r, x, y, z);
      for (int k = 0; k < ppc; ++k) {
        uint32_t ctr[4] = {(uint32_t)c, (uint32_t)((unsigned long long)c >> 32), (uint32_t)k, 0u};
        philox10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32));
        float* q = pos + 3 * (rank * ppc + k);
        q[0] = __fadd_rn(__fmul_rn(__fadd_rn((float)x, unit24(ctr[0])), g.hx), g.ox);
        q[1] = __fadd_rn(__fmul_rn(__fadd_rn((float)y, unit24(ctr[1])), g.hy), g.oy);
        q[2] = __fadd_rn(__fmul_rn(__fadd_rn((float)z, unit24(ctr[2])), g.hz), g.oz);
      }
    }
    __syncthreads();
  }
}
cudaError_t launchSeedWrite(const Geom& g, const float* fluidSDF, const uint8_t* solidIdx,
                            const unsigned int* blockOffsets, int cellsPerBlock, int ppc, unsigned long long seed,
                            float* pos, cudaStream_t s) {
  long long n = g.r.size();
  int nb = (int)((n + cellsPerBlock - 1) / cellsPerBlock);
  kSeedWrite<<<nb, kThreads, 0, s>>>(g, fluidSDF, solidIdx, blockOffsets, cellsPerBlock, ppc, seed, pos);
  return cudaGetLastError();
}

// Particle velocity update before advection:
//   PIC  (ParticleInCell.cpp:102-104):       v = G2P(vin)
//   FLIP (FluidImplicitParticle.cpp:107-119): v += G2P(vin - prev)
//   MIX  (MixPICAndFLIP.cpp:112-129):        v = (1-m)(v + G2P(vin - prev)) + m G2P(vin)
// with prev = the previous step's P2G output, or prev = 0 on the first FLIP step.
template <int ALG>
__global__ void kParticleVelUpdate(Geom g, int mode, ConstFaceField vin, ConstFaceField prev, int first, float mixing,
                                   const float* __restrict__ pos, float* __restrict__ vel, long long P) {
  const float keep = (float)(1.0 - (double)mixing);
  HFG_FOR(p, P) {
    float px = pos[3 * p], py = pos[3 * p + 1], pz = pos[3 * p + 2];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      Geom fg = faceGeom(g, a);
      float v = vel[3 * p + a];
      if (mode == MODE_PIC) {
        v = g2p<ALG>(vin.c[a], fg, px, py, pz);
      } else {
        float pic = (mode == MODE_MIX) ? g2p<ALG>(vin.c[a], fg, px, py, pz) : 0.f;
        float dv;
        if (first) {
          dv = g2p<ALG>(vin.c[a], fg, px, py, pz);
        } else {
          // G2P of the face-wise difference vin - prev
          Taps t;
          taps<ALG == G2PNEAREST ? LINEAR : ALG>(fg, px, py, pz, t);
          constexpr int n = TapsN<ALG>::n, sft = TapsN<ALG>::shift;
          dv = 0.f;
          if (ALG == G2PNEAREST) {
            long long i = binCell(fg, px, py, pz);
            dv = __fsub_rn(__ldg(vin.c[a] + i), __ldg(prev.c[a] + i));
          } else {
#pragma unroll
            for (int z = 0; z < n; ++z)
#pragma unroll
              for (int y = 0; y < n; ++y)
#pragma unroll
                for (int x = 0; x < n; ++x) {
                  float w = t.w[0][x] * t.w[1][y] * t.w[2][z];
                  long long i = linc(t.base[0] + x + sft, t.base[1] + y + sft, t.base[2] + z + sft, fg.r);
                  dv += w * __fsub_rn(__ldg(vin.c[a] + i), __ldg(prev.c[a] + i));
                }
          }
        }
        v = __fadd_rn(dv, v);
        if (mode == MODE_MIX) {
          v = __fmul_rn(v, keep);
          v = fmaf(mixing, pic, v);
        }
      }
      vel[3 * p + a] = v;
    }
  }
}

__device__ inline void blockMaxToGlobal(float m, unsigned int* dst);

// LINEAR transfers (the configuration of every benchmark scene), fused with the
// first velocity sample of the substep loop that follows
// (EulerParticles.cpp:249-251): one sampler per particle serves the PIC sample,
// the FLIP difference and all three components.  The PIC sample comes from the
// corner tables of vin and is also v0 of the substeps, with max |v0|.
template <typename I>
__global__ void kParticleVelUpdateLinear(Geom g, int mode, FaceQuads vinQ, ConstFaceField vin, ConstFaceField prev,
                                         int first, float mixing, const float* __restrict__ pos,
                                         float* __restrict__ vel, long long P, float* __restrict__ v0,
                                         SubstepState* st) {
  const float keep = (float)(1.0 - (double)mixing);
  const I stride = (I)gridDim.x * blockDim.x;
  float m = 0.f;
  HFG_FOR_T(I, p, P) {
    if (p + stride < (I)P) {  // the next iteration's lines (two or four ahead gained less)
      prefetchL2(pos + 3 * (p + stride));
      prefetchL2(vel + 3 * (p + stride));
    }
    FaceSampler fs(vinQ, pos[3 * p], pos[3 * p + 1], pos[3 * p + 2], FaceSampler::IndexClamp{});
    float pic[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      pic[a] = fs.sampleQuads(vinQ, a);
      v0[3 * p + a] = pic[a];
      m = fmaxf(m, fabsf(pic[a]));
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float v = vel[3 * p + a];
      if (mode == MODE_PIC) {
        v = pic[a];
      } else {
        float dv = first ? pic[a] : fs.sampleDiff(g, a, vin.c[a], prev.c[a]);
        v = __fadd_rn(dv, v);
        if (mode == MODE_MIX) {
          v = __fmul_rn(v, keep);
          v = fmaf(mixing, pic[a], v);
        }
      }
      vel[3 * p + a] = v;
    }
  }
  blockMaxToGlobal(m, &st[0].maxAbsBits);
}

cudaError_t launchParticleVelUpdate(const Geom& g, int mode, int alg, ConstFaceField vin, ConstFaceField prev,
                                    int firstFlip, float mixing, const float* pos, float* vel, long long P,
                                    cudaStream_t s, const FaceQuads* vinQ, float* v0, SubstepState* st) {
  if (P <= 0) return cudaSuccess;
  int gr = gridFor(P);
  switch (alg) {
    case LINEAR:
      if (!vinQ || !v0 || !st) return cudaErrorInvalidValue;
      if (index32(P))
        kParticleVelUpdateLinear<int><<<gr, kThreads, 0, s>>>(g, mode, *vinQ, vin, prev, firstFlip, mixing, pos, vel,
                                                              P, v0, st);
      else
        kParticleVelUpdateLinear<long long><<<gr, kThreads, 0, s>>>(g, mode, *vinQ, vin, prev, firstFlip, mixing, pos,
                                                                    vel, P, v0, st);
      break;
    case QUADRATIC: kParticleVelUpdate<QUADRATIC><<<gr, kThreads, 0, s>>>(g, mode, vin, prev, firstFlip, mixing, pos, vel, P); break;
    case CUBIC: kParticleVelUpdate<CUBIC><<<gr, kThreads, 0, s>>>(g, mode, vin, prev, firstFlip, mixing, pos, vel, P); break;
    case G2PNEAREST: kParticleVelUpdate<G2PNEAREST><<<gr, kThreads, 0, s>>>(g, mode, vin, prev, firstFlip, mixing, pos, vel, P); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// max of m over the block, then atomically into *dst (bits of a float >= 0)
__device__ inline void blockMaxToGlobal(float m, unsigned int* dst) {
  __shared__ float s[32];
  m = warpMaxF(m);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    int nw = blockDim.x >> 5;
    float v = (int)threadIdx.x < nw ? s[threadIdx.x] : 0.f;
    v = warpMaxF(v);
    if (threadIdx.x == 0) atomicMax(dst, __float_as_uint(v));
  }
}

// Corner tables of the three face grids (FaceQuads), one component per
// blockIdx.y; consecutive threads take consecutive jx.
__global__ void kFaceQuads(Dim3i r, ConstFaceField v, float4* q0, float4* q1, float4* q2) {
  const int a = blockIdx.y;
  const unsigned nx = (unsigned)(r.x + (a == 0)), ny = (unsigned)(r.y + (a == 1)), nz = (unsigned)(r.z + (a == 2));
  const unsigned lx = nx + 1, ly = ny + 1;
  const long long n = (long long)lx * ly * (nz + 2);
  const float* __restrict__ f = a == 0 ? v.c[0] : (a == 1 ? v.c[1] : v.c[2]);
  float4* __restrict__ out = a == 0 ? q0 : (a == 1 ? q1 : q2);
  HFG_FOR(e, n) {
    const unsigned t = (unsigned)(e / lx), jx = (unsigned)(e - (long long)t * lx);
    const unsigned L = t / ly, jy = t - L * ly;
    const unsigned z = L == 0 ? 0 : (L > nz ? nz - 1 : L - 1);
    const unsigned x0 = jx > 0 ? jx - 1 : 0, x1 = jx < nx ? jx : nx - 1;
    const unsigned y0 = jy > 0 ? jy - 1 : 0, y1 = jy < ny ? jy : ny - 1;
    const unsigned b0 = (z * ny + y0) * nx, b1 = (z * ny + y1) * nx;
    const float f00 = __ldg(f + b0 + x0), f01 = __ldg(f + b0 + x1), f10 = __ldg(f + b1 + x0), f11 = __ldg(f + b1 + x1);
    out[e] = make_float4(f00, __fsub_rn(f01, f00), f10, __fsub_rn(f11, f10));
  }
}
long long faceQuadCount(const Dim3i& r, int a) {
  return (long long)(r.x + (a == 0) + 1) * (r.y + (a == 1) + 1) * (r.z + (a == 2) + 2);
}
cudaError_t launchFaceQuads(const Dim3i& r, ConstFaceField v, float4* const out[3], cudaStream_t s) {
  long long n = faceQuadCount(r, 0);
  dim3 grid(gridFor(n), 3);
  kFaceQuads<<<grid, kThreads, 0, s>>>(r, v, out[0], out[1], out[2]);
  return cudaGetLastError();
}

// First velocity sample of the substep loop (EulerParticles.cpp:249-251):
// v0 = trilinear(vel, pos) and max |v0| over every component.
template <typename I>
__global__ void kSubstepBegin(Geom g, FaceQuads vel, const float* __restrict__ pos, float* __restrict__ v0,
                              long long P, SubstepState* st) {
  float m = 0.f;
  HFG_FOR_T(I, p, P) {
    float v[3];
    sampleFaceQuads(vel, pos[3 * p], pos[3 * p + 1], pos[3 * p + 2], v);
    v0[3 * p] = v[0]; v0[3 * p + 1] = v[1]; v0[3 * p + 2] = v[2];
    m = fmaxf(m, fmaxf(fabsf(v[0]), fmaxf(fabsf(v[1]), fabsf(v[2]))));
  }
  blockMaxToGlobal(m, &st[0].maxAbsBits);
}
cudaError_t launchSubstepBegin(const Geom& g, FaceQuads vel, const float* pos, float* v0, long long P,
                               SubstepState* st, cudaStream_t s) {
  if (index32(P))
    kSubstepBegin<int><<<gridFor(P > 0 ? P : 1), kThreads, 0, s>>>(g, vel, pos, v0, P, st);
  else
    kSubstepBegin<long long><<<gridFor(P > 0 ? P : 1), kThreads, 0, s>>>(g, vel, pos, v0, P, st);
  return cudaGetLastError();
}

// Substep size rule of EulerParticles.cpp:253-275, evaluated identically by
// every thread from the slot's state.
__device__ inline float substepSize(const SubstepState& s, float dt, float cfl, float minH, bool& last) {
  float amax = __uint_as_float(s.maxAbsBits);
  float d = (amax != 0.f) ? __fdiv_rn(__fmul_rn(cfl, minH), amax) : dt;
  last = false;
  if (__fadd_rn(s.subTime, d) >= dt) {
    d = __fsub_rn(dt, s.subTime);
    last = true;
  } else if (__fadd_rn(s.subTime, __fmul_rn(2.f, d)) >= dt) {
    d = (float)(0.5 * (double)__fsub_rn(dt, s.subTime));
  }
  return d;
}

// One RK1/2/3 substep (EulerParticles.cpp:277-318).  After the last substep the
// box clamp of fixParticlesPosWithBoundarys (EulerParticlesTool.cu:310-333) is
// applied to the first `nclamp` particles; otherwise the next v0 and its max
// are produced for slot+1.
// One particle's substep: RK1/2/3 from its v0, the box clamp after the last
// substep, otherwise the next v0 sampled and stored; returns max |v0 next|.
template <typename I>
__device__ __forceinline__ float substepParticle(const Geom& g, const FaceQuads& vel, float* __restrict__ pos,
                                                 float* __restrict__ v0, I p, int acc, float ds, float half, float tq,
                                                 float a29, float a39, float a49, bool last, bool clampIt) {
  float q[3] = {pos[3 * p], pos[3 * p + 1], pos[3 * p + 2]};
  float w0[3] = {v0[3 * p], v0[3 * p + 1], v0[3 * p + 2]};
  float m = 0.f;
  QuadCache qc;
  bool fresh = true;  // no entry cached yet
  if (acc == 0) {
#pragma unroll
    for (int a = 0; a < 3; ++a) q[a] = fmaf(ds, w0[a], q[a]);
  } else if (acc == 1) {
    float mid[3], w1[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) mid[a] = fmaf(half, w0[a], q[a]);
    sampleFaceQuadsCached(vel, mid[0], mid[1], mid[2], w1, qc, true);
    fresh = false;
#pragma unroll
    for (int a = 0; a < 3; ++a) q[a] = fmaf(ds, w1[a], q[a]);
  } else {
    // q + a29 w0 + a39 w1 + a49 w2, in that order, accumulated as soon as
    // each sample is known so that fewer values stay live across a sample
    float mid[3], tf[3], acc3[3], w[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      mid[a] = fmaf(half, w0[a], q[a]);
      acc3[a] = fmaf(a29, w0[a], q[a]);
    }
    sampleFaceQuadsCached(vel, mid[0], mid[1], mid[2], w, qc, true);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      tf[a] = fmaf(tq, w[a], q[a]);
      acc3[a] = fmaf(a39, w[a], acc3[a]);
    }
    sampleFaceQuadsCached(vel, tf[0], tf[1], tf[2], w, qc, false);
    fresh = false;
#pragma unroll
    for (int a = 0; a < 3; ++a) q[a] = fmaf(a49, w[a], acc3[a]);
  }
  if (last) {
    if (clampIt) {  // the box bounds are formed here, from the kernel parameters
      const float bmin[3] = {g.ox, g.oy, g.oz};
      const float bmax[3] = {g.ox + (float)g.r.x * g.hx, g.oy + (float)g.r.y * g.hy, g.oz + (float)g.r.z * g.hz};
#pragma unroll
      for (int a = 0; a < 3; ++a) q[a] = fmaxf(bmin[a], fminf(q[a], bmax[a]));
    }
  } else {
    float v[3];
    sampleFaceQuadsCached(vel, q[0], q[1], q[2], v, qc, fresh);
    v0[3 * p] = v[0]; v0[3 * p + 1] = v[1]; v0[3 * p + 2] = v[2];
    m = fmaxf(fabsf(v[0]), fmaxf(fabsf(v[1]), fabsf(v[2])));
  }
  pos[3 * p] = q[0]; pos[3 * p + 1] = q[1]; pos[3 * p + 2] = q[2];
  return m;
}

// The RK coefficients of a substep of size ds (EulerParticles.cpp:281-301).
struct SubstepCoef {
  float ds, half, tq, a29, a39, a49;
  SubstepCoef() = default;
  __device__ explicit SubstepCoef(float d)
      : ds(d), half((float)(0.5 * (double)d)), tq((float)(0.75 * (double)d)), a29((float)(2.0 / 9.0 * (double)d)),
        a39((float)(3.0 / 9.0 * (double)d)), a49((float)(4.0 / 9.0 * (double)d)) {}
};

// One RK1/2/3 substep (EulerParticles.cpp:277-318).  After the last substep the
// box clamp of fixParticlesPosWithBoundarys (EulerParticlesTool.cu:310-333) is
// applied to the first `nclamp` particles; otherwise the next v0 and its max
// are produced for slot+1.  ACC: the RK order (0, 1, 2), fixed per
// instantiation so that the particle loop carries no branch on it.
template <typename I, int ACC>
__global__ void __launch_bounds__(256, 4) kSubstep(Geom g, FaceQuads vel, float* __restrict__ pos,
                                                  float* __restrict__ v0, long long P, float dt, float cfl,
                                                  long long nclamp, SubstepState* st, int slot) {
  const SubstepState cur = st[slot];
  if (cur.finished) {
    // carry the finished state forward so later speculative launches no-op
    if (blockIdx.x == 0 && threadIdx.x == 0) st[slot + 1] = cur;
    return;
  }
  // the substep size and RK coefficients, formed once per block: held in
  // shared memory, a use is one load where registers would have to give way
  // to recomputing them (FP64 products) inside the particle loop
  __shared__ SubstepCoef sk;
  __shared__ int sLast;
  if (threadIdx.x == 0) {
    bool l;
    sk = SubstepCoef(substepSize(cur, dt, cfl, fminf(fminf(g.hx, g.hy), g.hz), l));
    sLast = l ? 1 : 0;
  }
  __syncthreads();
  const SubstepCoef& k = sk;
  const bool last = sLast != 0;
  float m = 0.f;
  const I stride = (I)gridDim.x * blockDim.x;
  HFG_FOR_T(I, p, P) {
    // the stream loads of a later iteration are DRAM misses; ask for them now
    // so that the chain of samples below does not start with one
    if (p + stride < (I)P) {
      prefetchL2(pos + 3 * (p + stride));
      prefetchL2(v0 + 3 * (p + stride));
    }
    m = fmaxf(m, substepParticle<I>(g, vel, pos, v0, p, ACC, k.ds, k.half, k.tq, k.a29, k.a39, k.a49, last,
                                    (long long)p < nclamp));
  }
  if (!last) blockMaxToGlobal(m, &st[slot + 1].maxAbsBits);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st[slot + 1].subTime = __fadd_rn(cur.subTime, k.ds);
    st[slot + 1].finished = last ? 1 : 0;
    st[slot + 1].count = cur.count + 1;
  }
}

// The substep `slot` of many scenes in one launch (the batched mode).  Scene
// s owns blocks [chunkStart[s], chunkStart[s + 1]), each a chunk of
// kMultiChunk of its particles; a block finds its scene by binary search and
// runs that scene's substep with the scene's own CFL state, exactly as
// kSubstep would.  Scenes whose substeps are finished do nothing.
constexpr int kMultiChunk = 8 * kThreads;
__global__ void __launch_bounds__(256, 3) kSubstepMulti(const SubstepTask* __restrict__ tasks,
                                                       const long long* __restrict__ chunkStart, int nScenes,
                                                       int slot) {
  __shared__ int sc;
  __shared__ FaceQuads sq;
  if (threadIdx.x == 0) {
    int lo = 0, hi = nScenes - 1;  // the last scene whose first chunk is <= blockIdx.x
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (chunkStart[mid] <= (long long)blockIdx.x) lo = mid;
      else hi = mid - 1;
    }
    sc = lo;
    sq = tasks[lo].vel;
  }
  __syncthreads();
  const SubstepTask& T = tasks[sc];
  const long long chunk = (long long)blockIdx.x - chunkStart[sc];
  const SubstepState cur = T.st[slot];
  if (cur.finished) {
    if (chunk == 0 && threadIdx.x == 0) T.st[slot + 1] = cur;
    return;
  }
  const Geom g = T.g;
  // the scene's tables and sampling constants, read from shared memory where
  // used (held in registers they spill)
  const FaceQuads& vel = sq;
  const float minH = fminf(fminf(g.hx, g.hy), g.hz);
  bool last;
  const SubstepCoef k(substepSize(cur, T.dt, T.cfl, minH, last));
  float m = 0.f;
  // the chunk's particles, indexed in 32 bits from the chunk's start
  const long long p0 = chunk * kMultiChunk;
  const int n = (int)(min(T.P, p0 + kMultiChunk) - p0);
  const long long nclamp = T.nclamp - p0;
  float* pos = T.pos + 3 * p0;
  float* v0 = T.v0 + 3 * p0;
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    m = fmaxf(m, substepParticle<int>(g, vel, pos, v0, i, T.acc, k.ds, k.half, k.tq, k.a29, k.a39, k.a49, last,
                                      (long long)i < nclamp));
  if (!last) blockMaxToGlobal(m, &T.st[slot + 1].maxAbsBits);
  if (chunk == 0 && threadIdx.x == 0) {
    T.st[slot + 1].subTime = __fadd_rn(cur.subTime, k.ds);
    T.st[slot + 1].finished = last ? 1 : 0;
    T.st[slot + 1].count = cur.count + 1;
  }
}
long long multiSubstepChunks(long long P) { return (P + kMultiChunk - 1) / kMultiChunk; }
cudaError_t launchSubstepMulti(const SubstepTask* tasks, const long long* chunkStart, int nScenes,
                               long long totalChunks, int slot, cudaStream_t s) {
  if (nScenes <= 0 || totalChunks <= 0) return cudaSuccess;
  kSubstepMulti<<<(unsigned)totalChunks, kThreads, 0, s>>>(tasks, chunkStart, nScenes, slot);
  return cudaGetLastError();
}

// finished flag and substep count of every scene's state slot `slot`, into
// host-mapped memory (two ints per scene)
__global__ void kGatherSubstepStates(const SubstepTask* __restrict__ tasks, int nScenes, int slot, int* out) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nScenes; s += gridDim.x * blockDim.x) {
    const SubstepState v = tasks[s].st[slot];
    out[2 * s] = v.finished;
    out[2 * s + 1] = v.count;
  }
}
cudaError_t launchGatherSubstepStates(const SubstepTask* tasks, int nScenes, int slot, int* out, cudaStream_t s) {
  if (nScenes <= 0) return cudaSuccess;
  kGatherSubstepStates<<<(nScenes + 255) / 256, 256, 0, s>>>(tasks, nScenes, slot, out);
  return cudaGetLastError();
}

cudaError_t launchSubstep(const Geom& g, FaceQuads vel, float* pos, float* v0, long long P, int acc, float dt,
                          float cfl, long long nclamp, SubstepState* st, int slot, cudaStream_t s) {
  const int grid = gridFor(P > 0 ? P : 1);
#define HFG_SUBSTEP(I, A) kSubstep<I, A><<<grid, kThreads, 0, s>>>(g, vel, pos, v0, P, dt, cfl, nclamp, st, slot)
  if (index32(P)) {
    if (acc == 0) HFG_SUBSTEP(int, 0);
    else if (acc == 1) HFG_SUBSTEP(int, 1);
    else HFG_SUBSTEP(int, 2);
  } else {
    if (acc == 0) HFG_SUBSTEP(long long, 0);
    else if (acc == 1) HFG_SUBSTEP(long long, 1);
    else HFG_SUBSTEP(long long, 2);
  }
#undef HFG_SUBSTEP
  return cudaGetLastError();
}

// P2G of particle velocities to the three face grids, value and weight packed
// as float2 so every corner is one vector atomic
// (accumulateParticles2CCSField, EulerParticlesTool.cu:79-196).
template <int ALG>
__device__ inline void p2gScatter(const Geom& fg, float px, float py, float pz, float val, float2* acc) {
  if (ALG == P2GSUM) {
    atomicAdd(&acc[binCell(fg, px, py, pz)].x, val);
    return;
  }
  Taps t;
  taps<ALG>(fg, px, py, pz, t);
  constexpr int n = TapsN<ALG>::n, s = TapsN<ALG>::shift;
#pragma unroll
  for (int z = 0; z < n; ++z)
#pragma unroll
    for (int y = 0; y < n; ++y)
#pragma unroll
      for (int x = 0; x < n; ++x) {
        float w = t.w[0][x] * t.w[1][y] * t.w[2][z];
        long long i = linc(t.base[0] + x + s, t.base[1] + y + s, t.base[2] + z + s, fg.r);
        atomicAdd(acc + i, make_float2(w * val, w));
      }
}

// LINEAR P2G to the three face grids.  Particles are stored in seeding order
// (the particles of a cell next to each other) and move coherently, so the
// lanes of an aligned pair, quad or octet of a warp often share all eight
// corners of a component.  Such a group first sums its contributions with
// lane shuffles (levels skipped when no lane of the warp merges there), and one
// lane adds the sums to the grid: up to eight times fewer L2 atomics.  The
// sums differ from lane-by-lane atomics in the order of the additions only,
// as the order of the atomics does anyway.
__global__ void kP2GFaceLinear(Geom g, const float* __restrict__ pos, const float* __restrict__ vel, long long P,
                               float2* a0, float2* a1, float2* a2) {
  constexpr unsigned kAll = 0xffffffffu;
  float2* acc[3] = {a0, a1, a2};
  const int lane = threadIdx.x & 31;
  const long long stride = (long long)gridDim.x * blockDim.x;
  // warp-uniform trip count: every lane takes part in the shuffles
  for (long long p0 = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); p0 < P; p0 += stride) {
    const long long p = p0 + lane;
    const bool live = p < P;
    FaceSampler fs(g, live ? pos[3 * p] : g.ox, live ? pos[3 * p + 1] : g.oy, live ? pos[3 * p + 2] : g.oz);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      unsigned idx[8];
      float w[8];
      fs.corners(g, a, idx, w);
      const float val = live ? vel[3 * p + a] : 0.f;
      float vx[8], vw[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        vx[k] = w[k] * val;
        vw[k] = w[k];
      }
      // lanes with the same clamped floor indices (AxisW::j, -1 .. n - 1, which
      // fix both corners of an axis) share all eight corners; the key is
      // their linear index in a grid one larger per axis, less a constant, in
      // 32-bit unsigned arithmetic: distinct triples give distinct keys, and
      // the keys that wrap below zero land above 2^32 - 2^31, never on a dead
      // lane's 0x80000000 | lane
      const AxisW& X = a == 0 ? fs.fc[0] : fs.cc[0];
      const AxisW& Y = a == 1 ? fs.fc[1] : fs.cc[1];
      const AxisW& Z = a == 2 ? fs.fc[2] : fs.cc[2];
      const unsigned lx = (unsigned)(g.r.x + (a == 0) + 1), ly = (unsigned)(g.r.y + (a == 1) + 1);
      const unsigned key = live ? ((unsigned)Z.j * ly + (unsigned)Y.j) * lx + (unsigned)X.j : 0x80000000u | (unsigned)lane;
      const unsigned m = __match_any_sync(kAll, key);
      int group = 1;
#pragma unroll
      for (int lvl = 1; lvl <= 4; lvl <<= 1) {
        const unsigned gm = (lvl == 1 ? 0x3u : (lvl == 2 ? 0xFu : 0xFFu));
        const bool merge = group == lvl && ((m >> (lane & ~(2 * lvl - 1))) & gm) == gm;
        if (!__any_sync(kAll, merge)) break;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const float ox = __shfl_xor_sync(kAll, vx[k], lvl), ow = __shfl_xor_sync(kAll, vw[k], lvl);
          if (merge) {
            vx[k] += ox;
            vw[k] += ow;
          }
        }
        if (merge) group = 2 * lvl;
      }
      if (live && (lane & (group - 1)) == 0) {
#pragma unroll
        for (int k = 0; k < 8; ++k) atomicAdd(acc[a] + idx[k], make_float2(vx[k], vw[k]));
      }
    }
  }
}

template <int ALG>
__global__ void kP2GFace(Geom g, const float* __restrict__ pos, const float* __restrict__ vel, long long P,
                         float2* a0, float2* a1, float2* a2) {
  HFG_FOR(p, P) {
    float px = pos[3 * p], py = pos[3 * p + 1], pz = pos[3 * p + 2];
    p2gScatter<ALG>(faceGeom(g, 0), px, py, pz, vel[3 * p], a0);
    p2gScatter<ALG>(faceGeom(g, 1), px, py, pz, vel[3 * p + 1], a1);
    p2gScatter<ALG>(faceGeom(g, 2), px, py, pz, vel[3 * p + 2], a2);
  }
}
cudaError_t launchP2GFace(const Geom& g, int alg, const float* pos, const float* vel, long long P, float2* acc[3],
                          cudaStream_t s) {
  if (P <= 0) return cudaSuccess;
  int gr = gridFor(P);
  switch (alg) {
    case LINEAR: kP2GFaceLinear<<<gr, kThreads, 0, s>>>(g, pos, vel, P, acc[0], acc[1], acc[2]); break;
    case QUADRATIC: kP2GFace<QUADRATIC><<<gr, kThreads, 0, s>>>(g, pos, vel, P, acc[0], acc[1], acc[2]); break;
    case CUBIC: kP2GFace<CUBIC><<<gr, kThreads, 0, s>>>(g, pos, vel, P, acc[0], acc[1], acc[2]); break;
    case P2GSUM: kP2GFace<P2GSUM><<<gr, kThreads, 0, s>>>(g, pos, vel, P, acc[0], acc[1], acc[2]); break;
    default: break;  // G2PNEAREST has no P2G branch in the reference: nothing is accumulated
  }
  return cudaGetLastError();
}

template <int ALG>
__global__ void kP2GCell(Geom g, const float* __restrict__ pos, const float* __restrict__ val, int span, int comp,
                         long long P, float2* acc) {
  HFG_FOR(p, P) p2gScatter<ALG>(g, pos[3 * p], pos[3 * p + 1], pos[3 * p + 2], val[span * p + comp], acc);
}
cudaError_t launchP2GCell(const Geom& g, int alg, const float* pos, const float* val, int span, int comp, long long P,
                          float2* acc, cudaStream_t s) {
  if (P <= 0) return cudaSuccess;
  int gr = gridFor(P);
  switch (alg) {
    case LINEAR: kP2GCell<LINEAR><<<gr, kThreads, 0, s>>>(g, pos, val, span, comp, P, acc); break;
    case QUADRATIC: kP2GCell<QUADRATIC><<<gr, kThreads, 0, s>>>(g, pos, val, span, comp, P, acc); break;
    case CUBIC: kP2GCell<CUBIC><<<gr, kThreads, 0, s>>>(g, pos, val, span, comp, P, acc); break;
    case P2GSUM: kP2GCell<P2GSUM><<<gr, kThreads, 0, s>>>(g, pos, val, span, comp, P, acc); break;
    default: break;
  }
  return cudaGetLastError();
}

// normalizeCCSField (EulerParticlesTool.cu:290-308) fused with the copy kept
// as the next FLIP "previous grid velocity" (MixPICAndFLIP.cpp:135) and the
// unit-field external-force axpys (ExternalForcesSolver.cpp:57-58).
__global__ void kNormalize(long long n, const float2* __restrict__ acc, float* __restrict__ out, float* __restrict__ copy,
                           float add, int doAdd, float add2, int doAdd2) {
  HFG_FOR(i, n) {
    float2 a = acc[i];
    float v = a.y > 0.f ? __fdiv_rn(a.x, a.y) : a.x;
    if (copy) copy[i] = v;
    if (doAdd) v = __fadd_rn(add, v);
    if (doAdd2) v = __fadd_rn(add2, v);
    out[i] = v;
  }
}
cudaError_t launchNormalize(long long n, const float2* acc, float* out, float* copy, float add, int doAdd, float add2,
                            int doAdd2, cudaStream_t s) {
  kNormalize<<<gridFor(n), kThreads, 0, s>>>(n, acc, out, copy, add, doAdd, add2, doAdd2);
  return cudaGetLastError();
}

template <int ALG>
__global__ void kG2PFace(Geom g, ConstFaceField f, const float* __restrict__ pos, long long P, float* __restrict__ out) {
  HFG_FOR(p, P) {
    float px = pos[3 * p], py = pos[3 * p + 1], pz = pos[3 * p + 2];
#pragma unroll
    for (int a = 0; a < 3; ++a) out[3 * p + a] = g2p<ALG>(f.c[a], faceGeom(g, a), px, py, pz);
  }
}
cudaError_t launchG2PFace(const Geom& g, int alg, ConstFaceField f, const float* pos, long long P, float* out,
                          cudaStream_t s) {
  if (P <= 0) return cudaSuccess;
  int gr = gridFor(P);
  switch (alg) {
    case LINEAR: kG2PFace<LINEAR><<<gr, kThreads, 0, s>>>(g, f, pos, P, out); break;
    case QUADRATIC: kG2PFace<QUADRATIC><<<gr, kThreads, 0, s>>>(g, f, pos, P, out); break;
    case CUBIC: kG2PFace<CUBIC><<<gr, kThreads, 0, s>>>(g, f, pos, P, out); break;
    case G2PNEAREST: kG2PFace<G2PNEAREST><<<gr, kThreads, 0, s>>>(g, f, pos, P, out); break;
    default: return cudaMemsetAsync(out, 0, sizeof(float) * 3 * P, s);  // P2GSUM: G2P writes 0 (:223)
  }
  return cudaGetLastError();
}

template <int ALG>
__global__ void kG2PCell(Geom g, const float* __restrict__ f, const float* __restrict__ pos, long long P,
                         float* __restrict__ out, int span, int comp) {
  HFG_FOR(p, P) out[span * p + comp] = g2p<ALG>(f, g, pos[3 * p], pos[3 * p + 1], pos[3 * p + 2]);
}
cudaError_t launchG2PCell(const Geom& g, int alg, const float* f, const float* pos, long long P, float* out, int span,
                          int comp, cudaStream_t s) {
  if (P <= 0) return cudaSuccess;
  int gr = gridFor(P);
  switch (alg) {
    case LINEAR: kG2PCell<LINEAR><<<gr, kThreads, 0, s>>>(g, f, pos, P, out, span, comp); break;
    case QUADRATIC: kG2PCell<QUADRATIC><<<gr, kThreads, 0, s>>>(g, f, pos, P, out, span, comp); break;
    case CUBIC: kG2PCell<CUBIC><<<gr, kThreads, 0, s>>>(g, f, pos, P, out, span, comp); break;
    case G2PNEAREST: kG2PCell<G2PNEAREST><<<gr, kThreads, 0, s>>>(g, f, pos, P, out, span, comp); break;
    default: break;
  }
  return cudaGetLastError();
}

__global__ void kSampleFace(Geom g, ConstFaceField f, const float* __restrict__ pos, long long M, float* __restrict__ out) {
  HFG_FOR(i, M) {
    float v[3];
    sampleFace(f, g, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], v);
    out[3 * i] = v[0]; out[3 * i + 1] = v[1]; out[3 * i + 2] = v[2];
  }
}
cudaError_t launchSampleFace(const Geom& g, ConstFaceField f, const float* pos, long long M, float* out, cudaStream_t s) {
  if (M <= 0) return cudaSuccess;
  kSampleFace<<<gridFor(M), kThreads, 0, s>>>(g, f, pos, M, out);
  return cudaGetLastError();
}
__global__ void kSampleCell(Geom g, const float* __restrict__ f, const float* __restrict__ pos, long long M,
                            float* __restrict__ out) {
  HFG_FOR(i, M) out[i] = trilerp(f, g, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
}
cudaError_t launchSampleCell(const Geom& g, const float* f, const float* pos, long long M, float* out, cudaStream_t s) {
  if (M <= 0) return cudaSuccess;
  kSampleCell<<<gridFor(M), kThreads, 0, s>>>(g, f, pos, M, out);
  return cudaGetLastError();
}

// ===========================================================================
// Semi-Lagrangian advection (SemiLagrangian.cpp:135-347): back-trace each
// face / cell centre through `vel` with RK1/2/3, then sample the source field
// there.  The position fields and the nine axpys of the reference are fused
// into one pass per output grid.
// ===========================================================================
__device__ inline void axpyPt(float a, const float v[3], float p[3]) {
  if (fabsf(a) < FLT_EPSILON) return;  // plusAlphaX skip
#pragma unroll
  for (int k = 0; k < 3; ++k) p[k] = fmaf(a, v[k], p[k]);
}

template <int SAMP>
__device__ inline void sampleVel(ConstFaceField vel, const Geom& g, float px, float py, float pz, float v[3]) {
  if (SAMP == 0) {
    sampleFaceFast(vel, g, px, py, pz, v);
  } else {
#pragma unroll
    for (int a = 0; a < 3; ++a) v[a] = cubicSample<SAMP>(vel.c[a], faceGeom(g, a), px, py, pz);
  }
}

// CSemiLagrangian::backTrace (SemiLagrangian.cpp:188-347); every velocity
// sample uses the advection's sampling algorithm.
template <int SAMP>
__device__ inline void backTrace(ConstFaceField vel, const Geom& g, float dt, int acc, const float in[3], float out[3]) {
  float v0[3], v1[3], v2[3], mid[3], tf[3];
  out[0] = in[0]; out[1] = in[1]; out[2] = in[2];
  sampleVel<SAMP>(vel, g, in[0], in[1], in[2], v0);
  if (acc == 0) {
    axpyPt(-dt, v0, out);
    return;
  }
  mid[0] = in[0]; mid[1] = in[1]; mid[2] = in[2];
  axpyPt(-0.5f * dt, v0, mid);
  sampleVel<SAMP>(vel, g, mid[0], mid[1], mid[2], v1);
  if (acc == 1) {
    axpyPt(-dt, v1, out);
    return;
  }
  tf[0] = in[0]; tf[1] = in[1]; tf[2] = in[2];
  axpyPt(-0.75f * dt, v1, tf);
  sampleVel<SAMP>(vel, g, tf[0], tf[1], tf[2], v2);
  axpyPt(-(float)(2.0 / 9.0) * dt, v0, out);
  axpyPt(-(float)(3.0 / 9.0) * dt, v1, out);
  axpyPt(-(float)(4.0 / 9.0) * dt, v2, out);
}

template <int SAMP>
__global__ void kSLFace(Geom g, int acc, float dt, ConstFaceField vel, ConstFaceField in, FaceField out, float ax,
                        float ay, float az, int doAdd, float bx, float by, float bz, int doAdd2) {
  const float add[3] = {ax, ay, az}, add2[3] = {bx, by, bz};
  for (int a = 0; a < 3; ++a) {
    Geom fg = faceGeom(g, a);
    HFG_FOR(f, fg.r.size()) {
      int x, y, z;
      cellCoord(f, fg.r, x, y, z);
      // SemiLagrangian.cpp:60-97 sample points
      float p[3] = {__fadd_rn(__fmul_rn(__fadd_rn((float)x, 0.5f), g.hx), g.ox),
                    __fadd_rn(__fmul_rn(__fadd_rn((float)y, 0.5f), g.hy), g.oy),
                    __fadd_rn(__fmul_rn(__fadd_rn((float)z, 0.5f), g.hz), g.oz)};
      if (a == 0) p[0] = __fadd_rn(__fmul_rn((float)x, g.hx), g.ox);
      if (a == 1) p[1] = __fadd_rn(__fmul_rn((float)y, g.hy), g.oy);
      if (a == 2) p[2] = __fadd_rn(__fmul_rn((float)z, g.hz), g.oz);
      float q[3];
      backTrace<SAMP>(vel, g, dt, acc, p, q);
      float v = sampleAlg<SAMP>(in.c[a], fg, q[0], q[1], q[2]);
      if (doAdd) v = __fadd_rn(add[a], v);
      if (doAdd2) v = __fadd_rn(add2[a], v);
      out.c[a][f] = v;
    }
  }
}
cudaError_t launchSLFace(const Geom& g, int acc, float dt, ConstFaceField vel, ConstFaceField in, FaceField out,
                         const float add[3], int doAdd, const float add2[3], int doAdd2, cudaStream_t s,
                         int sampling) {
#define HFG_SL_FACE(S)                                                                                              \
  kSLFace<S><<<gridFor(g.r.size()), kThreads, 0, s>>>(g, acc, dt, vel, in, out, add[0], add[1], add[2], doAdd,      \
                                                      add2[0], add2[1], add2[2], doAdd2)
  switch (sampling) {
    case 1: HFG_SL_FACE(1); break;
    case 2: HFG_SL_FACE(2); break;
    case 3: HFG_SL_FACE(3); break;
    case 4: HFG_SL_FACE(4); break;
    default: HFG_SL_FACE(0);
  }
#undef HFG_SL_FACE
  return cudaGetLastError();
}

struct CellFields {
  const float* in[4];
  float* out[4];
};
template <int SAMP>
__global__ void kSLCell(Geom g, int acc, float dt, ConstFaceField vel, CellFields cf, int nf) {
  HFG_FOR(c, g.r.size()) {
    int x, y, z;
    cellCoord(c, g.r, x, y, z);
    float p[3] = {__fadd_rn(__fmul_rn(__fadd_rn((float)x, 0.5f), g.hx), g.ox),
                  __fadd_rn(__fmul_rn(__fadd_rn((float)y, 0.5f), g.hy), g.oy),
                  __fadd_rn(__fmul_rn(__fadd_rn((float)z, 0.5f), g.hz), g.oz)};
    float q[3];
    backTrace<SAMP>(vel, g, dt, acc, p, q);
    for (int k = 0; k < nf; ++k) cf.out[k][c] = sampleAlg<SAMP>(cf.in[k], g, q[0], q[1], q[2]);
  }
}
cudaError_t launchSLCell(const Geom& g, int acc, float dt, ConstFaceField vel, const float* const* in, float* const* out,
                         int nfields, cudaStream_t s, int sampling) {
  CellFields cf{};
  for (int k = 0; k < nfields && k < 4; ++k) { cf.in[k] = in[k]; cf.out[k] = out[k]; }
  const int nf = nfields < 4 ? nfields : 4;
  switch (sampling) {
    case 1: kSLCell<1><<<gridFor(g.r.size()), kThreads, 0, s>>>(g, acc, dt, vel, cf, nf); break;
    case 2: kSLCell<2><<<gridFor(g.r.size()), kThreads, 0, s>>>(g, acc, dt, vel, cf, nf); break;
    case 3: kSLCell<3><<<gridFor(g.r.size()), kThreads, 0, s>>>(g, acc, dt, vel, cf, nf); break;
    case 4: kSLCell<4><<<gridFor(g.r.size()), kThreads, 0, s>>>(g, acc, dt, vel, cf, nf); break;
    default: kSLCell<0><<<gridFor(g.r.size()), kThreads, 0, s>>>(g, acc, dt, vel, cf, nf);
  }
  return cudaGetLastError();
}

// Sampling of a cell-centred scalar grid (FieldMathTool.cu:470-573) or of
// the three face grids (:783-1128) at n points with an ESamplingAlgorithm.
template <int SAMP>
__global__ void kSampleAlg(Geom g, int face, ConstFaceField f, const float* __restrict__ pos, long long n,
                           float* __restrict__ out) {
  HFG_FOR(i, n) {
    const float px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
    if (face) {
#pragma unroll
      for (int a = 0; a < 3; ++a) out[3 * i + a] = sampleAlg<SAMP>(f.c[a], faceGeom(g, a), px, py, pz);
    } else {
      out[i] = sampleAlg<SAMP>(f.c[0], g, px, py, pz);
    }
  }
}
cudaError_t launchSampleAlg(const Geom& g, int face, ConstFaceField f, const float* pos, long long n, int sampling,
                            float* out, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  switch (sampling) {
    case 1: kSampleAlg<1><<<gridFor(n), kThreads, 0, s>>>(g, face, f, pos, n, out); break;
    case 2: kSampleAlg<2><<<gridFor(n), kThreads, 0, s>>>(g, face, f, pos, n, out); break;
    case 3: kSampleAlg<3><<<gridFor(n), kThreads, 0, s>>>(g, face, f, pos, n, out); break;
    case 4: kSampleAlg<4><<<gridFor(n), kThreads, 0, s>>>(g, face, f, pos, n, out); break;
    default: kSampleAlg<0><<<gridFor(n), kThreads, 0, s>>>(g, face, f, pos, n, out);
  }
  return cudaGetLastError();
}

__global__ void kAddConst(long long n, float* __restrict__ v, float a) {
  HFG_FOR(i, n) v[i] = __fadd_rn(a, v[i]);
}
cudaError_t launchAddConst(long long n, float* v, float a, cudaStream_t s) {
  kAddConst<<<gridFor(n), kThreads, 0, s>>>(n, v, a);
  return cudaGetLastError();
}

// ===========================================================================
// Self-test of the bounded waits.  Every wait of the TMA-fed and cooperative
// kernels is bounded: past its limit it records an error and returns, so the
// context stays usable.  These two kernels make the shared wait helpers run
// out on purpose, on conditions that nothing will ever satisfy, without any
// fault: an mbarrier phase expecting bytes no copy will deliver, and a grid
// barrier expecting one arrival more than the grid has blocks.
// ===========================================================================
__global__ void kSelftestMbarrier(unsigned long long waitNs, int* out) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbarInit(&bar, 1);
    mbarFenceInit();
    mbarExpectTx(&bar, 16);  // this thread arrives; 16 bytes stay pending for good
    const bool done = mbarWait(&bar, 0, globalNs() + waitNs);
    out[0] = done ? 0 : 1;
  }
}
__global__ void kSelftestGridBarrier(unsigned* words, int* out) {
  // words: count, generation, error
  const bool ok = gridBarrier(words, words + 1, words + 2, gridDim.x + 1);
  if (threadIdx.x == 0 && blockIdx.x == 0) out[1] = ok ? 0 : 1;
}
cudaError_t launchSelftestWaits(unsigned long long waitNs, unsigned* words, int* out, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(words, 0, 3 * sizeof(unsigned), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(out, 0xff, 2 * sizeof(int), s);
  if (e != cudaSuccess) return e;
  kSelftestMbarrier<<<1, 32, 0, s>>>(waitNs, out);
  kSelftestGridBarrier<<<2, 32, 0, s>>>(words, out);
  return cudaGetLastError();
}

}  // namespace hfg
