// hfg_mg.cu -- mixed-precision geometric multigrid preconditioner for the
// pressure CG.
//
// The reference solves the pressure system with an unpreconditioned CG
// (PressureSolver.cpp:12-15 copies r into z).  This preconditioner is new: a
// cell-centred V-cycle on the level hierarchy of the fluid/air/solid markers,
// used inside an FP32 CG whose dot products and convergence test stay FP64.
//
//  * coarsening: a coarse cell is air (Dirichlet, p = 0) if any of its <= 8
//    children is air, else fluid if any child is fluid, else solid;
//  * level operators: the same matrix-free 7-point stencil rebuilt from each
//    level's markers with the scales dt / (rho h^2) of that level (h doubles);
//  * smoothing: damped Jacobi (omega = 2/3), nu sweeps before and after; on
//    level 0 each thread marches along z with the z neighbours in registers;
//  * transfers: restriction = mean of the children's residuals, prolongation =
//    piecewise-constant injection (the scaled transpose), so the V-cycle is a
//    symmetric operator and plain CG applies;
//  * coarsest level (<= 512 cells): many Jacobi sweeps in one block's shared
//    memory;
//  * precision: every coarser level stores its right-hand side and iterate
//    in BF16 and computes in FP32; level 0 keeps its right-hand side (the
//    CG's r) in FP32 and, with half mode 2, stores its smoothing iterates in
//    BF16 as well, all but the last sweep's, which the CG reads in FP32.
//
// Every kernel returns at once when the CG has converged (CgState::done), so
// chunks of iterations can be launched without host round trips.
#include <algorithm>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <functional>
#include <vector>

#include "hfg_solver.h"

namespace hfg {

namespace {
constexpr int BX = 32, BY = 4, BZ = 2;
constexpr float kOmega = 2.0f / 3.0f;
constexpr int kCoarseMax = 512;
constexpr int kCoarseSweeps = 48;

template <class T> __device__ __forceinline__ float ld(const T* p, unsigned i);
template <> __device__ __forceinline__ float ld<float>(const float* p, unsigned i) { return __ldg(p + i); }
template <> __device__ __forceinline__ float ld<__nv_bfloat16>(const __nv_bfloat16* p, unsigned i) {
  return __bfloat162float(p[i]);
}
template <class T> __device__ __forceinline__ T cvt(float v);
template <> __device__ __forceinline__ float cvt<float>(float v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 cvt<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

__device__ __forceinline__ bool nbF(Code k, int d) { return (k >> (7 + d)) & 1; }
__device__ __forceinline__ float diagOfC(Code k, float sx, float sy, float sz) {
  if (!(k & 1)) return 1.f;
  float d = 0.f;
  if (k & 2) d += sx;
  if (k & 4) d += sx;
  if (k & 8) d += sy;
  if (k & 16) d += sy;
  if (k & 32) d += sz;
  if (k & 64) d += sz;
  return d;
}

struct Lvl {
  Dim3i r;
  float sx, sy, sz;
};

dim3 gridOf(const Dim3i& r) { return dim3((r.x + BX - 1) / BX, (r.y + BY - 1) / BY, (r.z + BZ - 1) / BZ); }

__device__ __forceinline__ bool cellOf(const Dim3i& r, int& x, int& y, int& z, unsigned& c) {
  x = blockIdx.x * BX + threadIdx.x;
  y = blockIdx.y * BY + threadIdx.y;
  z = blockIdx.z * BZ + threadIdx.z;
  if (x >= r.x || y >= r.y || z >= r.z) return false;
  c = ((unsigned)z * r.y + y) * r.x + x;
  return true;
}

// (A v)_c with the value of neighbour d (left, right, down, up, back, front)
// fetched by get(d); only fluid neighbours are asked for.
template <class G>
__device__ __forceinline__ float applyA(const Lvl& L, Code k, float vc, G get) {
  if (!(k & 1)) return vc;
  float acc = diagOfC(k, L.sx, L.sy, L.sz) * vc;
  if (nbF(k, 0)) acc -= L.sx * get(0);
  if (nbF(k, 1)) acc -= L.sx * get(1);
  if (nbF(k, 2)) acc -= L.sy * get(2);
  if (nbF(k, 3)) acc -= L.sy * get(3);
  if (nbF(k, 4)) acc -= L.sz * get(4);
  if (nbF(k, 5)) acc -= L.sz * get(5);
  return acc;
}

__device__ __forceinline__ void nbrOf(int d, int& dx, int& dy, int& dz) {
  dx = d == 0 ? -1 : (d == 1 ? 1 : 0);
  dy = d == 2 ? -1 : (d == 3 ? 1 : 0);
  dz = d == 4 ? -1 : (d == 5 ? 1 : 0);
}

// Coarse markers: air if any child is air, else fluid if any child is fluid,
// else solid.
__global__ void kCoarsenMarkers(Dim3i rf, Dim3i rc, const uint8_t* __restrict__ mf, uint8_t* __restrict__ mc) {
  int X, Y, Z;
  unsigned C;
  if (!cellOf(rc, X, Y, Z, C)) return;
  bool anyAir = false, anyFluid = false;
  for (int k = 0; k < 2; ++k)
    for (int j = 0; j < 2; ++j)
      for (int i = 0; i < 2; ++i) {
        int x = 2 * X + i, y = 2 * Y + j, z = 2 * Z + k;
        if (x >= rf.x || y >= rf.y || z >= rf.z) continue;
        uint8_t m = mf[((unsigned)z * rf.y + y) * rf.x + x];
        anyAir |= m == kAir;
        anyFluid |= m == kFluid;
      }
  mc[C] = anyAir ? kAir : (anyFluid ? kFluid : kSolid);
}

// First pre-smoothing sweep from z = 0: z = omega b / diag.
template <class TB, class TZ>
__global__ void kJacobiFirst(Lvl L, const TB* __restrict__ b, TZ* __restrict__ z, const Code* __restrict__ code,
                             const CgState* st) {
  waitPrevGrid();
  if (st->done) return;
  allowNextGrid();
  int x, y, zz;
  unsigned c;
  if (!cellOf(L.r, x, y, zz, c)) return;
  Code k = code[c];
  float v = (k & 1) ? kOmega * ld(b, c) / diagOfC(k, L.sx, L.sy, L.sz) : 0.f;
  z[c] = cvt<TZ>(v);
}

// One damped-Jacobi sweep zo = zi + omega (b - A zi) / diag.  With a coarse
// correction `zc` the sweep acts on zi + P zc (prolongation fused in).  With
// `dot` the sweep also reduces r.z and finishes the CG's beta (level 0, last
// post-smoothing sweep).
template <class TB, class TZ, class TC, bool CORR, bool DOT>
__global__ void kJacobi(Lvl L, Dim3i rc, const TB* __restrict__ b, const TZ* __restrict__ zi, TZ* __restrict__ zo,
                        const TC* __restrict__ zc, const Code* __restrict__ code, double* partials, CgState* st,
                        int zPer) {
  waitPrevGrid();
  if (st->done) return;
  allowNextGrid();
  double rz = 0.0, dummy = 0.0;
  const int x = blockIdx.x * BX + threadIdx.x, y = blockIdx.y * BY + threadIdx.y;
  const int zb0 = blockIdx.z * zPer;
  const unsigned pl = (unsigned)L.r.x * L.r.y;
  for (int zb = zb0; zb < zb0 + zPer; ++zb) {
    const int z = zb * BZ + threadIdx.z;
    if (x >= L.r.x || y >= L.r.y || z >= L.r.z) break;
    const unsigned c = ((unsigned)z * L.r.y + y) * L.r.x + x;
    auto zAt = [&](int d) -> float {
      int dx, dy, dz;
      nbrOf(d, dx, dy, dz);
      unsigned i = c + dx + dy * L.r.x + dz * pl;
      float v = ld(zi, i);
      if (CORR) v += ld(zc, ((unsigned)((z + dz) >> 1) * rc.y + ((y + dy) >> 1)) * rc.x + ((x + dx) >> 1));
      return v;
    };
    Code k = code[c];
    float v = 0.f;
    float bv = ld(b, c);
    if (k & 1) {
      float vc = ld(zi, c);
      if (CORR) vc += ld(zc, ((unsigned)(z >> 1) * rc.y + (y >> 1)) * rc.x + (x >> 1));
      float az = applyA(L, k, vc, zAt);
      v = vc + kOmega * (bv - az) / diagOfC(k, L.sx, L.sy, L.sz);
    }
    zo[c] = cvt<TZ>(v);
    if (DOT) rz += (double)bv * (double)v;
  }
  if (DOT) {
    if (gridSum2(rz, dummy, partials, &st->ticket) && flatTid() == 0) {
      // first V-cycle after the RHS: beta stays 0, rz initialised
      if (st->iter == 0) {
        st->rz = rz;
        st->beta = 0.f;
      } else {
        st->beta = (float)(rz / st->rz);
        st->rz = rz;
      }
      st->ticket = 0;
    }
  }
}

// Launch shape of the sweeps: one z-block per thread block (zPer = 1), or for
// the sweeps that end in a grid reduction a few thousand blocks each walking
// several z-blocks, so that the last-block reduction stays short.
struct SweepGrid {
  dim3 grid;
  int zPer;
};
SweepGrid sweepGrid(const Dim3i& r, bool reduce) {
  dim3 g = gridOf(r);
  int zPer = 1;
  if (reduce) {
    long long want = (long long)numSMs() * 8;
    long long cols = (long long)g.x * g.y;
    long long zc = std::max<long long>(1, want / std::max<long long>(1, cols));
    zPer = (int)((g.z + zc - 1) / zc);
  }
  return SweepGrid{dim3(g.x, g.y, (g.z + zPer - 1) / zPer), zPer};
}

// The same sweep on level 0, marching along z: a 32 x 8 tile of threads
// walks zLen planes, and the z neighbours come from registers (the value of
// the plane below is the one just used as the centre, the plane above is
// loaded one plane ahead and its stencil code two planes ahead).  The values
// and the arithmetic are those of kJacobi, so the sweeps agree bit for bit;
// only the order of the r.z partial sums differs.
constexpr int MX = 32, MY = 8;
static_assert(MX == kCgTileX && 2 * MY == kCgTileY, "two sweep blocks per tile column of the CG schedule");

// The cells a level-0 marching block sweeps: with the CG schedule of the
// solve (launchCgSchedule), two blocks per work item, the lower and upper 8
// rows of its 32 x 16 tile column over its run of fluid planes (a block past
// the last item sweeps nothing); without, the dense grid (tile x, tile y, z
// chunk of zLen planes).  Cells off the fluid keep z = 0 and add nothing to
// r.z, so skipping the planes no fluid cell of the column occupies changes
// no value.
__device__ __forceinline__ void mgBlockWork(const int* sched, const Dim3i& r, int zLen, int& x0, int& y0, int& z0,
                                            int& z1) {
  if (!sched) {
    x0 = blockIdx.x * MX;
    y0 = blockIdx.y * MY;
    z0 = blockIdx.z * zLen;
    z1 = min(z0 + zLen, r.z);
    return;
  }
  const int tilesX = (r.x + kCgTileX - 1) / kCgTileX, cols = tilesX * ((r.y + kCgTileY - 1) / kCgTileY);
  const int item = blockIdx.x >> 1;
  x0 = y0 = z0 = z1 = 0;
  const int n = __ldg(sched + 2 * cols);
  if (item >= n || 2 * n > (int)gridDim.x) return;
  const int4 w = __ldg(reinterpret_cast<const int4*>(sched + schedItemsOffset(cols)) + item);
  // an item that is not a run of this grid is not swept (the CG kernels,
  // which read the same schedule, report it)
  if (w.x < 0 || w.x >= cols || w.y < 0 || w.y >= w.z || w.z > r.z) return;
  x0 = (w.x % tilesX) * kCgTileX;
  y0 = (w.x / tilesX) * kCgTileY + (blockIdx.x & 1) * MY;
  z0 = w.y;
  z1 = w.z;
}

template <class TC, bool CORR, bool DOT, class TZI = float, class TZO = float>
__global__ void __launch_bounds__(MX* MY)
    kJacobiZ(Lvl L, Dim3i rc, const float* __restrict__ b, const TZI* __restrict__ zi, TZO* __restrict__ zo,
             const TC* __restrict__ zc, const Code* __restrict__ code, double* partials, CgState* st, int zLen,
             const int* __restrict__ sched) {
  waitPrevGrid();
  if (st->done) return;
  allowNextGrid();
  double rz = 0.0, dummy = 0.0;
  int xb, yb, z0, z1;
  mgBlockWork(sched, L.r, zLen, xb, yb, z0, z1);
  const int x = xb + threadIdx.x, y = yb + threadIdx.y;
  if (x < L.r.x && y < L.r.y && z0 < z1) {
    const unsigned pl = (unsigned)L.r.x * L.r.y;
    auto par = [&](int i, int j, int k) { return ((unsigned)(k >> 1) * rc.y + (j >> 1)) * rc.x + (i >> 1); };
    // iterate (with the coarse correction) at cell i of plane zz, 0 off the fluid
    auto value = [&](unsigned i, int zz, Code ki) -> float {
      if (!(ki & 1)) return 0.f;
      float v = ld(zi, i);
      if (CORR) v += ld(zc, par(x, y, zz));
      return v;
    };
    unsigned c = ((unsigned)z0 * L.r.y + y) * L.r.x + x;
    const Code kb0 = z0 > 0 ? code[c - pl] : (Code)0;
    float vb = value(c - pl, z0 - 1, kb0);
    Code k = code[c];
    float vc = value(c, z0, k);
    Code ka = z0 + 1 < L.r.z ? code[c + pl] : (Code)0;
    for (int z = z0; z < z1; ++z, c += pl) {
      const Code kaa = z + 2 < L.r.z ? code[c + 2 * pl] : (Code)0;
      const float va = value(c + pl, z + 1, ka);
      const float bv = __ldg(b + c);
      float v = 0.f;
      if (k & 1) {
        auto zAt = [&](int d) -> float {
          if (d == 4) return vb;
          if (d == 5) return va;
          int dx, dy, dz;
          nbrOf(d, dx, dy, dz);
          float w = ld(zi, c + dx + dy * L.r.x);
          if (CORR) w += ld(zc, par(x + dx, y + dy, z));
          return w;
        };
        float az = applyA(L, k, vc, zAt);
        v = vc + kOmega * (bv - az) / diagOfC(k, L.sx, L.sy, L.sz);
      }
      if (k & 1) zo[c] = cvt<TZO>(v);  // zero off the fluid for the whole solve (memset by mgRunCg)
      if (DOT) rz += (double)bv * (double)v;
      vb = vc;
      k = ka;
      vc = va;
      ka = kaa;
    }
  }
  if (DOT) {
    if (gridSum2(rz, dummy, partials, &st->ticket) && flatTid() == 0) {
      if (st->iter == 0) {
        st->rz = rz;
        st->beta = 0.f;
      } else {
        st->beta = (float)(rz / st->rz);
        st->rz = rz;
      }
      st->ticket = 0;
    }
  }
}

// kJacobiFirst on level 0 with the launch shape of kJacobiZ: z = omega b /
// diag along a column of zLen planes.
template <class TZO>
__global__ void __launch_bounds__(MX* MY)
    kJacobiFirstZ(Lvl L, const float* __restrict__ b, TZO* __restrict__ z, const Code* __restrict__ code,
                  const CgState* st, int zLen, const int* __restrict__ sched) {
  waitPrevGrid();
  if (st->done) return;
  allowNextGrid();
  int xb, yb, z0, z1;
  mgBlockWork(sched, L.r, zLen, xb, yb, z0, z1);
  const int x = xb + threadIdx.x, y = yb + threadIdx.y;
  if (x >= L.r.x || y >= L.r.y) return;
  const unsigned pl = (unsigned)L.r.x * L.r.y;
  unsigned c = ((unsigned)z0 * L.r.y + y) * L.r.x + x;
#pragma unroll 4
  for (int zz = z0; zz < z1; ++zz, c += pl) {
    const Code k = code[c];
    if (k & 1) z[c] = cvt<TZO>(kOmega * __ldg(b + c) / diagOfC(k, L.sx, L.sy, L.sz));  // zero elsewhere already
  }
}

// Launch shape of the level-0 marching sweeps: enough z chunks for about 32
// blocks per SM (8 or 64 per SM, and 128, were slower at 256^3), but columns
// of at least 4 planes (shorter ones re-load more of their neighbours than
// they save; with concurrent scenes every load counts).
SweepGrid marchGrid(const Dim3i& r) {
  const long long cols = (long long)((r.x + MX - 1) / MX) * ((r.y + MY - 1) / MY);
  const long long want = (long long)numSMs() * 32;
  const long long chunks = std::min<long long>((r.z + 3) / 4, std::max<long long>(1, (want + cols - 1) / cols));
  const int zLen = (int)((r.z + chunks - 1) / chunks);
  return SweepGrid{dim3((r.x + MX - 1) / MX, (r.y + MY - 1) / MY, (r.z + zLen - 1) / zLen), zLen};
}

// Level 0 marches when that still gives two blocks per SM; smaller grids (64^3
// and below) keep the per-cell sweeps, whose many short blocks hide latency
// better there.
bool marchLevel0(const Dim3i& r) {
  const dim3 g = marchGrid(r).grid;
  return (long long)g.x * g.y * g.z >= 2LL * numSMs();
}

// Residual of level f restricted to level c: bc = mean over the children of
// (b - A z).
template <class TB, class TZ, class TBC>
__global__ void kResidualRestrict(Lvl Lf, Dim3i rc, const TB* __restrict__ b, const TZ* __restrict__ zf,
                                  const Code* __restrict__ code, TBC* __restrict__ bc, const CgState* st) {
  waitPrevGrid();
  if (st->done) return;
  allowNextGrid();
  int X, Y, Z;
  unsigned C;
  if (!cellOf(rc, X, Y, Z, C)) return;
  float s = 0.f;
  for (int kk = 0; kk < 2; ++kk)
    for (int j = 0; j < 2; ++j)
      for (int i = 0; i < 2; ++i) {
        int x = 2 * X + i, y = 2 * Y + j, z = 2 * Z + kk;
        if (x >= Lf.r.x || y >= Lf.r.y || z >= Lf.r.z) continue;
        unsigned c = ((unsigned)z * Lf.r.y + y) * Lf.r.x + x;
        Code k = code[c];
        if (!(k & 1)) continue;
        const unsigned pl = (unsigned)Lf.r.x * Lf.r.y;
        float az = applyA(Lf, k, ld(zf, c), [&](int d) {
          int dx, dy, dz;
          nbrOf(d, dx, dy, dz);
          return ld(zf, c + dx + dy * Lf.r.x + dz * pl);
        });
        s += ld(b, c) - az;
      }
  bc[C] = cvt<TBC>(0.125f * s);
}

// Coarsest level: Jacobi sweeps in one block's shared memory.
template <class TB, class TZ>
__global__ void kCoarseSolve(Lvl L, const TB* __restrict__ b, TZ* __restrict__ z, const Code* __restrict__ code,
                             const CgState* st) {
  waitPrevGrid();
  if (st->done) return;
  allowNextGrid();
  __shared__ float za[kCoarseMax], zb[kCoarseMax];
  unsigned n = (unsigned)L.r.size();
  for (unsigned c = threadIdx.x; c < n; c += blockDim.x) za[c] = 0.f;
  __syncthreads();
  float* cur = za;
  float* nxt = zb;
  for (int it = 0; it < kCoarseSweeps; ++it) {
    for (unsigned c = threadIdx.x; c < n; c += blockDim.x) {
      Code k = code[c];
      float v = 0.f;
      if (k & 1) {
        const unsigned pl = (unsigned)L.r.x * L.r.y;
        float az = applyA(L, k, cur[c], [&](int d) {
          int dx, dy, dz;
          nbrOf(d, dx, dy, dz);
          return cur[c + dx + dy * L.r.x + dz * pl];
        });
        v = cur[c] + kOmega * (ld(b, c) - az) / diagOfC(k, L.sx, L.sy, L.sz);
      }
      nxt[c] = v;
    }
    __syncthreads();
    float* t = cur;
    cur = nxt;
    nxt = t;
  }
  for (unsigned c = threadIdx.x; c < n; c += blockDim.x) z[c] = cvt<TZ>(cur[c]);
}
}  // namespace

// Work items a multigrid solve's schedule can hold: the larger of the two
// iterate types' targets (the sweeps do not know which one the CG uses).
int mgScheduleTarget() { return std::max(cgScheduleTarget(2, false), cgScheduleTarget(2, true)); }

struct Multigrid {
  Dim3i r0;                          // level 0 = the pitched grid of the pressure system
  Dim3i rLogical;                    // the solver's grid (level-0 markers are unpitched)
  int smooth = 2;
  bool half = true;                  // coarse levels in BF16
  bool half0 = false;                // level-0 smoothing iterates in BF16 too (marching sweeps only)
  std::vector<Dim3i> res;            // level resolutions, [0] = fine
  std::vector<DArray<uint8_t>*> mk;  // levels >= 1
  std::vector<DArray<Code>*> code;   // levels >= 1
  std::vector<DArray<uint16_t>*> b16, z16a, z16b;  // levels >= 1 (BF16 / FP16 storage)
  std::vector<DArray<float>*> b32, z32a, z32b;     // levels >= 1 when !half
  DArray<float> z0a, z0b;            // level 0 iterate (FP32)
  DArray<uint16_t> z0h[2];           // level 0 BF16 iterates (half0)
  DArray<float> p[2];
  DArray<double> partials;
  CUtensorMap zH[2], pH[2];          // halo tensor maps of z0a / z0b and p[0] / p[1]
  long long chunkLaunches = 0;       // kernels in one captured chunk of CG iterations
  const Code* code0 = nullptr;
  float s0[3] = {0, 0, 0};
  ~Multigrid() {
    for (auto* v : mk) delete v;
    for (auto* v : code) delete v;
    for (auto* v : b16) delete v;
    for (auto* v : z16a) delete v;
    for (auto* v : z16b) delete v;
    for (auto* v : b32) delete v;
    for (auto* v : z32a) delete v;
    for (auto* v : z32b) delete v;
  }
  int levels() const { return (int)res.size(); }
};

Multigrid* mgCreate(const Dim3i& r, int levels, int smooth, int halfMode, cudaStream_t s) {
  auto* m = new Multigrid();
  m->r0 = r;
  m->smooth = smooth > 0 ? smooth : 3;  // 3 sweeps: fewest ms per solve at 256^3 (2: 67.3, 3: 65.6, 4: 66.9 ms per step)
  const bool half = halfMode != 0;
  m->half = half;
  m->half0 = halfMode == 2 && marchLevel0(r);
  m->res.push_back(r);
  Dim3i cur = r;
  while ((levels <= 0 || (int)m->res.size() < levels) && cur.size() > kCoarseMax) {
    Dim3i nx{(cur.x + 1) / 2, (cur.y + 1) / 2, (cur.z + 1) / 2};
    if (nx.x == cur.x && nx.y == cur.y && nx.z == cur.z) break;
    m->res.push_back(nx);
    cur = nx;
  }
  if (m->res.back().size() > kCoarseMax) {
    delete m;
    throw CudaError("multigrid: coarsest level too large; allow more levels", HFG_ERR_INVALID);
  }
  long long N = r.size();
  m->z0a.alloc(N, s);
  m->z0b.alloc(N, s);
  if (m->half0) {
    m->z0h[0].alloc(N, s);
    m->z0h[1].alloc(N, s);
  }
  m->p[0].alloc(N, s);
  m->p[1].alloc(N, s);
  const dim3 mg = marchGrid(r).grid;
  m->partials.alloc(std::max({cgPartialsNeeded(r), 2 * (int)(gridOf(r).x * gridOf(r).y * gridOf(r).z),
                              2 * (int)(mg.x * mg.y * mg.z), 2 * 2 * (mgScheduleTarget() + cgColumns(r))}),
                    s);
  check(makeHaloMap(r, m->z0a.p, &m->zH[0]), "multigrid tensor map");
  check(makeHaloMap(r, m->z0b.p, &m->zH[1]), "multigrid tensor map");
  check(makeHaloMap(r, m->p[0].p, &m->pH[0]), "multigrid tensor map");
  check(makeHaloMap(r, m->p[1].p, &m->pH[1]), "multigrid tensor map");
  for (int l = 1; l < m->levels(); ++l) {
    long long n = m->res[l].size();
    auto* a = new DArray<uint8_t>();
    a->alloc(n, s);
    m->mk.push_back(a);
    auto* c = new DArray<Code>();
    c->alloc(n, s);
    m->code.push_back(c);
    if (half) {
      auto* b = new DArray<uint16_t>(); b->alloc(n, s); m->b16.push_back(b);
      auto* za = new DArray<uint16_t>(); za->alloc(n, s); m->z16a.push_back(za);
      auto* zb = new DArray<uint16_t>(); zb->alloc(n, s); m->z16b.push_back(zb);
    } else {
      auto* b = new DArray<float>(); b->alloc(n, s); m->b32.push_back(b);
      auto* za = new DArray<float>(); za->alloc(n, s); m->z32a.push_back(za);
      auto* zb = new DArray<float>(); zb->alloc(n, s); m->z32b.push_back(zb);
    }
  }
  return m;
}

void mgDestroy(Multigrid* m) { delete m; }

// Level markers and stencil codes for the current step's fine markers.
void mgSetupLevels(Multigrid* m, const uint8_t* mk0, const Code* code0, float sx, float sy, float sz, cudaStream_t s,
                   long long& launches) {
  m->code0 = code0;
  m->s0[0] = sx; m->s0[1] = sy; m->s0[2] = sz;
  const uint8_t* fine = mk0;
  for (int l = 1; l < m->levels(); ++l) {
    // level-0 markers are unpitched: children in the pitch padding are skipped
    Dim3i rf = l == 1 ? m->rLogical : m->res[l - 1], rc = m->res[l];
    kCoarsenMarkers<<<gridOf(rc), dim3(BX, BY, BZ), 0, s>>>(rf, rc, fine, m->mk[l - 1]->p);
    check(cudaGetLastError(), "coarsen markers");
    check(launchStencilCode(rc, rc.x, m->mk[l - 1]->p, m->code[l - 1]->p, s), "level stencil code");
    launches += 2;
    fine = m->mk[l - 1]->p;
  }
}

namespace {
template <class TS>
const float* vcycleT(Multigrid* m, const float* r0, CgState* st, cudaStream_t s, long long& launches, TS* const* bL,
                     TS* const* zaL, TS* const* zbL, const int* sched) {
  const int L = m->levels();
  std::vector<Lvl> lv(L);
  for (int l = 0; l < L; ++l) {
    float f = 1.f;
    for (int i = 0; i < l; ++i) f *= 0.25f;
    lv[l] = Lvl{m->res[l], m->s0[0] * f, m->s0[1] * f, m->s0[2] * f};
  }
  auto codeOf = [&](int l) -> const Code* { return l == 0 ? m->code0 : m->code[l - 1]->p; };
  const dim3 blk(BX, BY, BZ);
  const int nu = m->smooth;
  // every kernel of the V-cycle is a programmatic dependent launch: the launch
  // of the next one overlaps the tail of this one
  auto run = [&](auto kernel, dim3 grid, dim3 block, auto... args) {
    check(launchPdl(kernel, grid, block, s, args...), "multigrid");
    ++launches;
  };
  // a smoothing sweep (with the grid reduction of the CG's r.z when dot)
  auto sweep = [&](auto kernel, const Dim3i& r, bool dot, auto... args) {
    const SweepGrid g = sweepGrid(r, dot);
    run(kernel, g.grid, blk, args..., g.zPer);
  };
  // a level-0 sweep marching along z
  const SweepGrid mg0 = marchGrid(lv[0].r);
  const bool marching = marchLevel0(lv[0].r);
  // with the solve's CG schedule: two blocks per work item, fluid runs only
  const dim3 schedGrid(2 * (mgScheduleTarget() + cgColumns(lv[0].r)), 1, 1);
  auto march = [&](auto kernel, auto... args) {
    run(kernel, sched ? schedGrid : mg0.grid, dim3(MX, MY), args..., mg0.zPer, sched);
  };
  // which ping-pong buffer holds the current iterate of each level
  std::vector<int> curBuf(L, 0);
  float* z0[2] = {m->z0a.p, m->z0b.p};
  // half0: the level-0 iterates in BF16 (h0), except the last sweep's, which
  // goes to z0a in FP32 for the CG
  using BF = __nv_bfloat16;
  const bool h0 = m->half0 && marching && L > 1;
  BF* hz[2] = {(BF*)m->z0h[0].p, (BF*)m->z0h[1].p};
  // downward sweep
  for (int l = 0; l < L - 1; ++l) {
    if (l == 0 && h0) {
      march(kJacobiFirstZ<BF>, lv[0], r0, hz[0], codeOf(0), (const CgState*)st);
      int cb = 0;
      for (int k = 1; k < nu; ++k, cb ^= 1)
        march(kJacobiZ<float, false, false, BF, BF>, lv[0], lv[0].r, r0, (const BF*)hz[cb], hz[cb ^ 1],
              (const float*)nullptr, codeOf(0), (double*)nullptr, st);
      curBuf[0] = cb;
      run(kResidualRestrict<float, BF, TS>, gridOf(lv[1].r), blk, lv[0], lv[1].r, r0, (const BF*)hz[cb], codeOf(0),
          bL[1], (const CgState*)st);
    } else if (l == 0) {
      if (marching)
        march(kJacobiFirstZ<float>, lv[0], r0, z0[0], codeOf(0), (const CgState*)st);
      else
        run(kJacobiFirst<float, float>, gridOf(lv[0].r), blk, lv[0], r0, z0[0], codeOf(0), (const CgState*)st);
      int cb = 0;
      for (int k = 1; k < nu; ++k, cb ^= 1) {
        if (marching)
          march(kJacobiZ<float, false, false>, lv[0], lv[0].r, r0, (const float*)z0[cb], z0[cb ^ 1],
                (const float*)nullptr, codeOf(0), (double*)nullptr, st);
        else
          sweep(kJacobi<float, float, float, false, false>, lv[0].r, false, lv[0], lv[0].r, r0, (const float*)z0[cb],
                z0[cb ^ 1], (const float*)nullptr, codeOf(0), (double*)nullptr, st);
      }
      curBuf[0] = cb;
      run(kResidualRestrict<float, float, TS>, gridOf(lv[1].r), blk, lv[0], lv[1].r, r0, (const float*)z0[cb],
          codeOf(0), bL[1], (const CgState*)st);
    } else {
      TS* zl[2] = {zaL[l], zbL[l]};
      run(kJacobiFirst<TS, TS>, gridOf(lv[l].r), blk, lv[l], (const TS*)bL[l], zl[0], codeOf(l), (const CgState*)st);
      int cb = 0;
      for (int k = 1; k < nu; ++k, cb ^= 1)
        sweep(kJacobi<TS, TS, TS, false, false>, lv[l].r, false, lv[l], lv[l].r, (const TS*)bL[l], (const TS*)zl[cb],
              zl[cb ^ 1], (const TS*)nullptr, codeOf(l), (double*)nullptr, st);
      curBuf[l] = cb;
      run(kResidualRestrict<TS, TS, TS>, gridOf(lv[l + 1].r), blk, lv[l], lv[l + 1].r, (const TS*)bL[l],
          (const TS*)zl[cb], codeOf(l), bL[l + 1], (const CgState*)st);
    }
  }
  // coarsest
  {
    int l = L - 1;
    if (l == 0)
      run(kCoarseSolve<float, float>, dim3(1), dim3(1024), lv[0], r0, z0[0], codeOf(0), (const CgState*)st);
    else
      run(kCoarseSolve<TS, TS>, dim3(1), dim3(1024), lv[l], (const TS*)bL[l], zaL[l], codeOf(l), (const CgState*)st);
    curBuf[l] = 0;
  }
  // upward sweep: prolongation fused into the first post-smoothing sweep
  for (int l = L - 2; l >= 0; --l) {
    const TS* zc = (curBuf[l + 1] == 0) ? zaL[l + 1] : zbL[l + 1];
    if (l == 0 && h0) {
      int cb = curBuf[0];
      for (int k = 0; k < nu; ++k, cb ^= 1) {
        const bool last = k == nu - 1;
        const BF* zi = hz[cb];
        if (k == 0 && last)
          march(kJacobiZ<TS, true, true, BF, float>, lv[0], lv[1].r, r0, zi, z0[0], zc, codeOf(0), m->partials.p, st);
        else if (k == 0)
          march(kJacobiZ<TS, true, false, BF, BF>, lv[0], lv[1].r, r0, zi, hz[cb ^ 1], zc, codeOf(0), (double*)nullptr,
                st);
        else if (last)
          march(kJacobiZ<float, false, true, BF, float>, lv[0], lv[0].r, r0, zi, z0[0], (const float*)nullptr,
                codeOf(0), m->partials.p, st);
        else
          march(kJacobiZ<float, false, false, BF, BF>, lv[0], lv[0].r, r0, zi, hz[cb ^ 1], (const float*)nullptr,
                codeOf(0), (double*)nullptr, st);
      }
      curBuf[0] = 0;  // the result is in z0[0]
    } else if (l == 0) {
      int cb = curBuf[0];
      for (int k = 0; k < nu; ++k, cb ^= 1) {
        const bool last = k == nu - 1;
        const float* zi = z0[cb];
        if (!marching) {
          if (k == 0 && last)
            sweep(kJacobi<float, float, TS, true, true>, lv[0].r, true, lv[0], lv[1].r, r0, zi, z0[cb ^ 1], zc,
                  codeOf(0), m->partials.p, st);
          else if (k == 0)
            sweep(kJacobi<float, float, TS, true, false>, lv[0].r, false, lv[0], lv[1].r, r0, zi, z0[cb ^ 1], zc,
                  codeOf(0), (double*)nullptr, st);
          else if (last)
            sweep(kJacobi<float, float, float, false, true>, lv[0].r, true, lv[0], lv[0].r, r0, zi, z0[cb ^ 1],
                  (const float*)nullptr, codeOf(0), m->partials.p, st);
          else
            sweep(kJacobi<float, float, float, false, false>, lv[0].r, false, lv[0], lv[0].r, r0, zi, z0[cb ^ 1],
                  (const float*)nullptr, codeOf(0), (double*)nullptr, st);
        } else if (k == 0 && last)
          march(kJacobiZ<TS, true, true>, lv[0], lv[1].r, r0, zi, z0[cb ^ 1], zc, codeOf(0), m->partials.p, st);
        else if (k == 0)
          march(kJacobiZ<TS, true, false>, lv[0], lv[1].r, r0, zi, z0[cb ^ 1], zc, codeOf(0), (double*)nullptr, st);
        else if (last)
          march(kJacobiZ<float, false, true>, lv[0], lv[0].r, r0, zi, z0[cb ^ 1], (const float*)nullptr, codeOf(0),
                m->partials.p, st);
        else
          march(kJacobiZ<float, false, false>, lv[0], lv[0].r, r0, zi, z0[cb ^ 1], (const float*)nullptr, codeOf(0),
                (double*)nullptr, st);
      }
      curBuf[0] = cb;
    } else {
      TS* zl[2] = {zaL[l], zbL[l]};
      int cb = curBuf[l];
      for (int k = 0; k < nu; ++k, cb ^= 1) {
        if (k == 0)
          sweep(kJacobi<TS, TS, TS, true, false>, lv[l].r, false, lv[l], lv[l + 1].r, (const TS*)bL[l],
                (const TS*)zl[cb], zl[cb ^ 1], zc, codeOf(l), (double*)nullptr, st);
        else
          sweep(kJacobi<TS, TS, TS, false, false>, lv[l].r, false, lv[l], lv[l].r, (const TS*)bL[l],
                (const TS*)zl[cb], zl[cb ^ 1], (const TS*)nullptr, codeOf(l), (double*)nullptr, st);
      }
      curBuf[l] = cb;
    }
  }
  return z0[curBuf[0]];
}
}  // namespace

// z = V(r0) (returned: one of the two level-0 buffers), and st->rz /
// st->beta updated by the last sweep.
const float* mgVcycle(Multigrid* m, const float* r0, CgState* st, cudaStream_t s, long long& launches,
                      const int* sched) {
  const int L = m->levels();
  if (m->half) {
    std::vector<__nv_bfloat16*> b(L, nullptr), za(L, nullptr), zb(L, nullptr);
    for (int l = 1; l < L; ++l) {
      b[l] = (__nv_bfloat16*)m->b16[l - 1]->p;
      za[l] = (__nv_bfloat16*)m->z16a[l - 1]->p;
      zb[l] = (__nv_bfloat16*)m->z16b[l - 1]->p;
    }
    return vcycleT<__nv_bfloat16>(m, r0, st, s, launches, b.data(), za.data(), zb.data(), sched);
  } else {
    std::vector<float*> b(L, nullptr), za(L, nullptr), zb(L, nullptr);
    for (int l = 1; l < L; ++l) {
      b[l] = m->b32[l - 1]->p;
      za[l] = m->z32a[l - 1]->p;
      zb[l] = m->z32b[l - 1]->p;
    }
    return vcycleT<float>(m, r0, st, s, launches, b.data(), za.data(), zb.data(), sched);
  }
}

void mgSetup(Multigrid* m, const Dim3i& r, const uint8_t* mk0, const Code* code, float sx, float sy, float sz,
             cudaStream_t s, long long& launches) {
  m->rLogical = r;
  mgSetupLevels(m, mk0, code, sx, sy, sz, s, launches);
}

// Preconditioned CG with the V-cycle: the RHS kernel already set r = b,
// x = 0 and ||b||^2.  Iterations are launched in chunks; every kernel returns
// immediately once the state says done.
void mgRunCg(Multigrid* m, const Dim3i& cg, float sx, float sy, float sz, const CgMaps& maps, const CgCode* code, void* x,
             bool xDouble, float* rvec, CgState* st, CgState* stHost, cudaStream_t s, long long& launches,
             const std::function<cudaGraphExec_t(const std::function<void()>&)>& capture, cudaGraphExec_t* chunk,
             const int* colZ) {
  // both direction buffers start zero: the CG kernels never store at non-fluid
  // cells, and the fluid moves between solves
  check(cudaMemsetAsync(m->p[0].p, 0, m->p[0].bytes(), s), "memset");
  check(cudaMemsetAsync(m->p[1].p, 0, m->p[1].bytes(), s), "memset");
  // the marching level-0 sweeps store fluid cells only: the iterates start zero
  check(cudaMemsetAsync(m->z0a.p, 0, m->z0a.bytes(), s), "memset");
  check(cudaMemsetAsync(m->z0b.p, 0, m->z0b.bytes(), s), "memset");
  for (auto& h : m->z0h)
    if (h.p) check(cudaMemsetAsync(h.p, 0, h.bytes(), s), "memset");
  const float* z0 = mgVcycle(m, rvec, st, s, launches, colZ);  // z0 = V(b), rz = b.z0
  const int kChunk = 4;  // even: every chunk starts on p[0]
  auto body = [&] {
    const float* z = z0;
    long long before = launches;
    for (int it = 0; it < kChunk; ++it) {
      const int po = it & 1, pn = (it + 1) & 1;
      const int zi = z == m->z0a.p ? 0 : 1;
      check(launchCgDirection(cg, sx, sy, sz, m->zH[zi], m->pH[po], maps.codeH, code, z, m->p[po].p, m->p[pn].p,
                              m->partials.p, st, 2, s, colZ, xDouble),
            "cg direction");
      check(launchCgUpdate(cg, sx, sy, sz, m->pH[pn], maps.rI, maps.xI, maps.codeI, m->p[pn].p, x, xDouble, rvec,
                           m->partials.p, st, 2, s, colZ),
            "cg update");
      launches += 2;
      z = mgVcycle(m, rvec, st, s, launches, colZ);
    }
    m->chunkLaunches = launches - before;
    // the V-cycle always leaves its result in the same level-0 buffer
    if (z != z0) throw CudaError("multigrid: V-cycle output buffer changed between iterations", HFG_ERR_STATE);
  };
  if (!*chunk) *chunk = capture(body);
  for (;;) {
    check(cudaGraphLaunch(*chunk, s), "cg chunk");
    launches += m->chunkLaunches;
    readBack(stHost, st, sizeof(CgState), s);
    check(cudaStreamSynchronize(s), "cg sync");
    if (stHost->done) break;
  }
}

}  // namespace hfg
