// hfg_pressure.cu -- the matrix-free pressure Poisson system and its CG on
// sm_100a.
//
// The reference stores A as 4 floats per cell (buildPressureMatrixA,
// EulerSolverTool.cu:58-126) and runs CG with cuBLAS calls and three blocking
// host reads per iteration (CuMatrixFreePCG.cpp:22-65).  Here A is rebuilt in
// registers from a 16-bit stencil code per cell, every CG iteration is two
// kernels with FP64 block reductions finished by the last block (no host
// round trip), and the stencil kernels are 2.5-D: a 32x8 thread tile marches
// along z keeping the below / current / above planes in registers, so the z
// neighbours cost no extra loads and no division is needed for indexing.
#include <algorithm>

#include "hfg_kernels.h"

namespace hfg {

namespace {
constexpr int TX = 32, TY = 8;

struct CgGrid {
  dim3 grid, block;
  int zPer;
};

// Enough blocks to fill every SM several times over, each marching >= 4 planes.
CgGrid cgGrid(const Dim3i& r) {
  CgGrid g;
  g.block = dim3(TX, TY, 1);
  int bx = (r.x + TX - 1) / TX, by = (r.y + TY - 1) / TY;
  long long tiles = (long long)bx * by;
  long long want = (long long)numSMs() * 16;
  int zc = (int)std::max<long long>(1, (want + tiles - 1) / tiles);
  zc = std::min(zc, std::max(1, r.z / 4));
  g.zPer = (r.z + zc - 1) / zc;
  zc = (r.z + g.zPer - 1) / g.zPer;
  g.grid = dim3(bx, by, zc);
  return g;
}

__device__ __forceinline__ bool nbFluid(Code k, int d) { return (k >> (7 + d)) & 1; }

// Diagonal in the reference's accumulation order (EulerSolverTool.cu:85-120).
__device__ __forceinline__ float diagOf(Code k, float sx, float sy, float sz) {
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

// PC: 0 identity, 1 Jacobi, 2 z supplied by the caller (multigrid)
template <int PC>
__device__ __forceinline__ float precondZ(Code k, float rv, float sx, float sy, float sz) {
  return PC == 1 ? __fdiv_rn(rv, diagOf(k, sx, sy, sz)) : rv;
}

__device__ inline bool cgStop(const CgState* st, double rr) {
  double rn = sqrt(rr);
  if (st->tolMode == 0) return sqrt(rn) < st->tol;  // CuMatrixFreePCG.cpp:28,51
  double bn = sqrt(st->bb);
  return bn == 0.0 || rn / bn < st->tol;
}

// (A v)_c for a fluid cell given v at the centre and at its six neighbours
// (fdmMatrixVectorMul, EulerSolverTool.cu:219-226: products in float, sum in
// double as the reference's `: 0.0` ternaries make it).
__device__ __forceinline__ float applyRow(Code k, float sx, float sy, float sz, float vc, float vl, float vr, float vd,
                                          float vu, float vb, float vf) {
  if (!(k & 1)) return vc;
  double acc = (double)__fmul_rn(diagOf(k, sx, sy, sz), vc);
  if (nbFluid(k, 0)) acc += (double)__fmul_rn(-sx, vl);
  if (nbFluid(k, 1)) acc += (double)__fmul_rn(-sx, vr);
  if (nbFluid(k, 2)) acc += (double)__fmul_rn(-sy, vd);
  if (nbFluid(k, 3)) acc += (double)__fmul_rn(-sy, vu);
  if (nbFluid(k, 4)) acc += (double)__fmul_rn(-sz, vb);
  if (nbFluid(k, 5)) acc += (double)__fmul_rn(-sz, vf);
  return (float)acc;
}
}  // namespace

int cgPartialsNeeded(const Dim3i& r) {
  CgGrid g = cgGrid(r);
  return 2 * (int)(g.grid.x * g.grid.y * g.grid.z);
}

// ---------------------------------------------------------------------------
__global__ void kStencilCode(Dim3i r, const uint8_t* __restrict__ mk, Code* __restrict__ code, int zPer) {
  int x = blockIdx.x * TX + threadIdx.x, y = blockIdx.y * TY + threadIdx.y;
  if (x >= r.x || y >= r.y) return;
  int z0 = blockIdx.z * zPer, z1 = min(z0 + zPer, r.z);
  long long plane = (long long)r.x * r.y;
  for (int z = z0; z < z1; ++z) {
    long long c = (long long)z * plane + (long long)y * r.x + x;
    Code k = 0;
    if (mk[c] == kFluid) {
      k = 1;
      const bool in[6] = {x > 0, x + 1 < r.x, y > 0, y + 1 < r.y, z > 0, z + 1 < r.z};
      const long long o[6] = {-1, 1, -(long long)r.x, (long long)r.x, -plane, plane};
#pragma unroll
      for (int d = 0; d < 6; ++d) {
        if (!in[d]) continue;
        uint8_t m = mk[c + o[d]];
        if (m != kSolid) k |= (Code)(1u << (1 + d));
        if (m == kFluid) k |= (Code)(1u << (7 + d));
      }
    }
    code[c] = k;
  }
}
cudaError_t launchStencilCode(const Dim3i& r, const uint8_t* markers, Code* code, cudaStream_t s) {
  CgGrid g = cgGrid(r);
  kStencilCode<<<g.grid, g.block, 0, s>>>(r, markers, code, g.zPer);
  return cudaGetLastError();
}

// The reference's stored matrix [diag, +x, +y, +z] (EulerSolverTool.cu:58-126),
// bit-exact: used by the operator API and its tests only.
__global__ void kMatrixA(Dim3i r, float sx, float sy, float sz, const Code* __restrict__ code, float* __restrict__ A) {
  long long n = r.size();
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    Code k = code[c];
    float a0 = diagOf(k, sx, sy, sz), a1 = 0.f, a2 = 0.f, a3 = 0.f;
    if (k & 1) {
      if (nbFluid(k, 1)) a1 = -sx;
      if (nbFluid(k, 3)) a2 = -sy;
      if (nbFluid(k, 5)) a3 = -sz;
    }
    A[4 * c] = a0; A[4 * c + 1] = a1; A[4 * c + 2] = a2; A[4 * c + 3] = a3;
  }
}
cudaError_t launchMatrixA(const Dim3i& r, float sx, float sy, float sz, const Code* code, float* A, cudaStream_t s) {
  int blocks = (int)std::min<long long>((r.size() + 255) / 256, (long long)numSMs() * 16);
  kMatrixA<<<blocks, 256, 0, s>>>(r, sx, sy, sz, code, A);
  return cudaGetLastError();
}

// y = A x (fdmMatrixVectorMulInvoker, EulerSolverTool.cu:706-720)
__global__ void kApplyA(Dim3i r, float sx, float sy, float sz, const Code* __restrict__ code,
                        const float* __restrict__ xin, float* __restrict__ y, int zPer) {
  int x = blockIdx.x * TX + threadIdx.x, yy = blockIdx.y * TY + threadIdx.y;
  if (x >= r.x || yy >= r.y) return;
  int z0 = blockIdx.z * zPer, z1 = min(z0 + zPer, r.z);
  long long plane = (long long)r.x * r.y;
  long long c = (long long)z0 * plane + (long long)yy * r.x + x;
  float below = z0 > 0 ? xin[c - plane] : 0.f, cur = xin[c];
  for (int z = z0; z < z1; ++z, c += plane) {
    float above = z + 1 < r.z ? xin[c + plane] : 0.f;
    Code k = code[c];
    float vl = x > 0 ? xin[c - 1] : 0.f, vr = x + 1 < r.x ? xin[c + 1] : 0.f;
    float vd = yy > 0 ? xin[c - r.x] : 0.f, vu = yy + 1 < r.y ? xin[c + r.x] : 0.f;
    y[c] = applyRow(k, sx, sy, sz, cur, vl, vr, vd, vu, below, above);
    below = cur;
    cur = above;
  }
}
cudaError_t launchApplyA(const Dim3i& r, float sx, float sy, float sz, const Code* code, const float* x, float* y,
                         cudaStream_t s) {
  CgGrid g = cgGrid(r);
  kApplyA<<<g.grid, g.block, 0, s>>>(r, sx, sy, sz, code, x, y, g.zPer);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// RHS: divergence (FieldMathTool.cu:370-395) + solid terms
// (EulerSolverTool.cu:128-197), fused with the CG set-up of
// CuMatrixFreePCG.cpp:22-37 (x0 = 0 so r = b).
template <int PC>
__global__ void __launch_bounds__(TX* TY) kRhsInit(Geom g, ConstFaceField v, ConstFaceField svArr, SolidVelTable svTab,
                                                   const uint8_t* __restrict__ mk, const Code* __restrict__ code,
                                                   float sAx, float sAy, float sAz, float* __restrict__ bOut,
                                                   float* __restrict__ r, float* __restrict__ xv, float* __restrict__ p,
                                                   double* partials, CgState* st, int zPer) {
  const Dim3i R = g.r;
  const float ix = 1.0f / g.hx, iy = 1.0f / g.hy, iz = 1.0f / g.hz;
  int x = blockIdx.x * TX + threadIdx.x, y = blockIdx.y * TY + threadIdx.y;
  double bb = 0.0, rzs = 0.0;
  if (x < R.x && y < R.y) {
    int z0 = blockIdx.z * zPer, z1 = min(z0 + zPer, R.z);
    const long long plane = (long long)R.x * R.y;
    const long long fxRow = R.x + 1, fxPlane = (long long)(R.x + 1) * R.y;
    const long long fyPlane = (long long)R.x * (R.y + 1);
    for (int z = z0; z < z1; ++z) {
      long long c = (long long)z * plane + (long long)y * R.x + x;
      float b = 0.f;
      if (mk[c] == kFluid) {
        long long uL = (long long)z * fxPlane + (long long)y * fxRow + x, uR = uL + 1;
        long long vD = (long long)z * fyPlane + (long long)y * R.x + x, vU = vD + R.x;
        long long wB = c, wF = c + plane;
        float L = v.c[0][uL], Rr = v.c[0][uR], D = v.c[1][vD], U = v.c[1][vU], B = v.c[2][wB], F = v.c[2][wF];
        float div = __fadd_rn(__fadd_rn(__fdiv_rn(__fsub_rn(Rr, L), g.hx), __fdiv_rn(__fsub_rn(U, D), g.hy)),
                              __fdiv_rn(__fsub_rn(F, B), g.hz));
        b = -div;
        uint8_t me = svTab.solidIdx ? svTab.solidIdx[c] : 0;
        auto sv = [&](int axis, long long f, long long nb, bool nbIsHi) -> float {
          if (svArr.c[0]) return svArr.c[axis][f];
          uint8_t o = svTab.solidIdx[nb];
          return nbIsHi ? solidFaceVel(svTab, me, o, axis) : solidFaceVel(svTab, o, me, axis);
        };
        long long cl = x > 0 ? c - 1 : c, cr = x + 1 < R.x ? c + 1 : c;
        long long cd = y > 0 ? c - R.x : c, cu = y + 1 < R.y ? c + R.x : c;
        long long cb = z > 0 ? c - plane : c, cf = z + 1 < R.z ? c + plane : c;
        if (mk[cl] == kSolid) b = __fsub_rn(b, __fmul_rn(ix, __fsub_rn(L, sv(0, uL, cl, false))));
        if (mk[cr] == kSolid) b = __fadd_rn(b, __fmul_rn(ix, __fsub_rn(Rr, sv(0, uR, cr, true))));
        if (mk[cd] == kSolid) b = __fsub_rn(b, __fmul_rn(iy, __fsub_rn(D, sv(1, vD, cd, false))));
        if (mk[cu] == kSolid) b = __fadd_rn(b, __fmul_rn(iy, __fsub_rn(U, sv(1, vU, cu, true))));
        if (mk[cb] == kSolid) b = __fsub_rn(b, __fmul_rn(iz, __fsub_rn(B, sv(2, wB, cb, false))));
        if (mk[cf] == kSolid) b = __fadd_rn(b, __fmul_rn(iz, __fsub_rn(F, sv(2, wF, cf, true))));
      }
      if (bOut) bOut[c] = b;
      r[c] = b;
      xv[c] = 0.f;
      p[c] = 0.f;
      float zz = precondZ<PC>(code[c], b, sAx, sAy, sAz);
      bb += (double)b * (double)b;
      rzs += (double)b * (double)zz;
    }
  }
  if (gridSum2(bb, rzs, partials, &st->ticket) && flatTid() == 0) {
    st->bb = bb;
    st->rr = bb;
    st->rz = rzs;
    st->iter = 0;
    st->beta = 0.f;
    st->alpha = 0.f;
    st->done = cgStop(st, bb) || st->maxIter <= 0;  // CuMatrixFreePCG.cpp:28-32
    st->ticket = 0;
  }
}
cudaError_t launchRhsInit(const Geom& gm, ConstFaceField v, ConstFaceField svArr, const SolidVelTable& svTab,
                          const uint8_t* markers, const Code* code, float ax, float ay, float az, float* b, float* r,
                          float* x, float* p, double* partials, CgState* st, int precond, cudaStream_t s) {
  CgGrid g = cgGrid(gm.r);
  if (precond == 1)
    kRhsInit<1><<<g.grid, g.block, 0, s>>>(gm, v, svArr, svTab, markers, code, ax, ay, az, b, r, x, p, partials, st,
                                           g.zPer);
  else
    kRhsInit<0><<<g.grid, g.block, 0, s>>>(gm, v, svArr, svTab, markers, code, ax, ay, az, b, r, x, p, partials, st,
                                           g.zPer);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Fast row of A for the CG: the diagonal and its reciprocal come from a
// 64-entry table per launch (indexed by the six "not solid" bits; the entries
// are summed in the reference's order), the six off-diagonal terms are FP32
// FMAs on masked neighbour values.
struct DiagTab {
  float d[64], inv[64];
};

__device__ __forceinline__ void buildDiagTab(DiagTab& t, float sx, float sy, float sz) {
  const int tid = flatTid();
  if (tid < 64) {
    Code k = (Code)(1 | (tid << 1));
    float d = diagOf(k, sx, sy, sz);
    t.d[tid] = d;
    t.inv[tid] = d != 0.f ? 1.0f / d : 0.f;
  }
}

__device__ __forceinline__ float fastRow(const DiagTab& t, Code k, float sx, float sy, float sz, float vc, float vl,
                                         float vr, float vd, float vu, float vb, float vf) {
  if (!(k & 1)) return vc;
  float nx = ((k >> 7) & 1 ? vl : 0.f) + ((k >> 8) & 1 ? vr : 0.f);
  float ny = ((k >> 9) & 1 ? vd : 0.f) + ((k >> 10) & 1 ? vu : 0.f);
  float nz = ((k >> 11) & 1 ? vb : 0.f) + ((k >> 12) & 1 ? vf : 0.f);
  float q = t.d[(k >> 1) & 63] * vc;
  q = fmaf(-sx, nx, q);
  q = fmaf(-sy, ny, q);
  q = fmaf(-sz, nz, q);
  return q;
}

template <int PC>
__device__ __forceinline__ float fastZ(const DiagTab& t, Code k, float rv) {
  if (PC != 1) return rv;
  return (k & 1) ? rv * t.inv[(k >> 1) & 63] : rv;
}

// CG direction: p = z + beta p_old (scal then axpy with 1), q = A p and the
// reduction p.q; the last block forms alpha = r.z / p.Ap
// (CuMatrixFreePCG.cpp:40-47, :56-60).  p of the current plane (with a one-
// cell halo) sits in a double-buffered shared tile, p below / above in
// registers; every p value is formed once per cell plus the halo ring.
template <int PC>
__global__ void __launch_bounds__(TX* TY, 4) kCgDirection(Dim3i R, float sx, float sy, float sz,
                                                          const Code* __restrict__ code, const float* __restrict__ r,
                                                          const float* __restrict__ pOld, float* __restrict__ pNew,
                                                          double* partials, CgState* st, int zPer) {
  if (st->done) return;
  __shared__ float tile[2][TY + 2][TX + 2];
  __shared__ DiagTab tab;
  buildDiagTab(tab, sx, sy, sz);
  __syncthreads();
  const float beta = st->beta;
  double pq = 0.0, dummy = 0.0;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int x = blockIdx.x * TX + tx, y = blockIdx.y * TY + ty;
  const bool in = x < R.x && y < R.y;
  const int z0 = blockIdx.z * zPer, z1 = min(z0 + zPer, R.z);
  const unsigned plane = (unsigned)R.x * (unsigned)R.y;
  auto pn = [&](unsigned i) -> float {
    float zz = fastZ<PC>(tab, __ldg(code + i), __ldg(r + i));
    return fmaf(beta, __ldg(pOld + i), zz);
  };
  unsigned c = (unsigned)z0 * plane + (unsigned)y * (unsigned)R.x + (unsigned)x;
  float below = (in && z0 > 0) ? pn(c - plane) : 0.f;
  float cur = in ? pn(c) : 0.f;
  float acc = 0.f;
  int buf = 0;
  for (int z = z0; z < z1; ++z, c += plane, buf ^= 1) {
    float above = (in && z + 1 < R.z) ? pn(c + plane) : 0.f;
    Code k = in ? __ldg(code + c) : (Code)0;
    float (*t)[TX + 2] = tile[buf];
    t[ty + 1][tx + 1] = cur;
    if (tx == 0) t[ty + 1][0] = (in && x > 0) ? pn(c - 1) : 0.f;
    if (tx == TX - 1 || x == R.x - 1) t[ty + 1][tx + 2] = (in && x + 1 < R.x) ? pn(c + 1) : 0.f;
    if (ty == 0) t[0][tx + 1] = (in && y > 0) ? pn(c - R.x) : 0.f;
    if (ty == TY - 1 || y == R.y - 1) t[ty + 2][tx + 1] = (in && y + 1 < R.y) ? pn(c + R.x) : 0.f;
    __syncthreads();
    if (in) {
      float q = fastRow(tab, k, sx, sy, sz, cur, t[ty + 1][tx], t[ty + 1][tx + 2], t[ty][tx + 1], t[ty + 2][tx + 1],
                        below, above);
      pNew[c] = cur;
      acc = fmaf(cur, q, acc);
    }
    below = cur;
    cur = above;
  }
  pq = (double)acc;
  if (gridSum2(pq, dummy, partials, &st->ticket) && flatTid() == 0) {
    st->pAp = pq;
    st->alpha = (float)(st->rz / pq);
    st->ticket = 0;
  }
}

// CG update: x += alpha p, r -= alpha A p (A p recomputed from the stored p
// through the same shared tile), z = M^-1 r, the reductions r.r and r.z; the
// last block checks convergence and forms beta (CuMatrixFreePCG.cpp:49-63).
// The |alpha| < FLT_EPSILON skip of CCuDenseVector::plusAlphaX
// (CuDenseVector.cpp:178) is kept.  Per-thread partial sums run over one
// z-column segment in FP32 and are combined in FP64.
template <int PC>
__global__ void __launch_bounds__(TX* TY, 4) kCgUpdate(Dim3i R, float sx, float sy, float sz,
                                                       const Code* __restrict__ code, const float* __restrict__ p,
                                                       float* __restrict__ xv, float* __restrict__ r,
                                                       double* partials, CgState* st, int zPer) {
  if (st->done) return;
  __shared__ float tile[2][TY + 2][TX + 2];
  __shared__ DiagTab tab;
  buildDiagTab(tab, sx, sy, sz);
  __syncthreads();
  const float alpha = st->alpha;
  const bool skip = fabsf(alpha) < FLT_EPSILON;
  float arr = 0.f, arz = 0.f;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int x = blockIdx.x * TX + tx, y = blockIdx.y * TY + ty;
  const bool in = x < R.x && y < R.y;
  const int z0 = blockIdx.z * zPer, z1 = min(z0 + zPer, R.z);
  const unsigned plane = (unsigned)R.x * (unsigned)R.y;
  unsigned c = (unsigned)z0 * plane + (unsigned)y * (unsigned)R.x + (unsigned)x;
  float below = (in && z0 > 0) ? __ldg(p + c - plane) : 0.f;
  float cur = in ? __ldg(p + c) : 0.f;
  int buf = 0;
  for (int z = z0; z < z1; ++z, c += plane, buf ^= 1) {
    float above = (in && z + 1 < R.z) ? __ldg(p + c + plane) : 0.f;
    Code k = in ? __ldg(code + c) : (Code)0;
    float rv = in ? r[c] : 0.f;
    float xo = (in && !skip) ? xv[c] : 0.f;
    float (*t)[TX + 2] = tile[buf];
    t[ty + 1][tx + 1] = cur;
    if (tx == 0) t[ty + 1][0] = (in && x > 0) ? __ldg(p + c - 1) : 0.f;
    if (tx == TX - 1 || x == R.x - 1) t[ty + 1][tx + 2] = (in && x + 1 < R.x) ? __ldg(p + c + 1) : 0.f;
    if (ty == 0) t[0][tx + 1] = (in && y > 0) ? __ldg(p + c - R.x) : 0.f;
    if (ty == TY - 1 || y == R.y - 1) t[ty + 2][tx + 1] = (in && y + 1 < R.y) ? __ldg(p + c + R.x) : 0.f;
    __syncthreads();
    if (in) {
      if (!skip) {
        float q = fastRow(tab, k, sx, sy, sz, cur, t[ty + 1][tx], t[ty + 1][tx + 2], t[ty][tx + 1], t[ty + 2][tx + 1],
                          below, above);
        xv[c] = fmaf(alpha, cur, xo);
        rv = fmaf(-alpha, q, rv);
        r[c] = rv;
      }
      float zz = fastZ<PC>(tab, k, rv);
      arr = fmaf(rv, rv, arr);
      arz = fmaf(rv, zz, arz);
    }
    below = cur;
    cur = above;
  }
  double rr = (double)arr, rz = (double)arz;
  if (gridSum2(rr, rz, partials, &st->ticket) && flatTid() == 0) {
    st->rr = rr;
    st->iter += 1;
    bool stop = cgStop(st, rr);
    if (PC != 2) {  // with multigrid the V-cycle's last sweep forms r.z and beta
      st->beta = (float)(rz / st->rz);
      st->rz = rz;
    }
    st->done = stop || st->iter >= st->maxIter;
    st->ticket = 0;
  }
}

cudaError_t launchCgDirection(const Dim3i& r, float sx, float sy, float sz, const Code* code, const float* rr,
                              const float* pOld, float* pNew, double* partials, CgState* st, int precond,
                              cudaStream_t s) {
  CgGrid g = cgGrid(r);
  if (precond == 1)
    kCgDirection<1><<<g.grid, g.block, 0, s>>>(r, sx, sy, sz, code, rr, pOld, pNew, partials, st, g.zPer);
  else
    kCgDirection<0><<<g.grid, g.block, 0, s>>>(r, sx, sy, sz, code, rr, pOld, pNew, partials, st, g.zPer);
  return cudaGetLastError();
}
cudaError_t launchCgUpdate(const Dim3i& r, float sx, float sy, float sz, const Code* code, const float* p, float* x,
                           float* rr, double* partials, CgState* st, int precond, cudaStream_t s) {
  CgGrid g = cgGrid(r);
  if (precond == 1)
    kCgUpdate<1><<<g.grid, g.block, 0, s>>>(r, sx, sy, sz, code, p, x, rr, partials, st, g.zPer);
  else
    kCgUpdate<0><<<g.grid, g.block, 0, s>>>(r, sx, sy, sz, code, p, x, rr, partials, st, g.zPer);
  return cudaGetLastError();
}

// Multigrid flavour: z is read from memory (the V-cycle's output).
cudaError_t launchCgDirectionZ(const Dim3i& r, float sx, float sy, float sz, const Code* code, const float* z,
                               const float* pOld, float* pNew, double* partials, CgState* st, cudaStream_t s) {
  CgGrid g = cgGrid(r);
  kCgDirection<2><<<g.grid, g.block, 0, s>>>(r, sx, sy, sz, code, z, pOld, pNew, partials, st, g.zPer);
  return cudaGetLastError();
}
cudaError_t launchCgUpdateNoZ(const Dim3i& r, float sx, float sy, float sz, const Code* code, const float* p,
                              float* x, float* rr, double* partials, CgState* st, cudaStream_t s) {
  CgGrid g = cgGrid(r);
  kCgUpdate<2><<<g.grid, g.block, 0, s>>>(r, sx, sy, sz, code, p, x, rr, partials, st, g.zPer);
  return cudaGetLastError();
}

}  // namespace hfg
