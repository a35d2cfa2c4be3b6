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
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

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


// ---------------------------------------------------------------------------
__global__ void kStencilCode(Dim3i r, int px, const uint8_t* __restrict__ mk, Code* __restrict__ code,
                             CgCode* __restrict__ cgc, int zPer) {
  int x = blockIdx.x * TX + threadIdx.x, y = blockIdx.y * TY + threadIdx.y;
  if (x >= px || y >= r.y) return;
  int z0 = blockIdx.z * zPer, z1 = min(z0 + zPer, r.z);
  long long plane = (long long)r.x * r.y;
  for (int z = z0; z < z1; ++z) {
    long long c = (long long)z * plane + (long long)y * r.x + x;
    long long o = ((long long)z * r.y + y) * px + x;
    Code k = 0;
    if (x < r.x && mk[c] == kFluid) {
      k = 1;
      const bool in[6] = {x > 0, x + 1 < r.x, y > 0, y + 1 < r.y, z > 0, z + 1 < r.z};
      const long long d6[6] = {-1, 1, -(long long)r.x, (long long)r.x, -plane, plane};
#pragma unroll
      for (int d = 0; d < 6; ++d) {
        if (!in[d]) continue;
        uint8_t m = mk[c + d6[d]];
        if (m != kSolid) k |= (Code)(1u << (1 + d));
        if (m == kFluid) k |= (Code)(1u << (7 + d));
      }
    }
    code[o] = k;
    if (cgc) cgc[o] = (CgCode)(k & 0x7f);
  }
}
cudaError_t launchStencilCode(const Dim3i& r, int px, const uint8_t* markers, Code* code, cudaStream_t s,
                              CgCode* cgc) {
  CgGrid g = cgGrid(Dim3i{px, r.y, r.z});
  kStencilCode<<<g.grid, g.block, 0, s>>>(r, px, markers, code, cgc, g.zPer);
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
// b of one cell: -div u plus the solid-face terms (FieldMathTool.cu:370-395,
// EulerSolverTool.cu:128-197), in the reference's operation order; 0 for
// non-fluid cells.
__device__ __forceinline__ float rhsAt(const Geom& g, const ConstFaceField& v, const ConstFaceField& svArr,
                                       const SolidVelTable& svTab, const uint8_t* __restrict__ mk, int x, int y,
                                       int z) {
  const Dim3i R = g.r;
  const long long plane = (long long)R.x * R.y;
  const long long c = (long long)z * plane + (long long)y * R.x + x;
  if (mk[c] != kFluid) return 0.f;
  const float ix = 1.0f / g.hx, iy = 1.0f / g.hy, iz = 1.0f / g.hz;
  const long long fxRow = R.x + 1, fxPlane = (long long)(R.x + 1) * R.y;
  const long long fyPlane = (long long)R.x * (R.y + 1);
  long long uL = (long long)z * fxPlane + (long long)y * fxRow + x, uR = uL + 1;
  long long vD = (long long)z * fyPlane + (long long)y * R.x + x, vU = vD + R.x;
  long long wB = c, wF = c + plane;
  float L = v.c[0][uL], Rr = v.c[0][uR], D = v.c[1][vD], U = v.c[1][vU], B = v.c[2][wB], F = v.c[2][wF];
  float div = __fadd_rn(__fadd_rn(__fdiv_rn(__fsub_rn(Rr, L), g.hx), __fdiv_rn(__fsub_rn(U, D), g.hy)),
                        __fdiv_rn(__fsub_rn(F, B), g.hz));
  float b = -div;
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
  return b;
}

// Divergence residual of a projected field: sum of b^2 over the fluid cells
// (FP64, last-block reduction) and max |b| (ordered-bits atomic max).
__global__ void kDivergenceNorm(Geom g, ConstFaceField v, ConstFaceField svArr, SolidVelTable svTab,
                                const uint8_t* __restrict__ mk, double* partials, unsigned* ticket,
                                double* sumOut, unsigned* maxBits) {
  double s2 = 0.0, dummy = 0.0;
  float mx = 0.f;
  const long long n = g.r.size();
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(c % g.r.x);
    const long long t = c / g.r.x;
    const int y = (int)(t % g.r.y), z = (int)(t / g.r.y);
    float b = rhsAt(g, v, svArr, svTab, mk, x, y, z);
    s2 += (double)b * (double)b;
    mx = fmaxf(mx, fabsf(b));
  }
  mx = warpMaxF(mx);
  if ((threadIdx.x & 31) == 0) atomicMax(maxBits, __float_as_uint(mx));
  if (gridSum2(s2, dummy, partials, ticket) && flatTid() == 0) {
    *sumOut = s2;
    *ticket = 0;
  }
}

// The final residual check of a pressure solve, in FP64 on the GPU:
// ||b - A x||^2 and ||b||^2 over the fluid cells.  b is recomputed from the
// unprojected velocity (rhsAt, the reference's operation order), the entries
// of A are the FP32 system's scales promoted to FP64 (fdmMatrixVectorMul,
// EulerSolverTool.cu:199-227, with diagonal and neighbour terms from the
// stencil code) and x is read as stored (FP32 or FP64).  The CG's own
// recurrence residual drifts from this once FP32 round-off builds up.
__global__ void kTrueResidual(Geom g, ConstFaceField v, SolidVelTable svTab, const uint8_t* __restrict__ mk,
                              const Code* __restrict__ code, const void* __restrict__ xv, int xDouble, double sx,
                              double sy, double sz, double* partials, unsigned* ticket, double* out) {
  double rr = 0.0, bb = 0.0;
  const Dim3i R = g.r;
  const long long px = cgPitch(R.x), pl = px * R.y;
  const ConstFaceField none{{nullptr, nullptr, nullptr}};
  auto X = [&](long long i) -> double {
    return xDouble ? ((const double*)xv)[i] : (double)((const float*)xv)[i];
  };
  const long long n = R.size();
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    if (mk[c] != kFluid) continue;
    const int x = (int)(c % R.x);
    const long long t = c / R.x;
    const int y = (int)(t % R.y), z = (int)(t / R.y);
    const double b = (double)rhsAt(g, v, none, svTab, mk, x, y, z);
    const long long o = ((long long)z * R.y + y) * px + x;
    const Code k = code[o];
    double diag = 0.0;
    if (k & 2) diag += sx;
    if (k & 4) diag += sx;
    if (k & 8) diag += sy;
    if (k & 16) diag += sy;
    if (k & 32) diag += sz;
    if (k & 64) diag += sz;
    double ax = diag * X(o);
    if (nbFluid(k, 0)) ax -= sx * X(o - 1);
    if (nbFluid(k, 1)) ax -= sx * X(o + 1);
    if (nbFluid(k, 2)) ax -= sy * X(o - px);
    if (nbFluid(k, 3)) ax -= sy * X(o + px);
    if (nbFluid(k, 4)) ax -= sz * X(o - pl);
    if (nbFluid(k, 5)) ax -= sz * X(o + pl);
    const double r = b - ax;
    rr += r * r;
    bb += b * b;
  }
  if (gridSum2(rr, bb, partials, ticket) && flatTid() == 0) {
    out[0] = rr;
    out[1] = bb;
    *ticket = 0;
  }
}
cudaError_t launchTrueResidual(const Geom& g, ConstFaceField v, const SolidVelTable& svTab, const uint8_t* markers,
                               const Code* code, const void* x, bool xDouble, float sx, float sy, float sz,
                               double* scratch, unsigned* ticket, double* out, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(ticket, 0, sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  kTrueResidual<<<divergenceBlocks(), 256, 0, s>>>(g, v, svTab, markers, code, x, xDouble ? 1 : 0, (double)sx,
                                                   (double)sy, (double)sz, scratch, ticket, out);
  return cudaGetLastError();
}

template <int PC>
__global__ void __launch_bounds__(TX* TY) kRhsInit(Geom g, ConstFaceField v, ConstFaceField svArr, SolidVelTable svTab,
                                                   const uint8_t* __restrict__ mk, const Code* __restrict__ code,
                                                   float sAx, float sAy, float sAz, float* __restrict__ bOut,
                                                   float* __restrict__ r, void* __restrict__ xv, int xDouble,
                                                   float* __restrict__ p, double* partials, CgState* st, int zPer) {
  const Dim3i R = g.r;
  const int px = cgPitch(R.x);
  int x = blockIdx.x * TX + threadIdx.x, y = blockIdx.y * TY + threadIdx.y;
  double bb = 0.0, rzs = 0.0;
  if (x >= R.x && x < px && y < R.y) {  // pitch padding: inert cells
    int z0 = blockIdx.z * zPer, z1 = min(z0 + zPer, R.z);
    for (int z = z0; z < z1; ++z) {
      long long o = ((long long)z * R.y + y) * px + x;
      r[o] = 0.f;
      if (xDouble) ((double*)xv)[o] = 0.0;
      else ((float*)xv)[o] = 0.f;
      p[o] = 0.f;
    }
  }
  if (x < R.x && y < R.y) {
    int z0 = blockIdx.z * zPer, z1 = min(z0 + zPer, R.z);
    const long long plane = (long long)R.x * R.y;
    for (int z = z0; z < z1; ++z) {
      long long c = (long long)z * plane + (long long)y * R.x + x;
      float b = rhsAt(g, v, svArr, svTab, mk, x, y, z);
      if (bOut) bOut[c] = b;
      long long o = ((long long)z * R.y + y) * px + x;
      r[o] = b;
      if (xDouble) ((double*)xv)[o] = 0.0;
      else ((float*)xv)[o] = 0.f;
      p[o] = 0.f;
      float zz = precondZ<PC>(code[o], b, sAx, sAy, sAz);
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
                          void* x, bool xDouble, float* p, double* partials, CgState* st, int precond,
                          cudaStream_t s) {
  CgGrid g = cgGrid(cgDims(gm.r));
  const int xd = xDouble ? 1 : 0;
  if (precond == 1)
    kRhsInit<1><<<g.grid, g.block, 0, s>>>(gm, v, svArr, svTab, markers, code, ax, ay, az, b, r, x, xd, p, partials,
                                           st, g.zPer);
  else
    kRhsInit<0><<<g.grid, g.block, 0, s>>>(gm, v, svArr, svTab, markers, code, ax, ay, az, b, r, x, xd, p, partials,
                                           st, g.zPer);
  return cudaGetLastError();
}

cudaError_t launchDivergenceNorm(const Geom& g, ConstFaceField v, const SolidVelTable& svTab,
                                 const uint8_t* markers, double* scratch, unsigned* ticketAndMax, double* sumOut,
                                 cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(ticketAndMax, 0, 2 * sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  ConstFaceField none{{nullptr, nullptr, nullptr}};
  kDivergenceNorm<<<divergenceBlocks(), 256, 0, s>>>(g, v, none, svTab, markers, scratch, ticketAndMax, sumOut,
                                                     ticketAndMax + 1);
  return cudaGetLastError();
}

namespace {
// ---------------------------------------------------------------------------
// Fast row of A for the CG: the diagonal and its reciprocal come from a
// 128-entry table per launch, indexed by the whole 7-bit CG code (fluid bit
// and the six "not solid" bits; the entries are summed in the reference's
// order), and the six off-diagonal terms are FP32 FMAs on the neighbour
// values.  The non-fluid codes hold (-1, 1): the Jacobi preconditioner then
// needs no test of the fluid bit (r * 1 = r), and a negative diagonal marks
// a non-fluid cell (a fluid diagonal is a sum of positive scales, or 0).
struct DiagTab {
  float2 e[128];  // (diagonal, its reciprocal)
};

__device__ __forceinline__ void buildDiagTab(DiagTab& t, float sx, float sy, float sz) {
  const int tid = flatTid();
  if (tid < 128) {
    float d = -1.f, inv = 1.f;
    if (tid & 1) {
      d = diagOf((Code)tid, sx, sy, sz);
      inv = d != 0.f ? 1.0f / d : 0.f;
    }
    t.e[tid] = make_float2(d, inv);
  }
}

// Row sum of A at a fluid cell: d vc minus the six off-diagonal terms, d the
// diagonal of the cell's code.  The neighbour values need no masks here.  The
// CG vectors p, r and z are zero at every cell that is not fluid: b is zero
// there, the row of A is the identity, and the Jacobi and multigrid
// preconditioners write zero there, so r -= alpha A p and p = z + beta p keep
// them zero.  The halo outside the grid arrives zero-filled and the pitch
// padding is zero too.  So the only neighbours that add anything are the
// fluid ones, as in the reference's off-diagonal terms, and the sum is the
// masked sum up to the sign of a zero.  At a non-fluid cell the row is the
// identity and every CG vector stays zero for the whole solve (the RHS kernel
// zeroes x, r and p there, and the updates add alpha or beta times zero), so
// the CG kernels neither form the row nor store anything there.
__device__ __forceinline__ float rowSum(float d, float sx, float sy, float sz, float vc, float vl, float vr, float vd,
                                        float vu, float vb, float vf) {
  float q = d * vc;
  q = fmaf(-sx, vl + vr, q);
  q = fmaf(-sy, vd + vu, q);
  q = fmaf(-sz, vb + vf, q);
  return q;
}

template <int PC>
__device__ __forceinline__ float fastZ(float inv, float rv) {
  if (PC != 1) return rv;
  return rv * inv;
}

// ---------------------------------------------------------------------------
// TMA plumbing.  Each CG block owns a 32 x 8 column of the pitched grid and
// marches along z; one elected thread streams the planes ahead of the
// consumers into a ring of shared-memory stages with cp.async.bulk.tensor,
// completion tracked by one mbarrier per stage.  The halo boxes start 4
// floats (8 codes) left of the tile so that every box starts on a 16-byte
// boundary; boxes outside the grid arrive zero-filled.
constexpr int CTX = 32, CTY = 8;     // threads per block (x, y)
constexpr int RY = 2;                // rows per thread: thread (tx, ty) owns rows ty and ty + CTY
constexpr int CTR = CTY * RY;        // 16 tile rows per plane
static_assert(2 * CTR == CTX, "one warp computes both halo columns (one lane per halo cell)");
constexpr int HXF = 4, HXC = 16;     // left pad of the float / code halo boxes (16 bytes)
constexpr int FW = CTX + 2 * HXF;    // 40 floats
constexpr int CW = CTX + 2 * HXC;    // 64 codes
constexpr int FH = CTR + 2;          // 18 rows
constexpr int kDirStages = 4, kUpdStages = 5;
constexpr unsigned long long kWaitNs = 2000000000ull;  // a stage that takes 2 s to land is an error

__device__ __forceinline__ void tmaLoad3(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smemAddr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smemAddr(bar))
      : "memory");
}

// Marks the solve failed; the host sees `error` and stops.
__device__ __forceinline__ void cgFail(CgState* st, int code) {
  atomicExch(&st->error, code);
  atomicExch(&st->done, 1);
}

// Blocks that gave up still drain every stage they issued (bounded) before
// the shared memory is released.
template <int S>
__device__ void drainStages(uint64_t* bar, const int* issued, int waited) {
  unsigned long long deadline = globalNs() + kWaitNs;
  for (int i = waited; i < issued[0]; ++i)
    if (!mbarWait(&bar[i % S], (unsigned)((i / S) & 1), deadline)) break;
}

struct __align__(128) DirStage {
  alignas(128) float r[FH][FW];
  alignas(128) float po[FH][FW];
  alignas(128) CgCode code[FH][CW];
};
constexpr unsigned kDirStageBytes = sizeof(float) * FH * FW * 2 + sizeof(CgCode) * FH * CW;

// TX: the pressure iterate x in FP32 (the reference's Real) or FP64.
template <class TX> struct __align__(128) UpdStage {
  alignas(128) float p[FH][FW];
  alignas(128) float r[CTR][CTX];
  alignas(128) TX x[CTR][CTX];
  alignas(128) CgCode code[CTR][CTX];
};
template <class TX>
constexpr unsigned kUpdStageBytes = sizeof(float) * (FH * FW + CTR * CTX) + sizeof(TX) * CTR * CTX + sizeof(CgCode) * CTR * CTX;
template <class TX> constexpr int kUpdStagesT = sizeof(TX) == 8 ? 4 : kUpdStages;  // keeps static shared memory < 48 KB

struct CgLaunch {
  dim3 grid, block;
  int zPer;
};

// The CG schedule of a solve (launchCgSchedule), in one int array:
//   [0, cols)            the lowest plane holding a fluid cell of each tile
//                        column (CTX x CTR cells of the pitched grid, all z),
//   [cols, 2 cols)       the highest (a range no plane meets: no fluid),
//   [2 cols]             the number of work items,
//   [schedItemsOffset)   the items (column, z0, z1, 0): one per CG block, the
//                        fluid planes of the active columns cut into chunks
//                        so that the items about fill one wave of blocks.
// A block past the last item only joins the reductions.  Null: the dense
// grid, block (x, y, z) on tile (x, y) and planes [z zPer, (z + 1) zPer).
static_assert(CTX == kCgTileX && CTR == kCgTileY, "the schedule's tile is the CG kernels' tile");

// A work item that is not a run of planes of a column of this grid (or a
// count beyond the grid) is not used: the block stays idle and the solve
// reports error 4.
__device__ __forceinline__ bool cgBlockWork(const int* sched, const Dim3i& P, int zPer, int& x0, int& y0, int& z0,
                                            int& z1, CgState* st) {
  if (!sched) {
    x0 = blockIdx.x * CTX;
    y0 = blockIdx.y * CTR;
    z0 = blockIdx.z * zPer;
    z1 = min(z0 + zPer, P.z);
    return true;
  }
  x0 = y0 = z0 = z1 = 0;
  const int tilesX = (P.x + CTX - 1) / CTX, cols = tilesX * ((P.y + CTR - 1) / CTR);
  const int n = __ldg(sched + 2 * cols);
  if (n < 0 || n > (int)gridDim.x) {
    if (threadIdx.x == 0 && threadIdx.y == 0) cgFail(st, 4);
    return false;
  }
  if ((int)blockIdx.x >= n) return false;
  const int4 w = __ldg(reinterpret_cast<const int4*>(sched + schedItemsOffset(cols)) + blockIdx.x);
  if (w.x < 0 || w.x >= cols || w.y < 0 || w.y >= w.z || w.z > P.z) {
    if (threadIdx.x == 0 && threadIdx.y == 0) cgFail(st, 4);
    return false;
  }
  x0 = (w.x % tilesX) * CTX;
  y0 = (w.x / tilesX) * CTR;
  z0 = w.y;
  z1 = w.z;
  return true;
}

// Tiles over (x, y), z split into chunks so that the blocks fill whole waves
// of the resident slots (wave count x chunk length minimal, chunks of at
// least 3 planes).
int residentBlocks(const void* kernel) {
  static std::mutex mu;
  static std::map<const void*, int> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(kernel);
  if (it != cache.end()) return it->second;
  int per = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, CTX * CTY, 0) != cudaSuccess || per <= 0) per = 1;
  cache[kernel] = per;
  return per;
}

}  // namespace

// Work items of a CG schedule: one wave of the CG kernels of this
// preconditioner (the fewest resident blocks of the direction and both update
// kernels, at most kSchedPerSM per SM).
constexpr int kSchedPerSM = 8;
int cgScheduleTarget(int precond, bool xDouble);

// ---------------------------------------------------------------------------
// Launch shapes picked by measurement.  autotuneCg (driven by the solver)
// times the CG kernels of a grid for every z-chunk length in kTuneZPer and
// records the fastest per kernel family; cgLaunch prefers a recorded shape to
// its cost model.  The table is process wide and can be saved and loaded.
namespace {
constexpr int kTuneZPer[] = {3, 4, 5, 6, 8, 10, 12, 16, 20, 24, 32, 48, 64};
std::mutex g_tuneMu;
std::map<std::string, int> g_tune;  // "cg<family> nx ny nz" -> zPer

std::string tuneKey(int family, const Dim3i& cg) {
  return "cg" + std::to_string(family) + " " + std::to_string(cg.x) + " " + std::to_string(cg.y) + " " +
         std::to_string(cg.z);
}
int tunedZPer(int family, const Dim3i& cg) {
  std::lock_guard<std::mutex> lk(g_tuneMu);
  auto it = g_tune.find(tuneKey(family, cg));
  return it == g_tune.end() ? -1 : it->second;
}
}  // namespace

void setTunedCgZPer(int family, const Dim3i& cg, int zPer) {
  std::lock_guard<std::mutex> lk(g_tuneMu);
  if (zPer > 0) g_tune[tuneKey(family, cg)] = zPer;
  else g_tune.erase(tuneKey(family, cg));
}
int tunedCgZPer(int family, const Dim3i& cg) { return tunedZPer(family, cg); }
std::vector<int> cgZPerCandidates(const Dim3i& cg) {
  std::vector<int> v;
  for (int z : kTuneZPer)
    if (z <= cg.z) v.push_back(z);
  if (v.empty()) v.push_back(cg.z);
  return v;
}
bool saveTuning(const char* path) {
  std::lock_guard<std::mutex> lk(g_tuneMu);
  FILE* f = std::fopen(path, "w");
  if (!f) return false;
  std::fprintf(f, "# hfgrid launch shapes: cg<family 0 direction, 1 update> px ny nz zPer\n");
  for (const auto& kv : g_tune) std::fprintf(f, "%s %d\n", kv.first.c_str(), kv.second);
  return std::fclose(f) == 0;
}
int loadTuning(const char* path) {
  FILE* f = std::fopen(path, "r");
  if (!f) return -1;
  char name[16];
  int x, y, z, per, n = 0;
  char line[256];
  while (std::fgets(line, sizeof line, f)) {
    if (line[0] == '#') continue;
    if (std::sscanf(line, "%15s %d %d %d %d", name, &x, &y, &z, &per) != 5) continue;
    if ((std::string(name) != "cg0" && std::string(name) != "cg1") || per < 1 || per > z) continue;
    setTunedCgZPer(name[2] - '0', Dim3i{x, y, z}, per);
    ++n;
  }
  std::fclose(f);
  return n;
}

namespace {
// family: 0 for kCgDirection, 1 for kCgUpdate (the key of the tuning table).
// With a schedule the grid is one block per possible work item.
template <class K>
CgLaunch cgLaunch(const Dim3i& cg, K kernel, int family, const int* sched = nullptr, int precond = 1,
                  bool xDouble = false) {
  CgLaunch L;
  L.block = dim3(CTX, CTY, 1);
  if (sched) {
    L.zPer = 0;
    L.grid = dim3(cgScheduleTarget(precond, xDouble) + cgColumns(cg), 1, 1);
    return L;
  }
  int bx = (cg.x + CTX - 1) / CTX, by = (cg.y + CTR - 1) / CTR;
  const int tuned = tunedZPer(family, cg);
  if (tuned > 0) {
    L.zPer = std::min(tuned, cg.z);
    L.grid = dim3(bx, by, (cg.z + L.zPer - 1) / L.zPer);
    return L;
  }
  long long slots = (long long)numSMs() * residentBlocks((const void*)kernel);
  long long tiles = (long long)bx * by;
  long long best = -1;
  int bestPer = cg.z;
  // chunks of at least 3 planes: on small grids one-plane chunks pay the
  // ring's fill and a block's set-up for every plane (64^3: 16.1 us per
  // iteration with 1 plane, 15.2 with 3, 15.3 with 4, 19.2 with 8; 96^3:
  // 22.3 with 3, 24.1 with 4)
  for (int zPer = std::min(3, cg.z); zPer <= cg.z; ++zPer) {
    long long zc = (cg.z + zPer - 1) / zPer;
    long long waves = (tiles * zc + slots - 1) / slots;
    long long cost = waves * (zPer + 2);  // +2: pipeline fill per block
    if (best < 0 || cost < best) {
      best = cost;
      bestPer = zPer;
    }
  }
  L.zPer = bestPer;
  L.grid = dim3(bx, by, (cg.z + bestPer - 1) / bestPer);
  return L;
}

// CG direction: p = z + beta p_old (scal then axpy with 1), q = A p and the
// reduction p.q; the last block forms alpha = r.z / p.Ap
// (CuMatrixFreePCG.cpp:40-47, :56-60).  Stage i of the ring holds raw (z or r,
// p_old, code) of plane z0 + i with a one-cell halo; p of each plane (with
// halo) is formed once into a double-buffered tile, p above / below the
// current plane stay in registers.  PC: 0 identity, 1 Jacobi, 2 z from
// memory (multigrid).
template <int PC>
__global__ void __launch_bounds__(CTX* CTY, 4)
    kCgDirection(const __grid_constant__ CUtensorMap mZ, const __grid_constant__ CUtensorMap mPo,
                 const __grid_constant__ CUtensorMap mCode, Dim3i P, float sx, float sy, float sz,
                 const CgCode* __restrict__ code, const float* __restrict__ zr, const float* __restrict__ pOld,
                 float* __restrict__ pNew, double* partials, CgState* st, int zPer, const int* __restrict__ colZ) {
  __shared__ DirStage stg[kDirStages];
  __shared__ float pt[2][FH][CTX + 2];
  __shared__ DiagTab tab;
  __shared__ __align__(8) uint64_t bar[kDirStages];
  __shared__ int issued;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * CTX + tx;
  int x0 = 0, y0 = 0, z0 = 0, z1 = 0;
  auto issue = [&](int i) {
    DirStage& S = stg[i % kDirStages];
    uint64_t* b = &bar[i % kDirStages];
    mbarExpectTx(b, kDirStageBytes);
    tmaLoad3(&S.r[0][0], &mZ, x0 - HXF, y0 - 1, z0 + i, b);
    tmaLoad3(&S.po[0][0], &mPo, x0 - HXF, y0 - 1, z0 + i, b);
    tmaLoad3(&S.code[0][0], &mCode, x0 - HXC, y0 - 1, z0 + i, b);
  };
  if (tid == 0) {
    for (int s = 0; s < kDirStages; ++s) mbarInit(&bar[s], 1);
    mbarFenceInit();
  }
  buildDiagTab(tab, sx, sy, sz);
  __syncthreads();
  waitPrevGrid();
  if (st->done) return;  // the same value in every thread
  allowNextGrid();
  // a block with no work item (sched) writes nothing and adds zero to the
  // reduction; the schedule was written before the kernels before this one
  const bool active = cgBlockWork(colZ, P, zPer, x0, y0, z0, z1, st);
  const int nPlanes = active ? z1 - z0 : 0, nLoad = nPlanes + 1;  // plane z1 is the last "above"
  if (tid == 0) {
    int n = active ? min(kDirStages, nLoad) : 0;
    for (int i = 0; i < n; ++i) issue(i);
    issued = n;
  }
  const float beta = st->beta;
  const unsigned long long deadline = globalNs() + kWaitNs;
  const int x = x0 + tx;
  const unsigned plane = (unsigned)P.x * (unsigned)P.y;
  bool in[RY];
  unsigned c[RY];
  float below[RY], cur[RY], above[RY];
  float dCur[RY], dAbove[RY];
#pragma unroll
  for (int j = 0; j < RY; ++j) {
    const int y = y0 + ty + j * CTY;
    in[j] = x < P.x && y < P.y;
    c[j] = (unsigned)z0 * plane + (unsigned)y * (unsigned)P.x + (unsigned)x;
    // p of the plane below the chunk, own cell only
    below[j] = 0.f;
    if (active && in[j] && z0 > 0) {
      unsigned b = c[j] - plane;
      below[j] = fmaf(beta, __ldg(pOld + b), fastZ<PC>(tab.e[__ldg(code + b)].y, __ldg(zr + b)));
    }
  }
  // p of stage i's plane into tile t: the thread's RY cells, the x halo of its
  // rows and, for the edge warps, the y halo rows; own p and diagonals returned
  auto formTile = [&](int i, float (*t)[CTX + 2], float* v, float* dOwn) {
    const DirStage& S = stg[i % kDirStages];
    auto pAt = [&](int row, int colF, int colC) {
      return fmaf(beta, S.po[row][colF], fastZ<PC>(tab.e[S.code[row][colC]].y, S.r[row][colF]));
    };
#pragma unroll
    for (int j = 0; j < RY; ++j) {
      const int row = ty + 1 + j * CTY;
      const float2 e = tab.e[S.code[row][tx + HXC]];
      v[j] = fmaf(beta, S.po[row][tx + HXF], fastZ<PC>(e.y, S.r[row][tx + HXF]));
      dOwn[j] = e.x;
      t[row][tx + 1] = v[j];
    }
    // the halo ring, one warp-wide pass per side: warps 0 and CTY-1 take the
    // rows below and above; warp 3 takes both columns, lane l -> row
    // 1 + (l & 15), left for l < 16, right otherwise
    if (ty == 0) t[0][tx + 1] = pAt(0, tx + HXF, tx + HXC);
    if (ty == CTY - 1) t[CTR + 1][tx + 1] = pAt(CTR + 1, tx + HXF, tx + HXC);
    if (ty == 3) {
      const int row = 1 + (tx & (CTR - 1));
      const bool right = tx >= CTR;
      t[row][right ? CTX + 1 : 0] = pAt(row, right ? HXF + CTX : HXF - 1, right ? HXC + CTX : HXC - 1);
    }
  };
  bool ok = !active || mbarWait(&bar[0], 0, deadline);
  if (ok && active) formTile(0, pt[0], cur, dCur);
  int waited = active ? 1 : 0;
  bool fail = __syncthreads_or(!ok);
  if (active && !fail && tid == 0 && kDirStages < nLoad) issue(kDirStages), issued = kDirStages + 1;
  double acc = 0.0;  // FP64 dot partials: each product rounded to FP64, summed in FP64
  for (int i = 0; i < nPlanes && !fail; ++i) {
    ok = mbarWait(&bar[(i + 1) % kDirStages], (unsigned)(((i + 1) / kDirStages) & 1), deadline);
    waited = i + 2;
    if (ok) formTile(i + 1, pt[(i + 1) & 1], above, dAbove);
    float (*t)[CTX + 2] = pt[i & 1];
#pragma unroll
    for (int j = 0; j < RY; ++j) {
      if (in[j] && ok && dCur[j] >= 0.f) {  // fluid cells only
        const int row = ty + 1 + j * CTY;
        float q = rowSum(dCur[j], sx, sy, sz, cur[j], t[row][tx], t[row][tx + 2], t[row - 1][tx + 1],
                         t[row + 1][tx + 1], below[j], above[j]);
        pNew[c[j]] = cur[j];
        acc = fma((double)cur[j], (double)q, acc);
      }
      below[j] = cur[j];
      cur[j] = above[j];
      dCur[j] = dAbove[j];
      c[j] += plane;
    }
    fail = __syncthreads_or(!ok);
    if (!fail && tid == 0 && i + 1 + kDirStages < nLoad) issue(i + 1 + kDirStages), issued = i + 2 + kDirStages;
  }
  if (fail) {
    if (tid == 0) {
      cgFail(st, 1);
      drainStages<kDirStages>(bar, &issued, waited);
    }
    return;
  }
  double pq = acc, dummy = 0.0;
  if (gridSum2(pq, dummy, partials, &st->ticket) && flatTid() == 0) {
    st->pAp = pq;
    st->alpha = (float)(st->rz / pq);
    st->ticket = 0;
  }
}

// CG update: x += alpha p, r -= alpha A p (A p recomputed from the stored p
// of the stage ring), z = M^-1 r, the reductions r.r and r.z; the last block
// checks convergence and forms beta (CuMatrixFreePCG.cpp:49-63).  The
// |alpha| < FLT_EPSILON skip of CCuDenseVector::plusAlphaX
// (CuDenseVector.cpp:178) is kept.  The dot products accumulate in FP64 from
// the first product: per-thread partials over one z-column segment, then a
// fixed-order FP64 reduction over the grid.
template <int PC, class TX>
__global__ void __launch_bounds__(CTX* CTY, 4)
    kCgUpdate(const __grid_constant__ CUtensorMap mP, const __grid_constant__ CUtensorMap mR,
              const __grid_constant__ CUtensorMap mX, const __grid_constant__ CUtensorMap mCode, Dim3i P, float sx,
              float sy, float sz, const float* __restrict__ p, TX* __restrict__ xv, float* __restrict__ r,
              double* partials, CgState* st, int zPer, const int* __restrict__ colZ) {
  constexpr int kUpdStages = kUpdStagesT<TX>;
  using Stage = UpdStage<TX>;
  __shared__ Stage stg[kUpdStages];
  __shared__ DiagTab tab;
  __shared__ __align__(8) uint64_t bar[kUpdStages];
  __shared__ int issued;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * CTX + tx;
  int x0 = 0, y0 = 0, z0 = 0, z1 = 0;
  auto issue = [&](int i) {
    Stage& S = stg[i % kUpdStages];
    uint64_t* b = &bar[i % kUpdStages];
    mbarExpectTx(b, kUpdStageBytes<TX>);
    tmaLoad3(&S.p[0][0], &mP, x0 - HXF, y0 - 1, z0 + i, b);
    tmaLoad3(&S.r[0][0], &mR, x0, y0, z0 + i, b);
    tmaLoad3(&S.x[0][0], &mX, x0, y0, z0 + i, b);
    tmaLoad3(&S.code[0][0], &mCode, x0, y0, z0 + i, b);
  };
  if (tid == 0) {
    for (int s = 0; s < kUpdStages; ++s) mbarInit(&bar[s], 1);
    mbarFenceInit();
  }
  buildDiagTab(tab, sx, sy, sz);
  __syncthreads();
  waitPrevGrid();
  if (st->done) return;  // the same value in every thread
  allowNextGrid();
  const bool active = cgBlockWork(colZ, P, zPer, x0, y0, z0, z1, st);  // as in kCgDirection
  const int nPlanes = active ? z1 - z0 : 0, nLoad = nPlanes + 1;
  if (tid == 0) {
    int n = active ? min(kUpdStages, nLoad) : 0;
    for (int i = 0; i < n; ++i) issue(i);
    issued = n;
  }
  const float alpha = st->alpha;
  const bool skip = fabsf(alpha) < FLT_EPSILON;
  const unsigned long long deadline = globalNs() + kWaitNs;
  const int x = x0 + tx;
  const unsigned plane = (unsigned)P.x * (unsigned)P.y;
  bool in[RY];
  unsigned c[RY];
  float below[RY], cur[RY];
#pragma unroll
  for (int j = 0; j < RY; ++j) {
    const int y = y0 + ty + j * CTY;
    in[j] = x < P.x && y < P.y;
    c[j] = (unsigned)z0 * plane + (unsigned)y * (unsigned)P.x + (unsigned)x;
    below[j] = (active && in[j] && z0 > 0) ? __ldg(p + c[j] - plane) : 0.f;
  }
  bool ok = !active || mbarWait(&bar[0], 0, deadline);
#pragma unroll
  for (int j = 0; j < RY; ++j) cur[j] = (ok && active) ? stg[0].p[ty + 1 + j * CTY][tx + HXF] : 0.f;
  int waited = active ? 1 : 0;
  bool fail = __syncthreads_or(!ok);
  double arr = 0.0, arz = 0.0;  // FP64 dot partials
  for (int i = 0; i < nPlanes && !fail; ++i) {
    ok = mbarWait(&bar[(i + 1) % kUpdStages], (unsigned)(((i + 1) / kUpdStages) & 1), deadline);
    waited = i + 2;
    const Stage& A = stg[(i + 1) % kUpdStages];
    const Stage& S = stg[i % kUpdStages];
#pragma unroll
    for (int j = 0; j < RY; ++j) {
      const int row = ty + 1 + j * CTY, ir = ty + j * CTY;
      float above = ok ? A.p[row][tx + HXF] : 0.f;
      if (in[j] && ok) {
        CgCode k = S.code[ir][tx];
        const float2 e = tab.e[k];
        float rv = S.r[ir][tx];
        if (!skip && (k & 1)) {  // x, r and z stay zero off the fluid
          float q = rowSum(e.x, sx, sy, sz, cur[j], S.p[row][tx + HXF - 1], S.p[row][tx + HXF + 1],
                           S.p[row - 1][tx + HXF], S.p[row + 1][tx + HXF], below[j], above);
          if (sizeof(TX) == 8)  // FP64 accumulation: x + alpha p, each operation rounded once
            xv[c[j]] = (TX)__dadd_rn((double)S.x[ir][tx], __dmul_rn((double)alpha, (double)cur[j]));
          else
            xv[c[j]] = (TX)fmaf(alpha, cur[j], (float)S.x[ir][tx]);
          rv = fmaf(-alpha, q, rv);
          r[c[j]] = rv;
        }
        float zz = fastZ<PC>(e.y, rv);
        arr = fma((double)rv, (double)rv, arr);
        arz = fma((double)rv, (double)zz, arz);
      }
      below[j] = cur[j];
      cur[j] = above;
      c[j] += plane;
    }
    fail = __syncthreads_or(!ok);
    if (!fail && tid == 0 && i + kUpdStages < nLoad) issue(i + kUpdStages), issued = i + 1 + kUpdStages;
  }
  if (fail) {
    if (tid == 0) {
      cgFail(st, 1);
      drainStages<kUpdStages>(bar, &issued, waited);
    }
    return;
  }
  double rr = arr, rz = arz;
  if (gridSum2(rr, rz, partials, &st->ticket) && flatTid() == 0) {
    st->rr = rr;
    st->iter += 1;
    bool stop = cgStop(st, rr);
    if (PC != 2) {  // with multigrid the V-cycle's last sweep forms r.z and beta
      st->beta = (float)(rz / st->rz);
      st->rz = rz;
    }
    st->done = st->error || stop || st->iter >= st->maxIter;
    st->ticket = 0;
  }
}

// Tensor map of a pitched 3-D array (x fastest) with the given box.
cudaError_t encodeMap(CUtensorMap* m, const void* base, CUtensorMapDataType type, unsigned esize, const Dim3i& cg,
                      unsigned bx, unsigned by) {
  using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static Encode encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess) return e;
    if (q != cudaDriverEntryPointSuccess || !fn) return cudaErrorNotSupported;
    encode = (Encode)fn;
  }
  cuuint64_t dims[3] = {(cuuint64_t)cg.x, (cuuint64_t)cg.y, (cuuint64_t)cg.z};
  cuuint64_t strides[2] = {(cuuint64_t)cg.x * esize, (cuuint64_t)cg.x * cg.y * esize};
  cuuint32_t box[3] = {bx, by, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = encode(m, type, 3, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}
}  // namespace

cudaError_t makeHaloMap(const Dim3i& cg, const float* v, CUtensorMap* m) {
  return encodeMap(m, v, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, cg, FW, FH);
}

cudaError_t makeCgMaps(const Dim3i& cg, const CgCode* code, const float* r, const void* x, bool xDouble,
                       const float* p0, const float* p1, CgMaps* m) {
  if (cg.x % 16 != 0) return cudaErrorInvalidValue;  // rows of 8-bit codes must start on 16-byte boundaries
  cudaError_t e;
  if ((e = encodeMap(&m->codeH, code, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, cg, CW, FH)) != cudaSuccess) return e;
  if ((e = encodeMap(&m->codeI, code, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, cg, CTX, CTR)) != cudaSuccess) return e;
  if ((e = encodeMap(&m->rH, r, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, cg, FW, FH)) != cudaSuccess) return e;
  if ((e = encodeMap(&m->rI, r, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, cg, CTX, CTR)) != cudaSuccess) return e;
  if ((e = encodeMap(&m->xI, x, xDouble ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                     xDouble ? 8 : 4, cg, CTX, CTR)) != cudaSuccess)
    return e;
  if ((e = encodeMap(&m->pH[0], p0, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, cg, FW, FH)) != cudaSuccess) return e;
  return encodeMap(&m->pH[1], p1, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, cg, FW, FH);
}

void cgWarmLaunchCache() {
  residentBlocks((const void*)kCgDirection<0>);
  residentBlocks((const void*)kCgDirection<1>);
  residentBlocks((const void*)kCgDirection<2>);
  residentBlocks((const void*)kCgUpdate<0, float>);
  residentBlocks((const void*)kCgUpdate<1, float>);
  residentBlocks((const void*)kCgUpdate<2, float>);
  residentBlocks((const void*)kCgUpdate<0, double>);
  residentBlocks((const void*)kCgUpdate<1, double>);
  residentBlocks((const void*)kCgUpdate<2, double>);
}

int cgScheduleTarget(int precond, bool xDouble) {
  int per = kSchedPerSM;
  auto take = [&](const void* k) { per = std::min(per, residentBlocks(k)); };
  if (precond == 1) {
    take((const void*)kCgDirection<1>);
    take(xDouble ? (const void*)kCgUpdate<1, double> : (const void*)kCgUpdate<1, float>);
  } else if (precond == 2) {
    take((const void*)kCgDirection<2>);
    take(xDouble ? (const void*)kCgUpdate<2, double> : (const void*)kCgUpdate<2, float>);
  } else {
    take((const void*)kCgDirection<0>);
    take(xDouble ? (const void*)kCgUpdate<0, double> : (const void*)kCgUpdate<0, float>);
  }
  return numSMs() * std::max(1, per);
}

int cgScheduleInts(const Dim3i& cg) {
  const int cols = cgColumns(cg);
  return schedItemsOffset(cols) + 4 * (numSMs() * kSchedPerSM + cols);
}

int cgPartialsNeeded(const Dim3i& r) {
  const Dim3i cg = cgDims(r);
  CgGrid g = cgGrid(cg);
  long long n = (long long)g.grid.x * g.grid.y * g.grid.z;
  // the CG kernels, at the shortest z chunk any launch shape (tuned or not) uses
  const long long tiles = (long long)((cg.x + CTX - 1) / CTX) * ((cg.y + CTR - 1) / CTR);
  n = std::max(n, tiles * ((cg.z + std::min(3, cg.z) - 1) / std::min(3, cg.z)));
  n = std::max(n, (long long)numSMs() * kSchedPerSM + tiles);  // a schedule's grid
  return 2 * (int)n;
}

cudaError_t launchCgDirection(const Dim3i& cg, float sx, float sy, float sz, const CUtensorMap& mZ,
                              const CUtensorMap& mPo, const CUtensorMap& mCode, const CgCode* code, const float* zr,
                              const float* pOld, float* pNew, double* partials, CgState* st, int precond,
                              cudaStream_t s, const int* colZ, bool xDouble) {
  switch (precond) {
    case 1: {
      CgLaunch L = cgLaunch(cg, kCgDirection<1>, 0, colZ, 1, xDouble);
      cudaError_t e = launchPdl(kCgDirection<1>, L.grid, L.block, s, mZ, mPo, mCode, cg, sx, sy, sz, code, zr, pOld,
                                pNew, partials, st, L.zPer, colZ);
      if (e != cudaSuccess) return e;
      break;
    }
    case 2: {
      CgLaunch L = cgLaunch(cg, kCgDirection<2>, 0, colZ, 2, xDouble);
      cudaError_t e = launchPdl(kCgDirection<2>, L.grid, L.block, s, mZ, mPo, mCode, cg, sx, sy, sz, code, zr, pOld,
                                pNew, partials, st, L.zPer, colZ);
      if (e != cudaSuccess) return e;
      break;
    }
    default: {
      CgLaunch L = cgLaunch(cg, kCgDirection<0>, 0, colZ, 0, xDouble);
      cudaError_t e = launchPdl(kCgDirection<0>, L.grid, L.block, s, mZ, mPo, mCode, cg, sx, sy, sz, code, zr, pOld,
                                pNew, partials, st, L.zPer, colZ);
      if (e != cudaSuccess) return e;
    }
  }
  return cudaGetLastError();
}

cudaError_t launchCgUpdate(const Dim3i& cg, float sx, float sy, float sz, const CUtensorMap& mP, const CUtensorMap& mR,
                           const CUtensorMap& mX, const CUtensorMap& mCode, const float* p, void* x, bool xDouble,
                           float* r, double* partials, CgState* st, int precond, cudaStream_t s, const int* colZ) {
#define HFG_CG_UPDATE(PCV, TXV)                                                                                   \
  {                                                                                                               \
    CgLaunch L = cgLaunch(cg, kCgUpdate<PCV, TXV>, 1, colZ, PCV, xDouble);                                                             \
    cudaError_t e = launchPdl(kCgUpdate<PCV, TXV>, L.grid, L.block, s, mP, mR, mX, mCode, cg, sx, sy, sz, p,      \
                              (TXV*)x, r, partials, st, L.zPer, colZ);                                        \
    if (e != cudaSuccess) return e;                                                                             \
  }
  if (xDouble) {
    if (precond == 1) HFG_CG_UPDATE(1, double)
    else if (precond == 2) HFG_CG_UPDATE(2, double)
    else HFG_CG_UPDATE(0, double)
  } else {
    if (precond == 1) HFG_CG_UPDATE(1, float)
    else if (precond == 2) HFG_CG_UPDATE(2, float)
    else HFG_CG_UPDATE(0, float)
  }
#undef HFG_CG_UPDATE
  return cudaGetLastError();
}

// Fluid extent of every CG tile column: one block per (column, z slice)
// reduces the fluid planes of its slice; the column's range is their
// min / max (atomics into colZ, set up by the launcher).
__global__ void kFluidColumns(Dim3i cg, const CgCode* __restrict__ code, int zPer, int* colZ) {
  const int x = blockIdx.x * CTX + threadIdx.x, y = blockIdx.y * CTR + threadIdx.y;
  const int z0 = blockIdx.z * zPer, z1 = min(z0 + zPer, cg.z);
  int lo = 0x7fffffff, hi = -1;
  if (x < cg.x && y < cg.y)
    for (int z = z0; z < z1; ++z)
      if (code[((long long)z * cg.y + y) * cg.x + x] & 1) {
        lo = min(lo, z);
        hi = z;
      }
  __shared__ int sl[CTR], sh[CTR];
  lo = __reduce_min_sync(0xffffffffu, lo);
  hi = __reduce_max_sync(0xffffffffu, hi);
  if (threadIdx.x == 0) { sl[threadIdx.y] = lo; sh[threadIdx.y] = hi; }
  __syncthreads();
  if (threadIdx.y == 0 && threadIdx.x < CTR) {
    lo = __reduce_min_sync(0x0000ffffu, sl[threadIdx.x]);
    hi = __reduce_max_sync(0x0000ffffu, sh[threadIdx.x]);
    if (threadIdx.x == 0 && hi >= 0) {
      const unsigned cols = gridDim.x * gridDim.y, t = blockIdx.y * gridDim.x + blockIdx.x;
      atomicMin(colZ + t, lo);
      atomicMax(colZ + cols + t, hi);
    }
  }
}
int cgColumns(const Dim3i& cg) { return ((cg.x + CTX - 1) / CTX) * ((cg.y + CTR - 1) / CTR); }

// The work items of a schedule from the columns' fluid extents: chunks of
// zLen = max(zMin, ceil(S / target)) planes, S the fluid planes of all active
// columns, so the items are at most target + (active columns); they are
// written column by column, bottom to top.  One block.
constexpr int kListThreads = 1024;
__global__ void __launch_bounds__(kListThreads) kCgWorkList(int cols, int target, int zMin, int capacity, int* sched) {
  const int* lo = sched;
  const int* hi = sched + cols;
  int4* items = reinterpret_cast<int4*>(sched + schedItemsOffset(cols));
  __shared__ unsigned long long total;
  __shared__ int warpTot[kListThreads / 32];
  __shared__ int carry;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  if (t == 0) {
    total = 0;
    carry = 0;
  }
  __syncthreads();
  unsigned long long mine = 0;
  for (int c = t; c < cols; c += kListThreads)
    if (hi[c] >= lo[c]) mine += (unsigned long long)(hi[c] - lo[c] + 1);
  atomicAdd(&total, mine);
  __syncthreads();
  const long long S = (long long)total;
  const int zLen = (int)max((long long)zMin, (S + target - 1) / max(target, 1));
  for (int c0 = 0; c0 < cols; c0 += kListThreads) {
    const int c = c0 + t;
    int n = 0, l = 0;
    if (c < cols && hi[c] >= lo[c]) {
      l = lo[c];
      n = (hi[c] - l + zLen) / zLen;
    }
    int inc = n;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, inc, d);
      if (lane >= d) inc += y;
    }
    if (lane == 31) warpTot[w] = inc;
    __syncthreads();
    if (w == 0) {
      int x = warpTot[lane], xi = x;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, xi, d);
        if (lane >= d) xi += y;
      }
      warpTot[lane] = xi - x;
    }
    __syncthreads();
    int k = carry + warpTot[w] + inc - n;
    for (int i = 0; i < n; ++i, ++k) {
      const int z0 = l + i * zLen;
      if (k < capacity) items[k] = make_int4(c, z0, min(z0 + zLen, hi[c] + 1), 0);
    }
    __syncthreads();
    if (t == kListThreads - 1) carry = k;
    __syncthreads();
  }
  // more items than the buffer holds cannot happen (at most target + cols);
  // if it did, a count past the grid makes the CG kernels report error 4
  if (t == 0) sched[2 * cols] = carry;
}

cudaError_t launchCgSchedule(const Dim3i& cg, const CgCode* code, int* sched, int precond, bool xDouble,
                             cudaStream_t s) {
  const int cols = cgColumns(cg);
  cudaError_t e = cudaMemsetAsync(sched, 0x7f, sizeof(int) * cols, s);  // lo: 0x7f7f7f7f, above any plane
  if (e == cudaSuccess) e = cudaMemsetAsync(sched + cols, 0xff, sizeof(int) * cols, s);  // hi: -1
  if (e != cudaSuccess) return e;
  const int zPer = 16;
  dim3 grid((cg.x + CTX - 1) / CTX, (cg.y + CTR - 1) / CTR, (cg.z + zPer - 1) / zPer);
  kFluidColumns<<<grid, dim3(CTX, CTR), 0, s>>>(cg, code, zPer, sched);
  // the shortest chunk: the tuned z-chunk length of the direction kernel, else 3 planes
  const int tuned = tunedZPer(0, cg);
  const int zMin = tuned > 0 ? tuned : std::min(3, cg.z);
  kCgWorkList<<<1, kListThreads, 0, s>>>(cols, cgScheduleTarget(precond, xDouble), zMin,
                                         (cgScheduleInts(cg) - schedItemsOffset(cols)) / 4, sched);
  return cudaGetLastError();
}

}  // namespace hfg
