// hfg_kernels.h -- host-side launchers for the sm_100a kernels of the grid
// step.  Every launcher is asynchronous on the given stream and returns
// cudaGetLastError() of its launch.
#pragma once
#include <cstdint>
#include <vector>
#include <cuda.h>
#include <cuda_runtime.h>

#include "hfg_device.cuh"

namespace hfg {

constexpr int kMaxBoundaries = 32;

// Solid boundaries as the kernels see them: one cell-centred SDF per solid
// plus its current translation (MPhysics/Boundary.cpp:124-136).
struct BoundarySet {
  int n;
  const float* sdf[kMaxBoundaries];
  float tx[kMaxBoundaries], ty[kMaxBoundaries], tz[kMaxBoundaries];
  float vx[kMaxBoundaries], vy[kMaxBoundaries], vz[kMaxBoundaries];
};

// Device-resident scalars of one CG solve.  The last block of every reduction
// kernel updates them, so no host round trip is needed per iteration.
struct CgState {
  double rz;        // r.z of the current iteration
  double rr;        // ||r||^2 after the last update
  double bb;        // ||b||^2
  double pAp;
  float alpha, beta;
  int iter;         // iterations completed
  int done;         // 1 once converged or out of iterations
  int maxIter;
  int precond;      // 0 identity, 1 Jacobi
  int tolMode;      // 0 reference rule sqrt(||r||) < tol, 1 ||r||/||b|| < tol
  double tol;
  int error;        // nonzero: a kernel gave up (a stage load timed out); done is set too
  unsigned int ticket;  // last-block-done counter
};

// State of the CFL substep loop of one particle advection
// (MPhysics/EulerParticles.cpp:241-319).  Slot s is read by substep s and
// slot s+1 written by it.
struct SubstepState {
  unsigned int maxAbsBits;  // max |v| over all sampled components (float bits)
  float subTime;            // time advanced so far
  int finished;
  int count;
};

// One scene's CFL substep loop as a launch sees it (GridSolver::substepTask);
// the batch stepper runs the substeps of many scenes in one launch per slot.
struct SubstepTask {
  Geom g;
  FaceQuads vel;
  float* pos;
  float* v0;
  long long P;
  long long nclamp;
  SubstepState* st;
  int acc;
  float dt, cfl;
};

struct SolidVelTable {
  const uint8_t* solidIdx;  // 0 = not solid, i+1 = solid of boundary i
  float vx[kMaxBoundaries], vy[kMaxBoundaries], vz[kMaxBoundaries];
};

int numSMs();

// Solid face velocity of a face between cells lo (index i-1) and hi (index i)
// on `axis`: the six faces of a solid cell carry its solid's velocity
// (BoundaryTool.cu:28-83).  Where two different solids meet the reference
// races; the higher cell wins here.
__device__ inline float solidFaceVel(const SolidVelTable& t, uint8_t lo, uint8_t hi, int axis) {
  uint8_t s = hi ? hi : lo;
  if (!s) return 0.f;
  return axis == 0 ? t.vx[s - 1] : (axis == 1 ? t.vy[s - 1] : t.vz[s - 1]);
}


// ---- boundaries / classification -------------------------------------------
cudaError_t launchSolidClassify(const Geom& g, const BoundarySet& b, uint8_t* solidIdx, float* const* curSDF,
                                cudaStream_t s);
cudaError_t launchSolidFromSDF(long long n, const float* solidSDF, uint8_t* solidIdx, cudaStream_t s);
// Signed distance (negative inside the solid) of an analytic solid at every
// cell centre, evaluated in FP64 and stored as FP32.  type 0: the walls, i.e.
// everything outside the inner box [o + h, o + (n - 1) h]; 1: sphere
// (cx, cy, cz, r); 2: axis-aligned box (cx, cy, cz, sx, sy, sz full sides).
cudaError_t launchAnalyticSdf(const Geom& g, int type, const double* params, float* sdf, cudaStream_t s);
cudaError_t launchTotalSolidSDF(long long n, int nb, const uint8_t* solidIdx, float* out, cudaStream_t s);
cudaError_t launchSolidVelField(const Geom& g, const SolidVelTable& t, FaceField out, cudaStream_t s);
cudaError_t launchMarkersInit(long long n, const uint8_t* solidIdx, uint8_t* markers, cudaStream_t s);
cudaError_t launchMarkersFromParticles(const Geom& g, const float* pos, long long P, uint8_t* markers, cudaStream_t s);
cudaError_t launchBinCounts(const Geom& g, const float* pos, long long P, unsigned int* counts, cudaStream_t s);
cudaError_t launchMarkersFromSDF(long long n, const uint8_t* solidIdx, const float* fluidSDF, uint8_t* markers,
                                 cudaStream_t s);
cudaError_t launchFluidDomainFromBBox(const Geom& g, const float mn[3], const float mx[3], float* out, cudaStream_t s);

// ---- pressure projection ---------------------------------------------------
// Per-cell stencil code: bit 0 the cell is fluid; bits 1..6 its left, right,
// down, up, back, front neighbour is inside the grid and not solid (the
// diagonal of buildPressureMatrixA, EulerSolverTool.cu:85-120); bits 7..12
// that neighbour is inside the grid and fluid (the off-diagonals).
typedef uint16_t Code;
// Bits 0..6 of the code (fluid, the six "not solid" neighbours): all the CG
// kernels read.  The neighbour-is-fluid bits are not needed there because
// every CG vector is zero off the fluid.
typedef uint8_t CgCode;
// The pressure system lives on a pitched copy of the grid: rows of
// px = cgPitch(nx) >= nx cells, px a multiple of 16 so that every row of FP32
// values and of 8-bit CG codes starts on a 16-byte boundary (TMA tiles).  The
// cells x >= nx are inert: code 0 and every CG vector 0 there.  Index of cell
// (x, y, z): (z * ny + y) * px + x.
__host__ __device__ inline int cgPitch(int nx) { return (nx + 15) & ~15; }
__host__ __device__ inline Dim3i cgDims(const Dim3i& r) { return Dim3i{cgPitch(r.x), r.y, r.z}; }
// Codes of grid `r` written with row pitch px (px = r.x: unpitched).
// With `cgc`, the CG codes too (same pitch).
cudaError_t launchStencilCode(const Dim3i& r, int px, const uint8_t* markers, Code* code, cudaStream_t s,
                              CgCode* cgc = nullptr);
cudaError_t launchMatrixA(const Dim3i& r, float sx, float sy, float sz, const Code* code, float* A, cudaStream_t s);
cudaError_t launchApplyA(const Dim3i& r, float sx, float sy, float sz, const Code* code, const float* x, float* y,
                         cudaStream_t s);
// RHS (divergence + solid terms) fused with CG set-up: r = b, x = 0, p = 0,
// ||b||^2 and r.z into the state.  Solid face velocities come from `svArr`
// when non-null, else from the per-solid table.  `b` (optional) is unpitched;
// code, r, x and p are pitched.
cudaError_t launchRhsInit(const Geom& g, ConstFaceField v, ConstFaceField svArr, const SolidVelTable& svTab,
                          const uint8_t* markers, const Code* code, float ax, float ay, float az, float* b,
                          float* r, void* x, bool xDouble, float* p, double* partials, CgState* st, int precond,
                          cudaStream_t s);
// TMA descriptors of the CG vectors on the pitched grid cg = cgDims(r):
// halo boxes (H) for the arrays read with neighbours, plain tiles (I) else.
struct CgMaps {
  CUtensorMap codeH, codeI, rH, rI, xI, pH[2];
};
// x: the pressure iterate, FP32 or (xDouble) FP64
cudaError_t makeCgMaps(const Dim3i& cg, const CgCode* code, const float* r, const void* x, bool xDouble,
                       const float* p0, const float* p1, CgMaps* m);
cudaError_t makeHaloMap(const Dim3i& cg, const float* v, CUtensorMap* m);
// precond: 0 identity, 1 Jacobi, 2 z read through mZ (must match CgState::precond);
// mZ is the halo map of r (precond 0, 1) or of z (2); zr the same array.
// colZ (optional, from launchCgSchedule): the solve's schedule; the grid is
// then one block per work item (a tile column's run of fluid planes), sized
// for one wave.  Null: the dense grid over every tile and z chunk.
cudaError_t launchCgDirection(const Dim3i& cg, float sx, float sy, float sz, const CUtensorMap& mZ,
                              const CUtensorMap& mPo, const CUtensorMap& mCode, const CgCode* code, const float* zr,
                              const float* pOld, float* pNew, double* partials, CgState* st, int precond,
                              cudaStream_t s, const int* colZ = nullptr, bool xDouble = false);
cudaError_t launchCgUpdate(const Dim3i& cg, float sx, float sy, float sz, const CUtensorMap& mP, const CUtensorMap& mR,
                           const CUtensorMap& mX, const CUtensorMap& mCode, const float* p, void* x, bool xDouble,
                           float* r, double* partials, CgState* st, int precond, cudaStream_t s,
                           const int* colZ = nullptr);
// Measured launch shapes of the CG kernels (family 0 direction, 1 update):
// the z-chunk length used for the pitched grid cg, <= 0 erases.  The table is
// process wide; saveTuning/loadTuning keep it in a text file.
void setTunedCgZPer(int family, const Dim3i& cg, int zPer);
int tunedCgZPer(int family, const Dim3i& cg);  // -1: none
std::vector<int> cgZPerCandidates(const Dim3i& cg);
bool saveTuning(const char* path);
int loadTuning(const char* path);  // entries read, -1 if the file cannot be opened
// The schedule of the CG kernels for a solve, from the CG codes: the fluid
// extent of every tile column (32 x 16 cells of the pitched grid cg, all z)
// and the work items cut from it for one wave of blocks of the kernels of
// `precond`.  sched holds cgScheduleInts(cg) ints.
int cgColumns(const Dim3i& cg);
int cgScheduleInts(const Dim3i& cg);
// work items of one wave of the CG kernels of this preconditioner and
// iterate type (the schedule's grid: this + cgColumns)
int cgScheduleTarget(int precond, bool xDouble);
// Layout of a schedule: ints [0, cols) and [cols, 2 cols) the lowest and
// highest fluid plane of each tile column (kCgTileX x kCgTileY cells), [2 cols]
// the item count, from schedItemsOffset(cols) the items (column, z0, z1, 0).
constexpr int kCgTileX = 32, kCgTileY = 16;
__host__ __device__ inline int schedItemsOffset(int cols) { return (2 * cols + 1 + 3) & ~3; }
cudaError_t launchCgSchedule(const Dim3i& cg, const CgCode* code, int* sched, int precond, bool xDouble,
                             cudaStream_t s);
// Divergence residual of the projected velocity over the fluid cells:
// *sumOut = sum b^2 (FP64), ticketAndMax[1] = bits of max |b|.  `scratch`
// holds 2 * divergenceBlocks() doubles.
inline int divergenceBlocks() { return 1024; }
cudaError_t launchDivergenceNorm(const Geom& g, ConstFaceField v, const SolidVelTable& svTab,
                                 const uint8_t* markers, double* scratch, unsigned* ticketAndMax, double* sumOut,
                                 cudaStream_t s);
// FP64 residual of a solve: out[0] = ||b - A x||^2, out[1] = ||b||^2 over the
// fluid cells, b from the unprojected velocity v, A from the 16-bit codes
// (pitched) and the FP32 scales, x pitched (FP32 or FP64).  `scratch` holds
// 2 * divergenceBlocks() doubles.
cudaError_t launchTrueResidual(const Geom& g, ConstFaceField v, const SolidVelTable& svTab, const uint8_t* markers,
                               const Code* code, const void* x, bool xDouble, float sx, float sy, float sz,
                               double* scratch, unsigned* ticket, double* out, cudaStream_t s);
// p pitched, FP32 or (pDouble) FP64; the differences are rounded to FP32
cudaError_t launchGradient(const Geom& g, float gx, float gy, float gz, const uint8_t* markers, const void* p,
                           bool pDouble, FaceField v, ConstFaceField svArr, const SolidVelTable& svTab,
                           cudaStream_t s);
// Resolves the launch shapes of every CG kernel variant (occupancy queries) so
// that no query runs while a stream is being captured.
void cgWarmLaunchCache();
// doubles of reduction scratch the CG kernels need on grid `r`
int cgPartialsNeeded(const Dim3i& r);

// dst[0 .. words) = src[...] by one warp (dst may be mapped host memory)
cudaError_t launchCopyWords(const unsigned* src, unsigned* dst, int words, cudaStream_t s);

// ---- extrapolation ---------------------------------------------------------
struct ExtrapScratch {
  uint16_t* dist;          // total faces
  unsigned int* list;      // total faces
  unsigned int* hist;      // kExtrapHistWords: the layer histogram, then the grid-barrier words
  unsigned int* offsets;   // kMaxLayers + 2
  unsigned int* cursor;    // kMaxLayers + 2
  uint8_t* mask;           // total faces: per list entry, the neighbours (bit q in the order left, right,
                           // down, up, back, front) that lie in an earlier layer
};
constexpr int kMaxLayers = 1000;
// hist[0 .. kMaxLayers + 1] is the histogram; hist[kMaxLayers + 2 ..] the
// barrier count, generation and error word of the layer kernel
constexpr int kExtrapHistWords = kMaxLayers + 2 + 4;
cudaError_t launchExtrapDistance(const Dim3i rc[3], float* const vals[3], long long off[3], int nums,
                                 ExtrapScratch sc, cudaStream_t s);
// a layer of at most this many faces is filled by one block (runs of such
// layers without grid barriers between them)
constexpr unsigned kExtrapSmallLayer = 4096;
// Every layer 1 .. nums-1 in one cooperative launch, with a grid barrier
// between layers.  The barrier waits are bounded.  Afterwards the four words
// at extrapBarWords() hold: count, generation, error (nonzero: a barrier timed
// out and the layers are incomplete), deepest layer filled.
cudaError_t launchExtrapLayers(const Dim3i rc[3], float* const vals[3], const long long off[3], ExtrapScratch sc,
                               int nums, cudaStream_t s, long long* launches);
inline unsigned int* extrapBarWords(const ExtrapScratch& sc) { return sc.hist + kMaxLayers + 2; }
// Registers (+1) or drops (-1) a user of launchExtrapLayers (a solver, an
// operator call); the launch sizes its grid to a share of the GPU per user.
void extrapUsers(int delta);

// ---- fluid SDF (buildFluidSDF); frontier buffers hold N cells each; counts 2;
// hostCount pinned.  Blocks (one host read per layer).
// The hybrid coupler's inside / outside distance fields of a fluid density
// (frontier lists of r.size() entries each, two counters, one pinned host
// word; the stream is synchronised once per sweep) and its mixed outside field.
cudaError_t launchFluidSideSdf(const Dim3i& r, const float* density, const float* solid, bool outside, int distance,
                               float* out, unsigned int* frontA, unsigned int* frontB, unsigned int* counts,
                               unsigned int* hostCount, cudaStream_t s);
cudaError_t launchMixedOutsideSdf(const Dim3i& r, const float* gridDensity, const float* mixedDensity,
                                  const float* gridOutside, float* out, cudaStream_t s);
cudaError_t launchFluidSdf(const Dim3i& r, const float* dom, float* sdf, int layers, unsigned int* frontA,
                           unsigned int* frontB, unsigned int* counts, unsigned int* hostCount, cudaStream_t s);
// mixFieldWithDensity of a cell grid (face = 0, a[0], b[0]) or of the three
// face grids of r (face = 1); b is updated in place
cudaError_t launchMixFieldWithDensity(const Dim3i& r, int face, const float* const a[3], float* const b[3],
                                      const float* wa, const float* wb, cudaStream_t s);
cudaError_t launchMixParticleVel(const float* pic, const float* flip, const float* dist, long long n, float cell,
                                 float g, float gf, float f, float p, float* predict, cudaStream_t s);
// fluid density of buildFluidDensity; the solid is solidSdf < 0 when given,
// else solidIdx != 0
cudaError_t launchFluidDensity(const Dim3i& r, const float* dom, const float* solidSdf, const uint8_t* solidIdx,
                               float* out, cudaStream_t s);

// ---- particles -------------------------------------------------------------
enum ParticleMode : int { MODE_PIC = 0, MODE_FLIP = 1, MODE_MIX = 2 };
cudaError_t launchSeedCount(const Dim3i& r, const float* fluidSDF, const uint8_t* solidIdx, unsigned int* blockCounts,
                            int cellsPerBlock, cudaStream_t s);
cudaError_t launchSeedScan(unsigned int* blockCounts, int nBlocks, unsigned long long* total, cudaStream_t s);
cudaError_t launchSeedWrite(const Geom& g, const float* fluidSDF, const uint8_t* solidIdx,
                            const unsigned int* blockOffsets, int cellsPerBlock, int ppc, unsigned long long seed,
                            float* pos, cudaStream_t s);
// LINEAR (alg 2) also writes v0 = the PIC sample of vinQ (the corner tables of
// vin) and max |v0| into st[0], the start of the substep loop, which then
// needs no launchSubstepBegin; the other transfer kernels leave both alone.
cudaError_t launchParticleVelUpdate(const Geom& g, int mode, int alg, ConstFaceField vin, ConstFaceField prev,
                                    int firstFlip, float mixing, const float* pos, float* vel, long long P,
                                    cudaStream_t s, const FaceQuads* vinQ, float* v0, SubstepState* st);
// Corner tables of the face grids for the substep kernels; component a has
// faceQuadCount(r, a) entries.
long long faceQuadCount(const Dim3i& r, int a);
cudaError_t launchFaceQuads(const Dim3i& r, ConstFaceField v, float4* const out[3], cudaStream_t s);

// hfg_sort.cu: the stable permutation that orders P particles by cell
// (perm[j] = index of the j-th particle in cell order, ties in index order).
// Scratch: keyA, keyB, valA, valB of P entries, counts of
// sortCountEntries(P), sums of sortScanBlocks(sortCountEntries(P)); *perm
// is set to valA or valB.
struct SortScratch {
  unsigned int *keyA, *keyB, *valA, *valB, *counts, *sums;
};
long long sortCountEntries(long long P);
long long sortScanBlocks(long long entries);
int sortPassesLaunches(long long nCells, bool grouped);  // kernels one sort launches
// split in (0, P): particles [0, split) and [split, P) are sorted each within
// its own index range (stable); otherwise all together.
cudaError_t launchSortPermutation(const Geom& g, const float* pos, long long P, long long split, const SortScratch& sc,
                                  const unsigned int** perm, cudaStream_t s);
// out[width*j + k] = in[width*perm[j] + k], width 1 or 3
cudaError_t launchGather(const float* in, int width, const unsigned int* perm, long long P, float* out,
                         cudaStream_t s);
cudaError_t launchSubstepBegin(const Geom& g, FaceQuads vel, const float* pos, float* v0, long long P,
                               SubstepState* st, cudaStream_t s);
cudaError_t launchSubstep(const Geom& g, FaceQuads vel, float* pos, float* v0, long long P, int acc, float dt,
                          float cfl, long long nclamp, SubstepState* st, int slot, cudaStream_t s);
// Batched substeps: slot `slot` of every scene of `tasks` (device array) in one
// launch; chunkStart[s] = sum of multiSubstepChunks(P) over scenes < s (device
// array), totalChunks the sum over all scenes.
long long multiSubstepChunks(long long P);
cudaError_t launchSubstepMulti(const SubstepTask* tasks, const long long* chunkStart, int nScenes,
                               long long totalChunks, int slot, cudaStream_t s);
// out[2 s] = finished, out[2 s + 1] = count of scene s's state slot `slot`
cudaError_t launchGatherSubstepStates(const SubstepTask* tasks, int nScenes, int slot, int* out, cudaStream_t s);
cudaError_t launchP2GFace(const Geom& g, int alg, const float* pos, const float* vel, long long P, float2* acc[3],
                          cudaStream_t s);
cudaError_t launchP2GCell(const Geom& g, int alg, const float* pos, const float* val, int span, int comp, long long P,
                          float2* acc, cudaStream_t s);
cudaError_t launchNormalize(long long n, const float2* acc, float* out, float* copy, float add, int doAdd,
                            float add2, int doAdd2, cudaStream_t s);
cudaError_t launchG2PFace(const Geom& g, int alg, ConstFaceField f, const float* pos, long long P, float* out,
                          cudaStream_t s);
cudaError_t launchG2PCell(const Geom& g, int alg, const float* f, const float* pos, long long P, float* out, int span,
                          int comp, cudaStream_t s);
cudaError_t launchSampleFace(const Geom& g, ConstFaceField f, const float* pos, long long M, float* out,
                             cudaStream_t s);
cudaError_t launchSampleCell(const Geom& g, const float* f, const float* pos, long long M, float* out, cudaStream_t s);

// ---- semi-Lagrangian -------------------------------------------------------
// sampling: ESamplingAlgorithm of every sample (0 trilinear .. 4 clamped Bridson)
cudaError_t launchSLFace(const Geom& g, int acc, float dt, ConstFaceField vel, ConstFaceField in, FaceField out,
                         const float add[3], int doAdd, const float add2[3], int doAdd2, cudaStream_t s,
                         int sampling = 0);
cudaError_t launchSLCell(const Geom& g, int acc, float dt, ConstFaceField vel, const float* const* in, float* const* out,
                         int nfields, cudaStream_t s, int sampling = 0);
// n points (3n floats) sampled from one cell-centred grid (face = 0, f.c[0];
// out n floats) or from the three face grids of `g` (face = 1; out 3n floats)
cudaError_t launchSampleAlg(const Geom& g, int face, ConstFaceField f, const float* pos, long long n, int sampling,
                            float* out, cudaStream_t s);

// ---- external forces (unit-field axpy on every face) ------------------------
cudaError_t launchAddConst(long long n, float* v, float a, cudaStream_t s);

// Runs the bounded-wait helpers against conditions nothing satisfies: out[0]
// = 1 once an mbarrier wait of waitNs ran out, out[1] = 1 once a grid barrier
// missing one arrival gave up (its own 1 s limit).  words: 3 scratch words.
cudaError_t launchSelftestWaits(unsigned long long waitNs, unsigned* words, int* out, cudaStream_t s);

}  // namespace hfg
