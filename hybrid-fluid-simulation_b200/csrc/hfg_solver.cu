// hfg_solver.cu -- GridSolver: the reference grid step
// (MPhysics/GridFluidSolver.cpp:336-537) orchestrated as device-resident
// kernels on one stream.  Host round trips per step: one 4-byte read per
// chunk of CFL substeps, one per chunk of CG iterations, and one 4 KB read of
// the extrapolation layer offsets.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <mutex>

#include "hfg_solver.h"

namespace hfg {

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e), HFG_ERR_CUDA);
}

namespace {
constexpr size_t kPinnedBlock = 8192;
std::mutex g_pinnedMu;
std::vector<void*> g_pinnedFree;
}  // namespace

void* pinnedGet(size_t bytes) {
  if (bytes > kPinnedBlock) throw CudaError("pinned block too large", HFG_ERR_INVALID);
  {
    std::lock_guard<std::mutex> lk(g_pinnedMu);
    if (!g_pinnedFree.empty()) {
      void* p = g_pinnedFree.back();
      g_pinnedFree.pop_back();
      return p;
    }
  }
  void* p = nullptr;
  // mapped: kernels write the read-backs straight into these blocks
  check(cudaHostAlloc(&p, kPinnedBlock, cudaHostAllocMapped | cudaHostAllocPortable), "cudaHostAlloc");
  return p;
}

void pinnedPut(void* p) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(g_pinnedMu);
  g_pinnedFree.push_back(p);
}

// A small device-to-host read that does not use a copy engine: a one-warp
// kernel stores the words into the mapped pinned block over the bus.  A large
// copy on another stream (the particle mirror) occupies the copy engine for
// milliseconds, and a small cudaMemcpyAsync queued behind it would wait that
// long.  The caller synchronises the stream before reading `host`.
void readBack(void* host, const void* dev, size_t bytes, cudaStream_t s) {
  void* d = nullptr;
  check(cudaHostGetDevicePointer(&d, host, 0), "cudaHostGetDevicePointer");
  check(launchCopyWords((const unsigned*)dev, (unsigned*)d, (int)((bytes + 3) / 4), s), "read back");
}

namespace {
constexpr int kCgChunk = 16;       // CG iterations launched between convergence reads
constexpr int kSubstepChunk = 4;   // CFL substeps launched between completion reads
}  // namespace

// Multigrid preconditioner hooks (hfg_mg.cu).
Multigrid* mgCreate(const Dim3i& cg, int levels, int smooth, int halfMode, cudaStream_t s);
void mgDestroy(Multigrid* m);
void mgSetup(Multigrid* m, const Dim3i& r, const uint8_t* mk0, const Code* code, float sx, float sy, float sz,
             cudaStream_t s, long long& launches);
void mgRunCg(Multigrid* m, const Dim3i& cg, float sx, float sy, float sz, const CgMaps& maps, const CgCode* code, void* x,
             bool xDouble, float* rvec, CgState* st, CgState* stHost, cudaStream_t s, long long& launches,
             const std::function<cudaGraphExec_t(const std::function<void()>&)>& capture, cudaGraphExec_t* chunk,
             const int* colZ);

GridSolver::GridSolver(float dt, Dim3i res, const float origin[3], const float spacing[3]) {
  if (res.x <= 0 || res.y <= 0 || res.z <= 0) throw CudaError("resolution must be positive", HFG_ERR_INVALID);
  if (res.size() >= (1LL << 31)) throw CudaError("grid too large", HFG_ERR_INVALID);
  g_.r = res;
  g_.ox = origin[0]; g_.oy = origin[1]; g_.oz = origin[2];
  g_.hx = spacing[0]; g_.hy = spacing[1]; g_.hz = spacing[2];
  dt_ = dt;
  N_ = res.size();
  fr_[0] = Dim3i{res.x + 1, res.y, res.z};
  fr_[1] = Dim3i{res.x, res.y + 1, res.z};
  fr_[2] = Dim3i{res.x, res.y, res.z + 1};
  Ftot_ = 0;
  for (int a = 0; a < 3; ++a) { F_[a] = fr_[a].size(); Ftot_ += F_[a]; }
  hfg_default_options(&opt_);
  check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  own_.s = stream_;
  for (int b = 0; b < 2; ++b)
    for (int a = 0; a < 3; ++a) {
      vel_[b][a].alloc(F_[a], stream_);
      color_[b][a].alloc(N_, stream_);
    }
  for (int b = 0; b < 2; ++b) dom_[b].alloc(N_, stream_);
  for (int a = 0; a < 3; ++a) prev_[a].alloc(F_[a], stream_);
  cg_ = cgDims(res);
  NC_ = cg_.size();
  solidIdx_.alloc(N_, stream_); markers_.alloc(N_, stream_); code_.alloc(NC_, stream_); cgc_.alloc(NC_, stream_);
  cgx_.alloc(NC_, stream_);
  cgr_.alloc(NC_, stream_);
  cgp_[0].alloc(NC_, stream_);
  cgp_[1].alloc(NC_, stream_);
  partials_.alloc(cgPartialsNeeded(res), stream_);
  colZ_.alloc((size_t)cgScheduleInts(cgDims(res)), stream_);
  // an empty schedule (no work items) until the first solve builds one
  check(cudaMemsetAsync(colZ_.p, 0, colZ_.bytes(), stream_), "memset");
  check(makeCgMaps(cg_, cgc_.p, cgr_.p, cgx_.p, false, cgp_[0].p, cgp_[1].p, &maps_), "CG tensor maps");
  cgState_.alloc(1, stream_);
  subState_.alloc(subSlots_ + 1, stream_);
  dist_.alloc(Ftot_, stream_); list_.alloc(Ftot_, stream_); mask_.alloc(Ftot_, stream_);
  hist_.alloc(kExtrapHistWords, stream_);
  offsets_.alloc(kMaxLayers + 2, stream_);
  cursor_.alloc(kMaxLayers + 2, stream_);
  cgHost_ = (CgState*)pinnedGet(sizeof(CgState));
  subHost_ = (SubstepState*)pinnedGet(sizeof(SubstepState));
  extrapHost_ = (unsigned int*)pinnedGet(sizeof(unsigned int) * 4);
  // GridFluidSolver.cpp:179-195: every field starts at zero
  for (int b = 0; b < 2; ++b) {
    for (int a = 0; a < 3; ++a) {
      check(cudaMemsetAsync(vel_[b][a].p, 0, vel_[b][a].bytes(), stream_), "memset");
      check(cudaMemsetAsync(color_[b][a].p, 0, color_[b][a].bytes(), stream_), "memset");
    }
    check(cudaMemsetAsync(dom_[b].p, 0, dom_[b].bytes(), stream_), "memset");
  }
  for (int a = 0; a < 3; ++a) check(cudaMemsetAsync(prev_[a].p, 0, prev_[a].bytes(), stream_), "memset");
  check(cudaMemsetAsync(solidIdx_.p, 0, N_, stream_), "memset");
  check(cudaMemsetAsync(markers_.p, 0, N_, stream_), "memset");
  check(cudaMemsetAsync(cgx_.p, 0, cgx_.bytes(), stream_), "memset");
  check(cudaMemsetAsync(cgState_.p, 0, sizeof(CgState), stream_), "memset");
  for (int i = 0; i < kEvents; ++i) check(cudaEventCreate(&ev_[i]), "cudaEventCreate");
  check(cudaStreamSynchronize(stream_), "sync");
  extrapUsers(+1);  // last: a constructor that throws registers nothing
}

GridSolver::~GridSolver() {
  if (copy_.s) cudaStreamSynchronize(copy_.s);
  if (stream_) cudaStreamSynchronize(stream_);
  if (advDone_) cudaEventDestroy(advDone_);
  if (copyDone_) cudaEventDestroy(copyDone_);
  extrapUsers(-1);
  for (auto* b : bsdf_) delete b;
  dropGraphs();
  if (mg_) mgDestroy(mg_);
  pinnedPut(cgHost_);
  pinnedPut(subHost_);
  pinnedPut(extrapHost_);
  for (int i = 0; i < kEvents; ++i)
    if (ev_[i]) cudaEventDestroy(ev_[i]);
  // the stream itself goes with own_, after the member arrays are freed on it
}

void GridSolver::launched(cudaError_t e, const char* what, int count) {
  check(e, what);
  launches_ += count;
}

void GridSolver::stageBegin(int i) {
  if (timing_) check(cudaEventRecord(ev_[2 * i], stream_), "cudaEventRecord");
}
void GridSolver::stageEnd(int i) {
  if (timing_) check(cudaEventRecord(ev_[2 * i + 1], stream_), "cudaEventRecord");
}

void GridSolver::enableTiming(bool on) { timing_ = on; }

void GridSolver::addBoundary(const float* sdfHost, const float vel[3]) {
  if ((int)bsdf_.size() >= kMaxBoundaries) throw CudaError("too many solid boundaries", HFG_ERR_INVALID);
  auto* b = new DArray<float>();
  b->alloc(N_, stream_);
  check(cudaMemcpyAsync(b->p, sdfHost, N_ * sizeof(float), cudaMemcpyHostToDevice, stream_), "upload sdf");
  bsdf_.push_back(b);
  for (int a = 0; a < 3; ++a) { bvel_.push_back(vel ? vel[a] : 0.f); btrans_.push_back(0.f); }
  check(cudaStreamSynchronize(stream_), "sync");
}

void GridSolver::addAnalyticBoundary(int type, const double params[6], const float vel[3]) {
  if ((int)bsdf_.size() >= kMaxBoundaries) throw CudaError("too many solid boundaries", HFG_ERR_INVALID);
  if (type < 0 || type > 2) throw CudaError("unknown analytic solid type", HFG_ERR_INVALID);
  const double zero[6] = {0, 0, 0, 0, 0, 0};
  auto* b = new DArray<float>();
  try {
    b->alloc(N_, stream_);
    check(launchAnalyticSdf(g_, type, params ? params : zero, b->p, stream_), "analytic sdf");
  } catch (...) {
    delete b;
    throw;
  }
  bsdf_.push_back(b);
  for (int a = 0; a < 3; ++a) { bvel_.push_back(vel ? vel[a] : 0.f); btrans_.push_back(0.f); }
}

void GridSolver::setBoundaryVelocity(int index, const float vel[3]) {
  if (index < 0 || index >= (int)bsdf_.size()) throw CudaError("boundary index out of range", HFG_ERR_INVALID);
  for (int a = 0; a < 3; ++a) bvel_[3 * index + a] = vel[a];
}

void GridSolver::addExternalForce(const float f[3]) {
  for (int a = 0; a < 3; ++a) ext_[a] += f[a];  // ExternalForcesSolver.cpp:45-48
}

void GridSolver::setVelocity(const float* x, const float* y, const float* z) {
  const float* s[3] = {x, y, z};
  for (int b = 0; b < 2; ++b)
    for (int a = 0; a < 3; ++a)
      check(cudaMemcpyAsync(vel_[b][a].p, s[a], F_[a] * 4, cudaMemcpyHostToDevice, stream_), "upload velocity");
  check(cudaStreamSynchronize(stream_), "sync");
}

void GridSolver::setFluidDomain(const float* d) {
  for (int b = 0; b < 2; ++b) check(cudaMemcpyAsync(dom_[b].p, d, N_ * 4, cudaMemcpyHostToDevice, stream_), "upload");
  check(cudaStreamSynchronize(stream_), "sync");
}

void GridSolver::setColor(const float* x, const float* y, const float* z) {
  const float* s[3] = {x, y, z};
  for (int b = 0; b < 2; ++b)
    for (int a = 0; a < 3; ++a)
      check(cudaMemcpyAsync(color_[b][a].p, s[a], N_ * 4, cudaMemcpyHostToDevice, stream_), "upload colour");
  check(cudaStreamSynchronize(stream_), "sync");
}

// GridFluidSolver.cpp:551-555: bbox written into field 1, copied to field 2.
void GridSolver::fluidDomainFromBBox(const float mn[3], const float mx[3]) {
  launched(launchFluidDomainFromBBox(g_, mn, mx, dom_[0].p, stream_), "fluid domain");
  check(cudaMemcpyAsync(dom_[1].p, dom_[0].p, N_ * 4, cudaMemcpyDeviceToDevice, stream_), "copy");
  check(cudaStreamSynchronize(stream_), "sync");
}

void GridSolver::setAdvection(int kind, int acc, int alg, float cfl, float mixing) {
  if (kind < 0 || kind > 3 || acc < 0 || acc > 2 || alg < 0 || alg > 4)
    throw CudaError("invalid advection settings", HFG_ERR_INVALID);
  adv_ = kind; acc_rk_ = acc; alg_ = alg; cfl_ = cfl; mixing_ = mixing;
  sFlag_ = vFlag_ = velFlag_ = false;
}

void GridSolver::setParticles(const float* pos, const float* vel, long long n) {
  finishMirrorCopy();
  if (n < 0) throw CudaError("negative particle count", HFG_ERR_INVALID);
  P_ = n;
  ppos_.alloc(3 * n, stream_);
  pvel_.alloc(3 * n, stream_);
  pv0_.alloc(3 * n, stream_);
  pscalar_.alloc(n, stream_);
  pvector_.alloc(3 * n, stream_);
  if (n > 0) {
    check(cudaMemcpyAsync(ppos_.p, pos, 12 * n, cudaMemcpyHostToDevice, stream_), "upload particles");
    if (vel) check(cudaMemcpyAsync(pvel_.p, vel, 12 * n, cudaMemcpyHostToDevice, stream_), "upload particles");
    else check(cudaMemsetAsync(pvel_.p, 0, 12 * n, stream_), "memset");
    check(cudaMemsetAsync(pscalar_.p, 0, 4 * n, stream_), "memset");
    check(cudaMemsetAsync(pvector_.p, 0, 12 * n, stream_), "memset");
  }
  sFlag_ = vFlag_ = velFlag_ = false;
  check(cudaStreamSynchronize(stream_), "sync");
}

// EulerParticles.cpp:140-179 on the device: the fluid cells of the current
// fluid-domain field that are not inside a solid get `ppc` particles each.
void GridSolver::seedParticles(int ppc, unsigned long long seed) {
  finishMirrorCopy();
  if (ppc <= 0) throw CudaError("particles per cell must be positive", HFG_ERR_INVALID);
  // Cells inside a solid get no particles (findFluidGrid,
  // EulerParticlesTool.cu:20).  The solids are classified at their current
  // placement, so a scene seeded before its first step already excludes them.
  BoundarySet bs{};
  bs.n = (int)bsdf_.size();
  for (int i = 0; i < bs.n; ++i) {
    bs.sdf[i] = bsdf_[i]->p;
    bs.tx[i] = btrans_[3 * i]; bs.ty[i] = btrans_[3 * i + 1]; bs.tz[i] = btrans_[3 * i + 2];
  }
  classifySolids(bs);
  const int cellsPerBlock = 4096;
  int nb = (int)((N_ + cellsPerBlock - 1) / cellsPerBlock);
  DArray<unsigned int> counts;
  counts.alloc(nb, stream_);
  DArray<unsigned long long> total;
  total.alloc(1, stream_);
  const float* fsdf = dom_[cur()].p;
  launched(launchSeedCount(g_.r, fsdf, solidIdx_.p, counts.p, cellsPerBlock, stream_), "seed count");
  launched(launchSeedScan(counts.p, nb, total.p, stream_), "seed scan");
  unsigned long long nf = 0;
  check(cudaMemcpyAsync(&nf, total.p, 8, cudaMemcpyDeviceToHost, stream_), "read count");
  check(cudaStreamSynchronize(stream_), "sync");
  long long n = (long long)nf * ppc;
  P_ = n;
  ppos_.alloc(3 * n, stream_);
  pvel_.alloc(3 * n, stream_);
  pv0_.alloc(3 * n, stream_);
  pscalar_.alloc(n, stream_);
  pvector_.alloc(3 * n, stream_);
  if (n > 0) {
    launched(launchSeedWrite(g_, fsdf, solidIdx_.p, counts.p, cellsPerBlock, ppc, seed, ppos_.p, stream_), "seed write");
    check(cudaMemsetAsync(pvel_.p, 0, 12 * n, stream_), "memset");
    check(cudaMemsetAsync(pscalar_.p, 0, 4 * n, stream_), "memset");
    check(cudaMemsetAsync(pvector_.p, 0, 12 * n, stream_), "memset");
  }
  sFlag_ = vFlag_ = velFlag_ = false;
  check(cudaStreamSynchronize(stream_), "sync");
}

void GridSolver::setOptions(const hfg_options_t& o) {
  if (o.precond < 0 || o.precond > 2 || o.tol_mode < 0 || o.tol_mode > 1 || !(o.tol > 0))
    throw CudaError("invalid solver options", HFG_ERR_INVALID);
  if (o.sampling < 0 || o.sampling > 4) throw CudaError("sampling algorithm must be in [0, 4]", HFG_ERR_INVALID);
  if (o.extrapolation_layers < 0 || o.extrapolation_layers > kMaxLayers)
    throw CudaError("extrapolation layers must be in [0, 1000]", HFG_ERR_INVALID);
  if (o.sort_interval < 0) throw CudaError("sort interval must be >= 0", HFG_ERR_INVALID);
  if (o.mg_half < 0 || o.mg_half > 2) throw CudaError("mg_half must be 0, 1 or 2", HFG_ERR_INVALID);
  bool mgChanged = o.precond == HFG_PRECOND_MG &&
                   (!mg_ || o.mg_levels != opt_.mg_levels || o.mg_smooth != opt_.mg_smooth || o.mg_half != opt_.mg_half);
  const bool fp64Changed = (o.pressure_fp64 != 0) != (opt_.pressure_fp64 != 0);
  opt_ = o;
  if (fp64Changed) {
    // the pressure iterate changes type: new tensor map, recaptured graphs
    dropGraphs();
    if (o.pressure_fp64) {
      cgx64_.alloc(NC_, stream_);
      check(cudaMemsetAsync(cgx64_.p, 0, cgx64_.bytes(), stream_), "memset");
    }
    check(makeCgMaps(cg_, cgc_.p, cgr_.p, xPtr(), xDouble(), cgp_[0].p, cgp_[1].p, &maps_), "CG tensor maps");
  }
  if (mgChanged) {
    dropGraphs();
    if (mg_) mgDestroy(mg_);
    mg_ = mgCreate(cg_, o.mg_levels, o.mg_smooth, o.mg_half, stream_);
  }
}

SolidVelTable GridSolver::solidTable() const {
  SolidVelTable t{};
  t.solidIdx = solidIdx_.p;
  for (size_t i = 0; i < bsdf_.size(); ++i) {
    t.vx[i] = bvel_[3 * i]; t.vy[i] = bvel_[3 * i + 1]; t.vz[i] = bvel_[3 * i + 2];
  }
  return t;
}

// Boundary.cpp:115-122: move (translation += -dt * velocity), re-sample,
// classify.  Solid face velocities are formed on demand from the per-solid
// table, never stored.
void GridSolver::updateBoundarys() {
  BoundarySet b{};
  b.n = (int)bsdf_.size();
  for (int i = 0; i < b.n; ++i) {
    for (int a = 0; a < 3; ++a) btrans_[3 * i + a] = std::fma(-dt_, bvel_[3 * i + a], btrans_[3 * i + a]);
    b.sdf[i] = bsdf_[i]->p;
    b.tx[i] = btrans_[3 * i]; b.ty[i] = btrans_[3 * i + 1]; b.tz[i] = btrans_[3 * i + 2];
    b.vx[i] = bvel_[3 * i]; b.vy[i] = bvel_[3 * i + 1]; b.vz[i] = bvel_[3 * i + 2];
  }
  classifySolids(b);
}

// solidIdx_ from the boundaries at their current placement.  A placement
// equal to the one solidIdx_ already holds (same SDF arrays, same
// translations: solids at rest) needs no new classification.
void GridSolver::classifySolids(const BoundarySet& b) {
  std::vector<float> key;
  key.reserve(4 * b.n + 1);
  key.push_back((float)b.n);
  for (int i = 0; i < b.n; ++i) {
    key.push_back(b.tx[i]);
    key.push_back(b.ty[i]);
    key.push_back(b.tz[i]);
  }
  std::vector<const float*> ptrs(b.sdf, b.sdf + b.n);
  if (classified_ && key == classKey_ && ptrs == classSdf_) return;
  if (b.n == 0) check(cudaMemsetAsync(solidIdx_.p, 0, N_, stream_), "memset");
  else launched(launchSolidClassify(g_, b, solidIdx_.p, nullptr, stream_), "solid classify");
  classified_ = true;
  classKey_ = std::move(key);
  classSdf_ = std::move(ptrs);
}

// ExternalForcesSolver.cpp:50-58: two unit-field axpys, each skipped when all
// three of its coefficients are below FLT_EPSILON.
void GridSolver::forcesTerms(float gv[3], bool& doG, float ev[3], bool& doE) const {
  for (int a = 0; a < 3; ++a) { gv[a] = gravity_[a] * dt_; ev[a] = ext_[a] * dt_; }
  auto tiny = [](const float v[3]) {
    return std::fabs(v[0]) < 1.1920929e-07f && std::fabs(v[1]) < 1.1920929e-07f && std::fabs(v[2]) < 1.1920929e-07f;
  };
  doG = !tiny(gv);
  doE = !tiny(ev);
}

void GridSolver::p2gFace(const float* vel, float* const out[3], float* const copy[3], const float add[3], bool doAdd,
                         const float add2[3], bool doAdd2) {
  for (int a = 0; a < 3; ++a) {
    acc_[a].alloc(F_[a], stream_);
    check(cudaMemsetAsync(acc_[a].p, 0, acc_[a].bytes(), stream_), "memset");
  }
  float2* acc[3] = {acc_[0].p, acc_[1].p, acc_[2].p};
  launched(launchP2GFace(g_, alg_, ppos_.p, vel, P_, acc, stream_), "p2g");
  for (int a = 0; a < 3; ++a)
    launched(launchNormalize(F_[a], acc_[a].p, out[a], copy ? copy[a] : nullptr, add ? add[a] : 0.f, doAdd,
                             add2 ? add2[a] : 0.f, doAdd2, stream_),
             "normalize");
}

void GridSolver::p2gCell(const float* vals, int span, int comp, float* out) {
  cacc_.alloc(N_, stream_);
  check(cudaMemsetAsync(cacc_.p, 0, cacc_.bytes(), stream_), "memset");
  launched(launchP2GCell(g_, alg_, ppos_.p, vals, span, comp, P_, cacc_.p, stream_), "p2g cell");
  launched(launchNormalize(N_, cacc_.p, out, nullptr, 0.f, 0, 0.f, 0, stream_), "normalize cell");
}

// Corner tables of the advecting velocity (G2P and every substep sample read
// them) and a cleared substep state.
FaceQuads GridSolver::beginParticleStep(ConstFaceField vin) {
  float4* quads[3];
  for (int a = 0; a < 3; ++a) {
    quads_[a].alloc(faceQuadCount(g_.r, a), stream_);
    quads[a] = quads_[a].p;
  }
  launched(launchFaceQuads(g_.r, vin, quads, stream_), "face corner tables");
  check(cudaMemsetAsync(subState_.p, 0, sizeof(SubstepState) * (subSlots_ + 1), stream_), "memset");
  return makeFaceQuads(g_, quads[0], quads[1], quads[2]);
}

// EulerParticles.cpp:231-325.  Substeps are launched speculatively in chunks;
// a launch whose slot is already finished does nothing.  The first sample (v0
// and its max) is already in place (advectBegin).
void GridSolver::advectParticles(const FaceQuads& v) {
  long long nclamp = opt_.clamp_mode == 1 ? std::min<long long>(P_, N_) : P_;
  int slot = 0;
  partMs_[1] = 0.f;
  // the first batch runs up to two short of the previous step's count without
  // a read-back (the CFL rule changes the count slowly from step to step);
  // then chunks of kSubstepChunk.  A launch past the last substep does nothing.
  int batch = std::max(kSubstepChunk, substeps_ - 2);
  for (;;) {
    if (timing_) check(cudaEventRecord(ev_[18], stream_), "cudaEventRecord");
    for (int k = 0; k < batch && slot < subSlots_; ++k, ++slot)
      launched(launchSubstep(g_, v, ppos_.p, pv0_.p, P_, acc_rk_, dt_, cfl_, nclamp, subState_.p, slot, stream_),
               "substep");
    if (timing_) check(cudaEventRecord(ev_[19], stream_), "cudaEventRecord");
    readBack(subHost_, subState_.p + slot, sizeof(SubstepState), stream_);
    check(cudaStreamSynchronize(stream_), "substep sync");
    if (timing_) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, ev_[18], ev_[19]) == cudaSuccess) partMs_[1] += ms;
    }
    if (subHost_->finished) { substeps_ = subHost_->count; break; }
    if (slot >= subSlots_) throw CudaError("CFL substep limit reached", HFG_ERR_STATE);
    batch = kSubstepChunk;
  }
}

// GridFluidSolver.cpp:399-416 with the advection solvers' bodies
// (SemiLagrangian.cpp:135-186, ParticleInCell.cpp:93-108,
// FluidImplicitParticle.cpp:98-127, MixPICAndFLIP.cpp:64-136); the external
// forces of ExternalForcesSolver.cpp:50-58 are folded into the pass that
// writes the advected velocity.
void GridSolver::computeAdvection() {
  if (advectBegin()) {
    advectParticles(vq_);
    advectEnd();
  }
}

// The advection up to the CFL substeps: the whole semi-Lagrangian advection
// (returns false), or for the particle solvers the corner tables, the G2P
// velocity update and the first substep sample (returns true).
bool GridSolver::advectBegin() {
  finishMirrorCopy();
  int ci = cur(), ni = nxt();
  float gv[3], ev[3];
  bool doG, doE;
  forcesTerms(gv, doG, ev, doE);
  if (adv_ == HFG_ADV_SEMI_LAGRANGIAN) {
    stageBegin(1);
    launched(launchSLFace(g_, acc_rk_, dt_, cvel(ci), cvel(ci), mvel(ni), gv, doG, ev, doE, stream_, opt_.sampling),
             "sl face");
    if (opt_.advect_scalars) {
      const float* in[4] = {color_[ci][0].p, color_[ci][1].p, color_[ci][2].p, dom_[ci].p};
      float* out[4] = {color_[ni][0].p, color_[ni][1].p, color_[ni][2].p, dom_[ni].p};
      launched(launchSLCell(g_, acc_rk_, dt_, cvel(ci), in, out, 4, stream_, opt_.sampling), "sl cell");
    }
    stageEnd(1);
    return false;
  }
  if (P_ <= 0) throw CudaError("particle advection needs particles", HFG_ERR_STATE);
  stageBegin(1);
  if (opt_.sort_interval > 0) {
    // the sort's buffers are taken at the first particle step, not at the
    // first sort: growing the allocator's pool by about 1 GB can take 0.2 s
    reserveSortScratch();
    if (particleSteps_ > 0 && particleSteps_ % opt_.sort_interval == 0) sortParticles();
  }
  ++particleSteps_;
  ConstFaceField prev{{prev_[0].p, prev_[1].p, prev_[2].p}};
  int mode = adv_ == HFG_ADV_PIC ? MODE_PIC : (adv_ == HFG_ADV_FLIP ? MODE_FLIP : MODE_MIX);
  int first = (mode != MODE_PIC && !velFlag_) ? 1 : 0;
  vq_ = beginParticleStep(cvel(ci));
  if (timing_) check(cudaEventRecord(ev_[16], stream_), "cudaEventRecord");
  launched(launchParticleVelUpdate(g_, mode, alg_, cvel(ci), prev, first, mixing_, ppos_.p, pvel_.p, P_, stream_,
                                   &vq_, pv0_.p, subState_.p),
           "particle velocity");
  if (timing_) check(cudaEventRecord(ev_[17], stream_), "cudaEventRecord");
  if (mode != MODE_PIC) velFlag_ = true;
  // the LINEAR G2P also took the first substep sample (v0 and its max)
  if (alg_ != HFG_LINEAR)
    launched(launchSubstepBegin(g_, vq_, ppos_.p, pv0_.p, P_, subState_.p, stream_), "substep begin");
  startMirrorCopy(false);
  return true;
}

// The particles in cell order (hfg_sort.cu), with their velocities and
// carried colour / domain values.  v at the substep start is not carried: each
// step's velocity update writes it before the substeps read it.
// The sort's keys, values, digit counts and gather buffer for P_ particles
// (no-ops once they have that size).
void GridSolver::reserveSortScratch() {
  for (int i = 0; i < 2; ++i) {
    sortKey_[i].alloc(P_, stream_);
    sortVal_[i].alloc(P_, stream_);
  }
  const long long entries = sortCountEntries(P_);
  sortCounts_.alloc(entries, stream_);
  sortSums_.alloc(sortScanBlocks(entries), stream_);
  sortTmp_.alloc(3 * P_, stream_);
}

void GridSolver::sortParticles() {
  if (P_ <= 0) return;
  // With clamp_mode 1 the boundary fix reaches only the first min(N, P)
  // particles, as the reference's launch does (EulerParticlesTool.cu:880):
  // those stay the first ones, each group sorted within its own range.
  const long long split = (opt_.clamp_mode == 1 && P_ > N_) ? N_ : 0;
  finishMirrorCopy();
  reserveSortScratch();
  const SortScratch sc{sortKey_[0].p, sortKey_[1].p, sortVal_[0].p, sortVal_[1].p, sortCounts_.p, sortSums_.p};
  const unsigned int* perm = nullptr;
  launched(launchSortPermutation(g_, ppos_.p, P_, split, sc, &perm, stream_), "particle sort",
           sortPassesLaunches(N_, split > 0));
  for (DArray<float>* a : {&ppos_, &pvel_, &pvector_}) {
    if (!a->p || a->n != (size_t)(3 * P_)) continue;
    launched(launchGather(a->p, 3, perm, P_, sortTmp_.p, stream_), "particle gather");
    a->swap(sortTmp_);
  }
  if (pscalar_.p && pscalar_.n == (size_t)P_) {
    launched(launchGather(pscalar_.p, 1, perm, P_, sortTmp_.p, stream_), "particle gather");
    check(cudaMemcpyAsync(pscalar_.p, sortTmp_.p, sizeof(float) * P_, cudaMemcpyDeviceToDevice, stream_),
          "particle gather copy");
  }
}

// The CFL substeps of this scene alone, as the batch stepper's shared launches
// would run them (substepTask).
SubstepTask GridSolver::substepTask() {
  SubstepTask t;
  t.g = g_;
  t.vel = vq_;
  t.pos = ppos_.p;
  t.v0 = pv0_.p;
  t.P = P_;
  t.nclamp = opt_.clamp_mode == 1 ? std::min<long long>(P_, N_) : P_;
  t.st = subState_.p;
  t.acc = acc_rk_;
  t.dt = dt_;
  t.cfl = cfl_;
  return t;
}

// The particle advection after the substeps: P2G of the velocities (with the
// FLIP copy and the external forces) and of the carried scalars.
void GridSolver::advectEnd() {
  int ci = cur(), ni = nxt();
  float gv[3], ev[3];
  bool doG, doE;
  forcesTerms(gv, doG, ev, doE);
  float* vout[3] = {vel_[ni][0].p, vel_[ni][1].p, vel_[ni][2].p};
  int mode = adv_ == HFG_ADV_PIC ? MODE_PIC : (adv_ == HFG_ADV_FLIP ? MODE_FLIP : MODE_MIX);
  startMirrorCopy(true);
  float* copy[3] = {prev_[0].p, prev_[1].p, prev_[2].p};
  if (timing_) check(cudaEventRecord(ev_[20], stream_), "cudaEventRecord");
  p2gFace(pvel_.p, vout, mode == MODE_PIC ? nullptr : copy, gv, doG, ev, doE);
  if (timing_) check(cudaEventRecord(ev_[21], stream_), "cudaEventRecord");
  if (opt_.advect_scalars) {
    // colour (CC vector) then fluid domain (CC scalar): G2P once, P2G every step
    if (!vFlag_) {
      for (int a = 0; a < 3; ++a)
        launched(launchG2PCell(g_, alg_, color_[ci][a].p, ppos_.p, P_, pvector_.p, 3, a, stream_), "g2p colour");
      vFlag_ = true;
    }
    for (int a = 0; a < 3; ++a) p2gCell(pvector_.p, 3, a, color_[ni][a].p);
    if (!sFlag_) {
      launched(launchG2PCell(g_, alg_, dom_[ci].p, ppos_.p, P_, pscalar_.p, 1, 0, stream_), "g2p domain");
      sFlag_ = true;
    }
    p2gCell(pscalar_.p, 1, 0, dom_[ni].p);
  }
  stageEnd(1);
}

void GridSolver::cgIteration(int it, float sx, float sy, float sz, int pc) {
  const int po = it & 1, pn = (it + 1) & 1;
  launched(launchCgDirection(cg_, sx, sy, sz, maps_.rH, maps_.pH[po], maps_.codeH, cgc_.p, cgr_.p, cgp_[po].p,
                             cgp_[pn].p, partials_.p, cgState_.p, pc, stream_, colZ_.p, xDouble()),
           "cg direction");
  launched(launchCgUpdate(cg_, sx, sy, sz, maps_.pH[pn], maps_.rI, maps_.xI, maps_.codeI, cgp_[pn].p, xPtr(), xDouble(),
                          cgr_.p,
                          partials_.p, cgState_.p, pc, stream_, colZ_.p),
           "cg update");
}

template <class F> cudaGraphExec_t GridSolver::capture(F&& f) {
  cgWarmLaunchCache();  // launch-shape queries happen before the capture
  cudaGraph_t g = nullptr;
  cudaGraphExec_t e = nullptr;
  const long long saved = launches_;
  check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
  try {
    f();
  } catch (...) {
    cudaStreamEndCapture(stream_, &g);
    if (g) cudaGraphDestroy(g);
    launches_ = saved;
    throw;
  }
  check(cudaStreamEndCapture(stream_, &g), "end capture");
  launches_ = saved;
  cudaError_t r = cudaGraphInstantiate(&e, g, 0);
  cudaGraphDestroy(g);
  check(r, "graph instantiate");
  return e;
}

void GridSolver::dropGraphs() {
  for (auto& g : cgGraph_)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

void GridSolver::runCg() {
  const float sx = dt_ / (1.0f * g_.hx * g_.hx), sy = dt_ / (1.0f * g_.hy * g_.hy), sz = dt_ / (1.0f * g_.hz * g_.hz);
  if (opt_.precond == HFG_PRECOND_MG) {
    auto cap = [this](const std::function<void()>& f) { return capture(f); };
    mgRunCg(mg_, cg_, sx, sy, sz, maps_, cgc_.p, xPtr(), xDouble(), cgr_.p, cgState_.p, cgHost_, stream_, launches_, cap,
            &cgGraph_[2], colZ_.p);
  } else {
    const int pc = opt_.precond == HFG_PRECOND_JACOBI ? 1 : 0;
    // kCgChunk is even, so every chunk starts on the same p buffer
    if (!cgGraph_[pc])
      cgGraph_[pc] = capture([&] {
        for (int k = 0; k < kCgChunk; ++k) cgIteration(k, sx, sy, sz, pc);
      });
    // as many chunks as the previous solve needed, less one, go out before the
    // first convergence read; every kernel of a chunk past convergence returns
    // at once
    int batch = std::max(1, cgChunks_ - 1), chunks = 0;
    for (;;) {
      for (int k = 0; k < batch; ++k) {
        check(cudaGraphLaunch(cgGraph_[pc], stream_), "cg chunk");
        launches_ += 2 * kCgChunk;
        ++chunks;
      }
      readBack(cgHost_, cgState_.p, sizeof(CgState), stream_);
      check(cudaStreamSynchronize(stream_), "cg sync");
      if (cgHost_->done) break;
      batch = 1;
    }
    cgChunks_ = (cgHost_->iter + kCgChunk - 1) / kCgChunk;
  }
  if (cgHost_->error == 4) throw CudaError("pressure CG: a work item of the schedule is invalid", HFG_ERR_STATE);
  if (cgHost_->error) throw CudaError("pressure CG: a stage load did not complete in time", HFG_ERR_TIMEOUT);
}

// PressureSolver.cpp:194-197 + GridFluidSolver.cpp:435-525
void GridSolver::computePressure() {
  int ni = nxt();
  stageBegin(3);
  if (adv_ == HFG_ADV_SEMI_LAGRANGIAN) {
    launched(launchMarkersFromSDF(N_, solidIdx_.p, dom_[ni].p, markers_.p, stream_), "markers");
  } else {
    launched(launchMarkersInit(N_, solidIdx_.p, markers_.p, stream_), "markers");
    launched(launchMarkersFromParticles(g_, ppos_.p, P_, markers_.p, stream_), "markers");
  }
  launched(launchStencilCode(g_.r, cg_.x, markers_.p, code_.p, stream_, cgc_.p), "stencil code");
  const int schedPc =
      opt_.precond == HFG_PRECOND_MG ? 2 : (opt_.precond == HFG_PRECOND_JACOBI ? 1 : 0);
  launched(launchCgSchedule(cg_, cgc_.p, colZ_.p, schedPc, xDouble(), stream_), "cg schedule", 2);
  stageEnd(3);
  stageBegin(4);
  CgState init{};
  init.maxIter = (int)std::min<long long>(opt_.max_iter < 0 ? N_ : opt_.max_iter, 0x7fffffff);
  init.precond = opt_.precond == HFG_PRECOND_JACOBI ? 1 : 0;
  init.tolMode = opt_.tol_mode;
  init.tol = opt_.tol;
  *cgHost_ = init;
  check(cudaMemcpyAsync(cgState_.p, cgHost_, sizeof(CgState), cudaMemcpyHostToDevice, stream_), "cg state");
  const float sx = dt_ / (1.0f * g_.hx * g_.hx), sy = dt_ / (1.0f * g_.hy * g_.hy), sz = dt_ / (1.0f * g_.hz * g_.hz);
  ConstFaceField none{{nullptr, nullptr, nullptr}};
  launched(launchRhsInit(g_, cvel(ni), none, solidTable(), markers_.p, code_.p, sx, sy, sz, nullptr, cgr_.p, xPtr(),
                         xDouble(),
                         cgp_[0].p, partials_.p, cgState_.p, init.precond, stream_),
           "rhs");
  // the CG kernels never store at non-fluid cells, and the fluid moves between
  // solves: the second direction buffer starts zero too
  check(cudaMemsetAsync(cgp_[1].p, 0, cgp_[1].bytes(), stream_), "memset");
  if (opt_.autotune && opt_.precond != HFG_PRECOND_MG && tunedCgZPer(0, cg_) < 0) {
    // measure the launch shapes on this system, then set the solve up again
    autotuneCg(sx, sy, sz, init.precond);
    *cgHost_ = init;
    check(cudaMemcpyAsync(cgState_.p, cgHost_, sizeof(CgState), cudaMemcpyHostToDevice, stream_), "cg state");
    launched(launchRhsInit(g_, cvel(ni), none, solidTable(), markers_.p, code_.p, sx, sy, sz, nullptr, cgr_.p, xPtr(),
                           xDouble(), cgp_[0].p, partials_.p, cgState_.p, init.precond, stream_),
             "rhs");
    check(cudaMemsetAsync(cgp_[1].p, 0, cgp_[1].bytes(), stream_), "memset");
  }
  if (opt_.precond == HFG_PRECOND_MG) mgSetup(mg_, g_.r, markers_.p, code_.p, sx, sy, sz, stream_, launches_);
  stageEnd(4);
  stageBegin(5);
  runCg();
  cgIters_ = cgHost_->iter;
  cgResid_ = std::sqrt(cgHost_->rr);
  cgBnorm_ = std::sqrt(cgHost_->bb);
  // the stop rule of the solve (CuMatrixFreePCG.cpp:28,51, or relative) met
  cgConverged_ = cgHost_->tolMode == 0 ? (std::sqrt(cgResid_) < cgHost_->tol ? 1 : 0)
                                       : (cgBnorm_ == 0.0 || cgResid_ / cgBnorm_ < cgHost_->tol ? 1 : 0);
  cgTrueResid_ = -1.0;
  if (opt_.report_divergence) {
    // the final residual check, ||b - A x|| in FP64 on the unprojected velocity
    const int nb = divergenceBlocks();
    divScratch_.alloc(2 * nb + 2, stream_);
    divTicket_.alloc(2, stream_);
    launched(launchTrueResidual(g_, cvel(ni), solidTable(), markers_.p, code_.p, xPtr(), xDouble(), sx, sy, sz,
                                divScratch_.p, divTicket_.p, divScratch_.p + 2 * nb, stream_),
             "true residual");
    double rb[2] = {0.0, 0.0};
    check(cudaMemcpyAsync(rb, divScratch_.p + 2 * nb, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream_), "read");
    check(cudaStreamSynchronize(stream_), "sync");
    cgTrueResid_ = std::sqrt(rb[0]);
  }
  stageEnd(5);
  stageBegin(6);
  ConstFaceField noneSv{{nullptr, nullptr, nullptr}};
  launched(launchGradient(g_, dt_ / (1.0f * g_.hx), dt_ / (1.0f * g_.hy), dt_ / (1.0f * g_.hz), markers_.p, xPtr(),
                          xDouble(),
                          mvel(ni), noneSv, solidTable(), stream_),
           "gradient");
  if (opt_.report_divergence) {
    const int nb = divergenceBlocks();
    divScratch_.alloc(2 * nb + 2, stream_);
    divTicket_.alloc(2, stream_);
    launched(launchDivergenceNorm(g_, cvel(ni), solidTable(), markers_.p, divScratch_.p, divTicket_.p,
                                  divScratch_.p + 2 * nb, stream_),
             "divergence");
    double sum = 0.0;
    unsigned bits = 0;
    check(cudaMemcpyAsync(&sum, divScratch_.p + 2 * nb, sizeof(double), cudaMemcpyDeviceToHost, stream_), "read");
    check(cudaMemcpyAsync(&bits, divTicket_.p + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_), "read");
    check(cudaStreamSynchronize(stream_), "sync");
    divL2_ = std::sqrt(sum);
    float mx;
    std::memcpy(&mx, &bits, sizeof(mx));
    divMax_ = mx;
  }
  stageEnd(6);
}

// GridFluidSolver.cpp:527-537 -> EulerSolverTool.cu:904-969
void GridSolver::extrapolate() {
  stageBegin(7);
  int ni = nxt();
  int nums = opt_.extrapolation_layers;
  extrapDepth_ = 0;
  if (nums > 1) {
    float* vals[3] = {vel_[ni][0].p, vel_[ni][1].p, vel_[ni][2].p};
    long long off[3] = {0, F_[0], F_[0] + F_[1]};
    ExtrapScratch sc{dist_.p, list_.p, hist_.p, offsets_.p, cursor_.p, mask_.p};
    launched(launchExtrapDistance(fr_, vals, off, nums, sc, stream_), "extrapolation distance", 17);
    check(launchExtrapLayers(fr_, vals, off, sc, nums, stream_, &launches_), "extrapolation layers");
    readBack(extrapHost_, extrapBarWords(sc), sizeof(unsigned int) * 4, stream_);
    check(cudaStreamSynchronize(stream_), "extrapolation sync");
    if (extrapHost_[2] != 0u) throw CudaError("extrapolation: a grid barrier timed out", HFG_ERR_TIMEOUT);
    extrapDepth_ = (int)extrapHost_[3];
  }
  stageEnd(7);
}

void GridSolver::stepBoundaries() {
  stageBegin(0);
  updateBoundarys();
  stageEnd(0);
}

void GridSolver::updateWithoutPressure() {
  stepBoundaries();
  computeAdvection();
}

void GridSolver::solvePressure() {
  computePressure();
  extrapolate();
  finishMirrorCopy();
  bufferFlag_ = !bufferFlag_;  // GridFluidSolver.cpp:393-397
  time_ += dt_;
}

void GridSolver::update() {
  updateWithoutPressure();
  solvePressure();
  if (timing_) {
    check(cudaStreamSynchronize(stream_), "sync");
    for (int i = 0; i < 8; ++i) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, ev_[2 * i], ev_[2 * i + 1]) == cudaSuccess) stageMs_[i] = ms;
      else stageMs_[i] = 0.f;
    }
    if (adv_ != HFG_ADV_SEMI_LAGRANGIAN) {
      float ms = 0.f;
      partMs_[0] = cudaEventElapsedTime(&ms, ev_[16], ev_[17]) == cudaSuccess ? ms : 0.f;
      partMs_[2] = cudaEventElapsedTime(&ms, ev_[20], ev_[21]) == cudaSuccess ? ms : 0.f;
    }
    cudaGetLastError();
  }
}

void GridSolver::synchronize() { check(cudaStreamSynchronize(stream_), "sync"); }

// The autotuner: every candidate z-chunk length of the CG kernels is timed on
// the current system (a few iterations each, events around every kernel) and
// the fastest per kernel is recorded for this grid size.  The iterations
// change x, r and p; the caller sets the solve up again afterwards.  The
// captured CG graphs hold launch shapes, so they are dropped.
void GridSolver::autotuneCg(float sx, float sy, float sz, int pc) {
  constexpr int kIters = 4;
  const std::vector<int> cands = cgZPerCandidates(cg_);
  cudaEvent_t e[3 * kIters + 1];
  for (auto& x : e) check(cudaEventCreate(&x), "cudaEventCreate");
  float best[2] = {1e30f, 1e30f};
  int pick[2] = {cands[0], cands[0]};
  CgState st{};
  st.maxIter = 0x7fffffff;
  st.precond = pc;
  st.tolMode = HFG_TOL_RELATIVE;
  st.tol = 0.0;  // never converges: every launch does its work
  st.rz = 1.0;
  st.bb = 1.0;
  try {
    for (int z : cands) {
      setTunedCgZPer(0, cg_, z);
      setTunedCgZPer(1, cg_, z);
      // the schedule's shortest chunk is the tuned length
      launched(launchCgSchedule(cg_, cgc_.p, colZ_.p, pc, xDouble(), stream_), "cg schedule", 2);
      *cgHost_ = st;
      check(cudaMemcpyAsync(cgState_.p, cgHost_, sizeof(CgState), cudaMemcpyHostToDevice, stream_), "cg state");
      cgIteration(0, sx, sy, sz, pc);  // warm-up
      for (int it = 0; it < kIters; ++it) {
        const int po = it & 1, pn = po ^ 1;
        check(cudaEventRecord(e[3 * it], stream_), "event");
        launched(launchCgDirection(cg_, sx, sy, sz, maps_.rH, maps_.pH[po], maps_.codeH, cgc_.p, cgr_.p,
                                   cgp_[po].p, cgp_[pn].p, partials_.p, cgState_.p, pc, stream_, colZ_.p, xDouble()),
                 "cg direction");
        check(cudaEventRecord(e[3 * it + 1], stream_), "event");
        launched(launchCgUpdate(cg_, sx, sy, sz, maps_.pH[pn], maps_.rI, maps_.xI, maps_.codeI, cgp_[pn].p, xPtr(),
                                xDouble(), cgr_.p, partials_.p, cgState_.p, pc, stream_, colZ_.p),
                 "cg update");
        check(cudaEventRecord(e[3 * it + 2], stream_), "event");
      }
      check(cudaEventSynchronize(e[3 * kIters - 1]), "event sync");
      float t[2] = {0.f, 0.f};
      for (int it = 0; it < kIters; ++it)
        for (int k = 0; k < 2; ++k) {
          float ms = 0.f;
          check(cudaEventElapsedTime(&ms, e[3 * it + k], e[3 * it + k + 1]), "elapsed");
          t[k] += ms;
        }
      for (int k = 0; k < 2; ++k)
        if (t[k] < best[k]) { best[k] = t[k]; pick[k] = z; }
    }
  } catch (...) {
    for (auto& x : e) cudaEventDestroy(x);
    setTunedCgZPer(0, cg_, -1);
    setTunedCgZPer(1, cg_, -1);
    throw;
  }
  for (auto& x : e) cudaEventDestroy(x);
  setTunedCgZPer(0, cg_, pick[0]);
  setTunedCgZPer(1, cg_, pick[1]);
  launched(launchCgSchedule(cg_, cgc_.p, colZ_.p, pc, xDouble(), stream_), "cg schedule", 2);
  dropGraphs();
}

float GridSolver::timeCg(int iters) {
  if (iters <= 0) throw CudaError("iterations must be positive", HFG_ERR_INVALID);
  const float sx = dt_ / (1.0f * g_.hx * g_.hx), sy = dt_ / (1.0f * g_.hy * g_.hy), sz = dt_ / (1.0f * g_.hz * g_.hz);
  CgState st{};
  st.maxIter = 0x7fffffff;
  st.precond = opt_.precond == HFG_PRECOND_JACOBI ? 1 : 0;
  st.tolMode = HFG_TOL_RELATIVE;
  st.tol = 0.0;  // never converges: every launch does its work
  st.rz = 1.0;
  st.bb = 1.0;
  *cgHost_ = st;
  check(cudaMemcpyAsync(cgState_.p, cgHost_, sizeof(CgState), cudaMemcpyHostToDevice, stream_), "cg state");
  check(cudaEventRecord(ev_[14], stream_), "event");
  for (int it = 0; it < iters; ++it) cgIteration(it, sx, sy, sz, st.precond);
  check(cudaEventRecord(ev_[15], stream_), "event");
  check(cudaEventSynchronize(ev_[15]), "event sync");
  float ms = 0.f;
  check(cudaEventElapsedTime(&ms, ev_[14], ev_[15]), "elapsed");
  check(cudaMemcpy(cgHost_, cgState_.p, sizeof(CgState), cudaMemcpyDeviceToHost), "read cg state");
  if (cgHost_->error == 4) throw CudaError("pressure CG: a work item of the schedule is invalid", HFG_ERR_STATE);
  if (cgHost_->error) throw CudaError("pressure CG: a stage load did not complete in time", HFG_ERR_TIMEOUT);
  return ms / iters;
}

void GridSolver::getVelocity(int which, float* x, float* y, float* z) {
  int b = which == 0 ? cur() : nxt();
  float* d[3] = {x, y, z};
  for (int a = 0; a < 3; ++a)
    if (d[a]) check(cudaMemcpyAsync(d[a], vel_[b][a].p, F_[a] * 4, cudaMemcpyDeviceToHost, stream_), "download");
  synchronize();
}

void GridSolver::getFluidDomain(float* d) {
  check(cudaMemcpyAsync(d, dom_[cur()].p, N_ * 4, cudaMemcpyDeviceToHost, stream_), "download");
  synchronize();
}

void GridSolver::getColor(float* x, float* y, float* z) {
  float* d[3] = {x, y, z};
  for (int a = 0; a < 3; ++a)
    if (d[a]) check(cudaMemcpyAsync(d[a], color_[cur()][a].p, N_ * 4, cudaMemcpyDeviceToHost, stream_), "download");
  synchronize();
}

void GridSolver::getMarkers(uint8_t* m) {
  check(cudaMemcpyAsync(m, markers_.p, N_, cudaMemcpyDeviceToHost, stream_), "download");
  synchronize();
}

void GridSolver::getPressure(float* p) {
  if (xDouble()) {
    std::vector<double> tmp((size_t)N_);
    check(cudaMemcpy2DAsync(tmp.data(), (size_t)g_.r.x * 8, cgx64_.p, (size_t)cg_.x * 8, (size_t)g_.r.x * 8,
                            (size_t)g_.r.y * g_.r.z, cudaMemcpyDeviceToHost, stream_),
          "download");
    synchronize();
    for (long long i = 0; i < N_; ++i) p[i] = (float)tmp[i];
    return;
  }
  check(cudaMemcpy2DAsync(p, (size_t)g_.r.x * 4, cgx_.p, (size_t)cg_.x * 4, (size_t)g_.r.x * 4,
                          (size_t)g_.r.y * g_.r.z, cudaMemcpyDeviceToHost, stream_),
        "download");
  synchronize();
}

void GridSolver::getSolidSDF(float* s) {
  DArray<float> tmp;
  tmp.alloc(N_, stream_);
  launched(launchTotalSolidSDF(N_, (int)bsdf_.size(), solidIdx_.p, tmp.p, stream_), "total sdf");
  check(cudaMemcpyAsync(s, tmp.p, N_ * 4, cudaMemcpyDeviceToHost, stream_), "download");
  synchronize();
}

void GridSolver::getSolidVel(float* x, float* y, float* z) {
  DArray<float> t[3];
  for (int a = 0; a < 3; ++a) t[a].alloc(F_[a], stream_);
  FaceField f{{t[0].p, t[1].p, t[2].p}};
  launched(launchSolidVelField(g_, solidTable(), f, stream_), "solid vel");
  float* d[3] = {x, y, z};
  for (int a = 0; a < 3; ++a) check(cudaMemcpyAsync(d[a], t[a].p, F_[a] * 4, cudaMemcpyDeviceToHost, stream_), "download");
  synchronize();
}

// GridFluidSolver.cpp:571-591 generateCurFluidSDF on the current domain field
void GridSolver::getFluidSDF(float* out) {
  DArray<float> sdf;
  DArray<unsigned int> fa, fb, cnt;
  sdf.alloc(N_, stream_);
  fa.alloc(N_, stream_);
  fb.alloc(N_, stream_);
  cnt.alloc(2, stream_);
  unsigned int* host = (unsigned int*)pinnedGet(sizeof(unsigned int));
  cudaError_t e = launchFluidSdf(g_.r, dom_[cur()].p, sdf.p, opt_.extrapolation_layers, fa.p, fb.p, cnt.p, host, stream_);
  pinnedPut(host);
  check(e, "fluid sdf");
  check(cudaMemcpyAsync(out, sdf.p, N_ * 4, cudaMemcpyDeviceToHost, stream_), "download");
  synchronize();
}

// GridFluidSolver.cpp:593-613 generateCurFluidDensity: the current fluid
// domain against the total solid.
void GridSolver::getFluidDensity(float* out) {
  DArray<float> d;
  d.alloc(N_, stream_);
  check(launchFluidDensity(g_.r, dom_[cur()].p, nullptr, solidIdx_.p, d.p, stream_), "fluid density");
  check(cudaMemcpyAsync(out, d.p, N_ * 4, cudaMemcpyDeviceToHost, stream_), "download");
  synchronize();
}

// GridFluidSolver.cpp:615-642: into the velocity buffer the step in progress
// writes (the reference's Field1 while its buffer flag is set, else Field2).
void GridSolver::mixVelFieldWithOthers(const float* const other[3], const float* wOther, const float* wFluid) {
  float* b[3] = {vel_[nxt()][0].p, vel_[nxt()][1].p, vel_[nxt()][2].p};
  launched(launchMixFieldWithDensity(g_.r, 1, other, b, wOther, wFluid, stream_), "mix", 3);
  synchronize();
}

// GridFluidSolver.cpp:644-670: G2P from the current velocity buffer.
void GridSolver::transferVelToParticles(const float* pos, long long n, int alg, float* vel) {
  if (n > 0) launched(launchG2PFace(g_, alg, cvel(cur()), pos, n, vel, stream_), "g2p");
  synchronize();
}

void GridSolver::setParticleMirror(float* pos, float* vel, long long capacity) {
  finishMirrorCopy();
  if (!pos && !vel) {
    mirrorPos_ = mirrorVel_ = nullptr;
    mirrorCap_ = 0;
    return;
  }
  if (!copy_.s) check(cudaStreamCreateWithFlags(&copy_.s, cudaStreamNonBlocking), "cudaStreamCreate");
  if (!advDone_) check(cudaEventCreateWithFlags(&advDone_, cudaEventDisableTiming), "cudaEventCreate");
  if (!copyDone_) check(cudaEventCreateWithFlags(&copyDone_, cudaEventDisableTiming), "cudaEventCreate");
  mirrorPos_ = pos;
  mirrorVel_ = vel;
  mirrorCap_ = capacity;
}

// The particle velocities hold their values for the rest of the step once the
// G2P update has run, the positions once the substeps have: each copy to the
// mirror starts on the copy stream at that point, the velocities while the
// substeps run and the positions while the pressure solve runs.  Every writer
// of the particles (setParticles, seedParticles, the next advection) first
// waits for both (finishMirrorCopy), and so does the end of the step.
void GridSolver::startMirrorCopy(bool positions) {
  float* dst = positions ? mirrorPos_ : mirrorVel_;
  if (!dst || P_ <= 0) return;
  if (P_ > mirrorCap_) throw CudaError("particle mirror smaller than the particle count", HFG_ERR_INVALID);
  check(cudaEventRecord(advDone_, stream_), "event");
  check(cudaStreamWaitEvent(copy_.s, advDone_, 0), "wait");
  check(cudaMemcpyAsync(dst, positions ? ppos_.p : pvel_.p, 12 * P_, cudaMemcpyDeviceToHost, copy_.s), "mirror");
  check(cudaEventRecord(copyDone_, copy_.s), "event");
  copyPending_ = true;
}

void GridSolver::finishMirrorCopy() {
  if (!copyPending_) return;
  copyPending_ = false;
  check(cudaEventSynchronize(copyDone_), "mirror copy");
}

void GridSolver::getParticles(float* pos, float* vel) {
  if (P_ > 0) {
    if (pos) check(cudaMemcpyAsync(pos, ppos_.p, 12 * P_, cudaMemcpyDeviceToHost, stream_), "download");
    if (vel) check(cudaMemcpyAsync(vel, pvel_.p, 12 * P_, cudaMemcpyDeviceToHost, stream_), "download");
  }
  synchronize();
}

void GridSolver::getStats(hfg_stats_t* st) {
  std::memset(st, 0, sizeof(*st));
  st->cg_iterations = cgIters_;
  st->divergence_l2 = divL2_;
  st->divergence_max = divMax_;
  st->cg_residual = cgResid_;
  st->cg_rhs_norm = cgBnorm_;
  st->cg_true_residual = cgTrueResid_;
  st->cg_converged = cgConverged_;
  st->substeps = substeps_;
  st->extrapolation_layers = extrapDepth_;
  st->sim_time = time_;
  st->num_particles = P_;
  st->fluid_cells = fluidCells_;
  for (int i = 0; i < 8; ++i) st->stage_ms[i] = stageMs_[i];
  for (int i = 0; i < 3; ++i) st->particle_ms[i] = partMs_[i];
}

}  // namespace hfg
