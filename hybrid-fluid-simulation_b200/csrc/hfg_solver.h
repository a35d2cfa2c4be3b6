// hfg_solver.h -- host orchestration of one grid fluid scene on one GPU.
//
// GridSolver mirrors CGridFluidSolver (MPhysics/GridFluidSolver.h:17-137):
// double-buffered face velocities, colour / fluid-domain fields, solid
// boundaries, the advection solver (semi-Lagrangian, PIC, FLIP or the PIC/FLIP
// mix with its particles), external forces, the pressure projection and the
// velocity extrapolation.  All state is device resident; every stage is a
// kernel on the solver's own stream.
#pragma once
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/hfgrid.h"
#include "hfg_kernels.h"

namespace hfg {

struct CudaError : std::runtime_error {
  int code;
  CudaError(const std::string& m, int c) : std::runtime_error(m), code(c) {}
};

void check(cudaError_t e, const char* what);

// Host-side injection of a device allocation failure, for the failure-path
// tests: once armed with n >= 1, the n-th following DArray allocation fails
// as cudaMalloc would (HFG_ERR_NOMEM) without calling it.  Disarmed: 0.
bool injectedAllocFailure();

// Owning device array.  With a stream the memory comes from the
// stream-ordered allocator and is returned with cudaFreeAsync on the same
// stream, so creating and destroying scenes never synchronises the device
// (other scenes keep running); without one it is plain cudaMalloc / cudaFree.
template <class T> struct DArray {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = nullptr;
  bool async = false;
  DArray() = default;
  DArray(const DArray&) = delete;
  DArray& operator=(const DArray&) = delete;
  ~DArray() { release(); }
  void release() {
    if (p) {
      if (async) cudaFreeAsync(p, s);
      else cudaFree(p);
    }
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count, cudaStream_t stream = nullptr) {
    if (count == n && p) return;
    release();
    if (count == 0) return;
    if (injectedAllocFailure()) throw CudaError("device allocation failed: injected by the test hook", HFG_ERR_NOMEM);
    cudaError_t e;
    if (stream) e = cudaMallocAsync((void**)&p, count * sizeof(T), stream);
    else e = cudaMalloc((void**)&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      throw CudaError(std::string("device allocation failed: ") + cudaGetErrorString(e), HFG_ERR_NOMEM);
    }
    s = stream;
    async = stream != nullptr;
    n = count;
  }
  size_t bytes() const { return n * sizeof(T); }
  void swap(DArray& o) {
    std::swap(p, o.p);
    std::swap(n, o.n);
    std::swap(s, o.s);
    std::swap(async, o.async);
  }
};

// Small pinned host blocks (state read-backs) from a process-wide free list:
// cudaMallocHost / cudaFreeHost may synchronise the device, which a server
// creating scenes while others run must avoid.
void* pinnedGet(size_t bytes);
void pinnedPut(void* p);
// `bytes` from device memory into a pinned block of pinnedGet, by a kernel
// on stream s (no copy engine); valid on the host once s is synchronised.
void readBack(void* host, const void* dev, size_t bytes, cudaStream_t s);

// The solver's stream, destroyed after every member array has been freed
// on it (declared first in GridSolver, so destroyed last).
struct OwnedStream {
  cudaStream_t s = nullptr;
  ~OwnedStream() {
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
};

struct Multigrid;  // hfg_mg.cu

class GridSolver {
 public:
  GridSolver(float dt, Dim3i res, const float origin[3], const float spacing[3]);
  ~GridSolver();

  // ---- setters (GridFluidSolver.cpp:198-244) ----
  void addBoundary(const float* sdfHost, const float vel[3]);
  // type/params as launchAnalyticSdf; the SDF is built on the device
  void addAnalyticBoundary(int type, const double params[6], const float vel[3]);
  void addExternalForce(const float f[3]);
  void setBoundaryVelocity(int index, const float vel[3]);
  void setVelocity(const float* x, const float* y, const float* z);
  void setFluidDomain(const float* d);
  void setColor(const float* x, const float* y, const float* z);
  void fluidDomainFromBBox(const float mn[3], const float mx[3]);
  void setAdvection(int kind, int acc, int alg, float cfl, float mixing);
  void seedParticles(int ppc, unsigned long long seed);
  void setParticles(const float* pos, const float* vel, long long n);
  void setOptions(const hfg_options_t& o);
  void enableTiming(bool on);

  // ---- the step (GridFluidSolver.cpp:336-370) ----
  void update();
  void updateWithoutPressure();
  void solvePressure();

  // ---- getters ----
  void getVelocity(int which, float* x, float* y, float* z);
  void getFluidDomain(float* d);
  void getColor(float* x, float* y, float* z);
  void getMarkers(uint8_t* m);
  void getPressure(float* p);
  void getSolidSDF(float* s);
  void getSolidVel(float* x, float* y, float* z);
  void getFluidSDF(float* out);
  void getFluidDensity(float* out);
  // mixVelFieldWithOthers (device pointers)
  void mixVelFieldWithOthers(const float* const other[3], const float* wOther, const float* wFluid);
  // transferFluidVelField2Particles (device pointers)
  void transferVelToParticles(const float* pos, long long n, int alg, float* vel);
  void getParticles(float* pos, float* vel);
  // host mirror filled by every update (hfg_solver_set_particle_mirror)
  void setParticleMirror(float* pos, float* vel, long long capacity);
  // Reorders the particles (and their carried values) by cell, stable.
  void sortParticles();
  void reserveSortScratch();
  void getStats(hfg_stats_t* st);
  void synchronize();
  float timeCg(int iters);

  const Geom& geom() const { return g_; }
  cudaStream_t stream() const { return stream_; }
  int numBoundaries() const { return (int)bsdf_.size(); }
  long long numParticles() const { return P_; }
  long long launches() const { return launches_; }
  const hfg_options_t& options() const { return opt_; }

  // The step in phases, for a driver that runs the CFL substeps of several
  // scenes in shared launches (BatchStepper): updateWithoutPressure() is
  //   boundaries; advectBegin(); [substeps]; advectEnd()
  // and a true advectBegin() needs the substeps run on substepTask() and then
  // substepsDone(count) before advectEnd().
  void stepBoundaries();
  bool advectBegin();
  SubstepTask substepTask();
  void substepsDone(int count) { substeps_ = count; }
  void advectEnd();

 private:
  void updateBoundarys();
  void computeAdvection();
  FaceQuads beginParticleStep(ConstFaceField vin);
  void advectParticles(const FaceQuads& v);
  void p2gFace(const float* vel, float* const out[3], float* const copy[3], const float add[3], bool doAdd,
               const float add2[3], bool doAdd2);
  void p2gCell(const float* vals, int span, int comp, float* out);
  void computePressure();
  void runCg();
  void cgIteration(int it, float sx, float sy, float sz, int pc);
  void autotuneCg(float sx, float sy, float sz, int pc);
  // Records what f() launches on the solver's stream as an executable graph.
  template <class F> cudaGraphExec_t capture(F&& f);
  void dropGraphs();
  void extrapolate();
  void forcesTerms(float gv[3], bool& doG, float ev[3], bool& doE) const;
  int cur() const { return bufferFlag_ ? 1 : 0; }  // velocity/colour/domain "current" buffer
  int nxt() const { return bufferFlag_ ? 0 : 1; }
  ConstFaceField cvel(int b) const { return ConstFaceField{{vel_[b][0].p, vel_[b][1].p, vel_[b][2].p}}; }
  FaceField mvel(int b) { return FaceField{{vel_[b][0].p, vel_[b][1].p, vel_[b][2].p}}; }
  SolidVelTable solidTable() const;
  void launched(cudaError_t e, const char* what, int count = 1);
  void stageBegin(int i);
  void stageEnd(int i);

  OwnedStream own_;  // first member: outlives every array below
  OwnedStream copy_;  // the particle-mirror copies
  Geom g_;
  Dim3i fr_[3];
  long long N_, F_[3], Ftot_;
  float dt_;
  double time_ = 0.0;
  bool bufferFlag_ = true;
  hfg_options_t opt_;
  cudaStream_t stream_ = nullptr;
  long long launches_ = 0;

  DArray<float> vel_[2][3], prev_[3], color_[2][3], dom_[2], solidVel_[3];
  DArray<uint8_t> solidIdx_, markers_;
  DArray<Code> code_;
  DArray<CgCode> cgc_;
  float* mirrorPos_ = nullptr;
  float* mirrorVel_ = nullptr;
  long long mirrorCap_ = 0;
  cudaEvent_t advDone_ = nullptr, copyDone_ = nullptr;
  bool copyPending_ = false;
  void startMirrorCopy(bool positions);
  void finishMirrorCopy();
  Dim3i cg_;       // pitched grid of the pressure system
  long long NC_ = 0;
  CgMaps maps_;
  DArray<float> cgx_, cgr_, cgp_[2];
  DArray<double> cgx64_;  // the pressure iterate with pressure_fp64
  bool xDouble() const { return opt_.pressure_fp64 != 0; }
  void* xPtr() { return xDouble() ? (void*)cgx64_.p : (void*)cgx_.p; }
  DArray<double> partials_;
  DArray<int> colZ_;  // the CG schedule of the solve (launchCgSchedule)
  DArray<CgState> cgState_;
  CgState* cgHost_ = nullptr;  // pinned
  DArray<SubstepState> subState_;
  SubstepState* subHost_ = nullptr;  // pinned
  int subSlots_ = 4096;
  int cgChunks_ = 0;  // CG chunks the last Jacobi/identity solve needed
  DArray<float2> acc_[3], cacc_;
  DArray<float4> quads_[3];  // corner tables of the advecting velocity (particle substeps)
  FaceQuads vq_{};           // their pointers during an advection
  DArray<uint16_t> dist_;
  DArray<uint8_t> mask_;
  DArray<unsigned int> list_, hist_, offsets_, cursor_;
  unsigned int* extrapHost_ = nullptr;  // pinned

  long long P_ = 0;
  DArray<float> ppos_, pvel_, pv0_, pscalar_, pvector_;
  // the particle sort (option sort_interval, sortParticles)
  long long particleSteps_ = 0;
  DArray<unsigned int> sortKey_[2], sortVal_[2], sortCounts_, sortSums_;
  DArray<float> sortTmp_;

  std::vector<DArray<float>*> bsdf_;
  std::vector<float> bvel_, btrans_;
  // the placement solidIdx_ was last classified at (classifySolids)
  bool classified_ = false;
  std::vector<float> classKey_;
  std::vector<const float*> classSdf_;
  void classifySolids(const BoundarySet& b);
  float ext_[3] = {0, 0, 0};
  float gravity_[3] = {0.f, -9.8f, 0.f};  // ExternalForcesSolver.h:25

  int adv_ = HFG_ADV_SEMI_LAGRANGIAN, acc_rk_ = HFG_RK3, alg_ = HFG_LINEAR;
  float cfl_ = 1.f, mixing_ = 0.1f;
  bool sFlag_ = false, vFlag_ = false, velFlag_ = false;

  // last-step statistics
  long long cgIters_ = 0;
  double cgResid_ = 0, cgBnorm_ = 0;
  int cgConverged_ = 0, substeps_ = 0, extrapDepth_ = 0;
  double divL2_ = 0, divMax_ = 0, cgTrueResid_ = -1.0;
  DArray<double> divScratch_;     // with report_divergence: reduction partials + sum
  DArray<unsigned> divTicket_;
  long long fluidCells_ = -1;

  Multigrid* mg_ = nullptr;
  // one chunk of CG iterations as a CUDA graph, per preconditioner (identity,
  // Jacobi, multigrid): replayed until the device-side state says done
  cudaGraphExec_t cgGraph_[3] = {nullptr, nullptr, nullptr};

  bool timing_ = false;
  // stages 0-7: events 2i, 2i+1; the particle transfers of the advection
  // stage: G2P 16/17, each chunk of substeps 18/19, P2G 20/21
  static constexpr int kEvents = 22;
  cudaEvent_t ev_[kEvents] = {};
  float partMs_[3] = {0.f, 0.f, 0.f};  // G2P, substeps (sum over chunks), P2G
  float stageMs_[8] = {};
};

}  // namespace hfg
