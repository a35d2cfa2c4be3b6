// driver.cu -- a C ABI over the reference's own CGridFluidSolver, built from
// the reference's CUDA sources (unmodified, compiled where they lie) by
// oracle/refgpu/build.sh.  Test infrastructure: the GPU parity tests step it
// beside libhfgrid on the same seeded particles, and the reference arm of
// the bench times it.  It is never part of the product path.
//
// What it drives (reference files):
//   CGridFluidSolver(dt, res, origin, spacing)        GridFluidSolver.cpp:32-41, 161-196
//   addSolidBoundary / setFluidDomainField             GridFluidSolver.cpp:203-206, 214-218
//   generateFluidDomainFromBBox                        GridFluidSolver.cpp:551-555 (EulerSolverTool.cu:989-1013)
//   CMixPICAndFLIP::resizeMixPICAndFLIP               MixPICAndFLIP.cpp:30-60 (seeding EulerParticles.cpp:140-179)
//   CEulerParticles::setParticlesPos                  EulerParticles.cpp:125-128
//   setAdvectionSolver                                 GridFluidSolver.cpp:231-234
//   update()                                           GridFluidSolver.cpp:336-370
//   the pressure solve: CCuMatrixFreePCG::solvePCGInvDia, cap = N cells and
//   threshold 1e-3 as PressureSolver.cpp:80-82 and CuMatrixFreePCG.h:27-28 set them
//
// The reference's seeding draws positions with rand() after srand(time(0));
// rg_set_mix_pic_flip replaces them with the caller's (same count, checked),
// so both solvers start from identical particles.  To read the CG iteration
// count the driver wraps the solver's A*x callback with a counter; to bound a
// solve that cannot reach the absolute threshold in FP32 it can lower the
// iteration cap through CCuMatrixFreePCG::setIterationNum.  Both reach the
// PCG object through the pressure solver's private member, which is why the
// reference headers are included with private access opened below; no
// arithmetic of the reference is changed.  Built with -DDOUBLE_REAL (the
// reference's own switch) the whole step runs in FP64, and every array of
// this ABI is double.
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "Common.h"
#define private public
#include "GridFluidSolver.h"
#undef private
#include "CudaContextManager.h"

namespace {

thread_local std::string g_err;

struct RefScene {
  std::unique_ptr<CGridFluidSolver> solver;
  Vector3i res;
  Vector3 origin, spacing;
  std::shared_ptr<CMixPICAndFLIP> mix;
};

// A*x calls of the pressure solves since the counter was last read: one for
// the initial residual and one per CG iteration.
MatrixVecCGProd g_ax = nullptr;
unsigned long long g_axCalls = 0;
void countingAx(const CCuDenseVector& v, CCuDenseVector& out, void* user) {
  ++g_axCalls;
  g_ax(v, out, user);
}

template <class F> int guarded(F&& f) {
  try {
    f();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      g_err = std::string("CUDA error: ") + cudaGetErrorString(e);
      return 2;
    }
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

RefScene* scene(void* h) {
  if (!h) throw std::invalid_argument("null scene handle");
  return static_cast<RefScene*>(h);
}

template <class T> void toHost(const thrust::device_vector<T>& d, T* out) {
  cudaError_t e = cudaMemcpy(out, thrust::raw_pointer_cast(d.data()), d.size() * sizeof(T), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) throw std::runtime_error(std::string("read-back failed: ") + cudaGetErrorString(e));
}

CCuMatrixFreePCG* pcgOf(RefScene* s) {
  CCuMatrixFreePCG* p = s->solver->getPressureSolver()->m_MartixFreeCGSolver.get();
  if (!p) throw std::runtime_error("pressure solver has no PCG");
  return p;
}

}  // namespace

extern "C" {

const char* rg_last_error() { return g_err.c_str(); }

// sizeof(Real) of this build: 4, or 8 when built with -DDOUBLE_REAL.  Every
// array argument below is of that type.
int rg_real_size() { return (int)sizeof(Real); }

int rg_init() {
  return guarded([] {
    if (!CCudaContextManager::getInstance().getIsInit()) CCudaContextManager::getInstance().initCudaContext();
  });
}

void* rg_create(float dt, const int res[3], const float origin[3], const float spacing[3]) {
  RefScene* out = nullptr;
  int rc = guarded([&] {
    auto s = std::make_unique<RefScene>();
    s->res = Vector3i(res[0], res[1], res[2]);
    s->origin = Vector3(origin[0], origin[1], origin[2]);
    s->spacing = Vector3(spacing[0], spacing[1], spacing[2]);
    s->solver = std::make_unique<CGridFluidSolver>(dt, s->res, s->origin, s->spacing);
    CCuMatrixFreePCG* p = pcgOf(s.get());
    g_ax = p->m_AxCGProdFunc;
    p->m_AxCGProdFunc = countingAx;
    out = s.release();
  });
  return rc == 0 ? out : nullptr;
}

void rg_destroy(void* h) { delete static_cast<RefScene*>(h); }

int rg_add_solid(void* h, const Real* sdf) {
  return guarded([&] {
    RefScene* s = scene(h);
    CCellCenteredScalarField f(s->res, s->origin, s->spacing, const_cast<Real*>(sdf));
    s->solver->addSolidBoundary(f);
  });
}

// A solid moving at a constant velocity: CBoundarys::addBoundary(sdf, vel)
// (Boundary.cpp:92-113; each update moves it by -dt vel and resamples its
// SDF, Boundary.cpp:115-136).  GridFluidSolver::addSolidBoundary passes no
// velocity, so the driver reaches the boundaries directly.
int rg_add_moving_solid(void* h, const Real* sdf, const float vel[3]) {
  return guarded([&] {
    RefScene* s = scene(h);
    CCellCenteredScalarField f(s->res, s->origin, s->spacing, const_cast<Real*>(sdf));
    s->solver->m_Boundarys.addBoundary(f, Vector3(vel[0], vel[1], vel[2]));
  });
}

int rg_set_fluid_domain(void* h, const Real* dom) {
  return guarded([&] {
    RefScene* s = scene(h);
    CCellCenteredScalarField f(s->res, s->origin, s->spacing, const_cast<Real*>(dom));
    s->solver->setFluidDomainField(f);
  });
}

int rg_fluid_domain_bbox(void* h, const float mn[3], const float mx[3]) {
  return guarded([&] {
    scene(h)->solver->generateFluidDomainFromBBox(Vector3(mn[0], mn[1], mn[2]), Vector3(mx[0], mx[1], mx[2]));
  });
}

// Assembles the total boundary SDF, marker and velocity fields from the
// boundaries added so far (CBoundarys::updateBoundarys with dt = 0: no
// motion), as the first update() would.  The reference seeds its particles
// from the total SDF (EulerParticlesTool.cu:5-25) when the advection solver
// is built, which in its own setup (HybridSimulator.cpp:111-115) happens
// before any update, so the total SDF is still all zeros there and cells
// inside solids are seeded too; calling this first makes the seeding skip
// them, which is the rule libhfgrid seeds by.
int rg_update_boundaries(void* h) {
  return guarded([&] { scene(h)->solver->m_Boundarys.updateBoundarys(0); });
}

// PIC/FLIP mix with linear transfers, seeded by the reference from the fluid
// domain and the total solid SDF; returns the reference's particle count, or
// -1 on error.  When pos is given its n particles replace the seeded ones,
// and n must equal that count.
long long rg_set_mix_pic_flip(void* h, int ppc, float cfl, float mixing, const Real* pos, long long n) {
  long long count = -1;
  int rc = guarded([&] {
    RefScene* s = scene(h);
    auto mix = std::make_shared<CMixPICAndFLIP>();
    mix->resizeMixPICAndFLIP(s->solver->getFluidDomainField(), s->solver->getSolidSDFField(), (UInt)ppc, s->res,
                             s->origin, s->spacing, cfl, mixing, EPGTransferAlgorithm::LINEAR);
    count = (long long)mix->getEulerParticles().getNumOfParticles();
    if (pos) {
      if (n != count)
        throw std::invalid_argument("particle count " + std::to_string(n) + " differs from the reference's seeding (" +
                                    std::to_string(count) + ")");
      const_cast<CEulerParticles&>(mix->getEulerParticles()).setParticlesPos(pos);
    }
    s->mix = mix;
    s->solver->setAdvectionSolver(mix);
  });
  return rc == 0 ? count : -1;
}

int rg_set_cg_iteration_cap(void* h, unsigned cap) {
  return guarded([&] { pcgOf(scene(h))->setIterationNum(cap); });
}

int rg_update(void* h) {
  return guarded([&] { scene(h)->solver->update(); });
}

// A*x calls since the last read (0 when no solve ran), and reset.
unsigned long long rg_take_ax_calls() {
  unsigned long long c = g_axCalls;
  g_axCalls = 0;
  return c;
}

int rg_velocity(void* h, Real* x, Real* y, Real* z) {
  return guarded([&] {
    const CFaceCenteredVectorField& v = scene(h)->solver->getVelocityField();
    toHost(v.getConstGridDataX(), x);
    toHost(v.getConstGridDataY(), y);
    toHost(v.getConstGridDataZ(), z);
  });
}

long long rg_num_particles(void* h) {
  RefScene* s = static_cast<RefScene*>(h);
  return (s && s->mix) ? (long long)s->mix->getEulerParticles().getNumOfParticles() : 0;
}

int rg_particles(void* h, Real* pos, Real* vel) {
  return guarded([&] {
    RefScene* s = scene(h);
    if (!s->mix) throw std::runtime_error("no particles: the advection solver is not the PIC/FLIP mix");
    if (pos) toHost(s->mix->getEulerParticles().getParticlesPos(), pos);
    if (vel) toHost(s->mix->getEulerParticles().getParticlesVel(), vel);
  });
}

int rg_markers(void* h, Real* m) {
  return guarded([&] { toHost(scene(h)->solver->getPressureSolver()->getMarkers().getConstGridData(), m); });
}

int rg_pressure(void* h, Real* p) {
  return guarded([&] { toHost(scene(h)->solver->getPressureSolver()->getConstVectorx().getConstVectorValue(), p); });
}

int rg_synchronize() {
  return guarded([] {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) throw std::runtime_error(std::string("synchronize: ") + cudaGetErrorString(e));
  });
}

}  // extern "C"
