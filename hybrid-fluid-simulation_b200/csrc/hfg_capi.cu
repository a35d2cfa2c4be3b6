// hfg_capi.cu -- the extern "C" boundary of libhfgrid.so (declared in
// include/hfgrid.h).  Exceptions never cross it: every entry point returns a
// status and records the message for hfg_last_error().
#include <atomic>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>

#include "hfg_solver.h"

using namespace hfg;

struct hfg_solver_s {
  std::unique_ptr<GridSolver> s;
};

namespace {
thread_local std::string g_lastError;

int fail(int code, const std::string& msg) {
  g_lastError = msg;
  return code;
}

std::atomic<int> g_allocFailAfter{0};

template <class F> int guarded(F&& f) {
  try {
    return f();
  } catch (const CudaError& e) {
    return fail(e.code, e.what());
  } catch (const std::bad_alloc&) {
    return fail(HFG_ERR_NOMEM, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(HFG_ERR_INVALID, e.what());
  } catch (...) {
    return fail(HFG_ERR_INVALID, "unknown error");
  }
}

}  // namespace

bool hfg::injectedAllocFailure() {
  int n = g_allocFailAfter.load(std::memory_order_relaxed);
  while (n > 0 && !g_allocFailAfter.compare_exchange_weak(n, n - 1)) {
  }
  return n == 1;  // this allocation took the count from 1 to 0
}

namespace {

#define NEED(c, msg) \
  if (!(c)) return fail(HFG_ERR_INVALID, msg)

Dim3i toRes(const int r[3]) { return Dim3i{r[0], r[1], r[2]}; }
bool validRes(const int* r) { return r && r[0] > 0 && r[1] > 0 && r[2] > 0 && (long long)r[0] * r[1] * r[2] < (1LL << 31); }

Geom toGeom(const int r[3], const float* o, const float* h) {
  Geom g;
  g.r = toRes(r);
  g.ox = o ? o[0] : 0.f; g.oy = o ? o[1] : 0.f; g.oz = o ? o[2] : 0.f;
  g.hx = h ? h[0] : 1.f; g.hy = h ? h[1] : 1.f; g.hz = h ? h[2] : 1.f;
  return g;
}
cudaStream_t st(void* s) { return (cudaStream_t)s; }

// Stream-ordered scratch for the operator entry points.
template <class T> struct Scratch {
  T* p = nullptr;
  cudaStream_t s;
  Scratch(size_t n, cudaStream_t s_) : s(s_) {
    if (n && cudaMallocAsync((void**)&p, n * sizeof(T), s) != cudaSuccess) {
      p = nullptr;
      throw CudaError("cudaMallocAsync failed", HFG_ERR_NOMEM);
    }
  }
  ~Scratch() {
    if (p) cudaFreeAsync(p, s);
  }
};
}  // namespace

namespace hfg {
void setLastError(const std::string& msg) { g_lastError = msg; }
}  // namespace hfg

extern "C" {

HFG_API const char* hfg_last_error(void) { return g_lastError.c_str(); }
HFG_API const char* hfg_version(void) { return "hfgrid 0.1 (sm_100a)"; }

HFG_API int hfg_test_inject_alloc_failure(int after) {
  return guarded([&]() -> int {
    NEED(after >= 0, "invalid arguments");
    g_allocFailAfter.store(after);
    return HFG_OK;
  });
}

HFG_API int hfg_tune_save(const char* path) {
  return guarded([&]() -> int {
    NEED(path, "invalid arguments");
    if (!saveTuning(path)) return fail(HFG_ERR_INVALID, std::string("cannot write ") + path);
    return HFG_OK;
  });
}

HFG_API int hfg_tune_load(const char* path, int* entries) {
  return guarded([&]() -> int {
    NEED(path, "invalid arguments");
    const int n = loadTuning(path);
    if (n < 0) return fail(HFG_ERR_INVALID, std::string("cannot read ") + path);
    if (entries) *entries = n;
    return HFG_OK;
  });
}

HFG_API int hfg_selftest_bounded_waits(int wait_ms, int* mbarrier_timed_out, int* grid_barrier_timed_out) {
  return guarded([&]() -> int {
    NEED(wait_ms > 0 && wait_ms <= 10000 && mbarrier_timed_out && grid_barrier_timed_out, "invalid arguments");
    DArray<unsigned> words;
    DArray<int> out;
    words.alloc(3);
    out.alloc(2);
    check(launchSelftestWaits((unsigned long long)wait_ms * 1000000ull, words.p, out.p, nullptr), "self-test");
    int h[2] = {-1, -1};
    check(cudaMemcpy(h, out.p, sizeof(h), cudaMemcpyDeviceToHost), "read");
    *mbarrier_timed_out = h[0];
    *grid_barrier_timed_out = h[1];
    return HFG_OK;
  });
}

HFG_API void hfg_default_options(hfg_options_t* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->precond = HFG_PRECOND_IDENTITY;
  o->tol_mode = HFG_TOL_REFERENCE;
  o->tol = 1e-3;
  o->max_iter = -1;
  o->clamp_mode = 1;
  o->advect_scalars = 1;
  o->extrapolation_layers = 1000;
  o->mg_levels = 0;
  o->mg_smooth = 0;
  o->mg_half = 1;
}

HFG_API int hfg_init(int device) {
  return guarded([&]() -> int {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return fail(HFG_ERR_CUDA, "no CUDA device available");
    NEED(device >= 0 && device < n, "device index out of range");
    check(cudaSetDevice(device), "cudaSetDevice");
    check(cudaFree(nullptr), "context init");
    cudaDeviceProp p;
    check(cudaGetDeviceProperties(&p, device), "cudaGetDeviceProperties");
    if (p.major < 10) return fail(HFG_ERR_UNSUPPORTED, "libhfgrid is built for sm_100a (B200) only");
    return HFG_OK;
  });
}

// ---------------------------------------------------------------- solver --
HFG_API int hfg_solver_create(float dt, const int res[3], const float origin[3], const float spacing[3],
                              hfg_solver_t* out) {
  return guarded([&]() -> int {
    NEED(out && validRes(res), "invalid resolution");
    NEED(spacing == nullptr || (spacing[0] > 0 && spacing[1] > 0 && spacing[2] > 0), "spacing must be positive");
    const float o0[3] = {0, 0, 0}, h1[3] = {1, 1, 1};
    auto* h = new hfg_solver_s();
    try {
      h->s.reset(new GridSolver(dt, toRes(res), origin ? origin : o0, spacing ? spacing : h1));
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return HFG_OK;
  });
}

HFG_API int hfg_solver_destroy(hfg_solver_t s) {
  return guarded([&]() -> int {
    delete s;
    return HFG_OK;
  });
}

#define SOLVER(s) \
  NEED(s && s->s, "null solver handle"); \
  GridSolver& S = *s->s

HFG_API int hfg_solver_add_solid_boundary(hfg_solver_t s, const float* sdf, const float vel[3]) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(sdf, "null sdf");
    S.addBoundary(sdf, vel);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_add_analytic_solid(hfg_solver_t s, int type, const double params[6], const float vel[3]) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(type == HFG_SOLID_WALLS || params, "null parameters");
    S.addAnalyticBoundary(type, params, vel);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_set_boundary_velocity(hfg_solver_t s, int index, const float vel[3]) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(vel, "null velocity");
    S.setBoundaryVelocity(index, vel);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_add_external_force(hfg_solver_t s, const float force[3]) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(force, "null force");
    S.addExternalForce(force);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_set_velocity_field(hfg_solver_t s, const float* x, const float* y, const float* z) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(x && y && z, "null component");
    S.setVelocity(x, y, z);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_set_fluid_domain_field(hfg_solver_t s, const float* d) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(d, "null field");
    S.setFluidDomain(d);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_set_color_field(hfg_solver_t s, const float* x, const float* y, const float* z) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(x && y && z, "null component");
    S.setColor(x, y, z);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_generate_fluid_domain_from_bbox(hfg_solver_t s, const float mn[3], const float mx[3]) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(mn && mx, "null box");
    S.fluidDomainFromBBox(mn, mx);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_set_advection(hfg_solver_t s, int kind, int accuracy, int alg, float cfl, float mixing) {
  return guarded([&]() -> int {
    SOLVER(s);
    S.setAdvection(kind, accuracy, alg, cfl, mixing);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_seed_particles(hfg_solver_t s, int per_cell, unsigned long long seed) {
  return guarded([&]() -> int {
    SOLVER(s);
    S.seedParticles(per_cell, seed);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_set_particles(hfg_solver_t s, const float* pos, const float* vel, long long n) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(n >= 0 && (n == 0 || pos), "invalid particles");
    S.setParticles(pos, vel, n);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_set_options(hfg_solver_t s, const hfg_options_t* o) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(o, "null options");
    S.setOptions(*o);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_enable_timing(hfg_solver_t s, int on) {
  return guarded([&]() -> int {
    SOLVER(s);
    S.enableTiming(on != 0);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_update(hfg_solver_t s) {
  return guarded([&]() -> int {
    SOLVER(s);
    S.update();
    return HFG_OK;
  });
}
HFG_API int hfg_solver_update_steps(hfg_solver_t s, int steps) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(steps >= 0, "negative step count");
    for (int i = 0; i < steps; ++i) S.update();
    return HFG_OK;
  });
}
HFG_API int hfg_solver_update_without_pressure(hfg_solver_t s) {
  return guarded([&]() -> int {
    SOLVER(s);
    S.updateWithoutPressure();
    return HFG_OK;
  });
}
HFG_API int hfg_solver_solve_pressure(hfg_solver_t s) {
  return guarded([&]() -> int {
    SOLVER(s);
    S.solvePressure();
    return HFG_OK;
  });
}
HFG_API int hfg_solver_get_velocity_field(hfg_solver_t s, int which, float* x, float* y, float* z) {
  return guarded([&]() -> int {
    SOLVER(s);
    S.getVelocity(which, x, y, z);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_get_fluid_domain_field(hfg_solver_t s, float* d) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(d, "null output");
    S.getFluidDomain(d);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_get_color_field(hfg_solver_t s, float* x, float* y, float* z) {
  return guarded([&]() -> int {
    SOLVER(s);
    S.getColor(x, y, z);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_get_markers(hfg_solver_t s, uint8_t* m) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(m, "null output");
    S.getMarkers(m);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_get_pressure(hfg_solver_t s, float* p) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(p, "null output");
    S.getPressure(p);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_get_solid_sdf(hfg_solver_t s, float* sdf) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(sdf, "null output");
    S.getSolidSDF(sdf);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_get_solid_vel_field(hfg_solver_t s, float* x, float* y, float* z) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(x && y && z, "null output");
    S.getSolidVel(x, y, z);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_get_fluid_sdf(hfg_solver_t s, float* sdf) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(sdf, "null output");
    S.getFluidSDF(sdf);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_get_fluid_density(hfg_solver_t s, float* out) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(out, "null output");
    S.getFluidDensity(out);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_mix_vel_field_with_others(hfg_solver_t s, const float* vx, const float* vy, const float* vz,
                                                 const float* others_density, const float* fluid_density) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(vx && vy && vz && others_density && fluid_density, "null argument");
    const float* o[3] = {vx, vy, vz};
    S.mixVelFieldWithOthers(o, others_density, fluid_density);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_transfer_vel_to_particles(hfg_solver_t s, const float* pos, long long n, int alg, float* vel) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(n >= 0 && (n == 0 || (pos && vel)) && alg >= 0 && alg <= 4, "invalid arguments");
    S.transferVelToParticles(pos, n, alg, vel);
    return HFG_OK;
  });
}
HFG_API long long hfg_solver_num_particles(hfg_solver_t s) { return (s && s->s) ? s->s->numParticles() : -1; }
HFG_API int hfg_solver_get_particles(hfg_solver_t s, float* pos, float* vel) {
  return guarded([&]() -> int {
    SOLVER(s);
    S.getParticles(pos, vel);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_sort_particles(hfg_solver_t s) {
  return guarded([&]() -> int {
    SOLVER(s);
    S.sortParticles();
    return HFG_OK;
  });
}
HFG_API int hfg_solver_set_particle_mirror(hfg_solver_t s, float* pos, float* vel, long long capacity) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(capacity >= 0 && (capacity == 0 || pos || vel || (!pos && !vel)), "invalid arguments");
    S.setParticleMirror(pos, vel, capacity);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_get_stats(hfg_solver_t s, hfg_stats_t* out) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(out, "null output");
    S.getStats(out);
    return HFG_OK;
  });
}
HFG_API int hfg_solver_get_grid(hfg_solver_t s, int res[3], float origin[3], float spacing[3]) {
  return guarded([&]() -> int {
    SOLVER(s);
    const Geom& g = S.geom();
    if (res) { res[0] = g.r.x; res[1] = g.r.y; res[2] = g.r.z; }
    if (origin) { origin[0] = g.ox; origin[1] = g.oy; origin[2] = g.oz; }
    if (spacing) { spacing[0] = g.hx; spacing[1] = g.hy; spacing[2] = g.hz; }
    return HFG_OK;
  });
}
HFG_API void* hfg_solver_stream(hfg_solver_t s) { return (s && s->s) ? (void*)s->s->stream() : nullptr; }
HFG_API long long hfg_solver_launch_count(hfg_solver_t s) { return (s && s->s) ? s->s->launches() : -1; }
HFG_API int hfg_solver_synchronize(hfg_solver_t s) {
  return guarded([&]() -> int {
    SOLVER(s);
    S.synchronize();
    return HFG_OK;
  });
}

HFG_API int hfg_solver_time_cg(hfg_solver_t s, int iters, float* ms) {
  return guarded([&]() -> int {
    SOLVER(s);
    NEED(ms && iters > 0, "invalid arguments");
    *ms = S.timeCg(iters);
    return HFG_OK;
  });
}

// -------------------------------------------------------------- operators --
HFG_API int hfg_op_markers_from_particles(const int res[3], const float origin[3], const float spacing[3],
                                          const float* solid_sdf, const float* pos, long long n, uint8_t* markers,
                                          void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && solid_sdf && markers && (n == 0 || pos) && n >= 0, "invalid arguments");
    Geom g = toGeom(res, origin, spacing);
    long long N = g.r.size();
    Scratch<uint8_t> idx(N, st(stream));
    check(launchSolidFromSDF(N, solid_sdf, idx.p, st(stream)), "solid");
    check(launchMarkersInit(N, idx.p, markers, st(stream)), "markers");
    check(launchMarkersFromParticles(g, pos, n, markers, st(stream)), "markers");
    return HFG_OK;
  });
}
HFG_API int hfg_op_bin_counts(const int res[3], const float origin[3], const float spacing[3], const float* pos,
                              long long n, unsigned int* counts, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && counts && (n == 0 || pos) && n >= 0, "invalid arguments");
    Geom g = toGeom(res, origin, spacing);
    check(cudaMemsetAsync(counts, 0, sizeof(unsigned int) * g.r.size(), st(stream)), "memset");
    check(launchBinCounts(g, pos, n, counts, st(stream)), "bin counts");
    return HFG_OK;
  });
}
HFG_API int hfg_op_markers_from_sdf(const int res[3], const float* solid_sdf, const float* fluid_sdf,
                                    uint8_t* markers, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && solid_sdf && fluid_sdf && markers, "invalid arguments");
    long long N = toRes(res).size();
    Scratch<uint8_t> idx(N, st(stream));
    check(launchSolidFromSDF(N, solid_sdf, idx.p, st(stream)), "solid");
    check(launchMarkersFromSDF(N, idx.p, fluid_sdf, markers, st(stream)), "markers");
    return HFG_OK;
  });
}

namespace {
void scalesA(const float* h, float dt, float& sx, float& sy, float& sz) {
  sx = dt / (1.0f * h[0] * h[0]); sy = dt / (1.0f * h[1] * h[1]); sz = dt / (1.0f * h[2] * h[2]);
}
}  // namespace

HFG_API int hfg_op_build_matrix_a(const int res[3], const float spacing[3], float dt, const uint8_t* markers,
                                  float* A, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && spacing && markers && A, "invalid arguments");
    Dim3i r = toRes(res);
    Scratch<Code> code(r.size(), st(stream));
    float sx, sy, sz;
    scalesA(spacing, dt, sx, sy, sz);
    check(launchStencilCode(r, r.x, markers, code.p, st(stream)), "code");
    check(launchMatrixA(r, sx, sy, sz, code.p, A, st(stream)), "matrix");
    return HFG_OK;
  });
}
HFG_API int hfg_op_apply_a(const int res[3], const float spacing[3], float dt, const uint8_t* markers,
                           const float* x, float* y, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && spacing && markers && x && y, "invalid arguments");
    Dim3i r = toRes(res);
    Scratch<Code> code(r.size(), st(stream));
    float sx, sy, sz;
    scalesA(spacing, dt, sx, sy, sz);
    check(launchStencilCode(r, r.x, markers, code.p, st(stream)), "code");
    check(launchApplyA(r, sx, sy, sz, code.p, x, y, st(stream)), "apply");
    return HFG_OK;
  });
}
HFG_API int hfg_op_build_rhs(const int res[3], const float spacing[3], const float* vx, const float* vy,
                             const float* vz, const float* svx, const float* svy, const float* svz,
                             const uint8_t* markers, float* b, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && spacing && vx && vy && vz && svx && svy && svz && markers && b, "invalid arguments");
    Geom g = toGeom(res, nullptr, spacing);
    const Dim3i cg = cgDims(g.r);
    long long N = cg.size();
    Scratch<Code> code(N, st(stream));
    Scratch<float> r(N, st(stream)), x(N, st(stream)), p(N, st(stream));
    Scratch<double> part(cgPartialsNeeded(g.r), st(stream));
    Scratch<CgState> cs(1, st(stream));
    CgState init{};
    init.maxIter = 1;
    init.tol = 1e-3;
    check(cudaMemcpyAsync(cs.p, &init, sizeof(init), cudaMemcpyHostToDevice, st(stream)), "state");
    check(launchStencilCode(g.r, cg.x, markers, code.p, st(stream)), "code");
    ConstFaceField v{{vx, vy, vz}}, sv{{svx, svy, svz}};
    SolidVelTable none{};
    check(launchRhsInit(g, v, sv, none, markers, code.p, 1.f, 1.f, 1.f, b, r.p, x.p, false, p.p, part.p, cs.p, 0,
                        st(stream)),
          "rhs");
    check(cudaStreamSynchronize(st(stream)), "sync");
    return HFG_OK;
  });
}

HFG_API int hfg_op_project(const int res[3], const float spacing[3], float dt, const uint8_t* markers, float* vx,
                           float* vy, float* vz, const float* svx, const float* svy, const float* svz, int precond,
                           int tol_mode, double tol, long long max_iter, float* pOut, double* stats, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && spacing && markers && vx && vy && vz && svx && svy && svz, "invalid arguments");
    NEED(precond == HFG_PRECOND_IDENTITY || precond == HFG_PRECOND_JACOBI, "operator projection supports identity/Jacobi");
    NEED(tol_mode == 0 || tol_mode == 1, "invalid tolerance mode");
    Geom g = toGeom(res, nullptr, spacing);
    const Dim3i cg = cgDims(g.r);
    long long N = g.r.size(), NC = cg.size();
    cudaStream_t s = st(stream);
    Scratch<Code> code(NC, s);
    Scratch<CgCode> cgc(NC, s);
    Scratch<float> r(NC, s), x(NC, s), p0(NC, s), p1(NC, s);
    Scratch<double> part(cgPartialsNeeded(g.r), s);
    Scratch<CgState> cs(1, s);
    CgMaps maps;
    check(makeCgMaps(cg, cgc.p, r.p, x.p, false, p0.p, p1.p, &maps), "tensor maps");
    CgState init{};
    init.maxIter = (int)std::min<long long>(max_iter < 0 ? N : max_iter, 0x7fffffff);
    init.precond = precond == HFG_PRECOND_JACOBI ? 1 : 0;
    init.tolMode = tol_mode;
    init.tol = tol;
    check(cudaMemcpyAsync(cs.p, &init, sizeof(init), cudaMemcpyHostToDevice, s), "state");
    float sx, sy, sz;
    scalesA(spacing, dt, sx, sy, sz);
    check(launchStencilCode(g.r, cg.x, markers, code.p, s, cgc.p), "code");
    ConstFaceField v{{vx, vy, vz}}, sv{{svx, svy, svz}};
    SolidVelTable none{};
    check(launchRhsInit(g, v, sv, none, markers, code.p, sx, sy, sz, nullptr, r.p, x.p, false, p0.p, part.p, cs.p,
                        init.precond, s),
          "rhs");
    // the CG kernels never store at non-fluid cells: both directions start zero
    check(cudaMemsetAsync(p1.p, 0, sizeof(float) * NC, s), "memset");
    CgState host{};
    float* pb[2] = {p0.p, p1.p};
    int it = 0;
    for (;;) {
      for (int k = 0; k < 16; ++k, ++it) {
        const int po = it & 1, pn = (it + 1) & 1;
        check(launchCgDirection(cg, sx, sy, sz, maps.rH, maps.pH[po], maps.codeH, cgc.p, r.p, pb[po], pb[pn], part.p,
                                cs.p, init.precond, s),
              "cg");
        check(launchCgUpdate(cg, sx, sy, sz, maps.pH[pn], maps.rI, maps.xI, maps.codeI, pb[pn], x.p, false, r.p, part.p,
                             cs.p, init.precond, s),
              "cg");
      }
      check(cudaMemcpyAsync(&host, cs.p, sizeof(host), cudaMemcpyDeviceToHost, s), "read state");
      check(cudaStreamSynchronize(s), "sync");
      if (host.done) break;
    }
    if (host.error) return fail(HFG_ERR_TIMEOUT, "pressure CG: a stage load did not complete in time");
    FaceField vv{{vx, vy, vz}};
    check(launchGradient(g, dt / (1.0f * spacing[0]), dt / (1.0f * spacing[1]), dt / (1.0f * spacing[2]), markers,
                         x.p, false, vv, sv, none, s),
          "gradient");
    if (pOut)
      check(cudaMemcpy2DAsync(pOut, (size_t)g.r.x * 4, x.p, (size_t)cg.x * 4, (size_t)g.r.x * 4,
                              (size_t)g.r.y * g.r.z, cudaMemcpyDeviceToDevice, s),
            "copy");
    check(cudaStreamSynchronize(s), "sync");
    if (stats) {
      stats[0] = host.iter;
      stats[1] = std::sqrt(host.rr);
      stats[2] = std::sqrt(host.bb);
    }
    return host.iter >= host.maxIter && host.maxIter > 0 && !(tol_mode == 0 ? std::sqrt(std::sqrt(host.rr)) < tol
                                                                            : std::sqrt(host.rr) < tol * std::sqrt(host.bb))
               ? HFG_ERR_NOT_CONVERGED
               : HFG_OK;
  });
}

namespace {
int extrapolateGrids(int ngrids, const Dim3i* rc, float* const* vals, int layers, cudaStream_t s) {
  long long total = 0, off[3] = {0, 0, 0};
  Dim3i r3[3] = {rc[0], rc[0], rc[0]};
  float* v3[3] = {vals[0], vals[0], vals[0]};
  for (int a = 0; a < ngrids; ++a) { off[a] = total; total += rc[a].size(); r3[a] = rc[a]; v3[a] = vals[a]; }
  for (int a = ngrids; a < 3; ++a) { off[a] = total; r3[a] = Dim3i{1, 1, 0}; }
  Scratch<uint16_t> dist(total, s);
  Scratch<unsigned int> list(total, s), hist(kExtrapHistWords, s), offs(kMaxLayers + 2, s), cur(kMaxLayers + 2, s);
  Scratch<uint8_t> mask(total, s);
  ExtrapScratch sc{dist.p, list.p, hist.p, offs.p, cur.p, mask.p};
  if (layers > kMaxLayers) layers = kMaxLayers;
  if (layers <= 1) return HFG_OK;
  // grids with zero size contribute nothing
  check(launchExtrapDistance(r3, v3, off, layers, sc, s), "extrapolation distance");
  struct User {
    User() { extrapUsers(+1); }
    ~User() { extrapUsers(-1); }
  } user;
  check(launchExtrapLayers(r3, v3, off, sc, layers, s, nullptr), "extrapolation layers");
  unsigned int words[4] = {0, 0, 0, 0};
  check(cudaMemcpyAsync(words, extrapBarWords(sc), sizeof(words), cudaMemcpyDeviceToHost, s), "read");
  check(cudaStreamSynchronize(s), "sync");
  if (words[2] != 0u) return fail(HFG_ERR_TIMEOUT, "extrapolation: a grid barrier timed out");
  return HFG_OK;
}
}  // namespace

HFG_API int hfg_op_extrapolate_fc(const int res[3], float* vx, float* vy, float* vz, int layers, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && vx && vy && vz && layers >= 0, "invalid arguments");
    Dim3i rc[3] = {{res[0] + 1, res[1], res[2]}, {res[0], res[1] + 1, res[2]}, {res[0], res[1], res[2] + 1}};
    float* v[3] = {vx, vy, vz};
    return extrapolateGrids(3, rc, v, layers, st(stream));
  });
}
HFG_API int hfg_op_extrapolate_cc(const int res[3], float* f, int layers, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && f && layers >= 0, "invalid arguments");
    Dim3i rc[1] = {toRes(res)};
    float* v[1] = {f};
    return extrapolateGrids(1, rc, v, layers, st(stream));
  });
}

HFG_API int hfg_op_sample_fc(const int res[3], const float origin[3], const float spacing[3], const float* vx,
                             const float* vy, const float* vz, const float* pos, long long n, float* out,
                             void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && vx && vy && vz && n >= 0 && (n == 0 || (pos && out)), "invalid arguments");
    check(launchSampleFace(toGeom(res, origin, spacing), ConstFaceField{{vx, vy, vz}}, pos, n, out, st(stream)),
          "sample");
    return HFG_OK;
  });
}
HFG_API int hfg_op_sample_cc(const int res[3], const float origin[3], const float spacing[3], const float* f,
                             const float* pos, long long n, float* out, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && f && n >= 0 && (n == 0 || (pos && out)), "invalid arguments");
    check(launchSampleCell(toGeom(res, origin, spacing), f, pos, n, out, st(stream)), "sample");
    return HFG_OK;
  });
}
HFG_API int hfg_op_g2p_fc(const int res[3], const float origin[3], const float spacing[3], const float* vx,
                          const float* vy, const float* vz, const float* pos, long long n, int alg, float* out,
                          void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && vx && vy && vz && n >= 0 && (n == 0 || (pos && out)) && alg >= 0 && alg <= 4,
         "invalid arguments");
    check(launchG2PFace(toGeom(res, origin, spacing), alg, ConstFaceField{{vx, vy, vz}}, pos, n, out, st(stream)),
          "g2p");
    return HFG_OK;
  });
}
HFG_API int hfg_op_g2p_cc(const int res[3], const float origin[3], const float spacing[3], const float* f,
                          const float* pos, long long n, int alg, float* out, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && f && n >= 0 && (n == 0 || (pos && out)) && alg >= 0 && alg <= 4, "invalid arguments");
    if (alg == HFG_P2GSUM) {
      check(cudaMemsetAsync(out, 0, 4 * n, st(stream)), "memset");
      return HFG_OK;
    }
    check(launchG2PCell(toGeom(res, origin, spacing), alg, f, pos, n, out, 1, 0, st(stream)), "g2p");
    return HFG_OK;
  });
}
HFG_API int hfg_op_p2g_fc(const int res[3], const float origin[3], const float spacing[3], const float* pos,
                          const float* vel, long long n, int alg, float* vx, float* vy, float* vz, float* wx,
                          float* wy, float* wz, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && vx && vy && vz && n >= 0 && (n == 0 || (pos && vel)) && alg >= 0 && alg <= 4,
         "invalid arguments");
    Geom g = toGeom(res, origin, spacing);
    cudaStream_t s = st(stream);
    long long F[3] = {(long long)(res[0] + 1) * res[1] * res[2], (long long)res[0] * (res[1] + 1) * res[2],
                      (long long)res[0] * res[1] * (res[2] + 1)};
    Scratch<float2> a0(F[0], s), a1(F[1], s), a2(F[2], s);
    float2* acc[3] = {a0.p, a1.p, a2.p};
    for (int a = 0; a < 3; ++a) check(cudaMemsetAsync(acc[a], 0, 8 * F[a], s), "memset");
    check(launchP2GFace(g, alg, pos, vel, n, acc, s), "p2g");
    float* out[3] = {vx, vy, vz};
    float* w[3] = {wx, wy, wz};
    for (int a = 0; a < 3; ++a) {
      check(launchNormalize(F[a], acc[a], out[a], nullptr, 0.f, 0, 0.f, 0, s), "normalize");
      if (w[a]) check(cudaMemcpy2DAsync(w[a], 4, (const char*)acc[a] + 4, 8, 4, F[a], cudaMemcpyDeviceToDevice, s), "w");
    }
    check(cudaStreamSynchronize(s), "sync");
    return HFG_OK;
  });
}
HFG_API int hfg_op_p2g_cc(const int res[3], const float origin[3], const float spacing[3], const float* pos,
                          const float* val, long long n, int alg, int normalize, float* f, float* w, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && f && n >= 0 && (n == 0 || (pos && val)) && alg >= 0 && alg <= 4, "invalid arguments");
    Geom g = toGeom(res, origin, spacing);
    cudaStream_t s = st(stream);
    long long N = g.r.size();
    Scratch<float2> acc(N, s);
    check(cudaMemsetAsync(acc.p, 0, 8 * N, s), "memset");
    check(launchP2GCell(g, alg, pos, val, 1, 0, n, acc.p, s), "p2g");
    if (normalize) check(launchNormalize(N, acc.p, f, nullptr, 0.f, 0, 0.f, 0, s), "normalize");
    else check(cudaMemcpy2DAsync(f, 4, acc.p, 8, 4, N, cudaMemcpyDeviceToDevice, s), "copy");
    if (w) check(cudaMemcpy2DAsync(w, 4, (const char*)acc.p + 4, 8, 4, N, cudaMemcpyDeviceToDevice, s), "w");
    check(cudaStreamSynchronize(s), "sync");
    return HFG_OK;
  });
}
HFG_API int hfg_op_advect_particles(const int res[3], const float origin[3], const float spacing[3],
                                    const float* vx, const float* vy, const float* vz, float* pos, long long n,
                                    float dt, float cfl, int accuracy, int clamp_mode, int* substeps, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && vx && vy && vz && n >= 0 && (n == 0 || pos) && accuracy >= 0 && accuracy <= 2,
         "invalid arguments");
    Geom g = toGeom(res, origin, spacing);
    cudaStream_t s = st(stream);
    const int slots = 4096;
    Scratch<SubstepState> ss(slots + 1, s);
    Scratch<float> v0(3 * (n > 0 ? n : 1), s);
    check(cudaMemsetAsync(ss.p, 0, sizeof(SubstepState) * (slots + 1), s), "memset");
    Scratch<float4> q0(faceQuadCount(g.r, 0), s), q1(faceQuadCount(g.r, 1), s), q2(faceQuadCount(g.r, 2), s);
    float4* quads[3] = {q0.p, q1.p, q2.p};
    check(launchFaceQuads(g.r, ConstFaceField{{vx, vy, vz}}, quads, s), "face corner tables");
    FaceQuads v = makeFaceQuads(g, q0.p, q1.p, q2.p);
    check(launchSubstepBegin(g, v, pos, v0.p, n, ss.p, s), "substep");
    long long nclamp = clamp_mode == 1 ? std::min<long long>(n, g.r.size()) : n;
    SubstepState host{};
    int slot = 0;
    for (;;) {
      for (int k = 0; k < 4 && slot < slots; ++k, ++slot)
        check(launchSubstep(g, v, pos, v0.p, n, accuracy, dt, cfl, nclamp, ss.p, slot, s), "substep");
      check(cudaMemcpyAsync(&host, ss.p + slot, sizeof(host), cudaMemcpyDeviceToHost, s), "read");
      check(cudaStreamSynchronize(s), "sync");
      if (host.finished) break;
      if (slot >= slots) return fail(HFG_ERR_STATE, "CFL substep limit reached");
    }
    if (substeps) *substeps = host.count;
    return HFG_OK;
  });
}
HFG_API int hfg_op_sl_advect_fc(const int res[3], const float origin[3], const float spacing[3], const float* ix,
                                const float* iy, const float* iz, const float* vx, const float* vy, const float* vz,
                                float dt, int accuracy, float* ox, float* oy, float* oz, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && ix && iy && iz && vx && vy && vz && ox && oy && oz && accuracy >= 0 && accuracy <= 2,
         "invalid arguments");
    const float z3[3] = {0, 0, 0};
    check(launchSLFace(toGeom(res, origin, spacing), accuracy, dt, ConstFaceField{{vx, vy, vz}},
                       ConstFaceField{{ix, iy, iz}}, FaceField{{ox, oy, oz}}, z3, 0, z3, 0, st(stream)),
          "sl");
    return HFG_OK;
  });
}
HFG_API int hfg_op_sl_advect_cc(const int res[3], const float origin[3], const float spacing[3], const float* in,
                                const float* vx, const float* vy, const float* vz, float dt, int accuracy, float* out,
                                void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && in && vx && vy && vz && out && accuracy >= 0 && accuracy <= 2, "invalid arguments");
    const float* i1[1] = {in};
    float* o1[1] = {out};
    check(launchSLCell(toGeom(res, origin, spacing), accuracy, dt, ConstFaceField{{vx, vy, vz}}, i1, o1, 1,
                       st(stream)),
          "sl");
    return HFG_OK;
  });
}
HFG_API int hfg_op_sl_advect_fc_ex(const int res[3], const float origin[3], const float spacing[3], const float* ix,
                                   const float* iy, const float* iz, const float* vx, const float* vy,
                                   const float* vz, float dt, int accuracy, int sampling, float* ox, float* oy,
                                   float* oz, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && ix && iy && iz && vx && vy && vz && ox && oy && oz && accuracy >= 0 && accuracy <= 2 &&
             sampling >= 0 && sampling <= 4,
         "invalid arguments");
    const float z3[3] = {0, 0, 0};
    check(launchSLFace(toGeom(res, origin, spacing), accuracy, dt, ConstFaceField{{vx, vy, vz}},
                       ConstFaceField{{ix, iy, iz}}, FaceField{{ox, oy, oz}}, z3, 0, z3, 0, st(stream), sampling),
          "sl");
    return HFG_OK;
  });
}
HFG_API int hfg_op_sl_advect_cc_ex(const int res[3], const float origin[3], const float spacing[3], const float* in,
                                   const float* vx, const float* vy, const float* vz, float dt, int accuracy,
                                   int sampling, float* out, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && in && vx && vy && vz && out && accuracy >= 0 && accuracy <= 2 && sampling >= 0 &&
             sampling <= 4,
         "invalid arguments");
    const float* i1[1] = {in};
    float* o1[1] = {out};
    check(launchSLCell(toGeom(res, origin, spacing), accuracy, dt, ConstFaceField{{vx, vy, vz}}, i1, o1, 1,
                       st(stream), sampling),
          "sl");
    return HFG_OK;
  });
}
HFG_API int hfg_op_sample_cc_ex(const int res[3], const float origin[3], const float spacing[3], const float* f,
                                const float* pos, long long n, int sampling, float* out, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && f && n >= 0 && (n == 0 || (pos && out)) && sampling >= 0 && sampling <= 4,
         "invalid arguments");
    check(launchSampleAlg(toGeom(res, origin, spacing), 0, ConstFaceField{{f, nullptr, nullptr}}, pos, n, sampling,
                          out, st(stream)),
          "sample");
    return HFG_OK;
  });
}
HFG_API int hfg_op_sample_fc_ex(const int res[3], const float origin[3], const float spacing[3], const float* vx,
                                const float* vy, const float* vz, const float* pos, long long n, int sampling,
                                float* out, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && vx && vy && vz && n >= 0 && (n == 0 || (pos && out)) && sampling >= 0 && sampling <= 4,
         "invalid arguments");
    check(launchSampleAlg(toGeom(res, origin, spacing), 1, ConstFaceField{{vx, vy, vz}}, pos, n, sampling, out,
                          st(stream)),
          "sample");
    return HFG_OK;
  });
}
HFG_API int hfg_op_build_fluid_density(const int res[3], const float* domain, const float* solid_sdf, float* out,
                                       void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && domain && solid_sdf && out, "invalid arguments");
    check(launchFluidDensity(toRes(res), domain, solid_sdf, nullptr, out, st(stream)), "fluid density");
    return HFG_OK;
  });
}
HFG_API int hfg_op_mix_field_with_density_cc(long long n, const float* a, float* b, const float* wa, const float* wb,
                                             void* stream) {
  return guarded([&]() -> int {
    NEED(n >= 0 && (n == 0 || (a && b && wa && wb)), "invalid arguments");
    if (n == 0) return HFG_OK;
    const float* A[3] = {a, nullptr, nullptr};
    float* B[3] = {b, nullptr, nullptr};
    Dim3i r{(int)std::min<long long>(n, 1LL << 30), 1, 1};
    NEED(n < (1LL << 30), "too many entries");
    check(launchMixFieldWithDensity(r, 0, A, B, wa, wb, st(stream)), "mix");
    return HFG_OK;
  });
}
HFG_API int hfg_op_mix_field_with_density_fc(const int res[3], const float* ax, const float* ay, const float* az,
                                             float* bx, float* by, float* bz, const float* wa, const float* wb,
                                             void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && ax && ay && az && bx && by && bz && wa && wb, "invalid arguments");
    const float* A[3] = {ax, ay, az};
    float* B[3] = {bx, by, bz};
    check(launchMixFieldWithDensity(toRes(res), 1, A, B, wa, wb, st(stream)), "mix");
    return HFG_OK;
  });
}
HFG_API int hfg_op_mix_particle_vel_pic_flip(const float* pic, const float* flip, const float* dist, long long n,
                                             float cell, float g_rate, float gf_rate, float f_rate, float p_rate,
                                             float* predict, void* stream) {
  return guarded([&]() -> int {
    NEED(n >= 0 && (n == 0 || (pic && flip && dist && predict)), "invalid arguments");
    check(launchMixParticleVel(pic, flip, dist, n, cell, g_rate, gf_rate, f_rate, p_rate, predict, st(stream)),
          "mix");
    return HFG_OK;
  });
}
HFG_API int hfg_op_build_fluid_sdf(const int res[3], const float* domain, float* sdf, int layers, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && domain && sdf && layers >= 1 && layers <= 100000, "invalid arguments");
    Dim3i r = toRes(res);
    cudaStream_t s = st(stream);
    Scratch<unsigned int> fa(r.size(), s), fb(r.size(), s), cnt(2, s);
    unsigned int* host = nullptr;
    check(cudaMallocHost((void**)&host, sizeof(unsigned int)), "cudaMallocHost");
    cudaError_t e = launchFluidSdf(r, domain, sdf, layers, fa.p, fb.p, cnt.p, host, s);
    cudaFreeHost(host);
    check(e, "fluid sdf");
    check(cudaStreamSynchronize(s), "sync");
    return HFG_OK;
  });
}
namespace {
int fluidSideSdf(const int res[3], const float* density, const float* solid_sdf, float* out, int distance,
                 bool outside, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && density && solid_sdf && out && distance >= 0 && distance <= 100000, "invalid arguments");
    Dim3i r = toRes(res);
    cudaStream_t s = st(stream);
    Scratch<unsigned int> fa(r.size(), s), fb(r.size(), s), cnt(2, s);
    unsigned int* host = nullptr;
    check(cudaMallocHost((void**)&host, sizeof(unsigned int)), "cudaMallocHost");
    cudaError_t e = launchFluidSideSdf(r, density, solid_sdf, outside, distance, out, fa.p, fb.p, cnt.p, host, s);
    cudaFreeHost(host);
    check(e, outside ? "fluid outside sdf" : "fluid inside sdf");
    check(cudaStreamSynchronize(s), "sync");
    return HFG_OK;
  });
}
}  // namespace
HFG_API int hfg_op_build_fluid_outside_sdf(const int res[3], const float* density, const float* solid_sdf, float* out,
                                           int distance, void* stream) {
  return fluidSideSdf(res, density, solid_sdf, out, distance, true, stream);
}
HFG_API int hfg_op_build_fluid_inside_sdf(const int res[3], const float* density, const float* solid_sdf, float* out,
                                          int distance, void* stream) {
  return fluidSideSdf(res, density, solid_sdf, out, distance, false, stream);
}
HFG_API int hfg_op_build_mixed_fluid_outside_sdf(const int res[3], const float* grid_density,
                                                 const float* mixed_density, const float* grid_outside_sdf,
                                                 float* out, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && grid_density && mixed_density && grid_outside_sdf && out, "invalid arguments");
    check(launchMixedOutsideSdf(toRes(res), grid_density, mixed_density, grid_outside_sdf, out, st(stream)),
          "mixed outside sdf");
    return HFG_OK;
  });
}
HFG_API int hfg_op_fluid_domain_from_bbox(const int res[3], const float origin[3], const float spacing[3],
                                          const float mn[3], const float mx[3], float* out, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && mn && mx && out, "invalid arguments");
    check(launchFluidDomainFromBBox(toGeom(res, origin, spacing), mn, mx, out, st(stream)), "bbox");
    return HFG_OK;
  });
}
HFG_API int hfg_op_seed_particles(const int res[3], const float origin[3], const float spacing[3],
                                  const float* fluid_sdf, const float* solid_sdf, int per_cell,
                                  unsigned long long seed, float* pos, long long capacity, long long* count,
                                  void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && fluid_sdf && per_cell > 0, "invalid arguments");
    Geom g = toGeom(res, origin, spacing);
    cudaStream_t s = st(stream);
    long long N = g.r.size();
    const int cpb = 4096;
    int nb = (int)((N + cpb - 1) / cpb);
    Scratch<unsigned int> counts(nb, s);
    Scratch<unsigned long long> total(1, s);
    Scratch<uint8_t> idx(solid_sdf ? N : 0, s);
    if (solid_sdf) check(launchSolidFromSDF(N, solid_sdf, idx.p, s), "solid");
    check(launchSeedCount(g.r, fluid_sdf, idx.p, counts.p, cpb, s), "seed");
    check(launchSeedScan(counts.p, nb, total.p, s), "seed");
    unsigned long long nf = 0;
    check(cudaMemcpyAsync(&nf, total.p, 8, cudaMemcpyDeviceToHost, s), "read");
    check(cudaStreamSynchronize(s), "sync");
    long long n = (long long)nf * per_cell;
    if (count) *count = n;
    if (pos) {
      NEED(capacity >= n, "particle buffer too small");
      check(launchSeedWrite(g, fluid_sdf, idx.p, counts.p, cpb, per_cell, seed, pos, s), "seed");
      check(cudaStreamSynchronize(s), "sync");
    }
    return HFG_OK;
  });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// P2G onto the face grids with no device allocation (hfg_op_p2g_fc_static).
//
// hfg_op_p2g_fc takes its accumulators from the stream-ordered allocator on
// every call.  Some callers may not allocate at call time: a host that runs
// the transfer inside a fixed-memory real-time loop, or one whose own
// allocator reserves the whole device and forbids other allocations.  For
// them the accumulators live in one array that is part of the library image,
// sized at build time.
namespace {

// Total faces (x + y + z face grids together) one call may cover: 2^20 float2
// accumulators, 8 MiB of device memory (a 64 x 64 x 64 grid has 798,720 faces).
constexpr long long kStaticP2GFaces = 1LL << 20;
static __device__ __align__(256) float2 g_p2gStaticAcc[kStaticP2GFaces];

// Address of the array on the current device.  In host code the symbol
// g_p2gStaticAcc is a host-side stand-in, so the device address is looked up
// on every call (a host-side table lookup once the module is loaded): an
// address kept from an earlier call would go stale if the host reset the
// device or recreated its primary context, which reloads the module.
float2* staticP2GAccumulators() {
  float2* p = nullptr;
  check(cudaGetSymbolAddress((void**)&p, g_p2gStaticAcc), "cudaGetSymbolAddress");
  return p;
}

}  // namespace

extern "C" {

HFG_API int hfg_op_p2g_fc_static(const int res[3], const float origin[3], const float spacing[3], const float* pos,
                                 const float* vel, long long n, int alg, float* vx, float* vy, float* vz, float* wx,
                                 float* wy, float* wz, void* stream) {
  return guarded([&]() -> int {
    NEED(validRes(res) && vx && vy && vz && n >= 0 && (n == 0 || (pos && vel)) && alg >= 0 && alg <= 4,
         "invalid arguments");
    long long F[3] = {(long long)(res[0] + 1) * res[1] * res[2], (long long)res[0] * (res[1] + 1) * res[2],
                      (long long)res[0] * res[1] * (res[2] + 1)};
    if (F[0] + F[1] + F[2] > kStaticP2GFaces)
      return fail(HFG_ERR_INVALID, "hfg_op_p2g_fc_static: grid has " + std::to_string(F[0] + F[1] + F[2]) +
                                       " faces, above the fixed limit of " + std::to_string(kStaticP2GFaces) +
                                       " (use hfg_op_p2g_fc for larger grids)");
    Geom g = toGeom(res, origin, spacing);
    cudaStream_t s = st(stream);
    float2* base = staticP2GAccumulators();
    float2* acc[3] = {base, base + F[0], base + F[0] + F[1]};
    // the scatter accumulates with atomics: every call zeroes the part it uses
    check(cudaMemsetAsync(base, 0, sizeof(float2) * (F[0] + F[1] + F[2]), s), "memset");
    check(launchP2GFace(g, alg, pos, vel, n, acc, s), "p2g");
    float* out[3] = {vx, vy, vz};
    float* w[3] = {wx, wy, wz};
    for (int a = 0; a < 3; ++a) {
      check(launchNormalize(F[a], acc[a], out[a], nullptr, 0.f, 0, 0.f, 0, s), "normalize");
      if (w[a]) check(cudaMemcpy2DAsync(w[a], 4, (const char*)acc[a] + 4, 8, 4, F[a], cudaMemcpyDeviceToDevice, s), "w");
    }
    check(cudaStreamSynchronize(s), "sync");
    return HFG_OK;
  });
}

}  // extern "C"
