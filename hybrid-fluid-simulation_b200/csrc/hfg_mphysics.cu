// hfg_mphysics.cu -- the reference's MPhysicsAPI exports (include/mphysics.h)
// on top of the hfg_solver_* C ABI, plus the JSON scene loader
// (SceneManager.cpp:6-47, GridFluidSolver.cpp:48-159).
//
// Scene format: the reference's JSON.  Per HybridSimulator entry only "Name"
// and "GridSolver" are read: DeltaT, GridResolution (+2 ghost cells, origin
// moved out by one spacing, GridFluidSolver.cpp:48-73), SimulationDomain,
// EulerFluidDomain (each box rewrites the whole domain field, as
// generateFluidDomainFromBBoxInvoker does), AdvectionSolver {Type,
// NumOfParticlesPerCell, CFLNumber, MixingCoefficient, PGTransferAlg}.  Mesh
// boundaries ("Boundary", CLD grids) are not part of this library; solids are
// given analytically in GridSolver.Solids: {"Type": "Walls"} (the ghost-cell
// layer), {"Type": "Box", "Center", "Size", "Velocity"} or {"Type": "Sphere",
// "Center", "Radius", "Velocity"}.  Optional: GridSolver.Seed (particle
// seeding stream), GridSolver.PressureSolver {Preconditioner: "identity" |
// "jacobi" | "mg", ToleranceMode: "reference" | "relative", Tolerance,
// MaxIterations}, GridSolver.AdvectScalars.
#include <algorithm>
#include <cctype>
#include <stdexcept>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/hfgrid.h"
#include "../../include/mphysics.h"

namespace {

// ------------------------------------------------------------ minimal JSON --
struct Json {
  enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
  bool b = false;
  double n = 0;
  std::string s;
  std::vector<Json> a;
  std::vector<std::pair<std::string, Json>> o;
  const Json* get(const std::string& k) const {
    if (kind != OBJ) return nullptr;
    for (auto& kv : o)
      if (kv.first == k) return &kv.second;
    return nullptr;
  }
  const Json* path(const std::string& dotted) const {
    const Json* cur = this;
    size_t p = 0;
    while (cur && p <= dotted.size()) {
      size_t q = dotted.find('.', p);
      std::string k = dotted.substr(p, q == std::string::npos ? std::string::npos : q - p);
      cur = cur->get(k);
      if (q == std::string::npos) break;
      p = q + 1;
    }
    return cur;
  }
  double num(const std::string& dotted, double dflt) const {
    const Json* j = path(dotted);
    if (!j) return dflt;
    if (j->kind == NUM) return j->n;
    if (j->kind == BOOL) return j->b ? 1 : 0;
    if (j->kind == STR) return std::atof(j->s.c_str());
    return dflt;
  }
  std::string str(const std::string& dotted, const std::string& dflt) const {
    const Json* j = path(dotted);
    return (j && j->kind == STR) ? j->s : dflt;
  }
};

struct Parser {
  const char* p;
  const char* e;
  void ws() {
    while (p < e && std::isspace((unsigned char)*p)) ++p;
  }
  [[noreturn]] void fail(const char* what) { throw std::runtime_error(std::string("scene JSON: ") + what); }
  Json value() {
    ws();
    if (p >= e) fail("unexpected end");
    Json j;
    if (*p == '{') {
      j.kind = Json::OBJ;
      ++p;
      ws();
      if (p < e && *p == '}') { ++p; return j; }
      for (;;) {
        ws();
        Json k = value();
        if (k.kind != Json::STR) fail("object key must be a string");
        ws();
        if (p >= e || *p != ':') fail("expected ':'");
        ++p;
        j.o.emplace_back(k.s, value());
        ws();
        if (p < e && *p == ',') { ++p; continue; }
        if (p < e && *p == '}') { ++p; break; }
        fail("expected ',' or '}'");
      }
    } else if (*p == '[') {
      j.kind = Json::ARR;
      ++p;
      ws();
      if (p < e && *p == ']') { ++p; return j; }
      for (;;) {
        j.a.push_back(value());
        ws();
        if (p < e && *p == ',') { ++p; continue; }
        if (p < e && *p == ']') { ++p; break; }
        fail("expected ',' or ']'");
      }
    } else if (*p == '"') {
      j.kind = Json::STR;
      ++p;
      while (p < e && *p != '"') {
        if (*p == '\\' && p + 1 < e) {
          ++p;
          char c = *p;
          j.s.push_back(c == 'n' ? '\n' : (c == 't' ? '\t' : c));
        } else {
          j.s.push_back(*p);
        }
        ++p;
      }
      if (p >= e) fail("unterminated string");
      ++p;
    } else if (!std::strncmp(p, "true", 4)) {
      j.kind = Json::BOOL; j.b = true; p += 4;
    } else if (!std::strncmp(p, "false", 5)) {
      j.kind = Json::BOOL; j.b = false; p += 5;
    } else if (!std::strncmp(p, "null", 4)) {
      p += 4;
    } else {
      char* end = nullptr;
      j.kind = Json::NUM;
      j.n = std::strtod(p, &end);
      if (end == p) fail("bad value");
      p = end;
    }
    return j;
  }
};

Json parseJson(const std::string& text) {
  Parser ps{text.data(), text.data() + text.size()};
  Json j = ps.value();
  return j;
}

// ----------------------------------------------------------- scene manager --
struct Sim {
  hfg_solver_t s = nullptr;
  int res[3];
  float origin[3], spacing[3];
  ~Sim() {
    if (s) hfg_solver_destroy(s);
  }
};

std::mutex g_mu;
std::map<std::string, std::unique_ptr<Sim>> g_sims;  // name order, like the reference's std::map
std::string g_err;
bool g_init = false;

void setErr(const std::string& m) { g_err = m; }

void ok(int rc, const char* what) {
  if (rc != HFG_OK) throw std::runtime_error(std::string(what) + ": " + hfg_last_error());
}

void float3v(const Json* j, float out[3], float d0 = 0, float d1 = 0, float d2 = 0) {
  out[0] = d0; out[1] = d1; out[2] = d2;
  if (!j) return;
  out[0] = (float)j->num("x", d0);
  out[1] = (float)j->num("y", d1);
  out[2] = (float)j->num("z", d2);
}

// Signed distance at every cell centre (negative inside the solid).
std::vector<float> solidSdf(const Json& sol, const int r[3], const float o[3], const float h[3]) {
  std::string type = sol.str("Type", "");
  std::vector<float> out((size_t)r[0] * r[1] * r[2]);
  float c[3], sz[3];
  float3v(sol.get("Center"), c);
  float3v(sol.get("Size"), sz);
  double rad = sol.num("Radius", 0);
  for (int z = 0; z < r[2]; ++z)
    for (int y = 0; y < r[1]; ++y)
      for (int x = 0; x < r[0]; ++x) {
        double p[3] = {o[0] + (x + 0.5) * h[0], o[1] + (y + 0.5) * h[1], o[2] + (z + 0.5) * h[2]};
        double d;
        if (type == "Walls") {
          double lo[3] = {o[0] + h[0], o[1] + h[1], o[2] + h[2]};
          double hi[3] = {o[0] + (r[0] - 1) * h[0], o[1] + (r[1] - 1) * h[1], o[2] + (r[2] - 1) * h[2]};
          double in = 1e30, outsq = 0;
          for (int a = 0; a < 3; ++a) {
            double da = std::min(p[a] - lo[a], hi[a] - p[a]);
            in = std::min(in, da);
            if (da < 0) outsq += da * da;
          }
          d = in >= 0 ? in : -std::sqrt(outsq);
        } else if (type == "Sphere") {
          d = std::sqrt((p[0] - c[0]) * (p[0] - c[0]) + (p[1] - c[1]) * (p[1] - c[1]) + (p[2] - c[2]) * (p[2] - c[2])) - rad;
        } else if (type == "Box") {
          double q[3], outsq = 0, mx = -1e30;
          for (int a = 0; a < 3; ++a) {
            q[a] = std::fabs(p[a] - c[a]) - sz[a] / 2;
            if (q[a] > 0) outsq += q[a] * q[a];
            mx = std::max(mx, q[a]);
          }
          d = std::sqrt(outsq) + std::min(mx, 0.0);
        } else {
          throw std::runtime_error("unknown solid type '" + type + "'");
        }
        out[((size_t)z * r[1] + y) * r[0] + x] = (float)d;
      }
  return out;
}

int transferAlg(const std::string& s) {  // GridFluidSolver.cpp:3-25
  if (s == "P2GSUM") return HFG_P2GSUM;
  if (s == "G2PNEAREST") return HFG_G2PNEAREST;
  if (s == "QUADRATIC") return HFG_QUADRATIC;
  if (s == "CUBIC") return HFG_CUBIC;
  return HFG_LINEAR;
}

std::unique_ptr<Sim> buildSim(const Json& gs) {
  auto sim = std::make_unique<Sim>();
  // GridFluidSolver.cpp:48-73
  int res[3] = {(int)gs.num("GridResolution.x", 0), (int)gs.num("GridResolution.y", 0),
                (int)gs.num("GridResolution.z", 0)};
  float st[3], en[3];
  float3v(gs.path("SimulationDomain.Start"), st);
  float3v(gs.path("SimulationDomain.End"), en);
  for (int a = 0; a < 3; ++a) {
    if (res[a] <= 0) throw std::runtime_error("GridResolution must be positive");
    sim->spacing[a] = (en[a] - st[a]) / (float)res[a];
    sim->origin[a] = st[a] - sim->spacing[a];
    sim->res[a] = res[a] + 2;
  }
  float dt = (float)gs.num("DeltaT", 0.033);
  ok(hfg_solver_create(dt, sim->res, sim->origin, sim->spacing, &sim->s), "create solver");
  if (const Json* sols = gs.get("Solids"))
    for (auto& sol : sols->a) {
      std::vector<float> sdf = solidSdf(sol, sim->res, sim->origin, sim->spacing);
      float v[3];
      float3v(sol.get("Velocity"), v);
      ok(hfg_solver_add_solid_boundary(sim->s, sdf.data(), v), "add solid");
    }
  // GridFluidSolver.cpp:75-88
  if (const Json* fd = gs.get("EulerFluidDomain"))
    for (auto& d : fd->a) {
      float mn[3], mx[3];
      float3v(d.path("Range.Start"), mn);
      float3v(d.path("Range.End"), mx);
      ok(hfg_solver_generate_fluid_domain_from_bbox(sim->s, mn, mx), "fluid domain");
    }
  hfg_options_t o;
  hfg_default_options(&o);
  if (const Json* ps = gs.get("PressureSolver")) {
    std::string pc = ps->str("Preconditioner", "identity");
    o.precond = pc == "jacobi" ? HFG_PRECOND_JACOBI : (pc == "mg" ? HFG_PRECOND_MG : HFG_PRECOND_IDENTITY);
    o.tol_mode = ps->str("ToleranceMode", "reference") == "relative" ? HFG_TOL_RELATIVE : HFG_TOL_REFERENCE;
    o.tol = ps->num("Tolerance", o.tol);
    o.max_iter = (long long)ps->num("MaxIterations", (double)o.max_iter);
  }
  o.advect_scalars = (int)gs.num("AdvectScalars", 1);
  ok(hfg_solver_set_options(sim->s, &o), "options");
  // GridFluidSolver.cpp:90-158
  std::string type = gs.str("AdvectionSolver.Type", "SemiLagrangian");
  if (type != "SemiLagrangian") {
    int kind = type == "PIC" ? HFG_ADV_PIC : (type == "FLIP" ? HFG_ADV_FLIP : HFG_ADV_MIX_PIC_FLIP);
    if (type != "PIC" && type != "FLIP" && type != "MixPICAndFLIP")
      throw std::runtime_error("unknown advection solver '" + type + "'");
    ok(hfg_solver_set_advection(sim->s, kind, HFG_RK3, transferAlg(gs.str("AdvectionSolver.PGTransferAlg", "LINEAR")),
                                (float)gs.num("AdvectionSolver.CFLNumber", 1.0),
                                (float)gs.num("AdvectionSolver.MixingCoefficient", 0.1)),
       "advection");
    ok(hfg_solver_seed_particles(sim->s, (int)gs.num("AdvectionSolver.NumOfParticlesPerCell", 8),
                                 (unsigned long long)gs.num("Seed", 0)),
       "seed particles");
  } else {
    ok(hfg_solver_set_advection(sim->s, HFG_ADV_SEMI_LAGRANGIAN, HFG_RK3, HFG_LINEAR, 1.f, 0.f), "advection");
  }
  return sim;
}

Sim* find(const char* name) {
  if (!name) throw std::runtime_error("null simulator name");
  auto it = g_sims.find(name);
  if (it == g_sims.end()) throw std::runtime_error(std::string(name) + " does not exist");  // SceneManager.cpp:61-64
  return it->second.get();
}

template <class F> void guard(F&& f) {
  std::lock_guard<std::mutex> lk(g_mu);
  try {
    g_err.clear();
    f();
  } catch (const std::exception& e) {
    setErr(e.what());
  } catch (...) {
    setErr("unknown error");
  }
}

}  // namespace

namespace MPhysicsAPI {
extern "C" {

MPHYSICS_API const char* mphysics_last_error(void) { return g_err.c_str(); }

MPHYSICS_API void* mphysics_grid_solver(const char* name) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = name ? g_sims.find(name) : g_sims.end();
  return it == g_sims.end() ? nullptr : (void*)it->second->s;
}

// MPhysics.cpp:6-10
MPHYSICS_API void initMPhysics(void) {
  guard([] {
    ok(hfg_init(0), "init");
    g_init = true;
  });
}

// MPhysics.cpp:12-17
MPHYSICS_API void freeMPhysics(void) {
  guard([] {
    g_sims.clear();
    g_init = false;
  });
}

// MPhysics.cpp:19-25: every simulator steps once; the argument is ignored
// (HybridSimulator.cpp:119 uses GridSolver.DeltaT).
MPHYSICS_API void update(float) {
  guard([] {
    for (auto& kv : g_sims) ok(hfg_solver_update(kv.second->s), "update");
  });
}

// SceneManager.cpp:6-47
MPHYSICS_API void loadScene(const char* vSceneFile) {
  guard([&] {
    if (!vSceneFile) throw std::runtime_error("null scene");
    std::string text;
    std::ifstream f(vSceneFile);
    if (f.good()) {
      std::stringstream ss;
      ss << f.rdbuf();
      text = ss.str();
    } else {
      text = vSceneFile;
    }
    Json scene = parseJson(text);
    const Json* sims = scene.get("HybridSimulator");
    if (!sims || sims->kind != Json::ARR) throw std::runtime_error("scene has no HybridSimulator array");
    for (auto& sd : sims->a) {
      std::string name = sd.str("Name", "");
      if (g_sims.count(name)) return;  // SceneManager.cpp:38-43: an existing name stops the load
      const Json* gs = sd.get("GridSolver");
      if (!gs) throw std::runtime_error("simulator '" + name + "' has no GridSolver");
      g_sims[name] = buildSim(*gs);
    }
  });
}

MPHYSICS_API void copyPositionToCPU(const char*, float*) {
  guard([] { throw std::runtime_error("projective particles are not supported by this library"); });
}
MPHYSICS_API void copyVelToCPU(const char*, float*) {
  guard([] { throw std::runtime_error("projective particles are not supported by this library"); });
}

// MPhysics.cpp:183-205
MPHYSICS_API void copyEulerParticlesPosToCPU(const char* name, float* out) {
  guard([&] { ok(hfg_solver_get_particles(find(name)->s, out, nullptr), "particles"); });
}
MPHYSICS_API void copyEulerParticlesVelToCPU(const char* name, float* out) {
  guard([&] { ok(hfg_solver_get_particles(find(name)->s, nullptr, out), "particles"); });
}

// MPhysics.cpp:207-219: the hybrid simulator's fluid SDF grid (HybridSimulator.cpp:175-178).
MPHYSICS_API void copyFluidSDFToCPU(const char* name, float* out) {
  guard([&] {
    Sim* s = find(name);
    ok(hfg_solver_get_fluid_sdf(s->s, out), "fluid sdf");
  });
}

// MPhysics.cpp:220-247: central-difference gradient of the fluid SDF
// (gradientInvoker, FieldMathTool.cu:1130-1150).
MPHYSICS_API void copyFluidSDFGradientToCPU(const char* name, float* gx, float* gy, float* gz) {
  guard([&] {
    Sim* s = find(name);
    size_t n = (size_t)s->res[0] * s->res[1] * s->res[2];
    std::vector<float> f(n);
    ok(hfg_solver_get_fluid_sdf(s->s, f.data()), "fluid sdf");
    const int* r = s->res;
    auto at = [&](int x, int y, int z) {
      x = x < 0 ? 0 : (x >= r[0] ? r[0] - 1 : x);
      y = y < 0 ? 0 : (y >= r[1] ? r[1] - 1 : y);
      z = z < 0 ? 0 : (z >= r[2] ? r[2] - 1 : z);
      return f[((size_t)z * r[1] + y) * r[0] + x];
    };
    for (int z = 0; z < r[2]; ++z)
      for (int y = 0; y < r[1]; ++y)
        for (int x = 0; x < r[0]; ++x) {
          size_t c = ((size_t)z * r[1] + y) * r[0] + x;
          gx[c] = 0.5f * (at(x + 1, y, z) - at(x - 1, y, z)) / s->spacing[0];
          gy[c] = 0.5f * (at(x, y + 1, z) - at(x, y - 1, z)) / s->spacing[1];
          gz[c] = 0.5f * (at(x, y, z + 1) - at(x, y, z - 1)) / s->spacing[2];
        }
  });
}

MPHYSICS_API unsigned int instanceRigidBoundary(const char*, unsigned int, float, float, float, float, float, float,
                                                float, float, float, float, float, float) {
  guard([] { throw std::runtime_error("rigid boundary instances belong to the projective solver (not supported)"); });
  return 0;
}
MPHYSICS_API void transformRigidBoundary(const char*, unsigned int, unsigned int, float, float, float, float, float,
                                         float, float, float, float, float, float, float) {
  guard([] { throw std::runtime_error("rigid boundary instances belong to the projective solver (not supported)"); });
}
MPHYSICS_API unsigned int getParticleSize(const char*) { return 0; }

// MPhysics.cpp:262-266
MPHYSICS_API unsigned int getEulerParticleSize(const char* name) {
  unsigned int n = 0;
  guard([&] { n = (unsigned int)hfg_solver_num_particles(find(name)->s); });
  return n;
}
MPHYSICS_API unsigned int getNeighborDataSize(const char*) { return 0; }
MPHYSICS_API void copyParticleNeighborDataToCPU(const char*, unsigned int*, unsigned int*, unsigned int*) {
  guard([] { throw std::runtime_error("neighbour data belongs to the projective solver (not supported)"); });
}
MPHYSICS_API void getGridInfo(const char*, float& a, float& b, float& c, float& d, float& e, float& f, unsigned int& g,
                              unsigned int& h, unsigned int& i, unsigned int& j, unsigned int& k, unsigned int& l,
                              unsigned int& m, unsigned int& n, unsigned int& o, float& p) {
  a = b = c = d = e = f = p = 0.f;
  g = h = i = j = k = l = m = n = o = 0;
  guard([] { throw std::runtime_error("the projective neighbour grid is not supported"); });
}

// MPhysics.cpp:349-365
MPHYSICS_API void getEulerGridInfo(const char* name, float& ox, float& oy, float& oz, float& hx, float& hy,
                                   float& hz) {
  guard([&] {
    Sim* s = find(name);
    ox = s->origin[0]; oy = s->origin[1]; oz = s->origin[2];
    hx = s->spacing[0]; hy = s->spacing[1]; hz = s->spacing[2];
  });
}
MPHYSICS_API void copyCellDataToCPU(const char*, unsigned int*, unsigned int*) {
  guard([] { throw std::runtime_error("cell data belongs to the projective solver (not supported)"); });
}

}  // extern "C"
}  // namespace MPhysicsAPI
