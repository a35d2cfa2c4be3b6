// hfg_server.cu -- continuous-batching scene server (hfg_server_* in
// include/hfgrid.h).
//
// The reference steps its simulators one after another on the default stream
// (MPhysics.cpp:19-25).  Here each admitted request gets a worker thread that
// owns its GridSolver -- grids and particles resident on the device for all of
// the request's steps -- on the solver's own stream, so the kernels of
// different scenes overlap on the GPU.  Admission is by slot and by a device
// byte budget; scene memory comes from the stream-ordered allocator, so a
// scene arriving or leaving never synchronises the device under the others.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "hfg_solver.h"

using namespace hfg;

namespace hfg {
void setLastError(const std::string& msg);  // hfg_capi.cu
}

namespace {
using Clock = std::chrono::steady_clock;

// The dam break of a scene description: walls, its spheres, the fluid box,
// the PIC/FLIP mix and seeded particles.
std::unique_ptr<GridSolver> buildScene(const hfg_scene_desc_t& d) {
  Dim3i res{d.res[0], d.res[1], d.res[2]};
  const float origin[3] = {0.f, 0.f, 0.f};
  const float h[3] = {1.0f / d.res[0], 1.0f / d.res[1], 1.0f / d.res[2]};
  std::unique_ptr<GridSolver> sp(new GridSolver(d.dt, res, origin, h));
  GridSolver& s = *sp;
  const float still[3] = {0.f, 0.f, 0.f};
  s.addAnalyticBoundary(0, nullptr, still);
  for (int i = 0; i < d.n_spheres; ++i) {
    const double p[6] = {d.spheres[i][0], d.spheres[i][1], d.spheres[i][2], d.spheres[i][3], 0.0, 0.0};
    s.addAnalyticBoundary(1, p, still);
  }
  const float lo[3] = {0.f, 0.f, 0.f};
  s.fluidDomainFromBBox(lo, d.fluid_max);
  s.setAdvection(HFG_ADV_MIX_PIC_FLIP, HFG_RK3, HFG_LINEAR, d.cfl, d.mixing);
  s.setOptions(d.options);
  s.seedParticles(d.per_cell, d.seed);
  return sp;
}

double msBetween(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  double pos = q * (double)(v.size() - 1);
  size_t i = (size_t)pos;
  double f = pos - (double)i;
  return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

// Device bytes of one resident scene: the GridSolver allocations (face
// velocities x2 + FLIP copy, colour / domain double buffers, markers, solid
// index, stencil code and CG vectors on the pitched grid, P2G accumulators,
// face corner tables, extrapolation scratch, boundary SDFs, particles) plus
// the multigrid levels.
long long sceneBytes(const int res[3], long long particles, int boundaries, int precond, bool sorting = false) {
  const long long nx = res[0], ny = res[1], nz = res[2];
  const long long N = nx * ny * nz;
  const long long F = (nx + 1) * ny * nz + nx * (ny + 1) * nz + nx * ny * (nz + 1);
  const long long NC = ((nx + 15) & ~15LL) * ny * nz;
  long long b = 0;
  b += F * 4 * 3;              // velocity x2 + previous
  b += N * 4 * (6 + 2);        // colour x2 x3, domain x2
  b += N * 2;                  // markers, solid index
  b += NC * (2 + 1 + 4 * 4);   // code, CG code, x, r, p x2
  b += F * 8 + N * 8;          // P2G accumulators (faces, cells)
  b += ((nx + 2) * (ny + 1) * (nz + 2) + (nx + 1) * (ny + 2) * (nz + 2) + (nx + 1) * (ny + 1) * (nz + 3)) * 16;  // corner tables
  b += F * (2 + 4 + 1);        // extrapolation distance, list, neighbour masks
  b += N * 4 * (long long)boundaries;
  b += particles * (4 * 3 * 4 + 4);  // pos, vel, v0, vector scalars, scalar
  if (precond == HFG_PRECOND_MG) b += NC * 4 * 4 + N * 2;  // level-0 z x2, p x2; coarse levels
  if (sorting) b += particles * (16 + 12) + particles / 16;  // radix keys and values x2, gather buffer, digit counts
  b += 64ll << 20;             // partials, state, allocator granularity
  return b;
}

long long particlesBound(const hfg_scene_desc_t& d) {
  long long n = 1;
  for (int a = 0; a < 3; ++a) {
    // cells of the unit cube whose centre lies below fluid_max
    double h = 1.0 / d.res[a];
    long long k = (long long)std::ceil(d.fluid_max[a] / h - 0.5);
    n *= std::max(0LL, std::min<long long>(k, d.res[a]));
  }
  return n * std::max(0, d.per_cell);
}

bool validDesc(const hfg_scene_desc_t& d, std::string& why) {
  for (int a = 0; a < 3; ++a)
    if (d.res[a] < 4 || d.res[a] > 4096) return why = "res must be within [4, 4096]", false;
  if ((long long)d.res[0] * d.res[1] * d.res[2] >= (1LL << 31)) return why = "grid too large", false;
  if (!(d.dt > 0.f)) return why = "dt must be positive", false;
  if (d.n_spheres < 0 || d.n_spheres > 4) return why = "at most 4 spheres", false;
  if (d.per_cell <= 0) return why = "per_cell must be positive", false;
  if (d.steps < 0) return why = "steps must be non-negative", false;
  return true;
}

struct Request {
  long long id = 0;
  hfg_scene_desc_t d{};
  long long footprint = 0, cells = 0, particles = 0;
  Clock::time_point submitted, admitted, finished;
  int status = 0;  // 0 queued, 1 running, 2 done, < 0 failed
  bool rejected = false;
  std::string error;
  std::vector<double> stepMs;
  std::vector<float> pos;
  hfg_stats_t last{};
};

class Server {
 public:
  Server(int device, int slots, long long budget) : device_(device), slots_(slots), budget_(budget) {
    for (int i = 0; i < slots; ++i) workers_.emplace_back([this] { work(); });
  }
  ~Server() {
    drain();
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }

  long long submit(const hfg_scene_desc_t& d) {
    std::string why;
    if (!validDesc(d, why)) throw CudaError("scene description: " + why, HFG_ERR_INVALID);
    auto r = std::make_unique<Request>();
    r->d = d;
    r->cells = (long long)d.res[0] * d.res[1] * d.res[2];
    r->footprint = sceneBytes(d.res, particlesBound(d), 1 + d.n_spheres, d.options.precond,
                              d.options.sort_interval > 0);
    r->submitted = Clock::now();
    std::lock_guard<std::mutex> lk(mu_);
    r->id = ++nextId_;
    ++submitted_;
    if (firstSubmit_ == Clock::time_point{}) firstSubmit_ = r->submitted;
    long long id = r->id;
    if (r->footprint > budget_) {
      r->status = HFG_ERR_NOMEM;
      r->rejected = true;
      r->error = "scene footprint exceeds the server's byte budget";
      r->finished = r->submitted;
      ++rejected_;
      all_[id] = std::move(r);
      done_.notify_all();
      return id;
    }
    queue_.push_back(r.get());
    all_[id] = std::move(r);
    cv_.notify_all();
    return id;
  }

  Request* find(long long id) {
    auto it = all_.find(id);
    if (it == all_.end()) throw CudaError("unknown request id", HFG_ERR_INVALID);
    return it->second.get();
  }

  void info(long long id, hfg_request_info_t* out, bool wait) {
    std::unique_lock<std::mutex> lk(mu_);
    Request* r = find(id);
    if (wait) done_.wait(lk, [&] { return r->status == 2 || r->status < 0; });
    std::memset(out, 0, sizeof(*out));
    out->status = r->status;
    out->steps_done = (int)r->stepMs.size();
    out->cells = r->cells;
    out->particles = r->particles;
    out->footprint_bytes = r->footprint;
    if (r->admitted != Clock::time_point{}) {
      out->queue_ms = msBetween(r->submitted, r->admitted);
      if (r->status == 2 || r->status < 0) out->run_ms = msBetween(r->admitted, r->finished);
    }
    out->step_ms_p50 = percentile(r->stepMs, 0.5);
    out->step_ms_max = r->stepMs.empty() ? 0.0 : *std::max_element(r->stepMs.begin(), r->stepMs.end());
    out->last = r->last;
  }

  int stepTimes(long long id, double* ms, int cap) {
    std::lock_guard<std::mutex> lk(mu_);
    Request* r = find(id);
    int n = std::min<int>(cap, (int)r->stepMs.size());
    for (int i = 0; i < n; ++i) ms[i] = r->stepMs[i];
    return n;
  }

  void particles(long long id, float* pos, long long cap) {
    std::lock_guard<std::mutex> lk(mu_);
    Request* r = find(id);
    if (r->status != 2) throw CudaError("request is not done", HFG_ERR_STATE);
    if (!r->d.keep_particles) throw CudaError("request did not keep its particles", HFG_ERR_STATE);
    if (cap < (long long)r->pos.size()) throw CudaError("buffer too small", HFG_ERR_INVALID);
    std::copy(r->pos.begin(), r->pos.end(), pos);
  }

  void drain() {
    std::unique_lock<std::mutex> lk(mu_);
    done_.wait(lk, [&] { return queue_.empty() && running_ == 0; });
  }

  void stats(hfg_server_stats_t* st) {
    std::lock_guard<std::mutex> lk(mu_);
    std::memset(st, 0, sizeof(*st));
    std::vector<double> steps, reqs;
    Clock::time_point last{};
    for (auto& kv : all_) {
      Request* r = kv.second.get();
      if (r->status == 2) {
        ++st->completed;
        steps.insert(steps.end(), r->stepMs.begin(), r->stepMs.end());
        reqs.push_back(msBetween(r->submitted, r->finished));
        st->cell_steps += (double)r->cells * (double)r->stepMs.size();
        last = std::max(last, r->finished);
      } else if (r->status < 0 && !r->rejected) {
        ++st->failed;
      }
    }
    st->submitted = submitted_;
    st->rejected = rejected_;
    st->step_ms_p50 = percentile(steps, 0.5);
    st->step_ms_p99 = percentile(steps, 0.99);
    st->request_ms_p50 = percentile(reqs, 0.5);
    st->request_ms_p99 = percentile(reqs, 0.99);
    if (st->completed) st->wall_s = msBetween(firstSubmit_, last) / 1e3;
    st->peak_bytes = peakBytes_;
    st->budget_bytes = budget_;
    st->peak_running = peakRunning_;
    st->slots = slots_;
  }

 private:
  // The next admissible request: the first in arrival order whose footprint
  // fits, unless the head has waited more than a second (then only the head).
  Request* pick() {
    if (queue_.empty()) return nullptr;
    Request* head = queue_.front();
    auto fits = [&](Request* r) { return inUse_ + r->footprint <= budget_; };
    if (fits(head)) {
      queue_.pop_front();
      return head;
    }
    if (msBetween(head->submitted, Clock::now()) > 1000.0) return nullptr;
    for (auto it = queue_.begin(); it != queue_.end(); ++it)
      if (fits(*it)) {
        Request* r = *it;
        queue_.erase(it);
        return r;
      }
    return nullptr;
  }

  void work() {
    cudaSetDevice(device_);
    for (;;) {
      Request* r = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
          if (stop_) return;
          r = pick();
          if (r) break;
          // a head that stops being passed is re-examined at least every 50 ms
          cv_.wait_for(lk, std::chrono::milliseconds(50));
        }
        r->status = 1;
        r->admitted = Clock::now();
        inUse_ += r->footprint;
        peakBytes_ = std::max(peakBytes_, inUse_);
        ++running_;
        peakRunning_ = std::max(peakRunning_, running_);
      }
      int status = 2;
      std::string err;
      std::vector<double> stepMs;
      std::vector<float> pos;
      hfg_stats_t last{};
      long long particles = 0;
      try {
        run(*r, stepMs, pos, last, particles);
      } catch (const CudaError& e) {
        status = e.code < 0 ? e.code : HFG_ERR_CUDA;
        err = e.what();
      } catch (const std::exception& e) {
        status = HFG_ERR_INVALID;
        err = e.what();
      }
      {
        std::lock_guard<std::mutex> lk(mu_);
        r->stepMs = std::move(stepMs);
        r->pos = std::move(pos);
        r->last = last;
        r->particles = particles;
        r->error = err;
        r->finished = Clock::now();
        r->status = status;
        inUse_ -= r->footprint;
        --running_;
      }
      done_.notify_all();
      cv_.notify_all();
    }
  }

  // One request: build the dam break, step it, keep what was asked for.
  static void run(const Request& r, std::vector<double>& stepMs, std::vector<float>& pos, hfg_stats_t& last,
                  long long& particles) {
    const hfg_scene_desc_t& d = r.d;
    std::unique_ptr<GridSolver> sp = buildScene(d);
    GridSolver& s = *sp;
    particles = s.numParticles();
    stepMs.reserve(d.steps);
    for (int k = 0; k < d.steps; ++k) {
      auto t0 = Clock::now();
      s.update();
      s.synchronize();
      stepMs.push_back(msBetween(t0, Clock::now()));
    }
    s.getStats(&last);
    if (d.keep_particles && particles > 0) {
      pos.resize(3 * (size_t)particles);
      s.getParticles(pos.data(), nullptr);
    }
  }

  int device_, slots_;
  long long budget_;
  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable cv_, done_;
  std::deque<Request*> queue_;
  std::map<long long, std::unique_ptr<Request>> all_;
  long long nextId_ = 0, submitted_ = 0, rejected_ = 0, inUse_ = 0, peakBytes_ = 0;
  int running_ = 0, peakRunning_ = 0;
  bool stop_ = false;
  Clock::time_point firstSubmit_{};
};

template <class F> int guardedS(F&& f) {
  try {
    return f();
  } catch (const CudaError& e) {
    setLastError(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    setLastError("host allocation failed");
    return HFG_ERR_NOMEM;
  } catch (const std::exception& e) {
    setLastError(e.what());
    return HFG_ERR_INVALID;
  }
}
}  // namespace

struct hfg_server_s {
  std::unique_ptr<Server> s;
};

namespace {
// ---------------------------------------------------------------------------
// Batched lockstep stepping (hfg_batch_*).  All scenes stay resident and
// advance together, one step at a time:
//   A. every scene's boundaries and the advection up to the CFL substeps, on
//      its own stream (a pool of host threads issues them);
//   B. the substeps of all scenes: one kSubstepMulti launch per substep slot
//      covers the particles of every scene, each with its own CFL state; the
//      launches of a step form one CUDA graph (recaptured when the predicted
//      substep count changes), followed by one read-back of every scene's
//      state;
//   C. every scene's P2G, pressure solve (graph-replayed CG chunks) and
//      extrapolation, again on the scenes' own streams from the pool.
// A scene's results are those it has alone, up to the order of the P2G
// float atomics.
class WorkPool {
 public:
  WorkPool(int device, int threads) {
    for (int i = 0; i < threads; ++i)
      th_.emplace_back([this, device] {
        cudaSetDevice(device);
        long long seen = 0;
        for (;;) {
          std::function<void(int)> job;
          {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
            if (stop_) return;
            seen = gen_;
            job = job_;
          }
          drain(job);
        }
      });
  }
  ~WorkPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  // f(i) for every i in [0, n) on the pool (the caller takes part); the first
  // exception is rethrown here once all have finished
  void run(int n, const std::function<void(int)>& f) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      job_ = f;
      n_ = n;
      next_ = 0;
      done_ = 0;
      err_ = nullptr;
      ++gen_;
    }
    cv_.notify_all();
    drain(f);
    std::unique_lock<std::mutex> lk(mu_);
    fin_.wait(lk, [&] { return done_ == n_; });
    if (err_) std::rethrow_exception(err_);
  }

 private:
  void drain(const std::function<void(int)>& f) {
    for (;;) {
      int i;
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (next_ >= n_) return;
        i = next_++;
      }
      try {
        f(i);
      } catch (...) {
        std::lock_guard<std::mutex> lk(mu_);
        if (!err_) err_ = std::current_exception();
      }
      std::lock_guard<std::mutex> lk(mu_);
      if (++done_ == n_) fin_.notify_all();
    }
  }
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, fin_;
  std::function<void(int)> job_;
  int n_ = 0, next_ = 0, done_ = 0;
  long long gen_ = 0;
  bool stop_ = false;
  std::exception_ptr err_;
};

class Batch {
 public:
  Batch(int device, const hfg_scene_desc_t* d, int n, int threads) : device_(device), pool_(device, threads) {
    check(cudaSetDevice(device), "cudaSetDevice");
    std::string why;
    for (int i = 0; i < n; ++i)
      if (!validDesc(d[i], why)) throw CudaError("scene " + std::to_string(i) + ": " + why, HFG_ERR_INVALID);
    sc_.resize(n);
    pool_.run(n, [&](int i) { sc_[i] = buildScene(d[i]); });
    check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    ready_.resize(n);
    for (auto& e : ready_) check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    check(cudaEventCreateWithFlags(&subDone_, cudaEventDisableTiming), "cudaEventCreate");
    check(cudaHostAlloc((void**)&tasksHost_, sizeof(SubstepTask) * n, cudaHostAllocDefault), "cudaHostAlloc");
    check(cudaHostAlloc((void**)&startHost_, sizeof(long long) * (n + 1), cudaHostAllocDefault), "cudaHostAlloc");
    check(cudaHostAlloc((void**)&flags_, sizeof(int) * 2 * n, cudaHostAllocMapped), "cudaHostAlloc");
    check(cudaHostGetDevicePointer((void**)&flagsDev_, flags_, 0), "cudaHostGetDevicePointer");
    tasks_.alloc(n);
    start_.alloc(n + 1);
    counts_.assign(n, 0);
  }
  ~Batch() {
    if (stream_) cudaStreamSynchronize(stream_);
    if (graph_) cudaGraphExecDestroy(graph_);
    for (auto& e : ready_) cudaEventDestroy(e);
    if (subDone_) cudaEventDestroy(subDone_);
    if (tasksHost_) cudaFreeHost(tasksHost_);
    if (startHost_) cudaFreeHost(startHost_);
    if (flags_) cudaFreeHost(flags_);
    sc_.clear();
    tasks_.release();
    start_.release();
    if (stream_) cudaStreamDestroy(stream_);
  }

  void step() {
    const int n = (int)sc_.size();
    std::vector<char> particles(n, 0);
    // A: boundaries, G2P and the first substep sample of every scene
    pool_.run(n, [&](int i) {
      GridSolver& s = *sc_[i];
      s.stepBoundaries();
      particles[i] = s.advectBegin() ? 1 : 0;
      if (particles[i]) check(cudaEventRecord(ready_[i], s.stream()), "cudaEventRecord");
    });
    // B: the substeps of all scenes in shared launches
    std::vector<int> who;
    long long chunks = 0;
    for (int i = 0; i < n; ++i)
      if (particles[i]) {
        tasksHost_[who.size()] = sc_[i]->substepTask();
        startHost_[who.size()] = chunks;
        chunks += multiSubstepChunks(tasksHost_[who.size()].P);
        who.push_back(i);
      }
    const int m = (int)who.size();
    if (m > 0) {
      startHost_[m] = chunks;
      check(cudaMemcpyAsync(tasks_.p, tasksHost_, sizeof(SubstepTask) * m, cudaMemcpyHostToDevice, stream_), "copy");
      check(cudaMemcpyAsync(start_.p, startHost_, sizeof(long long) * (m + 1), cudaMemcpyHostToDevice, stream_),
            "copy");
      for (int i : who) check(cudaStreamWaitEvent(stream_, ready_[i], 0), "cudaStreamWaitEvent");
      int predicted = 4;
      for (int i : who) predicted = std::max(predicted, counts_[i]);
      // a graph of `predicted` launches (slots 0 ..) while the scene set and
      // its chunking stay the same; then chunks of 4 launches until done
      if (!graph_ || graphSlots_ != predicted || graphScenes_ != m || graphChunks_ != chunks) {
        if (graph_) cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
        cudaGraph_t g = nullptr;
        check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capture");
        cudaError_t e = cudaSuccess;
        for (int k = 0; k < predicted && e == cudaSuccess; ++k)
          e = launchSubstepMulti(tasks_.p, start_.p, m, chunks, k, stream_);
        if (e == cudaSuccess) e = launchGatherSubstepStates(tasks_.p, m, predicted, flagsDev_, stream_);
        cudaError_t ec = cudaStreamEndCapture(stream_, &g);
        check(e, "substep launches");
        check(ec, "capture");
        e = cudaGraphInstantiate(&graph_, g, 0);
        cudaGraphDestroy(g);
        check(e, "cudaGraphInstantiate");
        graphSlots_ = predicted;
        graphScenes_ = m;
        graphChunks_ = chunks;
      }
      check(cudaGraphLaunch(graph_, stream_), "substep graph");
      int slot = predicted;
      for (;;) {
        check(cudaStreamSynchronize(stream_), "substep sync");
        bool all = true;
        for (int j = 0; j < m; ++j) all = all && flags_[2 * j] != 0;
        if (all) break;
        if (slot >= 4000) throw CudaError("CFL substep limit reached", HFG_ERR_STATE);
        for (int k = 0; k < 4; ++k, ++slot)
          check(launchSubstepMulti(tasks_.p, start_.p, m, chunks, slot, stream_), "substep");
        check(launchGatherSubstepStates(tasks_.p, m, slot, flagsDev_, stream_), "gather");
      }
      for (int j = 0; j < m; ++j) counts_[who[j]] = flags_[2 * j + 1];
      check(cudaEventRecord(subDone_, stream_), "cudaEventRecord");
    }
    // C: P2G, pressure and extrapolation of every scene
    pool_.run(n, [&](int i) {
      GridSolver& s = *sc_[i];
      if (particles[i]) {
        check(cudaStreamWaitEvent(s.stream(), subDone_, 0), "cudaStreamWaitEvent");
        s.substepsDone(counts_[i]);
        s.advectEnd();
      }
      s.solvePressure();
      s.synchronize();
    });
  }

  GridSolver& scene(int i) { return *sc_.at(i); }
  int size() const { return (int)sc_.size(); }

 private:
  int device_;
  WorkPool pool_;
  std::vector<std::unique_ptr<GridSolver>> sc_;
  cudaStream_t stream_ = nullptr;
  std::vector<cudaEvent_t> ready_;
  cudaEvent_t subDone_ = nullptr;
  SubstepTask* tasksHost_ = nullptr;
  long long* startHost_ = nullptr;
  int* flags_ = nullptr;  // mapped: finished, count per scene
  int* flagsDev_ = nullptr;
  DArray<SubstepTask> tasks_;
  DArray<long long> start_;
  std::vector<int> counts_;
  cudaGraphExec_t graph_ = nullptr;
  int graphSlots_ = 0, graphScenes_ = 0;
  long long graphChunks_ = -1;
};

}  // namespace

struct hfg_batch_s {
  std::unique_ptr<Batch> b;
};

extern "C" {

HFG_API int hfg_scene_bytes(const int res[3], long long particles, int boundaries, int precond, long long* bytes) {
  return guardedS([&]() -> int {
    if (!res || !bytes || res[0] <= 0 || res[1] <= 0 || res[2] <= 0 || particles < 0 || boundaries < 0)
      throw CudaError("invalid arguments", HFG_ERR_INVALID);
    *bytes = sceneBytes(res, particles, boundaries, precond);
    return HFG_OK;
  });
}

HFG_API int hfg_scene_particles_bound(const hfg_scene_desc_t* d, long long* particles) {
  return guardedS([&]() -> int {
    if (!d || !particles) throw CudaError("invalid arguments", HFG_ERR_INVALID);
    std::string why;
    if (!validDesc(*d, why)) throw CudaError("scene description: " + why, HFG_ERR_INVALID);
    *particles = particlesBound(*d);
    return HFG_OK;
  });
}

HFG_API int hfg_server_create(int device, int slots, long long budget_bytes, hfg_server_t* out) {
  return guardedS([&]() -> int {
    if (!out || slots <= 0 || slots > 256 || budget_bytes <= 0) throw CudaError("invalid arguments", HFG_ERR_INVALID);
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) throw CudaError("no CUDA device available", HFG_ERR_CUDA);
    if (device < 0 || device >= n) throw CudaError("device index out of range", HFG_ERR_INVALID);
    auto* h = new hfg_server_s();
    h->s = std::make_unique<Server>(device, slots, budget_bytes);
    *out = h;
    return HFG_OK;
  });
}

#define SERVER(h)                                                        \
  if (!(h) || !(h)->s) throw CudaError("null server", HFG_ERR_INVALID); \
  Server& S = *(h)->s

HFG_API int hfg_server_submit(hfg_server_t srv, const hfg_scene_desc_t* desc, long long* id) {
  return guardedS([&]() -> int {
    SERVER(srv);
    if (!desc || !id) throw CudaError("invalid arguments", HFG_ERR_INVALID);
    *id = S.submit(*desc);
    return HFG_OK;
  });
}
HFG_API int hfg_server_info(hfg_server_t srv, long long id, hfg_request_info_t* info) {
  return guardedS([&]() -> int {
    SERVER(srv);
    if (!info) throw CudaError("invalid arguments", HFG_ERR_INVALID);
    S.info(id, info, false);
    return HFG_OK;
  });
}
HFG_API int hfg_server_wait(hfg_server_t srv, long long id, hfg_request_info_t* info) {
  return guardedS([&]() -> int {
    SERVER(srv);
    if (!info) throw CudaError("invalid arguments", HFG_ERR_INVALID);
    S.info(id, info, true);
    return HFG_OK;
  });
}
HFG_API int hfg_server_step_times(hfg_server_t srv, long long id, double* ms, int capacity) {
  return guardedS([&]() -> int {
    SERVER(srv);
    if (!ms || capacity < 0) throw CudaError("invalid arguments", HFG_ERR_INVALID);
    return S.stepTimes(id, ms, capacity);
  });
}
HFG_API int hfg_server_particles(hfg_server_t srv, long long id, float* pos, long long capacity) {
  return guardedS([&]() -> int {
    SERVER(srv);
    if (!pos) throw CudaError("invalid arguments", HFG_ERR_INVALID);
    S.particles(id, pos, capacity);
    return HFG_OK;
  });
}
HFG_API int hfg_server_drain(hfg_server_t srv) {
  return guardedS([&]() -> int {
    SERVER(srv);
    S.drain();
    return HFG_OK;
  });
}
HFG_API int hfg_server_stats(hfg_server_t srv, hfg_server_stats_t* st) {
  return guardedS([&]() -> int {
    SERVER(srv);
    if (!st) throw CudaError("invalid arguments", HFG_ERR_INVALID);
    S.stats(st);
    return HFG_OK;
  });
}
HFG_API int hfg_server_destroy(hfg_server_t srv) {
  return guardedS([&]() -> int {
    if (!srv) throw CudaError("null server", HFG_ERR_INVALID);
    delete srv;
    return HFG_OK;
  });
}

HFG_API int hfg_batch_create(int device, const hfg_scene_desc_t* scenes, int n, int threads, hfg_batch_t* out) {
  return guardedS([&]() -> int {
    if (!out || !scenes || n <= 0 || threads <= 0 || threads > 256)
      throw CudaError("invalid arguments", HFG_ERR_INVALID);
    auto* h = new hfg_batch_s();
    try {
      h->b.reset(new Batch(device, scenes, n, threads));
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return HFG_OK;
  });
}

HFG_API int hfg_batch_step(hfg_batch_t b, int steps, double* ms) {
  return guardedS([&]() -> int {
    if (!b || !b->b || steps < 0) throw CudaError("invalid arguments", HFG_ERR_INVALID);
    for (int k = 0; k < steps; ++k) {
      auto t0 = Clock::now();
      b->b->step();
      if (ms) ms[k] = msBetween(t0, Clock::now());
    }
    return HFG_OK;
  });
}

HFG_API int hfg_batch_scene_stats(hfg_batch_t b, int scene, hfg_stats_t* st) {
  return guardedS([&]() -> int {
    if (!b || !b->b || !st || scene < 0 || scene >= b->b->size()) throw CudaError("invalid arguments", HFG_ERR_INVALID);
    b->b->scene(scene).getStats(st);
    return HFG_OK;
  });
}

HFG_API int hfg_batch_particles(hfg_batch_t b, int scene, float* pos, long long capacity) {
  return guardedS([&]() -> int {
    if (!b || !b->b || !pos || scene < 0 || scene >= b->b->size()) throw CudaError("invalid arguments", HFG_ERR_INVALID);
    GridSolver& s = b->b->scene(scene);
    if (capacity < 3 * s.numParticles()) throw CudaError("particle buffer too small", HFG_ERR_INVALID);
    s.getParticles(pos, nullptr);
    return HFG_OK;
  });
}

HFG_API int hfg_batch_destroy(hfg_batch_t b) {
  return guardedS([&]() -> int {
    if (!b) throw CudaError("null batch", HFG_ERR_INVALID);
    delete b;
    return HFG_OK;
  });
}

}  // extern "C"
