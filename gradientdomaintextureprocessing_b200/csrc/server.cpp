// Solve server (see server.h).
#include "server.h"

#include <algorithm>
#include <cmath>
#include <exception>
#include <new>

#include "gdtp.h"

namespace gdtp {

Server::Server(int device, int64_t budget, int slots) : device_(device), policy_(budget), t0_(std::chrono::steady_clock::now()) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) { err_ = "no CUDA device"; return; }
  if (device < 0 || device >= n) { err_ = "invalid CUDA device"; return; }
  if (budget <= 0 || slots < 1 || slots > 64) { err_ = "invalid budget or slot count"; return; }
  for (int i = 0; i < slots; i++) workers_.emplace_back([this] { worker(); });
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  cv_.notify_all();
  for (auto& t : workers_) t.join();
  cudaSetDevice(device_);
  for (auto& kv : models_) free_device(*kv.second);
}

double Server::now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count(); }

int Server::add_model(const Mesh& mesh, int width, int height, int levels, int kind, double w, double s, const double* metric,
                      std::string& err) {
  if (kind < kKindFilter || kind > kKindLic) { err = "unknown model kind"; return -1; }
  if (kind == kKindLic && !metric) { err = "a line-integral-convolution model needs its parameter metric"; return -1; }
  std::unique_ptr<Model> m(new Model());
  m->kind = kind;
  m->w = w;
  m->s = s;
  m->mesh = mesh;
  if (metric) m->metric.assign(metric, metric + 4 * size_t(mesh.nt()));
  m->h.reset(new Hierarchy());
  m->be.reset(new BoundaryElements());
  if (!build_hierarchy(m->mesh, width, height, levels, BlockInfo(), *m->h, 2600, 12)) { err = "hierarchy: " + m->h->error; return -1; }
  if (!build_boundary_elements(*m->h, *m->be, err)) { err = "boundary elements: " + err; return -1; }
  // device bytes before the first build, corrected by the measured size once
  // built: FP64 operators, resident M and S of every level for the numeric
  // set-up, FP32 multigrid with up to 4 right-hand sides and coarse factor per
  // texel, dense boundary-block inverses and their value maps per boundary
  // texel (subdomains of up to 384), fixed allocations; the geodesic kind holds
  // two systems and its integration samples.  Fitted to measured sizes (torus,
  // icosphere, genus-2 from 256^2 to 2048^2): 3-77 % headroom.
  double sys = 700.0 * m->h->levels[0].numTexels + 5500.0 * m->h->levels[0].numBoundary + double(48 << 20);
  // boundary blocks small enough to be inverted whole hold a dense FP32 inverse
  const int denseMax = SolverKnobs().denseBoundaryMax;
  for (const GridLevel& g : m->h->levels)
    if (g.numBoundary <= denseMax) sys += 4.0 * double(g.numBoundary) * g.numBoundary;
  m->estimate = int64_t(kind == kKindGeodesic ? 1.75 * sys : sys);
  std::lock_guard<std::mutex> lk(mu_);
  const int id = (int)models_.size();
  m->id = id;
  models_[id] = std::move(m);
  return id;
}

int64_t Server::model_bytes(int model) {
  std::lock_guard<std::mutex> lk(mu_);
  auto it = models_.find(model);
  if (it == models_.end()) return -1;
  return it->second->a ? it->second->bytes : it->second->estimate;
}

int64_t Server::model_texels(int model) const {
  auto it = models_.find(model);
  return it == models_.end() ? -1 : it->second->h->levels[0].numTexels;
}

bool Server::build_device(Model& m, std::string& err) {
  cudaSetDevice(device_);
  auto make = [&](std::unique_ptr<DeviceSystem>& sys, double stiffness, double screen) {
    sys.reset(new DeviceSystem(*m.h, *m.be, device_));
    if (!sys->ok() || !sys->assemble(m.mesh, m.metric.empty() ? nullptr : m.metric.data()) || !sys->update(stiffness, screen)) {
      err = sys->error();
      return false;
    }
    return true;
  };
  if (m.kind == kKindGeodesic) {
    if (!make(m.a, m.w, 1.0) || !make(m.b, 1.0, m.s)) return false;
    m.g.reset(new GeodesicIntegrator(*m.a));
    if (!m.g->ok()) { err = m.g->error(); return false; }
  } else if (!make(m.a, m.w, 1.0)) {
    return false;
  } else if (m.kind == kKindLic) {
    m.a->knobs.krylov = 1;  // the anisotropic V-cycle contracts slowly: CG around it
  }
  return true;
}

// Runs a step of the worker that may allocate; a C++ exception becomes false
// and a message, so that it fails the batch instead of ending the process.
template <class F>
static bool without_exceptions(F&& f, std::string& err) {
  try {
    return f();
  } catch (const std::bad_alloc&) {
    err = "out of host memory";
  } catch (const std::exception& e) {
    err = e.what();
  } catch (...) {
    err = "unexpected exception";
  }
  return false;
}

void Server::free_device(Model& m) {
  m.g.reset();
  m.b.reset();
  m.a.reset();
  m.bytes = 0;
}

bool Server::admit(Model& m, std::unique_lock<std::mutex>& lk, std::string& err) {
  for (;;) {
    std::vector<int> victims;
    if (policy_.plan(m.estimate, victims, m.id)) {
      for (int v : victims) {
        free_device(*models_[v]);
        policy_.evict(v);
      }
      policy_.add(m.id, m.estimate, tick());
      policy_.set_busy(m.id, true, tick());
      return true;
    }
    bool anyBusy = false;
    for (auto& kv : models_) anyBusy = anyBusy || (kv.second->busy && kv.first != m.id && policy_.resident(kv.first));
    if (!anyBusy || stop_) {
      err = "HBM budget cannot hold the model";
      return false;
    }
    cv_.wait(lk);  // a running batch will release its model
  }
}

void Server::run_batch(Model& m, std::vector<ServerRequest*>& batch) {
  cudaSetDevice(device_);
  const int64_t n = m.h->levels[0].numTexels;
  int K = 0;
  for (auto* r : batch) K += r->k;
  std::vector<double> x(size_t(n) * K, 0.0);
  SolveReport rep, rep2;
  bool ok = true;
  std::string err;
  if (m.kind == kKindGeodesic) {
    std::vector<int> src;
    for (auto* r : batch) src.insert(src.end(), r->sources.begin(), r->sources.end());
    ok = m.g->distance(*m.a, *m.b, src.data(), K, batch[0]->tol, batch[0]->maxIters, x.data(), rep, rep2);
    if (!ok) err = m.g->error();
    rep.iterations += rep2.iterations;
    rep.vcycles += rep2.vcycles;
    rep.relMax = std::max(rep.relMax, rep2.relMax);
    rep.seconds += rep2.seconds;
  } else {
    std::vector<double> f(size_t(n) * K);
    int c0 = 0;
    for (auto* r : batch) {
      for (int64_t i = 0; i < n; i++)
        for (int c = 0; c < r->k; c++) f[size_t(i) * K + c0 + c] = r->signal[size_t(i) * r->k + c];
      c0 += r->k;
    }
    // M f + w s S f (filtering) or M f (LIC), formed on the device from one upload of f
    ok = m.a->solve_filtering(f.data(), x.data(), K, m.kind == kKindFilter ? m.w * m.s : 0.0, batch[0]->tol, batch[0]->maxIters, rep);
    if (!ok) err = m.a->error();
  }
  int c0 = 0;
  for (auto* r : batch) {
    r->status = ok ? (rep.relMax <= r->tol ? GDTP_OK : GDTP_ERR_NOT_CONVERGED) : GDTP_ERR_CUDA;
    r->error = err;
    r->rep = rep;
    r->batchSize = (int)batch.size();
    r->x.resize(size_t(n) * r->k);
    for (int64_t i = 0; i < n; i++)
      for (int c = 0; c < r->k; c++) r->x[size_t(i) * r->k + c] = x[size_t(i) * K + c0 + c];
    c0 += r->k;
  }
}

void Server::worker() {
  cudaSetDevice(device_);
  std::unique_lock<std::mutex> lk(mu_);
  for (;;) {
    // the oldest queued request whose model is idle
    ServerRequest* first = nullptr;
    Model* m = nullptr;
    cv_.wait(lk, [&] {
      if (stop_) return true;
      for (int64_t id : queue_) {
        ServerRequest* r = requests_[id].get();
        Model* mm = models_[r->model].get();
        if (!mm->busy) { first = r; m = mm; return true; }
      }
      return false;
    });
    if (stop_) return;
    // batch: queued requests of the same model, tolerance and iteration limit,
    // up to kMaxBatchRhs right-hand sides (a wider batch costs the same per
    // right-hand side, but holds wider vectors and delays its first request)
    std::vector<ServerRequest*> batch;
    int K = 0;
    for (auto it = queue_.begin(); it != queue_.end();) {
      ServerRequest* r = requests_[*it].get();
      if (r->model == m->id && r->tol == first->tol && r->maxIters == first->maxIters && K + r->k <= kMaxBatchRhs) {
        batch.push_back(r);
        K += r->k;
        it = queue_.erase(it);
      } else {
        ++it;
      }
    }
    m->busy = true;
    std::string err;
    bool ok = true;
    if (!m->a) {
      ok = admit(*m, lk, err);
      if (ok) {
        lk.unlock();
        ok = without_exceptions([&] { return build_device(*m, err); }, err);
        lk.lock();
        builds_++;
        if (!ok) {
          free_device(*m);
          policy_.evict(m->id);
        }
      }
    } else {
      policy_.set_busy(m->id, true, tick());
    }
    if (ok) {
      for (auto* r : batch) r->tStart = now();
      lk.unlock();
      std::string batchErr;
      if (!without_exceptions([&] { run_batch(*m, batch); return true; }, batchErr))
        for (auto* r : batch) {
          r->status = GDTP_ERR_SETUP;
          r->error = batchErr;
        }
      lk.lock();
      m->bytes = int64_t(m->a ? m->a->deviceBytes() : 0) + int64_t(m->b ? m->b->deviceBytes() : 0);
      m->estimate = std::max(m->estimate, m->bytes);
      policy_.add(m->id, m->bytes, tick());
      policy_.set_busy(m->id, false, tick());
    } else {
      for (auto* r : batch) {
        r->status = err.find("budget") != std::string::npos ? GDTP_ERR_BUDGET : GDTP_ERR_CUDA;
        r->error = err;
      }
    }
    m->busy = false;
    batches_++;
    batchedRequests_ += (int64_t)batch.size();
    const double t = now();
    for (auto* r : batch) {
      r->tEnd = t;
      r->done = true;
      if (r->status == GDTP_OK) {
        completed_++;
        latenciesMs_.push_back((r->tEnd - r->tSubmit) * 1e3);
        texelRhs_ += double(m->h->levels[0].numTexels) * r->k;
        lastEnd_ = std::max(lastEnd_, t);
      } else {
        failed_++;
      }
    }
    cv_.notify_all();
  }
}

bool Server::warm(int model, std::string& err) {
  std::unique_lock<std::mutex> lk(mu_);
  auto it = models_.find(model);
  if (it == models_.end()) { err = "unknown model"; return false; }
  Model& m = *it->second;
  cv_.wait(lk, [&] { return !m.busy; });
  if (m.a) return true;
  m.busy = true;
  bool ok = admit(m, lk, err);
  if (ok) {
    lk.unlock();
    // an exception here (a host allocation, say) must still clear busy and the
    // admission below, or every later warm / submit of this model waits forever
    ok = without_exceptions(
        [&] {
          if (!build_device(m, err)) return false;
          // settle the multigrid and work buffers with one zero-right-hand-side solve per system
          const size_t n = m.h->levels[0].numTexels;
          const int k = m.kind == kKindFilter ? 3 : 1;
          std::vector<double> b(n * k, 0.0), x(n * k, 0.0);
          SolveReport r;
          bool solved;
          if (m.kind == kKindGeodesic) {
            std::vector<int> src(1, int(n / 2));
            std::vector<double> d(n);
            SolveReport r2;
            solved = m.g->distance(*m.a, *m.b, src.data(), 1, 1e-6, 60, d.data(), r, r2);
          } else {
            solved = m.a->solve_mixed(b.data(), x.data(), nullptr, nullptr, k, 1e-6, 60, nullptr, r, true);
          }
          if (!solved) err = m.g ? m.g->error() : m.a->error();
          return solved;
        },
        err);
    lk.lock();
    builds_++;
    if (ok) {
      m.bytes = int64_t(m.a->deviceBytes()) + int64_t(m.b ? m.b->deviceBytes() : 0);
      m.estimate = std::max(m.estimate, m.bytes);
      policy_.add(m.id, m.bytes, tick());
      policy_.set_busy(m.id, false, tick());
    } else {
      free_device(m);
      policy_.evict(m.id);
    }
  }
  m.busy = false;
  cv_.notify_all();
  return ok;
}

int64_t Server::submit(int model, const double* signal, const int* sources, int k, double tol, int maxIters, std::string& err) {
  std::unique_ptr<ServerRequest> r(new ServerRequest());
  {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = models_.find(model);
    if (it == models_.end()) { err = "unknown model"; return -1; }
    const Model& m = *it->second;
    if (k < 1 || k > 64 || !(tol > 0) || maxIters < 1) { err = "bad k, tolerance or iteration limit"; return -1; }
    const int64_t n = m.h->levels[0].numTexels;
    if (m.kind == kKindGeodesic) {
      if (!sources) { err = "a geodesic request needs source texels"; return -1; }
      for (int c = 0; c < k; c++)
        if (sources[c] < 0 || sources[c] >= n) { err = "source texel out of range"; return -1; }
      r->sources.assign(sources, sources + k);
    } else {
      if (!signal) { err = "a filtering / convolution request needs its signal"; return -1; }
      r->signal.assign(signal, signal + size_t(n) * k);
    }
  }
  r->model = model;
  r->k = k;
  r->tol = tol;
  r->maxIters = maxIters;
  std::lock_guard<std::mutex> lk(mu_);
  r->id = nextId_++;
  r->tSubmit = now();
  if (firstSubmit_ < 0) firstSubmit_ = r->tSubmit;
  const int64_t id = r->id;
  requests_[id] = std::move(r);
  queue_.push_back(id);
  cv_.notify_all();
  return id;
}

bool Server::poll(int64_t id, bool& done) {
  std::lock_guard<std::mutex> lk(mu_);
  auto it = requests_.find(id);
  if (it == requests_.end()) return false;
  done = it->second->done;
  return true;
}

bool Server::wait(int64_t id, ServerRequest& out, std::string& err) {
  std::unique_lock<std::mutex> lk(mu_);
  auto it = requests_.find(id);
  if (it == requests_.end()) { err = "unknown request"; return false; }
  ServerRequest* r = it->second.get();
  cv_.wait(lk, [&] { return r->done; });
  out = std::move(*r);
  requests_.erase(id);
  return true;
}

ServerStats Server::stats() {
  std::lock_guard<std::mutex> lk(mu_);
  ServerStats s;
  s.completed = completed_;
  s.failed = failed_;
  s.batches = batches_;
  s.batchedRequests = batchedRequests_;
  s.evictions = policy_.evictions();
  s.builds = builds_;
  s.residentBytes = policy_.used();
  s.peakBytes = policy_.peak();
  s.budget = policy_.budget();
  if (!latenciesMs_.empty()) {
    std::vector<double> l = latenciesMs_;
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) { return l[std::min(l.size() - 1, size_t(std::ceil(p * l.size())) - (p > 0 ? 1 : 0))]; };
    s.p50Ms = pct(0.50);
    s.p99Ms = pct(0.99);
    double sum = 0;
    for (double v : l) sum += v;
    s.meanMs = sum / l.size();
  }
  if (lastEnd_ > firstSubmit_ && firstSubmit_ >= 0) s.texelRhsPerSec = texelRhs_ / (lastEnd_ - firstSubmit_);
  return s;
}

}  // namespace gdtp
