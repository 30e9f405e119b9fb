// Solve server: many meshes and resolutions resident on one device, requests
// admitted by an HBM budget, continuous batching.
//
// A model is one (mesh, resolution, kind) with its host hierarchy (built when the
// model is added) and its device systems (built on admission):
//   filtering  M + w S;  request signal f (n x k) -> rhs M f + w s S f   (TextureFiltering.cpp:693-700)
//   geodesic   (M + w S, s M + S) + integration samples; request = k source texels (Geodesics.cpp)
//   lic        metric given per triangle (anisotropic), M + w S; rhs M f   (LineIntegralConvolution.cpp:698-706)
// `slots` worker threads take requests in arrival order.  A worker claims an idle
// model, drains every queued request of that model (up to 16 right-hand sides)
// into one batched solve, and runs it on the model's own CUDA stream, so work of
// different models overlaps on the device while requests keep arriving.
// Converged right-hand sides are frozen inside a batch, so a request's result is
// the one it gets when solved alone.  Device memory is charged to the budget per
// resident model; idle models are evicted least recently used first.
#pragma once
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "geodesics.h"
#include "server_policy.h"
#include "system.h"

namespace gdtp {

enum ModelKind { kKindFilter = 0, kKindGeodesic = 1, kKindLic = 2 };
constexpr int kMaxBatchRhs = 16;  // right-hand sides per batched solve

struct ServerRequest {
  int64_t id = 0;
  int model = 0, k = 0, maxIters = 60;
  double tol = 1e-6;
  std::vector<double> signal;   // n x k (filtering, lic)
  std::vector<int> sources;     // k (geodesic)
  std::vector<double> x;        // n x k result
  SolveReport rep;
  int status = 0;               // gdtp status
  std::string error;
  bool done = false;
  int batchSize = 0;            // requests solved together with this one (itself included)
  double tSubmit = 0, tStart = 0, tEnd = 0;  // seconds on the server clock
};

struct ServerStats {
  int64_t completed = 0, failed = 0, batches = 0, batchedRequests = 0, evictions = 0, builds = 0;
  double p50Ms = 0, p99Ms = 0, meanMs = 0, texelRhsPerSec = 0;
  int64_t residentBytes = 0, peakBytes = 0, budget = 0;
};

class Server {
 public:
  Server(int device, int64_t budget, int slots);
  ~Server();
  bool ok() const { return err_.empty(); }
  const std::string& error() const { return err_; }

  // host hierarchy now; device systems on admission.  Returns the model id or -1.
  int add_model(const Mesh& mesh, int width, int height, int levels, int kind, double w, double s, const double* metric,
                std::string& err);
  int64_t model_texels(int model) const;
  // measured device bytes when resident, else the admission estimate
  int64_t model_bytes(int model);
  // device systems now (blocking); false if the budget cannot hold them
  bool warm(int model, std::string& err);

  int64_t submit(int model, const double* signal, const int* sources, int k, double tol, int maxIters, std::string& err);
  // blocks until the request is done, moves it out and forgets it
  bool wait(int64_t id, ServerRequest& out, std::string& err);
  bool poll(int64_t id, bool& done);
  ServerStats stats();

 private:
  struct Model {
    int id = 0, kind = 0;
    double w = 0, s = 0;
    Mesh mesh;
    std::vector<double> metric;
    std::unique_ptr<Hierarchy> h;
    std::unique_ptr<BoundaryElements> be;
    std::unique_ptr<DeviceSystem> a, b;        // filtering / lic: a; geodesic: a = smoothing, b = distance
    std::unique_ptr<GeodesicIntegrator> g;
    int64_t bytes = 0, estimate = 0;
    bool busy = false;
  };
  double now() const;
  uint64_t tick() { return ++tick_; }
  bool build_device(Model& m, std::string& err);   // no lock held
  void free_device(Model& m);
  bool admit(Model& m, std::unique_lock<std::mutex>& lk, std::string& err);  // lock held on entry and exit
  void run_batch(Model& m, std::vector<ServerRequest*>& batch);
  void worker();

  int device_ = 0;
  std::string err_;
  std::mutex mu_;
  std::condition_variable cv_;
  bool stop_ = false;
  uint64_t tick_ = 0;
  int64_t nextId_ = 1;
  AdmissionPolicy policy_;
  std::map<int, std::unique_ptr<Model>> models_;
  std::map<int64_t, std::unique_ptr<ServerRequest>> requests_;
  std::deque<int64_t> queue_;
  std::vector<std::thread> workers_;
  std::vector<double> latenciesMs_;
  double firstSubmit_ = -1, lastEnd_ = 0, texelRhs_ = 0;
  int64_t completed_ = 0, failed_ = 0, batches_ = 0, batchedRequests_ = 0, builds_ = 0;
  std::chrono::steady_clock::time_point t0_;
};

}  // namespace gdtp
