// Device-resident texel-FEM system: FP64 operators, multigrid levels (FP32 for
// the mixed-precision path, FP64 for the plain comparator), exact boundary
// solvers, coarsest dense inverse, and the solve drivers.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "kernels/vcycle.cuh"
#include "kernels/vcycle_kernels.h"
#include "numeric.h"
#include "setup/setup.h"

namespace gdtp {

// Owning device allocation.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept { std::swap(p, o.p); std::swap(bytes, o.bytes); return *this; }
  ~DevBuf() { if (p) cudaFree(p); }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

struct DeviceArena {
  std::vector<DevBuf> bufs;
  size_t total = 0;
  cudaError_t last = cudaSuccess;
  void* alloc(size_t bytes) {
    DevBuf b;
    if (bytes == 0) bytes = 16;
    last = cudaMalloc(&b.p, bytes);
    if (last != cudaSuccess) return nullptr;
    b.bytes = bytes;
    total += bytes;
    void* p = b.p;
    bufs.push_back(std::move(b));
    return p;
  }
  template <class T> T* upload(const std::vector<T>& v) {
    T* p = static_cast<T*>(alloc(v.size() * sizeof(T)));
    if (p && !v.empty()) last = cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    return p;
  }
  template <class T> T* zeros(size_t n) {
    T* p = static_cast<T*>(alloc(n * sizeof(T)));
    if (p) last = cudaMemset(p, 0, n * sizeof(T));
    return p;
  }
};

// Colour runs and raw FP64 stencil planes of one level's deep texels.
struct DeepRuns {
  std::vector<dev::ColourRun> runs;
  int runStart[5] = {0, 0, 0, 0, 0};
  std::vector<int> texel;       // run texel -> deep index (plane order)
  int count = 0;                // run texels = deep texels
  // per raster line: plane index of its first even- [2 l] and odd-column [2 l + 1]
  // texel (-1: none; deep runs only)
  std::vector<int> lineCoef;
};
DeepRuns build_deep_runs(const GridLevel& L);
DeepRuns build_line_runs(const GridLevel& L);

// Raster lines of even [0] and odd [1] rows packed into blocks of the row
// smoother (dev::launch_gs_rows)
struct RowBins {
  std::vector<dev::RowLine> lines[2];
  std::vector<int> lineOf[2];   // block * block size + thread -> line (-1: idle)
  int bins[2] = {0, 0};
  int block = 0, slots = 0;
};
bool build_row_bins(const GridLevel& L, const DeepRuns& R, RowBins& out);

template <typename T>
using LevelDev = dev::LevelDev<T>;

template <typename T>
struct Multigrid {
  std::vector<LevelDev<T>> levels;
  int coarseN = 0;
  const double* coarseInv = nullptr;    // scaled dense inverse of the coarsest operator
  const double* coarseScale = nullptr;
  int KP = 0;                           // channel stride the vectors were sized for
  const dev::LevelDev<T>* levelsDev = nullptr;  // copy of `levels` in device memory (cluster kernel)
  bool clusterOK = false;               // the device can run the coarse-level cluster
  bool gridOK = false;                  // the device can run the persistent coarse-level kernel
  dev::GridBarrierState* barrier = nullptr;  // its grid barrier
  int planGen = -1;                     // the numeric plan its layout follows (-1: host-built values)
  DeviceArena arena;
};

// Raw FP64 operator on level 0 (no reciprocals): y = A x.
struct RawOperator {
  const dev::ColourRun* runs = nullptr;
  int nRuns = 0;
  const double* coef = nullptr;         // 9 planes used
  int planeStride = 0;
  const int *bPtr = nullptr, *bCol = nullptr, *bGlobal = nullptr;
  const double* bVal = nullptr;
  int nB = 0;
};

// Defaults are the autotuner's choice on the 2048^2 icosphere filtering workload
// (3 + 3 deep sweeps on level 0, none before and 3 after the coarse correction on
// the coarser levels).
struct SolverKnobs {
  int preSweeps = 3, postSweeps = 3;
  int preBoundary = 0, postBoundary = 1;  // exact boundary solve before the pre / post sweeps
  int maxBlock = 384;                   // boundary subdomain size
  int denseBoundaryMax = 0;             // boundary blocks up to this size are inverted whole (0: off)
  int bsBlocksPerSm = 2;                // boundary products: chunk so that a wave has this many blocks per SM
  int maxCoarse = 2600;                 // coarsest level size limit (texels)
  int traceLevels = 0;                  // time every level's down / up leg (events in the graph)
  int clusterTexels = 0;                // levels up to this size run in one thread-block cluster (0: off)
  int gridTexels = 0;                   // levels up to this size run in one persistent whole-GPU kernel (0: off)
  int chartTexels = 1000;               // levels whose largest chart has at most this many deep texels
                                        // smooth all sweeps in one launch, a block per chart (0: off)
  int coarsePreSweeps = 0, coarsePostSweeps = 3;  // sweeps on levels >= coarseFrom (-1: as level 0)
  int coarseFrom = 1;
  int krylov = 0;                       // 1: flexible CG around the V-cycle instead of plain refinement
  int zeroStartSkip = 1;                // first sweep from a zero correction skips the zero neighbours
  int tileTexels = 0;                   // levels with at least this many deep texels run each smoothing
                                        // step with the fused tile smoother (0: off)
  int tilePreSweeps = 2, tilePostSweeps = 2;  // sweeps per smoothing step on tiled levels
  int tileRounds = 1;                   // passes over the four tile colours per smoothing step (the
                                        // step's sweeps split between them)
  int tileFinish = 0;                   // 1: one global colour sweep after each tiled smoothing step
  int deviceFactor = 1;                 // dense set-up inverses and products on the device (0: host)
  int rowSweeps = 1;                    // FP32 colour sweeps of k <= 4 channels as two row-smoother launches
                                        // (0: four colour passes)
};

struct SolveReport {
  int iterations = 0, vcycles = 0;
  double relMax = 0, seconds = 0;
  std::vector<double> rel;
};

class DeviceSystem {
 public:
  DeviceSystem(const Hierarchy& h, const BoundaryElements& be, int device);
  ~DeviceSystem();
  int device() const { return device_; }
  bool ok() const { return err_.empty(); }
  const std::string& error() const { return err_; }

  // assembly (FP64 on device) -> fine M and S
  bool assemble(const Mesh& mesh, const double* parameterMetric);
  const FineSystem& fine() const { return fine_; }
  // what the assembly was built from (for the geodesic integration samples)
  const Hierarchy& hierarchy() const { return h_; }
  const BoundaryElements& boundary_elements() const { return be_; }
  const ChartMetrics& metric() const { return metric_; }
  cudaStream_t stream() const { return stream_; }

  // A = screen*M + stiffness*S, Galerkin hierarchy, boundary solvers, coarse inverse
  bool update(double stiffness, double screen);
  // the coefficient hierarchy for the current weights (combined on the host on demand)
  const std::vector<LevelCoefficients>& coefficients();
  int levelsUsed() const { return levelsUsed_; }

  // host in/out, k right-hand sides (tight n x k)
  bool apply(int which, const double* x, double* y, int k);
  // y = a M x + b S x (one upload, one download)
  bool apply_combination(double a, double b, const double* x, double* y, int k);
  bool solve_mixed(const double* b_host, double* x_host, const double* b_dev, double* x_dev, int k, double tol, int maxIters,
                   cudaStream_t userStream, SolveReport& rep, bool zeroGuess = false);
  // plain FP64 V-cycles: host buffers (b_host, x_host) or the caller's device
  // buffers (b_dev, x_dev, ordered after userStream when given)
  bool solve_fp64(const double* b_host, double* x_host, const double* b_dev, double* x_dev, int k, double tol, int maxIters,
                  cudaStream_t userStream, SolveReport& rep);
  // count independent problems from host buffers, each from a zero guess: the
  // upload of b[i+1] and the download of x[i-1] run on two copy streams while
  // problem i is solved; returns once every x[i] is written
  bool solve_stream(const double* const* b_host, double* const* x_host, int count, int k, double tol, int maxIters,
                    SolveReport* reps);
  bool vcycle_host(float* x, const float* rhs, int k);
  // the filtering solve A x = M f + coefS S f from the host signal f (n x k):
  // the right-hand side is formed on the device, x (host) receives the solution
  bool solve_filtering(const double* f_host, double* x_host, int k, double coefS, double tol, int maxIters, SolveReport& rep);
  // one plain FP64 V-cycle on level-0 host vectors (the FP64 multigrid)
  bool vcycle_host64(double* x, const double* rhs, int k);
  // `sweeps` level-0 smoothing sweeps (host FP32 vectors, x in place) with the
  // level-0 smoother the V-cycle uses (colour passes or the fused tile smoother)
  bool relax_host(float* x, const float* rhs, int k, int sweeps, bool reverse);
  // times full solves of b (host, n x k) for a grid of smoother settings and
  // keeps the fastest that converges; returns the chosen knobs
  bool autotune(const double* b, int k, double tol, SolverKnobs& best, double& bestSeconds);
  bool residual_host(const double* b, const double* x, int k, double* rel);

  SolverKnobs knobs;
  bool profTiled() const { return profTiled_; }
  bool profRows() const { return profRows_; }
  template <typename T>
  void tile_smooth(Multigrid<T>& mg, dev::LevelDev<T>& D, int sweeps, bool reverse, bool zeroStart, cudaStream_t s, bool prof);
  // one 4-colour Gauss-Seidel sweep (colours 0..3, or 3..0 when reverse): two
  // row-smoother launches (knob row_sweeps, where the level has row blocks) or
  // four colour passes, the same updates either way.  fromZero: the first sweep
  // from a zero iterate (zero neighbours skipped); rhsEarly: the launch before
  // the sweep does not write the right-hand side.
  template <typename T, int W>
  void colour_sweep(const dev::LevelDev<T>& D, int KP, bool reverse, bool fromZero, bool rhsEarly, cudaStream_t s);
  // the row smoother runs this level's sweeps: FP32 vectors of one channel group
  template <typename T>
  bool row_sweeps_on(const dev::LevelDev<T>& D, int KP, size_t valueBytes, int W) const {
    if (!knobs.rowSweeps || valueBytes != 4 || KP != W || D.rowBlock == 0) return false;
    return W == 4 ? dev::gs_rows_available<T, 4>(D) : dev::gs_rows_available<T, 1>(D);
  }
  template <typename T>
  bool grouped(const dev::LevelDev<T>& D, int KP) const {
    return knobs.chartTexels > 0 && D.nGroups > 0 && D.maxGroupDeep <= knobs.chartTexels &&
           size_t(D.maxGroupSpan) * KP * sizeof(T) <= dev::kGroupSmemMax;
  }
  // the fused tile smoother runs this level (FP32 vectors of 1 or 4 channels)
  template <typename T>
  bool tiled(const dev::LevelDev<T>& D, int KP) const {
    return sizeof(T) == 4 && knobs.tileTexels > 0 && D.nTiles > 0 && D.nDeep >= knobs.tileTexels && (KP == 1 || KP == 4);
  }
  // sweeps of a smoothing step on a level: tiled levels have their own counts
  template <typename T>
  int pre_sweeps(int level, const dev::LevelDev<T>& D, int KP) const {
    return tiled(D, KP) ? knobs.tilePreSweeps : pre_sweeps(level);
  }
  template <typename T>
  int post_sweeps(int level, const dev::LevelDev<T>& D, int KP) const {
    return tiled(D, KP) ? knobs.tilePostSweeps : post_sweeps(level);
  }
  int pre_sweeps(int level) const {
    return (level >= knobs.coarseFrom && knobs.coarsePreSweeps >= 0) ? knobs.coarsePreSweeps : knobs.preSweeps;
  }
  int post_sweeps(int level) const {
    return (level >= knobs.coarseFrom && knobs.coarsePostSweeps >= 0) ? knobs.coarsePostSweeps : knobs.postSweeps;
  }
  size_t deviceBytes() const;
  // knobs that change the launch sequence take effect on the next solve
  // drop the multigrids (rebuilt by the next solve), e.g. when a knob changes their layout
  void invalidate_multigrids();
  void invalidate_graph();
  // live timing of the level-0 colour sweeps inside the captured step graphs:
  // {V-cycles timed, sum of their average full-sweep ms, deep texels per sweep}
  double profCount = 0, profMs = 0, profTexels = 0;
  // level trace (knob traceLevels): refinement steps timed, then per level l the
  // summed ms of its down leg (smoothing, residual, restriction), the coarse
  // solve, then per level its up leg (prolongation, boundary solve, smoothing)
  double traceCount = 0;
  std::vector<double> traceDownMs, traceUpMs;
  double traceCoarseMs = 0;
  // read-only views for entry points that bring their own buffers
  const RawOperator& raw_system_operator() const { return rawA_; }
  bool is_updated() const { return updated_; }
  int num_texels() const { return h_.levels[0].numTexels; }
  // per level of the FP32 multigrid (after a solve): texels, deep texels, boundary
  // texels, subdomain rows, separator rows, subdomain tasks x chunks, Schur tasks
  // x chunks, chart groups, largest chart (deep texels)
  std::vector<double> level_stats() const;
  // last set-up, ms: update (weights, Galerkin coarsening, FP64 operators),
  // boundary solver factorisations, coarsest inverse, other multigrid set-up
  // (device layouts, uploads); the last three when the multigrid is built;
  // then the boundary solver factorisations split into partition and sparse
  // assembly, subdomain inverses, Schur products, Schur complement inverse;
  // then the assembly {assembly work lists (host), device assembly with its
  // transfers, boundary blocks (host), level-0 operator layouts}, the Galerkin
  // coarsening of M and S (host, once per level count) and the numeric plan's
  // layout (host, once per level count and boundary partition)
  double setupMs[14] = {0};
  int graphKernels = 0;         // kernel nodes in the refinement-step graph
  int64_t kernelLaunches = 0;   // kernels launched by solve_mixed since the last profile reset

 private:
  template <typename T>
  bool build_multigrid(Multigrid<T>& mg, int KP);
  // numeric set-up on the device (numeric.h): used unless device_factor is 0 or
  // the tile smoother is on
  bool use_numeric() const;
  // the numeric plan for the current level count and boundary layout knobs; a
  // plan built here is combined for the current weights (*built: it was)
  bool ensure_plan(bool* built = nullptr);
  bool ensure_host_coefficients();
  bool refresh_raw_operator();
  bool refresh_multigrids();
  template <typename T>
  LevelValues<T> level_values(Multigrid<T>& mg, int l);
  template <typename T, int W>
  // zeroStart: the level-0 iterate is zero on entry (a correction), so the
  // first sweep skips the neighbours it has not updated yet (exact zeros)
  void vcycle(Multigrid<T>& mg, cudaStream_t s, bool zeroStart = false);
  bool ensure_work(int k);
  bool prepare_timing(const Multigrid<float>& mg);
  void collect_timing(const Multigrid<float>& mg);
  static int kernel_nodes(cudaGraph_t g);
  bool krylov_solve(Multigrid<float>& mg, const double* B, double* X, int k, double tol, int maxIters, cudaStream_t s,
                    SolveReport& rep, int& it, double& rm);
  bool raw_apply_dev(const RawOperator& op, const double* b, const double* x, double* out, int k, int mode, cudaStream_t s,
                     double* sumsHost);
  bool check(cudaError_t e, const char* what);

  const Hierarchy& h_;
  const BoundaryElements& be_;
  int device_ = 0;
  std::string err_;
  cudaStream_t stream_ = nullptr;
  FineSystem fine_;
  ChartMetrics metric_;
  std::vector<LevelCoefficients> coeffs_;
  std::vector<LevelCoefficients> coMass_, coStiff_;  // Galerkin hierarchies of M and S (levels coLevels_)
  // boundary solver set-ups per level, shared by the FP32 and FP64 multigrids of
  // one update (cleared by update; keyed by the knobs that shape them)
  std::vector<std::shared_ptr<BoundarySolverSetup>> bsCache_;
  int bsCacheKey_[3] = {-1, -1, -1};
  bool hostCoeffs_ = false;             // coeffs_ holds the current weights' combination
  std::unique_ptr<NumericPlan> plan_;
  int planCount_ = 0;                   // numeric plans built so far (their generation numbers)
  bool rawFromPlan_ = false;            // rawA_ holds the plan's boundary-row layout
  int coLevels_ = 0;
  int levelsUsed_ = 0;
  double stiffness_ = 0, screen_ = 0;
  bool updated_ = false;
  bool profiling_ = false;

  DeviceArena rawArena_;                // M and S operators (assembly)
  DeviceArena deepArena_;               // level-0 deep M and S coefficients (assembly)
  const double *deepMassDev_ = nullptr, *deepStiffDev_ = nullptr;
  DeviceArena rawAArena_;               // A = screen M + stiffness S (replaced by every update)
  RawOperator rawM_, rawS_, rawA_;
  DeepRuns runs0_;

  // FP32 multigrids, one per channel stride KP in use: the first holds the
  // level structure (coefficients, runs, boundary inverses), the others share
  // it and own only their KP-wide vectors, so small solves stay narrow after
  // a wide batch and a new width costs no rebuild
  std::vector<std::unique_ptr<Multigrid<float>>> mg32_;
  Multigrid<float>* mg32_for(int KP);
  template <typename T>
  bool derive_multigrid(const Multigrid<T>& base, Multigrid<T>& mg, int KP);
  std::unique_ptr<Multigrid<double>> mg64_;

  // solve work (tight n x k FP64)
  int* frozen_ = nullptr;              // per right-hand side: converged, x kept (device)
  DeviceArena krylovArena_;            // flexible CG: z, p, q (n x k FP64), scalars
  double *z_ = nullptr, *p_ = nullptr, *q_ = nullptr, *sc_ = nullptr;
  int krylovK_ = 0;
  std::vector<int> frozenHost_;
  DeviceArena workArena_;
  int workK_ = 0;
  double *b64_ = nullptr, *x64_ = nullptr, *r64_ = nullptr, *partials_ = nullptr, *sums_ = nullptr;
  DeviceArena filterArena_;                // signal and S f of solve_filtering
  double *fDev_ = nullptr, *sfDev_ = nullptr;
  int filterK_ = 0;
  double* sumsHost_ = nullptr;    // pinned, mapped
  double* sumsMapped_ = nullptr;  // its device address (null: norms come back by copy)
  // the solve loops' small host exchanges, by kernel: norms sums_ -> sumsHost_
  // (then waits for the stream), flags frozenHost_ -> frozen_
  bool read_norms(int k, cudaStream_t s, const char* what);
  bool upload_flags(int k, cudaStream_t s);
  // solve_stream: two slots of device b / x (n x k FP64), alternating between
  // problems, and the streams and events that order the copies around the solves
  DeviceArena slotArena_;
  int slotK_ = 0;
  double *slotB_[2] = {nullptr, nullptr}, *slotX_[2] = {nullptr, nullptr};
  cudaStream_t copyIn_ = nullptr, copyOut_ = nullptr;
  cudaEvent_t slotIn_[2] = {}, slotSolved_[2] = {}, slotOut_[2] = {};
  // captured step graphs (refinement or flexible-CG step), one per right-hand
  // side count and buffers, most recently used last: a server batching
  // requests of varying sizes reuses them instead of capturing again
  struct StepGraph {
    int kind = 0;  // 0 refinement (FP32 V-cycle), 1 flexible CG, 2 FP64 V-cycle
    int k = 0, kernels = 0;
    const double *b = nullptr, *x = nullptr;
    cudaGraphExec_t exec = nullptr;
  };
  std::vector<StepGraph> stepGraphs_;
  static constexpr size_t kMaxStepGraphs = 16;
  // the cached graph for this step (moved to the back), or null
  cudaGraphExec_t find_graph(int kind, int k, const double* b, const double* x);
  void add_graph(const StepGraph& g);
  cudaEvent_t profEv_[4] = {nullptr, nullptr, nullptr, nullptr};  // level-0 full pre sweeps, post sweeps
  int profSweeps_ = 0, profPostSweeps_ = 0;
  bool profTiled_ = false;              // the timed level-0 group is one fused tile-smoother launch
  bool profRows_ = false;               // the timed level-0 sweeps are row-smoother launches (two per sweep)
  std::vector<cudaEvent_t> traceEv_;   // 2 L markers of the captured V-cycle (traceLevels)
  void trace_mark(int i, cudaStream_t s);
  unsigned long long* timeline_ = nullptr;  // cluster phase timeline (traceLevels)
  bool usedGridBarrier_ = false;        // a captured V-cycle runs the persistent coarse-level kernel
  bool usedTileWait_ = false;           // ... or the tile smoother (bounded waits on neighbouring tiles)
  unsigned int* barrierErrHost_ = nullptr;  // pinned copy of its barrier's error word
  template <typename T>
  void queue_barrier_check(Multigrid<T>& mg, cudaStream_t s);
  template <typename T>
  bool barrier_ok(Multigrid<T>& mg);
  unsigned long long* clusterTimeline();
 public:
  // last cluster timeline: {code, ns} pairs (empty when not traced)
  bool cluster_timeline(std::vector<unsigned long long>& out);
};

}  // namespace gdtp
