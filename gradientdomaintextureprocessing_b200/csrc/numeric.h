// Numeric set-up of the multigrid on the device.
//
// Everything the V-cycle reads that depends on the weights (screen M +
// stiffness S) is recomputed on the device from the M and S coefficients kept
// resident in HBM: the reciprocal stencil planes of the smoother, the boundary
// rows, the exact boundary-block solver (scaled subdomain inverses, couplings,
// back-substitution blocks, separator Schur complement inverse), the coarsest
// dense inverse and the level-0 FP64 operator.  The host lays out the
// weight-independent structure once per level count (NumericPlan::build); an
// update then costs one pass of device kernels (UpdateLinearSystem and
// UpdateMultigridSolvers, UpdateCoefficients.inl:402-469, whose Eigen
// factorisations the blocked Gauss-Jordan inverses of kernels/dense_kernels.cu
// replace).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "kernels/vcycle_kernels.h"
#include "setup/setup.h"

namespace gdtp {

struct DeviceArena;

// One level's structure and resident sources.  Value sources: deep coefficient
// d * 10 + k of the level's deep texel d (M and S), and the entries of the union
// patterns of M's and S's boundary blocks (bb: boundary x boundary, bd:
// boundary x global texel), M and S aligned to the union (zeros where absent).
struct NumericLevel {
  int n = 0, nDeep = 0, nB = 0;
  bool coarsest = false;
  long long nBB = 0, nBD = 0;
  const double *deepM = nullptr, *deepS = nullptr;
  const double *bbM = nullptr, *bbS = nullptr, *bdM = nullptr, *bdS = nullptr;
  double *bbV = nullptr, *bdV = nullptr;  // combined for the current weights
  Csr bb, bd;                             // union patterns (values: M)
  // boundary rows of the smoother: per row the bd entries then the bb entries
  // (global columns); source per entry: >= 0 bd entry, < 0 bb entry -1 - code
  std::vector<int> bPtr, bCol;
  const int* bSrc = nullptr;
  long long nBRow = 0;
  // boundary solver
  BoundarySymbolic sym;
  const int *pos = nullptr, *order = nullptr, *bbRow = nullptr, *bbCol = nullptr, *diagEntry = nullptr;
  const int *fillEntry = nullptr, *ssEntry = nullptr, *aisEntry = nullptr, *asiEntry = nullptr, *bdEntry = nullptr;
  const long long *fillDest = nullptr, *ssDest = nullptr, *aisDest = nullptr;
  const int *subPtr = nullptr, *touchPtr = nullptr, *touch = nullptr;
  const long long *wOff = nullptr, *lOff = nullptr, *invOff = nullptr, *invOffPad = nullptr;
  std::vector<long long> invOffPadHost;   // padded rows (multiple of 4) as the solver kernels read them
  dev::SpdInverseLayout subLayout, schurLayout;
  dev::SpdInverseDevice subDev{}, schurDev{};
  std::vector<dev::GemmTask> gTasks, lTasks;
  const dev::GemmTask *gTasksDev = nullptr, *lTasksDev = nullptr;
  int maxM = 1, maxT = 1;
  // coarsest level: dense entries (row, column, source) and per-row diagonal
  // sources; a source is kind << 40 | index, kind 0 deep, 1 bd, 2 bb
  long long nDense = 0;
  const long long *denseSrc = nullptr, *diagSrc = nullptr;
  const int *denseRow = nullptr, *denseCol = nullptr;
  dev::SpdInverseLayout coarseLayout;
  dev::SpdInverseDevice coarseDev{};
  // smoother planes: run texel -> deep texel (the multigrid's run order)
  const int* runTexel = nullptr;
  int runCount = 0;
};

// Values of one multigrid level the numeric set-up writes (value type T).
template <typename T>
struct LevelValues {
  T* planes = nullptr;        // 10 x planeStride
  int planeStride = 0;
  T* bVal = nullptr;
  T *inv = nullptr, *sinv = nullptr, *scale = nullptr, *bdVal = nullptr, *asiVal = nullptr, *wt = nullptr;
  int nSp = 0;                // separator rows padded to a multiple of 4
  double *coarseInv = nullptr, *coarseScale = nullptr;
};

// Set-up scratch comes from the device's default memory pool, stream-ordered;
// freed blocks stay in the pool (no release threshold), so that the next
// set-up or update reuses them instead of mapping new memory.  Called once per
// device before the first StreamScratch.
void keep_pool_memory();

// Stream-ordered scratch buffers of one set-up step, released (to the pool) on
// destruction; `last` holds the first allocation or copy error.
struct StreamScratch {
  std::vector<void*> ptrs;
  cudaStream_t s;
  cudaError_t last = cudaSuccess;
  explicit StreamScratch(cudaStream_t stream) : s(stream) { keep_pool_memory(); }
  StreamScratch(const StreamScratch&) = delete;
  StreamScratch& operator=(const StreamScratch&) = delete;
  ~StreamScratch() {
    for (void* p : ptrs) cudaFreeAsync(p, s);
  }
  template <class T>
  T* get(size_t n) {
    void* p = nullptr;
    size_t bytes = (n ? n : 1) * sizeof(T);
    if (bytes < 16) bytes = 16;
    const cudaError_t e = cudaMallocAsync(&p, bytes, s);
    if (e != cudaSuccess) {
      if (last == cudaSuccess) last = e;
      return nullptr;
    }
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
  template <class T>
  T* upload(const std::vector<T>& v) {
    T* p = get<T>(v.size());
    if (p && !v.empty()) {
      const cudaError_t e = cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess && last == cudaSuccess) last = e;
    }
    return p;
  }
};

// planes[k][i] = deep[10 texel[i] + k], k < 9 (raw FP64 operator planes in run order)
void launch_gather_planes(int count, const int* texel, const double* deep, double* planes, cudaStream_t s);

class NumericPlan {
 public:
  NumericPlan() = default;
  NumericPlan(const NumericPlan&) = delete;
  NumericPlan& operator=(const NumericPlan&) = delete;
  ~NumericPlan();
  // structure of levels [0, L) and their resident M / S sources
  // (deep0M, deep0S: the level-0 deep coefficients already resident on the device)
  bool build(const Hierarchy& h, int L, const FineSystem& fine, const std::vector<LevelCoefficients>& coM,
             const std::vector<LevelCoefficients>& coS, const double* deep0M, const double* deep0S, int maxBlock, int denseMax,
             cudaStream_t s, std::string& err);
  // bbV, bdV of every level for screen M + stiffness S
  bool combine(double screen, double stiffness, cudaStream_t s, std::string& err);
  // run order of a level's smoother planes (the multigrid's deep runs)
  bool set_run_order(int l, const std::vector<int>& runTexel, std::string& err);
  // values of level l into up to two multigrids' buffers (FP32 and FP64; either
  // may be null): the factorisations run once, in FP64, and are converted
  bool fill_level(int l, LevelValues<float>* f32, LevelValues<double>* f64, cudaStream_t s, std::string& err);
  // the level-0 FP64 operator's boundary rows (same layout as the smoother's)
  bool fill_raw_rows(double* bVal, cudaStream_t s, std::string& err);

  std::vector<NumericLevel> levels;
  int L = 0, maxBlock = 0, denseMax = 0;
  int gen = 0;                // generation: multigrids laid out for this plan carry it
  double screen = 0, stiffness = 0;
  size_t deviceBytes() const;
  // ms of the fill_level calls since the caller last zeroed it, per phase
  // {values and conversions, subdomain inverses, Schur products and assembly,
  // Schur complement or coarsest inverse}
  double ms[4] = {0, 0, 0, 0};

 private:
  DeviceArena* arena_ = nullptr;
};

}  // namespace gdtp
