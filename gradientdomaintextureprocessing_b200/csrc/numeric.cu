// Numeric set-up of the multigrid on the device (numeric.h).
#include "numeric.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cmath>

#include "system.h"

namespace gdtp {
namespace {

double wall_ms() { return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

constexpr int kThreads = 256;
inline unsigned blocks_for(long long n) { return unsigned(std::max<long long>(1, (n + kThreads - 1) / kThreads)); }

// screen M + stiffness S, each product and the sum rounded once (the host's
// csr_axpby / update arithmetic, without contraction into a fused multiply-add)
__device__ __forceinline__ double combine_rn(double a, double m, double b, double s) { return __dadd_rn(__dmul_rn(a, m), __dmul_rn(b, s)); }

__global__ void k_combine(long long n, double a, const double* __restrict__ M, double b, const double* __restrict__ S, double* __restrict__ V) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) V[i] = combine_rn(a, M[i], b, S[i]);
}

// reciprocal planes of the smoother: planes[k][i] = c_k / c_4 (k != 4),
// planes[4][i] = 1 / c_4, planes[9][i] = c_4, c of run texel i's deep texel
template <typename T>
__global__ void k_planes(int count, const int* __restrict__ runTexel, const double* __restrict__ M, const double* __restrict__ S, double a,
                         double b, T* __restrict__ planes) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const long long d = 10LL * runTexel[i];
  const double c4 = combine_rn(a, M[d + 4], b, S[d + 4]), inv = 1.0 / c4;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const double c = combine_rn(a, M[d + k], b, S[d + k]);
    planes[(long long)k * count + i] = T(k == 4 ? inv : __dmul_rn(c, inv));
  }
  planes[9LL * count + i] = T(c4);
}

template <typename T>
__global__ void k_gather_rows(long long n, const int* __restrict__ src, const double* __restrict__ bdV, const double* __restrict__ bbV,
                              T* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = src[i];
  out[i] = T(c >= 0 ? bdV[c] : bbV[-1 - c]);
}

// s_k = 1 / sqrt(diagonal of the row at position k)
__global__ void k_scale_pos(int nb, const int* __restrict__ order, const int* __restrict__ diagEntry, const double* __restrict__ bbV,
                            double* __restrict__ scale) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nb) scale[k] = 1.0 / sqrt(bbV[diagEntry[order[k]]]);
}

struct Scaled {
  const double* bbV;
  const int *bbRow, *bbCol, *pos;
  const double* scale;
  __device__ __forceinline__ double operator()(int e) const {
    return __dmul_rn(__dmul_rn(bbV[e], scale[pos[bbRow[e]]]), scale[pos[bbCol[e]]]);
  }
};

__global__ void k_scatter_scaled(long long n, const int* __restrict__ entry, const long long* __restrict__ dest, Scaled sc,
                                 double* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[dest[i]] = sc(entry[i]);
}

template <typename T>
__global__ void k_scaled_values(long long n, const int* __restrict__ entry, Scaled sc, T* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = T(sc(entry[i]));
}

template <typename T>
__global__ void k_gather_values(long long n, const int* __restrict__ entry, const double* __restrict__ V, T* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = T(V[entry[i]]);
}

template <typename T>
__global__ void k_convert(long long n, const double* __restrict__ src, T* __restrict__ dst) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = T(src[i]);
}

// S -= sum_p scatter(local_p) in subdomain order: a block owns kRowsPerBlock
// separator rows and applies the subdomains one after the other, so every
// entry sees its contributions in the same order from run to run
constexpr int kRowsPerBlock = 16;
__global__ void k_schur_subtract(int nS, int nSub, const int* __restrict__ touchPtr, const int* __restrict__ touch,
                                 const long long* __restrict__ lOff, const double* __restrict__ local, double* __restrict__ S) {
  const int r0 = blockIdx.x * kRowsPerBlock, r1 = min(nS, r0 + kRowsPerBlock);
  for (int p = 0; p < nSub; p++) {
    const int* tp = touch + touchPtr[p];
    const int t = touchPtr[p + 1] - touchPtr[p];
    // the touch list is sorted: its entries in [r0, r1)
    int lo = 0, hi = t;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (tp[mid] < r0) lo = mid + 1; else hi = mid;
    }
    int end = lo;
    while (end < t && tp[end] < r1) end++;
    const int rows = end - lo;
    const double* Lp = local + lOff[p];
    for (int e = threadIdx.x; e < rows * t; e += blockDim.x) {
      const int c1 = lo + e / t, c2 = e % t;
      S[(long long)tp[c1] * nS + tp[c2]] -= Lp[(long long)c1 * t + c2];
    }
    __syncthreads();
  }
}

// S = (S + S^T) / 2 below and above the diagonal
__global__ void k_symmetrise_pairs(int n, double* __restrict__ S) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * n) return;
  const int a = int(e / n), c = int(e - (long long)a * n);
  if (c >= a) return;
  const double v = 0.5 * (S[(long long)a * n + c] + S[(long long)c * n + a]);
  S[(long long)a * n + c] = v;
  S[(long long)c * n + a] = v;
}

// subdomain inverses, rows padded to a multiple of 4 (zeros past m): block per subdomain
template <typename T>
__global__ void k_pad_blocks(const int* __restrict__ subPtr, const long long* __restrict__ invOff, const long long* __restrict__ invOffPad,
                             const double* __restrict__ src, T* __restrict__ dst) {
  const int p = blockIdx.x;
  const int m = subPtr[p + 1] - subPtr[p], mp = (m + 3) & ~3;
  const double* s = src + invOff[p];
  T* d = dst + invOffPad[p];
  for (long long e = threadIdx.x; e < (long long)m * mp; e += blockDim.x) {
    const int j = int(e / mp), a = int(e - (long long)j * mp);
    d[e] = a < m ? T(s[(long long)j * m + a]) : T(0);
  }
}

template <typename T>
__global__ void k_pad_square(int n, int np, const double* __restrict__ src, T* __restrict__ dst) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * np) return;
  const int j = int(e / np), a = int(e - (long long)j * np);
  dst[e] = a < n ? T(src[(long long)j * n + a]) : T(0);
}

// back-substitution blocks: W_p (m x t, column-major) from G_p (m x t, row-major)
template <typename T>
__global__ void k_wt(const int* __restrict__ subPtr, const int* __restrict__ touchPtr, const long long* __restrict__ wOff,
                     const double* __restrict__ G, T* __restrict__ wt) {
  const int p = blockIdx.x;
  const int m = subPtr[p + 1] - subPtr[p], t = touchPtr[p + 1] - touchPtr[p];
  const double* g = G + wOff[p];
  T* w = wt + wOff[p];
  for (long long e = threadIdx.x; e < (long long)m * t; e += blockDim.x) {
    const int c = int(e / m), a = int(e - (long long)c * m);
    w[e] = T(g[(long long)a * t + c]);
  }
}

// coarsest level: a source is kind << 40 | index (0 deep coefficient, 1 bd, 2 bb)
struct Sources {
  double a, b;
  const double *deepM, *deepS, *bdV, *bbV;
  __device__ __forceinline__ double operator()(long long src) const {
    const int kind = int(src >> 40);
    const long long i = src & ((1LL << 40) - 1);
    return kind == 0 ? combine_rn(a, deepM[i], b, deepS[i]) : kind == 1 ? bdV[i] : bbV[i];
  }
};

__global__ void k_coarse_scale(int n, const long long* __restrict__ diagSrc, Sources v, double* __restrict__ scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) scale[i] = 1.0 / sqrt(v(diagSrc[i]));
}

__global__ void k_coarse_fill(long long nD, int n, const long long* __restrict__ src, const int* __restrict__ row, const int* __restrict__ col,
                              Sources v, const double* __restrict__ scale, double* __restrict__ dense) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nD) return;
  const int r = row[e], c = col[e];
  dense[(long long)r * n + c] = __dmul_rn(__dmul_rn(v(src[e]), scale[r]), scale[c]);
}

template <class T>
std::vector<int> as_int(const std::vector<T>& v) {
  std::vector<int> out(v.size());
  for (size_t i = 0; i < v.size(); i++) out[i] = int(v[i]);
  return out;
}

std::vector<long long> as_ll(const std::vector<int64_t>& v) { return std::vector<long long>(v.begin(), v.end()); }

__global__ void k_gather_planes(int count, const int* __restrict__ texel, const double* __restrict__ deep, double* __restrict__ planes) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const double* c = deep + 10LL * texel[i];
#pragma unroll
  for (int k = 0; k < 9; k++) planes[(long long)k * count + i] = c[k];
}

}  // namespace

void launch_gather_planes(int count, const int* texel, const double* deep, double* planes, cudaStream_t s) {
  k_gather_planes<<<blocks_for(count), kThreads, 0, s>>>(count, texel, deep, planes);
}

NumericPlan::~NumericPlan() { delete arena_; }

size_t NumericPlan::deviceBytes() const { return arena_ ? arena_->total : 0; }

namespace {
// host side of one level's plan, built for all levels in parallel before the uploads
struct LevelHost {
  Csr bbS, bdS;                           // S aligned to the union patterns (N.bb, N.bd hold M)
  std::vector<int> bsrc;
  std::vector<long long> denseSrc, diagSrc;
  std::vector<int> denseRow, denseCol, m, t;
  std::string err;
};
}  // namespace

bool NumericPlan::build(const Hierarchy& h, int L_, const FineSystem& fine, const std::vector<LevelCoefficients>& coM,
                        const std::vector<LevelCoefficients>& coS, const double* deep0M, const double* deep0S, int maxBlock_,
                        int denseMax_, cudaStream_t s, std::string& err) {
  (void)s;
  delete arena_;
  arena_ = new DeviceArena();
  DeviceArena& A = *arena_;
  L = L_;
  maxBlock = maxBlock_;
  denseMax = denseMax_;
  levels.assign(L, NumericLevel());
  std::vector<LevelHost> host(L);
  // ---- structure of every level (host, levels in parallel)
#pragma omp parallel for schedule(dynamic, 1)
  for (int l = 0; l < L; l++) {
    const GridLevel& G = h.levels[l];
    NumericLevel& N = levels[l];
    LevelHost& H = host[l];
    N.n = G.numTexels;
    N.nDeep = G.numDeep;
    N.nB = G.numBoundary;
    N.coarsest = (l == L - 1);
    const Csr& bbM = l == 0 ? fine.bbMass : coM[l].bb;
    const Csr& bbS = l == 0 ? fine.bbStiffness : coS[l].bb;
    Csr bdM = l == 0 ? fine.bdMass : coM[l].bd, bdS = l == 0 ? fine.bdStiffness : coS[l].bd;
    bdM.cols = bdS.cols = G.numTexels;
    // union patterns, M and S aligned to them
    N.bb = csr_axpby(1.0, bbM, 0.0, bbS);
    H.bbS = csr_axpby(0.0, bbM, 1.0, bbS);
    N.bd = csr_axpby(1.0, bdM, 0.0, bdS);
    H.bdS = csr_axpby(0.0, bdM, 1.0, bdS);
    N.nBB = (long long)N.bb.col.size();
    N.nBD = (long long)N.bd.col.size();
    if (N.coarsest) {
      // dense entries: deep rows' 3x3 stencils, boundary rows' bd and bb entries
      // (the layout of full_matrix, galerkin.cpp)
      H.diagSrc.assign(G.numTexels, -1);
      for (int d = 0; d < G.numDeep; d++) {
        const int r = G.deepGlobal[d];
        const NodeInfo& nd = G.nodes[r];
        const GridChart& gc = G.charts[nd.chart];
        for (int oy = -1; oy <= 1; oy++)
          for (int ox = -1; ox <= 1; ox++) {
            const int c = gc.texel[gc.at(nd.ci + ox, nd.cj + oy)];
            const long long sIdx = 10LL * d + (oy + 1) * 3 + (ox + 1);
            H.denseRow.push_back(r);
            H.denseCol.push_back(c);
            H.denseSrc.push_back(sIdx);
            if (c == r) H.diagSrc[r] = sIdx;
          }
      }
      for (int b = 0; b < G.numBoundary; b++) {
        const int r = G.boundaryGlobal[b];
        for (int k = N.bd.ptr[b]; k < N.bd.ptr[b + 1]; k++) {
          H.denseRow.push_back(r);
          H.denseCol.push_back(N.bd.col[k]);
          H.denseSrc.push_back((1LL << 40) | k);
          if (N.bd.col[k] == r) H.diagSrc[r] = (1LL << 40) | k;
        }
        for (int k = N.bb.ptr[b]; k < N.bb.ptr[b + 1]; k++) {
          const int c = G.boundaryGlobal[N.bb.col[k]];
          H.denseRow.push_back(r);
          H.denseCol.push_back(c);
          H.denseSrc.push_back((2LL << 40) | k);
          if (c == r) H.diagSrc[r] = (2LL << 40) | k;
        }
      }
      for (int i = 0; i < G.numTexels && H.err.empty(); i++)
        if (H.diagSrc[i] < 0) H.err = "coarsest level: texel without a diagonal entry";
      for (int c : H.denseCol)
        if (H.err.empty() && (c < 0 || c >= G.numTexels)) H.err = "coarsest level: stencil column outside the level";
      if (H.err.empty())
        dev::spd_inverse_layout(std::vector<int64_t>(1, 0), std::vector<int>(1, G.numTexels), N.coarseLayout, H.err);
      continue;
    }
    // boundary rows of the smoother
    N.bPtr.assign(1, 0);
    for (int b = 0; b < G.numBoundary; b++) {
      for (int k = N.bd.ptr[b]; k < N.bd.ptr[b + 1]; k++) { N.bCol.push_back(N.bd.col[k]); H.bsrc.push_back(k); }
      for (int k = N.bb.ptr[b]; k < N.bb.ptr[b + 1]; k++) { N.bCol.push_back(G.boundaryGlobal[N.bb.col[k]]); H.bsrc.push_back(-1 - k); }
      N.bPtr.push_back((int)N.bCol.size());
    }
    N.nBRow = (long long)H.bsrc.size();
    // boundary solver structure
    BoundarySymbolic& sym = N.sym;
    if (!build_boundary_symbolic(N.bb, N.bd, maxBlock, denseMax, sym, H.err)) {
      H.err = "level " + std::to_string(l) + ": " + H.err;
      continue;
    }
    if (sym.nb == 0) continue;
    N.invOffPadHost.assign(sym.nSub + 1, 0);
    H.m.resize(sym.nSub);
    H.t.resize(sym.nSub);
    for (int p = 0; p < sym.nSub; p++) {
      H.m[p] = sym.subPtr[p + 1] - sym.subPtr[p];
      H.t[p] = sym.touchPtr[p + 1] - sym.touchPtr[p];
      N.invOffPadHost[p + 1] = N.invOffPadHost[p] + (long long)H.m[p] * ((H.m[p] + 3) & ~3);
    }
    std::vector<int64_t> invOff(sym.invOff.begin(), sym.invOff.end() - 1);
    if (!dev::spd_inverse_layout(invOff, H.m, N.subLayout, H.err)) continue;
    if (sym.nS > 0 && !dev::spd_inverse_layout(std::vector<int64_t>(1, 0), std::vector<int>(1, sym.nS), N.schurLayout, H.err)) continue;
    std::vector<int64_t> cOff(sym.wOff.begin(), sym.wOff.end() - 1), lOff(sym.lOff.begin(), sym.lOff.end() - 1);
    dev::schur_product_tasks(invOff, H.m, cOff, H.t, lOff, N.gTasks, N.lTasks, N.maxM, N.maxT);
  }
  for (const LevelHost& H : host)
    if (!H.err.empty()) {
      err = H.err;
      return false;
    }
  // ---- resident sources and structure arrays (device)
  auto layout_dev = [&](const dev::SpdInverseLayout& Ly) -> dev::SpdInverseDevice {
    return {A.upload(as_ll(Ly.offsets)), A.upload(Ly.sizes), A.upload(as_ll(Ly.first)), A.upload(as_ll(Ly.ws)), A.upload(Ly.tasks)};
  };
  for (int l = 0; l < L; l++) {
    NumericLevel& N = levels[l];
    const LevelHost& H = host[l];
    N.deepM = (l == 0 && deep0M) ? deep0M : A.upload(l == 0 ? fine.deepMass : coM[l].deep);
    N.deepS = (l == 0 && deep0S) ? deep0S : A.upload(l == 0 ? fine.deepStiffness : coS[l].deep);
    N.bbM = A.upload(N.bb.val);
    N.bbS = A.upload(H.bbS.val);
    N.bdM = A.upload(N.bd.val);
    N.bdS = A.upload(H.bdS.val);
    N.bbV = static_cast<double*>(A.alloc(std::max<long long>(1, N.nBB) * sizeof(double)));
    N.bdV = static_cast<double*>(A.alloc(std::max<long long>(1, N.nBD) * sizeof(double)));
    if (N.coarsest) {
      N.nDense = (long long)H.denseSrc.size();
      N.denseSrc = A.upload(H.denseSrc);
      N.diagSrc = A.upload(H.diagSrc);
      N.denseRow = A.upload(H.denseRow);
      N.denseCol = A.upload(H.denseCol);
      N.coarseDev = layout_dev(N.coarseLayout);
      continue;
    }
    N.bSrc = A.upload(H.bsrc);
    const BoundarySymbolic& sym = N.sym;
    if (sym.nb == 0) continue;
    N.pos = A.upload(sym.pos);
    N.order = A.upload(sym.order);
    N.bbRow = A.upload(sym.bbRow);
    N.bbCol = A.upload(N.bb.col);
    N.diagEntry = A.upload(sym.diagEntry);
    N.fillEntry = A.upload(sym.fillEntry);
    N.fillDest = A.upload(as_ll(sym.fillDest));
    N.ssEntry = A.upload(sym.ssEntry);
    N.ssDest = A.upload(as_ll(sym.ssDest));
    N.aisEntry = A.upload(as_int(sym.AIS.val));
    N.aisDest = A.upload(as_ll(sym.aisDest));
    N.asiEntry = A.upload(as_int(sym.ASI.val));
    N.bdEntry = A.upload(as_int(sym.BD.val));
    N.subPtr = A.upload(sym.subPtr);
    N.touchPtr = A.upload(sym.touchPtr);
    N.touch = A.upload(sym.touch);
    N.wOff = A.upload(as_ll(sym.wOff));
    N.lOff = A.upload(as_ll(sym.lOff));
    N.invOff = A.upload(as_ll(sym.invOff));
    N.invOffPad = A.upload(N.invOffPadHost);
    N.subDev = layout_dev(N.subLayout);
    if (sym.nS > 0) N.schurDev = layout_dev(N.schurLayout);
    N.gTasksDev = A.upload(N.gTasks);
    N.lTasksDev = A.upload(N.lTasks);
  }
  if (A.last != cudaSuccess) {
    err = std::string("numeric plan upload: ") + cudaGetErrorString(A.last);
    return false;
  }
  return true;
}

bool NumericPlan::set_run_order(int l, const std::vector<int>& runTexel, std::string& err) {
  NumericLevel& N = levels[l];
  if (N.runTexel && N.runCount == (int)runTexel.size()) return true;  // the runs are a function of the level's structure
  N.runTexel = arena_->upload(runTexel);
  N.runCount = (int)runTexel.size();
  if (arena_->last != cudaSuccess) {
    err = std::string("run order upload: ") + cudaGetErrorString(arena_->last);
    return false;
  }
  return true;
}

bool NumericPlan::combine(double a, double b, cudaStream_t s, std::string& err) {
  screen = a;
  stiffness = b;
  for (NumericLevel& N : levels) {
    if (N.nBB) k_combine<<<blocks_for(N.nBB), kThreads, 0, s>>>(N.nBB, a, N.bbM, b, N.bbS, N.bbV);
    if (N.nBD) k_combine<<<blocks_for(N.nBD), kThreads, 0, s>>>(N.nBD, a, N.bdM, b, N.bdS, N.bdV);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) err = std::string("combine: ") + cudaGetErrorString(e);
  return e == cudaSuccess;
}

bool NumericPlan::fill_raw_rows(double* bVal, cudaStream_t s, std::string& err) {
  const NumericLevel& N = levels[0];
  if (N.nBRow) k_gather_rows<double><<<blocks_for(N.nBRow), kThreads, 0, s>>>(N.nBRow, N.bSrc, N.bdV, N.bbV, bVal);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) err = std::string("operator rows: ") + cudaGetErrorString(e);
  return e == cudaSuccess;
}

namespace {

template <typename T>
void convert_boundary(const NumericLevel& N, const BoundarySymbolic& sym, const Scaled& sc, const double* invS, const double* G,
                      const double* Ss, const double* scale64, LevelValues<T>& v, cudaStream_t s) {
  if (sym.nSub > 0) {
    k_pad_blocks<T><<<sym.nSub, kThreads, 0, s>>>(N.subPtr, N.invOff, N.invOffPad, invS, v.inv);
    k_wt<T><<<sym.nSub, kThreads, 0, s>>>(N.subPtr, N.touchPtr, N.wOff, G, v.wt);
  }
  if (sym.nS > 0) {
    const long long e = (long long)sym.nS * v.nSp;
    k_pad_square<T><<<blocks_for(e), kThreads, 0, s>>>(sym.nS, v.nSp, Ss, v.sinv);
  }
  k_convert<T><<<blocks_for(sym.nb), kThreads, 0, s>>>(sym.nb, scale64, v.scale);
  const long long nAsi = (long long)sym.ASI.col.size(), nBd = (long long)sym.BD.col.size();
  if (nAsi) k_scaled_values<T><<<blocks_for(nAsi), kThreads, 0, s>>>(nAsi, N.asiEntry, sc, v.asiVal);
  if (nBd) k_gather_values<T><<<blocks_for(nBd), kThreads, 0, s>>>(nBd, N.bdEntry, N.bdV, v.bdVal);
}

}  // namespace

void keep_pool_memory() {
  static std::atomic<int> slots[dev::kMaxDevices];
  static const bool init = [] {
    for (auto& a : slots) a.store(dev::kUnset);
    return true;
  }();
  (void)init;
  dev::per_device_once(slots, [] {
    int d = 0;
    cudaMemPool_t pool;
    if (cudaGetDevice(&d) != cudaSuccess || cudaDeviceGetDefaultMemPool(&pool, d) != cudaSuccess) return 1;
    uint64_t keep = ~0ULL;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    return 1;
  });
}

bool NumericPlan::fill_level(int l, LevelValues<float>* f32, LevelValues<double>* f64, cudaStream_t s, std::string& err) {
  const NumericLevel& N = levels[l];
  StreamScratch S(s);
  int* bad = S.get<int>(1);
  if (!bad) {
    err = std::string("numeric scratch: ") + cudaGetErrorString(S.last);
    return false;
  }
  cudaMemsetAsync(bad, 0, sizeof(int), s);
  auto settle = [&](const char* what) -> bool {
    int badHost = 0;
    cudaError_t e = cudaMemcpyAsync(&badHost, bad, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess || S.last != cudaSuccess) {
      err = std::string(what) + ": " + cudaGetErrorString(e != cudaSuccess ? e : S.last);
      return false;
    }
    if (badHost) {
      err = std::string(what) + ": not positive definite";
      return false;
    }
    return true;
  };
  double t = wall_ms();
  auto lap = [&](int slot) {
    const double now = wall_ms();
    ms[slot] += now - t;
    t = now;
  };
  const Sources src{screen, stiffness, N.deepM, N.deepS, N.bdV, N.bbV};
  if (N.coarsest) {
    const int n = N.n;
    double* scale = f64 ? f64->coarseScale : f32->coarseScale;
    double* inv = f64 ? f64->coarseInv : f32->coarseInv;
    double* dense = S.get<double>(size_t(n) * n);
    double* scratch = S.get<double>(dev::spd_inverse_scratch_doubles(N.coarseLayout));
    if (!dense || !scratch) return settle("coarsest scratch");
    k_coarse_scale<<<blocks_for(n), kThreads, 0, s>>>(n, N.diagSrc, src, scale);
    cudaMemsetAsync(dense, 0, size_t(n) * n * sizeof(double), s);
    k_coarse_fill<<<blocks_for(N.nDense), kThreads, 0, s>>>(N.nDense, n, N.denseSrc, N.denseRow, N.denseCol, src, scale, dense);
    lap(0);
    if (!dev::launch_spd_inverse(N.coarseLayout, N.coarseDev, dense, inv, scratch, bad, s)) return settle("coarsest inverse launch");
    if (f64 && f32) {
      cudaMemcpyAsync(f32->coarseInv, inv, size_t(n) * n * sizeof(double), cudaMemcpyDeviceToDevice, s);
      cudaMemcpyAsync(f32->coarseScale, scale, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
    }
    const bool ok = settle("coarsest inverse");
    lap(3);
    return ok;
  }
  // smoother planes and boundary rows
  if (N.runCount > 0) {
    if (f32) k_planes<float><<<blocks_for(N.runCount), kThreads, 0, s>>>(N.runCount, N.runTexel, N.deepM, N.deepS, screen, stiffness, f32->planes);
    if (f64) k_planes<double><<<blocks_for(N.runCount), kThreads, 0, s>>>(N.runCount, N.runTexel, N.deepM, N.deepS, screen, stiffness, f64->planes);
  }
  if (N.nBRow) {
    if (f32) k_gather_rows<float><<<blocks_for(N.nBRow), kThreads, 0, s>>>(N.nBRow, N.bSrc, N.bdV, N.bbV, f32->bVal);
    if (f64) k_gather_rows<double><<<blocks_for(N.nBRow), kThreads, 0, s>>>(N.nBRow, N.bSrc, N.bdV, N.bbV, f64->bVal);
  }
  const BoundarySymbolic& sym = N.sym;
  if (sym.nb == 0) {
    const bool ok = settle("level values");
    lap(0);
    return ok;
  }
  // boundary solver: scaled subdomain blocks, their inverses
  double* scale64 = S.get<double>(sym.nb);
  const long long elems = std::max<long long>(1, N.subLayout.elems);
  double* blk = S.get<double>(elems);
  double* invS = S.get<double>(elems);
  const long long wTotal = std::max<int64_t>(1, sym.wOff.back()), lTotal = std::max<int64_t>(1, sym.lOff.back());
  double* C = S.get<double>(wTotal);
  double* G = S.get<double>(wTotal);
  double* Lc = S.get<double>(lTotal);
  double* subScratch = S.get<double>(std::max<size_t>(1, dev::spd_inverse_scratch_doubles(N.subLayout)));
  if (!scale64 || !blk || !invS || !C || !G || !Lc || !subScratch) return settle("boundary scratch");
  k_scale_pos<<<blocks_for(sym.nb), kThreads, 0, s>>>(sym.nb, N.order, N.diagEntry, N.bbV, scale64);
  const Scaled sc{N.bbV, N.bbRow, N.bbCol, N.pos, scale64};
  cudaMemsetAsync(blk, 0, size_t(elems) * sizeof(double), s);
  const long long nFill = (long long)sym.fillEntry.size();
  if (nFill) k_scatter_scaled<<<blocks_for(nFill), kThreads, 0, s>>>(nFill, N.fillEntry, N.fillDest, sc, blk);
  if (!settle("boundary values")) return false;
  lap(0);
  if (!dev::launch_spd_inverse(N.subLayout, N.subDev, blk, invS, subScratch, bad, s)) return settle("subdomain inverse launch");
  if (!settle("boundary subdomain inverses")) return false;
  lap(1);
  // couplings, back-substitution blocks G_p = Inv_p C_p, Schur complement
  cudaMemsetAsync(C, 0, size_t(wTotal) * sizeof(double), s);
  const long long nAis = (long long)sym.aisDest.size();
  if (nAis) k_scatter_scaled<<<blocks_for(nAis), kThreads, 0, s>>>(nAis, N.aisEntry, N.aisDest, sc, C);
  dev::launch_gemm_batch(N.gTasksDev, (int)N.gTasks.size(), N.maxM, N.maxT, invS, C, G, s);
  double* Ss = nullptr;
  double* Sm = nullptr;
  double* schurScratch = nullptr;
  if (sym.nS > 0) {
    const int nS = sym.nS;
    dev::launch_gemm_batch(N.lTasksDev, (int)N.lTasks.size(), N.maxT, N.maxT, C, G, Lc, s);
    Sm = S.get<double>(size_t(nS) * nS);
    Ss = S.get<double>(size_t(nS) * nS);
    schurScratch = S.get<double>(dev::spd_inverse_scratch_doubles(N.schurLayout));
    if (!Sm || !Ss || !schurScratch) return settle("Schur scratch");
    cudaMemsetAsync(Sm, 0, size_t(nS) * nS * sizeof(double), s);
    const long long nSS = (long long)sym.ssEntry.size();
    if (nSS) k_scatter_scaled<<<blocks_for(nSS), kThreads, 0, s>>>(nSS, N.ssEntry, N.ssDest, sc, Sm);
    if (sym.nSub > 0) k_schur_subtract<<<(nS + kRowsPerBlock - 1) / kRowsPerBlock, kThreads, 0, s>>>(nS, sym.nSub, N.touchPtr, N.touch, N.lOff, Lc, Sm);
    k_symmetrise_pairs<<<blocks_for((long long)nS * nS), kThreads, 0, s>>>(nS, Sm);
  }
  if (!settle("boundary Schur products")) return false;
  lap(2);
  if (sym.nS > 0) {
    if (!dev::launch_spd_inverse(N.schurLayout, N.schurDev, Sm, Ss, schurScratch, bad, s)) return settle("Schur inverse launch");
    if (!settle("boundary Schur complement inverse")) return false;
  }
  lap(3);
  if (f32) convert_boundary(N, sym, sc, invS, G, Ss, scale64, *f32, s);
  if (f64) convert_boundary(N, sym, sc, invS, G, Ss, scale64, *f64, s);
  const bool ok = settle("boundary solver values");
  lap(0);
  return ok;
}

}  // namespace gdtp
