// Dense FP64 set-up products on the device: the inverses and products of the
// exact boundary-block solve and the coarsest-level inverse (setup/bsolve.cpp,
// system.cu), which the reference factorises with Eigen's SimplicialLDLT
// (UpdateCoefficients.inl:402-439, Solver.h:144-259).
//
// Inverse: blocked Gauss-Jordan elimination without pivoting (the matrices are
// symmetric positive definite, so every pivot block is a principal block of a
// Schur complement, itself SPD).  Step k takes the 64 pivot rows and columns
// K = [64k, 64k + 64):
//   P    = A[K,K]^-1                                  (k_bgj_diag, one CTA)
//   R    = P [A[K,:] with A[K,K] replaced by I]       (k_bgj_panel, row tiles)
//   Cold = A[:,K] with rows K zeroed; A[i,K] = 0, i not in K (k_bgj_panel)
//   A[K,:] = R;  A -= Cold R                          (k_gemm, rank-64 update)
// after which A[K,K] = P, A[K,j] = P A[K,j], A[i,K] = -A[i,K] P and
// A[i,j] -= A[i,K] P A[K,j]: the n/64 steps leave A^-1.  Every matrix of a
// batch takes part in the steps k < ceil(m/64); the update is 2 n^3 flops in
// 64 x 64 register-tiled FP64 tiles.  A non-positive pivot sets an error flag
// (and the result is discarded).  The result is made exactly symmetric by
// averaging with its transpose.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "vcycle_kernels.h"

namespace gdtp {
namespace dev {
namespace {

constexpr int kPB = 64;  // pivot block of the blocked Gauss-Jordan elimination

// C (M x N) = alpha op(A) B + beta C over a batch of tasks (blockIdx.z); op(A)
// is A (M x K, leading dimension lda) or, with transA, the transpose of A
// stored K x M.  64 x 64 tiles, 256 threads of 4 x 4 outputs each (rows ty +
// 16 r, columns tx + 16 c), K in chunks of 16 through shared memory.
__global__ void __launch_bounds__(256) k_gemm(const GemmTask* __restrict__ tasks, const double* __restrict__ A,
                                              const double* __restrict__ B, double* __restrict__ C) {
  const GemmTask T = tasks[blockIdx.z];
  const int row0 = blockIdx.y * 64, col0 = blockIdx.x * 64;
  if (row0 >= T.M || col0 >= T.N) return;
  __shared__ double As[16][64 + 1], Bs[16][64];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  double acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int c = 0; c < 4; c++) acc[r][c] = 0.0;
  const double* Ab = A + T.a;
  const double* Bb = B + T.b;
  for (int k0 = 0; k0 < T.K; k0 += 16) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int e = tid + 256 * q;
      double av = 0.0;
      if (T.transA) {  // A stored K x M: consecutive threads along the rows of the tile
        const int kk = e >> 6, rr = e & 63, gr = row0 + rr, gk = k0 + kk;
        if (gr < T.M && gk < T.K) av = Ab[(long long)gk * T.lda + gr];
        As[kk][rr] = av;
      } else {  // A stored M x K: consecutive threads along k
        const int rr = e >> 4, kk = e & 15, gr = row0 + rr, gk = k0 + kk;
        if (gr < T.M && gk < T.K) av = Ab[(long long)gr * T.lda + gk];
        As[kk][rr] = av;
      }
      const int kk = e >> 6, cc = e & 63, gk = k0 + kk, gc = col0 + cc;
      Bs[kk][cc] = (gk < T.K && gc < T.N) ? Bb[(long long)gk * T.ldb + gc] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; kk++) {
      double a[4], b[4];
#pragma unroll
      for (int r = 0; r < 4; r++) a[r] = As[kk][ty + 16 * r];
#pragma unroll
      for (int c = 0; c < 4; c++) b[c] = Bs[kk][tx + 16 * c];
#pragma unroll
      for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[r][c] = fma(a[r], b[c], acc[r][c]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int gr = row0 + ty + 16 * r;
    if (gr >= T.M) continue;
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int gc = col0 + tx + 16 * c;
      if (gc >= T.N) continue;
      double* dst = C + T.c + (long long)gr * T.ldc + gc;
      *dst = T.alpha * acc[r][c] + (T.beta != 0.0 ? T.beta * *dst : 0.0);
    }
  }
}

// P_q = A_q[K,K]^-1 for every matrix q with m_q > 64k (one CTA each):
// unblocked Gauss-Jordan on the pivot block, held in registers.
__global__ void __launch_bounds__(256) k_bgj_diag(int k, const long long* __restrict__ off, const int* __restrict__ size,
                                                  const double* __restrict__ A, double* __restrict__ Pinv, int* __restrict__ bad) {
  const int q = blockIdx.x, m = size[q], kb = k * kPB;
  if (kb >= m) return;
  const int bs = min(kPB, m - kb);
  // thread (tr, tc) holds entries (tr + 16 a, tc + 16 b), a, b < 4, in
  // registers; the pivot row and column of each step go through shared
  // memory, double-buffered so that one barrier per step orders them
  const int tr = threadIdx.x >> 4, tc = threadIdx.x & 15;
  __shared__ double rowS[2][kPB], colS[2][kPB];
  const double* Aq = A + off[q];
  double P[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) {
      const int i = tr + 16 * a, j = tc + 16 * b;
      P[a][b] = (i < bs && j < bs) ? Aq[(long long)(kb + i) * m + kb + j] : 0.0;
    }
  for (int s = 0; s < bs; s++) {
    const int buf = s & 1;
    // the pivot row s and column s as they stand before step s
#pragma unroll
    for (int a = 0; a < 4; a++)
      if (tr + 16 * a == s)
#pragma unroll
        for (int b = 0; b < 4; b++) rowS[buf][tc + 16 * b] = P[a][b];
#pragma unroll
    for (int b = 0; b < 4; b++)
      if (tc + 16 * b == s)
#pragma unroll
        for (int a = 0; a < 4; a++) colS[buf][tr + 16 * a] = P[a][b];
    __syncthreads();
    double p = rowS[buf][s];
    if (!(p > 0.0)) {
      if (threadIdx.x == 0) atomicExch(bad, 1);
      p = 1.0;
    }
    const double ip = 1.0 / p;
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) {
        const int i = tr + 16 * a, j = tc + 16 * b;
        if (i >= bs || j >= bs) continue;
        double v;
        if (i == s && j == s) v = ip;
        else if (i == s) v = rowS[buf][j] * ip;
        else if (j == s) v = -colS[buf][i] * ip;
        else v = P[a][b] - colS[buf][i] * (rowS[buf][j] * ip);
        P[a][b] = v;
      }
  }
  double* Pq = Pinv + (long long)q * kPB * kPB;
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) Pq[(tr + 16 * a) * kPB + tc + 16 * b] = P[a][b];
}

// blockIdx.y == 0: row tile t of R = P [A[K,:], A[K,K] -> I], written to R
// (64 x m per matrix) and to A[K,:].  blockIdx.y == 1: row tile t of
// Cold = A[:,K] (rows K zeroed, 64 columns per row), A[i,K] = 0 for i not in K.
// The two roles touch disjoint entries of A (rows K, and columns K outside rows K).
__global__ void __launch_bounds__(256) k_bgj_panel(int k, const long long* __restrict__ off, const int* __restrict__ size,
                                                   const long long* __restrict__ wsOff, double* __restrict__ A,
                                                   const double* __restrict__ Pinv, double* __restrict__ R, double* __restrict__ Cold) {
  const int q = blockIdx.z, m = size[q], kb = k * kPB;
  if (kb >= m) return;
  const int bs = min(kPB, m - kb), t0 = blockIdx.x * kPB;
  if (t0 >= m) return;
  double* Aq = A + off[q];
  if (blockIdx.y == 1) {
    double* Cq = Cold + wsOff[q];
    for (int e = threadIdx.x; e < kPB * kPB; e += 256) {
      const int i = t0 + e / kPB, c = e % kPB;
      if (i >= m) continue;
      double v = 0.0;
      if (c < bs && (i < kb || i >= kb + bs)) {
        double* src = Aq + (long long)i * m + kb + c;
        v = *src;
        *src = 0.0;
      }
      Cq[(long long)i * kPB + c] = v;
    }
    return;
  }
  extern __shared__ double sm[];
  double(*Ps)[kPB + 1] = reinterpret_cast<double(*)[kPB + 1]>(sm);
  double(*Xs)[kPB + 1] = reinterpret_cast<double(*)[kPB + 1]>(sm + kPB * (kPB + 1));
  const double* Pq = Pinv + (long long)q * kPB * kPB;
  for (int e = threadIdx.x; e < kPB * kPB; e += 256) {
    const int r = e / kPB, c = e % kPB, j = t0 + c;
    Ps[r][c] = Pq[e];
    double x = 0.0;
    if (r < bs && j < m) x = (j >= kb && j < kb + bs) ? (j - kb == r ? 1.0 : 0.0) : Aq[(long long)(kb + r) * m + j];
    Xs[r][c] = x;
  }
  __syncthreads();
  double* Rq = R + wsOff[q];
  for (int e = threadIdx.x; e < kPB * kPB; e += 256) {
    const int r = e / kPB, c = e % kPB, j = t0 + c;
    if (r >= bs || j >= m) continue;
    double v = 0.0;
    for (int d = 0; d < bs; d++) v = fma(Ps[r][d], Xs[d][c], v);
    Rq[(long long)r * m + j] = v;
    Aq[(long long)(kb + r) * m + j] = v;
  }
}

__global__ void k_symmetrise(int nMat, const long long* __restrict__ off, const int* __restrict__ size,
                             const long long* __restrict__ first, long long total, const double* __restrict__ in, double* __restrict__ out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  int lo = 0, hi = nMat - 1;  // the matrix of item t: last with first[q] <= t
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (first[mid] <= t) lo = mid; else hi = mid - 1;
  }
  const int m = size[lo];
  const long long e = t - first[lo];
  const int i = int(e / m), j = int(e - (long long)i * m);
  const double* A = in + off[lo];
  out[off[lo] + e] = 0.5 * (A[e] + A[(long long)j * m + i]);
}

// stream-ordered scratch (no device-wide synchronisation on release, so the
// set-up of one system does not wait for the solves of others)
struct Buf {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  ~Buf() {
    if (p) cudaFreeAsync(p, s);
  }
  template <class T>
  T* as() const { return static_cast<T*>(p); }
};

bool check(cudaError_t e, const char* what, std::string& err) {
  if (e == cudaSuccess) return true;
  err = std::string(what) + ": " + cudaGetErrorString(e);
  return false;
}

bool alloc(Buf& b, size_t bytes, cudaStream_t s, std::string& err) {
  b.s = s;
  return check(cudaMallocAsync(&b.p, std::max<size_t>(16, bytes), s), "cudaMallocAsync", err);
}

template <class T>
bool upload(Buf& b, const T* v, size_t n, cudaStream_t s, std::string& err) {
  if (!alloc(b, n * sizeof(T), s, err)) return false;
  return n == 0 || check(cudaMemcpyAsync(b.p, v, n * sizeof(T), cudaMemcpyHostToDevice, s), "h2d", err);
}
template <class T>
bool upload(Buf& b, const std::vector<T>& v, cudaStream_t s, std::string& err) {
  return upload(b, v.data(), v.size(), s, err);
}

constexpr int kMaxGridZ = 65535;

}  // namespace

void launch_gemm_batch(const GemmTask* dTasks, int nTasks, int maxM, int maxN, const double* A, const double* B, double* C,
                       cudaStream_t s) {
  for (int t0 = 0; t0 < nTasks; t0 += kMaxGridZ) {
    const dim3 grid(unsigned((maxN + 63) / 64), unsigned((maxM + 63) / 64), unsigned(std::min(kMaxGridZ, nTasks - t0)));
    k_gemm<<<grid, 256, 0, s>>>(dTasks + t0, A, B, C);
  }
}

bool spd_inverse_layout(const std::vector<int64_t>& offsets, const std::vector<int>& sizes, SpdInverseLayout& L, std::string& err) {
  L = SpdInverseLayout();
  L.nMat = (int)sizes.size();
  if (L.nMat > kMaxGridZ) {
    err = "more dense blocks than one launch holds";
    return false;
  }
  L.offsets = offsets;
  L.sizes = sizes;
  L.first.resize(L.nMat);
  L.ws.resize(L.nMat);
  int mMax = 0;
  for (int q = 0; q < L.nMat; q++) {
    L.first[q] = L.total;
    L.ws[q] = L.wsTotal;
    L.total += (long long)sizes[q] * sizes[q];
    L.wsTotal += (long long)kPB * sizes[q];
    L.elems = std::max<long long>(L.elems, offsets[q] + (long long)sizes[q] * sizes[q]);
    mMax = std::max(mMax, sizes[q]);
  }
  L.steps = (mMax + kPB - 1) / kPB;
  // rank-64 update tasks of every step: A_q -= Cold_q R_q over the matrices still eliminating
  L.taskStart.assign(L.steps + 1, 0);
  L.stepMax.assign(L.steps, 0);
  for (int k = 0; k < L.steps; k++) {
    for (int q = 0; q < L.nMat; q++) {
      const int m = sizes[q], kb = k * kPB;
      if (kb >= m) continue;
      GemmTask T{};
      T.a = L.ws[q];
      T.b = L.ws[q];
      T.c = offsets[q];
      T.M = T.N = m;
      T.K = std::min(kPB, m - kb);
      T.lda = kPB;
      T.ldb = m;
      T.ldc = m;
      T.alpha = -1.0;
      T.beta = 1.0;
      L.tasks.push_back(T);
      L.stepMax[k] = std::max(L.stepMax[k], m);
    }
    L.taskStart[k + 1] = (int)L.tasks.size();
  }
  return true;
}

size_t spd_inverse_scratch_doubles(const SpdInverseLayout& L) { return size_t(L.nMat) * kPB * kPB + 2 * size_t(L.wsTotal); }

bool launch_spd_inverse(const SpdInverseLayout& L, const SpdInverseDevice& D, double* A, double* out, double* scratch, int* bad,
                        cudaStream_t s) {
  if (L.nMat == 0 || L.steps == 0) return true;
  static const int panelSmem = 2 * kPB * (kPB + 1) * sizeof(double);
  if (cudaFuncSetAttribute(k_bgj_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, panelSmem) != cudaSuccess) return false;
  double* pinv = scratch;
  double* rw = pinv + size_t(L.nMat) * kPB * kPB;
  double* cw = rw + L.wsTotal;
  for (int k = 0; k < L.steps; k++) {
    // matrices of size m <= 64k, and tiles past a matrix's own size, return at once
    k_bgj_diag<<<L.nMat, 256, 0, s>>>(k, D.off, D.size, A, pinv, bad);
    const dim3 pg(unsigned((L.stepMax[k] + kPB - 1) / kPB), 2, unsigned(L.nMat));
    k_bgj_panel<<<pg, 256, panelSmem, s>>>(k, D.off, D.size, D.ws, A, pinv, rw, cw);
    launch_gemm_batch(D.tasks + L.taskStart[k], L.taskStart[k + 1] - L.taskStart[k], L.stepMax[k], L.stepMax[k], cw, rw, A, s);
  }
  const unsigned blocks = unsigned((L.total + 255) / 256);
  k_symmetrise<<<blocks, 256, 0, s>>>(L.nMat, D.off, D.size, D.first, L.total, A, out);
  return cudaGetLastError() == cudaSuccess;
}

namespace {

// device copies of a layout's arrays in stream-ordered scratch
struct LayoutUpload {
  Buf off, size, first, ws, tasks;
  SpdInverseDevice dev;
  bool run(const SpdInverseLayout& L, cudaStream_t s, std::string& err) {
    if (!upload(off, L.offsets, s, err) || !upload(size, L.sizes, s, err) || !upload(first, L.first, s, err) ||
        !upload(ws, L.ws, s, err) || !upload(tasks, L.tasks, s, err))
      return false;
    dev = {off.as<long long>(), size.as<int>(), first.as<long long>(), ws.as<long long>(), tasks.as<GemmTask>()};
    return true;
  }
};

}  // namespace

bool gpu_spd_inverse_batched(double* data, const std::vector<int64_t>& offsets, const std::vector<int>& sizes, cudaStream_t s,
                             std::string& err) {
  SpdInverseLayout L;
  if (!spd_inverse_layout(offsets, sizes, L, err)) return false;
  if (L.nMat == 0 || L.steps == 0) return true;
  LayoutUpload U;
  Buf a, b, bad, scratch;
  if (!U.run(L, s, err) || !upload(a, data, size_t(L.elems), s, err) || !alloc(b, size_t(L.elems) * sizeof(double), s, err) ||
      !upload(bad, std::vector<int>(1, 0), s, err) || !alloc(scratch, spd_inverse_scratch_doubles(L) * sizeof(double), s, err))
    return false;
  if (!launch_spd_inverse(L, U.dev, a.as<double>(), b.as<double>(), scratch.as<double>(), bad.as<int>(), s)) {
    err = std::string("Gauss-Jordan: ") + cudaGetErrorString(cudaGetLastError());
    return false;
  }
  int badHost = 0;
  if (!check(cudaMemcpyAsync(&badHost, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s), "d2h", err) ||
      !check(cudaStreamSynchronize(s), "Gauss-Jordan", err))
    return false;
  if (badHost) {
    err = "dense block is not positive definite";
    return false;
  }
  for (int q = 0; q < L.nMat; q++) {
    const size_t bytes = size_t(sizes[q]) * sizes[q] * sizeof(double);
    if (bytes && !check(cudaMemcpyAsync(data + offsets[q], b.as<double>() + offsets[q], bytes, cudaMemcpyDeviceToHost, s), "d2h", err))
      return false;
  }
  return check(cudaStreamSynchronize(s), "Gauss-Jordan", err);
}

void schur_product_tasks(const std::vector<int64_t>& invOff, const std::vector<int>& m, const std::vector<int64_t>& cOff,
                         const std::vector<int>& t, const std::vector<int64_t>& localOff, std::vector<GemmTask>& gTasks,
                         std::vector<GemmTask>& lTasks, int& maxM, int& maxT) {
  gTasks.clear();
  lTasks.clear();
  maxM = maxT = 1;
  for (size_t p = 0; p < m.size(); p++) {
    if (t[p] == 0 || m[p] == 0) continue;
    GemmTask g{};  // G = Inv C   (m x t)
    g.a = invOff[p];
    g.b = cOff[p];
    g.c = cOff[p];
    g.M = m[p];
    g.N = t[p];
    g.K = m[p];
    g.lda = m[p];
    g.ldb = t[p];
    g.ldc = t[p];
    g.alpha = 1.0;
    gTasks.push_back(g);
    GemmTask l{};  // local = C^T G   (t x t)
    l.a = cOff[p];
    l.b = cOff[p];
    l.c = localOff[p];
    l.M = t[p];
    l.N = t[p];
    l.K = m[p];
    l.lda = t[p];
    l.ldb = t[p];
    l.ldc = t[p];
    l.transA = 1;
    l.alpha = 1.0;
    lTasks.push_back(l);
    maxM = std::max(maxM, m[p]);
    maxT = std::max(maxT, t[p]);
  }
}

bool gpu_schur_products(const std::vector<double>& inv, const std::vector<int64_t>& invOff, const std::vector<int>& m,
                        const std::vector<double>& C, const std::vector<int64_t>& cOff, const std::vector<int>& t, std::vector<double>& G,
                        std::vector<double>& local, const std::vector<int64_t>& localOff, cudaStream_t s, std::string& err) {
  const int nSub = (int)m.size();
  G.assign(C.size(), 0.0);
  long long localTotal = 0;
  for (int p = 0; p < nSub; p++) localTotal = std::max<long long>(localTotal, localOff[p] + (long long)t[p] * t[p]);
  local.assign(size_t(localTotal), 0.0);
  std::vector<GemmTask> gTasks, lTasks;
  int maxM = 1, maxT = 1;
  schur_product_tasks(invOff, m, cOff, t, localOff, gTasks, lTasks, maxM, maxT);
  if (gTasks.empty()) return true;
  Buf dInv, dC, dG, dL, dgt, dlt;
  if (!upload(dInv, inv, s, err) || !upload(dC, C, s, err) || !alloc(dG, C.size() * sizeof(double), s, err) ||
      !alloc(dL, size_t(localTotal) * sizeof(double), s, err) || !upload(dgt, gTasks, s, err) || !upload(dlt, lTasks, s, err))
    return false;
  launch_gemm_batch(dgt.as<GemmTask>(), (int)gTasks.size(), maxM, maxT, dInv.as<double>(), dC.as<double>(), dG.as<double>(), s);
  launch_gemm_batch(dlt.as<GemmTask>(), (int)lTasks.size(), maxT, maxT, dC.as<double>(), dG.as<double>(), dL.as<double>(), s);
  if (!check(cudaGetLastError(), "products", err) ||
      !check(cudaMemcpyAsync(G.data(), dG.p, G.size() * sizeof(double), cudaMemcpyDeviceToHost, s), "d2h", err) ||
      !check(cudaMemcpyAsync(local.data(), dL.p, local.size() * sizeof(double), cudaMemcpyDeviceToHost, s), "d2h", err) ||
      !check(cudaStreamSynchronize(s), "products", err))
    return false;
  return true;
}

}  // namespace dev
}  // namespace gdtp
