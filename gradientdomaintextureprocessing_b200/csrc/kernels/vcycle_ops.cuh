// Per-item bodies of the V-cycle operators, shared by the one-launch-per-phase
// kernels (vcycle_kernels.cu) and the cluster-resident coarse-level kernel
// (coarse_cycle.cu), so both run the same arithmetic in the same order.
//
// An "item" is one texel (or boundary row) and one group of W channels; a
// launch or a cluster loop hands out item indices.  LD selects how mutable
// vectors (x, rhs, residual, boundary work) are read: LoadDefault for kernels
// that only read data written by earlier launches, LoadL2 (ld.global.cg, L2
// only) for the cluster kernel, whose phases read what other CTAs wrote in the
// previous phase of the same launch.
#pragma once
#include "vcycle.cuh"
#include "vcycle_kernels.h"

namespace gdtp {
namespace dev {

struct LoadDefault {
  template <typename T, int W>
  static __device__ __forceinline__ Vec<T, W> ld(const T* p) { return vload<T, W>(p); }
  template <typename T>
  static __device__ __forceinline__ T coef(const T* p) { return *p; }
  template <typename T, int W>
  static __device__ __forceinline__ void st(T* p, const Vec<T, W>& v) { vstore<T, W>(p, v); }
};

struct LoadL2 {
  template <typename T, int W>
  static __device__ __forceinline__ Vec<T, W> ld(const T* p);
  template <typename T>
  static __device__ __forceinline__ T coef(const T* p) { return *p; }
  template <typename T, int W>
  static __device__ __forceinline__ void st(T* p, const Vec<T, W>& v) { vstore<T, W>(p, v); }
};
template <>
__device__ __forceinline__ Vec<float, 4> LoadL2::ld<float, 4>(const float* p) {
  const float4 v = __ldcg(reinterpret_cast<const float4*>(p));
  Vec<float, 4> r;
  r.v[0] = v.x; r.v[1] = v.y; r.v[2] = v.z; r.v[3] = v.w;
  return r;
}
template <>
__device__ __forceinline__ Vec<float, 1> LoadL2::ld<float, 1>(const float* p) {
  Vec<float, 1> r;
  r.v[0] = __ldcg(p);
  return r;
}
template <>
__device__ __forceinline__ Vec<double, 4> LoadL2::ld<double, 4>(const double* p) {
  const double2 a = __ldcg(reinterpret_cast<const double2*>(p)), b = __ldcg(reinterpret_cast<const double2*>(p + 2));
  Vec<double, 4> r;
  r.v[0] = a.x; r.v[1] = a.y; r.v[2] = b.x; r.v[3] = b.y;
  return r;
}
template <>
__device__ __forceinline__ Vec<double, 1> LoadL2::ld<double, 1>(const double* p) {
  Vec<double, 1> r;
  r.v[0] = __ldcg(p);
  return r;
}

// Four consecutive entries of a dense-inverse row (one vector load).
template <typename T>
struct Quad;
template <>
struct __align__(16) Quad<float> {
  float v[4];
};
template <>
struct __align__(32) Quad<double> {
  double v[4];
};

template <typename T, int W>
__device__ __forceinline__ void axpy(Vec<T, W>& acc, T a, const Vec<T, W>& v) {
#pragma unroll
  for (int c = 0; c < W; c++) acc.v[c] += a * v.v[c];
}

// Gauss-Seidel update of one colour-run texel: x = rhs*c4 - sum_{k!=4} c_k x_k
// (IterativeSolvers.inl:449-463).  Items: runs x 32 x G.
template <typename T, int W, typename LD>
__device__ __forceinline__ void gs_item(const ColourRun* runs, int nRuns, const T* coef, int planeStride, const T* rhs, T* x,
                                        int KP, int G, long long t, int skip = 0) {
  const int per = 32 * G;
  const long long r = t / per;
  if (r >= nRuns) return;
  const int rem = int(t - r * per);
  const int m = rem / G, q = rem - m * G;
  const ColourRun R = runs[r];
  if (m >= R.len) return;
  const int pos = R.pos0 + 2 * m, pp = R.prev0 + 2 * m, pn = R.next0 + 2 * m;
  const T* c = coef + R.coef0 + m;
  const int off = q * W;
  Vec<T, W> acc;
#pragma unroll
  for (int k = 0; k < W; k++) acc.v[k] = 0;
  // skip: neighbour slots known to hold exact zeros (their terms add nothing)
  if (!(skip & 1)) axpy(acc, LD::coef(c + 0 * planeStride), LD::template ld<T, W>(x + (long long)(pp - 1) * KP + off));
  if (!(skip & 2)) axpy(acc, LD::coef(c + 1 * planeStride), LD::template ld<T, W>(x + (long long)(pp)*KP + off));
  if (!(skip & 4)) axpy(acc, LD::coef(c + 2 * planeStride), LD::template ld<T, W>(x + (long long)(pp + 1) * KP + off));
  if (!(skip & 8)) axpy(acc, LD::coef(c + 3 * planeStride), LD::template ld<T, W>(x + (long long)(pos - 1) * KP + off));
  if (!(skip & 32)) axpy(acc, LD::coef(c + 5 * planeStride), LD::template ld<T, W>(x + (long long)(pos + 1) * KP + off));
  if (!(skip & 64)) axpy(acc, LD::coef(c + 6 * planeStride), LD::template ld<T, W>(x + (long long)(pn - 1) * KP + off));
  if (!(skip & 128)) axpy(acc, LD::coef(c + 7 * planeStride), LD::template ld<T, W>(x + (long long)(pn)*KP + off));
  if (!(skip & 256)) axpy(acc, LD::coef(c + 8 * planeStride), LD::template ld<T, W>(x + (long long)(pn + 1) * KP + off));
  const T c4 = LD::coef(c + 4 * planeStride);
  const Vec<T, W> b = LD::template ld<T, W>(rhs + (long long)pos * KP + off);
  Vec<T, W> out;
#pragma unroll
  for (int k = 0; k < W; k++) out.v[k] = b.v[k] * c4 - acc.v[k];
  LD::template st<T, W>(x + (long long)pos * KP + off, out);
}

// Deep residual r = rhs - (sum_{k!=4} c_k x_k + x) * c9 (IterativeSolvers.inl:479-493).
// Items: runs x 32 x G (all colours).
template <typename T, int W, typename LD>
__device__ __forceinline__ void residual_deep_item(const ColourRun* runs, int nRuns, const T* coef, int planeStride, const T* rhs,
                                                   const T* x, T* res, int KP, int G, long long t) {
  const int per = 32 * G;
  const long long r = t / per;
  if (r >= nRuns) return;
  const int rem = int(t - r * per);
  const int m = rem / G, q = rem - m * G;
  const ColourRun R = runs[r];
  if (m >= R.len) return;
  const int pos = R.pos0 + 2 * m, pp = R.prev0 + 2 * m, pn = R.next0 + 2 * m;
  const T* c = coef + R.coef0 + m;
  const int off = q * W;
  Vec<T, W> acc = LD::template ld<T, W>(x + (long long)pos * KP + off);
  axpy(acc, LD::coef(c + 0 * planeStride), LD::template ld<T, W>(x + (long long)(pp - 1) * KP + off));
  axpy(acc, LD::coef(c + 1 * planeStride), LD::template ld<T, W>(x + (long long)(pp)*KP + off));
  axpy(acc, LD::coef(c + 2 * planeStride), LD::template ld<T, W>(x + (long long)(pp + 1) * KP + off));
  axpy(acc, LD::coef(c + 3 * planeStride), LD::template ld<T, W>(x + (long long)(pos - 1) * KP + off));
  axpy(acc, LD::coef(c + 5 * planeStride), LD::template ld<T, W>(x + (long long)(pos + 1) * KP + off));
  axpy(acc, LD::coef(c + 6 * planeStride), LD::template ld<T, W>(x + (long long)(pn - 1) * KP + off));
  axpy(acc, LD::coef(c + 7 * planeStride), LD::template ld<T, W>(x + (long long)(pn)*KP + off));
  axpy(acc, LD::coef(c + 8 * planeStride), LD::template ld<T, W>(x + (long long)(pn + 1) * KP + off));
  const T c9 = LD::coef(c + 9 * planeStride);
  const Vec<T, W> b = LD::template ld<T, W>(rhs + (long long)pos * KP + off);
  Vec<T, W> out;
#pragma unroll
  for (int k = 0; k < W; k++) out.v[k] = b.v[k] - acc.v[k] * c9;
  vstore<T, W>(res + (long long)pos * KP + off, out);
}

// Boundary residual r_B = rhs_B - [BD BB] x (IterativeSolvers.inl:549-555).  Items: rows x G.
template <typename T, int W, typename LD>
__device__ __forceinline__ void residual_boundary_item(const int* bPtr, const int* bCol, const T* bVal, const int* bGlobal, int nB,
                                                       const T* rhs, const T* x, T* res, int KP, int G, long long t) {
  const long long row = t / G;
  if (row >= nB) return;
  const int q = int(t - row * G), off = q * W;
  const int g = bGlobal[row];
  Vec<T, W> acc = LD::template ld<T, W>(rhs + (long long)g * KP + off);
  for (int k = bPtr[row]; k < bPtr[row + 1]; k++) axpy(acc, -bVal[k], LD::template ld<T, W>(x + (long long)bCol[k] * KP + off));
  vstore<T, W>(res + (long long)g * KP + off, acc);
}

// Full-weighting restriction of deep lines (IterativeSolvers.inl:1037-1053).  Items: runs x 32 x G.
template <typename T, int W, typename LD>
__device__ __forceinline__ void restrict_deep_item(const RestrictRun* runs, int nRuns, const T* res, T* coarseRhs, int KP, int G,
                                                   long long t) {
  const int per = 32 * G;
  const long long r = t / per;
  if (r >= nRuns) return;
  const int rem = int(t - r * per);
  const int m = rem / G, q = rem - m * G;
  const RestrictRun R = runs[r];
  if (m >= R.len) return;
  const int f = R.f0 + 2 * m, fp = R.fp0 + 2 * m, fn = R.fn0 + 2 * m, off = q * W;
  const Vec<T, W> a0 = LD::template ld<T, W>(res + (long long)f * KP + off);
  const Vec<T, W> e1 = LD::template ld<T, W>(res + (long long)fp * KP + off), e2 = LD::template ld<T, W>(res + (long long)(f - 1) * KP + off),
                  e3 = LD::template ld<T, W>(res + (long long)(f + 1) * KP + off), e4 = LD::template ld<T, W>(res + (long long)fn * KP + off);
  const Vec<T, W> d1 = LD::template ld<T, W>(res + (long long)(fp - 1) * KP + off),
                  d2 = LD::template ld<T, W>(res + (long long)(fp + 1) * KP + off),
                  d3 = LD::template ld<T, W>(res + (long long)(fn - 1) * KP + off),
                  d4 = LD::template ld<T, W>(res + (long long)(fn + 1) * KP + off);
  Vec<T, W> out;
#pragma unroll
  for (int k = 0; k < W; k++)
    out.v[k] = a0.v[k] + (e1.v[k] + e2.v[k] + e3.v[k] + e4.v[k]) * T(0.5) + (d1.v[k] + d2.v[k] + d3.v[k] + d4.v[k]) * T(0.25);
  vstore<T, W>(coarseRhs + (long long)(R.out0 + m) * KP + off, out);
}

// Sparse boundary restriction rows.  Items: rows x G.
template <typename T, int W, typename LD>
__device__ __forceinline__ void restrict_boundary_item(const int* rPtr, const int* rCol, const T* rVal, const int* rOut, int nB,
                                                       const T* res, T* coarseRhs, int KP, int G, long long t) {
  const long long row = t / G;
  if (row >= nB) return;
  const int q = int(t - row * G), off = q * W;
  Vec<T, W> acc;
#pragma unroll
  for (int k = 0; k < W; k++) acc.v[k] = 0;
  for (int k = rPtr[row]; k < rPtr[row + 1]; k++) axpy(acc, rVal[k], LD::template ld<T, W>(res + (long long)rCol[k] * KP + off));
  vstore<T, W>(coarseRhs + (long long)rOut[row] * KP + off, acc);
}

// Bilinear prolongation added to the fine iterate (IterativeSolvers.inl:1128-1151).  Items: runs x 32 x G.
template <typename T, int W, typename LD>
__device__ __forceinline__ void prolong_item(const ProlongRun* runs, int nRuns, const T* coarse, T* fine, int KP, int G, long long t) {
  const int per = 32 * G;
  const long long r = t / per;
  if (r >= nRuns) return;
  const int rem = int(t - r * per);
  const int m = rem / G, q = rem - m * G;
  const ProlongRun R = runs[r];
  if (m >= R.len) return;
  const int i = R.i0 + m, o = R.aligned ? 0 : 1, off = q * W;
  const int p = (i + o) / 2, n = (i + o + 1) / 2;
  T* dst = fine + (long long)(R.f0 + m) * KP + off;
  Vec<T, W> acc = LD::template ld<T, W>(dst);
  if (R.center >= 0) {
    const Vec<T, W> a = LD::template ld<T, W>(coarse + (long long)(R.center + p) * KP + off),
                    b = LD::template ld<T, W>(coarse + (long long)(R.center + n) * KP + off);
#pragma unroll
    for (int k = 0; k < W; k++) acc.v[k] += (a.v[k] + b.v[k]) * T(0.5);
  } else {
    const Vec<T, W> a = LD::template ld<T, W>(coarse + (long long)(R.prev + p) * KP + off),
                    b = LD::template ld<T, W>(coarse + (long long)(R.prev + n) * KP + off),
                    c = LD::template ld<T, W>(coarse + (long long)(R.next + p) * KP + off),
                    d = LD::template ld<T, W>(coarse + (long long)(R.next + n) * KP + off);
#pragma unroll
    for (int k = 0; k < W; k++) acc.v[k] += (a.v[k] + b.v[k] + c.v[k] + d.v[k]) * T(0.25);
  }
  vstore<T, W>(dst, acc);
}

// ---- exact boundary solve, short-latency form.  Every sparse row sum of the
// boundary solve (BD x, A_SI y, W_p xs) is split over an aligned group of 8
// lanes (lane l takes terms l, l+8, ...) and added by a fixed shuffle tree
// ((v0+v4)+(v2+v6))+((v1+v5)+(v3+v7)), so a row costs a couple of dependent
// loads instead of a chain as long as the row, and the result does not depend
// on which kernel or thread ran it.  Callers run whole warps (every lane
// reaches the shuffles; items past the end contribute zeros).
template <typename T, int W>
__device__ __forceinline__ Vec<T, W> group8_sum(Vec<T, W> v) {
#pragma unroll
  for (int s = 4; s >= 1; s >>= 1)
#pragma unroll
    for (int c = 0; c < W; c++) v.v[c] += __shfl_down_sync(0xffffffffu, v.v[c], s);
  return v;  // valid in lane 0 of the group
}

// rhat_k = s_k (rhs_k - sum_e BD_ke x_e) for position k; group item gi = (k, q)
template <typename T, int W, typename LD>
__device__ __forceinline__ void bs_prep_group(const BoundaryDev<T>& B, const T* rhs, const T* x, int KP, int G, long long gi,
                                              int lane8) {
  const long long k = gi / G;
  const int q = int(gi - k * G), off = q * W;
  const bool valid = k < B.nb;
  Vec<T, W> acc;
#pragma unroll
  for (int c = 0; c < W; c++) acc.v[c] = 0;
  if (valid)
    for (int e = B.bdPtr[k] + lane8; e < B.bdPtr[k + 1]; e += 8)
      axpy(acc, B.bdVal[e], LD::template ld<T, W>(x + (long long)B.bdCol[e] * KP + off));
  acc = group8_sum(acc);
  if (valid && lane8 == 0) {
    Vec<T, W> r = LD::template ld<T, W>(rhs + (long long)B.posGlobal[k] * KP + off);
    const T sc = B.scale[k];
#pragma unroll
    for (int c = 0; c < W; c++) r.v[c] = (r.v[c] - acc.v[c]) * sc;
    vstore<T, W>(B.rhat + k * KP + off, r);
  }
}

// Separator input t_j = rhat_{nI+j} - sum_e A_SI,je y_e (valid in lane8 0)
template <typename T, int W, typename LD>
__device__ __forceinline__ Vec<T, W> bs_schur_input_group(const BoundaryDev<T>& B, int j, bool valid, int KP, int off, int lane8) {
  Vec<T, W> acc;
#pragma unroll
  for (int c = 0; c < W; c++) acc.v[c] = 0;
  if (valid)
    for (int e = B.asiPtr[j] + lane8; e < B.asiPtr[j + 1]; e += 8)
      axpy(acc, B.asiVal[e], LD::template ld<T, W>(B.y + (long long)B.asiCol[e] * KP + off));
  acc = group8_sum(acc);
  Vec<T, W> r;
#pragma unroll
  for (int c = 0; c < W; c++) r.v[c] = 0;
  if (valid && lane8 == 0) {
    r = LD::template ld<T, W>(B.rhat + (long long)(B.nI + j) * KP + off);
#pragma unroll
    for (int c = 0; c < W; c++) r.v[c] -= acc.v[c];
  }
  return r;
}

// Back substitution x_I = s (y - W_p xs) for interior position i; group item gi = (i, q)
template <typename T, int W, typename LD>
__device__ __forceinline__ void bs_back_group(const BoundaryDev<T>& B, T* x, int KP, int G, long long gi, int lane8) {
  const long long i = gi / G;
  const int q = int(gi - i * G), off = q * W;
  const bool valid = i < B.nI;
  Vec<T, W> acc;
#pragma unroll
  for (int c = 0; c < W; c++) acc.v[c] = 0;
  int p = 0, m = 0, a = 0;
  if (valid) {
    p = B.rowSub[i];
    const int b0 = B.subPtr[p];
    m = B.subPtr[p + 1] - b0;
    a = int(i) - b0;
    const T* Wp = B.wt + B.wOff[p] + a;
    const int e0 = B.touchPtr[p], e1 = B.touchPtr[p + 1];
    for (int e = e0 + lane8; e < e1; e += 8)
      axpy(acc, Wp[(long long)(e - e0) * m], LD::template ld<T, W>(B.xs + (long long)B.touch[e] * KP + off));
  }
  acc = group8_sum(acc);
  if (valid && lane8 == 0) {
    Vec<T, W> r = LD::template ld<T, W>(B.y + i * KP + off);
    const T sc = B.scale[i];
#pragma unroll
    for (int c = 0; c < W; c++) r.v[c] = (r.v[c] - acc.v[c]) * sc;
    vstore<T, W>(x + (long long)B.posGlobal[i] * KP + off, r);
  }
}

// Coarsest level: x = D Ainv^ D rhs (FP64 accumulation).  A row's j range is
// split into kCoarseParts contiguous parts; each part is summed by one warp
// (lanes stride the part, xor-tree reduction) and the parts are added in part
// order, so the launch kernel (a warp per part) and the coarse-level kernels
// (a warp per row, parts in turn) give the same bits.
constexpr int kCoarseParts = 4;
template <typename T, int W, typename LD>
__device__ __forceinline__ void coarse_part(int n, const double* ainv, const double* scale, const T* rhs, int KP, int off, int row,
                                            int part, int lane, double (&acc)[W]) {
  const int len = ((n + kCoarseParts - 1) / kCoarseParts + 31) & ~31;
  const int j0 = part * len, j1 = min(n, j0 + len);
  const double* arow = ainv + (long long)row * n;
#pragma unroll
  for (int c = 0; c < W; c++) acc[c] = 0;
  for (int j = j0 + lane; j < j1; j += 32) {
    const Vec<T, W> v = LD::template ld<T, W>(rhs + (long long)j * KP + off);
    const double w = arow[j] * scale[j];
#pragma unroll
    for (int c = 0; c < W; c++) acc[c] += w * double(v.v[c]);
  }
#pragma unroll
  for (int c = 0; c < W; c++)
    for (int s = 16; s > 0; s >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], s);
}

// One row by one warp (coarse-level kernels): the parts in turn
template <typename T, int W, typename LD>
__device__ __forceinline__ void coarse_row(int n, const double* ainv, const double* scale, const T* rhs, T* x, int KP, int G, int row,
                                           int lane) {
  for (int q = 0; q < G; q++) {
    const int off = q * W;
    double sum[W], acc[W];
#pragma unroll
    for (int c = 0; c < W; c++) sum[c] = 0;
    for (int p = 0; p < kCoarseParts; p++) {
      coarse_part<T, W, LD>(n, ainv, scale, rhs, KP, off, row, p, lane, acc);
#pragma unroll
      for (int c = 0; c < W; c++) sum[c] += acc[c];
    }
    if (lane == 0) {
      Vec<T, W> out;
#pragma unroll
      for (int c = 0; c < W; c++) out.v[c] = T(sum[c] * scale[row]);
      vstore<T, W>(x + (long long)row * KP + off, out);
    }
  }
}

}  // namespace dev
}  // namespace gdtp
