// V-cycle kernels: colour-run Gauss-Seidel, residual, transfer operators,
// exact boundary-block solve, coarsest dense solve, FP64 refinement.
// Reference operators restated (same arithmetic, different work partition):
//   deep update      IterativeSolvers.inl:449-463   x = rhs*c4 - sum_{k!=4} c_k x_k
//   deep residual    IterativeSolvers.inl:479-493   r = rhs - (sum_{k!=4} c_k x_k + x) * c9
//   restriction      IterativeSolvers.inl:1037-1053 full weighting 1, 1/2, 1/4 (+ sparse boundary rows)
//   prolongation     IterativeSolvers.inl:1128-1151 bilinear 1/2, 1/4 with aligned-start parity
//   boundary relax   IterativeSolvers.inl:414-430   x_B = BB^-1 (rhs_B - BD x)
//   boundary residual IterativeSolvers.inl:549-555  r_B = rhs_B - BD x - BB x_B
//   raw operator     IterativeSolvers.inl:881-950   y = A x (MultiplyBySystemMatrix_NoReciprocals)
#include <algorithm>

#include "vcycle.cuh"
#include "vcycle_kernels.h"

namespace gdtp {
namespace dev {

template <typename T, int W>
__device__ __forceinline__ void axpy(Vec<T, W>& acc, T a, const Vec<T, W>& v) {
#pragma unroll
  for (int c = 0; c < W; c++) acc.v[c] += a * v.v[c];
}

// ----------------------------------------------------------------------------
// Gauss-Seidel on one colour: x = rhs*c4 - sum_{k!=4} c_k x_k
// ----------------------------------------------------------------------------
template <typename T, int W>
__global__ void __launch_bounds__(256) k_gs_colour(const ColourRun* __restrict__ runs, int nRuns, const T* __restrict__ coef,
                                                   int planeStride, const T* __restrict__ rhs, T* __restrict__ x, int KP, int G) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
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
  axpy(acc, c[0 * planeStride], vload<T, W>(x + (long long)(pp - 1) * KP + off));
  axpy(acc, c[1 * planeStride], vload<T, W>(x + (long long)(pp)*KP + off));
  axpy(acc, c[2 * planeStride], vload<T, W>(x + (long long)(pp + 1) * KP + off));
  axpy(acc, c[3 * planeStride], vload<T, W>(x + (long long)(pos - 1) * KP + off));
  axpy(acc, c[5 * planeStride], vload<T, W>(x + (long long)(pos + 1) * KP + off));
  axpy(acc, c[6 * planeStride], vload<T, W>(x + (long long)(pn - 1) * KP + off));
  axpy(acc, c[7 * planeStride], vload<T, W>(x + (long long)(pn)*KP + off));
  axpy(acc, c[8 * planeStride], vload<T, W>(x + (long long)(pn + 1) * KP + off));
  const T c4 = c[4 * planeStride];
  const Vec<T, W> b = vload<T, W>(rhs + (long long)pos * KP + off);
  Vec<T, W> out;
#pragma unroll
  for (int k = 0; k < W; k++) out.v[k] = b.v[k] * c4 - acc.v[k];
  vstore<T, W>(x + (long long)pos * KP + off, out);
}

// ----------------------------------------------------------------------------
// Residual: deep rows by runs (all colours), boundary rows by CSR (global cols).
// Blocks [0, deepBlocks) handle deep texels, the rest boundary rows.
// ----------------------------------------------------------------------------
template <typename T, int W>
__global__ void __launch_bounds__(256) k_residual(const ColourRun* __restrict__ runs, int nRuns, const T* __restrict__ coef,
                                                  int planeStride, int deepBlocks, const int* __restrict__ bPtr,
                                                  const int* __restrict__ bCol, const T* __restrict__ bVal,
                                                  const int* __restrict__ bGlobal, int nB, const T* __restrict__ rhs,
                                                  const T* __restrict__ x, T* __restrict__ res, int KP, int G) {
  if ((int)blockIdx.x < deepBlocks) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
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
    Vec<T, W> acc = vload<T, W>(x + (long long)pos * KP + off);
    axpy(acc, c[0 * planeStride], vload<T, W>(x + (long long)(pp - 1) * KP + off));
    axpy(acc, c[1 * planeStride], vload<T, W>(x + (long long)(pp)*KP + off));
    axpy(acc, c[2 * planeStride], vload<T, W>(x + (long long)(pp + 1) * KP + off));
    axpy(acc, c[3 * planeStride], vload<T, W>(x + (long long)(pos - 1) * KP + off));
    axpy(acc, c[5 * planeStride], vload<T, W>(x + (long long)(pos + 1) * KP + off));
    axpy(acc, c[6 * planeStride], vload<T, W>(x + (long long)(pn - 1) * KP + off));
    axpy(acc, c[7 * planeStride], vload<T, W>(x + (long long)(pn)*KP + off));
    axpy(acc, c[8 * planeStride], vload<T, W>(x + (long long)(pn + 1) * KP + off));
    const T c9 = c[9 * planeStride];
    const Vec<T, W> b = vload<T, W>(rhs + (long long)pos * KP + off);
    Vec<T, W> out;
#pragma unroll
    for (int k = 0; k < W; k++) out.v[k] = b.v[k] - acc.v[k] * c9;
    vstore<T, W>(res + (long long)pos * KP + off, out);
  } else {
    const long long t = (long long)(blockIdx.x - deepBlocks) * blockDim.x + threadIdx.x;
    const long long row = t / G;
    if (row >= nB) return;
    const int q = int(t - row * G), off = q * W;
    const int g = bGlobal[row];
    Vec<T, W> acc = vload<T, W>(rhs + (long long)g * KP + off);
    for (int k = bPtr[row]; k < bPtr[row + 1]; k++) axpy(acc, -bVal[k], vload<T, W>(x + (long long)bCol[k] * KP + off));
    vstore<T, W>(res + (long long)g * KP + off, acc);
  }
}

// ----------------------------------------------------------------------------
// Restriction of the residual to the coarse right-hand side.
// ----------------------------------------------------------------------------
template <typename T, int W>
__global__ void __launch_bounds__(256) k_restrict(const RestrictRun* __restrict__ runs, int nRuns, int deepBlocks,
                                                  const int* __restrict__ rPtr, const int* __restrict__ rCol,
                                                  const T* __restrict__ rVal, const int* __restrict__ rOut, int nB,
                                                  const T* __restrict__ res, T* __restrict__ coarseRhs, int KP, int G) {
  if ((int)blockIdx.x < deepBlocks) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int per = 32 * G;
    const long long r = t / per;
    if (r >= nRuns) return;
    const int rem = int(t - r * per);
    const int m = rem / G, q = rem - m * G;
    const RestrictRun R = runs[r];
    if (m >= R.len) return;
    const int f = R.f0 + 2 * m, fp = R.fp0 + 2 * m, fn = R.fn0 + 2 * m, off = q * W;
    const Vec<T, W> a0 = vload<T, W>(res + (long long)f * KP + off);
    const Vec<T, W> e1 = vload<T, W>(res + (long long)fp * KP + off), e2 = vload<T, W>(res + (long long)(f - 1) * KP + off),
                    e3 = vload<T, W>(res + (long long)(f + 1) * KP + off), e4 = vload<T, W>(res + (long long)fn * KP + off);
    const Vec<T, W> d1 = vload<T, W>(res + (long long)(fp - 1) * KP + off), d2 = vload<T, W>(res + (long long)(fp + 1) * KP + off),
                    d3 = vload<T, W>(res + (long long)(fn - 1) * KP + off), d4 = vload<T, W>(res + (long long)(fn + 1) * KP + off);
    Vec<T, W> out;
#pragma unroll
    for (int k = 0; k < W; k++)
      out.v[k] = a0.v[k] + (e1.v[k] + e2.v[k] + e3.v[k] + e4.v[k]) * T(0.5) + (d1.v[k] + d2.v[k] + d3.v[k] + d4.v[k]) * T(0.25);
    vstore<T, W>(coarseRhs + (long long)(R.out0 + m) * KP + off, out);
  } else {
    const long long t = (long long)(blockIdx.x - deepBlocks) * blockDim.x + threadIdx.x;
    const long long row = t / G;
    if (row >= nB) return;
    const int q = int(t - row * G), off = q * W;
    Vec<T, W> acc;
#pragma unroll
    for (int k = 0; k < W; k++) acc.v[k] = 0;
    for (int k = rPtr[row]; k < rPtr[row + 1]; k++) axpy(acc, rVal[k], vload<T, W>(res + (long long)rCol[k] * KP + off));
    vstore<T, W>(coarseRhs + (long long)rOut[row] * KP + off, acc);
  }
}

// ----------------------------------------------------------------------------
// Prolongation of the coarse correction, added to the fine iterate.
// ----------------------------------------------------------------------------
template <typename T, int W>
__global__ void __launch_bounds__(256) k_prolong_add(const ProlongRun* __restrict__ runs, int nRuns, const T* __restrict__ coarse,
                                                     T* __restrict__ fine, int KP, int G) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
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
  Vec<T, W> acc = vload<T, W>(dst);
  if (R.center >= 0) {
    const Vec<T, W> a = vload<T, W>(coarse + (long long)(R.center + p) * KP + off), b = vload<T, W>(coarse + (long long)(R.center + n) * KP + off);
#pragma unroll
    for (int k = 0; k < W; k++) acc.v[k] += (a.v[k] + b.v[k]) * T(0.5);
  } else {
    const Vec<T, W> a = vload<T, W>(coarse + (long long)(R.prev + p) * KP + off), b = vload<T, W>(coarse + (long long)(R.prev + n) * KP + off),
                    c = vload<T, W>(coarse + (long long)(R.next + p) * KP + off), d = vload<T, W>(coarse + (long long)(R.next + n) * KP + off);
#pragma unroll
    for (int k = 0; k < W; k++) acc.v[k] += (a.v[k] + b.v[k] + c.v[k] + d.v[k]) * T(0.25);
  }
  vstore<T, W>(dst, acc);
}

// ----------------------------------------------------------------------------
// Exact boundary-block solve  x_B = BB^-1 (rhs_B - BD x), in four steps over
// the subdomain / separator split (scaled by s = BB_ii^-1/2).
// ----------------------------------------------------------------------------
// step 1 (block per subdomain): r^ = s (rhs - BD x) for the interior rows, y = Inv r^
template <typename T, int W>
__global__ void __launch_bounds__(256) k_bsolve_interior(const int* __restrict__ subPtr, const long long* __restrict__ invOff,
                                                         const T* __restrict__ inv, const int* __restrict__ posGlobal,
                                                         const T* __restrict__ scale, const int* __restrict__ bdPtr,
                                                         const int* __restrict__ bdCol, const T* __restrict__ bdVal,
                                                         const T* __restrict__ rhs, const T* __restrict__ x, T* __restrict__ y,
                                                         int KP, int G) {
  extern __shared__ unsigned char smem_raw[];
  T* rs = reinterpret_cast<T*>(smem_raw);  // m * KP
  const int p = blockIdx.x;
  const int b0 = subPtr[p], m = subPtr[p + 1] - b0;
  for (int e = threadIdx.x; e < m * G; e += blockDim.x) {
    const int a = e / G, q = e - a * G, off = q * W, k = b0 + a;
    const int g = posGlobal[k];
    Vec<T, W> acc = vload<T, W>(rhs + (long long)g * KP + off);
    for (int j = bdPtr[k]; j < bdPtr[k + 1]; j++) axpy(acc, -bdVal[j], vload<T, W>(x + (long long)bdCol[j] * KP + off));
    const T s = scale[k];
#pragma unroll
    for (int c = 0; c < W; c++) acc.v[c] *= s;
    vstore<T, W>(rs + a * KP + off, acc);
  }
  __syncthreads();
  const T* Inv = inv + invOff[p];
  // warp per output row; lanes stride the row (coalesced), reduce by shuffles
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int a = warp; a < m; a += nw) {
    const T* row = Inv + (long long)a * m;
    for (int q = 0; q < G; q++) {
      const int off = q * W;
      Vec<T, W> acc;
#pragma unroll
      for (int c = 0; c < W; c++) acc.v[c] = 0;
      for (int j = lane; j < m; j += 32) axpy(acc, row[j], vload<T, W>(rs + j * KP + off));
#pragma unroll
      for (int c = 0; c < W; c++)
        for (int s = 16; s > 0; s >>= 1) acc.v[c] += __shfl_xor_sync(0xffffffffu, acc.v[c], s);
      if (lane == 0) vstore<T, W>(y + (long long)(b0 + a) * KP + off, acc);
    }
  }
}

// step 2 (thread per separator row): t = s (rhs - BD x) - A_SI y
template <typename T, int W>
__global__ void __launch_bounds__(256) k_bsolve_separator_rhs(int nI, int nS, const int* __restrict__ posGlobal,
                                                              const T* __restrict__ scale, const int* __restrict__ bdPtr,
                                                              const int* __restrict__ bdCol, const T* __restrict__ bdVal,
                                                              const int* __restrict__ asiPtr, const int* __restrict__ asiCol,
                                                              const T* __restrict__ asiVal, const T* __restrict__ rhs,
                                                              const T* __restrict__ x, const T* __restrict__ y, T* __restrict__ t,
                                                              int KP, int G) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long s = tid / G;
  if (s >= nS) return;
  const int q = int(tid - s * G), off = q * W, k = nI + int(s);
  const int g = posGlobal[k];
  Vec<T, W> acc = vload<T, W>(rhs + (long long)g * KP + off);
  for (int j = bdPtr[k]; j < bdPtr[k + 1]; j++) axpy(acc, -bdVal[j], vload<T, W>(x + (long long)bdCol[j] * KP + off));
  const T sc = scale[k];
#pragma unroll
  for (int c = 0; c < W; c++) acc.v[c] *= sc;
  for (int j = asiPtr[s]; j < asiPtr[s + 1]; j++) axpy(acc, -asiVal[j], vload<T, W>(y + (long long)asiCol[j] * KP + off));
  vstore<T, W>(t + s * KP + off, acc);
}

// step 3 (warp per separator row): xs = Sinv t ; x[g] = s * xs
template <typename T, int W>
__global__ void __launch_bounds__(256) k_bsolve_separator(int nI, int nS, const T* __restrict__ sinv, const T* __restrict__ t,
                                                          const int* __restrict__ posGlobal, const T* __restrict__ scale,
                                                          T* __restrict__ xs, T* __restrict__ x, int KP, int G) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= nS) return;
  const T* row = sinv + (long long)warp * nS;
  for (int q = 0; q < G; q++) {
    const int off = q * W;
    Vec<T, W> acc;
#pragma unroll
    for (int c = 0; c < W; c++) acc.v[c] = 0;
    for (int j = lane; j < nS; j += 32) axpy(acc, row[j], vload<T, W>(t + (long long)j * KP + off));
#pragma unroll
    for (int c = 0; c < W; c++)
      for (int s = 16; s > 0; s >>= 1) acc.v[c] += __shfl_xor_sync(0xffffffffu, acc.v[c], s);
    if (lane == 0) {
      vstore<T, W>(xs + (long long)warp * KP + off, acc);
      const T sc = scale[nI + warp];
#pragma unroll
      for (int c = 0; c < W; c++) acc.v[c] *= sc;
      vstore<T, W>(x + (long long)posGlobal[nI + warp] * KP + off, acc);
    }
  }
}

// step 4 (block per subdomain): x_I = s (y - Inv (A_IS xs))
template <typename T, int W>
__global__ void __launch_bounds__(256) k_bsolve_back(const int* __restrict__ subPtr, const long long* __restrict__ invOff,
                                                     const T* __restrict__ inv, const int* __restrict__ posGlobal,
                                                     const T* __restrict__ scale, const int* __restrict__ aisPtr,
                                                     const int* __restrict__ aisCol, const T* __restrict__ aisVal,
                                                     const T* __restrict__ xs, const T* __restrict__ y, T* __restrict__ x, int KP,
                                                     int G) {
  extern __shared__ unsigned char smem_raw[];
  T* zs = reinterpret_cast<T*>(smem_raw);
  const int p = blockIdx.x;
  const int b0 = subPtr[p], m = subPtr[p + 1] - b0;
  for (int e = threadIdx.x; e < m * G; e += blockDim.x) {
    const int a = e / G, q = e - a * G, off = q * W, k = b0 + a;
    Vec<T, W> acc;
#pragma unroll
    for (int c = 0; c < W; c++) acc.v[c] = 0;
    for (int j = aisPtr[k]; j < aisPtr[k + 1]; j++) axpy(acc, aisVal[j], vload<T, W>(xs + (long long)aisCol[j] * KP + off));
    vstore<T, W>(zs + a * KP + off, acc);
  }
  __syncthreads();
  const T* Inv = inv + invOff[p];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int a = warp; a < m; a += nw) {
    const T* row = Inv + (long long)a * m;
    for (int q = 0; q < G; q++) {
      const int off = q * W;
      Vec<T, W> acc;
#pragma unroll
      for (int c = 0; c < W; c++) acc.v[c] = 0;
      for (int j = lane; j < m; j += 32) axpy(acc, row[j], vload<T, W>(zs + j * KP + off));
#pragma unroll
      for (int c = 0; c < W; c++)
        for (int s = 16; s > 0; s >>= 1) acc.v[c] += __shfl_xor_sync(0xffffffffu, acc.v[c], s);
      if (lane == 0) {
        const Vec<T, W> yy = vload<T, W>(y + (long long)(b0 + a) * KP + off);
        const T sc = scale[b0 + a];
        Vec<T, W> out;
#pragma unroll
        for (int c = 0; c < W; c++) out.v[c] = (yy.v[c] - acc.v[c]) * sc;
        vstore<T, W>(x + (long long)posGlobal[b0 + a] * KP + off, out);
      }
    }
  }
}

// ----------------------------------------------------------------------------
// Coarsest level: x = D Ainv^ D rhs with the scaled dense inverse (FP64).
// ----------------------------------------------------------------------------
template <typename T, int W>
__global__ void __launch_bounds__(256) k_coarse_solve(int n, const double* __restrict__ ainv, const double* __restrict__ scale,
                                                      const T* __restrict__ rhs, T* __restrict__ x, int KP, int G) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n) return;
  const double* row = ainv + (long long)warp * n;
  for (int q = 0; q < G; q++) {
    const int off = q * W;
    double acc[W];
#pragma unroll
    for (int c = 0; c < W; c++) acc[c] = 0;
    for (int j = lane; j < n; j += 32) {
      const Vec<T, W> v = vload<T, W>(rhs + (long long)j * KP + off);
      const double w = row[j] * scale[j];
#pragma unroll
      for (int c = 0; c < W; c++) acc[c] += w * double(v.v[c]);
    }
#pragma unroll
    for (int c = 0; c < W; c++)
      for (int s = 16; s > 0; s >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], s);
    if (lane == 0) {
      Vec<T, W> out;
#pragma unroll
      for (int c = 0; c < W; c++) out.v[c] = T(acc[c] * scale[warp]);
      vstore<T, W>(x + (long long)warp * KP + off, out);
    }
  }
}

// ----------------------------------------------------------------------------
// FP64 raw operator: res = b - A x (mode 0) or y = A x (mode 1) on tight
// n x K vectors.  Deep rows use 9 raw coefficients per run texel, boundary rows
// the merged BD/BB CSR.  A thread handles one texel and up to 4 channels
// (group q of G = KP/4 groups, or G = 1 for K = 1).  Per-block sums of res^2
// and b^2 per channel go to `partials` for a deterministic norm reduction.
// ----------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_raw_operator(const ColourRun* __restrict__ runs, int nRuns, const double* __restrict__ coef,
                                                      int planeStride, int deepBlocks, const int* __restrict__ bPtr,
                                                      const int* __restrict__ bCol, const double* __restrict__ bVal,
                                                      const int* __restrict__ bGlobal, int nB, const double* __restrict__ b,
                                                      const double* __restrict__ x, double* __restrict__ out, int K, int G, int mode,
                                                      double* __restrict__ partials) {
  double acc[4] = {0, 0, 0, 0};
  int g = -1, q = 0;
  if ((int)blockIdx.x < deepBlocks) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int per = 32 * G;
    const long long r = t / per;
    const int rem = int(t - r * per);
    const int m = rem / G;
    q = rem - m * G;
    if (r < nRuns) {
      const ColourRun R = runs[r];
      if (m < R.len) {
        const int pos = R.pos0 + 2 * m, pp = R.prev0 + 2 * m, pn = R.next0 + 2 * m;
        const double* c = coef + R.coef0 + m;
        const int nb[9] = {pp - 1, pp, pp + 1, pos - 1, pos, pos + 1, pn - 1, pn, pn + 1};
#pragma unroll
        for (int s = 0; s < 9; s++) {
          const double w = c[s * planeStride];
          const double* xs = x + (long long)nb[s] * K + 4 * q;
#pragma unroll
          for (int ch = 0; ch < 4; ch++)
            if (4 * q + ch < K) acc[ch] += w * xs[ch];
        }
        g = pos;
      }
    }
  } else {
    const long long t = (long long)(blockIdx.x - deepBlocks) * blockDim.x + threadIdx.x;
    const long long row = t / G;
    q = int(t - row * G);
    if (row < nB) {
      for (int k = bPtr[row]; k < bPtr[row + 1]; k++) {
        const double w = bVal[k];
        const double* xs = x + (long long)bCol[k] * K + 4 * q;
#pragma unroll
        for (int ch = 0; ch < 4; ch++)
          if (4 * q + ch < K) acc[ch] += w * xs[ch];
      }
      g = bGlobal[row];
    }
  }
  double rr[4] = {0, 0, 0, 0}, bb[4] = {0, 0, 0, 0};
  if (g >= 0) {
#pragma unroll
    for (int ch = 0; ch < 4; ch++) {
      const int c = 4 * q + ch;
      if (c >= K) continue;
      const double bv = b ? b[(long long)g * K + c] : 0.0;
      const double v = mode == 0 ? bv - acc[ch] : acc[ch];
      out[(long long)g * K + c] = v;
      rr[ch] = v * v;
      bb[ch] = bv * bv;
    }
  }
  if (!partials) return;
  // lanes l and l^s with s >= G share the group q: reduce across them
  __shared__ double red[8][2][64];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int ch = 0; ch < 4; ch++)
    for (int s = 16; s >= G; s >>= 1) {
      rr[ch] += __shfl_xor_sync(0xffffffffu, rr[ch], s);
      bb[ch] += __shfl_xor_sync(0xffffffffu, bb[ch], s);
    }
  if (lane < G)
#pragma unroll
    for (int ch = 0; ch < 4; ch++)
      if (4 * lane + ch < K) { red[warp][0][4 * lane + ch] = rr[ch]; red[warp][1][4 * lane + ch] = bb[ch]; }
  __syncthreads();
  if ((int)threadIdx.x < K) {
    double a = 0, c = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) { a += red[w][0][threadIdx.x]; c += red[w][1][threadIdx.x]; }
    partials[(long long)blockIdx.x * 2 * K + threadIdx.x] = a;
    partials[(long long)blockIdx.x * 2 * K + K + threadIdx.x] = c;
  }
}

// Sum of per-block partials in a fixed order (one block): sums[2K]
__global__ void k_sum_partials(const double* __restrict__ partials, int nBlocks, int K, double* __restrict__ sums) {
  __shared__ double sh[256];
  for (int c = 0; c < 2 * K; c++) {
    double s = 0;
    for (int b = threadIdx.x; b < nBlocks; b += blockDim.x) s += partials[(long long)b * 2 * K + c];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
      if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) sums[c] = sh[0];
    __syncthreads();
  }
}

// FP64 residual (n*K, tight) -> FP32 right-hand side (n*KP, padded)
template <typename T>
__global__ void k_pack_rhs(const double* __restrict__ r, T* __restrict__ rhs, long long n, int K, int KP) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * KP) return;
  const long long i = t / KP;
  const int c = int(t - i * KP);
  rhs[t] = c < K ? T(r[i * K + c]) : T(0);
}
// x64 += e (padded FP32/FP64 correction)
template <typename T>
__global__ void k_add_correction(double* __restrict__ x, const T* __restrict__ e, long long n, int K, int KP) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * K) return;
  const long long i = t / K;
  const int c = int(t - i * K);
  x[t] += double(e[i * KP + c]);
}

// ----------------------------------------------------------------------------
// launch wrappers
// ----------------------------------------------------------------------------
static inline int nblk(long long threads) { return int((threads + 255) / 256); }

template <typename T, int W>
void launch_gs_colour(const ColourRun* runs, int nRuns, const T* coef, int planeStride, const T* rhs, T* x, int KP,
                      cudaStream_t s) {
  if (nRuns == 0) return;
  const int G = KP / W;
  k_gs_colour<T, W><<<nblk((long long)nRuns * 32 * G), 256, 0, s>>>(runs, nRuns, coef, planeStride, rhs, x, KP, G);
}
template <typename T, int W>
void launch_residual(const ColourRun* runs, int nRuns, const T* coef, int planeStride, const int* bPtr, const int* bCol,
                     const T* bVal, const int* bGlobal, int nB, const T* rhs, const T* x, T* res, int KP, cudaStream_t s) {
  const int G = KP / W;
  const int db = nblk((long long)nRuns * 32 * G), bb = nblk((long long)nB * G);
  if (db + bb == 0) return;
  k_residual<T, W><<<db + bb, 256, 0, s>>>(runs, nRuns, coef, planeStride, db, bPtr, bCol, bVal, bGlobal, nB, rhs, x, res, KP, G);
}
template <typename T, int W>
void launch_restrict(const RestrictRun* runs, int nRuns, const int* rPtr, const int* rCol, const T* rVal, const int* rOut,
                     int nB, const T* res, T* coarseRhs, int KP, cudaStream_t s) {
  const int G = KP / W;
  const int db = nblk((long long)nRuns * 32 * G), bb = nblk((long long)nB * G);
  if (db + bb == 0) return;
  k_restrict<T, W><<<db + bb, 256, 0, s>>>(runs, nRuns, db, rPtr, rCol, rVal, rOut, nB, res, coarseRhs, KP, G);
}
template <typename T, int W>
void launch_prolong_add(const ProlongRun* runs, int nRuns, const T* coarse, T* fine, int KP, cudaStream_t s) {
  if (nRuns == 0) return;
  const int G = KP / W;
  k_prolong_add<T, W><<<nblk((long long)nRuns * 32 * G), 256, 0, s>>>(runs, nRuns, coarse, fine, KP, G);
}
template <typename T, int W>
void launch_boundary_solve(const BoundaryDev<T>& B, const T* rhs, T* x, int KP, cudaStream_t s) {
  if (B.nb == 0) return;
  const int G = KP / W;
  const size_t smem = size_t(B.maxBlock) * KP * sizeof(T);
  if (B.nSub > 0)
    k_bsolve_interior<T, W><<<B.nSub, 256, smem, s>>>(B.subPtr, B.invOff, B.inv, B.posGlobal, B.scale, B.bdPtr, B.bdCol, B.bdVal,
                                                      rhs, x, B.y, KP, G);
  if (B.nS > 0) {
    k_bsolve_separator_rhs<T, W><<<nblk((long long)B.nS * G), 256, 0, s>>>(B.nI, B.nS, B.posGlobal, B.scale, B.bdPtr, B.bdCol,
                                                                         B.bdVal, B.asiPtr, B.asiCol, B.asiVal, rhs, x, B.y,
                                                                         B.t, KP, G);
    k_bsolve_separator<T, W><<<nblk((long long)B.nS * 32), 256, 0, s>>>(B.nI, B.nS, B.sinv, B.t, B.posGlobal, B.scale, B.xs, x,
                                                                      KP, G);
  }
  if (B.nSub > 0)
    k_bsolve_back<T, W><<<B.nSub, 256, smem, s>>>(B.subPtr, B.invOff, B.inv, B.posGlobal, B.scale, B.aisPtr, B.aisCol, B.aisVal,
                                                  B.xs, B.y, x, KP, G);
}
template <typename T, int W>
cudaError_t configure_boundary_smem(size_t bytes) {
  const int b = int(std::max<size_t>(bytes, 48 * 1024));
  cudaError_t e = cudaFuncSetAttribute(k_bsolve_interior<T, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_bsolve_back<T, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
}
template <typename T, int W>
void launch_coarse_solve(int n, const double* ainv, const double* scale, const T* rhs, T* x, int KP, cudaStream_t s) {
  if (n == 0) return;
  k_coarse_solve<T, W><<<nblk((long long)n * 32), 256, 0, s>>>(n, ainv, scale, rhs, x, KP, KP / W);
}

static inline int raw_groups(int K) { int G = 1; while (4 * G < K) G *= 2; return G; }
void launch_raw_operator(const ColourRun* runs, int nRuns, const double* coef, int planeStride, const int* bPtr, const int* bCol,
                         const double* bVal, const int* bGlobal, int nB, const double* b, const double* x, double* out, int K,
                         int mode, double* partials, double* sums, cudaStream_t s) {
  const int G = raw_groups(K);
  const int db = nblk((long long)nRuns * 32 * G), bb = nblk((long long)nB * G);
  if (db + bb == 0) return;
  k_raw_operator<<<db + bb, 256, 0, s>>>(runs, nRuns, coef, planeStride, db, bPtr, bCol, bVal, bGlobal, nB, b, x, out, K, G,
                                         mode, partials);
  if (partials && sums) k_sum_partials<<<1, 256, 0, s>>>(partials, db + bb, K, sums);
}
int raw_operator_blocks(int nRuns, int nB, int K) {
  const int G = raw_groups(K);
  return nblk((long long)nRuns * 32 * G) + nblk((long long)nB * G);
}

template <typename T>
void launch_pack_rhs(const double* r, T* rhs, long long n, int K, int KP, cudaStream_t s) {
  k_pack_rhs<T><<<nblk(n * KP), 256, 0, s>>>(r, rhs, n, K, KP);
}
template <typename T>
void launch_add_correction(double* x, const T* e, long long n, int K, int KP, cudaStream_t s) {
  k_add_correction<T><<<nblk(n * K), 256, 0, s>>>(x, e, n, K, KP);
}

#define GDTP_INSTANTIATE(T, W)                                                                                             \
  template void launch_gs_colour<T, W>(const ColourRun*, int, const T*, int, const T*, T*, int, cudaStream_t);           \
  template void launch_residual<T, W>(const ColourRun*, int, const T*, int, const int*, const int*, const T*, const int*, \
                                      int, const T*, const T*, T*, int, cudaStream_t);                                   \
  template void launch_restrict<T, W>(const RestrictRun*, int, const int*, const int*, const T*, const int*, int,        \
                                      const T*, T*, int, cudaStream_t);                                                  \
  template void launch_prolong_add<T, W>(const ProlongRun*, int, const T*, T*, int, cudaStream_t);                       \
  template void launch_boundary_solve<T, W>(const BoundaryDev<T>&, const T*, T*, int, cudaStream_t);                     \
  template void launch_coarse_solve<T, W>(int, const double*, const double*, const T*, T*, int, cudaStream_t);     \
  template cudaError_t configure_boundary_smem<T, W>(size_t);
GDTP_INSTANTIATE(float, 1)
GDTP_INSTANTIATE(float, 4)
GDTP_INSTANTIATE(double, 1)
GDTP_INSTANTIATE(double, 4)
template void launch_pack_rhs<float>(const double*, float*, long long, int, int, cudaStream_t);
template void launch_pack_rhs<double>(const double*, double*, long long, int, int, cudaStream_t);
template void launch_add_correction<float>(double*, const float*, long long, int, int, cudaStream_t);
template void launch_add_correction<double>(double*, const double*, long long, int, int, cudaStream_t);

}  // namespace dev
}  // namespace gdtp
