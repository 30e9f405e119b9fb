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
#include <type_traits>

#include "vcycle.cuh"
#include "vcycle_kernels.h"
#include "vcycle_ops.cuh"

namespace gdtp {
namespace dev {

// ----------------------------------------------------------------------------
// Gauss-Seidel on one colour: x = rhs*c4 - sum_{k!=4} c_k x_k
// ----------------------------------------------------------------------------
template <typename T, int W>
__global__ void __launch_bounds__(256) k_gs_colour(const ColourRun* __restrict__ runs, int nRuns, const T* __restrict__ coef,
                                                   int planeStride, const T* __restrict__ rhs, T* __restrict__ x, int KP, int G,
                                                   int skip, int rhsEarly) {
  // What the previous launch cannot have written is loaded before waiting for
  // it, so that these loads overlap its tail: the run and its coefficients
  // (written at set-up), and the right-hand side when the previous launch is a
  // colour pass of the same smoothing step (rhsEarly).  x is read after the
  // wait.  The arithmetic is gs_item's, in the same order.
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int per = 32 * G;
  const long long r = t / per;
  const int rem = int(t - r * per);
  const int m = rem / G, q = rem - m * G;
  ColourRun R;
  R.len = 0;
  if (r < nRuns) R = runs[r];
  const bool active = r < nRuns && m < R.len;
  T w[10];
  Vec<T, W> b;
  int pos = 0, pp = 0, pn = 0;
  const int off = q * W;
  if (active) {
    pos = R.pos0 + 2 * m, pp = R.prev0 + 2 * m, pn = R.next0 + 2 * m;
    const T* c = coef + R.coef0 + m;
#pragma unroll
    for (int k = 0; k < 9; k++) w[k] = c[k * planeStride];
    if (rhsEarly) b = vload<T, W>(rhs + (long long)pos * KP + off);
  }
  grid_dependency_wait();
  grid_launch_dependents();
  if (!active) return;
  if (!rhsEarly) b = vload<T, W>(rhs + (long long)pos * KP + off);
  Vec<T, W> acc;
#pragma unroll
  for (int k = 0; k < W; k++) acc.v[k] = 0;
  if (!(skip & 1)) axpy(acc, w[0], vload<T, W>(x + (long long)(pp - 1) * KP + off));
  if (!(skip & 2)) axpy(acc, w[1], vload<T, W>(x + (long long)(pp)*KP + off));
  if (!(skip & 4)) axpy(acc, w[2], vload<T, W>(x + (long long)(pp + 1) * KP + off));
  if (!(skip & 8)) axpy(acc, w[3], vload<T, W>(x + (long long)(pos - 1) * KP + off));
  if (!(skip & 32)) axpy(acc, w[5], vload<T, W>(x + (long long)(pos + 1) * KP + off));
  if (!(skip & 64)) axpy(acc, w[6], vload<T, W>(x + (long long)(pn - 1) * KP + off));
  if (!(skip & 128)) axpy(acc, w[7], vload<T, W>(x + (long long)(pn)*KP + off));
  if (!(skip & 256)) axpy(acc, w[8], vload<T, W>(x + (long long)(pn + 1) * KP + off));
  Vec<T, W> out;
#pragma unroll
  for (int k = 0; k < W; k++) out.v[k] = b.v[k] * w[4] - acc.v[k];
  vstore<T, W>(x + (long long)pos * KP + off, out);
}

// Two colour passes of one row parity (launch_gs_rows).  Colours 0 and 1 hold
// the even rows, 2 and 3 the odd rows, and the 9-point stencil of a row reaches
// only its own row and the two rows of the other parity.  So the passes of one
// row parity update each raster line independently: the first colour (A) from
// the line's old values, then the second (B) from A's new values in the line.
// A block holds whole lines; thread q of a line owns its texels 2q and 2q + 1
// (A texel oA + 2q, B texel oB + 2q), which it stages with the rows above and
// below into shared memory (slot 0 of a line: texel -1, slot len + 1: texel
// len, the line's non-deep neighbours).  Coefficients and (rhsEarly) the
// right-hand side are loaded before the dependency wait, as in k_gs_colour; A
// texels of a line are consecutive in the colour-run planes, as are B texels.
// Each update is gs_item's sum in gs_item's order.
// blocks of BS threads per SM the row smoother is compiled for (registers)
template <typename T>
constexpr int rows_min_blocks(int bs) {
  return (sizeof(T) == 4 ? 1280 : 768) / bs > 0 ? (sizeof(T) == 4 ? 1280 : 768) / bs : 1;
}
template <typename T, int W, int BS>
__global__ void __launch_bounds__(BS) k_gs_rows(const RowLine* __restrict__ lines, const int* __restrict__ lineOf,
                                                           const T* __restrict__ coef, int planeStride, const T* __restrict__ rhs,
                                                           T* __restrict__ x, int KP, int slots, int oddFirst, int skip,
                                                           int rhsEarly) {
  extern __shared__ __align__(32) unsigned char smem_raw[];
  Vec<T, W>* up = reinterpret_cast<Vec<T, W>*>(smem_raw);
  Vec<T, W>* mid = up + slots;
  Vec<T, W>* dn = mid + slots;
  const int li = lineOf[(long long)blockIdx.x * BS + threadIdx.x];
  const int off = blockIdx.y * W;
  RowLine Ln;
  Ln.len = 0;
  int q = 0, a = 0, b = 0, s0 = 0, H = 0;
  bool hasA = false, hasB = false;
  T wA[9], wB[9];
  Vec<T, W> bA, bB;
  if (li >= 0) {
    Ln = lines[li];
    q = int(threadIdx.x) - (Ln.meta & 2047);
    s0 = (Ln.meta >> 11) & 8191;
    H = (Ln.len + 3) >> 1;
    const int oA = ((Ln.meta >> 24) & 1) ^ oddFirst;
    a = oA + 2 * q;
    b = (oA ^ 1) + 2 * q;
    hasA = a < Ln.len;
    hasB = b < Ln.len;
    const T* cA = coef + (oddFirst ? Ln.cOdd : Ln.cEven) + q;
    const T* cB = coef + (oddFirst ? Ln.cEven : Ln.cOdd) + q;
    if (hasA) {
#pragma unroll
      for (int k = 0; k < 9; k++) wA[k] = cA[k * planeStride];
      if (rhsEarly) bA = vload<T, W>(rhs + (long long)(Ln.pos + a) * KP + off);
    }
    if (hasB) {
#pragma unroll
      for (int k = 0; k < 9; k++) wB[k] = cB[k * planeStride];
      if (rhsEarly) bB = vload<T, W>(rhs + (long long)(Ln.pos + b) * KP + off);
    }
  }
  // shared slot of line texel i (-1 .. len): texels of even and odd i + 1 in
  // two halves, so that consecutive threads touch consecutive slots
  auto slot = [&](int i) { return s0 + (((i + 1) & 1) ? H + ((i + 1) >> 1) : ((i + 1) >> 1)); };
  grid_dependency_wait();
  grid_launch_dependents();
  const bool rowsA = !(skip & 1), rowsB = !(skip & 4);
  if (li >= 0) {
    const bool rows = rowsA || rowsB;
    auto stage = [&](int i) {
      const int sl = slot(i);
      mid[sl] = vload<T, W>(x + (long long)(Ln.pos + i) * KP + off);
      if (rows) {
        up[sl] = vload<T, W>(x + (long long)(Ln.prev + i) * KP + off);
        dn[sl] = vload<T, W>(x + (long long)(Ln.next + i) * KP + off);
      }
    };
    // the pair of texels (2q, 2q + 1) of the three rows, and the line's ends:
    // the first thread texel -1, the last thread texel len
    stage(2 * q);
    if (2 * q + 1 < Ln.len) stage(2 * q + 1);
    if (q == 0) stage(-1);
    if (2 * q + 2 >= Ln.len) stage(Ln.len);
    if (!rhsEarly) {
      if (hasA) bA = vload<T, W>(rhs + (long long)(Ln.pos + a) * KP + off);
      if (hasB) bB = vload<T, W>(rhs + (long long)(Ln.pos + b) * KP + off);
    }
  }
  __syncthreads();
  Vec<T, W> xa, xb;
  if (hasA) {
    const int sm = slot(a - 1), sc = slot(a), sp = slot(a + 1);
    Vec<T, W> acc;
#pragma unroll
    for (int k = 0; k < W; k++) acc.v[k] = 0;
    if (rowsA) {
      axpy(acc, wA[0], up[sm]);
      axpy(acc, wA[1], up[sc]);
      axpy(acc, wA[2], up[sp]);
    }
    if (!(skip & 2)) {
      axpy(acc, wA[3], mid[sm]);
      axpy(acc, wA[5], mid[sp]);
    }
    if (rowsA) {
      axpy(acc, wA[6], dn[sm]);
      axpy(acc, wA[7], dn[sc]);
      axpy(acc, wA[8], dn[sp]);
    }
#pragma unroll
    for (int k = 0; k < W; k++) xa.v[k] = bA.v[k] * wA[4] - acc.v[k];
    mid[sc] = xa;  // A slots are read only by B updates, after the barrier
  }
  __syncthreads();
  if (hasB) {
    const int sm = slot(b - 1), sc = slot(b), sp = slot(b + 1);
    Vec<T, W> acc;
#pragma unroll
    for (int k = 0; k < W; k++) acc.v[k] = 0;
    if (rowsB) {
      axpy(acc, wB[0], up[sm]);
      axpy(acc, wB[1], up[sc]);
      axpy(acc, wB[2], up[sp]);
    }
    if (!(skip & 8)) {
      axpy(acc, wB[3], mid[sm]);
      axpy(acc, wB[5], mid[sp]);
    }
    if (rowsB) {
      axpy(acc, wB[6], dn[sm]);
      axpy(acc, wB[7], dn[sc]);
      axpy(acc, wB[8], dn[sp]);
    }
#pragma unroll
    for (int k = 0; k < W; k++) xb.v[k] = bB.v[k] * wB[4] - acc.v[k];
  }
  // texels 2q and 2q + 1 of the line, in address order
  if (a < b) {
    if (hasA) vstore<T, W>(x + (long long)(Ln.pos + a) * KP + off, xa);
    if (hasB) vstore<T, W>(x + (long long)(Ln.pos + b) * KP + off, xb);
  } else {
    if (hasB) vstore<T, W>(x + (long long)(Ln.pos + b) * KP + off, xb);
    if (hasA) vstore<T, W>(x + (long long)(Ln.pos + a) * KP + off, xa);
  }
}

// Every sweep of one smoothing step on one chart per block: the colour passes
// of a chart only read texels of that chart (deep) or boundary texels, which
// the sweeps do not change, so block barriers order the passes.  The chart's
// texel span of x is staged in shared memory for all passes (the smoothing of
// a small level is a chain of dependent memory latencies, and shared memory
// has the shortest); the updated deep texels are written back at the end.  The
// arithmetic is gs_item's, so the result is the launch path's, bit for bit.
constexpr int kGroupBlockMax = 1024;
template <typename T, int W>
__global__ void __launch_bounds__(kGroupBlockMax, 1) k_gs_groups(const ColourRun* __restrict__ runs, const int* __restrict__ groups,
                                                               const T* __restrict__ coef, int planeStride, const T* __restrict__ rhs,
                                                               T* __restrict__ x, int KP, int G, int sweeps, int reverse) {
  grid_dependency_wait();
  grid_launch_dependents();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* xs = reinterpret_cast<T*>(smem_raw);
  const int* g = groups + 10 * blockIdx.x;
  const int lo = g[8], span = g[9];
  const int nt = blockDim.x;
  for (long long i = threadIdx.x; i < (long long)span * KP; i += nt) xs[i] = x[(long long)lo * KP + i];
  __syncthreads();
  for (int sw = 0; sw < sweeps; sw++)
    for (int cc = 0; cc < 4; cc++) {
      const int c = reverse ? 3 - cc : cc;
      const int nr = g[4 + c];
      const ColourRun* rc = runs + g[c];
      for (long long t = threadIdx.x; t < (long long)nr * 32 * G; t += nt) {
        const int per = 32 * G;
        const int r = int(t / per), rem = int(t - (long long)r * per);
        const int m = rem / G, q = rem - m * G;
        const ColourRun R = rc[r];
        if (m >= R.len) continue;
        // gs_item with positions relative to the span
        const int pos = R.pos0 + 2 * m - lo, pp = R.prev0 + 2 * m - lo, pn = R.next0 + 2 * m - lo;
        const T* cf = coef + R.coef0 + m;
        const int off = q * W;
        Vec<T, W> acc;
#pragma unroll
        for (int k = 0; k < W; k++) acc.v[k] = 0;
        axpy(acc, cf[0 * planeStride], vload<T, W>(xs + (pp - 1) * KP + off));
        axpy(acc, cf[1 * planeStride], vload<T, W>(xs + (pp)*KP + off));
        axpy(acc, cf[2 * planeStride], vload<T, W>(xs + (pp + 1) * KP + off));
        axpy(acc, cf[3 * planeStride], vload<T, W>(xs + (pos - 1) * KP + off));
        axpy(acc, cf[5 * planeStride], vload<T, W>(xs + (pos + 1) * KP + off));
        axpy(acc, cf[6 * planeStride], vload<T, W>(xs + (pn - 1) * KP + off));
        axpy(acc, cf[7 * planeStride], vload<T, W>(xs + (pn)*KP + off));
        axpy(acc, cf[8 * planeStride], vload<T, W>(xs + (pn + 1) * KP + off));
        const T c4 = cf[4 * planeStride];
        const Vec<T, W> bv = vload<T, W>(rhs + (long long)(pos + lo) * KP + off);
        Vec<T, W> out;
#pragma unroll
        for (int k = 0; k < W; k++) out.v[k] = bv.v[k] * c4 - acc.v[k];
        vstore<T, W>(xs + pos * KP + off, out);
      }
      __syncthreads();
    }
  // write back the chart's deep texels (the rest of the span is unchanged and
  // may not be written: boundary texels belong to the boundary solve's order)
  for (int c = 0; c < 4; c++) {
    const int nr = g[4 + c];
    const ColourRun* rc = runs + g[c];
    for (long long t = threadIdx.x; t < (long long)nr * 32; t += nt) {
      const int r = int(t >> 5), m = int(t & 31);
      const ColourRun R = rc[r];
      if (m >= R.len) continue;
      const int pos = R.pos0 + 2 * m;
      for (int k = 0; k < KP; k++) x[(long long)pos * KP + k] = xs[(pos - lo) * KP + k];
    }
  }
}

// The chart smoother for FP32 vectors of one channel group whose colour passes
// fit kGroupRegBlock threads: thread t owns item t of every colour (run t / 32,
// texel t % 32) and loads its run, coefficients and (rhsEarly) right-hand side
// for all four colours before the dependency wait, with independent loads;
// the passes then read x from shared memory only.  REV: colours 3..0.  Same
// updates, same order, same bits as k_gs_groups.
constexpr int kGroupRegBlock = 512;
template <int W, bool REV>
__global__ void __launch_bounds__(kGroupRegBlock, 1) k_gs_groups_reg(const ColourRun* __restrict__ runs,
                                                                   const int* __restrict__ groups, const float* __restrict__ coef,
                                                                   int planeStride, const float* __restrict__ rhs,
                                                                   float* __restrict__ x, int sweeps, int rhsEarly) {
  constexpr int KP = W;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* xs = reinterpret_cast<float*>(smem_raw);
  const int* g = groups + 10 * blockIdx.x;
  const int lo = g[8], span = g[9];
  const int t = threadIdx.x, m = t & 31;
  bool act[4];
  int pos[4], pp[4], pn[4];
  float w[4][9];
  Vec<float, W> bv[4];
#pragma unroll
  for (int c = 0; c < 4; c++) {
    act[c] = false;
    pos[c] = pp[c] = pn[c] = 0;
    if (t < g[4 + c] * 32) {
      const ColourRun R = runs[g[c] + (t >> 5)];
      if (m < R.len) {
        act[c] = true;
        pos[c] = R.pos0 + 2 * m - lo;
        pp[c] = R.prev0 + 2 * m - lo;
        pn[c] = R.next0 + 2 * m - lo;
        const float* cf = coef + R.coef0 + m;
#pragma unroll
        for (int k = 0; k < 9; k++) w[c][k] = cf[k * planeStride];
        if (rhsEarly) bv[c] = vload<float, W>(rhs + (long long)(pos[c] + lo) * KP);
      }
    }
  }
  grid_dependency_wait();
  grid_launch_dependents();
  for (int i = t; i < span * KP; i += blockDim.x) xs[i] = x[(long long)lo * KP + i];
  if (!rhsEarly)
#pragma unroll
    for (int c = 0; c < 4; c++)
      if (act[c]) bv[c] = vload<float, W>(rhs + (long long)(pos[c] + lo) * KP);
  __syncthreads();
  // the pass loop stays rolled (the per-colour arrays then live in local
  // memory, L1-resident): unrolled, the compiled passes did not reproduce the
  // launch path's bits
  for (int sw = 0; sw < sweeps; sw++) {
#pragma unroll 1
    for (int cc = 0; cc < 4; cc++) {
      const int c = REV ? 3 - cc : cc;
      if (act[c]) {
        Vec<float, W> acc;
#pragma unroll
        for (int k = 0; k < W; k++) acc.v[k] = 0;
        axpy(acc, w[c][0], vload<float, W>(xs + (pp[c] - 1) * KP));
        axpy(acc, w[c][1], vload<float, W>(xs + (pp[c]) * KP));
        axpy(acc, w[c][2], vload<float, W>(xs + (pp[c] + 1) * KP));
        axpy(acc, w[c][3], vload<float, W>(xs + (pos[c] - 1) * KP));
        axpy(acc, w[c][5], vload<float, W>(xs + (pos[c] + 1) * KP));
        axpy(acc, w[c][6], vload<float, W>(xs + (pn[c] - 1) * KP));
        axpy(acc, w[c][7], vload<float, W>(xs + (pn[c]) * KP));
        axpy(acc, w[c][8], vload<float, W>(xs + (pn[c] + 1) * KP));
        Vec<float, W> out;
#pragma unroll
        for (int k = 0; k < W; k++) out.v[k] = bv[c].v[k] * w[c][4] - acc.v[k];
        vstore<float, W>(xs + pos[c] * KP, out);
      }
      __syncthreads();
    }
  }
  // write back this thread's deep texels (boundary texels of the span stay)
#pragma unroll
  for (int c = 0; c < 4; c++)
    if (act[c]) vstore<float, W>(x + (long long)(pos[c] + lo) * KP, vload<float, W>(xs + pos[c] * KP));
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
                                                  const T* __restrict__ x, T* __restrict__ res, int KP, int G, int rhsEarly) {
  if ((int)blockIdx.x >= deepBlocks) {
    grid_dependency_wait();
    grid_launch_dependents();
    residual_boundary_item<T, W, LoadDefault>(bPtr, bCol, bVal, bGlobal, nB, rhs, x, res, KP, G,
                                              (long long)(blockIdx.x - deepBlocks) * blockDim.x + threadIdx.x);
    return;
  }
  // deep items (residual_deep_item's arithmetic, same order): the run and its
  // coefficients (set-up data), and rhs when the previous launch does not
  // write it (rhsEarly), are loaded before waiting for the previous launch
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int per = 32 * G;
  const long long r = t / per;
  const int rem = int(t - r * per);
  const int m = rem / G, q = rem - m * G;
  ColourRun R;
  R.len = 0;
  if (r < nRuns) R = runs[r];
  const bool active = r < nRuns && m < R.len;
  T w[10];
  Vec<T, W> b;
  int pos = 0, pp = 0, pn = 0;
  const int off = q * W;
  if (active) {
    pos = R.pos0 + 2 * m, pp = R.prev0 + 2 * m, pn = R.next0 + 2 * m;
    const T* c = coef + R.coef0 + m;
#pragma unroll
    for (int k = 0; k < 10; k++)
      if (k != 4) w[k] = c[k * planeStride];
    if (rhsEarly) b = vload<T, W>(rhs + (long long)pos * KP + off);
  }
  grid_dependency_wait();
  grid_launch_dependents();
  if (!active) return;
  if (!rhsEarly) b = vload<T, W>(rhs + (long long)pos * KP + off);
  Vec<T, W> acc = vload<T, W>(x + (long long)pos * KP + off);
  axpy(acc, w[0], vload<T, W>(x + (long long)(pp - 1) * KP + off));
  axpy(acc, w[1], vload<T, W>(x + (long long)(pp)*KP + off));
  axpy(acc, w[2], vload<T, W>(x + (long long)(pp + 1) * KP + off));
  axpy(acc, w[3], vload<T, W>(x + (long long)(pos - 1) * KP + off));
  axpy(acc, w[5], vload<T, W>(x + (long long)(pos + 1) * KP + off));
  axpy(acc, w[6], vload<T, W>(x + (long long)(pn - 1) * KP + off));
  axpy(acc, w[7], vload<T, W>(x + (long long)(pn)*KP + off));
  axpy(acc, w[8], vload<T, W>(x + (long long)(pn + 1) * KP + off));
  Vec<T, W> out;
#pragma unroll
  for (int k = 0; k < W; k++) out.v[k] = b.v[k] - acc.v[k] * w[9];
  vstore<T, W>(res + (long long)pos * KP + off, out);
}

// ----------------------------------------------------------------------------
// Restriction of the residual to the coarse right-hand side.
// ----------------------------------------------------------------------------
template <typename T, int W>
__global__ void __launch_bounds__(256) k_restrict(const RestrictRun* __restrict__ runs, int nRuns, int deepBlocks,
                                                  const int* __restrict__ rPtr, const int* __restrict__ rCol,
                                                  const T* __restrict__ rVal, const int* __restrict__ rOut, int nB,
                                                  const T* __restrict__ res, T* __restrict__ coarseRhs, T* __restrict__ coarseX,
                                                  long long coarseVals, int KP, int G) {
  // the coarse iterate starts from zero: cleared here (grid-stride), before
  // waiting for the previous launch (the residual of this level, which does
  // not touch the coarse level)
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < coarseVals; i += (long long)gridDim.x * blockDim.x)
    coarseX[i] = T(0);
  grid_dependency_wait();
  grid_launch_dependents();
  if ((int)blockIdx.x < deepBlocks)
    restrict_deep_item<T, W, LoadDefault>(runs, nRuns, res, coarseRhs, KP, G, (long long)blockIdx.x * blockDim.x + threadIdx.x);
  else
    restrict_boundary_item<T, W, LoadDefault>(rPtr, rCol, rVal, rOut, nB, res, coarseRhs, KP, G,
                                              (long long)(blockIdx.x - deepBlocks) * blockDim.x + threadIdx.x);
}

// ----------------------------------------------------------------------------
// Prolongation of the coarse correction, added to the fine iterate.
// ----------------------------------------------------------------------------
template <typename T, int W>
__global__ void __launch_bounds__(256) k_prolong_add(const ProlongRun* __restrict__ runs, int nRuns, const T* __restrict__ coarse,
                                                     T* __restrict__ fine, int KP, int G) {
  // prolong_item's arithmetic; the run and the fine value (this level's iterate,
  // which the previous launch, on the coarse level, does not write) are loaded
  // before waiting for it, the coarse values after
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int per = 32 * G;
  const long long r = t / per;
  const int rem = int(t - r * per);
  const int m = rem / G, q = rem - m * G;
  ProlongRun R{};
  if (r < nRuns) R = runs[r];
  const bool active = r < nRuns && m < R.len;
  const int off = q * W;
  T* dst = active ? fine + (long long)(R.f0 + m) * KP + off : nullptr;
  Vec<T, W> acc;
  if (active) acc = vload<T, W>(dst);
  grid_dependency_wait();
  grid_launch_dependents();
  if (!active) return;
  const int i = R.i0 + m, o = R.aligned ? 0 : 1;
  const int p = (i + o) / 2, n = (i + o + 1) / 2;
  if (R.center >= 0) {
    const Vec<T, W> a = vload<T, W>(coarse + (long long)(R.center + p) * KP + off),
                    b = vload<T, W>(coarse + (long long)(R.center + n) * KP + off);
#pragma unroll
    for (int k = 0; k < W; k++) acc.v[k] += (a.v[k] + b.v[k]) * T(0.5);
  } else {
    const Vec<T, W> a = vload<T, W>(coarse + (long long)(R.prev + p) * KP + off),
                    b = vload<T, W>(coarse + (long long)(R.prev + n) * KP + off),
                    c = vload<T, W>(coarse + (long long)(R.next + p) * KP + off),
                    d = vload<T, W>(coarse + (long long)(R.next + n) * KP + off);
#pragma unroll
    for (int k = 0; k < W; k++) acc.v[k] += (a.v[k] + b.v[k] + c.v[k] + d.v[k]) * T(0.25);
  }
  vstore<T, W>(dst, acc);
}

// ----------------------------------------------------------------------------
// Exact boundary-block solve  x_B = BB^-1 (rhs_B - BD x) over the subdomain /
// separator split (scaled by s = BB_ii^-1/2), four launches per level:
//   k_bs_prep:          r^ = s (rhs - BD x) for every boundary position
//   k_bs_dense mode 0:  y  = Inv_p r^_I
//   k_bs_dense mode 1:  xs = Sinv t,      t  = r^_S - A_SI y built in the prologue;
//                       x_S = s xs
//   k_bs_back:          x_I = s (y - W_p xs),  W_p = Inv_p A_{I_p,S} (m x t_p)
// The sparse row sums run on 8 lanes per row (group8_sum in vcycle_ops.cuh).
// The dense products are memory-bound streams of the symmetric inverses,
// stored row-major with rows padded to a multiple of 4: lane l of a warp reads
// rows 4l..4l+3 of matrix row j with one vector load, so a warp reads
// contiguous memory.  A block takes 128 rows of one matrix and a chunk of its
// j range (8 warps interleave j); the chunks of a row group (blockIdx.y) write
// partial sums and the last block to finish adds them in chunk order, so the
// result does not depend on scheduling.  Chunking keeps the dependent-load
// chain of each warp short on the small coarse levels.
// ----------------------------------------------------------------------------

template <typename T, int W>
__global__ void __launch_bounds__(256, 3) k_bs_dense(BoundaryDev<T> B, int mode, const T* __restrict__ rhs, T* __restrict__ x, int KP,
                                                  int G) {
  __shared__ T red[8][32][4 * W];
  __shared__ Vec<T, W> vin[kBoundaryChunkMax];
  __shared__ int lastFlag;
  // the block's task, its matrix and its rows of it are set-up data: read (and
  // the rows prefetched into L2) before waiting for the previous launch
  const int4 task = (mode == 0 ? B.subTasks : B.schurTasks)[blockIdx.x];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, rq = task.y + lane;
  const int r0 = mode == 0 ? B.subPtr[task.x] : 0;
  const int m = mode == 0 ? B.subPtr[task.x + 1] - r0 : B.nS, mp = (m + 3) & ~3;
  const T* M = mode == 0 ? B.inv + B.invOff[task.x] : B.sinv;
  const int nch = gridDim.y, chunk = blockIdx.y;
  const int clen = (m + nch - 1) / nch, j0 = min(m, chunk * clen), j1 = min(m, j0 + clen);
  {
    // rows j0..j1 of columns 4 task.y .. 4 task.y + 127 (clipped to the padded row)
    const int c0 = 4 * task.y, cols = max(0, min(mp - c0, 128));
    if (cols > 0)
      for (int j = j0 + warp; j < j1; j += 8)
        if (lane * 32 < cols * (int)sizeof(T)) asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<const char*>(M + (long long)j * mp + c0) + lane * 32));
  }
  grid_dependency_wait();
  grid_launch_dependents();
  const bool active = 4 * rq < m;
  T* part = mode == 0 ? B.subPart : B.schurPart;
  for (int q = 0; q < G; q++) {
    const int off = q * W;
    // prologue: the chunk's input vector (mode 0: the scaled right-hand side
    // from k_bs_prep; mode 1: minus the coupling to the interior solution)
    if (mode == 0) {
      for (int j = j0 + (int)threadIdx.x; j < j1; j += blockDim.x)
        vin[j - j0] = vload<T, W>(B.rhat + (long long)(r0 + j) * KP + off);
    } else {
      const int lane8 = threadIdx.x & 7, grp = threadIdx.x >> 3;
      for (int jb = j0; jb < j1; jb += 32) {  // 32 groups of 8 lanes
        const int j = jb + grp;
        const Vec<T, W> v = bs_schur_input_group<T, W, LoadDefault>(B, j, j < j1, KP, off, lane8);
        if (j < j1 && lane8 == 0) vin[j - j0] = v;
      }
    }
    __syncthreads();
    T acc[4][W];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int c = 0; c < W; c++) acc[a][c] = 0;
    if (active) {
#pragma unroll 8
      for (int j = j0 + warp; j < j1; j += 8) {
        const Quad<T> mq = *reinterpret_cast<const Quad<T>*>(M + (long long)j * mp + 4 * rq);
        const Vec<T, W> v = vin[j - j0];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int c = 0; c < W; c++) acc[a][c] += mq.v[a] * v.v[c];
      }
    }
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int c = 0; c < W; c++) red[warp][lane][a * W + c] = acc[a][c];
    __syncthreads();
    if (warp == 0 && active) {
#pragma unroll
      for (int a = 0; a < 4; a++) {
        const int row = 4 * rq + a;
        if (row >= m) continue;
        Vec<T, W> sum;
#pragma unroll
        for (int c = 0; c < W; c++) {
          T v = 0;
          for (int w = 0; w < 8; w++) v += red[w][lane][a * W + c];
          sum.v[c] = v;
        }
        if (nch > 1) {
          vstore<T, W>(part + (((long long)blockIdx.x * nch + chunk) * 128 + 4 * lane + a) * KP + off, sum);
        } else if (mode == 0) {
          vstore<T, W>(B.y + (long long)(r0 + row) * KP + off, sum);
        } else {
          vstore<T, W>(B.xs + (long long)row * KP + off, sum);
          const T sc = B.scale[B.nI + row];
#pragma unroll
          for (int c = 0; c < W; c++) sum.v[c] *= sc;
          vstore<T, W>(x + (long long)B.posGlobal[B.nI + row] * KP + off, sum);
        }
      }
    }
    __syncthreads();
  }
  if (nch == 1) return;
  // the last chunk of this row group to finish adds the partials in chunk order
  __threadfence();
  __syncthreads();
  int* counter = (mode == 0 ? B.subCount : B.schurCount) + blockIdx.x;
  if (threadIdx.x == 0) {
    const int prev = atomicAdd(counter, 1);
    lastFlag = prev == nch - 1;
    if (lastFlag) *counter = 0;  // ready for the next launch
  }
  __syncthreads();
  if (!lastFlag) return;
  __threadfence();
  for (int it = threadIdx.x; it < 128 * G; it += blockDim.x) {
    const int rt = it / G, q = it - rt * G, row = 4 * task.y + rt, off = q * W;
    if (row >= m) continue;
    Vec<T, W> sum;
#pragma unroll
    for (int c = 0; c < W; c++) sum.v[c] = 0;
#pragma unroll 4
    for (int ch = 0; ch < nch; ch++) {
      const T* src = part + (((long long)blockIdx.x * nch + ch) * 128 + rt) * KP + off;
#pragma unroll
      for (int c = 0; c < W; c++) sum.v[c] += __ldcg(src + c);
    }
    if (mode == 0) {
      vstore<T, W>(B.y + (long long)(r0 + row) * KP + off, sum);
    } else {
      vstore<T, W>(B.xs + (long long)row * KP + off, sum);
      const T sc = B.scale[B.nI + row];
#pragma unroll
      for (int c = 0; c < W; c++) sum.v[c] *= sc;
      vstore<T, W>(x + (long long)B.posGlobal[B.nI + row] * KP + off, sum);
    }
  }
}

// x_I = s (y - W_p xs[touch_p]) for every interior position (W_p column-major,
// so a warp reads consecutive rows of one column)
template <typename T, int W>
__global__ void __launch_bounds__(256) k_bs_back(BoundaryDev<T> B, T* __restrict__ x, int KP, int G, int yEarly) {
  // bs_back_group's arithmetic.  Before waiting for the previous launch (the
  // separator product, which writes xs): the row's subdomain, its W_p column
  // range and scale (set-up data), and y when yEarly (then y comes from the
  // subdomain product, which the previous launch itself waited for)
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long gi = t >> 3;
  const int lane8 = int(t & 7);
  const long long i = gi / G;
  const int q = int(gi - i * G), off = q * W;
  const bool valid = i < B.nI;
  int m = 0, e0 = 0, e1 = 0;
  const T* Wp = nullptr;
  Vec<T, W> yv;
  T sc = T(0);
  int g = 0;
  if (valid) {
    const int p = B.rowSub[i];
    const int b0 = B.subPtr[p];
    m = B.subPtr[p + 1] - b0;
    Wp = B.wt + B.wOff[p] + (int(i) - b0);
    e0 = B.touchPtr[p];
    e1 = B.touchPtr[p + 1];
    if (lane8 == 0) {
      if (yEarly) yv = vload<T, W>(B.y + i * KP + off);
      sc = B.scale[i];
      g = B.posGlobal[i];
    }
  }
  grid_dependency_wait();
  grid_launch_dependents();
  if (valid && lane8 == 0 && !yEarly) yv = vload<T, W>(B.y + i * KP + off);
  Vec<T, W> acc;
#pragma unroll
  for (int c = 0; c < W; c++) acc.v[c] = 0;
  if (valid)
    for (int e = e0 + lane8; e < e1; e += 8) axpy(acc, Wp[(long long)(e - e0) * m], vload<T, W>(B.xs + (long long)B.touch[e] * KP + off));
  acc = group8_sum(acc);
  if (valid && lane8 == 0) {
#pragma unroll
    for (int c = 0; c < W; c++) yv.v[c] = (yv.v[c] - acc.v[c]) * sc;
    vstore<T, W>(x + (long long)g * KP + off, yv);
  }
}

// rhat = s (rhs - BD x) for every boundary position, 8 lanes per position
template <typename T, int W>
__global__ void __launch_bounds__(256) k_bs_prep(BoundaryDev<T> B, const T* __restrict__ rhs, const T* __restrict__ x, int KP, int G,
                                                 int rhsEarly) {
  // bs_prep_group's arithmetic.  Before waiting for the previous launch: the
  // row's BD range, position and scale (set-up data), and rhs when the previous
  // launch does not write it (rhsEarly: the prolongation before a boundary solve
  // after the coarse correction)
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long gi = t >> 3;
  const int lane8 = int(t & 7);
  const long long k = gi / G;
  const int q = int(gi - k * G), off = q * W;
  const bool valid = k < B.nb;
  int e0 = 0, e1 = 0, g = 0;
  T sc = T(0);
  Vec<T, W> r;
  if (valid) {
    e0 = B.bdPtr[k];
    e1 = B.bdPtr[k + 1];
    if (lane8 == 0) {
      g = B.posGlobal[k];
      sc = B.scale[k];
      if (rhsEarly) r = vload<T, W>(rhs + (long long)g * KP + off);
    }
  }
  grid_dependency_wait();
  grid_launch_dependents();
  Vec<T, W> acc;
#pragma unroll
  for (int c = 0; c < W; c++) acc.v[c] = 0;
  if (valid)
    for (int e = e0 + lane8; e < e1; e += 8) axpy(acc, B.bdVal[e], vload<T, W>(x + (long long)B.bdCol[e] * KP + off));
  acc = group8_sum(acc);
  if (valid && lane8 == 0) {
    if (!rhsEarly) r = vload<T, W>(rhs + (long long)g * KP + off);
#pragma unroll
    for (int c = 0; c < W; c++) r.v[c] = (r.v[c] - acc.v[c]) * sc;
    vstore<T, W>(B.rhat + k * KP + off, r);
  }
}

// L2 prefetch of [p, p + bytes) by the threads of a block (128-byte lines);
// used for set-up matrices before a kernel waits for the previous launch
__device__ __forceinline__ void prefetch_l2_block(const void* p, long long bytes) {
  const char* c = static_cast<const char*>(p);
  for (long long o = (long long)threadIdx.x * 128; o < bytes; o += (long long)blockDim.x * 128)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(c + o));
}

// ----------------------------------------------------------------------------
// Coarsest level: x = D Ainv^ D rhs with the scaled dense inverse (FP64).
// ----------------------------------------------------------------------------
template <typename T, int W>
__global__ void __launch_bounds__(256) k_coarse_solve(int n, const double* __restrict__ ainv, const double* __restrict__ scale,
                                                      const T* __restrict__ rhs, T* __restrict__ x, int KP, int G) {
  // this block's two rows of the inverse (set-up data) start moving into L2
  // while the previous launch finishes
  {
    const int r0 = blockIdx.x * 2;
    if (r0 < n) prefetch_l2_block(ainv + (long long)r0 * n, (long long)min(2, n - r0) * n * sizeof(double));
  }
  grid_dependency_wait();
  grid_launch_dependents();
  // 2 rows per block, a warp per part of a row, parts added in order
  __shared__ double part[2][kCoarseParts][4 * W];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rl = warp / kCoarseParts, p = warp % kCoarseParts, row = blockIdx.x * 2 + rl;
  for (int q = 0; q < G; q++) {
    const int off = q * W;
    double acc[W];
    if (row < n) coarse_part<T, W, LoadDefault>(n, ainv, scale, rhs, KP, off, row, p, lane, acc);
    if (row < n && lane == 0)
#pragma unroll
      for (int c = 0; c < W; c++) part[rl][p][c] = acc[c];
    __syncthreads();
    if (threadIdx.x < 2 * W) {
      const int r2 = threadIdx.x / W, c = threadIdx.x % W, rr = blockIdx.x * 2 + r2;
      if (rr < n) {
        double sum = 0;
        for (int pp = 0; pp < kCoarseParts; pp++) sum += part[r2][pp][c];
        x[(long long)rr * KP + off + c] = T(sum * scale[rr]);
      }
    }
    __syncthreads();
  }
}

// Per-block sums of two per-channel accumulators into partials[block][0..K) and
// [K..2K): lanes l and l^s (s >= G) hold the same channel group, then the warps
// are added in a fixed order (deterministic).  All threads of the block call it.
__device__ __forceinline__ void block_partials(double (&ra)[4], double (&rb)[4], int G, int K, double* partials) {
  __shared__ double red[8][2][64];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int ch = 0; ch < 4; ch++)
    for (int s = 16; s >= G; s >>= 1) {
      ra[ch] += __shfl_xor_sync(0xffffffffu, ra[ch], s);
      rb[ch] += __shfl_xor_sync(0xffffffffu, rb[ch], s);
    }
  if (lane < G)
#pragma unroll
    for (int ch = 0; ch < 4; ch++)
      if (4 * lane + ch < K) { red[warp][0][4 * lane + ch] = ra[ch]; red[warp][1][4 * lane + ch] = rb[ch]; }
  __syncthreads();
  if ((int)threadIdx.x < K) {
    double a = 0, c = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) { a += red[w][0][threadIdx.x]; c += red[w][1][threadIdx.x]; }
    partials[(long long)blockIdx.x * 2 * K + threadIdx.x] = a;
    partials[(long long)blockIdx.x * 2 * K + K + threadIdx.x] = c;
  }
}

// ----------------------------------------------------------------------------
// FP64 raw operator: res = b - A x (mode 0), y = A x (mode 1), y = A x with
// the partial sums of x . y instead of y . y (mode 2), or res = b for x = 0
// (mode 3: the stencil and x are not read; A 0 sums signed zeros to +0, so
// mode 0 on x = 0 gives these bits) on tight n x K vectors.  Deep rows use 9 raw coefficients per run texel (line runs:
// up to 32 consecutive deep texels of a raster line), boundary rows
// the merged BD/BB CSR.  A thread handles one texel and up to 4 channels
// (group q of G = KP/4 groups, or G = 1 for K = 1).  Per-block sums of res^2
// and b^2 per channel go to `partials` for a deterministic norm reduction.
// ----------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_raw_operator(const ColourRun* __restrict__ runs, int nRuns, const double* __restrict__ coef,
                                                      int planeStride, const int* __restrict__ bPtr, const int* __restrict__ bCol,
                                                      const double* __restrict__ bVal, const int* __restrict__ bGlobal, int nB,
                                                      const double* __restrict__ b, const double* __restrict__ x,
                                                      double* __restrict__ out, int K, int G, int mode, double* __restrict__ partials,
                                                      float* __restrict__ out32 = nullptr, int KP = 0) {
  grid_dependency_wait();
  grid_launch_dependents();
  // grid-stride over deep items (runs x 32 x G) then boundary items (rows x G);
  // the stride is a multiple of G, so every thread keeps one channel group q
  const long long nDeepItems = (long long)nRuns * 32 * G, nItems = nDeepItems + (long long)nB * G;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int q = int(t0 % G);
  double rr[4] = {0, 0, 0, 0}, bb[4] = {0, 0, 0, 0};
  for (long long t = t0; t < nItems; t += stride) {
    double acc[4] = {0, 0, 0, 0};
    int g = -1;
    if (t < nDeepItems) {
      const long long r = t / (32 * G);
      const int m = int(t - r * 32 * G) / G;
      const ColourRun R = runs[r];
      if (m < R.len && mode == 3) {
        g = R.pos0 + m;
      } else if (m < R.len) {  // line runs: consecutive texels
        const int pos = R.pos0 + m, pp = R.prev0 + m, pn = R.next0 + m;
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
    } else {
      const long long row = (t - nDeepItems) / G;
      for (int k = mode == 3 ? bPtr[row + 1] : bPtr[row]; k < bPtr[row + 1]; k++) {
        const double w = bVal[k];
        const double* xs = x + (long long)bCol[k] * K + 4 * q;
#pragma unroll
        for (int ch = 0; ch < 4; ch++)
          if (4 * q + ch < K) acc[ch] += w * xs[ch];
      }
      g = bGlobal[row];
    }
    if (g >= 0) {
#pragma unroll
      for (int ch = 0; ch < 4; ch++) {
        const int c = 4 * q + ch;
        if (c >= K) continue;
        const double bv = b ? b[(long long)g * K + c] : 0.0;
        const double v = (mode == 0 || mode == 3) ? bv - acc[ch] : acc[ch];
        if (out32) out32[(long long)g * KP + c] = float(v);
        else out[(long long)g * K + c] = v;
        rr[ch] += mode == 2 ? x[(long long)g * K + c] * v : v * v;  // mode 2: x . A x
        bb[ch] += bv * bv;
      }
      if (out32)  // zero the padding channels of this group
        for (int c = max(K, 4 * q); c < min(KP, 4 * q + 4); c++) out32[(long long)g * KP + c] = 0.f;
    }
  }
  if (!partials) return;
  block_partials(rr, bb, G, K, partials);
}

// Small exchanges of the solve loops with the host, kept off the copy engines
// (which a streaming solve keeps busy with whole vectors): the norms are
// written into mapped pinned host memory, the per-right-hand-side flags come
// in as a kernel argument.  One block each.
__global__ void k_copy_f64(double* __restrict__ dst, const double* __restrict__ src, int n) {
  grid_dependency_wait();
  grid_launch_dependents();
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}
__global__ void k_set_flags(int* __restrict__ flags, unsigned long long mask, int k) {
  grid_dependency_wait();
  grid_launch_dependents();
  const int c = threadIdx.x;
  if (c < k) flags[c] = int((mask >> c) & 1ull);
}

// Sum of per-block partials in a fixed order (one block): sums[2K]; up to
// kSumWide sums (K <= 4: the solve's right-hand sides) reduced side by side
constexpr int kSumWide = 8;
__global__ void k_sum_partials(const double* __restrict__ partials, int nBlocks, int K, double* __restrict__ sums) {
  grid_dependency_wait();
  grid_launch_dependents();
  __shared__ double sh[256];
  if (2 * K <= kSumWide) {
    // every sum at once (one tree for all of them): per sum the same thread
    // partials, in the same order, and the same tree as the loop below
    __shared__ double shw[kSumWide][256];
    double s[kSumWide];
#pragma unroll
    for (int c = 0; c < kSumWide; c++) s[c] = 0;
    for (int b = threadIdx.x; b < nBlocks; b += blockDim.x)
#pragma unroll
      for (int c = 0; c < kSumWide; c++)
        if (c < 2 * K) s[c] += partials[(long long)b * 2 * K + c];
#pragma unroll
    for (int c = 0; c < kSumWide; c++) shw[c][threadIdx.x] = s[c];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
      if ((int)threadIdx.x < w)
#pragma unroll
        for (int c = 0; c < kSumWide; c++)
          if (c < 2 * K) shw[c][threadIdx.x] += shw[c][threadIdx.x + w];
      __syncthreads();
    }
    if ((int)threadIdx.x < 2 * K) sums[threadIdx.x] = shw[threadIdx.x][0];
    return;
  }
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

// ----------------------------------------------------------------------------
// Flexible preconditioned conjugate gradients around the FP32 V-cycle (FP64
// vectors, tight n x K; per right-hand side scalars in `sc`: alpha [0,K),
// beta [K,2K), rho [2K,3K), previous rho [3K,4K)).  Items are texels x channel
// groups of 4 over a fixed grid, so the partial sums have a fixed order.
// ----------------------------------------------------------------------------
// z = e (V-cycle output, FP32 padded), e cleared; partials: z . r and z . q
__global__ void __launch_bounds__(256) k_fcg_precond(long long n, int K, int KP, int G, float* __restrict__ e,
                                                     const double* __restrict__ r, const double* __restrict__ q,
                                                     double* __restrict__ z, double* __restrict__ partials) {
  grid_dependency_wait();
  grid_launch_dependents();
  const long long stride = (long long)gridDim.x * blockDim.x, t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int qg = int(t0 % G);
  double a[4] = {0, 0, 0, 0}, b[4] = {0, 0, 0, 0};
  for (long long t = t0; t < n * G; t += stride) {
    const long long i = t / G;
#pragma unroll
    for (int ch = 0; ch < 4; ch++) {
      const int c = 4 * qg + ch;
      if (c >= K) continue;
      const double v = double(e[i * KP + c]);
      e[i * KP + c] = 0.f;
      z[i * K + c] = v;
      a[ch] += v * r[i * K + c];
      b[ch] += v * q[i * K + c];
    }
  }
  block_partials(a, b, G, K, partials);
}

// beta = -alpha_old (z . q_old) / rho_old (0 on a (re)start, rho_old = 0); rho = z . r
__global__ void k_fcg_beta(int K, const double* __restrict__ sums, double* __restrict__ sc) {
  grid_dependency_wait();
  grid_launch_dependents();
  const int c = threadIdx.x;
  if (c >= K) return;
  const double rho = sums[c], gamma = sums[K + c], rhoOld = sc[3 * K + c];
  sc[K + c] = rhoOld != 0.0 ? -sc[c] * gamma / rhoOld : 0.0;
  sc[2 * K + c] = rho;
  sc[3 * K + c] = rho;
}

// p = z + beta p
__global__ void __launch_bounds__(256) k_fcg_direction(long long n, int K, const double* __restrict__ z, const double* __restrict__ sc,
                                                       double* __restrict__ p) {
  grid_dependency_wait();
  grid_launch_dependents();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * K) return;
  const int c = int(t % K);
  p[t] = z[t] + sc[K + c] * p[t];
}

// alpha = rho / (p . A p), 0 for frozen right-hand sides
__global__ void k_fcg_alpha(int K, const double* __restrict__ sums, const int* __restrict__ frozen, double* __restrict__ sc) {
  grid_dependency_wait();
  grid_launch_dependents();
  const int c = threadIdx.x;
  if (c >= K) return;
  const double pq = sums[c];
  sc[c] = (frozen && frozen[c]) || !(pq > 0) ? 0.0 : sc[2 * K + c] / pq;
}

// x += alpha p, r -= alpha q, r packed into the next V-cycle's FP32 right-hand
// side; partials: r . r and 0
__global__ void __launch_bounds__(256) k_fcg_update(long long n, int K, int KP, int G, const double* __restrict__ sc,
                                                    const double* __restrict__ p, const double* __restrict__ q, double* __restrict__ x,
                                                    double* __restrict__ r, float* __restrict__ rhs32, double* __restrict__ partials) {
  grid_dependency_wait();
  grid_launch_dependents();
  const long long stride = (long long)gridDim.x * blockDim.x, t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int qg = int(t0 % G);
  double a[4] = {0, 0, 0, 0}, b[4] = {0, 0, 0, 0};
  for (long long t = t0; t < n * G; t += stride) {
    const long long i = t / G;
#pragma unroll
    for (int ch = 0; ch < 4; ch++) {
      const int c = 4 * qg + ch;
      if (c >= K) continue;
      const double al = sc[c];
      x[i * K + c] += al * p[i * K + c];
      const double rv = r[i * K + c] - al * q[i * K + c];
      r[i * K + c] = rv;
      rhs32[i * KP + c] = float(rv);
      a[ch] += rv * rv;
    }
  }
  block_partials(a, b, G, K, partials);
}

// out = a x + b y (the system operator's planes from the mass and stiffness planes)
__global__ void k_axpby(double* __restrict__ out, double a, const double* __restrict__ x, double b, const double* __restrict__ y,
                        long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a * x[i] + b * y[i];
}

// FP64 residual (n*K, tight) -> FP32 right-hand side (n*KP, padded)
template <typename T>
__global__ void k_pack_rhs(const double* __restrict__ r, T* __restrict__ rhs, long long n, int K, int KP) {
  grid_dependency_wait();
  grid_launch_dependents();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * KP) return;
  const long long i = t / KP;
  const int c = int(t - i * KP);
  rhs[t] = c < K ? T(r[i * K + c]) : T(0);
}
// x64 += e (padded FP32/FP64 correction); e is cleared for the next V-cycle
// (its padding lanes stay zero through the V-cycle).  Columns with frozen[c]
// set keep their x: a right-hand side that has converged stops changing, so
// its result does not depend on what it was solved together with.
template <typename T>
__global__ void k_add_correction(double* __restrict__ x, T* __restrict__ e, long long n, int K, int KP, const int* __restrict__ frozen) {
  grid_dependency_wait();
  grid_launch_dependents();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * K) return;
  const long long i = t / K;
  const int c = int(t - i * K);
  if (!frozen || !frozen[c]) x[t] += double(e[i * KP + c]);
  e[i * KP + c] = T(0);
}

// ----------------------------------------------------------------------------
// launch wrappers
// ----------------------------------------------------------------------------
static inline int nblk(long long threads) { return int((threads + 255) / 256); }

static bool g_programmatic = true;
void set_programmatic_launch(bool on) { g_programmatic = on; }
bool programmatic_launch() { return g_programmatic; }

// Every V-cycle kernel is launched with programmatic stream serialization:
// inside a captured graph consecutive kernels get programmatic edges, so a
// kernel is scheduled while its predecessor drains (each kernel waits in
// grid_dependency_wait() before touching memory).
template <typename... P, typename... A>
static void launch(void (*kernel)(P...), dim3 grid, cudaStream_t s, A... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = g_programmatic ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kernel, static_cast<P>(args)...);
}

template <typename T, int W>
void launch_gs_colour(const ColourRun* runs, int nRuns, const T* coef, int planeStride, const T* rhs, T* x, int KP,
                      cudaStream_t s, int skip, bool rhsEarly) {
  if (nRuns == 0) return;
  const int G = KP / W;
  launch(k_gs_colour<T, W>, dim3(nblk((long long)nRuns * 32 * G)), s, runs, nRuns, coef, planeStride, rhs, x, KP, G, skip,
         rhsEarly ? 1 : 0);
}
template <typename T, int W>
size_t gs_rows_smem(const LevelDev<T>& D) {
  return size_t(3) * D.rowSlots * sizeof(Vec<T, W>);  // three rows
}
// The row smoother's shared memory fits this device (its attribute set): 1, else 0.
template <typename T, int W, int BS>
static int gs_rows_ready() {
  static std::atomic<int> slots[kMaxDevices];
  static const bool init = [] {
    for (auto& v : slots) v.store(kUnset);
    return true;
  }();
  (void)init;
  return per_device_once(slots, [] {
    const int smem = int(3 * row_slot_cap(BS) * sizeof(Vec<T, W>));
    if (cudaFuncSetAttribute(k_gs_rows<T, W, BS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    return 1;
  });
}
template <typename T, int W, int BS>
static bool launch_gs_rows_bs(const LevelDev<T>& D, int rows, bool oddFirst, int KP, cudaStream_t s, int skip, bool rhsEarly) {
  if (gs_rows_ready<T, W, BS>() <= 0) return false;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(D.nRowBins[rows]), unsigned(KP / W));
  cfg.blockDim = dim3(BS);
  cfg.dynamicSmemBytes = gs_rows_smem<T, W>(D);
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = g_programmatic ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k_gs_rows<T, W, BS>, D.rowLines[rows], D.rowLineOf[rows], D.coef, D.planeStride,
                     static_cast<const T*>(D.b), D.x, KP, D.rowSlots, oddFirst ? 1 : 0, skip, rhsEarly ? 1 : 0);
  return true;
}
template <typename T, int W>
bool gs_rows_available(const LevelDev<T>& D) {
  if (D.rowBlock == 256) return gs_rows_ready<T, W, 256>() > 0;
  if (D.rowBlock == 512) return gs_rows_ready<T, W, 512>() > 0;
  if (D.rowBlock == 1024) return gs_rows_ready<T, W, 1024>() > 0;
  return false;
}
template <typename T, int W>
bool launch_gs_rows(const LevelDev<T>& D, int rows, bool oddFirst, int KP, cudaStream_t s, int skip, bool rhsEarly) {
  if (D.nRowBins[rows] == 0) return true;
  if (D.rowBlock == 256) return launch_gs_rows_bs<T, W, 256>(D, rows, oddFirst, KP, s, skip, rhsEarly);
  if (D.rowBlock == 512) return launch_gs_rows_bs<T, W, 512>(D, rows, oddFirst, KP, s, skip, rhsEarly);
  if (D.rowBlock == 1024) return launch_gs_rows_bs<T, W, 1024>(D, rows, oddFirst, KP, s, skip, rhsEarly);
  return false;
}
template <typename T, int W>
size_t gs_groups_smem(const LevelDev<T>& D, int KP) {
  return size_t(D.maxGroupSpan) * KP * sizeof(T);
}
template <typename T, int W>
bool launch_gs_groups(const LevelDev<T>& D, int sweeps, bool reverse, int KP, cudaStream_t s, bool rhsEarly) {
  if (D.nGroups == 0 || sweeps <= 0) return true;
  const size_t smem = gs_groups_smem<T, W>(D, KP);
  if (smem > kGroupSmemMax) return false;
  if constexpr (std::is_same<T, float>::value) {
    // one channel group, every colour pass of a chart within one block: the
    // register-staged variant
    if (KP == W && D.maxGroupColourRuns > 0 && D.maxGroupColourRuns * 32 <= kGroupRegBlock) {
      auto kern = reverse ? k_gs_groups_reg<W, true> : k_gs_groups_reg<W, false>;
      static std::atomic<int> regAttr[2][kMaxDevices];
      static const bool regInit = [] {
        for (auto& r : regAttr)
          for (auto& a : r) a.store(kUnset);
        return true;
      }();
      (void)regInit;
      const int okReg = per_device_once(regAttr[reverse ? 1 : 0], [kern] {
        return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kGroupSmemMax)) == cudaSuccess ? 1 : 0;
      });
      if (okReg) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(D.nGroups);
        cfg.blockDim = dim3(std::max(128, D.maxGroupColourRuns * 32));
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = g_programmatic ? 1 : 0;
        return cudaLaunchKernelEx(&cfg, kern, D.runs, D.groups, (const float*)D.coef, D.planeStride, (const float*)D.b, D.x, sweeps,
                                  rhsEarly ? 1 : 0) == cudaSuccess;
      }
    }
  }
  static std::atomic<int> attr[kMaxDevices];
  static const bool init = [] {
    for (auto& a : attr) a.store(kUnset);
    return true;
  }();
  (void)init;
  const int ok = per_device_once(attr, [] {
    return cudaFuncSetAttribute(k_gs_groups<T, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kGroupSmemMax)) == cudaSuccess ? 1
                                                                                                                              : 0;
  });
  if (!ok) return false;
  const int G = KP / W;
  // threads: the largest colour pass of a chart, in warps, at most 1024
  const int items = 32 * G * std::max(1, (D.maxGroupDeep / 4 + 31) / 32 + 1);
  const int nt = std::min(kGroupBlockMax, std::max(128, (items + 31) / 32 * 32));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(D.nGroups);
  cfg.blockDim = dim3(nt);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = g_programmatic ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k_gs_groups<T, W>, D.runs, D.groups, (const T*)D.coef, D.planeStride, (const T*)D.b, D.x, KP, G,
                            sweeps, reverse ? 1 : 0) == cudaSuccess;
}
template <typename T, int W>
void launch_residual(const ColourRun* runs, int nRuns, const T* coef, int planeStride, const int* bPtr, const int* bCol,
                     const T* bVal, const int* bGlobal, int nB, const T* rhs, const T* x, T* res, int KP, cudaStream_t s,
                     bool rhsEarly) {
  const int G = KP / W;
  const int db = nblk((long long)nRuns * 32 * G), bb = nblk((long long)nB * G);
  if (db + bb == 0) return;
  launch(k_residual<T, W>, dim3(db + bb), s, runs, nRuns, coef, planeStride, db, bPtr, bCol, bVal, bGlobal, nB, rhs, x, res, KP, G,
         rhsEarly ? 1 : 0);
}
template <typename T, int W>
void launch_restrict(const RestrictRun* runs, int nRuns, const int* rPtr, const int* rCol, const T* rVal, const int* rOut,
                     int nB, const T* res, T* coarseRhs, T* coarseX, long long coarseTexels, int KP, cudaStream_t s) {
  const int G = KP / W;
  const int db = nblk((long long)nRuns * 32 * G), bb = nblk((long long)nB * G);
  if (db + bb == 0 && coarseTexels == 0) return;
  launch(k_restrict<T, W>, dim3(std::max(1, db + bb)), s, runs, nRuns, db, rPtr, rCol, rVal, rOut, nB, res, coarseRhs, coarseX,
         coarseTexels * KP, KP, G);
}
template <typename T, int W>
void launch_prolong_add(const ProlongRun* runs, int nRuns, const T* coarse, T* fine, int KP, cudaStream_t s) {
  if (nRuns == 0) return;
  const int G = KP / W;
  launch(k_prolong_add<T, W>, dim3(nblk((long long)nRuns * 32 * G)), s, runs, nRuns, coarse, fine, KP, G);
}
template <typename T, int W>
void launch_boundary_solve(const BoundaryDev<T>& B, const T* rhs, T* x, int KP, cudaStream_t s, bool rhsEarly) {
  if (B.nb == 0) return;
  const int G = KP / W;
  launch(k_bs_prep<T, W>, dim3(nblk((long long)B.nb * G * 8)), s, B, rhs, x, KP, G, rhsEarly ? 1 : 0);
  if (B.nSubTasks > 0) launch(k_bs_dense<T, W>, dim3(B.nSubTasks, B.subChunks), s, B, 0, rhs, x, KP, G);
  if (B.nS > 0) launch(k_bs_dense<T, W>, dim3(B.nSchurTasks, B.schurChunks), s, B, 1, rhs, x, KP, G);
  // y comes from the subdomain product: read early only when the separator
  // product sits between the two launches
  if (B.nI > 0) launch(k_bs_back<T, W>, dim3(nblk((long long)B.nI * G * 8)), s, B, x, KP, G, B.nS > 0 ? 1 : 0);
}
template <typename T, int W>
void launch_coarse_solve(int n, const double* ainv, const double* scale, const T* rhs, T* x, int KP, cudaStream_t s) {
  if (n == 0) return;
  launch(k_coarse_solve<T, W>, dim3((n + 1) / 2), s, n, ainv, scale, rhs, x, KP, KP / W);
}

static inline int raw_groups(int K) { int G = 1; while (4 * G < K) G *= 2; return G; }
// fixed grid (grid-stride): bounded number of partial sums, launch-shape-independent order
// Fixed grid of the FP64 operator and its reductions: 8 blocks per SM of the
// device (its partial sums are added in block order, so one device always gives
// the same bits), at most kRawMaxBlocks.
static int raw_blocks() {
  static std::atomic<int> slots[kMaxDevices];
  static const bool init = [] {
    for (auto& a : slots) a.store(kUnset);
    return true;
  }();
  (void)init;
  return per_device_once(slots, [] {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        sms <= 0)
      return kRawMaxBlocks;
    return std::min(kRawMaxBlocks, 8 * sms);
  });
}
void launch_raw_operator(const ColourRun* runs, int nRuns, const double* coef, int planeStride, const int* bPtr, const int* bCol,
                         const double* bVal, const int* bGlobal, int nB, const double* b, const double* x, double* out, int K,
                         int mode, double* partials, double* sums, cudaStream_t s) {
  const int G = raw_groups(K);
  const long long items = (long long)nRuns * 32 * G + (long long)nB * G;
  if (items == 0) return;
  const int blocks = int(std::min<long long>(raw_blocks(), nblk(items)));
  launch(k_raw_operator, dim3(blocks), s, runs, nRuns, coef, planeStride, bPtr, bCol, bVal, bGlobal, nB, b, x, out, K, G, mode,
         partials, (float*)nullptr, 0);
  if (partials && sums) launch(k_sum_partials, dim3(1), s, partials, blocks, K, sums);
}
int raw_operator_blocks(int nRuns, int nB, int K) { return raw_blocks(); }
void launch_raw_residual_f32(const ColourRun* runs, int nRuns, const double* coef, int planeStride, const int* bPtr,
                             const int* bCol, const double* bVal, const int* bGlobal, int nB, const double* b, const double* x,
                             float* rhs32, int K, int KP, double* partials, double* sums, cudaStream_t s, bool xZero) {
  const int G = raw_groups(K);
  const long long items = (long long)nRuns * 32 * G + (long long)nB * G;
  if (items == 0) return;
  const int blocks = int(std::min<long long>(raw_blocks(), nblk(items)));
  launch(k_raw_operator, dim3(blocks), s, runs, nRuns, coef, planeStride, bPtr, bCol, bVal, bGlobal, nB, b, x, (double*)nullptr, K,
         G, xZero ? 3 : 0, partials, rhs32, KP);
  if (partials && sums) launch(k_sum_partials, dim3(1), s, partials, blocks, K, sums);
}

// ---- flexible CG steps (fixed grids: partial sums in a fixed order)
static inline int fcg_blocks(long long n, int G) { return int(std::min<long long>(raw_blocks(), nblk(n * G))); }
void launch_fcg_precond(long long n, int K, int KP, float* e, const double* r, const double* q, double* z, double* partials,
                        double* sums, double* sc, cudaStream_t s) {
  const int G = raw_groups(K), blocks = fcg_blocks(n, G);
  launch(k_fcg_precond, dim3(blocks), s, n, K, KP, G, e, r, q, z, partials);
  launch(k_sum_partials, dim3(1), s, partials, blocks, K, sums);
  launch(k_fcg_beta, dim3(1), s, K, (const double*)sums, sc);
}
void launch_fcg_direction(long long n, int K, const double* z, const double* sc, double* p, cudaStream_t s) {
  launch(k_fcg_direction, dim3(nblk(n * K)), s, n, K, z, sc, p);
}
void launch_fcg_alpha(int K, const double* sums, const int* frozen, double* sc, cudaStream_t s) {
  launch(k_fcg_alpha, dim3(1), s, K, sums, frozen, sc);
}
void launch_fcg_update(long long n, int K, int KP, const double* sc, const double* p, const double* q, double* x, double* r, float* rhs32,
                       double* partials, double* sums, cudaStream_t s) {
  const int G = raw_groups(K), blocks = fcg_blocks(n, G);
  launch(k_fcg_update, dim3(blocks), s, n, K, KP, G, sc, p, q, x, r, rhs32, partials);
  launch(k_sum_partials, dim3(1), s, partials, blocks, K, sums);
}
void launch_raw_apply_dot(const ColourRun* runs, int nRuns, const double* coef, int planeStride, const int* bPtr, const int* bCol,
                          const double* bVal, const int* bGlobal, int nB, const double* x, double* out, int K, double* partials,
                          double* sums, cudaStream_t s) {
  const int G = raw_groups(K);
  const long long items = (long long)nRuns * 32 * G + (long long)nB * G;
  if (items == 0) return;
  const int blocks = int(std::min<long long>(raw_blocks(), nblk(items)));
  launch(k_raw_operator, dim3(blocks), s, runs, nRuns, coef, planeStride, bPtr, bCol, bVal, bGlobal, nB, (const double*)nullptr, x,
         out, K, G, 2, partials, (float*)nullptr, 0);
  launch(k_sum_partials, dim3(1), s, partials, blocks, K, sums);
}

void launch_axpby(double* out, double a, const double* x, double b, const double* y, long long n, cudaStream_t s) {
  if (n > 0) k_axpby<<<nblk(n), 256, 0, s>>>(out, a, x, b, y, n);
}
template <typename T>
void launch_pack_rhs(const double* r, T* rhs, long long n, int K, int KP, cudaStream_t s) {
  launch(k_pack_rhs<T>, dim3(nblk(n * KP)), s, r, rhs, n, K, KP);
}
void launch_copy_f64(double* dst, const double* src, int n, cudaStream_t s) { launch(k_copy_f64, dim3(1), s, dst, src, n); }
void launch_set_flags(int* flags, unsigned long long mask, int k, cudaStream_t s) {
  launch(k_set_flags, dim3(1), s, flags, mask, k);
}
template <typename T>
void launch_add_correction(double* x, T* e, long long n, int K, int KP, cudaStream_t s, const int* frozen) {
  launch(k_add_correction<T>, dim3(nblk(n * K)), s, x, e, n, K, KP, frozen);
}

#define GDTP_INSTANTIATE(T, W)                                                                                             \
  template void launch_gs_colour<T, W>(const ColourRun*, int, const T*, int, const T*, T*, int, cudaStream_t, int, bool); \
  template bool launch_gs_rows<T, W>(const LevelDev<T>&, int, bool, int, cudaStream_t, int, bool);                       \
  template bool gs_rows_available<T, W>(const LevelDev<T>&);                                                             \
  template size_t gs_rows_smem<T, W>(const LevelDev<T>&);                                                                \
  template bool launch_gs_groups<T, W>(const LevelDev<T>&, int, bool, int, cudaStream_t, bool);                          \
  template void launch_residual<T, W>(const ColourRun*, int, const T*, int, const int*, const int*, const T*, const int*, \
                                      int, const T*, const T*, T*, int, cudaStream_t, bool);                             \
  template void launch_restrict<T, W>(const RestrictRun*, int, const int*, const int*, const T*, const int*, int,        \
                                      const T*, T*, T*, long long, int, cudaStream_t);                                   \
  template void launch_prolong_add<T, W>(const ProlongRun*, int, const T*, T*, int, cudaStream_t);                       \
  template void launch_boundary_solve<T, W>(const BoundaryDev<T>&, const T*, T*, int, cudaStream_t, bool);               \
  template void launch_coarse_solve<T, W>(int, const double*, const double*, const T*, T*, int, cudaStream_t);
GDTP_INSTANTIATE(float, 1)
GDTP_INSTANTIATE(float, 4)
GDTP_INSTANTIATE(double, 1)
GDTP_INSTANTIATE(double, 4)
template void launch_pack_rhs<float>(const double*, float*, long long, int, int, cudaStream_t);
template void launch_pack_rhs<double>(const double*, double*, long long, int, int, cudaStream_t);
template void launch_add_correction<float>(double*, float*, long long, int, int, cudaStream_t, const int*);
template void launch_add_correction<double>(double*, double*, long long, int, int, cudaStream_t, const int*);

}  // namespace dev
}  // namespace gdtp
