// Device kernels of the multigrid V-cycle on the atlas texel grid.
//
// Vectors use the reference's texel order (chart by chart, raster order) with
// KP values per texel (KP = 1, or a multiple of 4 holding up to KP right-hand
// sides).  A thread handles one texel and W consecutive channels (W = 1 or 4),
// so a warp reads contiguous memory for every stencil tap.
//
// Work is described by "runs": up to 32 texels of one raster line.  For the
// smoother a run holds texels of one colour (chart-local parity (i&1, j&1)),
// which are every other texel of the line; runs of one colour are independent,
// so one launch updates a whole colour (4-colour Gauss-Seidel on the 9-point
// stencil).  Stencil coefficients are stored per run texel as 10 planes
// (c0..c8 pre-divided by the diagonal, c4 = 1/diag, c9 = diag), the layout of
// the reference's reciprocal coefficients (UpdateCoefficients.inl:374-397)
// transposed so that each plane is read with unit stride.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gdtp {
namespace dev {

struct ColourRun {       // texels pos0 + 2m, m < len
  int pos0, prev0, next0, coef0, len;
};
// One raster line of deep texels (row smoother): texels pos + i, i < len, the
// rows above and below start at prev and next; coefficient index of its first
// even- / odd-column texel (its texels of one colour are consecutive in the
// colour-run planes); meta = first thread of the line in its block (bits 0-10)
// | first shared-memory slot (bits 11-23, slot of texel -1) | 1 << 24 when its
// first texel is in an odd column.
struct __align__(16) RowLine {
  int pos, prev, next, len;
  int cEven, cOdd, meta, pad;
};
struct RestrictRun {     // coarse texel out0 + m reads fine f0 + 2m and rows fp0/fn0 + 2m
  int out0, f0, fp0, fn0, len;
};
struct ProlongRun {      // fine texels f0 + m, m < len, line position i0 + m
  int f0, i0, len, center, prev, next, aligned;
};

template <typename T, int W>
struct Vec;
template <>
struct Vec<float, 1> {
  float v[1];
};
template <>
struct Vec<double, 1> {
  double v[1];
};
template <>
struct __align__(16) Vec<float, 4> {
  float v[4];
};
template <>
struct __align__(32) Vec<double, 4> {
  double v[4];
};

// Programmatic dependent launch.  Every V-cycle kernel starts with
// grid_dependency_wait(): it returns once the grids this launch depends on have
// completed and their writes are visible (immediately when the launch carries
// no programmatic dependency).  grid_launch_dependents() then lets the next
// kernel in the stream be scheduled while this one still runs, so its launch
// latency overlaps this kernel's tail; the next kernel in turn waits before it
// touches memory.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename T, int W>
__device__ __forceinline__ Vec<T, W> vload(const T* p) {
  return *reinterpret_cast<const Vec<T, W>*>(p);
}
template <typename T, int W>
__device__ __forceinline__ void vstore(T* p, const Vec<T, W>& v) {
  *reinterpret_cast<Vec<T, W>*>(p) = v;
}

}  // namespace dev
}  // namespace gdtp
