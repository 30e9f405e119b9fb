// FP64 assembly kernels: one thread per interior cell / boundary triangle /
// deep texel, each running the shared element routines of assembly_math.h in
// the reference's accumulation order (MassAndStiffness.h:31-346), so results are
// deterministic and independent of the launch shape.
#include "assembly_math.h"
#include "vcycle_kernels.h"

namespace gdtp {
namespace dev {

__global__ void __launch_bounds__(128) k_interior_cells(int n, const int* __restrict__ cellPtr, const int* __restrict__ cellTri,
                                                        const int* __restrict__ cellIJ, const int* __restrict__ cellChart,
                                                        const double* __restrict__ chartCellSize, const double* __restrict__ triPos,
                                                        const double* __restrict__ triMetricInv, const double* __restrict__ triScale,
                                                        double* __restrict__ mass, double* __restrict__ stiff) {
  const int ic = blockIdx.x * blockDim.x + threadIdx.x;
  if (ic >= n) return;
  double m[16], s[16];
  am::interior_cell(ic, cellPtr, cellTri, cellIJ, cellChart, chartCellSize, triPos, triMetricInv, triScale, m, s);
#pragma unroll
  for (int q = 0; q < 16; q++) {
    mass[16 * (long long)ic + q] = m[q];
    stiff[16 * (long long)ic + q] = s[q];
  }
}

__global__ void __launch_bounds__(256) k_deep_gather(int nDeep, const int* __restrict__ deepCells, const double* __restrict__ cellMass,
                                                     const double* __restrict__ cellStiff, double* __restrict__ deepMass,
                                                     double* __restrict__ deepStiff) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= nDeep) return;
  double m[10], s[10];
  am::deep_gather(d, deepCells, cellMass, m);
  am::deep_gather(d, deepCells, cellStiff, s);
#pragma unroll
  for (int q = 0; q < 10; q++) {
    deepMass[10 * (long long)d + q] = m[q];
    deepStiff[10 * (long long)d + q] = s[q];
  }
}

__global__ void __launch_bounds__(64) k_boundary_triangles(int n, const int* __restrict__ btPtr, const int* __restrict__ btTri,
                                                           const double* __restrict__ btPos, const double* __restrict__ triPos,
                                                           const double* __restrict__ triMetric, const double* __restrict__ triMetricInv,
                                                           double* __restrict__ mass, double* __restrict__ stiff) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  double m[36], s[36];
  am::boundary_triangle(b, btPtr, btTri, btPos, triPos, triMetric, triMetricInv, m, s);
  for (int q = 0; q < 36; q++) {
    mass[36 * (long long)b + q] = m[q];
    stiff[36 * (long long)b + q] = s[q];
  }
}

__global__ void k_gather_cells(int n, const int* __restrict__ idx, const double* __restrict__ src, double* __restrict__ dst) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * 16) return;
  const long long c = t / 16;
  dst[t] = src[(long long)idx[c] * 16 + (t - c * 16)];
}

void launch_interior_cells(int n, const int* cellPtr, const int* cellTri, const int* cellIJ, const int* cellChart,
                           const double* chartCellSize, const double* triPos, const double* triMetricInv, const double* triScale,
                           double* mass, double* stiff, cudaStream_t s) {
  if (n <= 0) return;
  k_interior_cells<<<(n + 127) / 128, 128, 0, s>>>(n, cellPtr, cellTri, cellIJ, cellChart, chartCellSize, triPos, triMetricInv,
                                                   triScale, mass, stiff);
}
void launch_deep_gather(int nDeep, const int* deepCells, const double* cellMass, const double* cellStiff, double* deepMass,
                        double* deepStiff, cudaStream_t s) {
  if (nDeep <= 0) return;
  k_deep_gather<<<(nDeep + 255) / 256, 256, 0, s>>>(nDeep, deepCells, cellMass, cellStiff, deepMass, deepStiff);
}
void launch_boundary_triangles(int n, const int* btPtr, const int* btTri, const double* btPos, const double* triPos,
                               const double* triMetric, const double* triMetricInv, double* mass, double* stiff, cudaStream_t s) {
  if (n <= 0) return;
  k_boundary_triangles<<<(n + 63) / 64, 64, 0, s>>>(n, btPtr, btTri, btPos, triPos, triMetric, triMetricInv, mass, stiff);
}
void launch_gather_cells(int n, const int* idx, const double* src, double* dst, cudaStream_t s) {
  if (n <= 0) return;
  k_gather_cells<<<int(((long long)n * 16 + 255) / 256), 256, 0, s>>>(n, idx, src, dst);
}

}  // namespace dev
}  // namespace gdtp
