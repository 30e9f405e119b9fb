// Device data and launchers of the heat-method geodesic integration
// (geodesic_kernels.cu).
#pragma once
#include <cuda_runtime.h>

namespace gdtp {
namespace dev {

// Samples and gather lists on the device (built by GeodesicIntegrator).
struct GeoDev {
  int n = 0;                    // texels of the finest level
  int nCells = 0, nHex = 0, nFine = 0;
  float invW = 0, invH = 0;     // 1 / cell size of the finest level
  const int* cellPtr = nullptr;            // interior cell -> sample slots
  const int* corners = nullptr;            // 4 texels per interior cell: (i,j) (i+1,j) (i+1,j+1) (i,j+1)
  const float4* cellSamples = nullptr;     // 4 float4 per slot
  const int* slotBt = nullptr;             // boundary sample slot -> boundary element
  const int* btIdx = nullptr;              // 6 fine boundary nodes per element
  const double* hexSamples = nullptr;      // 20 doubles per slot
  const int *pPtr = nullptr, *pCol = nullptr;  // fine boundary node x coarse boundary texel prolongation
  const double* pVal = nullptr;
  const int* bGlobal = nullptr;            // boundary index -> texel
  const int *fPtr = nullptr, *fEnt = nullptr;  // fine node -> (slot * 6 + k) contributions
  const int *tPtr = nullptr, *tEnt = nullptr;  // texel -> (cell * 4 + k) contributions
  const int* texBoundary = nullptr;        // texel -> boundary index or -1
  const int *rPtr = nullptr, *rCol = nullptr;  // restriction = prolongation transposed
  const double* rVal = nullptr;
  double *fineU = nullptr, *fineRhs = nullptr, *hexOut = nullptr;  // work (boundary in FP64), sized for kMax channels
  float* cellOut = nullptr;
  int kMax = 0;
};

void launch_geo_cell_samples(int nSlots, const int* slotCell, const int* cellTri, const int* cellIJ, const int* cellChart,
                             const double* chartCellSize, const double* triPos, const double* triMetric, const double* triMetricInv,
                             const double* triScale, float4* out, cudaStream_t s);
void launch_geo_hex_samples(int nSlots, const int* slotBt, const int* btTri, const double* btPos, const double* triPos,
                            const double* triMetric, double* out, cudaStream_t s);
// rhs (n x K, FP64) of the potential u (n x K, FP64); K <= G.kMax
void launch_geo_rhs(const GeoDev& G, const double* u, double* rhs, int K, cudaStream_t s);
// b (n x K) = delta at sources[c] in column c
void launch_geo_impulses(long long n, int K, const int* sources, double* b, cudaStream_t s);
// d[:, c] -= d[sources[c], c]  (sourceValues: K doubles of scratch)
void launch_geo_shift(long long n, int K, const int* sources, double* d, double* sourceValues, cudaStream_t s);

}  // namespace dev
}  // namespace gdtp
