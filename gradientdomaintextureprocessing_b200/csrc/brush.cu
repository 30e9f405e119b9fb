// The sharpening brush of the filtering app on the device: the right-hand side
// M f + lambda sum_cells m_c S_c f of a per-cell stiffness mask m
// (TextureFiltering.cpp:562-570).  Restates CellStiffnessToTexelStiffness
// (IterativeSolvers.inl:1170-1208) over the per-cell stiffness contributions
// that InitializeMassAndStiffness computes with computeCellBasedStiffness
// (MassAndStiffness.h:304-333, 375-383, 542-546):
//   * deep texel d, its four surrounding cells q (previous cell row i, i+1,
//     next row i, i+1): coefficient (S_q f)[d], the row of cell q's 4x4
//     stiffness at d's corner applied to the signal at the cell's corners;
//   * boundary texels: the fine boundary nodes' rows of the same products
//     (interior cells touching a boundary texel with the texel signal, boundary
//     quadratic elements with the fine boundary signal P f_B), restricted to
//     the boundary texels by P^T, per channel a boundary x cells matrix.
// A stroke is then out = C m: four products per deep texel (in the reference's
// order) and one sparse row per boundary texel.  Set-up: element matrices from
// the assembly kernels, deep coefficients on the device (FP64), boundary
// matrices on the host.
#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "capi_internal.h"
#include "kernels/vcycle_kernels.h"
#include "system.h"

namespace gdtp {
namespace {

// deep texel d, slot q: the cell's corner slot of d (corners 0 (i,j), 1 (i+1,j),
// 2 (i+1,j+1), 3 (i,j+1)) is {2, 3, 1, 0}[q]
__global__ void k_brush_deep_coef(int nDeep, int k, const int* __restrict__ deepCells, const double* __restrict__ cellStiff,
                                  const int* __restrict__ cellCorners, const double* __restrict__ f, double* __restrict__ coef) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 4ll * nDeep) return;
  const int q = int(t & 3);
  const int corner = q == 0 ? 2 : q == 1 ? 3 : q == 2 ? 1 : 0;
  const int ic = deepCells[t];
  const double* S = cellStiff + 16 * (long long)ic + 4 * corner;
  for (int c = 0; c < k; c++) {
    double s = 0.0;
    for (int l = 0; l < 4; l++) s += S[l] * f[(long long)cellCorners[4 * (long long)ic + l] * k + c];
    coef[t * k + c] = s;
  }
}

// out[texel] = c0 m[prev i] + c1 m[prev i+1] + c2 m[next i] + c3 m[next i+1]
__global__ void k_brush_deep_apply(int nDeep, int k, const int* __restrict__ deepGlobal, const int4* __restrict__ cells,
                                   const double* __restrict__ coef, const double* __restrict__ mask, double* __restrict__ out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nDeep * k) return;
  const long long d = t / k;
  const int c = int(t - d * k);
  const int4 cl = cells[d];
  const double* a = coef + 4 * d * k + c;
  out[(long long)deepGlobal[d] * k + c] = a[0] * mask[cl.x] + a[k] * mask[cl.y] + a[2 * k] * mask[cl.z] + a[3 * k] * mask[cl.w];
}

// out[boundary texel] = row of channel c's boundary x cells matrix times m
__global__ void k_brush_boundary_apply(int nB, int k, int c, const int* __restrict__ bGlobal, const int* __restrict__ ptr,
                                       const int* __restrict__ col, const double* __restrict__ val, const double* __restrict__ mask,
                                       double* __restrict__ out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nB) return;
  double s = 0.0;
  for (int e = ptr[b]; e < ptr[b + 1]; e++) s += val[e] * mask[col[e]];
  out[(long long)bGlobal[b] * k + c] = s;
}

}  // namespace
}  // namespace gdtp

using namespace gdtp;

struct gdtp_brush {
  const DeviceSystem* sys = nullptr;
  int k = 0, nDeep = 0, nB = 0, nCells = 0, n = 0;
  DeviceArena arena;
  const int* deepGlobal = nullptr;
  const int4* deepCells = nullptr;  // global cell indices of the four cells
  double* coef = nullptr;
  const int* bGlobal = nullptr;
  const int* bPtr[4] = {nullptr, nullptr, nullptr, nullptr};
  const int* bCol[4] = {nullptr, nullptr, nullptr, nullptr};
  const double* bVal[4] = {nullptr, nullptr, nullptr, nullptr};
  double *maskDev = nullptr, *outDev = nullptr;  // host-API staging
};

extern "C" __attribute__((visibility("hidden"))) int gdtp_system_device_view(const gdtp_system* s, const void** sys);

static bool cuda_ok(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  fail(GDTP_ERR_CUDA, std::string("gdtp_brush: ") + what + ": " + cudaGetErrorString(e));
  return false;
}

extern "C" int gdtp_brush_create(gdtp_system* s, const double* signal, int k, gdtp_brush** out) {
  return guarded("gdtp_brush_create", [&]() -> int {
    if (!out) return fail(GDTP_ERR_INVALID, "gdtp_brush_create: null output");
    *out = nullptr;
    const void* view = nullptr;
    if (gdtp_system_device_view(s, &view) != GDTP_OK || !view) return fail(GDTP_ERR_INVALID, "gdtp_brush_create: null system");
    if (!signal || k < 1 || k > 4) return fail(GDTP_ERR_INVALID, "gdtp_brush_create: signal must be numTexels x k, 1 <= k <= 4");
    const DeviceSystem& sys = *static_cast<const DeviceSystem*>(view);
    const Hierarchy& h = sys.hierarchy();
    const BoundaryElements& be = sys.boundary_elements();
    const GridLevel& L = h.levels[0];
    if (cudaSetDevice(sys.device()) != cudaSuccess) return fail(GDTP_ERR_CUDA, "gdtp_brush_create: no usable device");
    std::unique_ptr<gdtp_brush> b(new gdtp_brush());
    b->sys = &sys;
    b->k = k;
    b->n = L.numTexels;
    b->nDeep = L.numDeep;
    b->nB = L.numBoundary;
    b->nCells = L.numCells;
    // element matrices of the assembly (same metric as the system)
    AssemblyWork w;
    build_assembly_work(h, be, sys.metric(), w);
    std::vector<int> cellBase(L.charts.size() + 1, 0);
    for (size_t c = 0; c < L.charts.size(); c++) cellBase[c + 1] = cellBase[c] + L.charts[c].numInteriorCells;
    // per interior cell: its four corner texels and its global cell index
    std::vector<int> corners(4 * size_t(w.numInteriorCells)), icGlobal(w.numInteriorCells);
    for (int ic = 0; ic < w.numInteriorCells; ic++) {
      const GridChart& gc = L.charts[w.cellChart[ic]];
      const int i = w.cellIJ[2 * ic], j = w.cellIJ[2 * ic + 1];
      const int pos[4] = {gc.at(i, j), gc.at(i + 1, j), gc.at(i + 1, j + 1), gc.at(i, j + 1)};
      for (int q = 0; q < 4; q++) corners[4 * size_t(ic) + q] = gc.texel[pos[q]];
      icGlobal[ic] = gc.cellOffset + gc.localCell[gc.cat(i, j)];
    }
    std::vector<int4> deepCellsGlobal(b->nDeep);
    std::vector<int> deepGlobal(L.deepGlobal.begin(), L.deepGlobal.end());
    for (int d = 0; d < b->nDeep; d++) {
      const int* q = &w.deepCells[4 * size_t(d)];
      deepCellsGlobal[d] = make_int4(icGlobal[q[0]], icGlobal[q[1]], icGlobal[q[2]], icGlobal[q[3]]);
    }
    DeviceArena tmp;
    DeviceArena& A = b->arena;
    const double* fDev = tmp.upload(std::vector<double>(signal, signal + size_t(b->n) * k));
    double* cs = tmp.zeros<double>(16 * size_t(w.numInteriorCells));
    double* cm = tmp.zeros<double>(16 * size_t(w.numInteriorCells));
    double* bm = tmp.zeros<double>(36 * size_t(w.numBoundaryTriangles));
    double* bs = tmp.zeros<double>(36 * size_t(w.numBoundaryTriangles));
    const int* deepCells = tmp.upload(w.deepCells);
    const int* cornersDev = tmp.upload(corners);
    if (!cuda_ok(tmp.last, "upload")) return GDTP_ERR_CUDA;
    cudaStream_t st = sys.stream();
    dev::launch_interior_cells(w.numInteriorCells, tmp.upload(w.cellPtr), tmp.upload(w.cellTri), tmp.upload(w.cellIJ),
                               tmp.upload(w.cellChart), tmp.upload(w.chartCellSize), tmp.upload(w.triPos), tmp.upload(w.triMetricInv),
                               tmp.upload(w.triScale), cm, cs, st);
    dev::launch_boundary_triangles(w.numBoundaryTriangles, tmp.upload(w.btPtr), tmp.upload(w.btTri), tmp.upload(w.btPos),
                                   tmp.upload(w.triPos), tmp.upload(w.triMetric), tmp.upload(w.triMetricInv), bm, bs, st);
    b->coef = static_cast<double*>(A.alloc(4 * size_t(b->nDeep) * k * sizeof(double)));
    if (!cuda_ok(tmp.last, "upload") || !cuda_ok(A.last, "alloc")) return GDTP_ERR_CUDA;
    if (b->nDeep > 0)
      k_brush_deep_coef<<<int((4ll * b->nDeep + 255) / 256), 256, 0, st>>>(b->nDeep, k, deepCells, cs, cornersDev, fDev, b->coef);
    // boundary rows on the host from the element matrices
    std::vector<double> hcs(16 * size_t(w.numInteriorCells)), hbs(36 * size_t(w.numBoundaryTriangles));
    if (!cuda_ok(cudaGetLastError(), "kernels") ||
        !cuda_ok(cudaMemcpyAsync(hcs.data(), cs, hcs.size() * 8, cudaMemcpyDeviceToHost, st), "d2h") ||
        !cuda_ok(cudaMemcpyAsync(hbs.data(), bs, hbs.size() * 8, cudaMemcpyDeviceToHost, st), "d2h") ||
        !cuda_ok(cudaStreamSynchronize(st), "set-up"))
      return GDTP_ERR_CUDA;
    // fine boundary signal: the boundary texels' signal prolonged to the fine boundary nodes
    std::vector<double> fB(size_t(b->nB) * k), fFine(size_t(be.numFineBoundary) * k, 0.0);
    for (int i = 0; i < b->nB; i++)
      for (int c = 0; c < k; c++) fB[size_t(i) * k + c] = signal[size_t(L.boundaryGlobal[i]) * k + c];
    const Csr& P = be.prolongation;
    for (int r = 0; r < P.rows; r++)
      for (int e = P.ptr[r]; e < P.ptr[r + 1]; e++)
        for (int c = 0; c < k; c++) fFine[size_t(r) * k + c] += P.val[e] * fB[size_t(P.col[e]) * k + c];
    std::vector<std::vector<Triplet>> trip(k);
    for (int ic = 0; ic < w.numInteriorCells; ic++) {
      const GridChart& gc = L.charts[w.cellChart[ic]];
      const int i = w.cellIJ[2 * ic], j = w.cellIJ[2 * ic + 1];
      const int pos[4] = {gc.at(i, j), gc.at(i + 1, j), gc.at(i + 1, j + 1), gc.at(i, j + 1)};
      for (int q = 0; q < 4; q++) {
        const int node = gc.texel[pos[q]];
        if (L.boundaryAndDeep[node] < 0) continue;  // deep rows: the device coefficients
        const int fk = be.fineBoundaryIndex[gc.interiorTexel[pos[q]]];
        if (fk < 0) return fail(GDTP_ERR_SETUP, "gdtp_brush_create: interior cell corner without a fine boundary node");
        const double* S = &hcs[16 * size_t(ic) + 4 * q];
        for (int c = 0; c < k; c++) {
          double v = 0.0;
          for (int l = 0; l < 4; l++) v += S[l] * signal[size_t(corners[4 * size_t(ic) + l]) * k + c];
          trip[c].push_back({fk, icGlobal[ic], v});
        }
      }
    }
    int bt = 0;
    for (size_t ch = 0; ch < L.charts.size(); ch++) {
      const GridChart& gc = L.charts[ch];
      for (size_t cell = 0; cell < be.charts[ch].cellTriangles.size(); cell++) {
        const int globalCell = gc.cellOffset + gc.boundaryCellToCell[cell];
        for (size_t t = 0; t < be.charts[ch].cellTriangles[cell].size(); t++, bt++) {
          const int* fi = &w.btIdx[6 * size_t(bt)];
          const double* S = &hbs[36 * size_t(bt)];
          for (int q = 0; q < 6; q++)
            for (int c = 0; c < k; c++) {
              double v = 0.0;
              for (int l = 0; l < 6; l++) v += S[6 * l + q] * fFine[size_t(fi[l]) * k + c];
              trip[c].push_back({fi[q], globalCell, v});
            }
        }
      }
    }
    const Csr R = csr_transpose(P);
    b->bGlobal = A.upload(L.boundaryGlobal);
    for (int c = 0; c < k; c++) {
      const Csr fine = csr_from_triplets(be.numFineBoundary, b->nCells, trip[c]);
      const Csr coarse = csr_multiply(R, fine);
      b->bPtr[c] = A.upload(coarse.ptr);
      b->bCol[c] = A.upload(coarse.col);
      b->bVal[c] = A.upload(coarse.val);
    }
    b->deepGlobal = A.upload(deepGlobal);
    b->deepCells = A.upload(deepCellsGlobal);
    b->maskDev = static_cast<double*>(A.alloc(size_t(std::max(1, b->nCells)) * sizeof(double)));
    b->outDev = static_cast<double*>(A.alloc(size_t(b->n) * k * sizeof(double)));
    if (!cuda_ok(A.last, "upload")) return GDTP_ERR_CUDA;
    *out = b.release();
    return GDTP_OK;
  });
}

extern "C" void gdtp_brush_free(gdtp_brush* b) { delete b; }

extern "C" int gdtp_brush_apply_device(gdtp_brush* b, const double* mask_dev, double* out_dev, void* stream) {
  return guarded("gdtp_brush_apply_device", [&]() -> int {
    if (!b || !mask_dev || !out_dev) return fail(GDTP_ERR_INVALID, "gdtp_brush_apply_device: null argument");
    if (cudaSetDevice(b->sys->device()) != cudaSuccess) return fail(GDTP_ERR_CUDA, "gdtp_brush_apply_device: no usable device");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int k = b->k;
    if (b->nDeep > 0)
      k_brush_deep_apply<<<int(((long long)b->nDeep * k + 255) / 256), 256, 0, st>>>(b->nDeep, k, b->deepGlobal, b->deepCells, b->coef,
                                                                                      mask_dev, out_dev);
    for (int c = 0; c < k && b->nB > 0; c++)
      k_brush_boundary_apply<<<(b->nB + 255) / 256, 256, 0, st>>>(b->nB, k, c, b->bGlobal, b->bPtr[c], b->bCol[c], b->bVal[c], mask_dev,
                                                                  out_dev);
    return cuda_ok(cudaGetLastError(), "apply") ? GDTP_OK : GDTP_ERR_CUDA;
  });
}

extern "C" int gdtp_brush_apply(gdtp_brush* b, const double* cell_mask, double* out) {
  return guarded("gdtp_brush_apply", [&]() -> int {
    if (!b || !cell_mask || !out) return fail(GDTP_ERR_INVALID, "gdtp_brush_apply: null argument");
    if (cudaSetDevice(b->sys->device()) != cudaSuccess) return fail(GDTP_ERR_CUDA, "gdtp_brush_apply: no usable device");
    cudaStream_t st = b->sys->stream();
    if (!cuda_ok(cudaMemcpyAsync(b->maskDev, cell_mask, size_t(b->nCells) * sizeof(double), cudaMemcpyHostToDevice, st), "h2d"))
      return GDTP_ERR_CUDA;
    const int code = gdtp_brush_apply_device(b, b->maskDev, b->outDev, st);
    if (code != GDTP_OK) return code;
    if (!cuda_ok(cudaMemcpyAsync(out, b->outDev, size_t(b->n) * b->k * sizeof(double), cudaMemcpyDeviceToHost, st), "d2h") ||
        !cuda_ok(cudaStreamSynchronize(st), "apply"))
      return GDTP_ERR_CUDA;
    return GDTP_OK;
  });
}
