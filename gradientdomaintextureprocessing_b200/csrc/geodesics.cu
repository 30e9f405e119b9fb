// Heat-method geodesics: sample construction (device, FP64 -> FP32) and the
// device pipeline.  See geodesics.h.
#include "geodesics.h"

#include <algorithm>

namespace gdtp {

bool GeodesicIntegrator::check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  err_ = std::string(what) + ": " + cudaGetErrorString(e);
  return false;
}

// counting-sort CSR of (row, entry) pairs given in the order the entries must keep
static void build_gather(int rows, const std::vector<std::pair<int, int>>& pairs, std::vector<int>& ptr, std::vector<int>& ent) {
  ptr.assign(rows + 1, 0);
  for (auto& p : pairs) ptr[p.first + 1]++;
  for (int r = 0; r < rows; r++) ptr[r + 1] += ptr[r];
  ent.resize(pairs.size());
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (auto& p : pairs) ent[fill[p.first]++] = p.second;
}

GeodesicIntegrator::GeodesicIntegrator(DeviceSystem& sys) : sys_(sys) {
  if (!sys.ok()) { err_ = sys.error(); return; }
  if (sys.metric().empty()) { err_ = "system not assembled"; return; }
  cudaSetDevice(sys.device());
  const Hierarchy& h = sys.hierarchy();
  const BoundaryElements& be = sys.boundary_elements();
  const GridLevel& L0 = h.levels[0];
  AssemblyWork w;
  build_assembly_work(h, be, sys.metric(), w);
  cudaStream_t s = sys.stream();

  // ---- samples (built on the device from the assembly's work lists)
  std::vector<int> slotCell(w.cellTri.size()), slotBt(w.btTri.size());
  for (int c = 0; c < w.numInteriorCells; c++)
    for (int e = w.cellPtr[c]; e < w.cellPtr[c + 1]; e++) slotCell[e] = c;
  for (int b = 0; b < w.numBoundaryTriangles; b++)
    for (int e = w.btPtr[b]; e < w.btPtr[b + 1]; e++) slotBt[e] = b;
  cellSlots = (int)slotCell.size();
  hexSlots = (int)slotBt.size();
  {
    DeviceArena tmp;
    const int* dSlotCell = tmp.upload(slotCell);
    const int* dCellTri = tmp.upload(w.cellTri);
    const int* dCellIJ = tmp.upload(w.cellIJ);
    const int* dCellChart = tmp.upload(w.cellChart);
    const double* dCell = tmp.upload(w.chartCellSize);
    const double* dTriPos = tmp.upload(w.triPos);
    const double* dTriMetric = tmp.upload(w.triMetric);
    const double* dTriInv = tmp.upload(w.triMetricInv);
    const double* dTriScale = tmp.upload(w.triScale);
    const int* dBtTri = tmp.upload(w.btTri);
    const double* dBtPos = tmp.upload(w.btPos);
    if (!check(tmp.last, "geodesic sample inputs")) return;
    float4* cellSamples = static_cast<float4*>(arena_.alloc(size_t(std::max(1, cellSlots)) * 4 * sizeof(float4)));
    double* hexSamples = static_cast<double*>(arena_.alloc(size_t(std::max(1, hexSlots)) * 20 * sizeof(double)));
    const int* dSlotBt = arena_.upload(slotBt);
    if (!check(arena_.last, "geodesic samples")) return;
    dev::launch_geo_cell_samples(cellSlots, dSlotCell, dCellTri, dCellIJ, dCellChart, dCell, dTriPos, dTriMetric, dTriInv, dTriScale,
                                 cellSamples, s);
    dev::launch_geo_hex_samples(hexSlots, dSlotBt, dBtTri, dBtPos, dTriPos, dTriMetric, hexSamples, s);
    if (!check(cudaGetLastError(), "geodesic sample kernels") || !check(cudaStreamSynchronize(s), "geodesic samples")) return;
    G_.cellSamples = cellSamples;
    G_.hexSamples = hexSamples;
    G_.slotBt = dSlotBt;
  }

  // ---- interior cells: corners and the texel gather
  std::vector<int> corners;
  for (const GridChart& gc : L0.charts) corners.insert(corners.end(), gc.interiorCellCorners.begin(), gc.interiorCellCorners.end());
  if ((int)corners.size() != 4 * w.numInteriorCells) { err_ = "interior cell corners do not match the cell lists"; return; }
  std::vector<std::pair<int, int>> tp;
  tp.reserve(corners.size());
  for (int c = 0; c < w.numInteriorCells; c++)
    for (int k = 0; k < 4; k++) tp.push_back({corners[4 * c + k], 4 * c + k});
  std::vector<int> tPtr, tEnt;
  build_gather(L0.numTexels, tp, tPtr, tEnt);

  // ---- boundary: fine nodes gather, prolongation / restriction, texel -> boundary
  const int nFine = be.prolongation.rows;
  std::vector<std::pair<int, int>> fp;
  for (int e = 0; e < hexSlots; e++)
    for (int k = 0; k < 6; k++) {
      const int f = w.btIdx[6 * slotBt[e] + k];
      if (f < 0 || f >= nFine) { err_ = "boundary element node without a fine boundary index"; return; }
      fp.push_back({f, 6 * e + k});
    }
  std::vector<int> fPtr, fEnt;
  build_gather(nFine, fp, fPtr, fEnt);
  const Csr& P = be.prolongation;
  const Csr R = csr_transpose(P);
  const std::vector<double>& pv = P.val;
  const std::vector<double>& rv = R.val;
  std::vector<int> texBoundary(L0.numTexels, -1);
  for (int b = 0; b < L0.numBoundary; b++) texBoundary[L0.boundaryGlobal[b]] = b;

  G_.n = L0.numTexels;
  G_.nCells = w.numInteriorCells;
  G_.nHex = hexSlots;
  G_.nFine = nFine;
  G_.invW = float(1.0 / L0.charts[0].cellSizeW);
  G_.invH = float(1.0 / L0.charts[0].cellSizeH);
  G_.cellPtr = arena_.upload(w.cellPtr);
  G_.corners = arena_.upload(corners);
  G_.btIdx = arena_.upload(w.btIdx);
  G_.pPtr = arena_.upload(P.ptr);
  G_.pCol = arena_.upload(P.col);
  G_.pVal = arena_.upload(pv);
  G_.bGlobal = arena_.upload(L0.boundaryGlobal);
  G_.fPtr = arena_.upload(fPtr);
  G_.fEnt = arena_.upload(fEnt);
  G_.tPtr = arena_.upload(tPtr);
  G_.tEnt = arena_.upload(tEnt);
  G_.texBoundary = arena_.upload(texBoundary);
  G_.rPtr = arena_.upload(R.ptr);
  G_.rCol = arena_.upload(R.col);
  G_.rVal = arena_.upload(rv);
  check(arena_.last, "geodesic gather lists");
}

bool GeodesicIntegrator::download(const std::string& name, std::vector<double>& out) {
  if (!err_.empty()) return false;
  cudaSetDevice(sys_.device());
  auto fetch_f = [&](const void* p, size_t n) {
    std::vector<float> t(n);
    if (!check(cudaMemcpy(t.data(), p, n * sizeof(float), cudaMemcpyDeviceToHost), "download")) return false;
    out.assign(t.begin(), t.end());
    return true;
  };
  auto fetch_i = [&](const int* p, size_t n) {
    std::vector<int> t(n);
    if (!check(cudaMemcpy(t.data(), p, n * sizeof(int), cudaMemcpyDeviceToHost), "download")) return false;
    out.assign(t.begin(), t.end());
    return true;
  };
  if (name == "cellSamples") return fetch_f(G_.cellSamples, size_t(cellSlots) * 16);
  if (name == "hexSamples") {
    out.resize(size_t(hexSlots) * 20);
    return check(cudaMemcpy(out.data(), G_.hexSamples, out.size() * sizeof(double), cudaMemcpyDeviceToHost), "download");
  }
  if (name == "cellPtr") return fetch_i(G_.cellPtr, size_t(G_.nCells) + 1);
  if (name == "corners") return fetch_i(G_.corners, size_t(G_.nCells) * 4);
  if (name == "slotBt") return fetch_i(G_.slotBt, size_t(hexSlots));
  if (name == "btIdx") {
    int nb = 0;
    std::vector<int> sb(hexSlots);
    if (hexSlots && !check(cudaMemcpy(sb.data(), G_.slotBt, hexSlots * sizeof(int), cudaMemcpyDeviceToHost), "download")) return false;
    for (int b : sb) nb = std::max(nb, b + 1);
    return fetch_i(G_.btIdx, size_t(nb) * 6);
  }
  err_ = "unknown array " + name;
  return false;
}

// buffer capacity for k right-hand sides: the next power of two (at most 64)
static int k_capacity(int k) {
  int c = 1;
  while (c < k) c *= 2;
  return std::min(c, 64);
}

bool GeodesicIntegrator::ensure_k(int kk) {
  if (kk <= G_.kMax) return true;
  const int k = k_capacity(kk);
  work_ = DeviceArena();
  G_.fineU = static_cast<double*>(work_.alloc(size_t(std::max(1, G_.nFine)) * k * sizeof(double)));
  G_.fineRhs = static_cast<double*>(work_.alloc(size_t(std::max(1, G_.nFine)) * k * sizeof(double)));
  G_.cellOut = static_cast<float*>(work_.alloc(size_t(std::max(1, G_.nCells)) * 4 * k * sizeof(float)));
  G_.hexOut = static_cast<double*>(work_.alloc(size_t(std::max(1, G_.nHex)) * 6 * k * sizeof(double)));
  if (!check(work_.last, "geodesic work")) return false;
  G_.kMax = k;
  return true;
}

bool GeodesicIntegrator::rhs_device(const double* u, double* rhs, int k, cudaStream_t s) {
  if (!err_.empty()) return false;
  if (k < 1 || k > 64) { err_ = "k must be in [1, 64]"; return false; }
  cudaSetDevice(sys_.device());
  if (!ensure_k(k)) return false;
  dev::launch_geo_rhs(G_, u, rhs, k, s);
  return check(cudaGetLastError(), "geodesic rhs");
}

bool GeodesicIntegrator::rhs_host(const double* u, double* rhs, int k) {
  if (!err_.empty()) return false;
  cudaSetDevice(sys_.device());
  DeviceArena a;
  const size_t bytes = size_t(G_.n) * k * sizeof(double);
  double* du = static_cast<double*>(a.alloc(bytes));
  double* dr = static_cast<double*>(a.alloc(bytes));
  cudaStream_t s = sys_.stream();
  return check(a.last, "geodesic rhs buffers") && check(cudaMemcpyAsync(du, u, bytes, cudaMemcpyHostToDevice, s), "h2d u") &&
         rhs_device(du, dr, k, s) && check(cudaMemcpyAsync(rhs, dr, bytes, cudaMemcpyDeviceToHost, s), "d2h rhs") &&
         check(cudaStreamSynchronize(s), "geodesic rhs");
}

bool GeodesicIntegrator::distance(DeviceSystem& smooth, DeviceSystem& dist, const int* sources, int k, double tol, int maxIters,
                                  double* d_host, SolveReport& smoothRep, SolveReport& distRep) {
  if (!err_.empty()) return false;
  if (k < 1 || k > 64) { err_ = "k must be in [1, 64]"; return false; }
  for (int c = 0; c < k; c++)
    if (sources[c] < 0 || sources[c] >= G_.n) { err_ = "source texel out of range"; return false; }
  cudaSetDevice(sys_.device());
  cudaStream_t s = sys_.stream();
  // the buffers only grow (to a power of two): varying batch sizes keep them,
  // and with them the solves' captured graphs
  if (k > dK_) {
    const int kc = k_capacity(k);
    const size_t nk = size_t(G_.n) * kc;
    dwork_ = DeviceArena();
    b_ = static_cast<double*>(dwork_.alloc(nk * sizeof(double)));
    u_ = static_cast<double*>(dwork_.alloc(nk * sizeof(double)));
    r_ = static_cast<double*>(dwork_.alloc(nk * sizeof(double)));
    d_ = static_cast<double*>(dwork_.alloc(nk * sizeof(double)));
    sv_ = static_cast<double*>(dwork_.alloc(kc * sizeof(double)));
    src_ = static_cast<int*>(dwork_.alloc(kc * sizeof(int)));
    if (!check(dwork_.last, "geodesic buffers")) { dK_ = 0; return false; }
    dK_ = kc;
  }
  const size_t nk = size_t(G_.n) * k;
  double *b = b_, *u = u_, *r = r_, *d = d_, *sv = sv_;
  int* src = src_;
  if (!check(cudaMemcpyAsync(src, sources, k * sizeof(int), cudaMemcpyHostToDevice, s), "h2d sources")) return false;
  dev::launch_geo_impulses((long long)G_.n, k, src, b, s);
  if (!smooth.solve_mixed(nullptr, nullptr, b, u, k, tol, maxIters, s, smoothRep, true)) { err_ = smooth.error(); return false; }
  if (!rhs_device(u, r, k, s)) return false;
  if (!dist.solve_mixed(nullptr, nullptr, r, d, k, tol, maxIters, s, distRep, true)) { err_ = dist.error(); return false; }
  dev::launch_geo_shift((long long)G_.n, k, src, d, sv, s);
  return check(cudaGetLastError(), "geodesic shift") && check(cudaMemcpyAsync(d_host, d, nk * sizeof(double), cudaMemcpyDeviceToHost, s), "d2h distance") &&
         check(cudaStreamSynchronize(s), "geodesic distance");
}

}  // namespace gdtp
