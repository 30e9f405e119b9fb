// Test-only CPU driver of the assembly element loops.  It runs the same
// per-element functions the assembly kernels run (kernels/assembly_math.h) in a
// plain host loop, so the FP64 element math and the host post-processing can be
// compared with the oracle on machines without a GPU.  Never linked into the
// product library.
//
// usage: assembly_check mesh.gdm out.gdd levels
#include <cstdio>
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../gradientdomaintextureprocessing_b200/csrc/kernels/assembly_math.h"
#include "../../gradientdomaintextureprocessing_b200/csrc/setup/setup.h"

using namespace gdtp;

static bool read_gdm(const char* path, Mesh& m, int& w, int& h) {
  FILE* f = fopen(path, "rb");
  if (!f) return false;
  char magic[8];
  int64_t hdr[5];
  if (fread(magic, 1, 8, f) != 8 || fread(hdr, 8, 5, f) != 5) { fclose(f); return false; }
  m.vertices.resize(hdr[0] * 3);
  m.triangles.resize(hdr[1] * 3);
  m.uv.resize(hdr[1] * 6);
  size_t ok = fread(m.vertices.data(), 8, m.vertices.size(), f) + fread(m.triangles.data(), 4, m.triangles.size(), f) +
              fread(m.uv.data(), 8, m.uv.size(), f);
  fclose(f);
  w = (int)hdr[2];
  h = (int)hdr[3];
  return ok == m.vertices.size() + m.triangles.size() + m.uv.size();
}

struct Out {
  FILE* f;
  explicit Out(const char* p) { f = fopen(p, "wb"); fwrite("GDTPDMP1", 1, 8, f); }
  ~Out() { fclose(f); }
  void put(const std::string& name, int code, int64_t n, int64_t cols, const void* d, size_t esz) {
    uint32_t l = (uint32_t)name.size();
    fwrite(&l, 4, 1, f);
    fwrite(name.data(), 1, l, f);
    uint8_t c = (uint8_t)code;
    fwrite(&c, 1, 1, f);
    uint32_t nd = cols > 1 ? 2 : 1;
    fwrite(&nd, 4, 1, f);
    int64_t dims[2] = {cols > 1 ? n / cols : n, cols};
    fwrite(dims, 8, nd, f);
    fwrite(d, esz, n, f);
  }
  void f64(const std::string& n, const std::vector<double>& v, int64_t cols = 1) { put(n, 2, v.size(), cols, v.data(), 8); }
  void i32(const std::string& n, const std::vector<int>& v) { put(n, 1, v.size(), 1, v.data(), 4); }
  void csr(const std::string& n, const Csr& m) { i32(n + "/ptr", m.ptr); i32(n + "/col", m.col); f64(n + "/val", m.val); }
};

int main(int argc, char** argv) {
  if (argc < 4) return 2;
  Mesh mesh;
  int W, H;
  if (!read_gdm(argv[1], mesh, W, H)) { fprintf(stderr, "bad mesh\n"); return 2; }
  Hierarchy h;
  if (!build_hierarchy(mesh, W, H, atoi(argv[3]), BlockInfo(), h)) { fprintf(stderr, "%s\n", h.error.c_str()); return 3; }
  BoundaryElements be;
  std::string err;
  if (!build_boundary_elements(h, be, err)) { fprintf(stderr, "%s\n", err.c_str()); return 3; }
  ChartMetrics g;
  embedding_metric(mesh, h.atlas, g);
  AssemblyWork w;
  build_assembly_work(h, be, g, w);
  std::vector<double> cm(16 * size_t(w.numInteriorCells)), cs(16 * size_t(w.numInteriorCells));
  for (int ic = 0; ic < w.numInteriorCells; ic++)
    am::interior_cell(ic, w.cellPtr.data(), w.cellTri.data(), w.cellIJ.data(), w.cellChart.data(), w.chartCellSize.data(),
                      w.triPos.data(), w.triMetricInv.data(), w.triScale.data(), &cm[16 * size_t(ic)], &cs[16 * size_t(ic)]);
  const int nd = h.levels[0].numDeep;
  FineSystem fs;
  fs.deepMass.resize(10 * size_t(nd));
  fs.deepStiffness.resize(10 * size_t(nd));
  for (int d = 0; d < nd; d++) {
    am::deep_gather(d, w.deepCells.data(), cm.data(), &fs.deepMass[10 * size_t(d)]);
    am::deep_gather(d, w.deepCells.data(), cs.data(), &fs.deepStiffness[10 * size_t(d)]);
  }
  std::vector<double> bm(36 * size_t(w.numBoundaryTriangles)), bs(36 * size_t(w.numBoundaryTriangles));
  for (int b = 0; b < w.numBoundaryTriangles; b++)
    am::boundary_triangle(b, w.btPtr.data(), w.btTri.data(), w.btPos.data(), w.triPos.data(), w.triMetric.data(),
                          w.triMetricInv.data(), &bm[36 * size_t(b)], &bs[36 * size_t(b)]);
  std::vector<double> am_(16 * w.boundaryAdjacentCells.size()), as_(16 * w.boundaryAdjacentCells.size());
  for (size_t a = 0; a < w.boundaryAdjacentCells.size(); a++)
    for (int q = 0; q < 16; q++) {
      am_[16 * a + q] = cm[16 * size_t(w.boundaryAdjacentCells[a]) + q];
      as_[16 * a + q] = cs[16 * size_t(w.boundaryAdjacentCells[a]) + q];
    }
  if (!assemble_boundary_blocks(h, be, w, am_, as_, bm, bs, fs, err)) { fprintf(stderr, "%s\n", err.c_str()); return 3; }
  Out out(argv[2]);
  // combined operator A = M + stiffness * S and its Galerkin hierarchy
  const double lam = argc > 4 ? atof(argv[4]) : 1e-3;
  std::vector<double> deepA(fs.deepMass.size());
  for (size_t i = 0; i < deepA.size(); i++) deepA[i] = fs.deepMass[i] + lam * fs.deepStiffness[i];
  Csr bbA = csr_axpby(1.0, fs.bbMass, lam, fs.bbStiffness), bdA = csr_axpby(1.0, fs.bdMass, lam, fs.bdStiffness);
  std::vector<LevelCoefficients> lc;
  if (!galerkin_hierarchy(h, 0, deepA, bbA, bdA, lc, err)) { fprintf(stderr, "%s\n", err.c_str()); return 3; }
  for (size_t l = 0; l < lc.size(); l++) {
    std::string p = "L" + std::to_string(l) + "/mine/";
    out.f64(p + "deep", lc[l].deep, 10);
    out.csr(p + "BB", lc[l].bb);
    out.csr(p + "BD", lc[l].bd);
  }
  // exact boundary solver: apply to r = BB * ones-ish vector and report the error
  for (size_t l = 0; l < lc.size(); l++) {
    BoundarySolverSetup bs;
    int maxBlock = argc > 5 ? atoi(argv[5]) : 384;
    int denseMax = argc > 6 ? atoi(argv[6]) : 0;
    if (!build_boundary_solver(lc[l].bb, lc[l].bd, maxBlock, denseMax, bs, err)) { fprintf(stderr, "bsolve: %s\n", err.c_str()); return 3; }
    const Csr& BB = lc[l].bb;
    std::vector<double> xt(bs.nb), r(bs.nb, 0.0), x(bs.nb, 0.0);
    for (int i = 0; i < bs.nb; i++) xt[i] = std::sin(0.37 * i) + 0.1 * std::cos(1.3 * i);
    for (int i = 0; i < bs.nb; i++)
      for (int k = BB.ptr[i]; k < BB.ptr[i + 1]; k++) r[i] += BB.val[k] * xt[BB.col[k]];
    // scaled solve
    std::vector<double> rh(bs.nb), y(bs.nI, 0.0), t(bs.nS), xs(bs.nS, 0.0), xh(bs.nb);
    for (int k = 0; k < bs.nb; k++) rh[k] = r[bs.order[k]] * bs.scale[k];
    for (int p = 0; p < bs.nSub; p++) {
      int b0 = bs.subPtr[p], m = bs.subPtr[p + 1] - b0;
      const double* Inv = &bs.inv[bs.invOff[p]];
      for (int a = 0; a < m; a++) { double s2 = 0; for (int q = 0; q < m; q++) s2 += Inv[size_t(a) * m + q] * rh[b0 + q]; y[b0 + a] = s2; }
    }
    for (int s2 = 0; s2 < bs.nS; s2++) {
      double v = rh[bs.nI + s2];
      for (int k = bs.ASI.ptr[s2]; k < bs.ASI.ptr[s2 + 1]; k++) v -= bs.ASI.val[k] * y[bs.ASI.col[k]];
      t[s2] = v;
    }
    for (int a = 0; a < bs.nS; a++) { double v = 0; for (int c = 0; c < bs.nS; c++) v += bs.Sinv[size_t(a) * bs.nS + c] * t[c]; xs[a] = v; }
    for (int p = 0; p < bs.nSub; p++) {
      int b0 = bs.subPtr[p], m = bs.subPtr[p + 1] - b0;
      std::vector<double> z(m, 0.0);
      for (int a = 0; a < m; a++)
        for (int k = bs.AIS.ptr[b0 + a]; k < bs.AIS.ptr[b0 + a + 1]; k++) z[a] += bs.AIS.val[k] * xs[bs.AIS.col[k]];
      const double* Inv = &bs.inv[bs.invOff[p]];
      for (int a = 0; a < m; a++) { double s2 = 0; for (int q = 0; q < m; q++) s2 += Inv[size_t(a) * m + q] * z[q]; xh[b0 + a] = y[b0 + a] - s2; }
    }
    for (int s2 = 0; s2 < bs.nS; s2++) xh[bs.nI + s2] = xs[s2];
    for (int k = 0; k < bs.nb; k++) x[bs.order[k]] = xh[k] * bs.scale[k];
    double emax = 0, xmax = 0, rres = 0, rn = 0;
    for (int i = 0; i < bs.nb; i++) { emax = std::max(emax, std::fabs(x[i] - xt[i])); xmax = std::max(xmax, std::fabs(xt[i])); }
    for (int i = 0; i < bs.nb; i++) {
      double v = r[i];
      for (int k = BB.ptr[i]; k < BB.ptr[i + 1]; k++) v -= BB.val[k] * x[BB.col[k]];
      rres += v * v; rn += r[i] * r[i];
    }
    fprintf(stderr, "level %zu boundary %d: %d subdomains, %d separator, rel residual %.2e, max err %.2e\n", l, bs.nb, bs.nSub, bs.nS,
            std::sqrt(rres / rn), emax / xmax);
  }
  out.f64("fine/deepMass", fs.deepMass, 10);
  out.f64("fine/deepStiffness", fs.deepStiffness, 10);
  out.csr("fine/BBmass", fs.bbMass);
  out.csr("fine/BBstiffness", fs.bbStiffness);
  out.csr("fine/BDmass", fs.bdMass);
  out.csr("fine/BDstiffness", fs.bdStiffness);
  {
    std::vector<int> bti;
    std::vector<double> btd;
    for (size_t c = 0; c < be.charts.size(); c++)
      for (size_t cell = 0; cell < be.charts[c].cellTriangles.size(); cell++)
        for (const BoundaryTriangle& t : be.charts[c].cellTriangles[cell]) {
          bti.insert(bti.end(), {(int)c, (int)cell, t.idx[0], t.idx[1], t.idx[2]});
          for (int k = 0; k < 3; k++) { btd.push_back(t.v[k].x); btd.push_back(t.v[k].y); }
        }
    out.put("fine/boundaryTriangles", 1, bti.size(), 5, bti.data(), 4);
    out.f64("fine/boundaryTrianglePos", btd, 6);
  }
  std::vector<int> info = {be.numBoundaryNodes, be.numMidPoints, be.numFineNodes, be.numFineBoundary, be.degenerateTriangulations};
  out.i32("fine/boundaryNodes", info);
  fprintf(stderr, "assembly_check: %d interior cells, %d boundary triangles, %d degenerate triangulations\n", w.numInteriorCells,
          w.numBoundaryTriangles, be.degenerateTriangulations);
  return 0;
}
// (appended) exact boundary solver check: BB x = r via the subdomain/Schur path, FP64
