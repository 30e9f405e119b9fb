// Host side of the FP64 assembly: parameter metric, device work lists, and the
// sparse boundary blocks built from element matrices computed on the device.
//
//   embedding metric                 Src/Metric.inl:248-276
//   parameter metric g = J^-T G J^-1 Src/Metric.inl:415-446
//   interior / boundary cell loops   Src/MassAndStiffness.h:31-284
//   deep coefficient scatter         Src/MassAndStiffness.h:287-346
//   boundary triplets and P^T B P    Src/MassAndStiffness.h:348-405, 490-549
#include <cmath>

#include "setup.h"

namespace gdtp {

bool embedding_metric(const Mesh& mesh, const Atlas& A, ChartMetrics& out) {
  std::vector<M2> G, P;
  if (!surface_metric(mesh, 0, true, G) || !parameter_metric(mesh, G, P)) return false;
  out.assign(A.charts.size(), {});
  for (size_t c = 0; c < A.charts.size(); c++) {
    const AtlasChart& ac = A.charts[c];
    out[c].resize(ac.meshTriangleIndices.size());
    for (size_t k = 0; k < ac.meshTriangleIndices.size(); k++) out[c][k] = P[ac.meshTriangleIndices[k]];
  }
  return true;
}

static void bbox_cells(const V2* p, double cw, double ch, int mn[2], int mx[2]) {
  double fminx = std::max(std::min(std::min(p[0].x, p[1].x), p[2].x), 0.0);
  double fminy = std::max(std::min(std::min(p[0].y, p[1].y), p[2].y), 0.0);
  double fmaxx = std::min(std::max(std::max(p[0].x, p[1].x), p[2].x), 1.0);
  double fmaxy = std::min(std::max(std::max(p[0].y, p[1].y), p[2].y), 1.0);
  double iw = 1.0 / cw, ih = 1.0 / ch;
  mn[0] = int(std::floor(fminx * iw)); mn[1] = int(std::floor(fminy * ih));
  mx[0] = int(std::ceil(fmaxx * iw)); mx[1] = int(std::ceil(fmaxy * ih));
}

void build_assembly_work(const Hierarchy& h, const BoundaryElements& be, const ChartMetrics& g, AssemblyWork& w) {
  const GridLevel& L = h.levels[0];
  const Atlas& A = h.atlas;
  w = AssemblyWork();
  // triangle table (chart-major) with grid-corner-relative positions and metric
  std::vector<int> triBase(A.charts.size() + 1, 0);
  for (size_t c = 0; c < A.charts.size(); c++) triBase[c + 1] = triBase[c] + (int)A.charts[c].triangles.size();
  w.numTriangles = triBase.back();
  w.triPos.resize(6 * size_t(w.numTriangles));
  w.triMetric.resize(4 * size_t(w.numTriangles));
  w.triMetricInv.resize(4 * size_t(w.numTriangles));
  w.triScale.resize(w.numTriangles);
  const int nCharts = (int)A.charts.size();
#pragma omp parallel for schedule(dynamic, 1)
  for (int c = 0; c < nCharts; c++) {
    const AtlasChart& ac = A.charts[c];
    const GridChart& gc = L.charts[c];
    for (size_t t = 0; t < ac.triangles.size(); t++) {
      size_t e = triBase[c] + t;
      for (int k = 0; k < 3; k++) {
        V2 p = ac.vertices[ac.triangles[t][k]] - gc.corner;
        w.triPos[6 * e + 2 * k] = p.x;
        w.triPos[6 * e + 2 * k + 1] = p.y;
      }
      const M2& m = g[c][t];
      M2 mi = m.inverse();
      double gm[4] = {m.c[0][0], m.c[0][1], m.c[1][0], m.c[1][1]};
      double gi[4] = {mi.c[0][0], mi.c[0][1], mi.c[1][0], mi.c[1][1]};
      for (int q = 0; q < 4; q++) { w.triMetric[4 * e + q] = gm[q]; w.triMetricInv[4 * e + q] = gi[q]; }
      w.triScale[e] = std::sqrt(m.det());
    }
  }
  // interior cells: global order = chart order, then interior cell order
  std::vector<int> icBase(L.charts.size() + 1, 0), btBase(L.charts.size() + 1, 0);
  for (size_t c = 0; c < L.charts.size(); c++) icBase[c + 1] = icBase[c] + L.charts[c].numInteriorCells;
  w.numInteriorCells = icBase.back();
  w.cellIJ.resize(2 * size_t(w.numInteriorCells));
  w.cellChart.resize(w.numInteriorCells);
#pragma omp parallel for schedule(dynamic, 1)
  for (int c = 0; c < nCharts; c++) {
    const GridChart& gc = L.charts[c];
    for (int j = 0; j < gc.height - 1; j++)
      for (int i = 0; i < gc.width - 1; i++) {
        int ic = gc.localInteriorCell[gc.cat(i, j)];
        if (ic < 0) continue;
        w.cellIJ[2 * (icBase[c] + ic)] = i;
        w.cellIJ[2 * (icBase[c] + ic) + 1] = j;
        w.cellChart[icBase[c] + ic] = (int)c;
      }
  }
  w.chartCellSize.resize(2 * L.charts.size());
  for (size_t c = 0; c < L.charts.size(); c++) {
    w.chartCellSize[2 * c] = L.charts[c].cellSizeW;
    w.chartCellSize[2 * c + 1] = L.charts[c].cellSizeH;
  }
  // boundary triangles: global order = chart order, boundary cell order, triangle order
  for (size_t c = 0; c < L.charts.size(); c++) {
    int n = 0;
    for (auto& v : be.charts[c].cellTriangles) n += (int)v.size();
    btBase[c + 1] = btBase[c] + n;
  }
  w.numBoundaryTriangles = btBase.back();
  w.btPos.resize(6 * size_t(w.numBoundaryTriangles));
  w.btIdx.resize(6 * size_t(w.numBoundaryTriangles));
  std::vector<std::vector<int>> cellFirstBt(L.charts.size());
  for (size_t c = 0; c < L.charts.size(); c++) {
    int b = btBase[c];
    cellFirstBt[c].resize(be.charts[c].cellTriangles.size() + 1);
    for (size_t cell = 0; cell < be.charts[c].cellTriangles.size(); cell++) {
      cellFirstBt[c][cell] = b;
      for (const BoundaryTriangle& bt : be.charts[c].cellTriangles[cell]) {
        for (int k = 0; k < 3; k++) { w.btPos[6 * size_t(b) + 2 * k] = bt.v[k].x; w.btPos[6 * size_t(b) + 2 * k + 1] = bt.v[k].y; }
        for (int k = 0; k < 6; k++) w.btIdx[6 * size_t(b) + k] = be.fineBoundaryIndex[bt.idx[k]];
        b++;
      }
    }
    cellFirstBt[c][be.charts[c].cellTriangles.size()] = b;
  }
  // (cell or boundary triangle, chart triangle) pairs, bucketed by cell and
  // boundary triangle in chart-triangle order.  A chart's pairs only touch its
  // own cells and boundary triangles, so the charts count and fill in parallel:
  // count, prefix sums, fill.
  w.cellPtr.assign(size_t(w.numInteriorCells) + 1, 0);
  w.btPtr.assign(size_t(w.numBoundaryTriangles) + 1, 0);
  auto visit_pairs = [&](int c, auto&& onCell, auto&& onBt) {
    const AtlasChart& ac = A.charts[c];
    const GridChart& gc = L.charts[c];
    for (size_t t = 0; t < ac.triangles.size(); t++) {
      V2 p[3];
      for (int k = 0; k < 3; k++) p[k] = ac.vertices[ac.triangles[t][k]] - gc.corner;
      int mn[2], mx[2];
      bbox_cells(p, gc.cellSizeW, gc.cellSizeH, mn, mx);
      const int tri = triBase[c] + (int)t;
      for (int j = mn[1]; j < mx[1]; j++)
        for (int i = mn[0]; i < mx[0]; i++) {
          int ic = gc.localInteriorCell[gc.cat(i, j)];
          if (ic >= 0) { onCell(icBase[c] + ic, tri); continue; }
          int bc = gc.localBoundaryCell[gc.cat(i, j)];
          if (bc >= 0)
            for (int b = cellFirstBt[c][bc]; b < cellFirstBt[c][bc + 1]; b++) onBt(b, tri);
        }
    }
  };
#pragma omp parallel for schedule(dynamic, 1)
  for (int c = 0; c < nCharts; c++)
    visit_pairs(c, [&](int cell, int) { w.cellPtr[size_t(cell) + 1]++; }, [&](int b, int) { w.btPtr[size_t(b) + 1]++; });
  for (int i = 0; i < w.numInteriorCells; i++) w.cellPtr[i + 1] += w.cellPtr[i];
  for (int i = 0; i < w.numBoundaryTriangles; i++) w.btPtr[i + 1] += w.btPtr[i];
  w.cellTri.resize(w.cellPtr.back());
  w.btTri.resize(w.btPtr.back());
  {
    std::vector<int> cellFill(w.cellPtr.begin(), w.cellPtr.end() - 1), btFill(w.btPtr.begin(), w.btPtr.end() - 1);
#pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < nCharts; c++)
      visit_pairs(c, [&](int cell, int tri) { w.cellTri[cellFill[cell]++] = tri; }, [&](int b, int tri) { w.btTri[btFill[b]++] = tri; });
  }

  // deep texels: the four surrounding interior cells (raster order) and the
  // texel's corner slot in each
  w.deepCells.resize(4 * size_t(L.numDeep));
#pragma omp parallel for schedule(dynamic, 1)
  for (int c = 0; c < nCharts; c++) {
    const GridChart& gc = L.charts[c];
    for (int j = 0; j < gc.height; j++)
      for (int i = 0; i < gc.width; i++) {
        int d = gc.deepTexel[gc.at(i, j)];
        if (d < 0) continue;
        const int ci[4] = {i - 1, i, i - 1, i}, cj[4] = {j - 1, j - 1, j, j};
        for (int q = 0; q < 4; q++) w.deepCells[4 * size_t(d) + q] = icBase[c] + gc.localInteriorCell[gc.cat(ci[q], cj[q])];
      }
  }
  // interior cells touching a boundary texel (their boundary rows are built on the host)
  std::vector<char> adjacent(w.numInteriorCells, 0);
#pragma omp parallel for schedule(static)
  for (int ic = 0; ic < w.numInteriorCells; ic++) {
    const GridChart& gc = L.charts[w.cellChart[ic]];
    int i = w.cellIJ[2 * ic], j = w.cellIJ[2 * ic + 1];
    int q[4] = {gc.at(i, j), gc.at(i + 1, j), gc.at(i + 1, j + 1), gc.at(i, j + 1)};
    for (int k = 0; k < 4; k++)
      if (gc.nodeType[q[k]] != 2) { adjacent[ic] = 1; break; }
  }
  for (int ic = 0; ic < w.numInteriorCells; ic++)
    if (adjacent[ic]) w.boundaryAdjacentCells.push_back(ic);
}

// Deep coefficient of texel slot k (corner of a cell) toward neighbour slot l.
static inline int neighbour_offset(int k, int l) {
  static const int oi[4] = {0, 1, 1, 0}, oj[4] = {0, 0, 1, 1};
  return (oj[l] - oj[k] + 1) * 3 + (oi[l] - oi[k] + 1);
}

bool assemble_boundary_blocks(const Hierarchy& h, const BoundaryElements& be, const AssemblyWork& w,
                              const std::vector<double>& adjCellMass, const std::vector<double>& adjCellStiffness,
                              const std::vector<double>& btMass, const std::vector<double>& btStiffness, FineSystem& fs,
                              std::string& err) {
  const GridLevel& L = h.levels[0];
  // entries in a fixed order (adjacent cells, then boundary triangles), each
  // cell's and triangle's slots computed first so that they fill in parallel
  const int nAdj = (int)w.boundaryAdjacentCells.size();
  std::vector<int> bbCount(size_t(nAdj) + 1, 0), bdCount(size_t(nAdj) + 1, 0);
  bool bad = false;
#pragma omp parallel for schedule(static) reduction(||: bad)
  for (int a = 0; a < nAdj; a++) {
    const int ic = w.boundaryAdjacentCells[a];
    const GridChart& gc = L.charts[w.cellChart[ic]];
    const int i = w.cellIJ[2 * ic], j = w.cellIJ[2 * ic + 1];
    const int pos[4] = {gc.at(i, j), gc.at(i + 1, j), gc.at(i + 1, j + 1), gc.at(i, j + 1)};
    int nbb = 0, nbd = 0;
    for (int k = 0; k < 4; k++) {
      if (L.boundaryAndDeep[gc.texel[pos[k]]] < 0) continue;  // deep rows come from the device gather
      for (int l = 0; l < 4; l++) {
        if (L.boundaryAndDeep[gc.texel[pos[l]]] < 0) nbd++;
        else {
          nbb++;
          if (be.fineBoundaryIndex[gc.interiorTexel[pos[k]]] < 0 || be.fineBoundaryIndex[gc.interiorTexel[pos[l]]] < 0) bad = true;
        }
      }
    }
    bbCount[a + 1] = nbb;
    bdCount[a + 1] = nbd;
  }
  if (bad) { err = "interior cell corner without fine boundary index"; return false; }
  for (int a = 0; a < nAdj; a++) {
    bbCount[a + 1] += bbCount[a];
    bdCount[a + 1] += bdCount[a];
  }
  const size_t nbbCells = size_t(bbCount[nAdj]), nbb = nbbCells + 36 * size_t(w.numBoundaryTriangles), nbd = size_t(bdCount[nAdj]);
  std::vector<int> bbR(nbb), bbC(nbb), bdR(nbd), bdC(nbd);
  std::vector<double> bbMv(nbb), bbSv(nbb), bdMv(nbd), bdSv(nbd);
#pragma omp parallel for schedule(static)
  for (int a = 0; a < nAdj; a++) {
    const int ic = w.boundaryAdjacentCells[a];
    const GridChart& gc = L.charts[w.cellChart[ic]];
    const int i = w.cellIJ[2 * ic], j = w.cellIJ[2 * ic + 1];
    const int pos[4] = {gc.at(i, j), gc.at(i + 1, j), gc.at(i + 1, j + 1), gc.at(i, j + 1)};
    const double* M = &adjCellMass[16 * size_t(a)];
    const double* S = &adjCellStiffness[16 * size_t(a)];
    size_t ob = size_t(bbCount[a]), od = size_t(bdCount[a]);
    for (int k = 0; k < 4; k++) {
      const int node = gc.texel[pos[k]];
      const int bdk = L.boundaryAndDeep[node];
      if (bdk < 0) continue;
      const int b = bdk - 1;
      for (int l = 0; l < 4; l++) {
        const int nb = gc.texel[pos[l]];
        if (L.boundaryAndDeep[nb] < 0) {
          bdR[od] = b;
          bdC[od] = nb;
          bdMv[od] = M[4 * k + l];
          bdSv[od++] = S[4 * k + l];
        } else {
          bbR[ob] = be.fineBoundaryIndex[gc.interiorTexel[pos[k]]];
          bbC[ob] = be.fineBoundaryIndex[gc.interiorTexel[pos[l]]];
          bbMv[ob] = M[4 * k + l];
          bbSv[ob++] = S[4 * k + l];
        }
      }
    }
  }
#pragma omp parallel for schedule(static)
  for (int b = 0; b < w.numBoundaryTriangles; b++) {
    const int* f = &w.btIdx[6 * size_t(b)];
    const double* M = &btMass[36 * size_t(b)];
    const double* S = &btStiffness[36 * size_t(b)];
    size_t o = nbbCells + 36 * size_t(b);
    for (int k = 0; k < 6; k++)
      for (int l = 0; l < 6; l++, o++) {
        bbR[o] = f[k];
        bbC[o] = f[l];
        bbMv[o] = M[6 * l + k];
        bbSv[o] = S[6 * l + k];
      }
  }
  // fine boundary blocks, then the texel boundary blocks P^T BB P (one pattern for M and S)
  Csr fineBBM, fineBBS;
  csr_from_pairs(be.numFineBoundary, be.numFineBoundary, bbR, bbC, bbMv, bbSv, fineBBM, fineBBS);
  const Csr R = csr_transpose(be.prolongation);
  Csr bbPM, bbPS;
  csr_multiply2(fineBBM, &fineBBS.val, be.prolongation, nullptr, bbPM, bbPS);
  csr_multiply2(R, nullptr, bbPM, &bbPS.val, fs.bbMass, fs.bbStiffness);
  csr_from_pairs(L.numBoundary, L.numTexels, bdR, bdC, bdMv, bdSv, fs.bdMass, fs.bdStiffness);
  return true;
}

}  // namespace gdtp
