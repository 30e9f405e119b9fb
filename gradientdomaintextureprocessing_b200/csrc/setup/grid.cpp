// Texel-grid hierarchy: per level and chart, node/cell classification, global,
// interior, deep and boundary indexing, raster lines, and the fine<->coarse
// line descriptors used by restriction and prolongation.
//
// Reference functions restated (same FP64 formulas, same orders, so indices are
// bit-exact):
//   grid chart extents           Src/HierarchyConstruction.inl:496-532
//   node / cell classification   Src/HierarchyConstruction.inl:39-229
//   enumeration + raster lines   Src/HierarchyConstruction.inl:231-395
//   boundary/deep indexing       Src/HierarchyConstruction.inl:3-35
//   restriction + deep lines     Src/ProlongationAndRestriction.inl:266-372
//   boundary restriction matrix  Src/ProlongationAndRestriction.inl:374-452
//   prolongation lines           Src/ProlongationAndRestriction.inl:99-171
// The reference's OpenMP block tasks (HierarchyConstruction.inl:397-490) are not
// built: the device smoother partitions work by colour runs instead.
#include <algorithm>
#include <cmath>

#include "setup.h"

namespace gdtp {

// Integer bounding box of a point set in cell units, clamped to the unit square.
// (GetTriangleIntegerBBox / GetEdgeIntegerBBox, Src/PolygonClipping.h:576-606)
static void integer_bbox(const V2* p, int n, double invW, double invH, int mn[2], int mx[2]) {
  double fminx = p[0].x, fminy = p[0].y, fmaxx = p[0].x, fmaxy = p[0].y;
  for (int i = 1; i < n; i++) {
    fminx = std::min(fminx, p[i].x); fminy = std::min(fminy, p[i].y);
    fmaxx = std::max(fmaxx, p[i].x); fmaxy = std::max(fmaxy, p[i].y);
  }
  fminx = std::max(fminx, 0.0); fminy = std::max(fminy, 0.0);
  fmaxx = std::min(fmaxx, 1.0); fmaxy = std::min(fmaxy, 1.0);
  mn[0] = int(std::floor(fminx * invW)); mn[1] = int(std::floor(fminy * invH));
  mx[0] = int(std::ceil(fmaxx * invW)); mx[1] = int(std::ceil(fmaxy * invH));
}

static M2 barycentric_map(const V2 t[3]) {
  M2 m;
  m.c[0][0] = t[1].x - t[0].x; m.c[0][1] = t[1].y - t[0].y;
  m.c[1][0] = t[2].x - t[0].x; m.c[1][1] = t[2].y - t[0].y;
  return m.inverse();
}

// (1)-(3): node and cell types of one chart (chart-local; charts in parallel)
static bool classify_chart(const AtlasChart& ac, GridChart& g, int deepRadius, std::string& err) {
  const int W = g.width, H = g.height;
  const double cw = g.cellSizeW, ch = g.cellSizeH;
  g.nodeType.assign(size_t(W) * H, -1);
  g.cellType.assign(size_t(W - 1) * (H - 1), -1);
  g.triangleId.assign(size_t(W) * H, -1);
  g.bary.assign(size_t(W) * H, V2());

  // (1) texels covered by a chart triangle (barycentric test in FP64)
  for (size_t t = 0; t < ac.triangles.size(); t++) {
    V2 tp[3];
    for (int k = 0; k < 3; k++) tp[k] = ac.vertices[ac.triangles[t][k]] - g.corner;
    int mn[2], mx[2];
    integer_bbox(tp, 3, 1.0 / cw, 1.0 / ch, mn, mx);
    M2 bm = barycentric_map(tp);
    for (int j = mn[1]; j <= mx[1]; j++)
      for (int i = mn[0]; i <= mx[0]; i++) {
        V2 b = bm * (V2(double(i) * cw, double(j) * ch) - tp[0]);
        if (b.x >= 0.0 && b.y >= 0.0 && (b.x + b.y) <= 1.0) {
          int n = g.at(i, j);
          if (g.nodeType[n] != -1) { err = "texel covered by two triangles (degenerate atlas)"; return false; }
          g.nodeType[n] = 1;
          g.triangleId[n] = ac.meshTriangleIndices[t];
          g.bary[n] = b;
        }
      }
  }

  // (2) texels around cells cut by boundary edges, or holding a whole boundary triangle
  auto mark_exterior = [&](int ni, int nj, const M2& bm, const V2& t0, int meshTri) {
    ni = std::min(std::max(0, ni), W - 1);
    nj = std::min(std::max(0, nj), H - 1);
    int n = g.at(ni, nj);
    if (g.nodeType[n] == 1) return;
    g.nodeType[n] = 0;
    V2 b = bm * (V2(double(ni) * cw, double(nj) * ch) - t0);
    if (g.triangleId[n] == -1) {
      g.triangleId[n] = meshTri;
      g.bary[n] = b;
    } else {  // keep the triangle the texel is closest to
      V2 o = g.bary[n];
      double minOld = std::min(std::min(1.0 - o.x - o.y, o.x), o.y);
      double minNew = std::min(std::min(1.0 - b.x - b.y, b.x), b.y);
      if (minNew > minOld) { g.triangleId[n] = meshTri; g.bary[n] = b; }
    }
  };
  for (int he : ac.boundaryHalfEdges) {
    int t = he / 3, k = he % 3;
    V2 e[2] = {ac.vertices[ac.triangles[t][k]] - g.corner, ac.vertices[ac.triangles[t][(k + 1) % 3]] - g.corner};
    int mn[2], mx[2];
    integer_bbox(e, 2, 1.0 / cw, 1.0 / ch, mn, mx);
    V2 tp[3];
    for (int q = 0; q < 3; q++) tp[q] = ac.vertices[ac.triangles[t][q]] - g.corner;
    M2 bm = barycentric_map(tp);
    const int meshTri = ac.meshTriangleIndices[t];
    V2 ed = e[1] - e[0];
    V2 en(ed.y, -ed.x);
    en = en / std::sqrt(en.x * en.x + en.y * en.y);
    double eLevel = (dot(en, e[0]) + dot(en, e[1])) / 2.0;
    for (int c = 0; c < 2; c++)
      for (int j = mn[1]; j <= mx[1]; j++)
        for (int i = mn[0]; i <= mx[0]; i++) {
          V2 n0(double(i) * cw, double(j) * ch), n1 = n0;
          if (c == 0) n1.x += cw; else n1.y += ch;
          V2 side = n1 - n0;
          V2 sn(side.y, -side.x);
          sn = sn / std::sqrt(sn.x * sn.x + sn.y * sn.y);
          double cLevel = (dot(sn, n0) + dot(sn, n1)) / 2.0;
          bool crossEdge = (dot(en, n0) - eLevel) * (dot(en, n1) - eLevel) < 0.0;
          bool crossSide = (dot(sn, e[1]) - cLevel) * (dot(sn, e[0]) - cLevel) < 0.0;
          if (!(crossEdge && crossSide)) continue;
          auto set_boundary_cell = [&](int ci, int cj) {
            if (ci >= 0 && cj >= 0 && ci < W - 1 && cj < H - 1) g.cellType[g.cat(ci, cj)] = 0;
          };
          if (c == 0) { set_boundary_cell(i, j - 1); set_boundary_cell(i, j); }
          else { set_boundary_cell(i - 1, j); set_boundary_cell(i, j); }
          for (int dn = -1; dn <= 1; dn++)
            for (int dc = 0; dc < 2; dc++) {
              int idx[2] = {i, j};
              idx[1 - c] += dn;
              idx[c] += dc;
              mark_exterior(idx[0], idx[1], bm, tp[0], meshTri);
            }
        }
    if (mn[0] + 1 == mx[0] && mn[1] + 1 == mx[1]) {
      g.cellType[g.cat(mn[0], mn[1])] = 0;
      for (int di = 0; di < 2; di++)
        for (int dj = 0; dj < 2; dj++) mark_exterior(mn[0] + di, mn[1] + dj, bm, tp[0], meshTri);
    }
  }

  // (3) interior cells and deep texels
  for (int j = 0; j < H - 1; j++)
    for (int i = 0; i < W - 1; i++)
      if (g.nodeType[g.at(i, j)] == 1 && g.nodeType[g.at(i + 1, j)] == 1 && g.nodeType[g.at(i, j + 1)] == 1 &&
          g.nodeType[g.at(i + 1, j + 1)] == 1 && g.cellType[g.cat(i, j)] == -1)
        g.cellType[g.cat(i, j)] = 1;
  for (int j = deepRadius; j < H - deepRadius; j++)
    for (int i = deepRadius; i < W - deepRadius; i++) {
      bool deep = true;
      for (int di = -deepRadius; di < deepRadius && deep; di++)
        for (int dj = -deepRadius; dj < deepRadius; dj++)
          if (g.cellType[g.cat(i + di, j + dj)] != 1) { deep = false; break; }
      if (deep) g.nodeType[g.at(i, j)] = 2;
    }
  return true;
}

// Texel and cell counts of one chart (its nodeType / cellType images).
struct ChartCounts { int texels = 0, interior = 0, boundary = 0, deep = 0, cells = 0; };
static ChartCounts count_chart(const GridChart& g) {
  ChartCounts k;
  for (int t : g.nodeType) {
    if (t != -1) k.texels++;
    if (t >= 1) k.interior++;
    if (t == 0 || t == 1) k.boundary++;
    if (t == 2) k.deep++;
  }
  for (int c : g.cellType)
    if (c != -1) k.cells++;
  return k;
}

// (4)-(5): global enumeration of one chart's texels and cells from its offsets
// (the counts of the charts before it): texels, cells, their nodes and raster
// lines in raster order.  Charts enumerate in parallel; L.nodes is presized.
static bool enumerate_chart(int chartId, GridChart& g, GridLevel& L, std::vector<Line>& lines, std::string& err) {
  const int W = g.width, H = g.height;
  // (4) enumeration
  int nTex = g.texelOffset, nInt = g.interiorTexelOffset, nBnd = g.boundaryOffset, nDeep = g.deepOffset;
  g.texel.assign(size_t(W) * H, -1);
  g.interiorTexel.assign(size_t(W) * H, -1);
  g.deepTexel.assign(size_t(W) * H, -1);
  g.boundaryTexel.assign(size_t(W) * H, -1);
  for (int j = 0; j < H; j++)
    for (int i = 0; i < W; i++) {
      int n = g.at(i, j), t = g.nodeType[n];
      if (t != -1) { L.nodes[nTex] = {chartId, i, j, t}; g.texel[n] = nTex++; }
      if (t >= 1) g.interiorTexel[n] = nInt++;
      if (t == 0 || t == 1) g.boundaryTexel[n] = nBnd++;
      if (t == 2) g.deepTexel[n] = nDeep++;
    }
  g.localCell.assign(size_t(W - 1) * (H - 1), -1);
  g.localInteriorCell.assign(size_t(W - 1) * (H - 1), -1);
  g.localBoundaryCell.assign(size_t(W - 1) * (H - 1), -1);
  int nCell = 0;
  for (int j = 0; j < H - 1; j++)
    for (int i = 0; i < W - 1; i++) {
      int c = g.cat(i, j);
      if (g.cellType[c] == -1) continue;
      g.localCell[c] = nCell++;
      int q[4] = {g.texel[g.at(i, j)], g.texel[g.at(i + 1, j)], g.texel[g.at(i + 1, j + 1)], g.texel[g.at(i, j + 1)]};
      if (q[0] < 0 || q[1] < 0 || q[2] < 0 || q[3] < 0) { err = "active cell adjacent to inactive texel"; return false; }
      g.cellCorners.insert(g.cellCorners.end(), q, q + 4);
      if (g.cellType[c] == 0) {
        g.localBoundaryCell[c] = g.numBoundaryCells++;
        g.boundaryCellToCell.push_back(nCell - 1);
      } else {
        g.localInteriorCell[c] = g.numInteriorCells++;
        g.interiorCellToCell.push_back(nCell - 1);
        g.interiorCellCorners.insert(g.interiorCellCorners.end(), q, q + 4);
      }
    }

  // (5) raster lines: maximal runs of deep texels per row
  for (int j = 0; j < H; j++) {
    int start = -1;
    bool prevDeep = false;
    for (int i = 0; i < W; i++) {
      bool deep = g.nodeType[g.at(i, j)] == 2;
      if (deep && !prevDeep) start = i;
      if (!deep && prevDeep) {
        Line l{g.texel[g.at(start, j)], g.texel[g.at(i - 1, j)], g.texel[g.at(start, j - 1)], g.texel[g.at(start, j + 1)],
               g.deepTexel[g.at(start, j)]};
        if (l.start < 0 || l.end < 0 || l.prev < 0 || l.next < 0) { err = "invalid raster line"; return false; }
        lines.push_back(l);
      }
      prevDeep = deep;
    }
  }
  return true;
}

static bool build_level(const Atlas& A, int level, int width, int height, const BlockInfo& info, GridLevel& L,
                        std::string& err) {
  const int factor = 1 << level;
  const double cw = double(factor) / double(width);
  const double ch = double(factor) / double(height);
  L.charts.assign(A.charts.size(), GridChart());
  const int nCharts = (int)A.charts.size();
  std::vector<std::string> chartErr(nCharts);
#pragma omp parallel for schedule(dynamic, 1)
  for (int c = 0; c < nCharts; c++) {
    const AtlasChart& ac = A.charts[c];
    GridChart& g = L.charts[c];
    int half[2][2];
    for (int d = 0; d < 2; d++) {
      double cs = d == 0 ? cw : ch;
      half[d][0] = int(std::ceil((ac.gridOrigin[d] - ac.minCorner[d]) / cs));
      half[d][1] = int(std::ceil((ac.maxCorner[d] - ac.gridOrigin[d]) / cs));
      g.corner[d] = ac.gridOrigin[d] - cs * double(half[d][0]);
      g.centerOffset[d] = half[d][0];
      g.cornerCoords[d] = ac.originCoords[d] - half[d][0];
    }
    g.width = half[0][0] + half[0][1] + 1;
    g.height = half[1][0] + half[1][1] + 1;
    g.cellSizeW = cw;
    g.cellSizeH = ch;
    int approx = std::max(int(std::ceil(1.0 / cw)), int(std::ceil(1.0 / ch)));
    g.gridIndexOffset = 2 * approx * approx * int(c);
    classify_chart(ac, g, info.boundaryDilation + 1, chartErr[c]);
  }
  for (int c = 0; c < nCharts; c++)
    if (!chartErr[c].empty()) { err = chartErr[c]; return false; }
  // offsets of every chart from the counts of the charts before it
  std::vector<ChartCounts> counts(nCharts);
#pragma omp parallel for schedule(dynamic, 1)
  for (int c = 0; c < nCharts; c++) counts[c] = count_chart(L.charts[c]);
  for (int c = 0; c < nCharts; c++) {
    GridChart& g = L.charts[c];
    g.texelOffset = L.numTexels;
    g.interiorTexelOffset = L.numInteriorTexels;
    g.cellOffset = L.numCells;
    g.deepOffset = L.numDeep;
    g.boundaryOffset = L.numBoundary;
    L.numTexels += counts[c].texels;
    L.numInteriorTexels += counts[c].interior;
    L.numBoundary += counts[c].boundary;
    L.numDeep += counts[c].deep;
    L.numCells += counts[c].cells;
  }
  L.nodes.resize(L.numTexels);
  std::vector<std::vector<Line>> lines(nCharts);
#pragma omp parallel for schedule(dynamic, 1)
  for (int c = 0; c < nCharts; c++) enumerate_chart(c, L.charts[c], L, lines[c], chartErr[c]);
  for (int c = 0; c < nCharts; c++) {
    if (!chartErr[c].empty()) { err = chartErr[c]; return false; }
    L.numBoundaryCells += L.charts[c].numBoundaryCells;
    L.numInteriorCells += L.charts[c].numInteriorCells;
    L.rasterLines.insert(L.rasterLines.end(), lines[c].begin(), lines[c].end());
  }
  if (L.numTexels != L.numBoundary + L.numDeep) { err = "boundary and deep texels do not partition the texels"; return false; }
  L.boundaryAndDeep.assign(L.numTexels, 0);
  int nb = 1, nd = -1, g = 0;
  for (auto& ch2 : L.charts)
    for (int n = 0; n < ch2.width * ch2.height; n++) {
      int t = ch2.nodeType[n];
      if (t == 0 || t == 1) { L.boundaryGlobal.push_back(g); L.boundaryAndDeep[g] = nb++; }
      else if (t == 2) { L.deepGlobal.push_back(g); L.boundaryAndDeep[g] = nd--; }
      else continue;
      if (ch2.texel[n] != g) { err = "unexpected global texel index"; return false; }
      g++;
    }
  return true;
}

static bool build_restriction(GridLevel& F, GridLevel& C, std::string& err) {
  C.restrictionLines.resize(C.rasterLines.size());
  C.deepLines.resize(C.rasterLines.size());
  for (size_t r = 0; r < C.rasterLines.size(); r++) {
    const Line& cl = C.rasterLines[r];
    const NodeInfo& sn = C.nodes[cl.start];
    if (sn.type != 2) { err = "restriction line does not start at a deep texel"; return false; }
    const GridChart& fc = F.charts[sn.chart];
    const GridChart& cc = C.charts[sn.chart];
    int fi = fc.centerOffset[0] + 2 * (sn.ci - cc.centerOffset[0]);
    int fj = fc.centerOffset[1] + 2 * (sn.cj - cc.centerOffset[1]);
    if (fi - 1 < 0 || fi + 1 > fc.width - 1 || fj - 1 < 0 || fj + 1 > fc.height - 1) { err = "restriction out of bounds"; return false; }
    Line& rl = C.restrictionLines[r];
    DeepLine& dl = C.deepLines[r];
    rl.coeff = cl.start;
    dl.coarseStart = cl.coeff;
    dl.coarseEnd = cl.coeff + (cl.end - cl.start);
    rl.start = fc.texel[fc.at(fi, fj)];
    rl.end = rl.start + 2 * (cl.end - cl.start);
    rl.prev = fc.texel[fc.at(fi, fj - 1)];
    rl.next = fc.texel[fc.at(fi, fj + 1)];
    dl.fineCurrent = fc.deepTexel[fc.at(fi, fj)];
    dl.finePrev = fc.deepTexel[fc.at(fi, fj - 1)];
    dl.fineNext = fc.deepTexel[fc.at(fi, fj + 1)];
    if (rl.start < 0 || rl.prev < 0 || rl.next < 0 || dl.fineCurrent < 0 || dl.finePrev < 0 || dl.fineNext < 0) {
      err = "invalid restriction line";
      return false;
    }
  }
  // boundary rows of the transfer operator: full weighting restricted to coarse boundary texels
  std::vector<Triplet> trip;
  for (size_t k = 0; k < F.charts.size(); k++) {
    const GridChart& fc = F.charts[k];
    const GridChart& cc = C.charts[k];
    for (int fj = 0; fj < fc.height; fj++)
      for (int fi = 0; fi < fc.width; fi++) {
        int fg = fc.texel[fc.at(fi, fj)];
        if (fg == -1) continue;
        int ri = fi - fc.centerOffset[0], rj = fj - fc.centerOffset[1];
        int si = ri < 0 ? -1 : (ri > 0 ? 1 : 0), sj = rj < 0 ? -1 : (rj > 0 ? 1 : 0);
        int ci[2], cj[2];
        double wi[2], wj[2];
        if (ri % 2 == 0) { ci[0] = ri / 2 + cc.centerOffset[0]; ci[1] = -1; wi[0] = 1.0; wi[1] = 0.0; }
        else { ci[0] = ri / 2 + cc.centerOffset[0]; ci[1] = (ri + si) / 2 + cc.centerOffset[0]; wi[0] = wi[1] = 0.5; }
        if (rj % 2 == 0) { cj[0] = rj / 2 + cc.centerOffset[1]; cj[1] = -1; wj[0] = 1.0; wj[1] = 0.0; }
        else { cj[0] = rj / 2 + cc.centerOffset[1]; cj[1] = (rj + sj) / 2 + cc.centerOffset[1]; wj[0] = wj[1] = 0.5; }
        for (int a = 0; a < 2; a++)
          for (int b = 0; b < 2; b++) {
            if (ci[a] == -1 || cj[b] == -1) continue;
            int cg = cc.texel[cc.at(ci[a], cj[b])];
            if (cg == -1) { err = "coarse texel inactive under an active fine texel"; return false; }
            int cb = C.boundaryAndDeep[cg] - 1;
            if (cb >= 0) trip.push_back({cb, fg, wi[a] * wj[b]});
          }
      }
  }
  F.boundaryRestriction = csr_from_triplets(C.numBoundary, F.numTexels, trip);
  return true;
}

static bool build_prolongation(GridLevel& F, const GridLevel& C, std::string& err) {
  for (size_t k = 0; k < F.charts.size(); k++) {
    const GridChart& fc = F.charts[k];
    const GridChart& cc = C.charts[k];
    const int W = fc.width;
    for (int j = 0; j < fc.height; j++) {
      int start = -1;
      bool prevValid = false;
      for (int i = 0; i < W; i++) {
        bool valid = fc.texel[fc.at(i, j)] != -1;
        if (valid && !prevValid) start = i;
        bool endsHere = (!valid && prevValid) || (valid && i == W - 1);
        if (endsHere) {
          int stop = (valid && i == W - 1) ? i + 1 : i;
          ProlongationLine pl;
          pl.start = fc.texel[fc.at(start, j)];
          pl.length = stop - start;
          int ri = start - fc.centerOffset[0], rj = j - fc.centerOffset[1];
          int di = (ri % 2 == 0) ? 0 : 1, dj = (rj % 2 == 0) ? 0 : 1;
          int ci = (ri - di) / 2 + cc.centerOffset[0];
          int cj = (rj - dj) / 2 + cc.centerOffset[1];
          pl.aligned = (ri % 2 == 0) ? 1 : 0;
          if (rj % 2 == 0) {
            pl.prev = pl.next = -1;
            pl.center = cc.texel[cc.at(ci, cj)];
            if (pl.center == -1) { err = "prolongation reads an inactive coarse texel"; return false; }
          } else {
            pl.center = -1;
            pl.prev = cc.texel[cc.at(ci, cj)];
            pl.next = cc.texel[cc.at(ci, cj + 1)];
            if (pl.prev == -1 || pl.next == -1) { err = "prolongation reads an inactive coarse texel"; return false; }
          }
          F.prolongationLines.push_back(pl);
        }
        prevValid = valid;
      }
    }
  }
  return true;
}

bool build_hierarchy(const Mesh& mesh, int width, int height, int levels, const BlockInfo& info, Hierarchy& h,
                     int extendToTexels, int maxLevels) {
  h.error.clear();
  if (levels < 1) { h.error = "levels must be >= 1"; return false; }
  if (!build_atlas(mesh, width, height, h.atlas, h.error)) return false;
  h.levels.clear();
  h.requestedLevels = levels;
  for (int l = 0;; l++) {
    if (l >= levels && (extendToTexels <= 0 || h.levels.back().numTexels <= extendToTexels || l >= maxLevels)) break;
    h.levels.emplace_back();
    if (!build_level(h.atlas, l, width, height, info, h.levels[l], h.error)) {
      if (l >= levels) {  // an optional extra level that does not exist: stop coarsening
        h.levels.pop_back();
        h.error.clear();
        break;
      }
      h.error = "level " + std::to_string(l) + ": " + h.error;
      return false;
    }
  }
  levels = (int)h.levels.size();
  for (int l = 0; l + 1 < levels; l++)
    if (!build_restriction(h.levels[l], h.levels[l + 1], h.error) || !build_prolongation(h.levels[l], h.levels[l + 1], h.error)) {
      h.error = "level " + std::to_string(l) + ": " + h.error;
      return false;
    }
  return true;
}

}  // namespace gdtp
