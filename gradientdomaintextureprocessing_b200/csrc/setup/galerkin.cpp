// Galerkin coefficient hierarchy A_{l+1} = P_l^T A_l P_l, where P_l is the
// per-chart bilinear prolongation (weights 1, 1/2, 1/4 around the aligned
// coarse texel, ProlongationAndRestriction.inl:99-216).
//
// The reference builds the same operator from hand-expanded pieces
// (UpdateCoefficients.inl:1-135, 285-371): a closed form for deep rows
// (DeepCoefficientRestriction) and sparse products plus index tables for the
// boundary rows.  Here deep rows use the equivalent stencil form of P^T A P
// and boundary rows the direct row-wise product R_b (A P); both only differ from
// the reference by summation order.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>

#include "setup.h"

namespace gdtp {

static inline double w1(int d) { return d == 0 ? 1.0 : ((d == 1 || d == -1) ? 0.5 : 0.0); }

static inline int floor_div2(int a) { return a >= 0 ? a / 2 : -((-a + 1) / 2); }

// Coarse texels (global) and weights of fine texel q's prolongation row P(q, .):
// an even offset from the chart centre sits on a coarse texel, an odd one
// between two (weights 1/2 per axis).
static int prolong_row(const GridLevel& F, const GridLevel& C, int q, int cols[4], double wts[4]) {
  const NodeInfo& n = F.nodes[q];
  const GridChart& fc = F.charts[n.chart];
  const GridChart& cc = C.charts[n.chart];
  const int ri = n.ci - fc.centerOffset[0], rj = n.cj - fc.centerOffset[1];
  const bool oddI = (ri & 1) != 0, oddJ = (rj & 1) != 0;
  const int ci0 = floor_div2(ri) + cc.centerOffset[0], cj0 = floor_div2(rj) + cc.centerOffset[1];
  int m = 0;
  for (int a = 0; a < (oddI ? 2 : 1); a++)
    for (int b = 0; b < (oddJ ? 2 : 1); b++) {
      int g = cc.texel[cc.at(ci0 + a, cj0 + b)];
      if (g < 0) return -1;
      cols[m] = g;
      wts[m] = (oddI ? 0.5 : 1.0) * (oddJ ? 0.5 : 1.0);
      m++;
    }
  return m;
}

bool galerkin_hierarchy(const Hierarchy& h, int L, const std::vector<double>& deep0, const Csr& bb0, const Csr& bd0,
                        std::vector<LevelCoefficients>& out, std::string& err) {
  if (L <= 0 || L > (int)h.levels.size()) L = (int)h.levels.size();
  out.assign(L, LevelCoefficients());
  out[0].deep = deep0;
  out[0].bb = bb0;
  out[0].bd = bd0;
  for (int l = 0; l + 1 < L; l++) {
    const GridLevel& F = h.levels[l];
    const GridLevel& C = h.levels[l + 1];
    const LevelCoefficients& A = out[l];
    LevelCoefficients& B = out[l + 1];
    // ---- deep rows: stencil form of P^T A P
    B.deep.assign(10 * size_t(C.numDeep), 0.0);
    bool bad = false;
#pragma omp parallel for schedule(static) reduction(||: bad)
    for (int d = 0; d < C.numDeep; d++) {
      const NodeInfo& n = C.nodes[C.deepGlobal[d]];
      const GridChart& fc = F.charts[n.chart];
      const GridChart& cc = C.charts[n.chart];
      int fi = fc.centerOffset[0] + 2 * (n.ci - cc.centerOffset[0]);
      int fj = fc.centerOffset[1] + 2 * (n.cj - cc.centerOffset[1]);
      double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          int fd = fc.deepTexel[fc.at(fi + dx, fj + dy)];
          if (fd < 0) { bad = true; continue; }
          const double wp = w1(dx) * w1(dy);
          const double* a = &A.deep[10 * size_t(fd)];
          for (int oy = -1; oy <= 1; oy++)
            for (int ox = -1; ox <= 1; ox++) {
              double av = a[(oy + 1) * 3 + (ox + 1)] * wp;
              for (int v = -1; v <= 1; v++) {
                double wy = w1(dy + oy - 2 * v);
                if (wy == 0.0) continue;
                for (int u = -1; u <= 1; u++) {
                  double wx = w1(dx + ox - 2 * u);
                  if (wx != 0.0) acc[(v + 1) * 3 + (u + 1)] += av * wx * wy;
                }
              }
            }
        }
      for (int k = 0; k < 9; k++) B.deep[10 * size_t(d) + k] = acc[k];
    }
    if (bad) { err = "coarse deep texel over a non-deep fine neighbourhood"; return false; }
    // ---- boundary rows: R_b (A P), one row at a time (rows in parallel
    // chunks, their triplets concatenated in row order)
    const Csr& Rb = F.boundaryRestriction;
    std::vector<Triplet> tbb, tbd;
    const int nChunks = std::max(1, std::min(256, C.numBoundary / 64));
    std::vector<std::vector<Triplet>> cbb(nChunks), cbd(nChunks);
#pragma omp parallel reduction(||: bad)
    {
      std::vector<double> acc(C.numTexels, 0.0);
      std::vector<int> mark(C.numTexels, -1), touched;
#pragma omp for schedule(dynamic, 1)
      for (int q = 0; q < nChunks; q++) {
        const int b0 = int(int64_t(C.numBoundary) * q / nChunks), b1 = int(int64_t(C.numBoundary) * (q + 1) / nChunks);
        for (int b = b0; b < b1; b++) {
          touched.clear();
          auto add = [&](int fineCol, double v) {
            int cols[4];
            double wts[4];
            int m = prolong_row(F, C, fineCol, cols, wts);
            if (m < 0) { bad = true; return; }
            for (int k = 0; k < m; k++) {
              int c = cols[k];
              if (mark[c] != b) { mark[c] = b; acc[c] = 0.0; touched.push_back(c); }
              acc[c] += v * wts[k];
            }
          };
          for (int e = Rb.ptr[b]; e < Rb.ptr[b + 1]; e++) {
            const int p = Rb.col[e];
            const double wp = Rb.val[e];
            const int bd = F.boundaryAndDeep[p];
            if (bd < 0) {  // deep fine row: 9-point stencil
              const NodeInfo& n = F.nodes[p];
              const GridChart& fc = F.charts[n.chart];
              const double* a = &A.deep[10 * size_t(-bd - 1)];
              for (int oy = -1; oy <= 1; oy++)
                for (int ox = -1; ox <= 1; ox++) add(fc.texel[fc.at(n.ci + ox, n.cj + oy)], wp * a[(oy + 1) * 3 + (ox + 1)]);
            } else {
              const int fb = bd - 1;
              for (int k = A.bd.ptr[fb]; k < A.bd.ptr[fb + 1]; k++) add(A.bd.col[k], wp * A.bd.val[k]);
              for (int k = A.bb.ptr[fb]; k < A.bb.ptr[fb + 1]; k++) add(F.boundaryGlobal[A.bb.col[k]], wp * A.bb.val[k]);
            }
          }
          for (int c : touched) {
            int cb = C.boundaryAndDeep[c];
            if (cb > 0) cbb[q].push_back({b, cb - 1, acc[c]});
            else cbd[q].push_back({b, c, acc[c]});
          }
        }
      }
    }
    for (int q = 0; q < nChunks; q++) {
      tbb.insert(tbb.end(), cbb[q].begin(), cbb[q].end());
      tbd.insert(tbd.end(), cbd[q].begin(), cbd[q].end());
    }
    if (bad) { err = "prolongation reads an inactive coarse texel"; return false; }
    B.bb = csr_from_triplets(C.numBoundary, C.numBoundary, tbb);
    B.bd = csr_from_triplets(C.numBoundary, C.numTexels, tbd);
  }
  return true;
}

void full_matrix(const GridLevel& g, const LevelCoefficients& c, Csr& full) {
  std::vector<Triplet> t;
  t.reserve(size_t(g.numDeep) * 9 + c.bb.nnz() + c.bd.nnz());
  for (int d = 0; d < g.numDeep; d++) {
    int row = g.deepGlobal[d];
    const NodeInfo& n = g.nodes[row];
    const GridChart& gc = g.charts[n.chart];
    for (int oy = -1; oy <= 1; oy++)
      for (int ox = -1; ox <= 1; ox++) t.push_back({row, gc.texel[gc.at(n.ci + ox, n.cj + oy)], c.deep[10 * size_t(d) + (oy + 1) * 3 + (ox + 1)]});
  }
  for (int b = 0; b < g.numBoundary; b++) {
    int row = g.boundaryGlobal[b];
    for (int k = c.bd.ptr[b]; k < c.bd.ptr[b + 1]; k++) t.push_back({row, c.bd.col[k], c.bd.val[k]});
    for (int k = c.bb.ptr[b]; k < c.bb.ptr[b + 1]; k++) t.push_back({row, g.boundaryGlobal[c.bb.col[k]], c.bb.val[k]});
  }
  full = csr_from_triplets(g.numTexels, g.numTexels, t);
}

}  // namespace gdtp
