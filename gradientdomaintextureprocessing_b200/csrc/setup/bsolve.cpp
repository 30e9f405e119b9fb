// Exact solve of the boundary block BB of one level, set up for the device.
//
// The reference relaxes boundary texels by a sparse LDLT of BB at every
// smoothing step (IterativeSolvers.inl:193-209, 414-430; factorised in
// UpdateCoefficients.inl:402-439 with Eigen SimplicialLDLT, Solver.h:144-203).
// Boundary rows include texels whose support barely meets the chart (diagonals
// down to 1e-17 of the typical one), and pointwise relaxation of them stalls, so
// the exactness matters.  A sparse triangular solve is a long sequential chain
// on a GPU; instead the boundary graph is split into subdomains of at most
// `maxBlock` texels plus a vertex separator, and
//     BB^-1 r  =  [interiors: A_II^-1 (r_I - A_IS x_S)] , x_S = S^-1 (r_S - A_SI A_II^-1 r_I)
// with S = A_SS - A_SI A_II^-1 A_IS, is applied with dense block inverses only:
// every step is a batch of independent dense products.  All inverses are of the
// Jacobi-scaled block D^-1/2 BB D^-1/2 (unit diagonal), which keeps the FP32
// copies well scaled; they are computed here in FP64.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <numeric>
#include <queue>

#include "setup.h"

namespace gdtp {

// Dot products of contiguous rows.  The simd reductions sum in vector lanes
// (a fixed order for a given build, so results repeat run to run).
static inline double dot(const double* a, const double* b, int n) {
  double s = 0;
#pragma omp simd reduction(+ : s)
  for (int p = 0; p < n; p++) s += a[p] * b[p];
  return s;
}
// four rows against one: each element of b is loaded once for four products
static inline void dot4(const double* a0, const double* a1, const double* a2, const double* a3, const double* b, int n, double* out) {
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
#pragma omp simd reduction(+ : s0, s1, s2, s3)
  for (int p = 0; p < n; p++) {
    const double v = b[p];
    s0 += a0[p] * v;
    s1 += a1[p] * v;
    s2 += a2[p] * v;
    s3 += a3[p] * v;
  }
  out[0] = s0;
  out[1] = s1;
  out[2] = s2;
  out[3] = s3;
}

// In-place inverse of a dense SPD matrix (row-major, n x n) via Cholesky.
// Returns false if not positive definite.  Every phase works on 4 rows or
// columns at a time, so that a streamed row serves 4 inner products (the
// matrices of the coarsest level do not fit in cache).  Built for the baseline
// x86-64 ISA and for AVX2 + FMA, picked at load time by the CPU that runs it.
#if defined(__x86_64__) && defined(__GNUC__) && !defined(__CUDACC__)
__attribute__((target_clones("default", "arch=haswell")))
#endif
bool dense_spd_inverse(double* A, int n, bool parallel) {
  auto row = [&](int i) { return &A[size_t(i) * n]; };
  // ---- Cholesky A = L L^T (lower triangle), columns in blocks of 4
  for (int k0 = 0; k0 < n; k0 += 4) {
    const int kb = std::min(4, n - k0);
    // the block's own rows: columns k0 .. k0 + kb - 1, one after another
    for (int k = k0; k < k0 + kb; k++) {
      double* rk = row(k);
      const double d2 = rk[k] - dot(rk, rk, k);
      if (!(d2 > 0)) return false;
      rk[k] = std::sqrt(d2);
      for (int i = k + 1; i < k0 + kb; i++) {
        double* ri = row(i);
        ri[k] = (ri[k] - dot(ri, rk, k)) / rk[k];
      }
    }
    // rows below: the block's 4 columns share the prefix [0, k0)
#pragma omp parallel for schedule(static) if (parallel && n - k0 > 256)
    for (int i = k0 + kb; i < n; i++) {
      double* ri = row(i);
      double pre[4] = {0, 0, 0, 0};
      if (kb == 4) dot4(row(k0), row(k0 + 1), row(k0 + 2), row(k0 + 3), ri, k0, pre);
      else
        for (int c = 0; c < kb; c++) pre[c] = dot(row(k0 + c), ri, k0);
      for (int c = 0; c < kb; c++) {
        const int k = k0 + c;
        const double* rk = row(k);
        double s = ri[k] - pre[c];
        for (int p = k0; p < k; p++) s -= ri[p] * rk[p];
        ri[k] = s / rk[k];
      }
    }
  }
  // ---- W = L^-1 (lower), stored transposed (Wt[j][i] = W[i][j], zero for i < j),
  // columns in blocks of 4: row i of L is streamed once for the 4 columns
  std::vector<double> Wt(size_t(n) * n, 0.0);
  const int nb4 = (n + 3) / 4;
#pragma omp parallel for schedule(dynamic, 2) if (parallel)
  for (int jb = 0; jb < nb4; jb++) {
    const int j0 = 4 * jb, cb = std::min(4, n - j0);
    double* w[4];
    for (int c = 0; c < 4; c++) w[c] = &Wt[size_t(j0 + std::min(c, cb - 1)) * n];
    for (int c = 0; c < cb; c++) w[c][j0 + c] = 1.0 / A[size_t(j0 + c) * n + j0 + c];
    for (int i = j0 + 1; i < n; i++) {
      const double* ri = row(i);
      double s[4];
      // sum over p in [j0, i): the zeros of Wt below each column's start add nothing
      dot4(w[0] + j0, w[1] + j0, w[2] + j0, w[3] + j0, ri + j0, i - j0, s);
      for (int c = 0; c < cb; c++)
        if (i > j0 + c) w[c][i] = -s[c] / ri[i];
    }
  }
  // ---- A^-1 = W^T W: (i, j) = sum_p Wt[i][p] Wt[j][p], rows i in blocks of 4
#pragma omp parallel for schedule(dynamic, 2) if (parallel)
  for (int ib = 0; ib < nb4; ib++) {
    const int i0 = 4 * ib, rb = std::min(4, n - i0);
    const double* wi[4];
    for (int c = 0; c < 4; c++) wi[c] = &Wt[size_t(i0 + std::min(c, rb - 1)) * n];
    for (int j = 0; j < i0 + rb; j++) {
      // p from i0: Wt[i][p] is zero for p < i, so the common start adds zeros only
      double s[4];
      dot4(wi[0] + i0, wi[1] + i0, wi[2] + i0, wi[3] + i0, &Wt[size_t(j) * n] + i0, n - i0, s);
      for (int c = 0; c < rb; c++)
        if (j <= i0 + c) A[size_t(i0 + c) * n + j] = s[c];
    }
  }
  for (int i = 0; i < n; i++)
    for (int j = 0; j < i; j++) A[size_t(j) * n + i] = A[size_t(i) * n + j];
  return true;
}

void partition_boundary(const Csr& BB, int maxBlock, int denseMax, std::vector<int>& order, std::vector<int>& subPtr, int& nI) {
  const int nb = BB.rows;
  order.clear();
  subPtr.assign(1, 0);
  nI = 0;
  if (nb == 0) return;
  // ---- subdomains: breadth-first growth from the lowest unassigned row
  std::vector<int> part(nb, -1);
  int nSub = 0;
  if (nb <= maxBlock) {
    std::fill(part.begin(), part.end(), 0);
    nSub = 1;
  } else {
    for (int seed = 0; seed < nb; seed++) {
      if (part[seed] != -1) continue;
      std::queue<int> q;
      q.push(seed);
      part[seed] = nSub;
      int size = 1;
      while (!q.empty() && size < maxBlock) {
        int u = q.front();
        q.pop();
        for (int k = BB.ptr[u]; k < BB.ptr[u + 1] && size < maxBlock; k++) {
          int v = BB.col[k];
          if (part[v] == -1) { part[v] = nSub; size++; q.push(v); }
        }
      }
      nSub++;
    }
  }
  // ---- vertex separator: for every cut edge the endpoint in the higher subdomain
  std::vector<char> sep(nb, 0);
  for (int u = 0; u < nb; u++)
    for (int k = BB.ptr[u]; k < BB.ptr[u + 1]; k++) {
      int v = BB.col[k];
      if (part[u] != part[v]) sep[part[u] > part[v] ? u : v] = 1;
    }
  // a small block is inverted whole: every row in the "separator", whose Schur
  // complement is then the scaled block itself (one dense product per solve
  // instead of four dependent steps)
  if (nb <= denseMax) std::fill(sep.begin(), sep.end(), 1);
  // order: interiors grouped by subdomain, then separators
  std::vector<std::vector<int>> members(nSub);
  for (int u = 0; u < nb; u++)
    if (!sep[u]) members[part[u]].push_back(u);
  subPtr.assign(1, 0);
  for (int p = 0; p < nSub; p++) {
    if (members[p].empty()) continue;
    order.insert(order.end(), members[p].begin(), members[p].end());
    subPtr.push_back((int)order.size());
  }
  nI = (int)order.size();
  for (int u = 0; u < nb; u++)
    if (sep[u]) order.push_back(u);
}

namespace {
double wall_ms() { return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count(); }
}  // namespace

bool build_boundary_solver(const Csr& BB, const Csr& BD, int maxBlock, int denseMax, BoundarySolverSetup& bs, std::string& err,
                           DenseBackend* dense) {
  double tMark = wall_ms();
  auto lap = [&](int slot) {
    const double t = wall_ms();
    bs.ms[slot] += t - tMark;
    tMark = t;
  };
  const int nb = BB.rows;
  bs = BoundarySolverSetup();
  bs.nb = nb;
  if (nb == 0) return true;
  std::vector<double> diag(nb, 0.0);
  for (int i = 0; i < nb; i++)
    for (int k = BB.ptr[i]; k < BB.ptr[i + 1]; k++)
      if (BB.col[k] == i) diag[i] = BB.val[k];
  for (int i = 0; i < nb; i++)
    if (!(diag[i] > 0)) { err = "boundary block has a non-positive diagonal"; return false; }

  // ---- subdomains and separator; order: interiors grouped by subdomain, then separators
  partition_boundary(BB, maxBlock, denseMax, bs.order, bs.subPtr, bs.nI);
  bs.nSub = (int)bs.subPtr.size() - 1;
  bs.nS = nb - bs.nI;
  std::vector<int> pos(nb);
  for (int k = 0; k < nb; k++) pos[bs.order[k]] = k;
  bs.scale.resize(nb);
  for (int k = 0; k < nb; k++) bs.scale[k] = 1.0 / std::sqrt(diag[bs.order[k]]);
  auto scaled = [&](int i, int kk) { return BB.val[kk] * bs.scale[pos[i]] * bs.scale[pos[BB.col[kk]]]; };

  // ---- subdomain inverses (scaled), and the interior/separator couplings
  lap(0);
  bs.invOff.assign(bs.nSub + 1, 0);
  for (int p = 0; p < bs.nSub; p++) {
    int64_t m = bs.subPtr[p + 1] - bs.subPtr[p];
    bs.invOff[p + 1] = bs.invOff[p] + m * m;
  }
  bs.inv.assign(size_t(bs.invOff[bs.nSub]), 0.0);
  bool ok = true;
  std::vector<int> subSize(bs.nSub);
#pragma omp parallel for schedule(dynamic, 1) reduction(&& : ok)
  for (int p = 0; p < bs.nSub; p++) {
    const int b0 = bs.subPtr[p], m = bs.subPtr[p + 1] - b0;
    subSize[p] = m;
    double* D = &bs.inv[size_t(bs.invOff[p])];
    for (int a = 0; a < m; a++) {
      int i = bs.order[b0 + a];
      for (int kk = BB.ptr[i]; kk < BB.ptr[i + 1]; kk++) {
        int c = pos[BB.col[kk]] - b0;
        if (c >= 0 && c < m) D[size_t(a) * m + c] = scaled(i, kk);
      }
    }
    if (!dense) ok = dense_spd_inverse(D, m, false) && ok;
  }
  if (dense && bs.nSub > 0) {
    std::vector<int64_t> off(bs.invOff.begin(), bs.invOff.end() - 1);
    ok = dense->spd_inverse_batched(bs.inv.data(), off, subSize, err);
  }
  if (!ok) { err = "boundary subdomain block is not positive definite" + (err.empty() ? std::string() : ": " + err); return false; }
  lap(1);
  std::vector<Triplet> tIS;
  for (int k = 0; k < bs.nI; k++) {
    int i = bs.order[k];
    for (int kk = BB.ptr[i]; kk < BB.ptr[i + 1]; kk++) {
      int c = pos[BB.col[kk]];
      if (c >= bs.nI) tIS.push_back({k, c - bs.nI, scaled(i, kk)});
    }
  }
  bs.AIS = csr_from_triplets(bs.nI, bs.nS, tIS);
  bs.ASI = csr_transpose(bs.AIS);

  // ---- separator columns each subdomain touches, and W_p = Inv_p A_{I_p,S}
  // restricted to them (m x t, stored column-major): the back substitution
  // x_I = Inv_p (r_I - A_IS x_S) = y_p - W_p x_S reads W_p instead of Inv_p.
  bs.touchPtr.assign(bs.nSub + 1, 0);
  std::vector<std::vector<int>> touches(bs.nSub);
#pragma omp parallel for schedule(dynamic, 4)
  for (int p = 0; p < bs.nSub; p++) {
    std::vector<int>& touch = touches[p];
    for (int a = bs.subPtr[p]; a < bs.subPtr[p + 1]; a++)
      for (int kk = bs.AIS.ptr[a]; kk < bs.AIS.ptr[a + 1]; kk++) touch.push_back(bs.AIS.col[kk]);
    std::sort(touch.begin(), touch.end());
    touch.erase(std::unique(touch.begin(), touch.end()), touch.end());
  }
  bs.wOff.assign(bs.nSub + 1, 0);
  for (int p = 0; p < bs.nSub; p++) {
    bs.touchPtr[p + 1] = bs.touchPtr[p] + (int)touches[p].size();
    bs.wOff[p + 1] = bs.wOff[p] + int64_t(bs.subPtr[p + 1] - bs.subPtr[p]) * (int64_t)touches[p].size();
  }
  bs.touch.resize(bs.touchPtr[bs.nSub]);
  for (int p = 0; p < bs.nSub; p++) std::copy(touches[p].begin(), touches[p].end(), bs.touch.begin() + bs.touchPtr[p]);
  bs.W.assign(size_t(bs.wOff[bs.nSub]), 0.0);

  // ---- Schur complement on the separator, S = A_SS - A_SI A_II^-1 A_IS (scaled)
  if (bs.nS > 0) {
    const int nS = bs.nS;
    bs.Sinv.assign(size_t(nS) * nS, 0.0);
    for (int s = 0; s < nS; s++) {
      int i = bs.order[bs.nI + s];
      for (int kk = BB.ptr[i]; kk < BB.ptr[i + 1]; kk++) {
        int c = pos[BB.col[kk]];
        if (c >= bs.nI) bs.Sinv[size_t(s) * nS + (c - bs.nI)] = scaled(i, kk);
      }
    }
    // per-subdomain contributions, subtracted afterwards in subdomain order so
    // that the complement is bit-identical from run to run
    std::vector<std::vector<double>> contrib(bs.nSub);
    if (dense) {
      // C_p (m x t, row-major) for every subdomain, then G_p and C_p^T G_p on the device
      std::vector<int64_t> cOff(bs.nSub, 0), lOff(bs.nSub, 0);
      std::vector<int> tSize(bs.nSub);
      int64_t cTotal = 0, lTotal = 0;
      for (int p = 0; p < bs.nSub; p++) {
        const int m = bs.subPtr[p + 1] - bs.subPtr[p];
        tSize[p] = (int)touches[p].size();
        cOff[p] = cTotal;
        lOff[p] = lTotal;
        cTotal += int64_t(m) * tSize[p];
        lTotal += int64_t(tSize[p]) * tSize[p];
      }
      std::vector<double> C(size_t(cTotal), 0.0), G, local;
#pragma omp parallel for schedule(dynamic, 4)
      for (int p = 0; p < bs.nSub; p++) {
        const int b0 = bs.subPtr[p], m = bs.subPtr[p + 1] - b0, t = tSize[p];
        const std::vector<int>& touch = touches[p];
        for (int a = 0; a < m; a++)
          for (int kk = bs.AIS.ptr[b0 + a]; kk < bs.AIS.ptr[b0 + a + 1]; kk++) {
            int c = int(std::lower_bound(touch.begin(), touch.end(), bs.AIS.col[kk]) - touch.begin());
            C[size_t(cOff[p]) + size_t(a) * t + c] = bs.AIS.val[kk];
          }
      }
      std::vector<int64_t> invOff(bs.invOff.begin(), bs.invOff.end() - 1);
      if (!dense->schur_products(bs.inv, invOff, subSize, C, cOff, tSize, G, local, lOff, err)) return false;
      for (int p = 0; p < bs.nSub; p++) {
        const int m = bs.subPtr[p + 1] - bs.subPtr[p], t = tSize[p];
        double* Wp = &bs.W[size_t(bs.wOff[p])];
        for (int a = 0; a < m; a++)
          for (int c = 0; c < t; c++) Wp[size_t(c) * m + a] = G[size_t(cOff[p]) + size_t(a) * t + c];
        contrib[p].assign(local.begin() + lOff[p], local.begin() + lOff[p] + int64_t(t) * t);
      }
    } else
#pragma omp parallel
    {
#pragma omp for schedule(dynamic, 1)
      for (int p = 0; p < bs.nSub; p++) {
        const int b0 = bs.subPtr[p], m = bs.subPtr[p + 1] - b0;
        const std::vector<int>& touch = touches[p];
        const int t = (int)touch.size();
        if (!t) continue;
        // C = A_IS restricted (m x t), then G = Inv C, contribution C^T G
        std::vector<double> C(size_t(m) * t, 0.0), G(size_t(m) * t, 0.0);
        for (int a = 0; a < m; a++)
          for (int kk = bs.AIS.ptr[b0 + a]; kk < bs.AIS.ptr[b0 + a + 1]; kk++) {
            int c = int(std::lower_bound(touch.begin(), touch.end(), bs.AIS.col[kk]) - touch.begin());
            C[size_t(a) * t + c] = bs.AIS.val[kk];
          }
        const double* Inv = &bs.inv[size_t(bs.invOff[p])];
        for (int a = 0; a < m; a++)
          for (int q = 0; q < m; q++) {
            double w = Inv[size_t(a) * m + q];
            if (w == 0.0) continue;
            const double* cq = &C[size_t(q) * t];
            double* ga = &G[size_t(a) * t];
            for (int c = 0; c < t; c++) ga[c] += w * cq[c];
          }
        double* Wp = &bs.W[size_t(bs.wOff[p])];
        for (int a = 0; a < m; a++)
          for (int c = 0; c < t; c++) Wp[size_t(c) * m + a] = G[size_t(a) * t + c];
        std::vector<double>& local = contrib[p];
        local.assign(size_t(t) * t, 0.0);
        for (int a = 0; a < m; a++)
          for (int c1 = 0; c1 < t; c1++) {
            double cv = C[size_t(a) * t + c1];
            if (cv == 0.0) continue;
            for (int c2 = 0; c2 < t; c2++) local[size_t(c1) * t + c2] += cv * G[size_t(a) * t + c2];
          }
      }
    }
    for (int p = 0; p < bs.nSub; p++) {
      const std::vector<int>& touch = touches[p];
      const int t = (int)touch.size();
      for (int c1 = 0; c1 < t; c1++)
        for (int c2 = 0; c2 < t; c2++) bs.Sinv[size_t(touch[c1]) * nS + touch[c2]] -= contrib[p][size_t(c1) * t + c2];
    }
    // symmetrise against rounding, then invert
    lap(2);
    for (int a = 0; a < nS; a++)
      for (int c = 0; c < a; c++) {
        double v = 0.5 * (bs.Sinv[size_t(a) * nS + c] + bs.Sinv[size_t(c) * nS + a]);
        bs.Sinv[size_t(a) * nS + c] = bs.Sinv[size_t(c) * nS + a] = v;
      }
    const bool inverted = dense ? dense->spd_inverse_batched(bs.Sinv.data(), std::vector<int64_t>(1, 0), std::vector<int>(1, nS), err)
                                : dense_spd_inverse(bs.Sinv.data(), nS, true);
    if (!inverted) { err = "boundary Schur complement is not positive definite" + (err.empty() ? std::string() : ": " + err); return false; }
    lap(3);
  }
  // ---- boundary-deep coupling rows in solver order (unscaled, global texel columns)
  std::vector<Triplet> tBD;
  for (int k = 0; k < nb; k++) {
    int i = bs.order[k];
    for (int kk = BD.ptr[i]; kk < BD.ptr[i + 1]; kk++) tBD.push_back({k, BD.col[kk], BD.val[kk]});
  }
  bs.BD = csr_from_triplets(nb, BD.cols, tBD);
  lap(0);
  return true;
}

bool build_boundary_symbolic(const Csr& BB, const Csr& BD, int maxBlock, int denseMax, BoundarySymbolic& sym, std::string& err) {
  const int nb = BB.rows;
  sym = BoundarySymbolic();
  sym.nb = nb;
  if (nb == 0) return true;
  sym.bbRow.resize(BB.col.size());
  sym.diagEntry.assign(nb, -1);
  for (int i = 0; i < nb; i++)
    for (int k = BB.ptr[i]; k < BB.ptr[i + 1]; k++) {
      sym.bbRow[k] = i;
      if (BB.col[k] == i) sym.diagEntry[i] = k;
    }
  for (int i = 0; i < nb; i++)
    if (sym.diagEntry[i] < 0) { err = "boundary block has no diagonal entry"; return false; }
  partition_boundary(BB, maxBlock, denseMax, sym.order, sym.subPtr, sym.nI);
  sym.nSub = (int)sym.subPtr.size() - 1;
  sym.nS = nb - sym.nI;
  sym.pos.resize(nb);
  for (int k = 0; k < nb; k++) sym.pos[sym.order[k]] = k;
  std::vector<int> subOf(nb, -1);
  for (int p = 0; p < sym.nSub; p++)
    for (int k = sym.subPtr[p]; k < sym.subPtr[p + 1]; k++) subOf[k] = p;
  // subdomain blocks (row-major m x m per subdomain) and the separator block
  sym.invOff.assign(sym.nSub + 1, 0);
  for (int p = 0; p < sym.nSub; p++) {
    const int64_t m = sym.subPtr[p + 1] - sym.subPtr[p];
    sym.invOff[p + 1] = sym.invOff[p] + m * m;
  }
  // entries between interior and separator rows: AIS (interior rows), with the
  // BB entry in place of the value
  std::vector<Triplet> tIS;
  for (int i = 0; i < nb; i++)
    for (int k = BB.ptr[i]; k < BB.ptr[i + 1]; k++) {
      const int a = sym.pos[i], c = sym.pos[BB.col[k]];
      if (a < sym.nI && c < sym.nI) {
        const int p = subOf[a];
        if (subOf[c] != p) continue;  // no coupling between different subdomains' interiors
        const int b0 = sym.subPtr[p], m = sym.subPtr[p + 1] - b0;
        sym.fillEntry.push_back(k);
        sym.fillDest.push_back(sym.invOff[p] + int64_t(a - b0) * m + (c - b0));
      } else if (a < sym.nI) {
        tIS.push_back({a, c - sym.nI, double(k)});
      } else if (c >= sym.nI) {
        sym.ssEntry.push_back(k);
        sym.ssDest.push_back(int64_t(a - sym.nI) * sym.nS + (c - sym.nI));
      }
    }
  sym.AIS = csr_from_triplets(sym.nI, sym.nS, tIS);
  sym.ASI = csr_transpose(sym.AIS);
  // separator columns per subdomain, and the m x t blocks of C_p = A_{I_p,touch}
  sym.touchPtr.assign(sym.nSub + 1, 0);
  std::vector<std::vector<int>> touches(sym.nSub);
  for (int p = 0; p < sym.nSub; p++) {
    std::vector<int>& touch = touches[p];
    for (int a = sym.subPtr[p]; a < sym.subPtr[p + 1]; a++)
      for (int kk = sym.AIS.ptr[a]; kk < sym.AIS.ptr[a + 1]; kk++) touch.push_back(sym.AIS.col[kk]);
    std::sort(touch.begin(), touch.end());
    touch.erase(std::unique(touch.begin(), touch.end()), touch.end());
    sym.touchPtr[p + 1] = sym.touchPtr[p] + (int)touch.size();
  }
  sym.wOff.assign(sym.nSub + 1, 0);
  sym.lOff.assign(sym.nSub + 1, 0);
  for (int p = 0; p < sym.nSub; p++) {
    const int64_t m = sym.subPtr[p + 1] - sym.subPtr[p], t = (int64_t)touches[p].size();
    sym.wOff[p + 1] = sym.wOff[p] + m * t;
    sym.lOff[p + 1] = sym.lOff[p] + t * t;
    sym.touch.insert(sym.touch.end(), touches[p].begin(), touches[p].end());
  }
  sym.aisDest.resize(sym.AIS.col.size());
  for (int p = 0; p < sym.nSub; p++) {
    const int b0 = sym.subPtr[p];
    const std::vector<int>& touch = touches[p];
    const int t = (int)touch.size();
    for (int a = b0; a < sym.subPtr[p + 1]; a++)
      for (int kk = sym.AIS.ptr[a]; kk < sym.AIS.ptr[a + 1]; kk++) {
        const int c = int(std::lower_bound(touch.begin(), touch.end(), sym.AIS.col[kk]) - touch.begin());
        sym.aisDest[kk] = sym.wOff[p] + int64_t(a - b0) * t + c;
      }
  }
  // boundary-deep rows in solver order, with the BD entry in place of the value
  std::vector<Triplet> tBD;
  for (int k = 0; k < nb; k++) {
    const int i = sym.order[k];
    for (int kk = BD.ptr[i]; kk < BD.ptr[i + 1]; kk++) tBD.push_back({k, BD.col[kk], double(kk)});
  }
  sym.BD = csr_from_triplets(nb, BD.cols, tBD);
  return true;
}

}  // namespace gdtp
