// Compressed sparse rows with sorted, duplicate-free columns: the host form of
// the reference's SparseMatrix<double,int> after SparseMatrixParser
// (Src/SparseMatrixParser.h:77-115 sorts each row and sums duplicates).
#include <algorithm>
#include <cstdint>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "setup.h"

namespace gdtp {

// Rows by a stable counting sort, each row's entries by a stable sort of its
// columns (rows in parallel), duplicates summed in input order: the same sums,
// term for term, as one stable sort of all entries by (row, column).  nv value
// sets share the pattern.
static void from_pairs(int rows, int cols, size_t n, const int* R, const int* Cc, int nv, const double* const* V, Csr* out) {
  std::vector<size_t> start(size_t(rows) + 1, 0);
  for (size_t i = 0; i < n; i++) start[size_t(R[i]) + 1]++;
  for (int r = 0; r < rows; r++) start[r + 1] += start[r];
  std::vector<size_t> ord(n);  // entries grouped by row, input order within a row
  {
    std::vector<size_t> fill(start.begin(), start.end() - 1);
    for (size_t i = 0; i < n; i++) ord[fill[R[i]]++] = i;
  }
  std::vector<int> distinct(size_t(rows) + 1, 0);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int r = 0; r < rows; r++) {
    size_t* b = ord.data() + start[r];
    size_t* e = ord.data() + start[r + 1];
    if (e - b <= 32) {
      for (size_t* i = b + 1; i < e; i++) {
        const size_t v = *i;
        size_t* j = i;
        while (j > b && Cc[*(j - 1)] > Cc[v]) { *j = *(j - 1); j--; }
        *j = v;
      }
    } else {
      std::stable_sort(b, e, [&](size_t x, size_t y) { return Cc[x] < Cc[y]; });
    }
    int d = 0;
    for (size_t* i = b; i < e; i++)
      if (i == b || Cc[*i] != Cc[*(i - 1)]) d++;
    distinct[r + 1] = d;
  }
  Csr& m = out[0];
  m.rows = rows;
  m.cols = cols;
  m.ptr.assign(rows + 1, 0);
  for (int r = 0; r < rows; r++) m.ptr[r + 1] = m.ptr[r] + distinct[r + 1];
  m.col.resize(m.ptr[rows]);
  for (int q = 0; q < nv; q++) out[q].val.assign(m.ptr[rows], 0.0);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int r = 0; r < rows; r++) {
    int o = m.ptr[r] - 1;
    for (size_t i = start[r]; i < start[r + 1]; i++) {
      const size_t k = ord[i];
      if (i == start[r] || Cc[k] != Cc[ord[i - 1]]) m.col[++o] = Cc[k];
      for (int q = 0; q < nv; q++) out[q].val[o] += V[q][k];
    }
  }
  for (int q = 1; q < nv; q++) {
    out[q].rows = rows;
    out[q].cols = cols;
    out[q].ptr = m.ptr;
    out[q].col = m.col;
  }
}

Csr csr_from_triplets(int rows, int cols, std::vector<Triplet>& t) {
  const size_t n = t.size();
  std::vector<int> R(n), Cc(n);
  std::vector<double> V(n);
  for (size_t i = 0; i < n; i++) {
    R[i] = t[i].r;
    Cc[i] = t[i].c;
    V[i] = t[i].v;
  }
  const double* vs[1] = {V.data()};
  Csr m;
  from_pairs(rows, cols, n, R.data(), Cc.data(), 1, vs, &m);
  return m;
}

void csr_from_pairs(int rows, int cols, const std::vector<int>& r, const std::vector<int>& c, const std::vector<double>& v1,
                    const std::vector<double>& v2, Csr& m1, Csr& m2) {
  const double* vs[2] = {v1.data(), v2.data()};
  Csr out[2];
  from_pairs(rows, cols, r.size(), r.data(), c.data(), 2, vs, out);
  m1 = std::move(out[0]);
  m2 = std::move(out[1]);
}

Csr csr_transpose(const Csr& a) {
  Csr t;
  t.rows = a.cols;
  t.cols = a.rows;
  t.ptr.assign(a.cols + 1, 0);
  for (int c : a.col) t.ptr[c + 1]++;
  for (int r = 0; r < a.cols; r++) t.ptr[r + 1] += t.ptr[r];
  t.col.resize(a.col.size());
  t.val.resize(a.val.size());
  std::vector<int> fill(t.ptr.begin(), t.ptr.end() - 1);
  for (int r = 0; r < a.rows; r++)
    for (int k = a.ptr[r]; k < a.ptr[r + 1]; k++) {
      int p = fill[a.col[k]]++;
      t.col[p] = r;
      t.val[p] = a.val[k];
    }
  return t;
}

// Row by row (rows in parallel chunks, concatenated in row order); each row's
// products accumulate in the order of a's entries, then b's.  A second value
// set (a2 for a's pattern, b2 for b's) gives a second product on the same
// pattern, each value as the one-set product would compute it.
static void multiply(const Csr& a, const double* a2, const Csr& b, const double* b2, Csr& c, std::vector<double>* c2) {
  c = Csr();
  c.rows = a.rows;
  c.cols = b.cols;
  c.ptr.assign(a.rows + 1, 0);
  int nChunks = 1;
#ifdef _OPENMP
  nChunks = std::max(1, std::min(omp_get_max_threads() * 4, a.rows / 256));
#endif
  std::vector<std::vector<int>> chunkCol(nChunks);
  std::vector<std::vector<double>> chunkVal(nChunks), chunkVal2(nChunks);
#pragma omp parallel
  {
    std::vector<double> acc(b.cols, 0.0), acc2(c2 ? b.cols : 0, 0.0);
    std::vector<int> mark(b.cols, -1), cols;
#pragma omp for schedule(dynamic, 1)
    for (int q = 0; q < nChunks; q++) {
      const int r0 = int(int64_t(a.rows) * q / nChunks), r1 = int(int64_t(a.rows) * (q + 1) / nChunks);
      std::vector<int>& oc = chunkCol[q];
      std::vector<double>& ov = chunkVal[q];
      std::vector<double>& ov2 = chunkVal2[q];
      for (int r = r0; r < r1; r++) {
        cols.clear();
        for (int k = a.ptr[r]; k < a.ptr[r + 1]; k++) {
          const int m = a.col[k];
          const double av = a.val[k], av2 = a2 ? a2[k] : av;
          for (int p = b.ptr[m]; p < b.ptr[m + 1]; p++) {
            const int j = b.col[p];
            if (mark[j] != r) {
              mark[j] = r;
              acc[j] = 0.0;
              if (c2) acc2[j] = 0.0;
              cols.push_back(j);
            }
            acc[j] += av * b.val[p];
            if (c2) acc2[j] += av2 * (b2 ? b2[p] : b.val[p]);
          }
        }
        std::sort(cols.begin(), cols.end());
        for (int j : cols) {
          oc.push_back(j);
          ov.push_back(acc[j]);
          if (c2) ov2.push_back(acc2[j]);
        }
        c.ptr[r + 1] = (int)cols.size();
      }
    }
  }
  for (int r = 0; r < a.rows; r++) c.ptr[r + 1] += c.ptr[r];
  c.col.reserve(c.ptr[a.rows]);
  c.val.reserve(c.ptr[a.rows]);
  if (c2) {
    c2->clear();
    c2->reserve(c.ptr[a.rows]);
  }
  for (int q = 0; q < nChunks; q++) {
    c.col.insert(c.col.end(), chunkCol[q].begin(), chunkCol[q].end());
    c.val.insert(c.val.end(), chunkVal[q].begin(), chunkVal[q].end());
    if (c2) c2->insert(c2->end(), chunkVal2[q].begin(), chunkVal2[q].end());
  }
}

Csr csr_multiply(const Csr& a, const Csr& b) {
  Csr c;
  multiply(a, nullptr, b, nullptr, c, nullptr);
  return c;
}

void csr_multiply2(const Csr& a, const std::vector<double>* a2, const Csr& b, const std::vector<double>* b2, Csr& c1, Csr& c2) {
  std::vector<double> v2;
  multiply(a, a2 ? a2->data() : nullptr, b, b2 ? b2->data() : nullptr, c1, &v2);
  c2.rows = c1.rows;
  c2.cols = c1.cols;
  c2.ptr = c1.ptr;
  c2.col = c1.col;
  c2.val = std::move(v2);
}

Csr csr_axpby(double a, const Csr& A, double b, const Csr& B) {
  Csr c;
  c.rows = A.rows;
  c.cols = std::max(A.cols, B.cols);
  c.ptr.assign(A.rows + 1, 0);
  for (int r = 0; r < A.rows; r++) {
    int i = A.ptr[r], j = B.ptr[r];
    while (i < A.ptr[r + 1] || j < B.ptr[r + 1]) {
      int ca = i < A.ptr[r + 1] ? A.col[i] : 0x7fffffff;
      int cb = j < B.ptr[r + 1] ? B.col[j] : 0x7fffffff;
      if (ca == cb) { c.col.push_back(ca); c.val.push_back(a * A.val[i++] + b * B.val[j++]); }
      else if (ca < cb) { c.col.push_back(ca); c.val.push_back(a * A.val[i++]); }
      else { c.col.push_back(cb); c.val.push_back(b * B.val[j++]); }
    }
    c.ptr[r + 1] = (int)c.col.size();
  }
  return c;
}

}  // namespace gdtp
