// Compressed sparse rows with sorted, duplicate-free columns: the host form of
// the reference's SparseMatrix<double,int> after SparseMatrixParser
// (Src/SparseMatrixParser.h:77-115 sorts each row and sums duplicates).
#include <algorithm>

#include "setup.h"

namespace gdtp {

Csr csr_from_triplets(int rows, int cols, std::vector<Triplet>& t) {
  std::stable_sort(t.begin(), t.end(), [](const Triplet& a, const Triplet& b) { return a.r != b.r ? a.r < b.r : a.c < b.c; });
  Csr m;
  m.rows = rows;
  m.cols = cols;
  m.ptr.assign(rows + 1, 0);
  m.col.reserve(t.size());
  m.val.reserve(t.size());
  size_t i = 0;
  for (int r = 0; r < rows; r++) {
    while (i < t.size() && t[i].r == r) {
      int c = t[i].c;
      double v = 0;
      while (i < t.size() && t[i].r == r && t[i].c == c) v += t[i++].v;
      m.col.push_back(c);
      m.val.push_back(v);
    }
    m.ptr[r + 1] = (int)m.col.size();
  }
  return m;
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

Csr csr_multiply(const Csr& a, const Csr& b) {
  Csr c;
  c.rows = a.rows;
  c.cols = b.cols;
  c.ptr.assign(a.rows + 1, 0);
  std::vector<double> acc(b.cols, 0.0);
  std::vector<int> mark(b.cols, -1), cols;
  for (int r = 0; r < a.rows; r++) {
    cols.clear();
    for (int k = a.ptr[r]; k < a.ptr[r + 1]; k++) {
      int m = a.col[k];
      double av = a.val[k];
      for (int q = b.ptr[m]; q < b.ptr[m + 1]; q++) {
        int j = b.col[q];
        if (mark[j] != r) { mark[j] = r; acc[j] = 0.0; cols.push_back(j); }
        acc[j] += av * b.val[q];
      }
    }
    std::sort(cols.begin(), cols.end());
    for (int j : cols) { c.col.push_back(j); c.val.push_back(acc[j]); }
    c.ptr[r + 1] = (int)c.col.size();
  }
  return c;
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
