// The CSR builders of the set-up (rows in parallel; one or two value sets on
// a shared pattern) against a serial restatement: one stable sort of the
// triplets by (row, column) with duplicates summed in input order, and a
// row-by-row sparse product.  Every array must agree bit for bit.
#include <algorithm>
#include <cstdio>
#include <random>
#include "setup/setup.h"
using namespace gdtp;
static Csr ref_from_triplets(int rows, int cols, std::vector<Triplet> t) {
  std::stable_sort(t.begin(), t.end(), [](const Triplet& a, const Triplet& b) { return a.r != b.r ? a.r < b.r : a.c < b.c; });
  Csr m; m.rows = rows; m.cols = cols; m.ptr.assign(rows + 1, 0); size_t i = 0;
  for (int r = 0; r < rows; r++) { while (i < t.size() && t[i].r == r) { int c = t[i].c; double v = 0; while (i < t.size() && t[i].r == r && t[i].c == c) v += t[i++].v; m.col.push_back(c); m.val.push_back(v);} m.ptr[r + 1] = (int)m.col.size(); }
  return m;
}
int main() {
  std::mt19937 g(1);
  for (int trial = 0; trial < 20; trial++) {
    int rows = 1 + g() % 5000, cols = 1 + g() % 3000; size_t n = g() % 200000;
    std::vector<Triplet> t(n);
    for (auto& e : t) { e.r = g() % rows; e.c = g() % (trial % 2 ? 8 : cols); e.v = std::uniform_real_distribution<double>(-1, 1)(g); }
    Csr a = ref_from_triplets(rows, cols, t);
    std::vector<Triplet> t2 = t; Csr b = csr_from_triplets(rows, cols, t2);
    if (a.ptr != b.ptr || a.col != b.col || a.val != b.val) { printf("triplets mismatch %d\n", trial); return 1; }
    Csr bt = csr_transpose(b);
    Csr p1 = csr_multiply(b, bt);
    // serial reference product
    Csr p0; p0.rows = b.rows; p0.cols = bt.cols; p0.ptr.assign(b.rows + 1, 0);
    std::vector<double> acc(bt.cols, 0.0); std::vector<int> mark(bt.cols, -1), cl;
    for (int r = 0; r < b.rows; r++) { cl.clear(); for (int k = b.ptr[r]; k < b.ptr[r + 1]; k++) { int m = b.col[k]; double av = b.val[k]; for (int q = bt.ptr[m]; q < bt.ptr[m + 1]; q++) { int j = bt.col[q]; if (mark[j] != r) { mark[j] = r; acc[j] = 0; cl.push_back(j);} acc[j] += av * bt.val[q]; } } std::sort(cl.begin(), cl.end()); for (int j : cl) { p0.col.push_back(j); p0.val.push_back(acc[j]); } p0.ptr[r + 1] = (int)p0.col.size(); }
    if (p0.ptr != p1.ptr || p0.col != p1.col || p0.val != p1.val) { printf("multiply mismatch %d\n", trial); return 1; }
    // two value sets on one pattern
    std::vector<int> rr(n), cc(n);
    std::vector<double> v1(n), v2(n);
    std::vector<Triplet> t3 = t;
    for (size_t i = 0; i < n; i++) { rr[i] = t[i].r; cc[i] = t[i].c; v1[i] = t[i].v; v2[i] = std::uniform_real_distribution<double>(-1, 1)(g); t3[i].v = v2[i]; }
    Csr m1, m2;
    csr_from_pairs(rows, cols, rr, cc, v1, v2, m1, m2);
    Csr r2 = ref_from_triplets(rows, cols, t3);
    if (m1.ptr != a.ptr || m1.col != a.col || m1.val != a.val || m2.ptr != r2.ptr || m2.col != r2.col || m2.val != r2.val) {
      printf("pairs mismatch %d\n", trial);
      return 1;
    }
    Csr q1, q2;
    csr_multiply2(b, &r2.val, bt, nullptr, q1, q2);
    Csr q2ref = csr_multiply(r2, bt);
    if (q1.ptr != p0.ptr || q1.col != p0.col || q1.val != p0.val || q2.ptr != q2ref.ptr || q2.col != q2ref.col || q2.val != q2ref.val) {
      printf("multiply2 mismatch %d\n", trial);
      return 1;
    }
  }
  printf("ok\n");
  return 0;
}
