// Dense SPD inverse used for the coarsest level and the boundary blocks:
// A * inv(A) = I to 1e-12 and inv(A) symmetric, for sizes that end in a
// partial block of 4 and for the parallel path; an indefinite matrix is
// rejected.  Prints "ok".
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "setup/setup.h"

static bool check(int n, bool parallel) {
  std::mt19937 rng(n);
  std::uniform_real_distribution<double> u(-1, 1);
  std::vector<double> B(size_t(n) * n), A(size_t(n) * n);
  for (auto& v : B) v = u(rng);
  for (int i = 0; i < n; i++)
    for (int j = 0; j <= i; j++) {
      double s = 0;
      for (int k = 0; k < n; k++) s += B[size_t(i) * n + k] * B[size_t(j) * n + k];
      A[size_t(i) * n + j] = A[size_t(j) * n + i] = s / n + (i == j ? 0.5 : 0.0);
    }
  std::vector<double> X = A;
  if (!gdtp::dense_spd_inverse(X.data(), n, parallel)) { printf("n=%d: rejected an SPD matrix\n", n); return false; }
  double err = 0, asym = 0;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      double s = 0;
      for (int k = 0; k < n; k++) s += A[size_t(i) * n + k] * X[size_t(k) * n + j];
      err = std::fmax(err, std::fabs(s - (i == j ? 1.0 : 0.0)));
      asym = std::fmax(asym, std::fabs(X[size_t(i) * n + j] - X[size_t(j) * n + i]));
    }
  if (err > 1e-12 || asym != 0.0) { printf("n=%d: |A X - I| = %g, asymmetry %g\n", n, err, asym); return false; }
  return true;
}

int main() {
  bool ok = true;
  for (int n : {1, 2, 3, 5, 8, 67, 384}) ok = check(n, false) && ok;
  ok = check(601, true) && ok;
  std::vector<double> indef = {1, 2, 2, 1};  // eigenvalues 3 and -1
  if (gdtp::dense_spd_inverse(indef.data(), 2, false)) { printf("accepted an indefinite matrix\n"); ok = false; }
  printf(ok ? "ok\n" : "failed\n");
  return ok ? 0 : 1;
}
