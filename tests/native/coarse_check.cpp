// The coarsest level's direct solve set-up on given coefficients: the full
// operator assembled by full_matrix (csrc/setup/galerkin.cpp) and its
// Jacobi-scaled dense inverse (dense_spd_inverse, csrc/setup/bsolve.cpp),
// applied to a right-hand side on the host.  The Jacobi scaling and the apply
// loop are restated here (the solver's own versions run on the device: the
// host build in system.cu, or the numeric set-up of numeric.cu, and
// k_coarse_solve); what this check pins is full_matrix and the dense inverse.
//
//   coarse_check <mesh.gdm> <levels> <in.bin> <out.bin>
//
// in.bin: the coarsest level's coefficients (int64 n + n float64 deep, 10 per
// deep texel; CSR BB; CSR BD, as int64 rows, cols, nnz + int32 ptr, int32 col,
// float64 val), then int64 m + m float64 right-hand side.  out.bin: the full
// operator as CSR, then m float64 solution.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "setup/setup.h"

using namespace gdtp;

namespace {

template <class T>
bool rd(std::ifstream& f, T* p, size_t n) {
  return bool(f.read(reinterpret_cast<char*>(p), std::streamsize(n * sizeof(T))));
}
template <class T>
void wr(std::ofstream& f, const T* p, size_t n) {
  f.write(reinterpret_cast<const char*>(p), std::streamsize(n * sizeof(T)));
}
bool read_csr(std::ifstream& f, Csr& c) {
  int64_t h[3];
  if (!rd(f, h, 3)) return false;
  c.rows = int(h[0]), c.cols = int(h[1]);
  c.ptr.resize(size_t(h[0]) + 1), c.col.resize(size_t(h[2])), c.val.resize(size_t(h[2]));
  return rd(f, c.ptr.data(), c.ptr.size()) && rd(f, c.col.data(), c.col.size()) && rd(f, c.val.data(), c.val.size());
}
bool read_gdm(const char* path, Mesh& m, int& width, int& height) {
  std::ifstream f(path, std::ios::binary);
  char magic[8];
  int64_t h[5];
  if (!rd(f, magic, 8) || !rd(f, h, 5)) return false;
  m.vertices.resize(size_t(h[0]) * 3), m.triangles.resize(size_t(h[1]) * 3), m.uv.resize(size_t(h[1]) * 6);
  width = int(h[2]), height = int(h[3]);
  return rd(f, m.vertices.data(), m.vertices.size()) && rd(f, m.triangles.data(), m.triangles.size()) &&
         rd(f, m.uv.data(), m.uv.size());
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 5) { std::fprintf(stderr, "usage: %s mesh.gdm levels in.bin out.bin\n", argv[0]); return 2; }
  Mesh mesh;
  int width = 0, height = 0;
  if (!read_gdm(argv[1], mesh, width, height)) return 2;
  const int levels = std::atoi(argv[2]);
  Hierarchy h;
  BlockInfo info;
  if (!build_hierarchy(mesh, width, height, levels, info, h, 0, levels)) { std::fprintf(stderr, "%s\n", h.error.c_str()); return 3; }
  std::ifstream fin(argv[3], std::ios::binary);
  LevelCoefficients c;
  int64_t n = 0, m = 0;
  if (!rd(fin, &n, 1)) return 2;
  c.deep.resize(static_cast<size_t>(n));
  if (!rd(fin, c.deep.data(), c.deep.size()) || !read_csr(fin, c.bb) || !read_csr(fin, c.bd) || !rd(fin, &m, 1)) return 2;
  std::vector<double> r(static_cast<size_t>(m));
  if (!rd(fin, r.data(), r.size())) return 2;
  Csr full;
  full_matrix(h.levels[levels - 1], c, full);
  if (full.rows != m) { std::fprintf(stderr, "size mismatch %d %lld\n", full.rows, (long long)m); return 3; }
  // Jacobi-scaled dense inverse: A = S^-1 (S A S) S^-1 with S = diag(A)^-1/2
  std::vector<double> s(static_cast<size_t>(m), 0.0), A(size_t(m) * size_t(m), 0.0);
  for (int i = 0; i < full.rows; i++)
    for (int k = full.ptr[i]; k < full.ptr[i + 1]; k++)
      if (full.col[k] == i) s[i] = 1.0 / std::sqrt(full.val[k]);
  for (int i = 0; i < full.rows; i++)
    for (int k = full.ptr[i]; k < full.ptr[i + 1]; k++) A[size_t(i) * m + full.col[k]] = s[i] * full.val[k] * s[full.col[k]];
  if (!dense_spd_inverse(A.data(), int(m), true)) { std::fprintf(stderr, "not positive definite\n"); return 3; }
  std::vector<double> x(static_cast<size_t>(m));
  for (int64_t i = 0; i < m; i++) {
    double acc = 0;
    for (int64_t j = 0; j < m; j++) acc += A[size_t(i) * m + j] * s[j] * r[j];
    x[i] = s[i] * acc;
  }
  std::ofstream fo(argv[4], std::ios::binary);
  const int64_t hdr[3] = {full.rows, full.cols, int64_t(full.col.size())};
  wr(fo, hdr, 3);
  wr(fo, full.ptr.data(), full.ptr.size());
  wr(fo, full.col.data(), full.col.size());
  wr(fo, full.val.data(), full.val.size());
  wr(fo, x.data(), x.size());
  std::printf("ok n=%lld\n", (long long)m);
  return 0;
}
