// Galerkin coarsening (csrc/setup/galerkin.cpp) driven from given fine
// coefficients: builds the texel hierarchy of a mesh, coarsens the fine operator
// and writes every level's coefficients.  The test feeds it the reference's own
// fine operator and compares the levels with the reference's coarse operators.
//
//   galerkin_check <mesh.gdm> <levels> <fine.bin> <out.bin>
//
// fine.bin / out.bin: int64 n + n float64 (deep, 10 per deep texel), then two CSR
// blocks (BB, BD) as int64 rows, cols, nnz + int32 ptr, int32 col, float64 val;
// out.bin repeats the three for every level.
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
void write_csr(std::ofstream& f, const Csr& c) {
  const int64_t h[3] = {c.rows, c.cols, int64_t(c.col.size())};
  wr(f, h, 3);
  wr(f, c.ptr.data(), c.ptr.size());
  wr(f, c.col.data(), c.col.size());
  wr(f, c.val.data(), c.val.size());
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
  if (argc != 5) { std::fprintf(stderr, "usage: %s mesh.gdm levels fine.bin out.bin\n", argv[0]); return 2; }
  Mesh mesh;
  int width = 0, height = 0;
  if (!read_gdm(argv[1], mesh, width, height)) { std::fprintf(stderr, "cannot read %s\n", argv[1]); return 2; }
  const int levels = std::atoi(argv[2]);
  Hierarchy h;
  BlockInfo info;
  if (!build_hierarchy(mesh, width, height, levels, info, h, 0, levels)) { std::fprintf(stderr, "%s\n", h.error.c_str()); return 3; }
  std::ifstream fin(argv[3], std::ios::binary);
  int64_t n = 0;
  if (!rd(fin, &n, 1)) return 2;
  std::vector<double> deep0(static_cast<size_t>(n));
  Csr bb0, bd0;
  if (!rd(fin, deep0.data(), deep0.size()) || !read_csr(fin, bb0) || !read_csr(fin, bd0)) { std::fprintf(stderr, "bad %s\n", argv[3]); return 2; }
  std::vector<LevelCoefficients> out;
  std::string err;
  if (!galerkin_hierarchy(h, levels, deep0, bb0, bd0, out, err)) { std::fprintf(stderr, "%s\n", err.c_str()); return 3; }
  std::ofstream fo(argv[4], std::ios::binary);
  for (const LevelCoefficients& c : out) {
    const int64_t m = int64_t(c.deep.size());
    wr(fo, &m, 1);
    wr(fo, c.deep.data(), c.deep.size());
    write_csr(fo, c.bb);
    write_csr(fo, c.bd);
  }
  std::printf("ok %zu levels\n", out.size());
  return 0;
}
