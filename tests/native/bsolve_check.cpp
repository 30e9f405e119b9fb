// The exact boundary-block solve's set-up (csrc/setup/bsolve.cpp) applied on the
// host: x = BB^-1 r through the subdomain inverses, the separator's Schur
// complement and the back substitution, the same sequence as the device
// kernels (k_bs_prep, k_bs_dense, k_bs_back).  The test feeds it boundary blocks
// of the reference's own operator and checks the residual BB x - r.  It also
// checks that build_boundary_symbolic (the device numeric set-up's layout)
// gives the host set-up's partition, patterns and scaled couplings.
//
//   bsolve_check <in.bin> <out.bin>
//
// in.bin: CSR BB (int64 rows, cols, nnz + int32 ptr, int32 col, float64 val),
// int64 n + n float64 right-hand side.  out.bin: n float64 solution.
#include <cmath>
#include <cstdint>
#include <cstdio>
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

bool read_csr(std::ifstream& f, Csr& c) {
  int64_t h[3];
  if (!rd(f, h, 3)) return false;
  c.rows = int(h[0]), c.cols = int(h[1]);
  c.ptr.resize(size_t(h[0]) + 1), c.col.resize(size_t(h[2])), c.val.resize(size_t(h[2]));
  return rd(f, c.ptr.data(), c.ptr.size()) && rd(f, c.col.data(), c.col.size()) && rd(f, c.val.data(), c.val.size());
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) { std::fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]); return 2; }
  std::ifstream fin(argv[1], std::ios::binary);
  Csr BB;
  int64_t n = 0;
  if (!read_csr(fin, BB) || !rd(fin, &n, 1) || n != BB.rows) { std::fprintf(stderr, "bad input\n"); return 2; }
  std::vector<double> r(static_cast<size_t>(n));
  if (!rd(fin, r.data(), r.size())) return 2;
  Csr BD;  // no deep couplings: the deep iterate is zero
  BD.rows = BB.rows, BD.cols = 1, BD.ptr.assign(size_t(BB.rows) + 1, 0);
  BoundarySolverSetup bs;
  std::string err;
  if (!build_boundary_solver(BB, BD, 384, 0, bs, err)) { std::fprintf(stderr, "%s\n", err.c_str()); return 3; }
  // the device numeric set-up lays the solver out from build_boundary_symbolic:
  // the same partition and patterns, and values made from the recorded entries
  // (scaled BB entry k of rows i, j: (BB_k s_pos(i)) s_pos(j)) equal to the
  // host set-up's bit for bit
  {
    BoundarySymbolic sym;
    if (!build_boundary_symbolic(BB, BD, 384, 0, sym, err)) { std::fprintf(stderr, "symbolic: %s\n", err.c_str()); return 3; }
    auto scaled = [&](int e) { return BB.val[e] * bs.scale[sym.pos[sym.bbRow[e]]] * bs.scale[sym.pos[BB.col[e]]]; };
    bool same = sym.nb == bs.nb && sym.nSub == bs.nSub && sym.nI == bs.nI && sym.nS == bs.nS && sym.order == bs.order &&
                sym.subPtr == bs.subPtr && sym.touchPtr == bs.touchPtr && sym.touch == bs.touch && sym.wOff == bs.wOff &&
                sym.invOff == bs.invOff && sym.AIS.ptr == bs.AIS.ptr && sym.AIS.col == bs.AIS.col && sym.ASI.ptr == bs.ASI.ptr &&
                sym.ASI.col == bs.ASI.col && sym.BD.ptr == bs.BD.ptr && sym.BD.col == bs.BD.col;
    for (size_t k = 0; same && k < sym.AIS.val.size(); k++) same = scaled(int(sym.AIS.val[k])) == bs.AIS.val[k];
    for (size_t k = 0; same && k < sym.ASI.val.size(); k++) same = scaled(int(sym.ASI.val[k])) == bs.ASI.val[k];
    for (int k = 0; same && k < bs.nb; k++) same = 1.0 / std::sqrt(BB.val[sym.diagEntry[bs.order[k]]]) == bs.scale[k];
    if (!same) { std::fprintf(stderr, "symbolic layout differs from the host set-up\n"); return 4; }
  }
  // scaled right-hand side by position
  std::vector<double> rhat(bs.nb), y(bs.nI, 0.0), xs(bs.nS, 0.0), x(static_cast<size_t>(n), 0.0);
  for (int k = 0; k < bs.nb; k++) rhat[k] = bs.scale[k] * r[bs.order[k]];
  // interior: y = Inv_p rhat_I per subdomain
  for (int p = 0; p < bs.nSub; p++) {
    const int r0 = bs.subPtr[p], m = bs.subPtr[p + 1] - r0;
    const double* inv = bs.inv.data() + bs.invOff[p];
    for (int i = 0; i < m; i++) {
      double acc = 0;
      for (int j = 0; j < m; j++) acc += inv[size_t(i) * m + j] * rhat[r0 + j];
      y[r0 + i] = acc;
    }
  }
  // separator: xs = Sinv (rhat_S - A_SI y); x_S = s xs
  std::vector<double> t(bs.nS);
  for (int j = 0; j < bs.nS; j++) {
    double acc = 0;
    for (int e = bs.ASI.ptr[j]; e < bs.ASI.ptr[j + 1]; e++) acc += bs.ASI.val[e] * y[bs.ASI.col[e]];
    t[j] = rhat[bs.nI + j] - acc;
  }
  for (int i = 0; i < bs.nS; i++) {
    double acc = 0;
    for (int j = 0; j < bs.nS; j++) acc += bs.Sinv[size_t(i) * bs.nS + j] * t[j];
    xs[i] = acc;
    x[bs.order[bs.nI + i]] = bs.scale[bs.nI + i] * acc;
  }
  // back substitution: x_I = s (y - W_p xs[touch_p]), W_p column-major m x t
  for (int p = 0; p < bs.nSub; p++) {
    const int r0 = bs.subPtr[p], m = bs.subPtr[p + 1] - r0;
    const double* W = bs.W.data() + bs.wOff[p];
    for (int i = 0; i < m; i++) {
      double acc = y[r0 + i];
      for (int a = bs.touchPtr[p], c = 0; a < bs.touchPtr[p + 1]; a++, c++) acc -= W[size_t(c) * m + i] * xs[bs.touch[a]];
      x[bs.order[r0 + i]] = bs.scale[r0 + i] * acc;
    }
  }
  std::ofstream fo(argv[2], std::ios::binary);
  fo.write(reinterpret_cast<const char*>(x.data()), std::streamsize(x.size() * sizeof(double)));
  std::printf("ok nb=%d subdomains=%d interior=%d separator=%d\n", bs.nb, bs.nSub, bs.nI, bs.nS);
  return 0;
}
