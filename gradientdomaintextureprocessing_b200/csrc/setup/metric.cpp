// Per-triangle metrics that drive the assembly.
//
// A surface metric is a 2x2 SPD matrix per mesh triangle expressed in the basis
// of the triangle's edges (p1 - p0, p2 - p0); the assembly consumes its pull-back
// to texture coordinates (the parameter metric).  Restated from the reference:
//   embedding metric      InitializeEmbeddingMetric    include/Src/Metric.inl:248-275
//   uniform metric        InitializeUniformMetric      include/Src/Metric.inl:277-303
//   tangent-field metric  InitializeVectorFieldMetric  include/Src/Metric.inl:12-67
//   parameter metric      InitializeParameterMetric    include/Src/Metric.inl:415-446
// Matrices use the column-major M2 of setup.h (c[column][row]).
#include <cmath>

#include "setup.h"

namespace gdtp {

static void normalise_by_area(std::vector<M2>& G, double total) {
  for (M2& g : G)
    for (int k = 0; k < 2; k++)
      for (int l = 0; l < 2; l++) g.c[k][l] /= total;
}

bool surface_metric(const Mesh& mesh, int mode, bool normalizeArea, std::vector<M2>& G) {
  const int nt = mesh.nt();
  G.assign(nt, M2());
  double total = 0;
  for (int t = 0; t < nt; t++) {
    double d[2][3] = {{0, 0, 0}, {0, 0, 0}};
    int dims = 3;
    if (mode == 0) {  // edges in space
      const double* p0 = &mesh.vertices[3 * size_t(mesh.triangles[3 * t])];
      for (int e = 0; e < 2; e++) {
        const double* p = &mesh.vertices[3 * size_t(mesh.triangles[3 * t + 1 + e])];
        for (int k = 0; k < 3; k++) d[e][k] = p[k] - p0[k];
      }
    } else {  // edges in texture space
      dims = 2;
      const V2 q0 = mesh.corner(t, 0);
      for (int e = 0; e < 2; e++) {
        const V2 q = mesh.corner(t, 1 + e);
        d[e][0] = q.x - q0.x;
        d[e][1] = q.y - q0.y;
      }
    }
    M2& g = G[t];
    for (int k = 0; k < 2; k++)
      for (int l = 0; l < 2; l++) {
        double s = 0;
        for (int j = 0; j < dims; j++) s += d[k][j] * d[l][j];
        g.c[k][l] = s;
      }
    total += std::sqrt(g.det()) / 2;
  }
  if (normalizeArea) {
    if (!(total > 0)) return false;
    normalise_by_area(G, total);
  }
  return true;
}

bool vector_field_metric(const std::vector<M2>& G, const double* vf, double across, double isotropic, bool normalizeArea,
                         std::vector<M2>& out) {
  const size_t nt = G.size();
  out.assign(nt, M2());
  double total = 0;
  for (size_t t = 0; t < nt; t++) {
    const M2& g = G[t];
    const V2 v0(vf[2 * t], vf[2 * t + 1]);
    const V2 gv0 = g * v0;
    const double n0 = v0.x * gv0.x + v0.y * gv0.y;
    M2 u;  // zero when the field vanishes on the triangle
    if (n0 > 0) {
      // frame: the field and its g-orthogonal complement, both of unit g-length
      V2 e[2] = {v0, V2(-gv0.y, gv0.x)};
      for (int k = 0; k < 2; k++) {
        const V2 ge = g * e[k];
        const double len = std::sqrt(e[k].x * ge.x + e[k].y * ge.y);
        e[k] = V2(e[k].x / len, e[k].y / len);
      }
      M2 B, D;
      B.c[0][0] = e[0].x; B.c[0][1] = e[0].y;  // column 0 = field direction
      B.c[1][0] = e[1].x; B.c[1][1] = e[1].y;  // column 1 = across the field
      D.c[1][1] = across;                       // the metric vanishes along the field (before the isotropic term)
      u = ((g * B) * D) * B.inverse();
    }
    M2& o = out[t];
    for (int k = 0; k < 2; k++)
      for (int l = 0; l < 2; l++) o.c[k][l] = u.c[k][l] + g.c[k][l] * isotropic;
    total += std::sqrt(o.det()) / 2;
  }
  if (normalizeArea) {
    if (!(total > 0)) return false;
    normalise_by_area(out, total);
  }
  return true;
}

bool parameter_metric(const Mesh& mesh, const std::vector<M2>& G, std::vector<M2>& out) {
  const int nt = mesh.nt();
  out.assign(nt, M2());
  for (int t = 0; t < nt; t++) {
    const V2 q0 = mesh.corner(t, 0), q1 = mesh.corner(t, 1), q2 = mesh.corner(t, 2);
    M2 J;  // columns: texture-space edges
    J.c[0][0] = q1.x - q0.x; J.c[0][1] = q1.y - q0.y;
    J.c[1][0] = q2.x - q0.x; J.c[1][1] = q2.y - q0.y;
    if (J.det() == 0) return false;
    const M2 Ji = J.inverse();
    out[t] = (Ji.transpose() * G[t]) * Ji;
  }
  return true;
}

}  // namespace gdtp
