// FP64 element integrals shared by the assembly kernels.
//
// Interior cells (bilinear basis on one texel cell, MassAndStiffness.h:58-160):
//   the chart triangle is clipped to the cell (ClipTriangleToPrimalCell,
//   PolygonClipping.h:85-124), fan-triangulated, and each fan triangle is
//   integrated with the 6-point rule on the unit right triangle
//   (RightTriangleQuadrature.h:6-22).
// Boundary cells (quadratic basis on a boundary triangle, MassAndStiffness.h:160-280):
//   the boundary triangle is clipped to the chart triangle, fan-triangulated and
//   integrated the same way with the 6 quadratic shape functions of the boundary
//   triangle (Basis.h:54-106); each piece is symmetrised before accumulation.
// Both use the chart triangle's parameter metric g: mass density sqrt(det g),
// stiffness density sqrt(det g) * g^-1.
#pragma once
#include <math.h>

#ifdef __CUDACC__
#define GDTP_HD __host__ __device__ __forceinline__
#else
#define GDTP_HD inline
#endif

namespace gdtp {
namespace am {

struct P2 {
  double x, y;
};

GDTP_HD P2 mk(double x, double y) { P2 p; p.x = x; p.y = y; return p; }

// 6-point degree-4 rule on the unit right triangle (published Dunavant-type
// rule; positions in (s,t), weights summing to 1/2 * 2 = 1 with area factor 1/2 applied by callers)
GDTP_HD double qx(int s) {
  const double a = 0.816847572980459, b = 0.0915762135097705, c = 0.108103018168070, d = 0.445948490915965;
  switch (s) { case 0: return a; case 1: return b; case 2: return b; case 3: return c; case 4: return d; default: return d; }
}
GDTP_HD double qy(int s) {
  const double a = 0.816847572980459, b = 0.0915762135097705, c = 0.108103018168070, d = 0.445948490915965;
  switch (s) { case 0: return b; case 1: return a; case 2: return b; case 3: return d; case 4: return c; default: return d; }
}
GDTP_HD double qw(int s) { return s < 3 ? 0.109951743655322 : 0.223381589678011; }

// Sutherland-Hodgman step against the half-plane dot(p, n) - off > 0.
GDTP_HD int clip_half(const P2* in, int n, P2* out, double nx, double ny, double off) {
  if (n == 0) return 0;
  int m = 0;
  P2 prev = in[n - 1];
  double pl = prev.x * nx + prev.y * ny - off;
  bool pin = pl > 0;
  for (int i = 0; i < n; i++) {
    P2 cur = in[i];
    double cl = cur.x * nx + cur.y * ny - off;
    bool cin = cl > 0;
    if (cin) {
      if (!pin) {
        double a = -cl / (pl - cl);
        out[m++] = mk(prev.x * a + cur.x * (1.0 - a), prev.y * a + cur.y * (1.0 - a));
      }
      out[m++] = cur;
    } else if (pin) {
      double a = -cl / (pl - cl);
      out[m++] = mk(prev.x * a + cur.x * (1.0 - a), prev.y * a + cur.y * (1.0 - a));
    }
    prev = cur;
    pl = cl;
    pin = cin;
  }
  return m;
}

// Triangle (3 points) clipped to the texel cell [i,i+1]x[j,j+1] (in cell units
// cw, ch).  Up to 7 output vertices; buffers must hold 8.
GDTP_HD int clip_to_cell(P2* poly, int n, int i, int j, double cw, double ch, P2* tmp) {
  n = clip_half(poly, n, tmp, 0, 1, double(j) * ch);
  if (!n) return 0;
  n = clip_half(tmp, n, poly, 0, -1, -(double(j + 1) * ch));
  if (!n) return 0;
  n = clip_half(poly, n, tmp, 1, 0, double(i) * cw);
  if (!n) return 0;
  n = clip_half(tmp, n, poly, -1, 0, -(double(i + 1) * cw));
  return n;
}

// Convex polygon clipped to a triangle (inward normals from the centroid).
GDTP_HD int clip_to_triangle(P2* poly, int n, const P2* t, P2* tmp) {
  P2 c = mk((t[0].x + t[1].x + t[2].x) / 3.0, (t[0].y + t[1].y + t[2].y) / 3.0);
  for (int k = 0; k < 3 && n; k++) {
    P2 a = t[k], b = t[(k + 1) % 3];
    double dx = b.x - a.x, dy = b.y - a.y;
    double nx = -dy, ny = dx;
    double len = sqrt(nx * nx + ny * ny);
    nx /= len;
    ny /= len;
    double off = ((a.x + b.x) / 2.0) * nx + ((a.y + b.y) / 2.0) * ny;
    if (c.x * nx + c.y * ny < off) { nx = -nx; ny = -ny; off = -off; }
    n = clip_half(poly, n, tmp, nx, ny, off);
    for (int q = 0; q < n; q++) poly[q] = tmp[q];
  }
  return n;
}

GDTP_HD double bilinear(int k, double x, double y) {
  switch (k) { case 0: return (1.0 - x) * (1.0 - y); case 1: return x * (1.0 - y); case 2: return x * y; default: return (1.0 - x) * y; }
}
GDTP_HD P2 bilinear_grad(int k, double x, double y) {
  switch (k) { case 0: return mk(y - 1.0, x - 1.0); case 1: return mk(1.0 - y, -x); case 2: return mk(y, x); default: return mk(-y, 1.0 - x); }
}

// Adds the bilinear mass / stiffness of one clipped polygon of an interior cell.
// ginv: g^-1 column-major (c00, c01, c10, c11), scale: sqrt(det g).
// mass/stiff: 16 entries, row k (texel corner) col l.
GDTP_HD void integrate_cell_polygon(const P2* poly, int n, int i, int j, double cw, double ch, const double* ginv, double scale,
                                    double* mass, double* stiff) {
  double pm[16], ps[16];
  for (int q = 0; q < 16; q++) pm[q] = ps[q] = 0.0;
  for (int p = 2; p < n; p++) {
    P2 d0 = mk(poly[p - 1].x - poly[0].x, poly[p - 1].y - poly[0].y);
    P2 d1 = mk(poly[p].x - poly[0].x, poly[p].y - poly[0].y);
    double jac = fabs(d0.x * d1.y - d0.y * d1.x);
    double val[4][6];
    P2 grd[4][6];
    for (int s = 0; s < 6; s++) {
      double sx = (poly[0].x + d0.x * qx(s) + d1.x * qy(s)) / cw - double(i);
      double sy = (poly[0].y + d0.y * qx(s) + d1.y * qy(s)) / ch - double(j);
      for (int k = 0; k < 4; k++) {
        val[k][s] = bilinear(k, sx, sy);
        P2 g = bilinear_grad(k, sx, sy);
        grd[k][s] = mk(g.x / cw, g.y / ch);
      }
    }
    for (int k = 0; k < 4; k++)
      for (int l = 0; l < 4; l++) {
        double im = 0.0, is = 0.0;
        for (int s = 0; s < 6; s++) {
          im += val[k][s] * val[l][s] * qw(s);
          // dot(grad_l, g^-1 grad_k)
          P2 gk = grd[k][s], gl = grd[l][s];
          double mx = ginv[0] * gk.x + ginv[2] * gk.y, my = ginv[1] * gk.x + ginv[3] * gk.y;
          is += (gl.x * mx + gl.y * my) * qw(s) * scale * jac / 2.0;
        }
        pm[4 * l + k] += im * scale * jac / 2.0;
        ps[4 * l + k] += is;
      }
  }
  for (int q = 0; q < 16; q++) { mass[q] += pm[q]; stiff[q] += ps[q]; }
}

GDTP_HD double quad_value(int k, double x, double y) {
  switch (k) {
    case 0: return 2 * x * x + 4 * x * y + 2 * y * y - 3 * x - 3 * y + 1;
    case 1: return 2 * x * x - 1 * x;
    case 2: return 2 * y * y - 1 * y;
    case 3: return 4 * x * y;
    case 4: return -4 * x * y - 4 * y * y + 4 * y;
    default: return -4 * x * x - 4 * x * y + 4 * x;
  }
}
GDTP_HD P2 quad_grad(int k, double x, double y) {
  switch (k) {
    case 0: return mk(4 * x + 4 * y - 3.0, 4 * x + 4 * y - 3.0);
    case 1: return mk(4 * x - 1.0, 0.0);
    case 2: return mk(0.0, 4 * y - 1.0);
    case 3: return mk(4 * y, 4 * x);
    case 4: return mk(-4 * y, -4 * x - 8 * y + 4.0);
    default: return mk(-8 * x - 4 * y + 4, -4 * x);
  }
}

// Adds the quadratic-element mass / stiffness of the part `poly` (n vertices) of
// boundary triangle bt (3 corners) lying in one chart triangle with metric g
// (column-major c00,c01,c10,c11).  mass/stiff: 36 entries [l*6+k] = (l,k) as the
// reference's polygonMass(l,k); symmetrised by the caller per polygon.
GDTP_HD void integrate_boundary_polygon(const P2* poly, int n, const P2* bt, const double* g, const double* ginv, double* mass,
                                        double* stiff) {
  // barycentric map of the boundary triangle: columns (b1-b0), (b2-b0)
  double m00 = bt[1].x - bt[0].x, m01 = bt[1].y - bt[0].y, m10 = bt[2].x - bt[0].x, m11 = bt[2].y - bt[0].y;
  double det = m00 * m11 - m01 * m10;
  double d = 1.0 / det;
  double i00 = m11 * d, i11 = m00 * d, i01 = -m01 * d, i10 = -m10 * d;  // inverse, column-major
  for (int p = 2; p < n; p++) {
    P2 d0 = mk(poly[p - 1].x - poly[0].x, poly[p - 1].y - poly[0].y);
    P2 d1 = mk(poly[p].x - poly[0].x, poly[p].y - poly[0].y);
    // unit-map metric U^T g U with U columns (d0, d1)
    double gu00 = g[0] * d0.x + g[2] * d0.y, gu01 = g[1] * d0.x + g[3] * d0.y;  // g * d0
    double gv00 = g[0] * d1.x + g[2] * d1.y, gv01 = g[1] * d1.x + g[3] * d1.y;  // g * d1
    double a = d0.x * gu00 + d0.y * gu01, b = d0.x * gv00 + d0.y * gv01, c = d1.x * gu00 + d1.y * gu01,
           e = d1.x * gv00 + d1.y * gv01;
    double triMass = sqrt(fabs(a * e - b * c)) / 2.0;
    if (!(triMass > 0)) continue;
    double val[6][6];
    P2 grd[6][6];
    for (int s = 0; s < 6; s++) {
      double px = poly[0].x + d0.x * qx(s) + d1.x * qy(s) - bt[0].x;
      double py = poly[0].y + d0.y * qx(s) + d1.y * qy(s) - bt[0].y;
      double sx = i00 * px + i10 * py, sy = i01 * px + i11 * py;
      sx = sx > 0 ? sx : 0.0;
      sy = sy > 0 ? sy : 0.0;
      double excess = sx + sy - 1.0;
      if (excess > 0) { sx -= excess / 2; sy -= excess / 2; }
      for (int k = 0; k < 6; k++) {
        val[k][s] = quad_value(k, sx, sy);
        P2 q = quad_grad(k, sx, sy);
        // barycentricMap^T * q
        grd[k][s] = mk(i00 * q.x + i01 * q.y, i10 * q.x + i11 * q.y);
      }
    }
    for (int k = 0; k < 6; k++)
      for (int l = 0; l < 6; l++) {
        double im = 0.0, is = 0.0;
        for (int s = 0; s < 6; s++) {
          im += val[k][s] * val[l][s] * qw(s);
          P2 gk = grd[k][s], gl = grd[l][s];
          double mx = ginv[0] * gl.x + ginv[2] * gl.y, my = ginv[1] * gl.x + ginv[3] * gl.y;
          is += (gk.x * mx + gk.y * my) * qw(s);
        }
        mass[6 * l + k] += im * triMass;
        stiff[6 * l + k] += is * triMass;
      }
  }
}

}  // namespace am
}  // namespace gdtp

namespace gdtp {
namespace am {

// One interior cell: accumulate over its chart triangles (pairs in ptr/tri).
// mass/stiff: 16 entries each, [4*a+b] = reference (a,b).
GDTP_HD void interior_cell(int ic, const int* cellPtr, const int* cellTri, const int* cellIJ, const int* cellChart,
                           const double* chartCellSize, const double* triPos, const double* triMetricInv,
                           const double* triScale, double* mass, double* stiff) {
  for (int q = 0; q < 16; q++) mass[q] = stiff[q] = 0.0;
  const int i = cellIJ[2 * ic], j = cellIJ[2 * ic + 1], c = cellChart[ic];
  const double cw = chartCellSize[2 * c], ch = chartCellSize[2 * c + 1];
  for (int e = cellPtr[ic]; e < cellPtr[ic + 1]; e++) {
    const int t = cellTri[e];
    P2 poly[8], tmp[8];
    for (int k = 0; k < 3; k++) poly[k] = mk(triPos[6 * t + 2 * k], triPos[6 * t + 2 * k + 1]);
    int n = clip_to_cell(poly, 3, i, j, cw, ch, tmp);
    if (n >= 3) integrate_cell_polygon(poly, n, i, j, cw, ch, &triMetricInv[4 * t], triScale[t], mass, stiff);
  }
}

// One boundary triangle: accumulate over the chart triangles overlapping its
// cell; each piece is symmetrised.  mass/stiff: 36 entries [6*l+k].
GDTP_HD void boundary_triangle(int b, const int* btPtr, const int* btTri, const double* btPos, const double* triPos,
                               const double* triMetric, const double* triMetricInv, double* mass, double* stiff) {
  for (int q = 0; q < 36; q++) mass[q] = stiff[q] = 0.0;
  P2 bt[3];
  for (int k = 0; k < 3; k++) bt[k] = mk(btPos[6 * b + 2 * k], btPos[6 * b + 2 * k + 1]);
  for (int e = btPtr[b]; e < btPtr[b + 1]; e++) {
    const int t = btTri[e];
    P2 tri[3], poly[16], tmp[16];
    for (int k = 0; k < 3; k++) tri[k] = mk(triPos[6 * t + 2 * k], triPos[6 * t + 2 * k + 1]);
    for (int k = 0; k < 3; k++) poly[k] = bt[k];
    int n = clip_to_triangle(poly, 3, tri, tmp);
    if (n < 3) continue;
    double pm[36], ps[36];
    for (int q = 0; q < 36; q++) pm[q] = ps[q] = 0.0;
    integrate_boundary_polygon(poly, n, bt, &triMetric[4 * t], &triMetricInv[4 * t], pm, ps);
    for (int k = 0; k < 6; k++)
      for (int l = 0; l < 6; l++) {
        mass[6 * k + l] += (pm[6 * k + l] + pm[6 * l + k]) / 2.0;
        stiff[6 * k + l] += (ps[6 * k + l] + ps[6 * l + k]) / 2.0;
      }
  }
}

// Deep texel d: 9 stencil coefficients from its four interior cells (raster
// order), texel slot in those cells {2,3,1,0}.  cell matrices [4*a+b].
GDTP_HD void deep_gather(int d, const int* deepCells, const double* cellMat, double* coef10) {
  const int oi[4] = {0, 1, 1, 0}, oj[4] = {0, 0, 1, 1}, slot[4] = {2, 3, 1, 0};
  for (int q = 0; q < 10; q++) coef10[q] = 0.0;
  for (int q = 0; q < 4; q++) {
    const double* M = &cellMat[16 * (long long)deepCells[4 * d + q]];
    const int k = slot[q];
    for (int l = 0; l < 4; l++) coef10[(oj[l] - oj[k] + 1) * 3 + (oi[l] - oi[k] + 1)] += M[4 * k + l];
  }
}

}  // namespace am
}  // namespace gdtp
