// Heat-method geodesics: integration of the normalised gradient field of a
// potential against the texel basis, on the device.
//
// Reference (include/Src/VectorFieldIntergration.inl):
//   samples   InitializeChartNormalizedVectorField  :77-426 (built once, FP64, stored in FP32)
//   integral  IntergrateNormalizedVectorFieldFromSamples :453-582
// Interior cells carry one sample per overlapping chart triangle (FP32): the clipped
// polygon's barycentre (cell units), the inverse parameter metric, and the
// integrals v_k of the 4 bilinear basis gradients over the polygon.  Boundary
// elements carry one sample per overlapping chart triangle (FP64): barycentre in the
// element's barycentric frame, the inverse boundary metric and the integrals of
// the 6 quadratic basis gradients.  At evaluation every sample contributes
//   X . v_k,   X = T (-grad u) / sqrt((-grad u) . T (-grad u))   (0 if that is 0)
// to its corners.  The reference scatters along cell lines; here every cell
// (boundary sample) writes its corner contributions and a gather in fixed order
// sums them per texel (fine boundary node), so results do not depend on
// scheduling.
#include "assembly_math.h"
#include "geodesic_kernels.h"

namespace gdtp {
namespace dev {

using am::mk;
using am::P2;

// 2x2 column-major (c[col][row]) helpers with the reference's product convention
struct Mat2 {
  double c00, c01, c10, c11;  // c[col][row]
};
__device__ __forceinline__ Mat2 mat_mul(const Mat2& a, const Mat2& b) {  // (a*b)(j,i) = sum_k a(k,i) b(j,k)
  Mat2 r;
  r.c00 = a.c00 * b.c00 + a.c10 * b.c01;
  r.c01 = a.c01 * b.c00 + a.c11 * b.c01;
  r.c10 = a.c00 * b.c10 + a.c10 * b.c11;
  r.c11 = a.c01 * b.c10 + a.c11 * b.c11;
  return r;
}
__device__ __forceinline__ Mat2 mat_t(const Mat2& a) { return Mat2{a.c00, a.c10, a.c01, a.c11}; }
__device__ __forceinline__ Mat2 mat_inv(const Mat2& a) {
  const double d = 1.0 / (a.c00 * a.c11 - a.c01 * a.c10);
  return Mat2{a.c11 * d, -a.c01 * d, -a.c10 * d, a.c00 * d};
}
__device__ __forceinline__ double mat_det(const Mat2& a) { return a.c00 * a.c11 - a.c01 * a.c10; }
__device__ __forceinline__ P2 mat_vec(const Mat2& a, P2 v) { return mk(a.c00 * v.x + a.c10 * v.y, a.c01 * v.x + a.c11 * v.y); }

// area-weighted barycentre of a fan-triangulated polygon
__device__ __forceinline__ P2 polygon_barycentre(const P2* poly, int n) {
  double bx = 0, by = 0, area = 0;
  for (int p = 2; p < n; p++) {
    const double d0x = poly[p - 1].x - poly[0].x, d0y = poly[p - 1].y - poly[0].y;
    const double d1x = poly[p].x - poly[0].x, d1y = poly[p].y - poly[0].y;
    const double a = fabs(d0x * d1y - d0y * d1x) / 2.0;
    bx += a * (poly[0].x + poly[p - 1].x + poly[p].x) / 3.0;
    by += a * (poly[0].y + poly[p - 1].y + poly[p].y) / 3.0;
    area += a;
  }
  return mk(bx / area, by / area);
}

// One interior-cell sample per (interior cell, chart triangle) slot
// (InitializeChartNormalizedVectorField, VectorFieldIntergration.inl:113-239).
// Layout: 16 floats: pos(2), tensor(4, column-major), v_0..v_3 (8), 0, 0.
__global__ void __launch_bounds__(256) k_geo_cell_samples(int nSlots, const int* __restrict__ slotCell,
                                                          const int* __restrict__ cellTri, const int* __restrict__ cellIJ,
                                                          const int* __restrict__ cellChart, const double* __restrict__ chartCellSize,
                                                          const double* __restrict__ triPos, const double* __restrict__ triMetric,
                                                          const double* __restrict__ triMetricInv, const double* __restrict__ triScale,
                                                          float4* __restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nSlots) return;
  const int c = slotCell[e], t = cellTri[e];
  const int i = cellIJ[2 * c], j = cellIJ[2 * c + 1], ch = cellChart[c];
  const double cw = chartCellSize[2 * ch], chh = chartCellSize[2 * ch + 1];
  P2 poly[8], tmp[8];
  for (int k = 0; k < 3; k++) poly[k] = mk(triPos[6 * t + 2 * k], triPos[6 * t + 2 * k + 1]);
  const int n = am::clip_to_cell(poly, 3, i, j, cw, chh, tmp);
  float s[16];
  for (int q = 0; q < 16; q++) s[q] = 0.f;
  if (n >= 3) {
    const Mat2 g{triMetric[4 * t], triMetric[4 * t + 1], triMetric[4 * t + 2], triMetric[4 * t + 3]};
    const Mat2 gi{triMetricInv[4 * t], triMetricInv[4 * t + 1], triMetricInv[4 * t + 2], triMetricInv[4 * t + 3]};
    const double scale = triScale[t];
    const P2 b = polygon_barycentre(poly, n);
    s[0] = float(b.x / cw - double(i));
    s[1] = float(b.y / chh - double(j));
    s[2] = float(gi.c00); s[3] = float(gi.c01); s[4] = float(gi.c10); s[5] = float(gi.c11);
    double v[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
    for (int p = 2; p < n; p++) {
      const P2 d0 = mk(poly[p - 1].x - poly[0].x, poly[p - 1].y - poly[0].y);
      const P2 d1 = mk(poly[p].x - poly[0].x, poly[p].y - poly[0].y);
      const double ums = fabs(d0.x * d1.y - d0.y * d1.x);
      for (int q = 0; q < 6; q++) {
        const double sx = (poly[0].x + d0.x * am::qx(q) + d1.x * am::qy(q)) / cw - double(i);
        const double sy = (poly[0].y + d0.y * am::qx(q) + d1.y * am::qy(q)) / chh - double(j);
        for (int k = 0; k < 4; k++) {
          const P2 gr = am::bilinear_grad(k, sx, sy);
          const P2 sg = mat_vec(gi, mk(gr.x / cw, gr.y / chh));   // g^-1 grad
          const P2 vd = mat_vec(g, sg);                           // g (g^-1 grad), as the reference forms it
          const double f = am::qw(q) * scale * ums / 2.0;
          v[k][0] += vd.x * f;
          v[k][1] += vd.y * f;
        }
      }
    }
    for (int k = 0; k < 4; k++) { s[6 + 2 * k] = float(v[k][0]); s[7 + 2 * k] = float(v[k][1]); }
  }
  for (int q = 0; q < 4; q++) out[4 * (long long)e + q] = make_float4(s[4 * q], s[4 * q + 1], s[4 * q + 2], s[4 * q + 3]);
}

// One boundary sample per (boundary element, chart triangle) slot
// (VectorFieldIntergration.inl:240-406).  Layout: 20 doubles: pos(2), tensor(4),
// v_0..v_5 (12), 0, 0.  Kept in FP64: boundary elements include slivers whose
// metric is nearly singular (condition ~1e12), where X = T g / |g|_T is only
// resolved in double precision.
__global__ void __launch_bounds__(256) k_geo_hex_samples(int nSlots, const int* __restrict__ slotBt, const int* __restrict__ btTri,
                                                         const double* __restrict__ btPos, const double* __restrict__ triPos,
                                                         const double* __restrict__ triMetric, double* __restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nSlots) return;
  const int b = slotBt[e], t = btTri[e];
  P2 bt[3], tri[3], poly[16], tmp[16];
  for (int k = 0; k < 3; k++) {
    bt[k] = mk(btPos[6 * b + 2 * k], btPos[6 * b + 2 * k + 1]);
    tri[k] = mk(triPos[6 * t + 2 * k], triPos[6 * t + 2 * k + 1]);
    poly[k] = bt[k];
  }
  const int n = am::clip_to_triangle(poly, 3, tri, tmp);
  double s[20];
  for (int q = 0; q < 20; q++) s[q] = 0.0;
  if (n >= 3) {
    const Mat2 g{triMetric[4 * t], triMetric[4 * t + 1], triMetric[4 * t + 2], triMetric[4 * t + 3]};
    const Mat2 M{bt[1].x - bt[0].x, bt[1].y - bt[0].y, bt[2].x - bt[0].x, bt[2].y - bt[0].y};
    const Mat2 Mi = mat_inv(M);                               // barycentric map
    const Mat2 bm = mat_mul(mat_mul(mat_t(M), g), M);         // boundary metric
    const Mat2 bmi = mat_inv(bm);
    const P2 c = polygon_barycentre(poly, n);
    const P2 pos = mat_vec(Mi, mk(c.x - bt[0].x, c.y - bt[0].y));
    s[0] = pos.x; s[1] = pos.y;
    s[2] = bmi.c00; s[3] = bmi.c01; s[4] = bmi.c10; s[5] = bmi.c11;
    double v[6][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}};
    for (int p = 2; p < n; p++) {
      const P2 d0 = mk(poly[p - 1].x - poly[0].x, poly[p - 1].y - poly[0].y);
      const P2 d1 = mk(poly[p].x - poly[0].x, poly[p].y - poly[0].y);
      const Mat2 U{d0.x, d0.y, d1.x, d1.y};
      const double triMass = sqrt(fabs(mat_det(mat_mul(mat_mul(mat_t(U), g), U)))) / 2.0;
      if (!(triMass > 0)) continue;
      for (int q = 0; q < 6; q++) {
        const P2 sp = mat_vec(Mi, mk(poly[0].x + d0.x * am::qx(q) + d1.x * am::qy(q) - bt[0].x,
                                     poly[0].y + d0.y * am::qx(q) + d1.y * am::qy(q) - bt[0].y));
        double sx = sp.x > 0 ? sp.x : 0.0, sy = sp.y > 0 ? sp.y : 0.0;
        const double excess = sx + sy - 1.0;
        if (excess > 0) { sx -= excess / 2; sy -= excess / 2; }
        for (int k = 0; k < 6; k++) {
          const P2 gr = am::quad_grad(k, sx, sy);
          v[k][0] += gr.x * am::qw(q) * triMass;
          v[k][1] += gr.y * am::qw(q) * triMass;
        }
      }
    }
    for (int k = 0; k < 6; k++) { s[6 + 2 * k] = v[k][0]; s[7 + 2 * k] = v[k][1]; }
  }
  for (int q = 0; q < 20; q++) out[20 * (long long)e + q] = s[q];
}

// X = T g / sqrt(g . T g), 0 when g . T g <= 0 (T column-major)
__device__ __forceinline__ void normalise(float& gx, float& gy, float t00, float t01, float t10, float t11) {
  const float ax = t00 * gx + t10 * gy, ay = t01 * gx + t11 * gy;
  const double len = double(gx) * double(ax) + double(gy) * double(ay);
  if (len > 0) {
    const double l = sqrt(len);
    gx = float(double(ax) / l);
    gy = float(double(ay) / l);
  } else {
    gx = gy = 0.f;
  }
}

// Fine boundary potential  u_f = P u_B  (Geodesics.cpp:519-522), items: fine nodes x K
__global__ void __launch_bounds__(256) k_geo_fine_potential(int nFine, int K, const int* __restrict__ pPtr, const int* __restrict__ pCol,
                                                            const double* __restrict__ pVal, const int* __restrict__ bGlobal,
                                                            const double* __restrict__ u, double* __restrict__ fineU) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nFine * K) return;
  const int f = int(t / K), c = int(t - (long long)f * K);
  double acc = 0.0;
  for (int e = pPtr[f]; e < pPtr[f + 1]; e++) acc += pVal[e] * u[(long long)bGlobal[pCol[e]] * K + c];
  fineU[t] = acc;
}

// Interior cells: contributions of every sample to the 4 corners, items: cells x K
__global__ void __launch_bounds__(256) k_geo_cells(int nCells, int K, const int* __restrict__ cellPtr, const int* __restrict__ corners,
                                                   const float4* __restrict__ samples, const double* __restrict__ u, float invW,
                                                   float invH, float* __restrict__ cellOut) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nCells * K) return;
  const int cell = int(t / K), ch = int(t - (long long)cell * K);
  float cv[4];
  for (int k = 0; k < 4; k++) cv[k] = float(u[(long long)corners[4 * cell + k] * K + ch]);
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  for (int e = cellPtr[cell]; e < cellPtr[cell + 1]; e++) {
    const float4 a = samples[4 * (long long)e], b = samples[4 * (long long)e + 1], c = samples[4 * (long long)e + 2],
                 d = samples[4 * (long long)e + 3];
    const float px = a.x, py = a.y;
    // negative gradient of the bilinear interpolant (VectorFieldIntergration.inl:514)
    float gx = -((py - 1.f) * cv[0] + (1.f - py) * cv[1] + py * cv[2] - py * cv[3]);
    float gy = -((px - 1.f) * cv[0] - px * cv[1] + px * cv[2] + (1.f - px) * cv[3]);
    gx *= invW;
    gy *= invH;
    normalise(gx, gy, a.z, a.w, b.x, b.y);
    acc[0] += gx * b.z + gy * b.w;
    acc[1] += gx * c.x + gy * c.y;
    acc[2] += gx * c.z + gy * c.w;
    acc[3] += gx * d.x + gy * d.y;
  }
  for (int k = 0; k < 4; k++) cellOut[((long long)cell * 4 + k) * K + ch] = acc[k];
}

// Boundary samples: contributions to the 6 fine nodes (FP64), items: slots x K
__global__ void __launch_bounds__(256) k_geo_hex(int nSlots, int K, const int* __restrict__ slotBt, const int* __restrict__ btIdx,
                                                 const double* __restrict__ samples, const double* __restrict__ fineU,
                                                 double* __restrict__ hexOut) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nSlots * K) return;
  const int e = int(t / K), ch = int(t - (long long)e * K);
  const int b = slotBt[e];
  double cv[6];
  for (int k = 0; k < 6; k++) cv[k] = fineU[(long long)btIdx[6 * b + k] * K + ch];
  const double* s = samples + 20 * (long long)e;
  const double x = s[0], y = s[1];
  // negative gradient of the quadratic interpolant (VectorFieldIntergration.inl:556-562)
  double gx = -((4 * x + 4 * y - 3.0) * cv[0] + (4 * x - 1.0) * cv[1] + (4 * y) * cv[3] + (-4 * y) * cv[4] + (-8 * x - 4 * y + 4.0) * cv[5]);
  double gy = -((4 * x + 4 * y - 3.0) * cv[0] + (4 * y - 1.0) * cv[2] + (4 * x) * cv[3] + (-4 * x - 8 * y + 4.0) * cv[4] + (-4 * x) * cv[5]);
  const double ax = s[2] * gx + s[4] * gy, ay = s[3] * gx + s[5] * gy;
  const double len = gx * ax + gy * ay;
  if (len > 0) {
    const double l = sqrt(len);
    gx = ax / l;
    gy = ay / l;
  } else {
    gx = gy = 0.0;
  }
  for (int k = 0; k < 6; k++) hexOut[((long long)e * 6 + k) * K + ch] = gx * s[6 + 2 * k] + gy * s[7 + 2 * k];
}

// Fine boundary right-hand side: the node's boundary-sample contributions in
// fixed order, items: fine nodes x K
__global__ void __launch_bounds__(256) k_geo_gather_fine(int nFine, int K, const int* __restrict__ ptr, const int* __restrict__ ent,
                                                         const double* __restrict__ hexOut, double* __restrict__ fineRhs) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nFine * K) return;
  const int f = int(t / K), c = int(t - (long long)f * K);
  double acc = 0.0;
  for (int e = ptr[f]; e < ptr[f + 1]; e++) acc += hexOut[(long long)ent[e] * K + c];
  fineRhs[t] = acc;
}

// Texel right-hand side: cell contributions in fixed order, plus the restricted
// fine boundary right-hand side on boundary texels (Geodesics.cpp:529-532),
// items: texels x K
__global__ void __launch_bounds__(256) k_geo_gather_texels(int n, int K, const int* __restrict__ ptr, const int* __restrict__ ent,
                                                           const float* __restrict__ cellOut, const int* __restrict__ texBoundary,
                                                           const int* __restrict__ rPtr, const int* __restrict__ rCol,
                                                           const double* __restrict__ rVal, const double* __restrict__ fineRhs,
                                                           double* __restrict__ rhs) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * K) return;
  const int i = int(t / K), c = int(t - (long long)i * K);
  float acc = 0.f;
  for (int e = ptr[i]; e < ptr[i + 1]; e++) acc += cellOut[(long long)ent[e] * K + c];
  double out = double(acc);
  const int b = texBoundary[i];
  if (b >= 0) {
    double r = 0.0;
    for (int e = rPtr[b]; e < rPtr[b + 1]; e++) r += rVal[e] * fineRhs[(long long)rCol[e] * K + c];
    out += r;
  }
  rhs[t] = out;
}

// sv[c] = d[source_c, c]; then d[:, c] -= sv[c] (distance 0 at the source)
__global__ void k_geo_source_values(int K, const int* __restrict__ sources, const double* __restrict__ d, double* __restrict__ sv) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < K) sv[c] = d[(long long)sources[c] * K + c];
}
__global__ void __launch_bounds__(256) k_geo_subtract(long long n, int K, const double* __restrict__ sv, double* __restrict__ d) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n * K) d[t] -= sv[t % K];
}

// RHS of the smoothing solve: delta at each column's source texel
__global__ void __launch_bounds__(256) k_geo_impulses(long long n, int K, const int* __restrict__ sources, double* __restrict__ b) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * K) return;
  const long long i = t / K;
  const int c = int(t - i * K);
  b[t] = (sources[c] == i) ? 1.0 : 0.0;
}

static inline int blocks(long long items) { return int((items + 255) / 256); }

void launch_geo_cell_samples(int nSlots, const int* slotCell, const int* cellTri, const int* cellIJ, const int* cellChart,
                             const double* chartCellSize, const double* triPos, const double* triMetric, const double* triMetricInv,
                             const double* triScale, float4* out, cudaStream_t s) {
  if (nSlots > 0)
    k_geo_cell_samples<<<blocks(nSlots), 256, 0, s>>>(nSlots, slotCell, cellTri, cellIJ, cellChart, chartCellSize, triPos, triMetric,
                                                      triMetricInv, triScale, out);
}
void launch_geo_hex_samples(int nSlots, const int* slotBt, const int* btTri, const double* btPos, const double* triPos,
                            const double* triMetric, double* out, cudaStream_t s) {
  if (nSlots > 0) k_geo_hex_samples<<<blocks(nSlots), 256, 0, s>>>(nSlots, slotBt, btTri, btPos, triPos, triMetric, out);
}
void launch_geo_rhs(const GeoDev& G, const double* u, double* rhs, int K, cudaStream_t s) {
  if (G.nFine > 0) {
    k_geo_fine_potential<<<blocks((long long)G.nFine * K), 256, 0, s>>>(G.nFine, K, G.pPtr, G.pCol, G.pVal, G.bGlobal, u, G.fineU);
    if (G.nHex > 0) k_geo_hex<<<blocks((long long)G.nHex * K), 256, 0, s>>>(G.nHex, K, G.slotBt, G.btIdx, G.hexSamples, G.fineU, G.hexOut);
    k_geo_gather_fine<<<blocks((long long)G.nFine * K), 256, 0, s>>>(G.nFine, K, G.fPtr, G.fEnt, G.hexOut, G.fineRhs);
  }
  if (G.nCells > 0)
    k_geo_cells<<<blocks((long long)G.nCells * K), 256, 0, s>>>(G.nCells, K, G.cellPtr, G.corners, G.cellSamples, u, G.invW, G.invH,
                                                               G.cellOut);
  k_geo_gather_texels<<<blocks((long long)G.n * K), 256, 0, s>>>(G.n, K, G.tPtr, G.tEnt, G.cellOut, G.texBoundary, G.rPtr, G.rCol,
                                                                 G.rVal, G.fineRhs, rhs);
}
void launch_geo_impulses(long long n, int K, const int* sources, double* b, cudaStream_t s) {
  k_geo_impulses<<<blocks(n * K), 256, 0, s>>>(n, K, sources, b);
}
void launch_geo_shift(long long n, int K, const int* sources, double* d, double* sourceValues, cudaStream_t s) {
  k_geo_source_values<<<blocks(K), 256, 0, s>>>(K, sources, d, sourceValues);
  k_geo_subtract<<<blocks(n * K), 256, 0, s>>>(n, K, sourceValues, d);
}

}  // namespace dev
}  // namespace gdtp
