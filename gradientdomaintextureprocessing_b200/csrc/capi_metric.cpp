// C ABI: per-triangle parameter metrics for gdtp_system_create (host only).
#include <vector>

#include "gdtp.h"
#include "capi_internal.h"

using namespace gdtp;

static bool make_mesh(const double* vertices, int64_t nv, const int32_t* triangles, int64_t nt, const double* uv, Mesh& m) {
  if (!vertices || !triangles || !uv || nv <= 0 || nt <= 0) return false;
  for (int64_t k = 0; k < 3 * nt; k++)
    if (triangles[k] < 0 || triangles[k] >= nv) return false;
  m.vertices.assign(vertices, vertices + nv * 3);
  m.triangles.assign(triangles, triangles + nt * 3);
  m.uv.assign(uv, uv + nt * 6);
  return true;
}

static void emit(const std::vector<M2>& P, double* out) {
  for (size_t t = 0; t < P.size(); t++) {
    out[4 * t] = P[t].c[0][0];
    out[4 * t + 1] = P[t].c[0][1];
    out[4 * t + 2] = P[t].c[1][0];
    out[4 * t + 3] = P[t].c[1][1];
  }
}

extern "C" int gdtp_surface_metric(const double* vertices, int64_t nv, const int32_t* triangles, int64_t nt, const double* uv,
                                   int mode, double* metric_out) {
  return guarded("gdtp_surface_metric", [&]() -> int {
    Mesh m;
    if (!metric_out || (mode != 0 && mode != 1) || !make_mesh(vertices, nv, triangles, nt, uv, m))
      return fail(GDTP_ERR_INVALID, "gdtp_surface_metric: invalid arguments");
    std::vector<M2> G, P;
    if (!surface_metric(m, mode, true, G)) return fail(GDTP_ERR_SETUP, "gdtp_surface_metric: zero total area");
    if (!parameter_metric(m, G, P)) return fail(GDTP_ERR_SETUP, "gdtp_surface_metric: degenerate texture triangle");
    emit(P, metric_out);
    return GDTP_OK;
  });
}

extern "C" int gdtp_anisotropic_metric(const double* vertices, int64_t nv, const int32_t* triangles, int64_t nt, const double* uv,
                                       const double* vf, double across, double isotropic, double* metric_out) {
  return guarded("gdtp_anisotropic_metric", [&]() -> int {
    Mesh m;
    if (!metric_out || !vf || !(across >= 0) || !(isotropic > 0) || !make_mesh(vertices, nv, triangles, nt, uv, m))
      return fail(GDTP_ERR_INVALID, "gdtp_anisotropic_metric: invalid arguments");
    std::vector<M2> G, U, P;
    if (!surface_metric(m, 0, true, G)) return fail(GDTP_ERR_SETUP, "gdtp_anisotropic_metric: zero total area");
    if (!vector_field_metric(G, vf, across, isotropic, true, U)) return fail(GDTP_ERR_SETUP, "gdtp_anisotropic_metric: zero metric area");
    if (!parameter_metric(m, U, P)) return fail(GDTP_ERR_SETUP, "gdtp_anisotropic_metric: degenerate texture triangle");
    emit(P, metric_out);
    return GDTP_OK;
  });
}
