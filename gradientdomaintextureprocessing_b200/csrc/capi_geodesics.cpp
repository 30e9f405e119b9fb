// C ABI: heat-method geodesics (samples, normalised-field integration, distances).
#include <algorithm>
#include <memory>
#include <vector>

#include "gdtp.h"
#include "capi_internal.h"
#include "geodesics.h"

using namespace gdtp;

extern "C" __attribute__((visibility("hidden"))) int gdtp_system_device_view(const gdtp_system* s, const void** sys);

struct gdtp_geodesics {
  std::unique_ptr<GeodesicIntegrator> g;
};

static DeviceSystem* system_of(gdtp_system* s) {
  const void* p = nullptr;
  if (!s || gdtp_system_device_view(s, &p) != GDTP_OK || !p) return nullptr;
  return const_cast<DeviceSystem*>(static_cast<const DeviceSystem*>(p));
}

extern "C" int gdtp_geodesics_create(gdtp_system* s, gdtp_geodesics** out) {
  return guarded("gdtp_geodesics_create", [&]() -> int {
    DeviceSystem* d = system_of(s);
    if (!d || !out) return fail(GDTP_ERR_INVALID, "gdtp_geodesics_create: bad arguments");
    *out = nullptr;
    std::unique_ptr<gdtp_geodesics> g(new gdtp_geodesics());
    g->g.reset(new GeodesicIntegrator(*d));
    if (!g->g->ok()) return fail(GDTP_ERR_CUDA, g->g->error());
    *out = g.release();
    return GDTP_OK;
  });
}

extern "C" void gdtp_geodesics_free(gdtp_geodesics* g) { delete g; }

extern "C" int gdtp_geodesics_counts(const gdtp_geodesics* g, int64_t* counts) {
  return guarded("gdtp_geodesics_counts", [&]() -> int {
    if (!g || !g->g || !counts) return fail(GDTP_ERR_INVALID, "gdtp_geodesics_counts: bad arguments");
    counts[0] = g->g->cellSlots;
    counts[1] = g->g->hexSlots;
    return GDTP_OK;
  });
}

extern "C" int gdtp_geodesics_array(gdtp_geodesics* g, const char* name, double* out, int64_t* count) {
  return guarded("gdtp_geodesics_array", [&]() -> int {
    if (!g || !g->g || !name) return fail(GDTP_ERR_INVALID, "gdtp_geodesics_array: bad arguments");
    std::vector<double> v;
    if (!g->g->download(name, v)) return fail(GDTP_ERR_INVALID, g->g->error());
    if (count) *count = (int64_t)v.size();
    if (out) std::copy(v.begin(), v.end(), out);
    return GDTP_OK;
  });
}

extern "C" int gdtp_geodesic_rhs(gdtp_geodesics* g, const double* potential, double* rhs, int k) {
  return guarded("gdtp_geodesic_rhs", [&]() -> int {
    if (!g || !g->g || !potential || !rhs) return fail(GDTP_ERR_INVALID, "gdtp_geodesic_rhs: bad arguments");
    return g->g->rhs_host(potential, rhs, k) ? GDTP_OK : fail(GDTP_ERR_CUDA, g->g->error());
  });
}

extern "C" int gdtp_geodesic_rhs_device(gdtp_geodesics* g, const double* potential_dev, double* rhs_dev, int k, void* stream) {
  return guarded("gdtp_geodesic_rhs_device", [&]() -> int {
    if (!g || !g->g || !potential_dev || !rhs_dev) return fail(GDTP_ERR_INVALID, "gdtp_geodesic_rhs_device: bad arguments");
    return g->g->rhs_device(potential_dev, rhs_dev, k, static_cast<cudaStream_t>(stream)) ? GDTP_OK : fail(GDTP_ERR_CUDA, g->g->error());
  });
}

extern "C" int gdtp_geodesic_distance(gdtp_geodesics* g, gdtp_system* smooth, gdtp_system* distance, const int32_t* sources, int k,
                                      double tol, int max_iters, double* distance_out, gdtp_report* report) {
  return guarded("gdtp_geodesic_distance", [&]() -> int {
    DeviceSystem* a = system_of(smooth);
    DeviceSystem* b = system_of(distance);
    if (!g || !g->g || !a || !b || !sources || !distance_out || !(tol > 0) || max_iters < 0)
      return fail(GDTP_ERR_INVALID, "gdtp_geodesic_distance: bad arguments");
    SolveReport ra, rb;
    if (!g->g->distance(*a, *b, sources, k, tol, max_iters, distance_out, ra, rb)) return fail(GDTP_ERR_CUDA, g->g->error());
    if (report) {  // both solves: iterations and V-cycles summed, worst residual, total device time
      report->iterations = ra.iterations + rb.iterations;
      report->vcycles = ra.vcycles + rb.vcycles;
      report->rel_residual_max = std::max(ra.relMax, rb.relMax);
      report->seconds = ra.seconds + rb.seconds;
    }
    return (ra.relMax <= tol && rb.relMax <= tol) ? GDTP_OK : fail(GDTP_ERR_NOT_CONVERGED, "relative residual above tolerance after max_iters");
  });
}
