// C ABI: device system (assembly, update, apply, V-cycle, solves).
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "gdtp.h"
#include "capi_internal.h"
#include "system.h"

using namespace gdtp;

struct gdtp_system {
  gdtp_hierarchy* h = nullptr;
  std::unique_ptr<DeviceSystem> sys;
};

#define GDTP_SYS_CHECK(s)                                                       \
  do {                                                                          \
    if (!(s) || !(s)->sys) return fail(GDTP_ERR_INVALID, "null system handle"); \
  } while (0)

static int sys_fail(gdtp_system* s, int code) { return fail(code, s->sys->error()); }

extern "C" int gdtp_system_create(gdtp_hierarchy* h, int device, int metric_mode, const double* parameter_metric,
                                  const double* vertices, int64_t nv, gdtp_system** out) {
  return guarded("gdtp_system_create", [&]() -> int {
    if (!h || !out) return fail(GDTP_ERR_INVALID, "gdtp_system_create: null argument");
    if (metric_mode != 0 && metric_mode != 1 && !parameter_metric)
      return fail(GDTP_ERR_INVALID, "gdtp_system_create: unknown metric mode");
    *out = nullptr;
    std::unique_ptr<gdtp_system> s(new gdtp_system());
    s->h = h;
    Mesh mesh = h->mesh;
    if (vertices) {
      if (nv != mesh.nv()) return fail(GDTP_ERR_INVALID, "gdtp_system_create: vertex count differs from the hierarchy's mesh");
      mesh.vertices.assign(vertices, vertices + nv * 3);
    }
    std::vector<double> uniform;
    if (!parameter_metric && metric_mode == 1) {  // uniform metric, per mesh triangle
      std::vector<M2> G, P;
      if (!surface_metric(mesh, 1, true, G) || !gdtp::parameter_metric(mesh, G, P))
        return fail(GDTP_ERR_SETUP, "gdtp_system_create: degenerate texture triangles");
      uniform.resize(4 * P.size());
      for (size_t t = 0; t < P.size(); t++) {
        uniform[4 * t] = P[t].c[0][0]; uniform[4 * t + 1] = P[t].c[0][1];
        uniform[4 * t + 2] = P[t].c[1][0]; uniform[4 * t + 3] = P[t].c[1][1];
      }
      parameter_metric = uniform.data();
    }
    s->sys.reset(new DeviceSystem(h->h, h->be, device));
    if (!s->sys->ok()) return fail(GDTP_ERR_CUDA, s->sys->error());
    if (!s->sys->assemble(mesh, parameter_metric)) return fail(GDTP_ERR_CUDA, s->sys->error());
    *out = s.release();
    return GDTP_OK;
  });
}

extern "C" void gdtp_system_free(gdtp_system* s) { delete s; }

extern "C" int gdtp_system_update(gdtp_system* s, double stiffness_weight, double screen_weight) {
  return guarded("gdtp_system_update", [&]() -> int {
    GDTP_SYS_CHECK(s);
    if (!(screen_weight >= 0) || !(stiffness_weight >= 0) || screen_weight + stiffness_weight == 0)
      return fail(GDTP_ERR_INVALID, "gdtp_system_update: weights must be non-negative and not both zero");
    if (!s->sys->update(stiffness_weight, screen_weight)) return sys_fail(s, GDTP_ERR_NUMERIC);
    return GDTP_OK;
  });
}

extern "C" int gdtp_system_array(const gdtp_system* s, const char* cname, int level, void* out, int64_t* count) {
  return guarded("gdtp_system_array", [&]() -> int {
    if (!s || !s->sys || !cname) return fail(GDTP_ERR_INVALID, "gdtp_system_array: bad arguments");
    const std::string name(cname);
    const FineSystem& f = s->sys->fine();
    auto vec = [&](const std::vector<double>& v) {
      if (count) *count = (int64_t)v.size();
      if (out && !v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(double));
      return GDTP_OK;
    };
    if (name == "deepMass") return vec(f.deepMass);
    if (name == "deepStiffness") return vec(f.deepStiffness);
    auto part = [&](const std::string& prefix) { return name.substr(prefix.size()); };
    if (name.rfind("bbMass.", 0) == 0) return emit_csr(f.bbMass, part("bbMass."), out, count);
    if (name.rfind("bbStiffness.", 0) == 0) return emit_csr(f.bbStiffness, part("bbStiffness."), out, count);
    if (name.rfind("bdMass.", 0) == 0) return emit_csr(f.bdMass, part("bdMass."), out, count);
    if (name.rfind("bdStiffness.", 0) == 0) return emit_csr(f.bdStiffness, part("bdStiffness."), out, count);
    const auto& co = s->sys->coefficients();
    if (name.rfind("coef.", 0) == 0) {
      if (level < 0 || level >= (int)co.size()) return fail(GDTP_ERR_STATE, "coefficients not available for this level (update first)");
      if (name == "coef.deep") return vec(co[level].deep);
      if (name.rfind("coef.bb.", 0) == 0) return emit_csr(co[level].bb, part("coef.bb."), out, count);
      if (name.rfind("coef.bd.", 0) == 0) return emit_csr(co[level].bd, part("coef.bd."), out, count);
    }
    if (name == "profile") {  // {timed groups, total ms, deep texels per group, kernels per step graph, kernels launched,
                              //  smoother of the timed group: 1 one fused tile-smoother launch, 2 a sweep of two
                              //  row-smoother launches, 0 a sweep of four colour passes}
      double v[6] = {s->sys->profCount, s->sys->profMs, s->sys->profTexels, double(s->sys->graphKernels),
                     double(s->sys->kernelLaunches), s->sys->profTiled() ? 1.0 : (s->sys->profRows() ? 2.0 : 0.0)};
      if (count) *count = 6;
      if (out) std::memcpy(out, v, sizeof(v));
      return GDTP_OK;
    }
    if (name == "profile.levels") {  // {steps timed, levels L, down ms x (L-1), coarse ms, up ms x (L-1)}
      const DeviceSystem& d = *s->sys;
      std::vector<double> v{d.traceCount, double(d.traceDownMs.size() + 1)};
      v.insert(v.end(), d.traceDownMs.begin(), d.traceDownMs.end());
      v.push_back(d.traceCoarseMs);
      v.insert(v.end(), d.traceUpMs.begin(), d.traceUpMs.end());
      return vec(v);
    }
    if (name == "profile.cluster") {  // {code, ns} pairs of the last traced cluster launch, start at [1022]
      std::vector<unsigned long long> t;
      if (!const_cast<DeviceSystem*>(s->sys.get())->cluster_timeline(t)) return fail(GDTP_ERR_CUDA, s->sys->error());
      std::vector<double> v(t.begin(), t.end());
      return vec(v);
    }
    if (name == "profile.reset") {
      DeviceSystem* d = const_cast<DeviceSystem*>(s->sys.get());
      d->profCount = 0;
      d->profMs = 0;
      d->kernelLaunches = 0;
      d->traceCount = 0;
      d->traceCoarseMs = 0;
      d->traceDownMs.clear();
      d->traceUpMs.clear();
      if (count) *count = 0;
      return GDTP_OK;
    }
    if (name == "profile.setup") return vec(std::vector<double>(s->sys->setupMs, s->sys->setupMs + 14));
    if (name == "levelStats") return vec(s->sys->level_stats());  // 9 per level, see DeviceSystem::level_stats
    if (name == "levelsUsed") {
      if (count) *count = 1;
      if (out) *static_cast<int32_t*>(out) = s->sys->levelsUsed();
      return GDTP_OK;
    }
    return fail(GDTP_ERR_INVALID, "gdtp_system_array: unknown array " + name);
  });
}

extern "C" int gdtp_apply(gdtp_system* s, int which, const double* x, double* y, int k) {
  return guarded("gdtp_apply", [&]() -> int {
    GDTP_SYS_CHECK(s);
    if (!x || !y || which < 0 || which > 2) return fail(GDTP_ERR_INVALID, "gdtp_apply: bad arguments");
    return s->sys->apply(which, x, y, k) ? GDTP_OK : sys_fail(s, GDTP_ERR_CUDA);
  });
}

extern "C" int gdtp_apply_mass_stiffness(gdtp_system* s, double mass_weight, double stiffness_weight, const double* x, double* y, int k) {
  return guarded("gdtp_apply_mass_stiffness", [&]() -> int {
    GDTP_SYS_CHECK(s);
    if (!x || !y) return fail(GDTP_ERR_INVALID, "gdtp_apply_mass_stiffness: bad arguments");
    return s->sys->apply_combination(mass_weight, stiffness_weight, x, y, k) ? GDTP_OK : sys_fail(s, GDTP_ERR_CUDA);
  });
}

extern "C" int gdtp_vcycle(gdtp_system* s, float* x, const float* rhs, int k) {
  return guarded("gdtp_vcycle", [&]() -> int {
    GDTP_SYS_CHECK(s);
    if (!x || !rhs) return fail(GDTP_ERR_INVALID, "gdtp_vcycle: null vector");
    return s->sys->vcycle_host(x, rhs, k) ? GDTP_OK : sys_fail(s, GDTP_ERR_CUDA);
  });
}

extern "C" int gdtp_vcycle64(gdtp_system* s, double* x, const double* rhs, int k) {
  return guarded("gdtp_vcycle64", [&]() -> int {
    GDTP_SYS_CHECK(s);
    if (!x || !rhs) return fail(GDTP_ERR_INVALID, "gdtp_vcycle64: null vector");
    return s->sys->vcycle_host64(x, rhs, k) ? GDTP_OK : sys_fail(s, GDTP_ERR_CUDA);
  });
}

extern "C" int gdtp_relax(gdtp_system* s, float* x, const float* rhs, int k, int sweeps, int reverse) {
  return guarded("gdtp_relax", [&]() -> int {
    GDTP_SYS_CHECK(s);
    if (!x || !rhs || sweeps < 0 || sweeps > 64) return fail(GDTP_ERR_INVALID, "gdtp_relax: bad arguments");
    return s->sys->relax_host(x, rhs, k, sweeps, reverse != 0) ? GDTP_OK : sys_fail(s, GDTP_ERR_CUDA);
  });
}

static void fill_report(gdtp_report* r, const SolveReport& rep) {
  if (!r) return;
  r->iterations = rep.iterations;
  r->vcycles = rep.vcycles;
  r->rel_residual_max = rep.relMax;
  r->seconds = rep.seconds;
}

extern "C" int gdtp_solve(gdtp_system* s, const double* b, double* x, int k, double tol, int max_iters, gdtp_report* report) {
  return guarded("gdtp_solve", [&]() -> int {
    GDTP_SYS_CHECK(s);
    if (!b || !x || !(tol > 0) || max_iters < 0) return fail(GDTP_ERR_INVALID, "gdtp_solve: bad arguments");
    SolveReport rep;
    if (!s->sys->solve_mixed(b, x, nullptr, nullptr, k, tol, max_iters, nullptr, rep)) return sys_fail(s, GDTP_ERR_CUDA);
    fill_report(report, rep);
    return rep.relMax <= tol ? GDTP_OK : fail(GDTP_ERR_NOT_CONVERGED, "relative residual above tolerance after max_iters");
  });
}

extern "C" int gdtp_solve_ex(gdtp_system* s, const double* b, double* x, int k, double tol, int max_iters, int flags,
                             gdtp_report* report) {
  return guarded("gdtp_solve_ex", [&]() -> int {
    GDTP_SYS_CHECK(s);
    if (!b || !x || !(tol > 0) || max_iters < 0 || (flags & ~GDTP_ZERO_GUESS)) return fail(GDTP_ERR_INVALID, "gdtp_solve_ex: bad arguments");
    SolveReport rep;
    if (!s->sys->solve_mixed(b, x, nullptr, nullptr, k, tol, max_iters, nullptr, rep, (flags & GDTP_ZERO_GUESS) != 0))
      return sys_fail(s, GDTP_ERR_CUDA);
    fill_report(report, rep);
    return rep.relMax <= tol ? GDTP_OK : fail(GDTP_ERR_NOT_CONVERGED, "relative residual above tolerance after max_iters");
  });
}

extern "C" int gdtp_solve_stream(gdtp_system* s, const double* const* b, double* const* x, int count, int k, double tol, int max_iters,
                                 gdtp_report* reports) {
  return guarded("gdtp_solve_stream", [&]() -> int {
    GDTP_SYS_CHECK(s);
    if (count < 0 || (count > 0 && (!b || !x)) || !(tol > 0) || max_iters < 0)
      return fail(GDTP_ERR_INVALID, "gdtp_solve_stream: bad arguments");
    for (int i = 0; i < count; i++)
      if (!b[i] || !x[i]) return fail(GDTP_ERR_INVALID, "gdtp_solve_stream: null vector");
    std::vector<SolveReport> reps(count);
    if (!s->sys->solve_stream(b, x, count, k, tol, max_iters, reps.data())) return sys_fail(s, GDTP_ERR_CUDA);
    bool converged = true;
    for (int i = 0; i < count; i++) {
      if (reports) fill_report(reports + i, reps[i]);
      converged = converged && reps[i].relMax <= tol;
    }
    return converged ? GDTP_OK : fail(GDTP_ERR_NOT_CONVERGED, "relative residual above tolerance after max_iters");
  });
}

extern "C" int gdtp_solve_device(gdtp_system* s, const double* b_dev, double* x_dev, int k, double tol, int max_iters, void* stream,
                                 gdtp_report* report) {
  return guarded("gdtp_solve_device", [&]() -> int {
    GDTP_SYS_CHECK(s);
    if (!b_dev || !x_dev || !(tol > 0) || max_iters < 0) return fail(GDTP_ERR_INVALID, "gdtp_solve_device: bad arguments");
    SolveReport rep;
    if (!s->sys->solve_mixed(nullptr, nullptr, b_dev, x_dev, k, tol, max_iters, static_cast<cudaStream_t>(stream), rep))
      return sys_fail(s, GDTP_ERR_CUDA);
    fill_report(report, rep);
    return rep.relMax <= tol ? GDTP_OK : fail(GDTP_ERR_NOT_CONVERGED, "relative residual above tolerance after max_iters");
  });
}

extern "C" int gdtp_solve_fp64(gdtp_system* s, const double* b, double* x, int k, double tol, int max_iters, gdtp_report* report) {
  return guarded("gdtp_solve_fp64", [&]() -> int {
    GDTP_SYS_CHECK(s);
    if (!b || !x || !(tol > 0) || max_iters < 0) return fail(GDTP_ERR_INVALID, "gdtp_solve_fp64: bad arguments");
    SolveReport rep;
    if (!s->sys->solve_fp64(b, x, nullptr, nullptr, k, tol, max_iters, nullptr, rep)) return sys_fail(s, GDTP_ERR_CUDA);
    fill_report(report, rep);
    return rep.relMax <= tol ? GDTP_OK : fail(GDTP_ERR_NOT_CONVERGED, "relative residual above tolerance after max_iters");
  });
}

extern "C" int gdtp_solve_fp64_device(gdtp_system* s, const double* b_dev, double* x_dev, int k, double tol, int max_iters,
                                      void* stream, gdtp_report* report) {
  return guarded("gdtp_solve_fp64_device", [&]() -> int {
    GDTP_SYS_CHECK(s);
    if (!b_dev || !x_dev || !(tol > 0) || max_iters < 0) return fail(GDTP_ERR_INVALID, "gdtp_solve_fp64_device: bad arguments");
    SolveReport rep;
    if (!s->sys->solve_fp64(nullptr, nullptr, b_dev, x_dev, k, tol, max_iters, static_cast<cudaStream_t>(stream), rep))
      return sys_fail(s, GDTP_ERR_CUDA);
    fill_report(report, rep);
    return rep.relMax <= tol ? GDTP_OK : fail(GDTP_ERR_NOT_CONVERGED, "relative residual above tolerance after max_iters");
  });
}

extern "C" int gdtp_residual(gdtp_system* s, const double* b, const double* x, int k, double* rel) {
  return guarded("gdtp_residual", [&]() -> int {
    GDTP_SYS_CHECK(s);
    if (!b || !x || !rel) return fail(GDTP_ERR_INVALID, "gdtp_residual: null argument");
    return s->sys->residual_host(b, x, k, rel) ? GDTP_OK : sys_fail(s, GDTP_ERR_CUDA);
  });
}

extern "C" int gdtp_system_set(gdtp_system* s, const char* knob, double value) {
  return guarded("gdtp_system_set", [&]() -> int {
    GDTP_SYS_CHECK(s);
    if (!knob) return fail(GDTP_ERR_INVALID, "gdtp_system_set: null knob");
    const std::string k(knob);
    SolverKnobs& kn = s->sys->knobs;
    const int v = int(value);
    if (k == "pre_sweeps" && v >= 0 && v <= 16) kn.preSweeps = v;
    else if (k == "post_sweeps" && v >= 0 && v <= 16) kn.postSweeps = v;
    else if (k == "pre_boundary" && (v == 0 || v == 1)) kn.preBoundary = v;
    else if (k == "post_boundary" && (v == 0 || v == 1)) kn.postBoundary = v;
    else if (k == "max_block" && v >= 16 && v <= dev::kBoundaryChunkMax) kn.maxBlock = v;
    else if (k == "max_coarse" && v >= 16 && v <= 12000) kn.maxCoarse = v;
    else if (k == "bs_blocks_per_sm" && v >= 1 && v <= 16) kn.bsBlocksPerSm = v;
    else if (k == "dense_boundary_max" && v >= 0 && v <= 8192) kn.denseBoundaryMax = v;
    else if (k == "programmatic_launch" && (v == 0 || v == 1)) dev::set_programmatic_launch(v != 0);
    else if (k == "trace_levels" && (v == 0 || v == 1)) kn.traceLevels = v;
    else if (k == "cluster_texels" && v >= 0) kn.clusterTexels = v;
    else if (k == "grid_texels" && v >= 0) kn.gridTexels = v;
    else if (k == "chart_texels" && v >= 0) kn.chartTexels = v;
    else if (k == "tile_texels" && v >= 0) kn.tileTexels = v;
    else if (k == "tile_rounds" && v >= 1 && v <= 16) kn.tileRounds = v;
    else if (k == "tile_pre_sweeps" && v >= 0 && v <= 16) kn.tilePreSweeps = v;
    else if (k == "tile_post_sweeps" && v >= 0 && v <= 16) kn.tilePostSweeps = v;
    else if (k == "tile_finish" && (v == 0 || v == 1)) kn.tileFinish = v;
    else if (k == "coarse_pre_sweeps" && v >= -1 && v <= 16) kn.coarsePreSweeps = v;
    else if (k == "coarse_post_sweeps" && v >= -1 && v <= 16) kn.coarsePostSweeps = v;
    else if (k == "coarse_from" && v >= 1 && v <= 16) kn.coarseFrom = v;
    else if (k == "krylov" && (v == 0 || v == 1)) kn.krylov = v;
    else if (k == "zero_start_skip" && (v == 0 || v == 1)) kn.zeroStartSkip = v;
    else if (k == "device_factor" && (v == 0 || v == 1)) kn.deviceFactor = v;
    else if (k == "row_sweeps" && (v == 0 || v == 1)) kn.rowSweeps = v;
    else return fail(GDTP_ERR_INVALID, "gdtp_system_set: unknown knob or value out of range: " + k);
    if (k == "tile_texels" || k == "device_factor" || k == "max_block" || k == "dense_boundary_max" || k == "max_coarse")
      s->sys->invalidate_multigrids();  // the multigrids are laid out and factorised by these knobs
    s->sys->invalidate_graph();
    return GDTP_OK;
  });
}

extern "C" int gdtp_system_get(const gdtp_system* s, const char* knob, double* value) {
  return guarded("gdtp_system_get", [&]() -> int {
    if (!s || !s->sys || !knob || !value) return fail(GDTP_ERR_INVALID, "gdtp_system_get: bad arguments");
    const std::string k(knob);
    const SolverKnobs& kn = s->sys->knobs;
    if (k == "pre_sweeps") *value = kn.preSweeps;
    else if (k == "post_sweeps") *value = kn.postSweeps;
    else if (k == "pre_boundary") *value = kn.preBoundary;
    else if (k == "post_boundary") *value = kn.postBoundary;
    else if (k == "max_block") *value = kn.maxBlock;
    else if (k == "max_coarse") *value = kn.maxCoarse;
    else if (k == "bs_blocks_per_sm") *value = kn.bsBlocksPerSm;
    else if (k == "dense_boundary_max") *value = kn.denseBoundaryMax;
    else if (k == "programmatic_launch") *value = dev::programmatic_launch() ? 1 : 0;
    else if (k == "trace_levels") *value = kn.traceLevels;
    else if (k == "cluster_texels") *value = kn.clusterTexels;
    else if (k == "coarse_pre_sweeps") *value = kn.coarsePreSweeps;
    else if (k == "coarse_post_sweeps") *value = kn.coarsePostSweeps;
    else if (k == "coarse_from") *value = kn.coarseFrom;
    else if (k == "krylov") *value = kn.krylov;
    else if (k == "zero_start_skip") *value = kn.zeroStartSkip;
    else if (k == "device_factor") *value = kn.deviceFactor;
    else if (k == "row_sweeps") *value = kn.rowSweeps;
    else if (k == "grid_texels") *value = kn.gridTexels;
    else if (k == "chart_texels") *value = kn.chartTexels;
    else if (k == "tile_texels") *value = kn.tileTexels;
    else if (k == "tile_rounds") *value = kn.tileRounds;
    else if (k == "tile_pre_sweeps") *value = kn.tilePreSweeps;
    else if (k == "tile_post_sweeps") *value = kn.tilePostSweeps;
    else if (k == "tile_finish") *value = kn.tileFinish;
    else return fail(GDTP_ERR_INVALID, "gdtp_system_get: unknown knob " + k);
    return GDTP_OK;
  });
}

extern "C" int gdtp_system_autotune(gdtp_system* s, const double* b, int k, double tol, double* knobs_out) {
  return guarded("gdtp_system_autotune", [&]() -> int {
    GDTP_SYS_CHECK(s);
    if (!b || !(tol > 0)) return fail(GDTP_ERR_INVALID, "gdtp_system_autotune: bad arguments");
    SolverKnobs best;
    double secs = 0;
    if (!s->sys->autotune(b, k, tol, best, secs)) return sys_fail(s, GDTP_ERR_CUDA);
    if (knobs_out) {
      knobs_out[0] = best.preSweeps;
      knobs_out[1] = best.postSweeps;
      knobs_out[2] = best.preBoundary;
      knobs_out[3] = best.postBoundary;
      knobs_out[4] = secs;
    }
    return GDTP_OK;
  });
}

extern "C" int gdtp_system_device_bytes(const gdtp_system* s, int64_t* bytes) {
  return guarded("gdtp_system_device_bytes", [&]() -> int {
    if (!s || !s->sys || !bytes) return fail(GDTP_ERR_INVALID, "gdtp_system_device_bytes: bad arguments");
    *bytes = (int64_t)s->sys->deviceBytes();
    return GDTP_OK;
  });
}

// Internal accessor for entry points compiled in other translation units (not exported).
extern "C" __attribute__((visibility("hidden"))) int gdtp_system_device_view(const gdtp_system* s, const void** sys) {
  if (!s || !s->sys || !sys) return fail(GDTP_ERR_INVALID, "null system handle");
  *sys = s->sys.get();
  return GDTP_OK;
}
