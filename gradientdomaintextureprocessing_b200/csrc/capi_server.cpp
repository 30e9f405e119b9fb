// C ABI: the solve server (resident models, HBM admission, continuous batching).
#include <cstring>
#include <memory>

#include "gdtp.h"
#include "capi_internal.h"
#include "server.h"

using namespace gdtp;

struct gdtp_server {
  std::unique_ptr<Server> s;
};

extern "C" int gdtp_server_create(int device, int64_t hbm_budget_bytes, int slots, gdtp_server** out) {
  return guarded("gdtp_server_create", [&]() -> int {
    if (!out) return fail(GDTP_ERR_INVALID, "gdtp_server_create: null output");
    *out = nullptr;
    std::unique_ptr<gdtp_server> s(new gdtp_server());
    s->s.reset(new Server(device, hbm_budget_bytes, slots));
    if (!s->s->ok()) return fail(GDTP_ERR_INVALID, s->s->error());
    *out = s.release();
    return GDTP_OK;
  });
}

extern "C" void gdtp_server_free(gdtp_server* s) { delete s; }

extern "C" int gdtp_server_add_model(gdtp_server* s, const double* vertices, int64_t nv, const int32_t* triangles, int64_t nt,
                                     const double* uv, int width, int height, int levels, int kind, double weight, double second,
                                     const double* parameter_metric, int* model_out) {
  return guarded("gdtp_server_add_model", [&]() -> int {
    if (!s || !s->s || !vertices || !triangles || !uv || nv <= 0 || nt <= 0 || !model_out || width <= 1 || height <= 1 || levels < 1)
      return fail(GDTP_ERR_INVALID, "gdtp_server_add_model: bad arguments");
    for (int64_t i = 0; i < 3 * nt; i++)
      if (triangles[i] < 0 || triangles[i] >= nv) return fail(GDTP_ERR_INVALID, "gdtp_server_add_model: triangle index out of range");
    Mesh mesh;
    mesh.vertices.assign(vertices, vertices + 3 * nv);
    mesh.triangles.assign(triangles, triangles + 3 * nt);
    mesh.uv.assign(uv, uv + 6 * nt);
    std::string err;
    const int id = s->s->add_model(mesh, width, height, levels, kind, weight, second, parameter_metric, err);
    if (id < 0) return fail(GDTP_ERR_SETUP, err);
    *model_out = id;
    return GDTP_OK;
  });
}

extern "C" int gdtp_server_model_texels(gdtp_server* s, int model, int64_t* texels) {
  return guarded("gdtp_server_model_texels", [&]() -> int {
    if (!s || !s->s || !texels) return fail(GDTP_ERR_INVALID, "gdtp_server_model_texels: bad arguments");
    *texels = s->s->model_texels(model);
    return *texels < 0 ? fail(GDTP_ERR_INVALID, "unknown model") : GDTP_OK;
  });
}

extern "C" int gdtp_server_model_bytes(gdtp_server* s, int model, int64_t* bytes) {
  return guarded("gdtp_server_model_bytes", [&]() -> int {
    if (!s || !s->s || !bytes) return fail(GDTP_ERR_INVALID, "gdtp_server_model_bytes: bad arguments");
    *bytes = s->s->model_bytes(model);
    return *bytes < 0 ? fail(GDTP_ERR_INVALID, "unknown model") : GDTP_OK;
  });
}

extern "C" int gdtp_server_warm(gdtp_server* s, int model) {
  return guarded("gdtp_server_warm", [&]() -> int {
    if (!s || !s->s) return fail(GDTP_ERR_INVALID, "gdtp_server_warm: null server");
    std::string err;
    if (s->s->warm(model, err)) return GDTP_OK;
    return fail(err.find("budget") != std::string::npos ? GDTP_ERR_BUDGET : GDTP_ERR_CUDA, err);
  });
}

extern "C" int gdtp_server_submit(gdtp_server* s, int model, const double* signal, const int32_t* sources, int k, double tol,
                                  int max_iters, int64_t* request_out) {
  return guarded("gdtp_server_submit", [&]() -> int {
    if (!s || !s->s || !request_out) return fail(GDTP_ERR_INVALID, "gdtp_server_submit: bad arguments");
    std::string err;
    const int64_t id = s->s->submit(model, signal, sources, k, tol, max_iters, err);
    if (id < 0) return fail(GDTP_ERR_INVALID, err);
    *request_out = id;
    return GDTP_OK;
  });
}

extern "C" int gdtp_server_poll(gdtp_server* s, int64_t request, int* done) {
  return guarded("gdtp_server_poll", [&]() -> int {
    if (!s || !s->s || !done) return fail(GDTP_ERR_INVALID, "gdtp_server_poll: bad arguments");
    bool d = false;
    if (!s->s->poll(request, d)) return fail(GDTP_ERR_INVALID, "unknown request");
    *done = d ? 1 : 0;
    return GDTP_OK;
  });
}

extern "C" int gdtp_server_wait(gdtp_server* s, int64_t request, double* out, gdtp_report* report, double* timing) {
  return guarded("gdtp_server_wait", [&]() -> int {
    if (!s || !s->s) return fail(GDTP_ERR_INVALID, "gdtp_server_wait: null server");
    ServerRequest r;
    std::string err;
    if (!s->s->wait(request, r, err)) return fail(GDTP_ERR_INVALID, err);
    if (out && !r.x.empty()) std::memcpy(out, r.x.data(), r.x.size() * sizeof(double));
    if (report) {
      report->iterations = r.rep.iterations;
      report->vcycles = r.rep.vcycles;
      report->rel_residual_max = r.rep.relMax;
      report->seconds = r.rep.seconds;
    }
    if (timing) {  // {latency ms, queue ms, batch size}
      timing[0] = (r.tEnd - r.tSubmit) * 1e3;
      timing[1] = (r.tStart - r.tSubmit) * 1e3;
      timing[2] = r.batchSize;
    }
    return r.status == GDTP_OK ? GDTP_OK : fail(r.status, r.error.empty() ? "request failed" : r.error);
  });
}

extern "C" int gdtp_server_stats(gdtp_server* s, double* stats) {
  return guarded("gdtp_server_stats", [&]() -> int {
    if (!s || !s->s || !stats) return fail(GDTP_ERR_INVALID, "gdtp_server_stats: bad arguments");
    const ServerStats t = s->s->stats();
    const double v[14] = {double(t.completed), double(t.failed), t.p50Ms, t.p99Ms, t.meanMs, t.texelRhsPerSec, double(t.batches),
                          double(t.batchedRequests), double(t.evictions), double(t.builds), double(t.residentBytes),
                          double(t.peakBytes), double(t.budget), 0.0};
    std::memcpy(stats, v, sizeof(v));
    return GDTP_OK;
  });
}
