// C ABI: hierarchy construction and host-array getters (no CUDA involved).
#include <cstring>
#include <memory>
#include <string>

#include "gdtp.h"
#include "capi_internal.h"

namespace gdtp {
thread_local std::string g_last_error;
int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
}  // namespace gdtp

using namespace gdtp;

extern "C" const char* gdtp_last_error(void) { return g_last_error.c_str(); }
extern "C" int gdtp_version(void) { return 1; }

extern "C" int gdtp_hierarchy_build(const double* vertices, int64_t nv, const int32_t* triangles, int64_t nt, const double* uv,
                                    int width, int height, int levels, const int32_t* block_info, gdtp_hierarchy** out) {
  return guarded("gdtp_hierarchy_build", [&]() -> int {
    if (!out || !vertices || !triangles || !uv || nv <= 0 || nt <= 0 || width <= 1 || height <= 1 || levels < 1 || levels > 16)
      return fail(GDTP_ERR_INVALID, "gdtp_hierarchy_build: invalid arguments");
    *out = nullptr;
    std::unique_ptr<gdtp_hierarchy> h(new gdtp_hierarchy());
    h->mesh.vertices.assign(vertices, vertices + nv * 3);
    h->mesh.triangles.assign(triangles, triangles + nt * 3);
    h->mesh.uv.assign(uv, uv + nt * 6);
    for (int64_t i = 0; i < nt * 3; i++)
      if (triangles[i] < 0 || triangles[i] >= nv) return fail(GDTP_ERR_INVALID, "gdtp_hierarchy_build: triangle index out of range");
    BlockInfo info;
    if (block_info) {
      info.blockWidth = block_info[0];
      info.blockHeight = block_info[1];
      info.paddingWidth = block_info[2];
      info.paddingHeight = block_info[3];
      info.boundaryDilation = block_info[4];
    }
    h->width = width;
    h->height = height;
    // levels beyond the requested ones are added until the coarsest level is small
    // enough for the dense direct solve of the device V-cycle
    if (!build_hierarchy(h->mesh, width, height, levels, info, h->h, 2600, 12)) return fail(GDTP_ERR_SETUP, "hierarchy: " + h->h.error);
    std::string err;
    if (!build_boundary_elements(h->h, h->be, err)) return fail(GDTP_ERR_SETUP, "boundary elements: " + err);
    *out = h.release();
    return GDTP_OK;
  });
}

extern "C" void gdtp_hierarchy_free(gdtp_hierarchy* h) { delete h; }
extern "C" int gdtp_hierarchy_levels(const gdtp_hierarchy* h) { return h ? (int)h->h.levels.size() : 0; }
extern "C" int gdtp_hierarchy_charts(const gdtp_hierarchy* h) { return h ? h->h.atlas.numCharts : 0; }

extern "C" int gdtp_hierarchy_counts(const gdtp_hierarchy* h, int level, int64_t* c) {
  return guarded("gdtp_hierarchy_counts", [&]() -> int {
    if (!h || !c || level < 0 || level >= (int)h->h.levels.size()) return fail(GDTP_ERR_INVALID, "gdtp_hierarchy_counts: bad level");
    const GridLevel& L = h->h.levels[level];
    int64_t v[8] = {L.numTexels, L.numDeep, L.numBoundary, L.numCells, L.numBoundaryCells, L.numInteriorCells, L.numInteriorTexels,
                    h->h.atlas.numCharts};
    std::memcpy(c, v, sizeof(v));
    return GDTP_OK;
  });
}

namespace {
template <class T, class F>
int emit(void* out, int64_t* count, int64_t n, F&& f) {
  if (count) *count = n;
  if (out) {
    T* o = static_cast<T*>(out);
    for (int64_t i = 0; i < n; i++) o[i] = f(i);
  }
  return GDTP_OK;
}
template <class T>
int emit_vec(void* out, int64_t* count, const std::vector<T>& v) {
  if (count) *count = (int64_t)v.size();
  if (out && !v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(T));
  return GDTP_OK;
}
}  // namespace

int gdtp::emit_csr(const Csr& m, const std::string& part, void* out, int64_t* count) {
  if (part == "ptr") return emit_vec(out, count, m.ptr);
  if (part == "col") return emit_vec(out, count, m.col);
  if (part == "val") return emit_vec(out, count, m.val);
  return fail(GDTP_ERR_INVALID, "unknown CSR part " + part);
}

extern "C" int gdtp_hierarchy_array(const gdtp_hierarchy* h, const char* cname, int level, void* out, int64_t* count) {
  return guarded("gdtp_hierarchy_array", [&]() -> int {
    if (!h || !cname || level < 0 || level >= (int)h->h.levels.size()) return fail(GDTP_ERR_INVALID, "gdtp_hierarchy_array: bad arguments");
    const std::string name(cname);
    const GridLevel& L = h->h.levels[level];
    if (name == "nodeinfo")
      return emit<int32_t>(out, count, 4 * (int64_t)L.nodes.size(), [&](int64_t i) {
        const NodeInfo& n = L.nodes[i / 4];
        int v[4] = {n.chart, n.ci, n.cj, n.type};
        return v[i % 4];
      });
    if (name == "boundaryAndDeep") return emit_vec(out, count, L.boundaryAndDeep);
    if (name == "boundaryGlobal") return emit_vec(out, count, L.boundaryGlobal);
    if (name == "deepGlobal") return emit_vec(out, count, L.deepGlobal);
    auto lines5 = [&](const std::vector<Line>& v) {
      return emit<int32_t>(out, count, 5 * (int64_t)v.size(), [&](int64_t i) {
        const Line& l = v[i / 5];
        int a[5] = {l.start, l.end, l.prev, l.next, l.coeff};
        return a[i % 5];
      });
    };
    if (name == "rasterLines") return lines5(L.rasterLines);
    if (name == "restrictionLines") return lines5(L.restrictionLines);
    if (name == "interiorTexelToCellLines") {
      // InitializeInteriorTexelToCellLines (InteriorTexelToCellLines.inl:3-29): per
      // raster line its texels, coefficient offset, and the global index of the
      // first cell of the row above (cells (ci-1, cj-1)...) and below ((ci-1, cj)...)
      if (level != 0) return fail(GDTP_ERR_INVALID, "interiorTexelToCellLines exist on level 0 only");
      return emit<int32_t>(out, count, 5 * (int64_t)L.rasterLines.size(), [&](int64_t i) {
        const Line& r = L.rasterLines[i / 5];
        const NodeInfo& n = L.nodes[r.start];
        const GridChart& c = L.charts[n.chart];
        const int prev = c.localCell[(n.cj - 1) * (c.width - 1) + (n.ci - 1)] + c.cellOffset;
        const int next = c.localCell[n.cj * (c.width - 1) + (n.ci - 1)] + c.cellOffset;
        const int a[5] = {r.start, r.end, r.coeff, prev, next};
        return a[i % 5];
      });
    }
    if (name == "deepLines")
      return emit<int32_t>(out, count, 5 * (int64_t)L.deepLines.size(), [&](int64_t i) {
        const DeepLine& l = L.deepLines[i / 5];
        int a[5] = {l.coarseStart, l.coarseEnd, l.finePrev, l.fineCurrent, l.fineNext};
        return a[i % 5];
      });
    if (name == "prolongationLines")
      return emit<int32_t>(out, count, 6 * (int64_t)L.prolongationLines.size(), [&](int64_t i) {
        const ProlongationLine& l = L.prolongationLines[i / 6];
        int a[6] = {l.start, l.length, l.center, l.prev, l.next, l.aligned};
        return a[i % 6];
      });
    if (name == "charts")
      return emit<int32_t>(out, count, 12 * (int64_t)L.charts.size(), [&](int64_t i) {
        const GridChart& c = L.charts[i / 12];
        int a[12] = {c.cornerCoords[0], c.cornerCoords[1], c.centerOffset[0], c.centerOffset[1], c.width, c.height,
                     c.texelOffset, c.deepOffset, c.boundaryOffset, c.cellOffset, c.numInteriorCells, c.numBoundaryCells};
        return a[i % 12];
      });
    if (name == "chartsd")
      return emit<double>(out, count, 4 * (int64_t)L.charts.size(), [&](int64_t i) {
        const GridChart& c = L.charts[i / 4];
        double a[4] = {c.corner.x, c.corner.y, c.cellSizeW, c.cellSizeH};
        return a[i % 4];
      });
    if (name == "nodeType" || name == "cellType" || name == "cellCorners") {
      std::vector<int> all;
      for (const GridChart& c : L.charts) {
        const std::vector<int>& v = name == "nodeType" ? c.nodeType : name == "cellType" ? c.cellType : c.cellCorners;
        all.insert(all.end(), v.begin(), v.end());
      }
      return emit_vec(out, count, all);
    }
    if (name == "textureNodes" || name == "textureBary") {
      if (level != 0) return fail(GDTP_ERR_INVALID, "texture nodes exist on level 0 only");
      std::vector<int> ti;
      std::vector<double> tb;
      for (size_t c = 0; c < L.charts.size(); c++) {
        const GridChart& g = L.charts[c];
        for (int j = 0; j < g.height; j++)
          for (int i = 0; i < g.width; i++) {
            int n = g.at(i, j);
            if (g.texel[n] == -1) continue;
            ti.insert(ti.end(), {g.cornerCoords[0] + i, g.cornerCoords[1] + j, (int)c, g.triangleId[n], g.nodeType[n] > 0 ? 1 : 0});
            tb.insert(tb.end(), {g.bary[n].x, g.bary[n].y});
          }
      }
      return name == "textureNodes" ? emit_vec(out, count, ti) : emit_vec(out, count, tb);
    }
    if (name.rfind("boundaryRestriction.", 0) == 0) return emit_csr(L.boundaryRestriction, name.substr(20), out, count);
    if (name == "boundaryNodes") {
      const BoundaryElements& be = h->be;
      std::vector<int> v = {be.numBoundaryNodes, be.numMidPoints, be.numFineNodes, be.numFineBoundary};
      return emit_vec(out, count, v);
    }
    if (name.rfind("boundaryProlongation.", 0) == 0) return emit_csr(h->be.prolongation, name.substr(21), out, count);
    return fail(GDTP_ERR_INVALID, "gdtp_hierarchy_array: unknown array " + name);
  });
}

extern "C" int gdtp_texel_signal(const gdtp_hierarchy* h, const void* texture, int width, int height, int channels, int bytes_per_value,
                                 int64_t row_stride, int64_t pixel_stride, int64_t channel_stride, double* out) {
  return guarded("gdtp_texel_signal", [&]() -> int {
    if (!h || !texture || !out || width <= 0 || height <= 0 || channels <= 0 || (bytes_per_value != 4 && bytes_per_value != 8))
      return fail(GDTP_ERR_INVALID, "gdtp_texel_signal: bad arguments");
    const GridLevel& L = h->h.levels[0];
    const int nCharts = (int)L.charts.size();
    bool outside = false;
#pragma omp parallel for schedule(dynamic, 1) reduction(||: outside)
    for (int c = 0; c < nCharts; c++) {
      const GridChart& g = L.charts[c];
      for (int j = 0; j < g.height; j++)
        for (int i = 0; i < g.width; i++) {
          const int t = g.texel[g.at(i, j)];
          if (t == -1) continue;
          const int x = g.cornerCoords[0] + i, y = g.cornerCoords[1] + j;
          if (x < 0 || y < 0 || x >= width || y >= height) { outside = true; continue; }
          const char* px = static_cast<const char*>(texture) + int64_t(y) * row_stride + int64_t(x) * pixel_stride;
          for (int q = 0; q < channels; q++) {
            const char* v = px + int64_t(q) * channel_stride;
            out[size_t(t) * channels + q] = bytes_per_value == 4 ? double(*reinterpret_cast<const float*>(v)) : *reinterpret_cast<const double*>(v);
          }
        }
    }
    if (outside) return fail(GDTP_ERR_INVALID, "gdtp_texel_signal: a texel lies outside the texture");
    return GDTP_OK;
  });
}
