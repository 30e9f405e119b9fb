// Atlas construction from per-corner texture coordinates.
//
// Follows the reference's chart decomposition and atlas indexing so that every
// downstream index (charts, chart vertices, atlas edges, boundary half-edges)
// is identical:
//   chart components           Src/ChartDecomposition.h:30-73
//   atlas vertices / edges     Src/AtlasMesh.inl:3-101
//   boundary half-edges        Src/AtlasMesh.inl:103-163
//   boundary vertices          Src/AtlasMesh.inl:165-184
//   chart tables, grid origin  Src/AtlasCharts.inl:3-76
#include <cmath>
#include <cstring>
#include <queue>
#include <vector>

#include "setup.h"

namespace gdtp {

// Directed edges (a, b) of a triangle list, grouped by their first vertex:
// edge lookups scan the few edges leaving a vertex instead of hashing.
struct DirectedEdges {
  std::vector<int> start;              // vertex -> first outgoing edge (nv + 1)
  std::vector<int> to, halfEdge;       // per outgoing edge: end vertex, half-edge 3 t + k
  // false on a repeated directed edge
  bool build(const int* tri, int nt, int nv) {
    start.assign(size_t(nv) + 1, 0);
    for (int h = 0; h < 3 * nt; h++) start[size_t(tri[h]) + 1]++;
    for (int v = 0; v < nv; v++) start[v + 1] += start[v];
    to.resize(3 * size_t(nt));
    halfEdge.resize(3 * size_t(nt));
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (int t = 0; t < nt; t++)
      for (int k = 0; k < 3; k++) {
        const int a = tri[3 * t + k], b = tri[3 * t + (k + 1) % 3];
        for (int e = start[a]; e < fill[a]; e++)
          if (to[e] == b) return false;
        to[fill[a]] = b;
        halfEdge[fill[a]++] = 3 * t + k;
      }
    return true;
  }
  int find(int a, int b) const {
    for (int e = start[a]; e < start[a + 1]; e++)
      if (to[e] == b) return halfEdge[e];
    return -1;
  }
};

static bool same_uv(const V2& a, const V2& b) { return a.x == b.x && a.y == b.y; }

bool build_atlas(const Mesh& mesh, int width, int height, Atlas& A, std::string& err) {
  const int nt = mesh.nt();
  A.width = width;
  A.height = height;
  const int* T = mesh.triangles.data();

  // directed half-edge table of the input mesh
  DirectedEdges half;
  if (!half.build(T, nt, mesh.nv())) { err = "non-manifold mesh (repeated directed edge)"; return false; }
  auto opposite = [&](int t, int k) -> int { return half.find(T[3 * t + (k + 1) % 3], T[3 * t + k]); };
  // an edge is interior to a chart when its twin carries the same texture coordinates
  auto uv_continuous = [&](int t, int k, int o) {
    int s = o / 3, m = o % 3;
    return same_uv(mesh.corner(t, (k + 1) % 3), mesh.corner(s, m)) && same_uv(mesh.corner(t, k), mesh.corner(s, (m + 1) % 3));
  };

  // ---- charts: edge-connected components with continuous texture coordinates
  A.triangleChart.assign(nt, -1);
  int comp = -1;
  std::vector<int> nb;
  for (int seed = 0; seed < nt; seed++) {
    if (A.triangleChart[seed] != -1) continue;
    comp++;
    std::queue<int> q;
    A.triangleChart[seed] = comp;
    q.push(seed);
    while (!q.empty()) {
      int t = q.front();
      q.pop();
      for (int k = 0; k < 3; k++) {
        int o = opposite(t, k);
        if (o < 0 || !uv_continuous(t, k, o)) continue;
        int s = o / 3;
        if (A.triangleChart[s] == -1) { A.triangleChart[s] = comp; q.push(s); }
        else if (A.triangleChart[s] != comp) { err = "inconsistent chart components"; return false; }
      }
    }
  }
  A.numCharts = comp + 1;

  // ---- atlas vertices: one per distinct (texture coordinate, mesh vertex) pair,
  // first-seen order; the atlas vertices of a mesh vertex are chained
  // (bitwise comparison of the coordinates)
  A.triangles.resize(nt);
  {
    std::vector<int> firstOf(mesh.nv(), -1), nextOf;
    for (int t = 0; t < nt; t++)
      for (int k = 0; k < 3; k++) {
        const V2 p = mesh.corner(t, k);
        const int m = T[3 * t + k];
        int id = firstOf[m];
        while (id != -1 && std::memcmp(&A.vertices[id], &p, sizeof(V2)) != 0) id = nextOf[id];
        if (id == -1) {
          id = (int)A.vertices.size();
          A.vertices.push_back(p);
          A.vertexMap.push_back(m);
          nextOf.push_back(firstOf[m]);
          firstOf[m] = id;
        }
        A.triangles[t][k] = id;
      }
  }

  // ---- vertices within 1e-6 texel of a texel-centre line are moved off it
  // (the reference does this with rand(); a deterministic offset keeps the atlas
  // reproducible -- inputs from the bundled generators never need it)
  const double precision = 1e-6;
  for (size_t i = 0; i < A.vertices.size(); i++)
    for (int c = 0; c < 2; c++) {
      double dim = c == 0 ? double(width) : double(height);
      double scaled = A.vertices[i][c] * dim - 0.5;
      double off = scaled - double(std::round(scaled));
      if (std::fabs(off) < precision) {
        double h = 1.0 + double((i * 2654435761u + c) % 1000) / 1000.0;
        scaled = off > 0 ? std::round(scaled) + precision * h : std::round(scaled) - precision * h;
        A.vertices[i][c] = (scaled + 0.5) / dim;
        A.gridJitterCount++;
      }
    }

  // ---- atlas edge indices
  std::vector<int> atlasTri(3 * size_t(nt));
  for (int t = 0; t < nt; t++)
    for (int k = 0; k < 3; k++) atlasTri[3 * t + k] = A.triangles[t][k];
  DirectedEdges ahalf;
  if (!ahalf.build(atlasTri.data(), nt, (int)A.vertices.size())) { err = "non-oriented-manifold atlas"; return false; }
  const int res = std::max(width, height);
  int nextEdge = 2 * res * res * A.numCharts;
  A.halfEdgeToEdgeIndex.assign(3 * nt, -1);
  for (int t = 0; t < nt; t++)
    for (int k = 0; k < 3; k++) {
      int cur = 3 * t + k;
      const int o = ahalf.find(A.triangles[t][(k + 1) % 3], A.triangles[t][k]);
      if (o >= 0) {
        if (cur < o) A.halfEdgeToEdgeIndex[cur] = A.halfEdgeToEdgeIndex[o] = nextEdge++;
      } else {
        A.halfEdgeToEdgeIndex[cur] = nextEdge++;
      }
    }

  // ---- boundary half-edges of the input mesh (open edges and texture seams)
  A.oppositeHalfEdge.assign(3 * nt, -1);
  A.isBoundaryHalfEdge.assign(3 * nt, 0);
  A.isClosed = true;
  std::vector<int> boundaryHalfEdges;
  for (int t = 0; t < nt; t++)
    for (int k = 0; k < 3; k++) {
      int cur = 3 * t + k;
      int o = opposite(t, k);
      if (o >= 0) {
        if (cur < o) { A.oppositeHalfEdge[cur] = o; A.oppositeHalfEdge[o] = cur; }
        if (!uv_continuous(t, k, o) && cur < o) {
          boundaryHalfEdges.push_back(cur);
          boundaryHalfEdges.push_back(o);
          A.isBoundaryHalfEdge[cur] = A.isBoundaryHalfEdge[o] = 1;
        }
      } else {
        A.isClosed = false;
        boundaryHalfEdges.push_back(cur);
        A.isBoundaryHalfEdge[cur] = 1;
      }
    }
  A.boundaryVertexIndex.assign(mesh.nv(), -1);
  A.numBoundaryVertices = 0;
  for (int he : boundaryHalfEdges) {
    int t = he / 3, k = he % 3;
    for (int e = 0; e < 2; e++) {
      int v = T[3 * t + (k + e) % 3];
      if (A.boundaryVertexIndex[v] == -1) A.boundaryVertexIndex[v] = A.numBoundaryVertices++;
    }
  }

  // ---- chart tables
  A.charts.assign(A.numCharts, AtlasChart());
  for (auto& c : A.charts) { c.minCorner = V2(1, 1); c.maxCorner = V2(0, 0); }
  std::vector<int> chartVertex(A.vertices.size(), -1), chartVertexCount(A.numCharts, 0);
  for (int t = 0; t < nt; t++) {
    AtlasChart& C = A.charts[A.triangleChart[t]];
    C.meshTriangleIndices.push_back(t);
    I3 tri;
    for (int k = 0; k < 3; k++) {
      C.atlasEdgeIndices.push_back(A.halfEdgeToEdgeIndex[3 * t + k]);
      int av = A.triangles[t][k];
      if (chartVertex[av] == -1) {
        chartVertex[av] = chartVertexCount[A.triangleChart[t]]++;
        V2 p = A.vertices[av];
        for (int c = 0; c < 2; c++) {
          C.minCorner[c] = std::min(p[c], C.minCorner[c]);
          C.maxCorner[c] = std::max(p[c], C.maxCorner[c]);
        }
        C.vertices.push_back(p);
        C.meshVertexIndices.push_back(A.vertexMap[av]);
      }
      tri[k] = chartVertex[av];
    }
    C.triangles.push_back(tri);
  }
  // grid origin as the reference's release build computes it: its Makefile
  // builds with -ffast-math, which turns the loop-invariant divisions by width
  // and height into multiplies by their reciprocals (exact for powers of two,
  // the last bit may differ otherwise)
  const double invW = 1.0 / double(width), invH = 1.0 / double(height);
  for (auto& C : A.charts) {
    V2 mid = (C.minCorner + C.maxCorner) / 2.0;
    mid.x *= double(width);
    mid.y *= double(height);
    mid = mid - V2(0.5, 0.5);
    mid = V2(std::floor(mid.x), std::floor(mid.y));
    C.originCoords[0] = int(std::round(mid.x));
    C.originCoords[1] = int(std::round(mid.y));
    mid = mid + V2(0.5, 0.5);
    mid.x *= invW;
    mid.y *= invH;
    C.gridOrigin = mid;
    for (size_t t = 0; t < C.meshTriangleIndices.size(); t++)
      for (int k = 0; k < 3; k++)
        if (A.isBoundaryHalfEdge[3 * C.meshTriangleIndices[t] + k]) C.boundaryHalfEdges.push_back(3 * int(t) + k);
  }
  return true;
}

}  // namespace gdtp
