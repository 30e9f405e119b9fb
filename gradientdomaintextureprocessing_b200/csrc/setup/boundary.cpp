// Boundary-cell elements of the finest level: the part of every boundary cell
// covered by its chart, cut into triangles that carry quadratic (6-node)
// elements, the auxiliary nodes those elements add, and the prolongation from
// boundary texels to all fine boundary nodes.
//
// Restates the reference algorithm:
//   boundary edge / grid intersections    Src/BoundaryQuadraticElements.inl:37-167
//   cell polygons and seam node insertion Src/BoundaryQuadraticElements.inl:196-521
//   indexed cell/triangle clipping        Src/PolygonClipping.h:434-566
//   quadratic elements + mid-edge nodes   Src/BoundaryQuadraticElements.inl:525-616
//   texel -> fine boundary prolongation   Src/BoundaryQuadraticElements.inl:652-772
// Two deliberate differences, both without effect on the assembled operator
// beyond rounding:
//   * polygons are triangulated by the constrained Delaunay triangulation
//     computed here (ear clipping + Lawson flips) instead of the vendored
//     Triangle library (ConstrainedTriangulation.h:14-68); for points in general
//     position the CDT is unique, so the triangles are the same, only their
//     order (and hence mid-edge node numbering) differs;
//   * seam nodes inserted on a boundary segment are placed exactly on it; the
//     reference adds a rand()-driven 1e-10 perpendicular offset
//     (BoundaryQuadraticElements.inl:433-436) only to shield Triangle from
//     collinear input, which the triangulator here handles directly.
#include <algorithm>
#include <cmath>
#include <unordered_map>
#include <unordered_set>
#include <cstdio>
#include <cstdlib>

#include "setup.h"

namespace gdtp {

static const uint32_t kNone = 0xFFFFFFFFu;
static inline uint64_t pair_key(uint32_t a, uint32_t b) { return (uint64_t(a) << 32) | uint64_t(b); }
static inline uint32_t key_hi(uint64_t k) { return uint32_t(k >> 32); }
static inline uint32_t key_lo(uint64_t k) { return uint32_t(k & 0xFFFFFFFFu); }

struct Intersection {
  uint64_t key;
  int node;
  V2 pos;
  double time;
};
struct SegmentInfo {
  double t0, t1;
  int halfEdge;
};

// ----------------------------------------------------------------------------
// polygon clipped against a triangle, vertices carrying combinatorial keys
// ----------------------------------------------------------------------------
struct KeyedPolygon {
  std::vector<V2> v;
  std::vector<uint64_t> key;
  std::vector<int> edge;  // edge[i] joins vertex i and i+1
};

static void clip_keyed(KeyedPolygon& p, const V2& normal, double offset, int edgeIndex) {
  const int n = (int)p.v.size();
  if (n == 0) return;
  KeyedPolygon o;
  V2 prev = p.v[n - 1];
  uint64_t prevKey = p.key[n - 1];
  int nextEdge = p.edge[n - 1];
  double prevLevel = dot(prev, normal) - offset;
  bool prevIn = prevLevel > 0;
  for (int i = 0; i < n; i++) {
    V2 cur = p.v[i];
    uint64_t curKey = p.key[i];
    int prevEdge = nextEdge;
    nextEdge = p.edge[i];
    double curLevel = dot(cur, normal) - offset;
    bool curIn = curLevel > 0;
    if (!prevIn) {
      if (curIn) {
        double a = -curLevel / (prevLevel - curLevel);
        o.v.push_back(prev * a + cur * (1.0 - a));
        o.key.push_back(pair_key(uint32_t(edgeIndex), uint32_t(prevEdge)));
        o.edge.push_back(prevEdge);
      }
    } else {
      o.v.push_back(prev);
      o.key.push_back(prevKey);
      o.edge.push_back(prevEdge);
      if (!curIn) {
        double a = -curLevel / (prevLevel - curLevel);
        o.v.push_back(prev * a + cur * (1.0 - a));
        o.key.push_back(pair_key(uint32_t(edgeIndex), uint32_t(prevEdge)));
        o.edge.push_back(edgeIndex);
      }
    }
    prev = cur;
    prevLevel = curLevel;
    prevKey = curKey;
    prevIn = curIn;
  }
  p = std::move(o);
}

// Clips the polygon to a triangle whose corners have keys tkey[] and edges tedge[]
// (edge k joins corner k and k+1).  Intersection keys that name a triangle corner
// (two triangle edges) are replaced by the corner's key.
static void clip_to_triangle(KeyedPolygon& p, const V2 tv[3], const uint64_t tkey[3], const int tedge[3]) {
  V2 centre = (tv[0] + tv[1] + tv[2]) / 3.0;
  uint64_t cornerKeys[6], cornerIdx[6];
  for (int k = 0; k < 3; k++) {
    cornerKeys[2 * k] = pair_key(uint32_t(tedge[k]), uint32_t(tedge[(k + 2) % 3]));
    cornerKeys[2 * k + 1] = pair_key(uint32_t(tedge[(k + 2) % 3]), uint32_t(tedge[k]));
    cornerIdx[2 * k] = cornerIdx[2 * k + 1] = tkey[k];
  }
  bool reversed = false;
  for (int k = 0; k < 3; k++) {
    V2 dir = tv[(k + 1) % 3] - tv[k];
    V2 mid = (tv[(k + 1) % 3] + tv[k]) / 2.0;
    V2 nrm(-dir.y, dir.x);
    nrm = nrm / std::sqrt(nrm.x * nrm.x + nrm.y * nrm.y);
    double off = dot(mid, nrm);
    if (dot(centre, nrm) < off) { nrm = nrm * -1.0; off = -off; reversed = true; }
    clip_keyed(p, nrm, off, tedge[k]);
  }
  for (auto& k : p.key)
    for (int c = 0; c < 6; c++)
      if (k == cornerKeys[c]) k = cornerIdx[c];
  if (reversed) {
    int n = (int)p.v.size();
    KeyedPolygon r;
    r.v.resize(n); r.key.resize(n); r.edge.resize(n);
    for (int k = 0; k < n; k++) {
      r.v[k] = p.v[n - 1 - k];
      r.key[k] = p.key[n - 1 - k];
      r.edge[k] = p.edge[(2 * n - k - 2) % n];
    }
    p = std::move(r);
  }
}

// ----------------------------------------------------------------------------
// constrained Delaunay triangulation of a simple polygon (small n)
// ----------------------------------------------------------------------------
static double orient(const V2& a, const V2& b, const V2& c) { return (b.x - a.x) * (c.y - a.y) - (b.y - a.y) * (c.x - a.x); }
static double incircle(const V2& a, const V2& b, const V2& c, const V2& d) {
  double adx = a.x - d.x, ady = a.y - d.y, bdx = b.x - d.x, bdy = b.y - d.y, cdx = c.x - d.x, cdy = c.y - d.y;
  double ad = adx * adx + ady * ady, bd = bdx * bdx + bdy * bdy, cd = cdx * cdx + cdy * cdy;
  return adx * (bdy * cd - bd * cdy) - ady * (bdx * cd - bd * cdx) + ad * (bdx * cdy - bdy * cdx);
}

// Returns counter-clockwise triangles (polygon vertex ids); false if the polygon
// could not be fully triangulated (self-intersecting input).
static bool triangulate_polygon(const std::vector<V2>& in, std::vector<I3>& tris) {
  tris.clear();
  const int n = (int)in.size();
  if (n < 3) return false;
  // local frame: translate and scale for well-conditioned predicates
  double minx = in[0].x, miny = in[0].y, maxx = in[0].x, maxy = in[0].y;
  for (auto& p : in) { minx = std::min(minx, p.x); miny = std::min(miny, p.y); maxx = std::max(maxx, p.x); maxy = std::max(maxy, p.y); }
  double s = std::max(maxx - minx, maxy - miny);
  if (!(s > 0)) return false;
  double area = 0;
  for (int i = 0; i < n; i++) area += (in[i].x - minx) * (in[(i + 1) % n].y - miny) - (in[(i + 1) % n].x - minx) * (in[i].y - miny);
  // work on a counter-clockwise copy Q; perm maps Q ids back to input ids
  std::vector<int> perm(n);
  for (int i = 0; i < n; i++) perm[i] = area >= 0 ? i : n - 1 - i;
  std::vector<V2> Q(n);
  for (int i = 0; i < n; i++) Q[i] = V2((in[perm[i]].x - minx) / s, (in[perm[i]].y - miny) / s);
  const double eps = 1e-10;  // relative to the polygon extent; absorbs rounding of seam nodes placed on segments

  std::vector<int> ring(n);
  for (int i = 0; i < n; i++) ring[i] = i;
  while (ring.size() > 3) {
    const int m = (int)ring.size();
    int best = -1;
    double bestScore = -1;
    for (int q = 0; q < m; q++) {
      int a = ring[(q + m - 1) % m], b = ring[q], c = ring[(q + 1) % m];
      double o = orient(Q[a], Q[b], Q[c]);
      if (o <= eps) continue;  // reflex or flat corner
      bool empty = true;
      for (int r = 0; r < m && empty; r++) {
        int d = ring[r];
        if (d == a || d == b || d == c) continue;
        if (orient(Q[a], Q[b], Q[d]) >= -eps && orient(Q[b], Q[c], Q[d]) >= -eps && orient(Q[c], Q[a], Q[d]) >= -eps) empty = false;
      }
      if (!empty) continue;
      double l2 = (Q[b].x - Q[a].x) * (Q[b].x - Q[a].x) + (Q[b].y - Q[a].y) * (Q[b].y - Q[a].y) +
                  (Q[c].x - Q[b].x) * (Q[c].x - Q[b].x) + (Q[c].y - Q[b].y) * (Q[c].y - Q[b].y) +
                  (Q[a].x - Q[c].x) * (Q[a].x - Q[c].x) + (Q[a].y - Q[c].y) * (Q[a].y - Q[c].y);
      double score = o / l2;  // prefer well-shaped ears
      if (score > bestScore) { bestScore = score; best = q; }
    }
    if (best < 0) return false;
    const int m2 = (int)ring.size();
    tris.push_back(I3{{ring[(best + m2 - 1) % m2], ring[best], ring[(best + 1) % m2]}});
    ring.erase(ring.begin() + best);
  }
  if (orient(Q[ring[0]], Q[ring[1]], Q[ring[2]]) <= eps) return false;
  tris.push_back(I3{{ring[0], ring[1], ring[2]}});

  // Lawson flips of unconstrained diagonals until every one is locally Delaunay
  auto constrained = [&](int a, int b) { return b == (a + 1) % n || a == (b + 1) % n; };
  for (int pass = 0; pass < 16 * n; pass++) {
    bool flipped = false;
    for (size_t t = 0; t < tris.size() && !flipped; t++)
      for (int e = 0; e < 3 && !flipped; e++) {
        int a = tris[t][e], b = tris[t][(e + 1) % 3], c = tris[t][(e + 2) % 3];
        if (constrained(a, b)) continue;
        for (size_t u = 0; u < tris.size(); u++) {
          if (u == t) continue;
          int f = -1;
          for (int g = 0; g < 3; g++)
            if (tris[u][g] == b && tris[u][(g + 1) % 3] == a) f = g;
          if (f < 0) continue;
          int d = tris[u][(f + 2) % 3];
          if (incircle(Q[a], Q[b], Q[c], Q[d]) > 1e-10 && orient(Q[a], Q[d], Q[c]) > eps && orient(Q[d], Q[b], Q[c]) > eps) {
            tris[t] = I3{{a, d, c}};
            tris[u] = I3{{d, b, c}};
            flipped = true;
          }
          break;
        }
      }
    if (!flipped) break;
  }
  for (auto& t : tris)
    for (int k = 0; k < 3; k++) t[k] = perm[t[k]];
  for (auto& t : tris)
    if (orient(in[t[0]], in[t[1]], in[t[2]]) < 0) std::swap(t[1], t[2]);
  return true;
}

// ----------------------------------------------------------------------------
bool build_boundary_elements(const Hierarchy& H, BoundaryElements& be, std::string& err) {
  const Atlas& A = H.atlas;
  const GridLevel& L = H.levels[0];
  const int nCharts = (int)L.charts.size();
  const int numInterior = L.numInteriorTexels;
  be.charts.assign(nCharts, ChartBoundary());
  be.numBoundaryVertices = A.numBoundaryVertices;

  // (1) intersections of boundary edges with grid lines, chart by chart
  int nextNode = A.numBoundaryVertices;
  std::unordered_map<int, std::vector<Intersection>> edgeHits;  // mesh half-edge -> sorted hits
  std::vector<std::unordered_map<uint64_t, SegmentInfo>> segInfo(nCharts);
  std::vector<std::unordered_map<uint64_t, int>> nodeOf(nCharts);
  std::vector<std::unordered_map<uint64_t, V2>> nodePos(nCharts);
  for (int c = 0; c < nCharts; c++) {
    const AtlasChart& ac = A.charts[c];
    const GridChart& g = L.charts[c];
    ChartBoundary& cb = be.charts[c];
    for (int che : ac.boundaryHalfEdges) {
      const int t = che / 3, k = che % 3;
      const int meshHalfEdge = ac.meshTriangleIndices[t] * 3 + k;
      V2 e[2] = {ac.vertices[ac.triangles[t][k]] - g.corner, ac.vertices[ac.triangles[t][(k + 1) % 3]] - g.corner};
      std::vector<Intersection> hits;
      for (int v = 0; v < 2; v++) hits.push_back({pair_key(uint32_t(ac.triangles[t][(k + v) % 3]), kNone), -1, e[v], double(v)});
      const int atlasEdge = ac.atlasEdgeIndices[che];
      double fmn[2], fmx[2];
      for (int d = 0; d < 2; d++) {
        fmn[d] = std::max(std::min(e[0][d], e[1][d]), 0.0);
        fmx[d] = std::min(std::max(e[0][d], e[1][d]), 1.0);
      }
      int imn[2] = {int(std::floor(fmn[0] / g.cellSizeW)), int(std::floor(fmn[1] / g.cellSizeH))};
      int imx[2] = {int(std::floor(fmx[0] / g.cellSizeW)), int(std::floor(fmx[1] / g.cellSizeH))};
      for (int d = 0; d < 2; d++)
        for (int s = imn[d]; s <= imx[d]; s++) {
          double cs = d == 0 ? g.cellSizeW : g.cellSizeH, ocs = d == 0 ? g.cellSizeH : g.cellSizeW;
          double level = double(s) * cs;
          double alpha = (level - e[0][d]) / (e[1][d] - e[0][d]);
          if (alpha > 0 && alpha < 1.0) {
            V2 pos = e[0] * (1.0 - alpha) + e[1] * alpha;
            int other = int(std::floor(pos[1 - d] / ocs));
            int cell[2];
            cell[d] = s;
            cell[1 - d] = other;
            uint32_t gridEdge = uint32_t(g.gridIndexOffset + d * g.width * g.height + cell[0] + cell[1] * g.width);
            hits.push_back({pair_key(uint32_t(atlasEdge), gridEdge), -1, pos, alpha});
          }
        }
      std::sort(hits.begin(), hits.end(), [](const Intersection& a, const Intersection& b) { return a.time < b.time; });
      for (auto& hit : hits) {
        auto it = nodeOf[c].find(hit.key);
        if (it == nodeOf[c].end()) {
          nodePos[c][hit.key] = hit.pos;
          int node;
          if (key_lo(hit.key) == kNone) {
            int meshVertex = ac.meshVertexIndices[key_hi(hit.key)];
            node = A.boundaryVertexIndex[meshVertex];
            if (node < 0) { err = "boundary vertex without index"; return false; }
          } else {
            node = nextNode++;
          }
          nodeOf[c][hit.key] = node;
          cb.aux.push_back({hit.pos, node + numInterior});
          hit.node = node;
        } else {
          hit.node = it->second;
        }
      }
      for (size_t i = 0; i + 1 < hits.size(); i++) {
        uint64_t sk = pair_key(uint32_t(hits[i].node), uint32_t(hits[i + 1].node));
        if (!segInfo[c].emplace(sk, SegmentInfo{hits[i].time, hits[i + 1].time, meshHalfEdge}).second) {
          err = "replicated boundary segment";
          return false;
        }
      }
      edgeHits[meshHalfEdge] = hits;
    }
  }
  be.numBoundaryNodes = nextNode;
  std::vector<int> oppositeCovered(std::max(0, be.numBoundaryNodes - A.numBoundaryVertices), 0);

  // (2) cell polygons: union of (cell ^ triangle) pieces, reduced to grid and boundary nodes
  struct Poly {
    std::vector<V2> v;
    std::vector<int> idx, atlasVertex, atlasEdge, parentEdge;
  };
  std::vector<std::vector<std::vector<Poly>>> cellPolys(nCharts);
  // charts in parallel: each writes its own polygons and auxiliary nodes; the
  // seam-node coverage counts are summed atomically
  std::vector<std::string> chartErr(nCharts);
#pragma omp parallel for schedule(dynamic, 1)
  for (int c = 0; c < nCharts; c++) {
    auto chart_polygons = [&](std::string& err) -> bool {
    const AtlasChart& ac = A.charts[c];
    const GridChart& g = L.charts[c];
    ChartBoundary& cb = be.charts[c];
    std::vector<std::vector<std::pair<uint64_t, uint64_t>>> segs(g.numBoundaryCells);
    for (size_t t = 0; t < ac.triangles.size(); t++) {
      V2 tv[3];
      uint64_t tkey[3];
      int tedge[3];
      for (int k = 0; k < 3; k++) {
        tv[k] = ac.vertices[ac.triangles[t][k]] - g.corner;
        tkey[k] = pair_key(uint32_t(ac.triangles[t][k]), kNone);
        tedge[k] = ac.atlasEdgeIndices[3 * t + k];
      }
      double fmn[2] = {std::max(std::min({tv[0].x, tv[1].x, tv[2].x}), 0.0), std::max(std::min({tv[0].y, tv[1].y, tv[2].y}), 0.0)};
      double fmx[2] = {std::min(std::max({tv[0].x, tv[1].x, tv[2].x}), 1.0), std::min(std::max({tv[0].y, tv[1].y, tv[2].y}), 1.0)};
      int mn[2] = {int(std::floor(fmn[0] * (1.0 / g.cellSizeW))), int(std::floor(fmn[1] * (1.0 / g.cellSizeH)))};
      int mx[2] = {int(std::ceil(fmx[0] * (1.0 / g.cellSizeW))), int(std::ceil(fmx[1] * (1.0 / g.cellSizeH)))};
      for (int j = mn[1]; j < mx[1]; j++)
        for (int i = mn[0]; i < mx[0]; i++) {
          if (g.cellType[g.cat(i, j)] != 0) continue;
          int cell = g.localBoundaryCell[g.cat(i, j)];
          KeyedPolygon p;
          const int W = g.width, Hh = g.height, go = g.gridIndexOffset;
          p.v = {V2(double(i) * g.cellSizeW, double(j) * g.cellSizeH), V2(double(i + 1) * g.cellSizeW, double(j) * g.cellSizeH),
                 V2(double(i + 1) * g.cellSizeW, double(j + 1) * g.cellSizeH), V2(double(i) * g.cellSizeW, double(j + 1) * g.cellSizeH)};
          p.key = {pair_key(kNone, uint32_t(go + i + j * W)), pair_key(kNone, uint32_t(go + i + 1 + j * W)),
                   pair_key(kNone, uint32_t(go + i + 1 + (j + 1) * W)), pair_key(kNone, uint32_t(go + i + (j + 1) * W))};
          p.edge = {go + W * Hh + i + j * W, go + i + 1 + j * W, go + W * Hh + i + (j + 1) * W, go + i + j * W};
          clip_to_triangle(p, tv, tkey, tedge);
          for (size_t s = 0; s < p.key.size(); s++) segs[cell].push_back({p.key[s], p.key[(s + 1) % p.key.size()]});
        }
    }
    cellPolys[c].resize(g.numBoundaryCells);
    for (int cell = 0; cell < g.numBoundaryCells; cell++) {
      auto& S = segs[cell];
      if (S.empty()) continue;
      // boundary of the union: directed segments whose reverse is absent
      std::unordered_set<uint64_t> present;
      std::unordered_map<uint64_t, int> local;
      auto lid = [&](uint64_t k) { auto it = local.find(k); if (it != local.end()) return it->second; int id = (int)local.size(); local.emplace(k, id); return id; };
      std::vector<std::pair<int, int>> ls;
      for (auto& s : S) { int a = lid(s.first), b = lid(s.second); ls.push_back({a, b}); present.insert(pair_key(a, b)); }
      std::unordered_map<uint64_t, uint64_t> fwd;
      std::vector<uint64_t> order;  // deterministic loop starts: first-seen order
      for (size_t k = 0; k < S.size(); k++)
        if (!present.count(pair_key(ls[k].second, ls[k].first))) {
          if (fwd.emplace(S[k].first, S[k].second).second) order.push_back(S[k].first);
        }
      std::unordered_set<uint64_t> visited;
      for (uint64_t start : order) {
        if (visited.count(start)) continue;
        std::vector<uint64_t> loop;
        uint64_t cur = start;
        while (true) {
          if (visited.count(cur)) {
            if (cur != start) { err = "non-simple boundary loop in a cell"; return false; }
            break;
          }
          visited.insert(cur);
          loop.push_back(cur);
          auto it = fwd.find(cur);
          if (it == fwd.end()) { err = "open boundary loop in a cell"; return false; }
          cur = it->second;
        }
        // keep grid nodes and boundary nodes
        Poly P;
        std::vector<uint64_t> keep;
        for (uint64_t k : loop) {
          uint32_t hi = key_hi(k), lo = key_lo(k);
          if (hi == kNone) {
            int v = int(lo) - g.gridIndexOffset, pi = v % g.width, pj = v / g.width;
            int it2 = g.interiorTexel[g.at(pi, pj)];
            if (it2 == -1) { err = "cell polygon corner is not an interior texel"; return false; }
            keep.push_back(k);
            P.v.push_back(V2(double(pi) * g.cellSizeW, double(pj) * g.cellSizeH));
            P.idx.push_back(it2);
            P.atlasVertex.push_back(-1);
          } else if (nodeOf[c].count(k)) {
            keep.push_back(k);
            P.v.push_back(nodePos[c][k]);
            P.idx.push_back(nodeOf[c][k] + numInterior);
            P.atlasVertex.push_back(lo == kNone ? int(hi) : -1);
          }
        }
        if (keep.empty()) { err = "empty reduced cell loop"; return false; }
        // insert the other side's seam nodes on each boundary segment
        const int m = (int)keep.size();
        Poly Q;
        for (int j = 0; j < m; j++) {
          uint64_t ck = keep[j], nk = keep[(j + 1) % m];
          int parent = (key_hi(ck) != kNone && key_lo(ck) != kNone) ? int(key_hi(ck)) : -1;
          int segEdge = -1;
          std::vector<std::pair<double, int>> ins;
          auto ci = nodeOf[c].find(ck), ni = nodeOf[c].find(nk);
          if (ci != nodeOf[c].end() && ni != nodeOf[c].end()) {
            auto si = segInfo[c].find(pair_key(uint32_t(ci->second), uint32_t(ni->second)));
            if (si != segInfo[c].end()) {
              segEdge = A.halfEdgeToEdgeIndex[si->second.halfEdge];
              int opp = A.oppositeHalfEdge[si->second.halfEdge];
              if (opp != -1) {
                auto oh = edgeHits.find(opp);
                if (oh == edgeHits.end()) { err = "opposite edge intersections not found"; return false; }
                const auto& hits = oh->second;
                for (int q = (int)hits.size() - 2; q > 0; q--) {
                  double tt = ((1.0 - hits[q].time) - si->second.t0) / (si->second.t1 - si->second.t0);
                  if (tt > 0 && tt < 1) ins.push_back({tt, hits[q].node});
                }
              }
            }
          }
          Q.v.push_back(P.v[j]);
          Q.idx.push_back(P.idx[j]);
          Q.atlasVertex.push_back(P.atlasVertex[j]);
          Q.atlasEdge.push_back(segEdge);
          Q.parentEdge.push_back(parent);
          for (auto& in : ins) {
            if (in.second < A.numBoundaryVertices || in.second > be.numBoundaryNodes) { err = "seam node index out of range"; return false; }
#pragma omp atomic
            oppositeCovered[in.second - A.numBoundaryVertices]++;
            V2 pos = P.v[j] * (1.0 - in.first) + P.v[(j + 1) % m] * in.first;
            cb.aux.push_back({pos, in.second + numInterior});
            Q.v.push_back(pos);
            Q.idx.push_back(in.second + numInterior);
            Q.atlasVertex.push_back(-1);
            Q.atlasEdge.push_back(segEdge);
            Q.parentEdge.push_back(segEdge);
          }
        }
        cellPolys[c][cell].push_back(std::move(Q));
      }
    }
        return true;
    };
    chart_polygons(chartErr[c]);
  }
  for (const std::string& e : chartErr)
    if (!e.empty()) { err = e; return false; }
  if (A.isClosed)
    for (size_t i = 0; i < oppositeCovered.size(); i++)
      if (oppositeCovered[i] != 1) { err = "seam node " + std::to_string(i) + " not matched on the opposite side"; return false; }

  // (3) quadratic elements: triangulate every cell polygon, add mid-edge nodes
  const int firstMid = be.numBoundaryNodes + numInterior;
  // triangulations of every polygon (charts in parallel), then the mid-edge
  // nodes numbered in chart, cell and polygon order
  std::vector<std::vector<std::vector<std::vector<I3>>>> polyTris(nCharts);
  std::vector<std::vector<std::vector<char>>> polyOk(nCharts);
#pragma omp parallel for schedule(dynamic, 1)
  for (int c = 0; c < nCharts; c++) {
    const int nCells = (int)cellPolys[c].size();
    polyTris[c].resize(nCells);
    polyOk[c].resize(nCells);
    for (int cell = 0; cell < nCells; cell++) {
      const std::vector<Poly>& polys = cellPolys[c][cell];
      polyTris[c][cell].resize(polys.size());
      polyOk[c][cell].resize(polys.size());
      for (size_t q = 0; q < polys.size(); q++) {
        std::vector<I3>& tris = polyTris[c][cell][q];
        polyOk[c][cell][q] = triangulate_polygon(polys[q].v, tris) && tris.size() + 2 == polys[q].v.size();
      }
    }
  }
  // mid-edge node of edge (a, b), a < b: chained per a, numbered in first-seen order
  std::vector<int> midHead(size_t(firstMid), -1), midNext, midTo;
  int nextMid = 0;
  for (int c = 0; c < nCharts; c++) {
    const GridChart& g = L.charts[c];
    ChartBoundary& cb = be.charts[c];
    cb.cellTriangles.assign(g.numBoundaryCells, {});
    for (int cell = 0; cell < g.numBoundaryCells; cell++)
      for (size_t q = 0; q < cellPolys[c][cell].size(); q++) {
        const Poly& P = cellPolys[c][cell][q];
        const std::vector<I3>& tris = polyTris[c][cell][q];
        const int n = (int)P.v.size();
        if (!polyOk[c][cell][q]) {
          be.degenerateTriangulations++;
          if (getenv("GDTP_DEBUG_POLY")) {
            fprintf(stderr, "degenerate polygon chart %d cell %d n=%d tris=%d\n", c, cell, n, (int)tris.size());
            for (int q = 0; q < n; q++) fprintf(stderr, "  %.17g %.17g idx %d\n", P.v[q].x / g.cellSizeW, P.v[q].y / g.cellSizeH, P.idx[q]);
          }
        }
        for (const I3& t : tris) {
          BoundaryTriangle bt;
          for (int v = 0; v < 3; v++) {
            int pv = t[v];
            bt.v[v] = P.v[pv];
            bt.idx[v] = P.idx[pv];
            bt.atlasVertex[v] = P.atlasVertex[pv];
            bt.parentEdge[v] = P.parentEdge[pv];
            bt.atlasEdge[v] = -1;
            if (t[(v + 1) % 3] == (pv + 1) % n) bt.atlasEdge[v] = P.atlasEdge[pv];
            int prevv = (pv + n - 1) % n;
            if (t[(v + 1) % 3] == prevv) bt.atlasEdge[v] = P.atlasEdge[prevv];
          }
          for (int v = 0; v < 3; v++) {
            int a = bt.idx[(v + 1) % 3], b = bt.idx[(v + 2) % 3];
            if (a > b) std::swap(a, b);
            if (a < 0 || a >= firstMid) { err = "boundary triangle vertex out of range"; return false; }
            int mid = midHead[a];
            while (mid != -1 && midTo[mid] != b) mid = midNext[mid];
            if (mid == -1) {
              mid = nextMid++;
              midTo.push_back(b);
              midNext.push_back(midHead[a]);
              midHead[a] = mid;
            }
            bt.idx[3 + v] = mid + firstMid;
            cb.aux.push_back({(bt.v[(v + 1) % 3] + bt.v[(v + 2) % 3]) / 2.0, mid + firstMid});
          }
          cb.cellTriangles[cell].push_back(bt);
        }
      }
  }
  be.numMidPoints = nextMid;
  be.numFineNodes = numInterior + be.numBoundaryNodes + be.numMidPoints;

  // (4) fine boundary numbering and the texel -> fine boundary prolongation
  be.fineBoundaryIndex.assign(be.numFineNodes, -1);
  std::vector<Triplet> trip;
  int nextFine = 0;
  for (const GridChart& g : L.charts)
    for (int n = 0; n < g.width * g.height; n++)
      if (g.interiorTexel[n] != -1 && g.deepTexel[n] == -1) {
        int bidx = L.boundaryAndDeep[g.texel[n]] - 1;
        if (bidx < 0) { err = "interior non-deep texel is not a boundary texel"; return false; }
        trip.push_back({nextFine, bidx, 1.0});
        be.fineBoundaryIndex[g.interiorTexel[n]] = nextFine++;
      }
  for (int i = numInterior; i < be.numFineNodes; i++) be.fineBoundaryIndex[i] = nextFine++;
  be.numFineBoundary = nextFine;
  const int numAux = be.numFineNodes - numInterior;
  std::vector<int> degree(numAux, 0);
  for (const ChartBoundary& cb : be.charts)
    for (const AuxNode& a : cb.aux) degree[a.index - numInterior]++;
  // auxiliary-node rows, charts in parallel, concatenated in chart order
  std::vector<std::vector<Triplet>> auxTrip(nCharts);
  std::vector<std::string> auxErr(nCharts);
#pragma omp parallel for schedule(dynamic, 1)
  for (int c = 0; c < nCharts; c++) {
    const GridChart& g = L.charts[c];
    auto aux_rows = [&](std::vector<Triplet>& trip, std::string& err) -> bool {
    for (const AuxNode& a : be.charts[c].aux) {
      int fid = be.fineBoundaryIndex[a.index];
      int deg = degree[a.index - numInterior];
      int ci = int(std::floor(a.pos.x / g.cellSizeW)), cj = int(std::floor(a.pos.y / g.cellSizeH));
      if (ci < 0 || cj < 0 || ci >= g.width - 1 || cj >= g.height - 1 || g.localCell[g.cat(ci, cj)] == -1) {
        err = "auxiliary node outside the active cells";
        return false;
      }
      int cellId = g.localCell[g.cat(ci, cj)];
      double x = a.pos.x / g.cellSizeW - double(ci), y = a.pos.y / g.cellSizeH - double(cj);
      const double tol = 1e-10;
      if (x < -tol || x > 1 + tol || y < -tol || y > 1 + tol) { err = "auxiliary node out of its cell"; return false; }
      double w[4] = {(1.0 - x) * (1.0 - y), x * (1.0 - y), x * y, (1.0 - x) * y};
      for (int k = 0; k < 4; k++) {
        double tw = w[k] / double(deg);
        if (std::fabs(tw) <= 1e-11) continue;
        int texel = g.cellCorners[4 * cellId + k];
        if (L.nodes[texel].type == 2) { err = "deep texel in the support of an auxiliary node"; return false; }
        int bidx = L.boundaryAndDeep[texel] - 1;
        if (bidx < 0) { err = "auxiliary node supported by a non-boundary texel"; return false; }
        trip.push_back({fid, bidx, tw});
      }
    }
      return true;
    };
    aux_rows(auxTrip[c], auxErr[c]);
  }
  for (int c = 0; c < nCharts; c++) {
    if (!auxErr[c].empty()) { err = auxErr[c]; return false; }
    trip.insert(trip.end(), auxTrip[c].begin(), auxTrip[c].end());
  }
  be.prolongation = csr_from_triplets(be.numFineBoundary, L.numBoundary, trip);
  return true;
}

}  // namespace gdtp
