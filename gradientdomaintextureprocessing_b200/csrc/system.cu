// Device-resident texel-FEM system (see system.h).
//
// Solve path (mixed precision, every RHS at once):
//   r = b - A x            FP64 operator, FP64 vectors, per-RHS norms
//   e = V(r)               one FP32 V-cycle from e = 0
//   x += e                 FP64
// repeated until max_k ||r_k|| / ||b_k|| <= tol.  The V-cycle follows the
// reference's schedule (IterativeSolvers.inl:1211-1333): on the way down each
// level relaxes (boundary block solved exactly, then deep texels by colour-run
// Gauss-Seidel), forms the residual and restricts it; the coarsest level is
// solved directly; on the way up the correction is prolongated and relaxed
// again.  The sequence of launches of one refinement step is captured once into
// a CUDA graph and replayed.
#include <algorithm>
#include <climits>
#include <chrono>
#include <cmath>
#include <cstring>

#include <map>
#include <stdexcept>
#include <thread>
#include <tuple>

#include "system.h"

namespace gdtp {

// coarsest levels up to this size are solved inside the coarse-level cluster

static inline int kp_for(int k) {
  if (k <= 1) return 1;
  int kp = 4;
  while (kp < k) kp *= 2;
  return kp;
}

// Line runs for the FP64 operator (no colouring needed): up to 32 consecutive
// deep texels of a raster line, so a warp's loads of a neighbour row are
// contiguous.  texel[i] = deep index of plane position i.
DeepRuns build_line_runs(const GridLevel& L) {
  DeepRuns R;
  R.texel.reserve(L.numDeep);
  for (const Line& l : L.rasterLines) {
    const int len = l.end - l.start + 1;
    for (int p = 0; p < len; p += 32) {
      dev::ColourRun r;
      r.pos0 = l.start + p;
      r.prev0 = l.prev + p;
      r.next0 = l.next + p;
      r.coef0 = R.count;
      r.len = std::min(32, len - p);
      for (int m = 0; m < r.len; m++) R.texel.push_back(l.coeff + p + m);
      R.count += r.len;
      R.runs.push_back(r);
    }
  }
  R.runStart[4] = (int)R.runs.size();
  return R;
}

DeepRuns build_deep_runs(const GridLevel& L) {
  DeepRuns R;
  R.texel.reserve(L.numDeep);
  R.lineCoef.assign(L.rasterLines.size() * 2, -1);
  for (int c = 0; c < 4; c++) {
    R.runStart[c] = (int)R.runs.size();
    const int ci = c & 1, cj = c >> 1;
    for (size_t li = 0; li < L.rasterLines.size(); li++) {
      const Line& l = L.rasterLines[li];
      const NodeInfo& n = L.nodes[l.start];
      if ((n.cj & 1) != cj) continue;
      const int len = l.end - l.start + 1;
      const int o = (ci - (n.ci & 1)) & 1;
      if (o < len) R.lineCoef[2 * li + ci] = R.count;
      for (int p = o; p < len; p += 64) {
        dev::ColourRun r;
        r.pos0 = l.start + p;
        r.prev0 = l.prev + p;
        r.next0 = l.next + p;
        r.coef0 = R.count;
        r.len = std::min(32, (len - p + 1) / 2);
        for (int m = 0; m < r.len; m++) R.texel.push_back(l.coeff + p + 2 * m);
        R.count += r.len;
        R.runs.push_back(r);
      }
    }
  }
  R.runStart[4] = (int)R.runs.size();
  return R;
}

// Raster lines of each row parity packed, in raster order, into blocks of
// `block` threads (a line of len texels takes (len + 1) / 2 threads and len + 2
// shared-memory slots).  The block size is the smallest of 256, 512 and 1024
// threads that holds the longest line; false (row smoother unused) when a line
// is longer than 2 kRowBlockMax texels.
bool build_row_bins(const GridLevel& L, const DeepRuns& R, RowBins& out) {
  out = RowBins();
  int maxThr = 0;
  for (const Line& l : L.rasterLines) maxThr = std::max(maxThr, (l.end - l.start + 2) / 2);
  int bs = 256;
  while (bs < maxThr && bs < dev::kRowBlockMax) bs *= 2;
  if (maxThr > bs || L.rasterLines.empty()) return false;
  out.block = bs;
  out.slots = dev::row_slot_cap(bs);
  for (int rows = 0; rows < 2; rows++) {
    std::vector<dev::RowLine>& lines = out.lines[rows];
    std::vector<int>& lineOf = out.lineOf[rows];
    int thr = bs, slot = out.slots;  // the current block is full: open one on the first line
    for (size_t li = 0; li < L.rasterLines.size(); li++) {
      const Line& l = L.rasterLines[li];
      const NodeInfo& n = L.nodes[l.start];
      if ((n.cj & 1) != rows) continue;
      const int len = l.end - l.start + 1, nt = (len + 1) / 2;
      if (thr + nt > bs || slot + len + 2 > out.slots) {
        lineOf.resize(lineOf.size() + bs, -1);
        out.bins[rows]++;
        thr = slot = 0;
      }
      const int oddStart = n.ci & 1;
      dev::RowLine r;
      r.pos = l.start;
      r.prev = l.prev;
      r.next = l.next;
      r.len = len;
      // the line's first texel of even / odd column (colour-run coefficient index)
      r.cEven = R.lineCoef[2 * li + 0];
      r.cOdd = R.lineCoef[2 * li + 1];
      r.meta = thr | (slot << 11) | (oddStart << 24);
      r.pad = 0;
      if ((r.cEven < 0 && len > oddStart) || (r.cOdd < 0 && len > 1 - oddStart)) return false;
      const int idx = (int)lines.size();
      lines.push_back(r);
      const size_t base = lineOf.size() - bs;
      for (int t = 0; t < nt; t++) lineOf[base + thr + t] = idx;
      thr += nt;
      slot += len + 2;
    }
  }
  return true;
}

// Per chart and colour, the range of that colour's runs that lie in the chart:
// grp[10 g + c] = first run, grp[10 g + 4 + c] = run count, then the chart's
// texel span (first texel, count) that its updates touch.  Runs of a colour
// follow the raster lines, chart by chart; false if a chart's runs of some
// colour are not contiguous (the grouped smoother is then not used).
static bool chart_groups(const GridLevel& L, const DeepRuns& R, std::vector<int>& grp, int& maxDeep, int& maxSpan) {
  grp.clear();
  maxDeep = 0;
  maxSpan = 0;
  const int nc = (int)L.charts.size();
  if (nc == 0 || R.runs.empty()) return false;
  std::vector<int> first(size_t(nc) * 4, -1), count(size_t(nc) * 4, 0), deep(nc, 0);
  for (int c = 0; c < 4; c++) {
    int last = -1;
    for (int r = R.runStart[c]; r < R.runStart[c + 1]; r++) {
      const int ch = L.nodes[R.runs[r].pos0].chart;
      if (ch < 0 || ch >= nc) return false;
      int& f = first[size_t(ch) * 4 + c];
      if (f < 0) f = r;
      else if (ch != last) return false;  // the chart's runs of this colour are split
      count[size_t(ch) * 4 + c]++;
      deep[ch] += R.runs[r].len;
      last = ch;
    }
  }
  // texel span [lo, hi] every update of the chart reads or writes; the span
  // must hold texels of that chart only (charts are contiguous in texel order)
  for (int ch = 0; ch < nc; ch++) {
    if (deep[ch] == 0) continue;
    int lo = INT_MAX, hi = INT_MIN;
    for (int c = 0; c < 4; c++)
      for (int r = first[size_t(ch) * 4 + c], e = r + count[size_t(ch) * 4 + c]; r >= 0 && r < e; r++) {
        const dev::ColourRun& u = R.runs[r];
        const int last = 2 * (u.len - 1);
        lo = std::min({lo, u.pos0 - 1, u.prev0 - 1, u.next0 - 1});
        hi = std::max({hi, u.pos0 + last + 1, u.prev0 + last + 1, u.next0 + last + 1});
      }
    if (lo < 0 || hi >= L.numTexels) return false;
    for (int i = lo; i <= hi; i++)
      if (L.nodes[i].chart != ch) return false;
    for (int c = 0; c < 4; c++) grp.push_back(std::max(0, first[size_t(ch) * 4 + c]));
    for (int c = 0; c < 4; c++) grp.push_back(count[size_t(ch) * 4 + c]);
    grp.push_back(lo);
    grp.push_back(hi - lo + 1);
    maxDeep = std::max(maxDeep, deep[ch]);
    maxSpan = std::max(maxSpan, hi - lo + 1);
  }
  return !grp.empty();
}

// Levels with at least this many deep texels get tiles for the fused smoother
// (the tile_texels knob then chooses where they are used).
static constexpr int kTileBuildMin = 4096;

// Tiles of the fused smoother over one level: kTileW x kTileH texels of a
// chart's grid with origins at multiples of the tile size, every tile holding
// at least one active texel.  Per tile the reciprocal-form coefficients of its
// deep texels (the colour-run planes' arithmetic: c_k / c_4, 1 / c_4, c_4; zeros
// elsewhere) and the runs of consecutive global texels on each row of the tile
// with its one-texel ring (the layout launch_tile_smooth documents).
struct TileLayout {
  std::vector<int4> tiles;              // ordered by tile colour
  int tileStart[5] = {0, 0, 0, 0, 0};
  std::vector<int4> segs;
  std::vector<int> nbrs;                // 8 per tile: the tiles around it (-1: none)
  std::vector<float> coef;
};
static void build_tiles(const GridLevel& G, const LevelCoefficients& C, TileLayout& T) {
  using dev::kTileH;
  using dev::kTileSlots;
  using dev::kTileW;
  constexpr int perColour = kTileSlots / 4, halfW = kTileW / 2;
  std::vector<int4> byColour[4];
  std::vector<int3> where[4];           // chart, tile column, tile row of each tile
  for (int ch = 0; ch < (int)G.charts.size(); ch++) {
    const GridChart& gc = G.charts[ch];
    const int w = gc.width, h = gc.height;
    auto texel = [&](int i, int j) { return (i < 0 || j < 0 || i >= w || j >= h) ? -1 : gc.texel[gc.at(i, j)]; };
    for (int j0 = 0; j0 < h; j0 += kTileH)
      for (int i0 = 0; i0 < w; i0 += kTileW) {
        bool any = false;
        for (int j = j0; j < std::min(h, j0 + kTileH) && !any; j++)
          for (int i = i0; i < std::min(w, i0 + kTileW) && !any; i++) any = texel(i, j) >= 0;
        if (!any) continue;
        int4 tile;
        tile.x = (int)T.coef.size();
        tile.y = (int)T.segs.size();
        T.coef.resize(T.coef.size() + size_t(10) * kTileSlots, 0.f);
        float* block = T.coef.data() + tile.x;
        for (int cc = 0; cc < 4; cc++)
          for (int q = 0; q < kTileH / 2; q++)
            for (int p = 0; p < halfW; p++) {
              const int i = i0 + 2 * p + (cc & 1), j = j0 + 2 * q + (cc >> 1);
              if (i >= w || j >= h) continue;
              const int d = gc.deepTexel[gc.at(i, j)];
              if (d < 0) continue;
              const double* c = &C.deep[10 * size_t(d)];
              const double c4 = c[4], inv = 1.0 / c4;
              const int slot = cc * perColour + q * halfW + p;
              for (int k = 0; k < 9; k++) block[size_t(k) * kTileSlots + slot] = float(k == 4 ? inv : c[k] * inv);
              block[size_t(9) * kTileSlots + slot] = float(c4);
            }
        int elems = 0;
        for (int r = 0; r <= kTileH + 1; r++) {
          const int j = j0 - 1 + r;
          for (int u = 0; u <= kTileW + 1;) {
            const int g0 = texel(i0 - 1 + u, j);
            if (g0 < 0) { u++; continue; }
            int len = 1;
            while (u + len <= kTileW + 1 && texel(i0 - 1 + u + len, j) == g0 + len) len++;
            T.segs.push_back(make_int4(g0, r | (u << 6) | (len << 12), elems, 0));
            elems += len;
            u += len;
          }
        }
        tile.z = (int)T.segs.size() - tile.y;
        tile.w = elems;
        // a ring row holds at most every other texel as its own segment
        if (tile.z > dev::kTileMaxSegs) throw std::logic_error("tile segment bound exceeded");
        const int colour = ((i0 / kTileW) & 1) | (((j0 / kTileH) & 1) << 1);
        byColour[colour].push_back(tile);
        where[colour].push_back(make_int3(ch, i0 / kTileW, j0 / kTileH));
      }
  }
  std::map<std::tuple<int, int, int>, int> index;
  std::vector<int3> at;
  for (int c = 0; c < 4; c++) {
    T.tileStart[c] = (int)T.tiles.size();
    for (size_t k = 0; k < byColour[c].size(); k++) {
      index[std::make_tuple(where[c][k].x, where[c][k].y, where[c][k].z)] = (int)T.tiles.size();
      T.tiles.push_back(byColour[c][k]);
      at.push_back(where[c][k]);
    }
  }
  T.tileStart[4] = (int)T.tiles.size();
  T.nbrs.assign(size_t(8) * T.tiles.size(), -1);
  for (size_t t = 0; t < T.tiles.size(); t++) {
    int k = 0;
    for (int dj = -1; dj <= 1; dj++)
      for (int di = -1; di <= 1; di++) {
        if (!di && !dj) continue;
        auto it = index.find(std::make_tuple(at[t].x, at[t].y + di, at[t].z + dj));
        T.nbrs[8 * t + k++] = it == index.end() ? -1 : it->second;
      }
  }
}

DeviceSystem::DeviceSystem(const Hierarchy& h, const BoundaryElements& be, int device) : h_(h), be_(be), device_(device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) { err_ = "no CUDA device"; return; }
  if (device < 0 || device >= n) { err_ = "invalid CUDA device"; return; }
  if (!check(cudaSetDevice(device), "cudaSetDevice")) return;
  if (!check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate")) return;
}

DeviceSystem::~DeviceSystem() {
  cudaSetDevice(device_);
  for (StepGraph& g : stepGraphs_) cudaGraphExecDestroy(g.exec);
  for (cudaEvent_t e : profEv_)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : traceEv_) cudaEventDestroy(e);
  if (sumsHost_) cudaFreeHost(sumsHost_);
  if (barrierErrHost_) cudaFreeHost(barrierErrHost_);
  for (int j = 0; j < 2; j++)
    for (cudaEvent_t e : {slotIn_[j], slotSolved_[j], slotOut_[j]})
      if (e) cudaEventDestroy(e);
  if (copyIn_) cudaStreamDestroy(copyIn_);
  if (copyOut_) cudaStreamDestroy(copyOut_);
  mg32_.clear();
  mg64_.reset();
  if (stream_) cudaStreamDestroy(stream_);
}

void DeviceSystem::invalidate_multigrids() {
  invalidate_graph();
  mg32_.clear();
  mg64_.reset();
}

void DeviceSystem::invalidate_graph() {
  cudaSetDevice(device_);
  for (StepGraph& g : stepGraphs_) cudaGraphExecDestroy(g.exec);
  stepGraphs_.clear();
}

cudaGraphExec_t DeviceSystem::find_graph(int kind, int k, const double* b, const double* x) {
  for (size_t i = 0; i < stepGraphs_.size(); i++) {
    const StepGraph g = stepGraphs_[i];
    if (g.kind == kind && g.k == k && g.b == b && g.x == x) {
      stepGraphs_.erase(stepGraphs_.begin() + i);
      stepGraphs_.push_back(g);
      graphKernels = g.kernels;
      return g.exec;
    }
  }
  return nullptr;
}

void DeviceSystem::add_graph(const StepGraph& g) {
  if (stepGraphs_.size() >= kMaxStepGraphs) {
    cudaGraphExecDestroy(stepGraphs_.front().exec);
    stepGraphs_.erase(stepGraphs_.begin());
  }
  stepGraphs_.push_back(g);
  graphKernels = g.kernels;
}

// capacity for k right-hand sides: the next power of two (at most 64), so a
// stream of varying batch sizes reallocates (and re-captures) rarely
static int k_capacity(int k) {
  int c = 1;
  while (c < k) c *= 2;
  return std::min(c, 64);
}

bool DeviceSystem::check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  err_ = std::string(what) + ": " + cudaGetErrorString(e);
  return false;
}

size_t DeviceSystem::deviceBytes() const {
  size_t b = rawArena_.total + rawAArena_.total + workArena_.total + slotArena_.total + deepArena_.total;
  for (const auto& m : mg32_) b += m->arena.total;
  if (mg64_) b += mg64_->arena.total;
  if (plan_) b += plan_->deviceBytes();
  return b;
}

// ----------------------------------------------------------------------------
// assembly
// ----------------------------------------------------------------------------
static double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

bool DeviceSystem::assemble(const Mesh& mesh, const double* parameterMetric) {
  if (!err_.empty()) return false;
  const double tAssembly = now_ms();
  // a new assembly replaces everything built from the previous one
  mg32_.clear();
  mg64_.reset();
  invalidate_graph();
  plan_.reset();
  bsCache_.clear();
  coLevels_ = 0;
  hostCoeffs_ = false;
  rawFromPlan_ = false;
  cudaSetDevice(device_);
  ChartMetrics g;
  if (parameterMetric) {
    g.assign(h_.atlas.charts.size(), {});
    for (size_t c = 0; c < h_.atlas.charts.size(); c++)
      for (int t : h_.atlas.charts[c].meshTriangleIndices) {
        M2 m;
        m.c[0][0] = parameterMetric[4 * t]; m.c[0][1] = parameterMetric[4 * t + 1];
        m.c[1][0] = parameterMetric[4 * t + 2]; m.c[1][1] = parameterMetric[4 * t + 3];
        g[c].push_back(m);
      }
  } else if (!embedding_metric(mesh, h_.atlas, g)) {
    err_ = "degenerate mesh (zero area)";
    return false;
  }
  metric_ = g;
  AssemblyWork w;
  build_assembly_work(h_, be_, g, w);
  setupMs[8] = now_ms() - tAssembly;
  // temporaries from the stream-ordered pool (every output below is written in
  // full by its kernel, so nothing is zeroed)
  StreamScratch A(stream_);
  int* cellPtr = A.upload(w.cellPtr);
  int* cellTri = A.upload(w.cellTri);
  int* cellIJ = A.upload(w.cellIJ);
  int* cellChart = A.upload(w.cellChart);
  double* cellSize = A.upload(w.chartCellSize);
  double* triPos = A.upload(w.triPos);
  double* triMetric = A.upload(w.triMetric);
  double* triInv = A.upload(w.triMetricInv);
  double* triScale = A.upload(w.triScale);
  int* deepCells = A.upload(w.deepCells);
  int* adj = A.upload(w.boundaryAdjacentCells);
  int* btPtr = A.upload(w.btPtr);
  int* btTri = A.upload(w.btTri);
  double* btPos = A.upload(w.btPos);
  double* cm = A.get<double>(16 * size_t(w.numInteriorCells));
  double* cs = A.get<double>(16 * size_t(w.numInteriorCells));
  const int nd = h_.levels[0].numDeep;
  // the level-0 deep coefficients stay resident: the operators' planes and the
  // numeric set-up read them on the device
  deepArena_ = DeviceArena();
  double* dm = static_cast<double*>(deepArena_.alloc(10 * std::max<size_t>(1, size_t(nd)) * sizeof(double)));
  double* ds = static_cast<double*>(deepArena_.alloc(10 * std::max<size_t>(1, size_t(nd)) * sizeof(double)));
  deepMassDev_ = dm;
  deepStiffDev_ = ds;
  if (!check(deepArena_.last, "deep coefficients")) return false;
  const size_t na = w.boundaryAdjacentCells.size();
  double* am = A.get<double>(16 * na);
  double* as = A.get<double>(16 * na);
  double* bm = A.get<double>(36 * size_t(w.numBoundaryTriangles));
  double* bs = A.get<double>(36 * size_t(w.numBoundaryTriangles));
  if (!check(A.last, "assembly buffers")) return false;
  dev::launch_interior_cells(w.numInteriorCells, cellPtr, cellTri, cellIJ, cellChart, cellSize, triPos, triInv, triScale, cm, cs,
                             stream_);
  dev::launch_deep_gather(nd, deepCells, cm, cs, dm, ds, stream_);
  dev::launch_gather_cells((int)na, adj, cm, am, stream_);
  dev::launch_gather_cells((int)na, adj, cs, as, stream_);
  dev::launch_boundary_triangles(w.numBoundaryTriangles, btPtr, btTri, btPos, triPos, triMetric, triInv, bm, bs, stream_);
  if (!check(cudaGetLastError(), "assembly launch")) return false;
  fine_ = FineSystem();
  fine_.deepMass.resize(10 * size_t(nd));
  fine_.deepStiffness.resize(10 * size_t(nd));
  std::vector<double> ham(16 * na), has(16 * na), hbm(36 * size_t(w.numBoundaryTriangles)), hbs(hbm.size());
  bool ok = check(cudaMemcpyAsync(ham.data(), am, ham.size() * 8, cudaMemcpyDeviceToHost, stream_), "d2h") &&
            check(cudaMemcpyAsync(has.data(), as, has.size() * 8, cudaMemcpyDeviceToHost, stream_), "d2h") &&
            check(cudaMemcpyAsync(hbm.data(), bm, hbm.size() * 8, cudaMemcpyDeviceToHost, stream_), "d2h") &&
            check(cudaMemcpyAsync(hbs.data(), bs, hbs.size() * 8, cudaMemcpyDeviceToHost, stream_), "d2h") &&
            check(cudaStreamSynchronize(stream_), "assembly");
  if (!ok) return false;
  setupMs[9] = now_ms() - tAssembly - setupMs[8];
  // the host copies of the deep coefficients (read by the Galerkin coarsening)
  // come down on a helper thread while this one builds the boundary blocks
  cudaError_t deepCopy = cudaSuccess;
  std::thread deepDown([&] {
    deepCopy = cudaSetDevice(device_);
    if (deepCopy == cudaSuccess)
      deepCopy = cudaMemcpyAsync(fine_.deepMass.data(), dm, fine_.deepMass.size() * 8, cudaMemcpyDeviceToHost, stream_);
    if (deepCopy == cudaSuccess)
      deepCopy = cudaMemcpyAsync(fine_.deepStiffness.data(), ds, fine_.deepStiffness.size() * 8, cudaMemcpyDeviceToHost, stream_);
    if (deepCopy == cudaSuccess) deepCopy = cudaStreamSynchronize(stream_);
  });
  const bool blocks = assemble_boundary_blocks(h_, be_, w, ham, has, hbm, hbs, fine_, err_);
  deepDown.join();
  if (!blocks || !check(deepCopy, "deep coefficients d2h")) return false;
  setupMs[10] = now_ms() - tAssembly - setupMs[8] - setupMs[9];

  // raw FP64 operators of M and S on level 0 (deep planes in line-run order)
  runs0_ = build_line_runs(h_.levels[0]);
  const GridLevel& L0 = h_.levels[0];
  rawArena_ = DeviceArena();
  const int* runTexel = rawArena_.upload(runs0_.texel);
  auto make_raw = [&](const double* deepDev, const Csr& bb, const Csr& bd, RawOperator& op) {
    const int cnt = runs0_.count;
    double* planes = static_cast<double*>(rawArena_.alloc(size_t(9) * std::max(1, cnt) * sizeof(double)));
    if (planes && cnt > 0) launch_gather_planes(cnt, runTexel, deepDev, planes, stream_);
    std::vector<int> ptr(1, 0), col;
    std::vector<double> val;
    for (int b = 0; b < L0.numBoundary; b++) {
      for (int k = bd.ptr[b]; k < bd.ptr[b + 1]; k++) { col.push_back(bd.col[k]); val.push_back(bd.val[k]); }
      for (int k = bb.ptr[b]; k < bb.ptr[b + 1]; k++) { col.push_back(L0.boundaryGlobal[bb.col[k]]); val.push_back(bb.val[k]); }
      ptr.push_back((int)col.size());
    }
    op.runs = rawArena_.upload(runs0_.runs);
    op.nRuns = (int)runs0_.runs.size();
    op.coef = planes;
    op.planeStride = cnt;
    op.bPtr = rawArena_.upload(ptr);
    op.bCol = rawArena_.upload(col);
    op.bVal = rawArena_.upload(val);
    op.bGlobal = rawArena_.upload(L0.boundaryGlobal);
    op.nB = L0.numBoundary;
  };
  make_raw(dm, fine_.bbMass, fine_.bdMass, rawM_);
  make_raw(ds, fine_.bbStiffness, fine_.bdStiffness, rawS_);
  if (!check(cudaStreamSynchronize(stream_), "operator planes")) return false;
  setupMs[11] = now_ms() - tAssembly - setupMs[8] - setupMs[9] - setupMs[10];
  return check(rawArena_.last, "operator upload");
}

// ----------------------------------------------------------------------------
// coefficient hierarchy + device multigrid
// ----------------------------------------------------------------------------
namespace {
bool fill_one(NumericPlan& p, int l, LevelValues<float>& v, cudaStream_t s, std::string& e) { return p.fill_level(l, &v, nullptr, s, e); }
bool fill_one(NumericPlan& p, int l, LevelValues<double>& v, cudaStream_t s, std::string& e) { return p.fill_level(l, nullptr, &v, s, e); }

// the dense inverses and products of the set-up on the device (kernels/dense_kernels.cu)
struct DeviceDense final : DenseBackend {
  cudaStream_t s;
  explicit DeviceDense(cudaStream_t stream) : s(stream) {}
  bool spd_inverse_batched(double* data, const std::vector<int64_t>& off, const std::vector<int>& size, std::string& err) override {
    return dev::gpu_spd_inverse_batched(data, off, size, s, err);
  }
  bool schur_products(const std::vector<double>& inv, const std::vector<int64_t>& invOff, const std::vector<int>& m,
                      const std::vector<double>& C, const std::vector<int64_t>& cOff, const std::vector<int>& t, std::vector<double>& G,
                      std::vector<double>& local, const std::vector<int64_t>& localOff, std::string& err) override {
    return dev::gpu_schur_products(inv, invOff, m, C, cOff, t, G, local, localOff, s, err);
  }
};
}  // namespace


bool DeviceSystem::update(double stiffness, double screen) {
  if (!err_.empty()) return false;
  const double tUpdate = now_ms();
  if (fine_.deepMass.empty() && h_.levels[0].numDeep > 0) { err_ = "update before assembly"; return false; }
  cudaSetDevice(device_);
  const GridLevel& L0 = h_.levels[0];
  // levels used: stop once the coarsest fits the dense direct solve
  int L = (int)h_.levels.size();
  for (int l = 0; l < (int)h_.levels.size(); l++)
    if (h_.levels[l].numTexels <= knobs.maxCoarse) { L = l + 1; break; }
  if (h_.levels[L - 1].numTexels > 12000) { err_ = "coarsest level too large for the dense direct solve; build more levels"; return false; }
  // Galerkin coarsening is linear in the weights: the mass and stiffness
  // hierarchies are coarsened once (per level count) and every update
  // combines them, so a re-weighting costs one pass over the coefficients
  if (coLevels_ != L) {
    const double t0 = now_ms();
    Csr bdM = fine_.bdMass, bdS = fine_.bdStiffness;
    bdM.cols = bdS.cols = L0.numTexels;
    // M and S coarsen side by side (each with its own parallel loops)
    std::string errS;
    bool okS = false;
    std::thread stiff([&] { okS = galerkin_hierarchy(h_, L, fine_.deepStiffness, fine_.bbStiffness, bdS, coStiff_, errS); });
    const bool okM = galerkin_hierarchy(h_, L, fine_.deepMass, fine_.bbMass, bdM, coMass_, err_);
    stiff.join();
    if (!okM) return false;
    if (!okS) {
      err_ = errS;
      return false;
    }
    coLevels_ = L;
    setupMs[12] = now_ms() - t0;
  }
  const bool sameLevels = (levelsUsed_ == L);
  levelsUsed_ = L;
  stiffness_ = stiffness;
  screen_ = screen;
  hostCoeffs_ = false;
  bsCache_.clear();
  if (use_numeric()) {
    // values on the device from the resident M and S: the multigrids built by
    // this path keep their layout and are refilled in place
    bool built = false;
    if (!ensure_plan(&built) || (!built && !plan_->combine(screen, stiffness, stream_, err_))) return false;
    if (!refresh_raw_operator()) return false;
    bool keep = sameLevels && (!mg32_.empty() || mg64_);
    if (!mg32_.empty()) keep = keep && mg32_.front()->planGen == plan_->gen;
    if (mg64_) keep = keep && mg64_->planGen == plan_->gen;
    if (keep) {
      if (!refresh_multigrids()) return false;
      invalidate_graph();
    } else {
      mg32_.clear();
      mg64_.reset();
      invalidate_graph();
    }
  } else {
    if (!ensure_host_coefficients()) return false;
    // raw FP64 A on level 0: its own arena, released on every update (the
    // deep planes are screen M + stiffness S of the resident M and S planes)
    const LevelCoefficients& c0 = coeffs_[0];
    const int cnt = runs0_.count;
    rawAArena_ = DeviceArena();
    rawFromPlan_ = false;
    double* planes = static_cast<double*>(rawAArena_.alloc(size_t(9) * std::max(1, cnt) * sizeof(double)));
    if (!check(rawAArena_.last, "operator planes")) return false;
    dev::launch_axpby(planes, screen, rawM_.coef, stiffness, rawS_.coef, (long long)9 * cnt, stream_);
    std::vector<int> ptr(1, 0), col;
    std::vector<double> val;
    for (int b = 0; b < L0.numBoundary; b++) {
      for (int k = c0.bd.ptr[b]; k < c0.bd.ptr[b + 1]; k++) { col.push_back(c0.bd.col[k]); val.push_back(c0.bd.val[k]); }
      for (int k = c0.bb.ptr[b]; k < c0.bb.ptr[b + 1]; k++) { col.push_back(L0.boundaryGlobal[c0.bb.col[k]]); val.push_back(c0.bb.val[k]); }
      ptr.push_back((int)col.size());
    }
    rawA_ = RawOperator();
    rawA_.runs = rawM_.runs;
    rawA_.nRuns = rawM_.nRuns;
    rawA_.coef = planes;
    rawA_.planeStride = cnt;
    rawA_.bPtr = rawAArena_.upload(ptr);
    rawA_.bCol = rawAArena_.upload(col);
    rawA_.bVal = rawAArena_.upload(val);
    rawA_.bGlobal = rawM_.bGlobal;
    rawA_.nB = L0.numBoundary;
    if (!check(rawAArena_.last, "operator upload") || !check(cudaStreamSynchronize(stream_), "operator planes")) return false;
    mg32_.clear();
    mg64_.reset();
    invalidate_graph();
  }
  updated_ = true;
  setupMs[0] = now_ms() - tUpdate;
  return true;
}

bool DeviceSystem::use_numeric() const { return knobs.deviceFactor != 0 && knobs.tileTexels == 0; }

// host combination of the coefficient hierarchy for the current weights (the
// host-built multigrid, the tile layout and the coefficient export read it)
bool DeviceSystem::ensure_host_coefficients() {
  if (hostCoeffs_) return true;
  const int L = levelsUsed_;
  const GridLevel& L0 = h_.levels[0];
  std::vector<LevelCoefficients> co(L);
  co[0].deep.resize(fine_.deepMass.size());
  for (size_t i = 0; i < co[0].deep.size(); i++) co[0].deep[i] = screen_ * fine_.deepMass[i] + stiffness_ * fine_.deepStiffness[i];
  co[0].bb = csr_axpby(screen_, fine_.bbMass, stiffness_, fine_.bbStiffness);
  co[0].bd = csr_axpby(screen_, fine_.bdMass, stiffness_, fine_.bdStiffness);
  co[0].bd.cols = L0.numTexels;
  for (int l = 1; l < L; l++) {
    const LevelCoefficients &m = coMass_[l], &k = coStiff_[l];
    co[l].deep.resize(m.deep.size());
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)m.deep.size(); i++) co[l].deep[i] = screen_ * m.deep[i] + stiffness_ * k.deep[i];
    co[l].bb = csr_axpby(screen_, m.bb, stiffness_, k.bb);
    co[l].bd = csr_axpby(screen_, m.bd, stiffness_, k.bd);
  }
  coeffs_ = std::move(co);
  hostCoeffs_ = true;
  return true;
}

const std::vector<LevelCoefficients>& DeviceSystem::coefficients() {
  if (updated_ && !ensure_host_coefficients()) coeffs_.clear();
  return coeffs_;
}

bool DeviceSystem::ensure_plan(bool* built) {
  const int L = levelsUsed_;
  if (built) *built = false;
  if (plan_ && plan_->L == L && plan_->maxBlock == knobs.maxBlock && plan_->denseMax == knobs.denseBoundaryMax) return true;
  // multigrids laid out for an earlier plan keep their own buffers; an update
  // rebuilds them (their generation differs)
  plan_.reset(new NumericPlan());
  plan_->gen = ++planCount_;
  const double t0 = now_ms();
  if (!plan_->build(h_, L, fine_, coMass_, coStiff_, deepMassDev_, deepStiffDev_, knobs.maxBlock, knobs.denseBoundaryMax, stream_,
                    err_)) {
    plan_.reset();
    return false;
  }
  setupMs[13] = now_ms() - t0;
  rawFromPlan_ = false;
  // a knob change rebuilds the plan after the update: its combined values come
  // from the weights already in force
  if (!plan_->combine(screen_, stiffness_, stream_, err_)) {
    plan_.reset();
    return false;
  }
  if (built) *built = true;
  return true;
}

// level-0 FP64 operator: structure once per plan, values from the combined M and S
bool DeviceSystem::refresh_raw_operator() {
  const GridLevel& L0 = h_.levels[0];
  const int cnt = runs0_.count;
  if (!rawFromPlan_) {
    const NumericLevel& N = plan_->levels[0];
    rawAArena_ = DeviceArena();
    rawA_ = RawOperator();
    rawA_.runs = rawM_.runs;
    rawA_.nRuns = rawM_.nRuns;
    rawA_.coef = static_cast<double*>(rawAArena_.alloc(size_t(9) * std::max(1, cnt) * sizeof(double)));
    rawA_.planeStride = cnt;
    if (N.coarsest) {  // a single-level system: the boundary rows of the union patterns
      std::vector<int> ptr(1, 0), col;
      for (int b = 0; b < L0.numBoundary; b++) {
        for (int k = N.bd.ptr[b]; k < N.bd.ptr[b + 1]; k++) col.push_back(N.bd.col[k]);
        for (int k = N.bb.ptr[b]; k < N.bb.ptr[b + 1]; k++) col.push_back(L0.boundaryGlobal[N.bb.col[k]]);
        ptr.push_back((int)col.size());
      }
      rawA_.bPtr = rawAArena_.upload(ptr);
      rawA_.bCol = rawAArena_.upload(col);
      rawA_.bVal = static_cast<double*>(rawAArena_.alloc(std::max<size_t>(1, col.size()) * sizeof(double)));
    } else {
      rawA_.bPtr = rawAArena_.upload(N.bPtr);
      rawA_.bCol = rawAArena_.upload(N.bCol);
      rawA_.bVal = static_cast<double*>(rawAArena_.alloc(std::max<size_t>(1, N.bCol.size()) * sizeof(double)));
    }
    rawA_.bGlobal = rawM_.bGlobal;
    rawA_.nB = L0.numBoundary;
    if (!check(rawAArena_.last, "operator upload")) return false;
    rawFromPlan_ = true;
  }
  dev::launch_axpby(const_cast<double*>(rawA_.coef), screen_, rawM_.coef, stiffness_, rawS_.coef, (long long)9 * cnt, stream_);
  const NumericLevel& N = plan_->levels[0];
  if (N.coarsest) {
    // the operator's boundary rows in the union layout: bd entries, then bb entries
    std::vector<int> src;
    for (int b = 0; b < L0.numBoundary; b++) {
      for (int k = N.bd.ptr[b]; k < N.bd.ptr[b + 1]; k++) src.push_back(k);
      for (int k = N.bb.ptr[b]; k < N.bb.ptr[b + 1]; k++) src.push_back(-1 - k);
    }
    if (!src.empty()) {
      std::vector<double> bd(N.nBD), bb(N.nBB), v(src.size());
      if (!check(cudaMemcpyAsync(bd.data(), N.bdV, bd.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_), "operator rows") ||
          !check(cudaMemcpyAsync(bb.data(), N.bbV, bb.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_), "operator rows") ||
          !check(cudaStreamSynchronize(stream_), "operator rows"))
        return false;
      for (size_t i = 0; i < src.size(); i++) v[i] = src[i] >= 0 ? bd[src[i]] : bb[-1 - src[i]];
      if (!check(cudaMemcpyAsync(const_cast<double*>(rawA_.bVal), v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, stream_),
                 "operator rows"))
        return false;
    }
  } else if (!plan_->fill_raw_rows(const_cast<double*>(rawA_.bVal), stream_, err_)) {
    return false;
  }
  return check(cudaStreamSynchronize(stream_), "operator values");
}

template <typename T>
LevelValues<T> DeviceSystem::level_values(Multigrid<T>& mg, int l) {
  LevelValues<T> v;
  if (l == (int)mg.levels.size() - 1) {
    v.coarseInv = const_cast<double*>(mg.coarseInv);
    v.coarseScale = const_cast<double*>(mg.coarseScale);
    return v;
  }
  LevelDev<T>& D = mg.levels[l];
  v.planes = const_cast<T*>(D.coef);
  v.planeStride = D.planeStride;
  v.bVal = const_cast<T*>(D.bVal);
  dev::BoundaryDev<T>& B = D.B;
  v.inv = const_cast<T*>(B.inv);
  v.sinv = const_cast<T*>(B.sinv);
  v.scale = const_cast<T*>(B.scale);
  v.bdVal = const_cast<T*>(B.bdVal);
  v.asiVal = const_cast<T*>(B.asiVal);
  v.wt = const_cast<T*>(B.wt);
  v.nSp = (B.nS + 3) & ~3;
  return v;
}

// values of the resident multigrids (the FP32 base, whose derived widths share
// its buffers, and the FP64 one) for the current weights
bool DeviceSystem::refresh_multigrids() {
  Multigrid<float>* m32 = mg32_.empty() ? nullptr : mg32_.front().get();
  Multigrid<double>* m64 = mg64_.get();
  if (m32 && m32->planGen != plan_->gen) m32 = nullptr;
  if (m64 && m64->planGen != plan_->gen) m64 = nullptr;
  std::fill(plan_->ms, plan_->ms + 4, 0.0);
  double t0 = now_ms();
  for (int l = 0; l < levelsUsed_; l++) {
    if (l == levelsUsed_ - 1) {
      // boundary factorisations {values, subdomain inverses, Schur products, Schur inverse}
      setupMs[1] = plan_->ms[0] + plan_->ms[1] + plan_->ms[2] + plan_->ms[3];
      std::copy(plan_->ms, plan_->ms + 4, setupMs + 4);
      t0 = now_ms();
    }
    LevelValues<float> v32;
    LevelValues<double> v64;
    if (m32) v32 = level_values(*m32, l);
    if (m64) v64 = level_values(*m64, l);
    if (!plan_->fill_level(l, m32 ? &v32 : nullptr, m64 ? &v64 : nullptr, stream_, err_)) {
      err_ = "level " + std::to_string(l) + ": " + err_;
      return false;
    }
  }
  setupMs[2] = now_ms() - t0;
  setupMs[3] = 0;
  return true;
}

template <typename T>
bool DeviceSystem::build_multigrid(Multigrid<T>& mg, int KP) {
  const double tBuild = now_ms();
  double tBoundary = 0, tCoarse = 0, tBs[4] = {0, 0, 0, 0};
  const int L = levelsUsed_;
  // numeric: the layout here, every value by the device numeric set-up below;
  // otherwise values from the host coefficients and host (or backend) factorisations
  const bool numeric = use_numeric();
  if (numeric ? !ensure_plan() : !ensure_host_coefficients()) return false;
  DeviceDense deviceDense(stream_);
  DenseBackend* dense = knobs.deviceFactor ? &deviceDense : nullptr;
  const int bsKey[3] = {knobs.maxBlock, knobs.denseBoundaryMax, knobs.deviceFactor};
  if (!std::equal(bsKey, bsKey + 3, bsCacheKey_) || (int)bsCache_.size() != L) {
    bsCache_.assign(L, nullptr);
    std::copy(bsKey, bsKey + 3, bsCacheKey_);
  }
  DeviceArena& A = mg.arena;
  mg.levels.assign(L, LevelDev<T>());
  mg.KP = KP;
  for (int l = 0; l < L; l++) {
    const GridLevel& G = h_.levels[l];
    const LevelCoefficients* C = numeric ? nullptr : &coeffs_[l];
    LevelDev<T>& D = mg.levels[l];
    D.n = G.numTexels;
    D.nDeep = G.numDeep;
    D.nB = G.numBoundary;
    D.x = static_cast<T*>(A.alloc(size_t(D.n) * KP * sizeof(T)));
    D.b = static_cast<T*>(A.alloc(size_t(D.n) * KP * sizeof(T)));
    D.r = static_cast<T*>(A.alloc(size_t(D.n) * KP * sizeof(T)));
    if (l == L - 1) {
      const int n = G.numTexels;
      mg.coarseN = n;
      if (numeric) {
        mg.coarseInv = static_cast<double*>(A.alloc(size_t(n) * n * sizeof(double)));
        mg.coarseScale = static_cast<double*>(A.alloc(size_t(n) * sizeof(double)));
        continue;
      }
      // coarsest: scaled dense inverse (FP64)
      Csr full;
      full_matrix(G, *C, full);
      std::vector<double> denseA(size_t(n) * n, 0.0), scale(n);
      for (int i = 0; i < n; i++)
        for (int k = full.ptr[i]; k < full.ptr[i + 1]; k++)
          if (full.col[k] == i) scale[i] = 1.0 / std::sqrt(full.val[k]);
      for (int i = 0; i < n; i++)
        for (int k = full.ptr[i]; k < full.ptr[i + 1]; k++) denseA[size_t(i) * n + full.col[k]] = full.val[k] * scale[i] * scale[full.col[k]];
      const double t0 = now_ms();
      std::string e;
      const bool inverted = dense ? dense->spd_inverse_batched(denseA.data(), std::vector<int64_t>(1, 0), std::vector<int>(1, n), e)
                                  : dense_spd_inverse(denseA.data(), n, true);
      if (!inverted) { err_ = "coarsest operator is not positive definite" + (e.empty() ? std::string() : ": " + e); return false; }
      tCoarse += now_ms() - t0;
      mg.coarseInv = A.upload(denseA);
      mg.coarseScale = A.upload(scale);
      continue;
    }
    // deep runs + reciprocal coefficient planes
    DeepRuns R = build_deep_runs(G);
    if (numeric) {
      if ((int)R.texel.size() != R.count) { err_ = "deep runs: texel list and count differ"; return false; }
      if (!plan_->set_run_order(l, R.texel, err_)) return false;
      D.coef = static_cast<T*>(A.alloc(size_t(10) * std::max(1, R.count) * sizeof(T)));
    } else {
      std::vector<T> planes(size_t(10) * std::max(1, R.count));
#pragma omp parallel for schedule(static)
      for (int i = 0; i < R.count; i++) {
        const double* c = &C->deep[10 * size_t(R.texel[i])];
        const double c4 = c[4], inv = 1.0 / c4;
        for (int k = 0; k < 9; k++) planes[size_t(k) * R.count + i] = T(k == 4 ? inv : c[k] * inv);
        planes[size_t(9) * R.count + i] = T(c4);
      }
      D.coef = A.upload(planes);
    }
    D.runs = A.upload(R.runs);
    D.nRuns = (int)R.runs.size();
    std::copy(R.runStart, R.runStart + 5, D.runStart);
    D.planeStride = R.count;
    // raster lines in blocks for the row smoother (two colours per launch)
    {
      RowBins RB;
      if (build_row_bins(G, R, RB)) {
        for (int p = 0; p < 2; p++) {
          D.rowLines[p] = A.upload(RB.lines[p]);
          D.rowLineOf[p] = A.upload(RB.lineOf[p]);
          D.nRowBins[p] = RB.bins[p];
        }
        D.rowBlock = RB.block;
        D.rowSlots = RB.slots;
      }
    }
    // tiles of the fused smoother (FP32 levels it runs on; the tile_texels knob
    // drops the multigrids when it changes; host-built values only)
    if (!numeric && sizeof(T) == 4 && G.numDeep >= kTileBuildMin && knobs.tileTexels > 0 && G.numDeep >= knobs.tileTexels) {
      TileLayout TL;
      build_tiles(G, *C, TL);
      D.tiles = A.upload(TL.tiles);
      D.nTiles = (int)TL.tiles.size();
      D.tileSegs = A.upload(TL.segs);
      D.tileCoef = A.upload(TL.coef);
      D.tileNbrs = A.upload(TL.nbrs);
      D.tileSync = A.zeros<int>(2 + TL.tiles.size());
      std::copy(TL.tileStart, TL.tileStart + 5, D.tileStart);
    }
    // chart groups of the runs (grouped smoother): deep texels of different
    // charts never neighbour each other, so during Gauss-Seidel sweeps (which
    // leave boundary texels alone) every chart is independent
    {
      std::vector<int> grp;
      int maxDeep = 0, maxSpan = 0;
      if (chart_groups(G, R, grp, maxDeep, maxSpan)) {
        D.groups = A.upload(grp);
        D.nGroups = (int)grp.size() / 10;
        D.maxGroupDeep = maxDeep;
        D.maxGroupSpan = maxSpan;
        for (int gi = 0; gi < D.nGroups; gi++)
          for (int c = 0; c < 4; c++) D.maxGroupColourRuns = std::max(D.maxGroupColourRuns, grp[10 * gi + 4 + c]);
      }
    }
    // boundary rows (merged BD + BB, global columns)
    if (numeric) {
      const NumericLevel& N = plan_->levels[l];
      D.bPtr = A.upload(N.bPtr);
      D.bCol = A.upload(N.bCol);
      D.bVal = static_cast<T*>(A.alloc(std::max<size_t>(1, N.bCol.size()) * sizeof(T)));
    } else {
      std::vector<int> ptr(1, 0), col;
      std::vector<T> val;
      for (int b = 0; b < G.numBoundary; b++) {
        for (int k = C->bd.ptr[b]; k < C->bd.ptr[b + 1]; k++) { col.push_back(C->bd.col[k]); val.push_back(T(C->bd.val[k])); }
        for (int k = C->bb.ptr[b]; k < C->bb.ptr[b + 1]; k++) { col.push_back(G.boundaryGlobal[C->bb.col[k]]); val.push_back(T(C->bb.val[k])); }
        ptr.push_back((int)col.size());
      }
      D.bPtr = A.upload(ptr);
      D.bCol = A.upload(col);
      D.bVal = A.upload(val);
    }
    D.bGlobal = A.upload(G.boundaryGlobal);
    // exact boundary solver: the layout of its structure (a host set-up with
    // values, or the numeric plan's structure with value buffers left to fill)
    auto layout_boundary = [&](const auto& bs, const BoundarySolverSetup* vals) -> bool {
      dev::BoundaryDev<T>& B = D.B;
      B.nb = bs.nb;
      B.nSub = bs.nSub;
      B.nI = bs.nI;
      B.nS = bs.nS;
      // subdomain inverses, rows padded to a multiple of 4; one task per 128 rows
      std::vector<long long> off(bs.nSub + 1, 0);
      std::vector<int4> tasks;
      int maxM = 0;
      for (int p = 0; p < bs.nSub; p++) {
        const int m = bs.subPtr[p + 1] - bs.subPtr[p], mp = (m + 3) & ~3;
        off[p + 1] = off[p] + (long long)m * mp;
        maxM = std::max(maxM, m);
        for (int rq = 0; rq < mp / 4; rq += 32) tasks.push_back(make_int4(p, rq, 0, m));
      }
      if (maxM > dev::kBoundaryChunkMax) { err_ = "boundary subdomain larger than the device chunk limit"; return false; }
      if (vals) {
        std::vector<T> inv(size_t(off[bs.nSub]), T(0));
#pragma omp parallel for schedule(dynamic, 4)
        for (int p = 0; p < bs.nSub; p++) {
          const int m = bs.subPtr[p + 1] - bs.subPtr[p], mp = (m + 3) & ~3;
          const double* src = &vals->inv[size_t(vals->invOff[p])];
          for (int j = 0; j < m; j++)
            for (int a = 0; a < m; a++) inv[size_t(off[p]) + size_t(j) * mp + a] = T(src[size_t(j) * m + a]);
        }
        B.inv = A.upload(inv);
      } else {
        B.inv = static_cast<T*>(A.alloc(std::max<size_t>(1, size_t(off[bs.nSub])) * sizeof(T)));
      }
      // blocks per row group: enough chunks for one wave of bsBlocksPerSm
      // resident blocks on each of the 148 SMs, each warp still taking >= 4 j steps
      const int target = knobs.bsBlocksPerSm * 148;
      auto chunks_for = [target](int tasks, int m, int minChunks) {
        int c = (target + std::max(1, tasks) - 1) / std::max(1, tasks);
        c = std::min(c, std::max(1, m / 32));
        return std::max(c, std::max(1, minChunks));
      };
      std::vector<int> rowSub(std::max(1, bs.nI));
      for (int p = 0; p < bs.nSub; p++)
        for (int k = bs.subPtr[p]; k < bs.subPtr[p + 1]; k++) rowSub[k] = p;
      B.subPtr = A.upload(bs.subPtr);
      B.rowSub = A.upload(rowSub);
      B.invOff = A.upload(off);
      B.subTasks = A.upload(tasks);
      B.nSubTasks = (int)tasks.size();
      B.subChunks = chunks_for(B.nSubTasks, maxM, 1);
      B.subPart = static_cast<T*>(A.alloc(size_t(std::max(1, B.nSubTasks)) * B.subChunks * 128 * KP * sizeof(T)));
      B.subCount = A.zeros<int>(std::max(1, B.nSubTasks));
      // separator Schur complement inverse, same layout
      if (bs.nS > 0) {
        const int nS = bs.nS, nSp = (nS + 3) & ~3;
        if (vals) {
          std::vector<T> sinv(size_t(nS) * nSp, T(0));
          for (int j = 0; j < nS; j++)
            for (int a = 0; a < nS; a++) sinv[size_t(j) * nSp + a] = T(vals->Sinv[size_t(j) * nS + a]);
          B.sinv = A.upload(sinv);
        } else {
          B.sinv = static_cast<T*>(A.alloc(size_t(nS) * nSp * sizeof(T)));
        }
        std::vector<int4> st;
        for (int rq = 0; rq < nSp / 4; rq += 32) st.push_back(make_int4(0, rq, 0, nS));
        B.schurTasks = A.upload(st);
        B.nSchurTasks = (int)st.size();
        B.schurChunks = chunks_for(B.nSchurTasks, nS, (nS + dev::kBoundaryChunkMax - 1) / dev::kBoundaryChunkMax);
        B.schurPart = static_cast<T*>(A.alloc(size_t(B.nSchurTasks) * B.schurChunks * 128 * KP * sizeof(T)));
        B.schurCount = A.zeros<int>(B.nSchurTasks);
      }
      // back substitution: W_p column-major with its separator columns
      std::vector<long long> wOff(bs.wOff.begin(), bs.wOff.end());
      B.touchPtr = A.upload(bs.touchPtr);
      B.touch = A.upload(bs.touch);
      B.wOff = A.upload(wOff);
      std::vector<int> pg(bs.nb);
      for (int k = 0; k < bs.nb; k++) pg[k] = G.boundaryGlobal[bs.order[k]];
      B.posGlobal = A.upload(pg);
      B.bdPtr = A.upload(bs.BD.ptr);
      B.bdCol = A.upload(bs.BD.col);
      B.asiPtr = A.upload(bs.ASI.ptr);
      B.asiCol = A.upload(bs.ASI.col);
      auto values = [&](const std::vector<double>& v, size_t n) -> const T* {
        if (!vals) return static_cast<T*>(A.alloc(std::max<size_t>(1, n) * sizeof(T)));
        std::vector<T> t(v.begin(), v.end());
        return A.upload(t);
      };
      B.wt = values(vals ? vals->W : std::vector<double>(), size_t(bs.wOff.back()));
      B.scale = values(vals ? vals->scale : std::vector<double>(), size_t(bs.nb));
      B.bdVal = values(vals ? vals->BD.val : std::vector<double>(), bs.BD.col.size());
      B.asiVal = values(vals ? vals->ASI.val : std::vector<double>(), bs.ASI.col.size());
      B.y = static_cast<T*>(A.alloc(size_t(std::max(1, bs.nI)) * KP * sizeof(T)));
      B.xs = static_cast<T*>(A.alloc(size_t(std::max(1, bs.nS)) * KP * sizeof(T)));
      B.rhat = static_cast<T*>(A.alloc(size_t(std::max(1, bs.nb)) * KP * sizeof(T)));
      return true;
    };
    if (numeric) {
      if (!layout_boundary(plan_->levels[l].sym, nullptr)) return false;
    } else {
      if (!bsCache_[l]) {
        auto built = std::make_shared<BoundarySolverSetup>();
        const double t0 = now_ms();
        if (!build_boundary_solver(C->bb, C->bd, knobs.maxBlock, knobs.denseBoundaryMax, *built, err_, dense)) {
          err_ = "level " + std::to_string(l) + ": " + err_;
          return false;
        }
        tBoundary += now_ms() - t0;
        for (int q = 0; q < 4; q++) tBs[q] += built->ms[q];
        bsCache_[l] = built;
      }
      if (!layout_boundary(*bsCache_[l], bsCache_[l].get())) return false;
    }
    // transfers to / from level l+1
    {
      const GridLevel& Cg = h_.levels[l + 1];
      std::vector<dev::RestrictRun> rr;
      for (const Line& ln : Cg.restrictionLines) {
        const int len = (ln.end - ln.start) / 2 + 1;
        for (int p = 0; p < len; p += 32) rr.push_back({ln.coeff + p, ln.start + 2 * p, ln.prev + 2 * p, ln.next + 2 * p, std::min(32, len - p)});
      }
      D.rruns = A.upload(rr);
      D.nRRuns = (int)rr.size();
      const Csr& Rb = G.boundaryRestriction;
      std::vector<T> rv(Rb.val.begin(), Rb.val.end());
      D.rbPtr = A.upload(Rb.ptr);
      D.rbCol = A.upload(Rb.col);
      D.rbVal = A.upload(rv);
      D.rbOut = A.upload(Cg.boundaryGlobal);
      D.nRB = Rb.rows;
      std::vector<dev::ProlongRun> pr;
      for (const ProlongationLine& pl : G.prolongationLines)
        for (int p = 0; p < pl.length; p += 32)
          pr.push_back({pl.start + p, p, std::min(32, pl.length - p), pl.center, pl.prev, pl.next, pl.aligned});
      D.pruns = A.upload(pr);
      D.nPRuns = (int)pr.size();
    }
  }
  if (!check(A.last, "multigrid upload")) return false;
  // whether this device can run the coarse-level kernels (queried outside any capture)
  mg.clusterOK = dev::coarse_cycle_cluster_ctas(sizeof(T) == 8, (KP % 4 == 0) ? 4 : 1) > 0;
  mg.gridOK = dev::coarse_cycle_grid_ctas(sizeof(T) == 8, (KP % 4 == 0) ? 4 : 1) > 0;
  mg.levelsDev = A.upload(mg.levels);
  mg.barrier = static_cast<dev::GridBarrierState*>(A.alloc(sizeof(dev::GridBarrierState)));
  if (!check(A.last, "multigrid upload")) return false;
  if (numeric) {
    // every value of the layout above, on the device
    const double tLayout = now_ms() - tBuild;
    std::fill(plan_->ms, plan_->ms + 4, 0.0);
    for (int l = 0; l + 1 < L; l++) {
      LevelValues<T> v = level_values(mg, l);
      if (!fill_one(*plan_, l, v, stream_, err_)) {
        err_ = "level " + std::to_string(l) + ": " + err_;
        return false;
      }
    }
    std::copy(plan_->ms, plan_->ms + 4, tBs);
    tBoundary = tBs[0] + tBs[1] + tBs[2] + tBs[3];
    const double t0 = now_ms();
    LevelValues<T> vc = level_values(mg, L - 1);
    if (!fill_one(*plan_, L - 1, vc, stream_, err_)) {
      err_ = "coarsest level: " + err_;
      return false;
    }
    tCoarse = now_ms() - t0;
    mg.planGen = plan_->gen;
    setupMs[1] = tBoundary;
    setupMs[2] = tCoarse;
    setupMs[3] = tLayout;
    std::copy(tBs, tBs + 4, setupMs + 4);
  } else {
    mg.planGen = -1;
    setupMs[1] = tBoundary;
    setupMs[2] = tCoarse;
    setupMs[3] = now_ms() - tBuild - tBoundary - tCoarse;
    std::copy(tBs, tBs + 4, setupMs + 4);
  }
  return check(cudaMemset(mg.barrier, 0, sizeof(dev::GridBarrierState)), "grid barrier");
}

template bool DeviceSystem::build_multigrid<float>(Multigrid<float>&, int);
template bool DeviceSystem::build_multigrid<double>(Multigrid<double>&, int);

// Another channel stride on the same levels: the structure is base's (shared,
// base outlives it), the vectors and the boundary solve's work are new.
template <typename T>
bool DeviceSystem::derive_multigrid(const Multigrid<T>& base, Multigrid<T>& mg, int KP) {
  DeviceArena& A = mg.arena;
  mg.levels = base.levels;
  mg.KP = KP;
  mg.coarseN = base.coarseN;
  mg.coarseInv = base.coarseInv;
  mg.coarseScale = base.coarseScale;
  mg.planGen = base.planGen;
  for (LevelDev<T>& D : mg.levels) {
    D.x = static_cast<T*>(A.alloc(size_t(D.n) * KP * sizeof(T)));
    D.b = static_cast<T*>(A.alloc(size_t(D.n) * KP * sizeof(T)));
    D.r = static_cast<T*>(A.alloc(size_t(D.n) * KP * sizeof(T)));
    if (D.nTiles > 0) D.tileSync = A.zeros<int>(2 + size_t(D.nTiles));
    dev::BoundaryDev<T>& B = D.B;
    if (B.nb == 0) continue;
    B.subPart = static_cast<T*>(A.alloc(size_t(std::max(1, B.nSubTasks)) * B.subChunks * 128 * KP * sizeof(T)));
    B.subCount = A.zeros<int>(std::max(1, B.nSubTasks));
    if (B.nS > 0) {
      B.schurPart = static_cast<T*>(A.alloc(size_t(B.nSchurTasks) * B.schurChunks * 128 * KP * sizeof(T)));
      B.schurCount = A.zeros<int>(B.nSchurTasks);
    }
    B.y = static_cast<T*>(A.alloc(size_t(std::max(1, B.nI)) * KP * sizeof(T)));
    B.xs = static_cast<T*>(A.alloc(size_t(std::max(1, B.nS)) * KP * sizeof(T)));
    B.rhat = static_cast<T*>(A.alloc(size_t(std::max(1, B.nb)) * KP * sizeof(T)));
  }
  if (!check(A.last, "multigrid vectors")) return false;
  mg.clusterOK = dev::coarse_cycle_cluster_ctas(sizeof(T) == 8, (KP % 4 == 0) ? 4 : 1) > 0;
  mg.gridOK = dev::coarse_cycle_grid_ctas(sizeof(T) == 8, (KP % 4 == 0) ? 4 : 1) > 0;
  mg.levelsDev = A.upload(mg.levels);
  mg.barrier = static_cast<dev::GridBarrierState*>(A.alloc(sizeof(dev::GridBarrierState)));
  if (!check(A.last, "multigrid vectors")) return false;
  return check(cudaMemset(mg.barrier, 0, sizeof(dev::GridBarrierState)), "grid barrier");
}

Multigrid<float>* DeviceSystem::mg32_for(int KP) {
  for (auto& m : mg32_)
    if (m->KP == KP) return m.get();
  std::unique_ptr<Multigrid<float>> m(new Multigrid<float>());
  const bool ok = mg32_.empty() ? build_multigrid(*m, KP) : derive_multigrid(*mg32_.front(), *m, KP);
  if (!ok) return nullptr;
  mg32_.push_back(std::move(m));
  return mg32_.back().get();
}

// ----------------------------------------------------------------------------
// V-cycle
// ----------------------------------------------------------------------------
std::vector<double> DeviceSystem::level_stats() const {
  std::vector<double> v;
  if (mg32_.empty()) return v;
  for (const LevelDev<float>& D : mg32_.front()->levels) {
    const dev::BoundaryDev<float>& B = D.B;
    const double row[] = {double(D.n), double(D.nDeep), double(D.nB), double(B.nI), double(B.nS),
                          double(B.nSubTasks) * B.subChunks, double(B.nSchurTasks) * B.schurChunks, double(D.nGroups),
                          double(D.maxGroupDeep)};
    v.insert(v.end(), row, row + 9);
  }
  return v;
}

bool DeviceSystem::cluster_timeline(std::vector<unsigned long long>& out) {
  out.clear();
  if (!timeline_) return true;
  out.resize(1024);
  return check(cudaMemcpy(out.data(), timeline_, 1024 * sizeof(unsigned long long), cudaMemcpyDeviceToHost), "timeline");
}

unsigned long long* DeviceSystem::clusterTimeline() {
  // allocated before the refinement graph is captured (solve_mixed)
  return (profiling_ && knobs.traceLevels) ? timeline_ : nullptr;
}

void DeviceSystem::trace_mark(int i, cudaStream_t s) {
  if (!profiling_ || !knobs.traceLevels || i >= (int)traceEv_.size()) return;
  cudaEventRecordWithFlags(traceEv_[i], s, cudaEventRecordExternal);
}

// The persistent coarse-level kernel records a grid-barrier timeout in its
// barrier state; after a solve that used it, the word is copied back with the
// results and checked once the stream is done.
template <typename T>
void DeviceSystem::queue_barrier_check(Multigrid<T>& mg, cudaStream_t s) {
  if (!(usedGridBarrier_ || usedTileWait_) || !mg.barrier) return;
  if (!barrierErrHost_ && cudaMallocHost(&barrierErrHost_, sizeof(unsigned int)) != cudaSuccess) {
    barrierErrHost_ = nullptr;
    return;
  }
  *barrierErrHost_ = 0;
  cudaMemcpyAsync(barrierErrHost_, &mg.barrier->error, sizeof(unsigned int), cudaMemcpyDeviceToHost, s);
}
template <typename T>
bool DeviceSystem::barrier_ok(Multigrid<T>& mg) {
  if (!(usedGridBarrier_ || usedTileWait_) || !mg.barrier || !barrierErrHost_ || *barrierErrHost_ == 0) return true;
  const unsigned int code = *barrierErrHost_;
  cudaMemset(mg.barrier, 0, sizeof(dev::GridBarrierState));  // usable again for the next solve
  err_ = code == 2 ? "tile smoother: a wait for a neighbouring tile timed out (results discarded)"
                   : "coarse-level kernel: a grid barrier timed out (results discarded)";
  return false;
}

// Neighbour slots (k = 3 (dy + 1) + dx + 1, centre 4 excluded) that a colour
// pass of the first sweep from a zero iterate may skip: a neighbour is read
// only when its colour comes earlier in the sweep (updated) -- later colours
// and boundary texels still hold exact zeros, whose terms add nothing.
static int zero_start_skip(int c) {
  int skip = 0;
  for (int k = 0; k < 9; k++) {
    if (k == 4) continue;
    const int dx = k % 3 - 1, dy = k / 3 - 1;
    const int nc = c ^ ((dx != 0 ? 1 : 0) | (dy != 0 ? 2 : 0));
    if (nc > c) skip |= 1 << k;
  }
  return skip;
}

template <typename T, int W>
void DeviceSystem::colour_sweep(const LevelDev<T>& D, int KP, bool reverse, bool fromZero, bool rhsEarly, cudaStream_t s) {
  // FP32 multigrids with one channel group only (k <= 4): with FP64 vectors
  // the row smoother's blocks need twice the shared memory and more registers,
  // and with several channel groups every group's block loads the
  // coefficients again (a colour pass shares them across a warp); both were
  // measured slower than the colour passes
  if (row_sweeps_on(D, KP, sizeof(T), W)) {
    // a colour's zero-start skips cover its rows above and below, or its own
    // row, whole: the row smoother skips them as groups
    constexpr int kRows = 1 | 2 | 4 | 64 | 128 | 256, kOwn = 8 | 32;
    for (int h = 0; h < 2; h++) {
      const int rows = reverse ? 1 - h : h;
      const int cA = 2 * rows + (reverse ? 1 : 0), cB = cA ^ 1;
      int skip = 0;
      if (fromZero) {
        const int sa = zero_start_skip(cA), sb = zero_start_skip(cB);
        skip = ((sa & kRows) ? 1 : 0) | ((sa & kOwn) ? 2 : 0) | ((sb & kRows) ? 4 : 0) | ((sb & kOwn) ? 8 : 0);
      }
      dev::launch_gs_rows<T, W>(D, rows, reverse, KP, s, skip, h > 0 || rhsEarly);
    }
    return;
  }
  for (int p = 0; p < 4; p++) {
    const int c = reverse ? 3 - p : p;
    dev::launch_gs_colour<T, W>(D.runs + D.runStart[c], D.runStart[c + 1] - D.runStart[c], D.coef, D.planeStride, D.b, D.x, KP, s,
                                fromZero ? zero_start_skip(c) : 0, p > 0 || rhsEarly);
  }
}
template void DeviceSystem::colour_sweep<float, 1>(const LevelDev<float>&, int, bool, bool, bool, cudaStream_t);
template void DeviceSystem::colour_sweep<float, 4>(const LevelDev<float>&, int, bool, bool, bool, cudaStream_t);
template void DeviceSystem::colour_sweep<double, 1>(const LevelDev<double>&, int, bool, bool, bool, cudaStream_t);
template void DeviceSystem::colour_sweep<double, 4>(const LevelDev<double>&, int, bool, bool, bool, cudaStream_t);

// One smoothing step of `sweeps` sweeps with the fused tile smoother, in
// place: `tileRounds` rounds (one launch each) over the tiles in tile-colour
// order (3..0 with reverse), the sweeps split between the rounds; only the
// first round may start from a zero iterate.  With tileFinish, one global
// colour sweep follows.
template <typename T>
void DeviceSystem::tile_smooth(Multigrid<T>& mg, LevelDev<T>& D, int sweeps, bool reverse, bool zeroStart, cudaStream_t s,
                               bool prof) {
  const int KP = mg.KP;
  const int rounds = std::max(1, std::min(knobs.tileRounds, sweeps));
  dev::TileRound a;
  a.tiles = D.tiles;
  a.segs = D.tileSegs;
  a.nbrs = D.tileNbrs;
  a.coef = D.tileCoef;
  a.rhs = reinterpret_cast<const float*>(D.b);
  a.sync = D.tileSync;
  a.err = &mg.barrier->error;
  a.nTiles = D.nTiles;
  std::copy(D.tileStart, D.tileStart + 5, a.tileStart);
  a.reverse = reverse ? 1 : 0;
  // profiling: the rounds are timed as `rounds` launch groups (the closing
  // colour sweep is not part of them)
  if (prof) cudaEventRecordWithFlags(profEv_[2], s, cudaEventRecordExternal);
  for (int r = 0; r < rounds; r++) {
    a.sweeps = sweeps / rounds + (r < sweeps % rounds ? 1 : 0);
    a.zeroStart = zeroStart && r == 0 ? 1 : 0;
    dev::launch_tile_smooth(a, reinterpret_cast<float*>(D.x), KP, s);
  }
  if (prof) {
    cudaEventRecordWithFlags(profEv_[3], s, cudaEventRecordExternal);
    profPostSweeps_ = rounds;
    profTiled_ = true;
    profRows_ = false;
  }
  usedTileWait_ = true;
  if (knobs.tileFinish) {
    if (KP % 4 == 0)
      colour_sweep<T, 4>(D, KP, reverse, false, false, s);
    else
      colour_sweep<T, 1>(D, KP, reverse, false, false, s);
  }
}

template <typename T, int W>
void DeviceSystem::vcycle(Multigrid<T>& mg, cudaStream_t s, bool zeroStart) {
  const int L = (int)mg.levels.size();
  const int KP = mg.KP;
  // levels [lc, L) run in the coarse-level cluster when it is enabled: from the
  // first level below the finest with at most clusterTexels texels
  int lc = L - 1;
  bool grid = false;
  if (knobs.gridTexels > 0 && mg.gridOK) {
    for (int l = 1; l + 1 < L; l++)
      if (mg.levels[l].n <= knobs.gridTexels) { lc = l; grid = true; break; }
  } else if (knobs.clusterTexels > 0 && mg.clusterOK) {
    for (int l = 1; l + 1 < L; l++)
      if (mg.levels[l].n <= knobs.clusterTexels) { lc = l; break; }
  }
  const dev::CoarseSweeps sw{knobs.preSweeps, knobs.postSweeps, knobs.coarsePreSweeps, knobs.coarsePostSweeps, knobs.coarseFrom,
                             knobs.preBoundary, knobs.postBoundary};
  dev::GridBarrierState* barrier = grid ? mg.barrier : nullptr;
  trace_mark(0, s);
  if (profiling_) profSweeps_ = profPostSweeps_ = 0;
  for (int l = 0; l < lc; l++) {
    LevelDev<T>& D = mg.levels[l];
    LevelDev<T>& C = mg.levels[l + 1];
    // D.x of levels > 0 was cleared by the restriction into this level
    if (knobs.preBoundary) dev::launch_boundary_solve<T, W>(D.B, D.b, D.x, KP, s);
    if (tiled(D, KP) && knobs.tilePreSweeps > 0) {
      // x = 0 on entry (a refinement step's correction, or a level entered
      // through the restriction) unless a boundary solve ran first
      tile_smooth(mg, D, knobs.tilePreSweeps, false, (l > 0 || zeroStart) && !knobs.preBoundary, s, false);
    } else if (grouped(D, KP) && pre_sweeps(l) > 0) {
      dev::launch_gs_groups<T, W>(D, pre_sweeps(l), false, KP, s);
    } else {
      // timed on level 0: every full sweep (all but a first sweep that skips
      // zeros), here and in the post-smoothing; the sweep average is reported
      const bool fromZero0 = zeroStart && knobs.zeroStartSkip && l == 0 && !knobs.preBoundary;
      const int firstFull = fromZero0 ? 1 : 0;
      for (int sw = 0; sw < pre_sweeps(l); sw++) {
        const bool prof = profiling_ && l == 0;
        if (prof && sw == firstFull) cudaEventRecordWithFlags(profEv_[0], s, cudaEventRecordExternal);
        colour_sweep<T, W>(D, KP, false, fromZero0 && sw == 0, sw > 0, s);
        if (prof && sw == pre_sweeps(l) - 1 && sw >= firstFull) {
          cudaEventRecordWithFlags(profEv_[1], s, cudaEventRecordExternal);
          profSweeps_ = pre_sweeps(l) - firstFull;
        }
      }
    }
    // a level entered with a zero iterate and left unsmoothed (no pre-sweeps, no
    // boundary solve) has residual b - A 0 = b exactly: restrict b itself
    const bool unsmoothed = knobs.zeroStartSkip && (l > 0 || zeroStart) && pre_sweeps(l, D, KP) == 0 && !knobs.preBoundary;
    // after smoothing or a boundary solve (x written) the right-hand side of this
    // level is not what the previous launch wrote
    if (!unsmoothed)
      dev::launch_residual<T, W>(D.runs, D.nRuns, D.coef, D.planeStride, D.bPtr, D.bCol, D.bVal, D.bGlobal, D.nB, D.b, D.x, D.r, KP, s,
                                 pre_sweeps(l, D, KP) > 0 || knobs.preBoundary);
    dev::launch_restrict<T, W>(D.rruns, D.nRRuns, D.rbPtr, D.rbCol, D.rbVal, D.rbOut, D.nRB, unsmoothed ? D.b : D.r, C.b, C.x, C.n, KP,
                               s);
    trace_mark(l + 1, s);
  }
  if (lc < L - 1) {
    // coarse levels in one kernel (one cluster, or every SM with grid barriers);
    // a large coarsest level is solved by an ordinary launch in between
    const bool whole = mg.coarseN <= dev::kCoarseInKernelMax(grid);
    if (whole) {
      dev::launch_coarse_cycle<T, W>(mg.levelsDev, lc, L, 2, sw, KP, mg.coarseN, mg.coarseInv, mg.coarseScale, clusterTimeline(),
                                     barrier, s);
    } else {
      dev::launch_coarse_cycle<T, W>(mg.levelsDev, lc, L, 0, sw, KP, mg.coarseN, mg.coarseInv, mg.coarseScale, clusterTimeline(),
                                     barrier, s);
      dev::launch_coarse_solve<T, W>(mg.coarseN, mg.coarseInv, mg.coarseScale, mg.levels[L - 1].b, mg.levels[L - 1].x, KP, s);
      dev::launch_coarse_cycle<T, W>(mg.levelsDev, lc, L, 1, sw, KP, mg.coarseN, mg.coarseInv, mg.coarseScale, clusterTimeline(),
                                     barrier, s);
    }
    usedGridBarrier_ = usedGridBarrier_ || grid;
    for (int i = lc + 1; i <= L + 1 + (L - 2 - lc); i++) trace_mark(i, s);  // the cluster's levels count as one segment
  } else {
    dev::launch_coarse_solve<T, W>(mg.coarseN, mg.coarseInv, mg.coarseScale, mg.levels[L - 1].b, mg.levels[L - 1].x, KP, s);
    trace_mark(L, s);
  }
  for (int l = std::min(lc, L - 1) - 1; l >= 0; l--) {
    LevelDev<T>& D = mg.levels[l];
    dev::launch_prolong_add<T, W>(D.pruns, D.nPRuns, mg.levels[l + 1].x, D.x, KP, s);
    if (knobs.postBoundary) dev::launch_boundary_solve<T, W>(D.B, D.b, D.x, KP, s, true);
    if (tiled(D, KP) && knobs.tilePostSweeps > 0) {
      // timed on level 0: the post-smoothing rounds (coefficients, rhs, x read
      // and written once each per round)
      tile_smooth(mg, D, knobs.tilePostSweeps, true, false, s, profiling_ && l == 0);
    } else if (grouped(D, KP) && post_sweeps(l) > 0) {
      // after the prolongation and the boundary solve, which leave the right-hand side alone
      dev::launch_gs_groups<T, W>(D, post_sweeps(l), true, KP, s, true);
    } else {
      const bool prof = profiling_ && l == 0 && post_sweeps(l) > 0;
      if (prof) cudaEventRecordWithFlags(profEv_[2], s, cudaEventRecordExternal);
      for (int sw = 0; sw < post_sweeps(l); sw++) colour_sweep<T, W>(D, KP, true, false, sw > 0, s);
      if (prof) {
        cudaEventRecordWithFlags(profEv_[3], s, cudaEventRecordExternal);
        profPostSweeps_ = post_sweeps(l);
        profTiled_ = false;
        profRows_ = row_sweeps_on(D, KP, sizeof(T), W);
      }
    }
    trace_mark(L + 1 + (L - 2 - l), s);
  }
}

template void DeviceSystem::vcycle<float, 1>(Multigrid<float>&, cudaStream_t, bool);
template void DeviceSystem::vcycle<float, 4>(Multigrid<float>&, cudaStream_t, bool);
template void DeviceSystem::vcycle<double, 1>(Multigrid<double>&, cudaStream_t, bool);
template void DeviceSystem::vcycle<double, 4>(Multigrid<double>&, cudaStream_t, bool);

// ----------------------------------------------------------------------------
// solve work and drivers
// ----------------------------------------------------------------------------
bool DeviceSystem::ensure_work(int kk) {
  if (kk <= workK_) return true;
  const int k = k_capacity(kk);
  workArena_ = DeviceArena();
  const size_t n = h_.levels[0].numTexels;
  b64_ = workArena_.zeros<double>(n * k);
  x64_ = workArena_.zeros<double>(n * k);
  r64_ = workArena_.zeros<double>(n * k);
  const int blocks = dev::raw_operator_blocks(rawM_.nRuns, h_.levels[0].numBoundary, k);
  partials_ = workArena_.zeros<double>(size_t(blocks) * 2 * k);
  frozen_ = workArena_.zeros<int>(size_t(k));
  frozenHost_.assign(k, 0);
  sums_ = workArena_.zeros<double>(2 * size_t(k));
  if (sumsHost_) cudaFreeHost(sumsHost_);
  sumsMapped_ = nullptr;
  if (!check(cudaHostAlloc(&sumsHost_, 2 * size_t(k) * sizeof(double), cudaHostAllocMapped), "cudaHostAlloc")) return false;
  if (cudaHostGetDevicePointer(&sumsMapped_, sumsHost_, 0) != cudaSuccess) {
    sumsMapped_ = nullptr;
    cudaGetLastError();  // not mappable here: the norms come back by copy
  }
  if (!check(workArena_.last, "work allocation")) return false;
  workK_ = k;
  invalidate_graph();
  return true;
}

bool DeviceSystem::read_norms(int k, cudaStream_t s, const char* what) {
  if (sumsMapped_) {
    kernelLaunches += 1;
    dev::launch_copy_f64(sumsMapped_, sums_, 2 * k, s);
    if (!check(cudaGetLastError(), "norms to host")) return false;
  } else if (!check(cudaMemcpyAsync(sumsHost_, sums_, 2 * size_t(k) * sizeof(double), cudaMemcpyDeviceToHost, s), "d2h norms")) {
    return false;
  }
  return check(cudaStreamSynchronize(s), what);
}

bool DeviceSystem::upload_flags(int k, cudaStream_t s) {
  unsigned long long mask = 0;
  for (int c = 0; c < k; c++)
    if (frozenHost_[c] == 1) mask |= 1ull << c;
  kernelLaunches += 1;
  dev::launch_set_flags(frozen_, mask, k, s);
  return check(cudaGetLastError(), "frozen flags");
}

bool DeviceSystem::raw_apply_dev(const RawOperator& op, const double* b, const double* x, double* out, int k, int mode,
                                 cudaStream_t s, double* sumsHost) {
  dev::launch_raw_operator(op.runs, op.nRuns, op.coef, op.planeStride, op.bPtr, op.bCol, op.bVal, op.bGlobal, op.nB, b, x, out, k,
                           mode, partials_, sums_, s);
  if (!sumsHost) return check(cudaGetLastError(), "raw operator");
  return check(cudaMemcpyAsync(sumsHost, sums_, 2 * size_t(k) * sizeof(double), cudaMemcpyDeviceToHost, s), "d2h norms") &&
         check(cudaStreamSynchronize(s), "raw operator");
}

bool DeviceSystem::apply(int which, const double* x, double* y, int k) {
  if (!err_.empty()) return false;
  cudaSetDevice(device_);
  if (k < 1 || k > 64) { err_ = "k must be in [1, 64]"; return false; }
  const RawOperator* op = which == 1 ? &rawM_ : which == 2 ? &rawS_ : &rawA_;
  if (which == 0 && !updated_) { err_ = "apply(A) before update"; return false; }
  if (!ensure_work(k)) return false;
  const size_t n = h_.levels[0].numTexels;
  return check(cudaMemcpyAsync(x64_, x, n * k * 8, cudaMemcpyHostToDevice, stream_), "h2d") &&
         raw_apply_dev(*op, nullptr, x64_, r64_, k, 1, stream_, nullptr) &&
         check(cudaMemcpyAsync(y, r64_, n * k * 8, cudaMemcpyDeviceToHost, stream_), "d2h") &&
         check(cudaStreamSynchronize(stream_), "apply");
}

bool DeviceSystem::apply_combination(double a, double b, const double* x, double* y, int k) {
  if (!err_.empty()) return false;
  cudaSetDevice(device_);
  if (k < 1 || k > 64) { err_ = "k must be in [1, 64]"; return false; }
  if (!ensure_work(k)) return false;
  const size_t n = h_.levels[0].numTexels;
  if (!check(cudaMemcpyAsync(x64_, x, n * k * 8, cudaMemcpyHostToDevice, stream_), "h2d") ||
      !raw_apply_dev(rawM_, nullptr, x64_, r64_, k, 1, stream_, nullptr) ||
      !raw_apply_dev(rawS_, nullptr, x64_, b64_, k, 1, stream_, nullptr))
    return false;
  dev::launch_axpby(r64_, a, r64_, b, b64_, (long long)(n * k), stream_);
  return check(cudaMemcpyAsync(y, r64_, n * k * 8, cudaMemcpyDeviceToHost, stream_), "d2h") &&
         check(cudaStreamSynchronize(stream_), "apply");
}

bool DeviceSystem::residual_host(const double* b, const double* x, int k, double* rel) {
  if (!err_.empty()) return false;
  cudaSetDevice(device_);
  if (!updated_) { err_ = "residual before update"; return false; }
  if (k < 1 || k > 64) { err_ = "k must be in [1, 64]"; return false; }
  if (!ensure_work(k)) return false;
  const size_t n = h_.levels[0].numTexels;
  if (!check(cudaMemcpyAsync(b64_, b, n * k * 8, cudaMemcpyHostToDevice, stream_), "h2d") ||
      !check(cudaMemcpyAsync(x64_, x, n * k * 8, cudaMemcpyHostToDevice, stream_), "h2d") ||
      !raw_apply_dev(rawA_, b64_, x64_, r64_, k, 0, stream_, sumsHost_))
    return false;
  for (int c = 0; c < k; c++) rel[c] = std::sqrt(sumsHost_[c] / std::max(sumsHost_[k + c], 1e-300));
  return true;
}

bool DeviceSystem::solve_filtering(const double* f_host, double* x_host, int k, double coefS, double tol, int maxIters,
                                   SolveReport& rep) {
  if (!err_.empty()) return false;
  cudaSetDevice(device_);
  if (!updated_) { err_ = "solve before update"; return false; }
  if (k < 1 || k > 64) { err_ = "k must be in [1, 64]"; return false; }
  if (!ensure_work(k)) return false;
  const size_t n = h_.levels[0].numTexels;
  if (filterK_ < workK_) {  // signal and S f work vectors, grown with the other work buffers
    filterArena_ = DeviceArena();
    fDev_ = static_cast<double*>(filterArena_.alloc(n * workK_ * sizeof(double)));
    sfDev_ = static_cast<double*>(filterArena_.alloc(n * workK_ * sizeof(double)));
    if (!check(filterArena_.last, "filtering buffers")) return false;
    filterK_ = workK_;
  }
  // b = M f (+ coefS S f) on the device from one upload of f
  if (!check(cudaMemcpyAsync(fDev_, f_host, n * k * sizeof(double), cudaMemcpyHostToDevice, stream_), "h2d f") ||
      !raw_apply_dev(rawM_, nullptr, fDev_, b64_, k, 1, stream_, nullptr))
    return false;
  kernelLaunches += 1;
  if (coefS != 0.0) {
    if (!raw_apply_dev(rawS_, nullptr, fDev_, sfDev_, k, 1, stream_, nullptr)) return false;
    dev::launch_axpby(b64_, 1.0, b64_, coefS, sfDev_, (long long)(n * k), stream_);
    kernelLaunches += 2;
  }
  return solve_mixed(nullptr, x_host, b64_, x64_, k, tol, maxIters, nullptr, rep, true);
}

bool DeviceSystem::vcycle_host64(double* x, const double* rhs, int k) {
  if (!err_.empty()) return false;
  cudaSetDevice(device_);
  if (!updated_) { err_ = "vcycle before update"; return false; }
  if (k < 1 || k > 64) { err_ = "k must be in [1, 64]"; return false; }
  const int KP = kp_for(k);
  if (!mg64_ || mg64_->KP < KP) {
    invalidate_graph();  // captured FP64 steps use the multigrid being replaced
    mg64_.reset(new Multigrid<double>());
    if (!build_multigrid(*mg64_, KP)) return false;
  }
  Multigrid<double>& mg = *mg64_;
  const size_t n = h_.levels[0].numTexels;
  std::vector<double> px(n * mg.KP, 0.0), pb(n * mg.KP, 0.0);
  for (size_t i = 0; i < n; i++)
    for (int c = 0; c < k; c++) { px[i * mg.KP + c] = x[i * k + c]; pb[i * mg.KP + c] = rhs[i * k + c]; }
  LevelDev<double>& D0 = mg.levels[0];
  if (!check(cudaMemcpyAsync(D0.x, px.data(), px.size() * 8, cudaMemcpyHostToDevice, stream_), "h2d") ||
      !check(cudaMemcpyAsync(D0.b, pb.data(), pb.size() * 8, cudaMemcpyHostToDevice, stream_), "h2d"))
    return false;
  if (mg.KP == 1) vcycle<double, 1>(mg, stream_); else vcycle<double, 4>(mg, stream_);
  queue_barrier_check(mg, stream_);
  if (!check(cudaGetLastError(), "vcycle") ||
      !check(cudaMemcpyAsync(px.data(), D0.x, px.size() * 8, cudaMemcpyDeviceToHost, stream_), "d2h") ||
      !check(cudaStreamSynchronize(stream_), "vcycle") || !barrier_ok(mg))
    return false;
  for (size_t i = 0; i < n; i++)
    for (int c = 0; c < k; c++) x[i * k + c] = px[i * mg.KP + c];
  return true;
}

bool DeviceSystem::relax_host(float* x, const float* rhs, int k, int sweeps, bool reverse) {
  if (!err_.empty()) return false;
  cudaSetDevice(device_);
  if (!updated_) { err_ = "relax before update"; return false; }
  if (k < 1 || k > 64 || sweeps < 0 || sweeps > 64) { err_ = "k must be in [1, 64] and sweeps in [0, 64]"; return false; }
  Multigrid<float>* mgp = mg32_for(kp_for(k));
  if (!mgp) return false;
  Multigrid<float>& mg = *mgp;
  const size_t n = h_.levels[0].numTexels;
  std::vector<float> px(n * mg.KP, 0.f), pb(n * mg.KP, 0.f);
  for (size_t i = 0; i < n; i++)
    for (int c = 0; c < k; c++) { px[i * mg.KP + c] = x[i * k + c]; pb[i * mg.KP + c] = rhs[i * k + c]; }
  LevelDev<float>& D0 = mg.levels[0];
  if (!check(cudaMemcpyAsync(D0.x, px.data(), px.size() * 4, cudaMemcpyHostToDevice, stream_), "h2d") ||
      !check(cudaMemcpyAsync(D0.b, pb.data(), pb.size() * 4, cudaMemcpyHostToDevice, stream_), "h2d"))
    return false;
  if (tiled(D0, mg.KP)) {
    if (sweeps > 0) tile_smooth(mg, D0, sweeps, reverse, false, stream_, false);
  } else {
    for (int sw = 0; sw < sweeps; sw++) {
      if (mg.KP % 4 == 0)
        colour_sweep<float, 4>(D0, mg.KP, reverse, false, sw > 0, stream_);
      else
        colour_sweep<float, 1>(D0, mg.KP, reverse, false, sw > 0, stream_);
    }
  }
  queue_barrier_check(mg, stream_);
  if (!check(cudaGetLastError(), "relax") ||
      !check(cudaMemcpyAsync(px.data(), D0.x, px.size() * 4, cudaMemcpyDeviceToHost, stream_), "d2h") ||
      !check(cudaStreamSynchronize(stream_), "relax") || !barrier_ok(mg))
    return false;
  for (size_t i = 0; i < n; i++)
    for (int c = 0; c < k; c++) x[i * k + c] = px[i * mg.KP + c];
  return true;
}

bool DeviceSystem::vcycle_host(float* x, const float* rhs, int k) {
  if (!err_.empty()) return false;
  cudaSetDevice(device_);
  if (!updated_) { err_ = "vcycle before update"; return false; }
  if (k < 1 || k > 64) { err_ = "k must be in [1, 64]"; return false; }
  Multigrid<float>* mgp = mg32_for(kp_for(k));
  if (!mgp) return false;
  Multigrid<float>& mg = *mgp;
  const size_t n = h_.levels[0].numTexels;
  std::vector<float> px(n * mg.KP, 0.f), pb(n * mg.KP, 0.f);
  for (size_t i = 0; i < n; i++)
    for (int c = 0; c < k; c++) { px[i * mg.KP + c] = x[i * k + c]; pb[i * mg.KP + c] = rhs[i * k + c]; }
  LevelDev<float>& D0 = mg.levels[0];
  if (!check(cudaMemcpyAsync(D0.x, px.data(), px.size() * 4, cudaMemcpyHostToDevice, stream_), "h2d") ||
      !check(cudaMemcpyAsync(D0.b, pb.data(), pb.size() * 4, cudaMemcpyHostToDevice, stream_), "h2d"))
    return false;
  if (mg.KP == 1) vcycle<float, 1>(mg, stream_); else vcycle<float, 4>(mg, stream_);
  queue_barrier_check(mg, stream_);
  if (!check(cudaGetLastError(), "vcycle") ||
      !check(cudaMemcpyAsync(px.data(), D0.x, px.size() * 4, cudaMemcpyDeviceToHost, stream_), "d2h") ||
      !check(cudaStreamSynchronize(stream_), "vcycle") || !barrier_ok(mg))
    return false;
  for (size_t i = 0; i < n; i++)
    for (int c = 0; c < k; c++) x[i * k + c] = px[i * mg.KP + c];
  return true;
}

bool DeviceSystem::solve_mixed(const double* b_host, double* x_host, const double* b_dev, double* x_dev, int k, double tol,
                               int maxIters, cudaStream_t userStream, SolveReport& rep, bool zeroGuess) {
  if (!err_.empty()) return false;
  cudaSetDevice(device_);
  if (!updated_) { err_ = "solve before update"; return false; }
  if (k < 1 || k > 64) { err_ = "k must be in [1, 64]"; return false; }
  Multigrid<float>* mgp = mg32_for(kp_for(k));
  if (!mgp || !ensure_work(k)) return false;
  Multigrid<float>& mg = *mgp;
  const size_t n = h_.levels[0].numTexels;
  cudaStream_t s = stream_;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  if (userStream) {
    cudaEventRecord(e0, userStream);
    cudaStreamWaitEvent(s, e0, 0);
  }
  cudaEventRecord(e0, s);
  const double* B = b_dev ? b_dev : b64_;
  double* X = x_dev ? x_dev : x64_;
  if (b_host && !check(cudaMemcpyAsync(b64_, b_host, n * k * 8, cudaMemcpyHostToDevice, s), "h2d b")) return false;
  if (x_host && !zeroGuess && !check(cudaMemcpyAsync(x64_, x_host, n * k * 8, cudaMemcpyHostToDevice, s), "h2d x")) return false;
  if (zeroGuess && !check(cudaMemsetAsync(X, 0, n * k * 8, s), "zero x")) return false;
  int it = 0;
  double rm = 0;
  if (knobs.krylov) {
    if (!krylov_solve(mg, B, X, k, tol, maxIters, s, rep, it, rm)) return false;
  } else {
    // refinement step graph: rhs <- r, e <- V(rhs), x += e, r <- b - A x (+ norms)
    cudaGraphExec_t iterGraph = find_graph(0, k, B, X);
    if (!iterGraph) {
      cudaGraph_t g;
      if (!prepare_timing(mg)) return false;
      profiling_ = true;
      if (!check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "capture")) return false;
      // D0.x (the correction) is zero on entry: cleared before the first step
      // and by the correction update of every step
      LevelDev<float>& D0 = mg.levels[0];
      if (mg.KP == 1) vcycle<float, 1>(mg, s, true); else vcycle<float, 4>(mg, s, true);
      dev::launch_add_correction<float>(X, D0.x, (long long)n, k, mg.KP, s, frozen_);
      // r = b - A x, written straight into the FP32 right-hand side of the next V-cycle
      dev::launch_raw_residual_f32(rawA_.runs, rawA_.nRuns, rawA_.coef, rawA_.planeStride, rawA_.bPtr, rawA_.bCol, rawA_.bVal,
                                   rawA_.bGlobal, rawA_.nB, B, X, D0.b, k, mg.KP, partials_, sums_, s);
      profiling_ = false;
      if (!check(cudaStreamEndCapture(s, &g), "capture end")) return false;
      StepGraph sg;
      sg.k = k;
      sg.b = B;
      sg.x = X;
      sg.kernels = kernel_nodes(g);
      if (!check(cudaGraphInstantiate(&sg.exec, g, 0), "graph instantiate")) { cudaGraphDestroy(g); return false; }
      cudaGraphDestroy(g);
      add_graph(sg);
      iterGraph = sg.exec;
    }
    // zero correction, initial residual straight into the FP32 right-hand side
    // (from a zero guess r = b: the operator is skipped, same bits)
    if (!check(cudaMemsetAsync(mg.levels[0].x, 0, n * mg.KP * sizeof(float), s), "zero correction")) return false;
    kernelLaunches += 2;  // operator + norm reduction
    dev::launch_raw_residual_f32(rawA_.runs, rawA_.nRuns, rawA_.coef, rawA_.planeStride, rawA_.bPtr, rawA_.bCol, rawA_.bVal,
                                 rawA_.bGlobal, rawA_.nB, B, X, mg.levels[0].b, k, mg.KP, partials_, sums_, s, zeroGuess);
    if (!read_norms(k, s, "initial residual")) return false;
    rep = SolveReport();
    rep.rel.assign(k, 0.0);
    auto rel_max = [&]() {
      double m = 0;
      for (int c = 0; c < k; c++) {
        rep.rel[c] = std::sqrt(sumsHost_[c] / std::max(sumsHost_[k + c], 1e-300));
        m = std::max(m, rep.rel[c]);
      }
      return m;
    };
    rm = rel_max();
    // right-hand sides at tolerance are frozen (their x no longer changes)
    auto update_frozen = [&]() {
      bool changed = false;
      for (int c = 0; c < k; c++) {
        const int f = rep.rel[c] <= tol ? 1 : 0;
        if (f != frozenHost_[c]) { frozenHost_[c] = f; changed = true; }
      }
      return !changed || upload_flags(k, s);
    };
    for (int c = 0; c < k; c++) frozenHost_[c] = 2;  // not a flag value: forces the first upload
    if (!update_frozen()) return false;
    while (rm > tol && it < maxIters) {
      kernelLaunches += graphKernels;
      if (!check(cudaGraphLaunch(iterGraph, s), "graph launch") || !read_norms(k, s, "refinement step")) return false;
      it++;
      rm = rel_max();
      if (rm > tol && !update_frozen()) return false;
      collect_timing(mg);
    }
  }
  if (x_host && !check(cudaMemcpyAsync(x_host, x64_, n * k * 8, cudaMemcpyDeviceToHost, s), "d2h x")) return false;
  queue_barrier_check(mg, s);
  cudaEventRecord(e1, s);
  if (userStream) cudaStreamWaitEvent(userStream, e1, 0);
  if (!check(cudaEventSynchronize(e1), "solve") || !barrier_ok(mg)) return false;
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  rep.iterations = it;
  rep.vcycles = it;
  rep.relMax = rm;
  rep.seconds = ms * 1e-3;
  return true;
}

// Problem i runs on slot i % 2.  Order of the work on the three streams:
//   copyIn:  b[i] -> slot            after problem i-2 (same slot) has finished
//   solve:   waits for b[i] and for the download of x[i-2] (same slot)
//   copyOut: slot -> x[i]            after problem i has finished
// so the upload of b[i+1] and the download of x[i-1] overlap solve i.  The
// solves are those of solve_mixed on device buffers, unchanged.
bool DeviceSystem::solve_stream(const double* const* b_host, double* const* x_host, int count, int k, double tol, int maxIters,
                                SolveReport* reps) {
  if (!err_.empty()) return false;
  cudaSetDevice(device_);
  if (!updated_) { err_ = "solve before update"; return false; }
  if (k < 1 || k > 64) { err_ = "k must be in [1, 64]"; return false; }
  if (count <= 0) return true;
  if (!copyIn_) {
    if (!check(cudaStreamCreateWithFlags(&copyIn_, cudaStreamNonBlocking), "copy stream") ||
        !check(cudaStreamCreateWithFlags(&copyOut_, cudaStreamNonBlocking), "copy stream"))
      return false;
    for (int j = 0; j < 2; j++)
      for (cudaEvent_t* e : {&slotIn_[j], &slotSolved_[j], &slotOut_[j]})
        if (!check(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "copy event")) return false;
  }
  const size_t n = h_.levels[0].numTexels, bytes = n * size_t(k) * sizeof(double);
  if (k > slotK_) {
    const int kc = k_capacity(k);
    slotArena_ = DeviceArena();
    slotK_ = 0;
    for (int j = 0; j < 2; j++) {
      slotB_[j] = static_cast<double*>(slotArena_.alloc(n * size_t(kc) * sizeof(double)));
      if (!slotB_[j]) return check(slotArena_.last, "slot buffers");
      slotX_[j] = static_cast<double*>(slotArena_.alloc(n * size_t(kc) * sizeof(double)));
      if (!slotX_[j]) return check(slotArena_.last, "slot buffers");
    }
    slotK_ = kc;
    invalidate_graph();  // graphs of freed slots must not match new ones at the same address
  }
  // every copy issued here has finished when this returns, on success or not
  auto drain = [&]() {
    cudaStreamSynchronize(copyIn_);
    cudaStreamSynchronize(copyOut_);
  };
  auto upload = [&](int i) {
    const int sl = i & 1;
    if (i >= 2 && !check(cudaStreamWaitEvent(copyIn_, slotSolved_[sl], 0), "copy order")) return false;
    return check(cudaMemcpyAsync(slotB_[sl], b_host[i], bytes, cudaMemcpyHostToDevice, copyIn_), "h2d b") &&
           check(cudaEventRecord(slotIn_[sl], copyIn_), "copy event");
  };
  for (int i = 0; i < std::min(count, 2); i++)
    if (!upload(i)) { drain(); return false; }
  for (int i = 0; i < count; i++) {
    const int sl = i & 1;
    bool ok = check(cudaStreamWaitEvent(stream_, slotIn_[sl], 0), "copy order") &&
              (i < 2 || check(cudaStreamWaitEvent(stream_, slotOut_[sl], 0), "copy order")) &&
              solve_mixed(nullptr, nullptr, slotB_[sl], slotX_[sl], k, tol, maxIters, nullptr, reps[i], true) &&
              check(cudaEventRecord(slotSolved_[sl], stream_), "copy event") &&
              check(cudaStreamWaitEvent(copyOut_, slotSolved_[sl], 0), "copy order") &&
              check(cudaMemcpyAsync(x_host[i], slotX_[sl], bytes, cudaMemcpyDeviceToHost, copyOut_), "d2h x") &&
              check(cudaEventRecord(slotOut_[sl], copyOut_), "copy event") && (i + 2 >= count || upload(i + 2));
    if (!ok) { drain(); return false; }
  }
  return check(cudaStreamSynchronize(copyOut_), "d2h x") && check(cudaStreamSynchronize(copyIn_), "h2d b");
}

// events for the level-0 sweep timing (and the per-level trace), created
// outside any capture
bool DeviceSystem::prepare_timing(const Multigrid<float>& mg) {
  if (!profEv_[0]) {
    for (cudaEvent_t& e : profEv_) cudaEventCreate(&e);
  }
  if (knobs.traceLevels && !timeline_) {
    timeline_ = static_cast<unsigned long long*>(rawArena_.alloc(1024 * sizeof(unsigned long long)));
    if (!check(rawArena_.last, "timeline") || !check(cudaMemset(timeline_, 0, 1024 * sizeof(unsigned long long)), "timeline"))
      return false;
  }
  if (knobs.traceLevels && traceEv_.size() != size_t(2 * mg.levels.size())) {
    for (cudaEvent_t e : traceEv_) cudaEventDestroy(e);
    traceEv_.assign(2 * mg.levels.size(), nullptr);
    for (cudaEvent_t& e : traceEv_) cudaEventCreate(&e);
  }
  return true;
}

int DeviceSystem::kernel_nodes(cudaGraph_t g) {
  size_t nn = 0;
  cudaGraphGetNodes(g, nullptr, &nn);
  std::vector<cudaGraphNode_t> nodes(nn);
  cudaGraphGetNodes(g, nodes.data(), &nn);
  int c = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    cudaGraphNodeGetType(nd, &t);
    if (t == cudaGraphNodeTypeKernel) c++;
  }
  return c;
}

// after a completed step: accumulate the events recorded inside its graph
void DeviceSystem::collect_timing(const Multigrid<float>& mg) {
  if (knobs.traceLevels && traceEv_.size() == size_t(2 * mg.levels.size())) {
    const int L = (int)mg.levels.size();
    std::vector<float> t(2 * L, 0.f);
    bool okT = true;
    for (int i = 1; i < 2 * L; i++) okT = okT && cudaEventElapsedTime(&t[i], traceEv_[i - 1], traceEv_[i]) == cudaSuccess;
    if (okT) {
      traceDownMs.resize(L - 1, 0.0);
      traceUpMs.resize(L - 1, 0.0);
      for (int l = 0; l + 1 < L; l++) traceDownMs[l] += t[l + 1];
      traceCoarseMs += t[L];
      for (int l = L - 2; l >= 0; l--) traceUpMs[l] += t[L + 1 + (L - 2 - l)];
      traceCount += 1;
    } else {
      cudaGetLastError();
    }
  }
  // average full level-0 sweep of this V-cycle (pre-smoothing and post-smoothing)
  float pre = 0, post = 0;
  const bool okPre = profSweeps_ > 0 && cudaEventElapsedTime(&pre, profEv_[0], profEv_[1]) == cudaSuccess;
  const bool okPost = profPostSweeps_ > 0 && cudaEventElapsedTime(&post, profEv_[2], profEv_[3]) == cudaSuccess;
  const int sweeps = (okPre ? profSweeps_ : 0) + (okPost ? profPostSweeps_ : 0);
  if (sweeps > 0) {
    profCount += 1;
    profMs += ((okPre ? pre : 0.f) + (okPost ? post : 0.f)) / sweeps;
    profTexels = mg.levels[0].nDeep;
  }
  cudaGetLastError();  // a missing timing leaves no error for the next caller
}

bool DeviceSystem::krylov_solve(Multigrid<float>& mg, const double* B, double* X, int k, double tol, int maxIters, cudaStream_t s,
                                SolveReport& rep, int& it, double& rm) {
  const size_t n = h_.levels[0].numTexels;
  if (k > krylovK_) {
    const int cap = k_capacity(k);
    krylovArena_ = DeviceArena();
    z_ = static_cast<double*>(krylovArena_.alloc(n * cap * sizeof(double)));
    p_ = static_cast<double*>(krylovArena_.alloc(n * cap * sizeof(double)));
    q_ = static_cast<double*>(krylovArena_.alloc(n * cap * sizeof(double)));
    sc_ = static_cast<double*>(krylovArena_.alloc(4 * size_t(cap) * sizeof(double)));
    if (!check(krylovArena_.last, "krylov vectors")) return false;
    krylovK_ = cap;
    invalidate_graph();  // the captured steps use the old vectors
  }
  LevelDev<float>& D0 = mg.levels[0];
  const int KP = mg.KP;
  rep = SolveReport();
  rep.rel.assign(k, 0.0);
  std::vector<double> bb(k, 0.0);
  auto rel_from = [&](bool setB) {
    double m = 0;
    for (int c = 0; c < k; c++) {
      if (setB) bb[c] = sumsHost_[k + c];
      rep.rel[c] = std::sqrt(sumsHost_[c] / std::max(bb[c], 1e-300));
      m = std::max(m, rep.rel[c]);
    }
    return m;
  };
  auto fetch = [&](const char* what) { return read_norms(k, s, what); };
  // r = b - A x with the FP64 operator
  auto true_residual = [&]() {
    kernelLaunches += 2;  // operator + norm reduction
    dev::launch_raw_operator(rawA_.runs, rawA_.nRuns, rawA_.coef, rawA_.planeStride, rawA_.bPtr, rawA_.bCol, rawA_.bVal, rawA_.bGlobal,
                             rawA_.nB, B, X, r64_, k, 0, partials_, sums_, s);
    return fetch("residual");
  };
  // (re)start: p = q = 0, rho_old = 0, the V-cycle's right-hand side = r, e = 0
  auto restart = [&]() {
    if (!check(cudaMemsetAsync(p_, 0, n * k * sizeof(double), s), "krylov restart") ||
        !check(cudaMemsetAsync(q_, 0, n * k * sizeof(double), s), "krylov restart") ||
        !check(cudaMemsetAsync(sc_, 0, 4 * size_t(k) * sizeof(double), s), "krylov restart"))
      return false;
    kernelLaunches += 1;
    dev::launch_pack_rhs<float>(r64_, D0.b, (long long)n, k, KP, s);
    return check(cudaMemsetAsync(D0.x, 0, n * KP * sizeof(float), s), "krylov restart");
  };
  auto update_frozen = [&]() {
    bool changed = false;
    for (int c = 0; c < k; c++) {
      const int f = rep.rel[c] <= tol ? 1 : 0;
      if (f != frozenHost_[c]) { frozenHost_[c] = f; changed = true; }
    }
    return !changed || upload_flags(k, s);
  };
  cudaGraphExec_t krylovGraph = find_graph(1, k, nullptr, X);
  if (!krylovGraph) {
    cudaGraph_t g;
    if (!prepare_timing(mg)) return false;
    profiling_ = true;
    if (!check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "capture")) return false;
    if (KP == 1) vcycle<float, 1>(mg, s, true); else vcycle<float, 4>(mg, s, true);
    profiling_ = false;
    dev::launch_fcg_precond((long long)n, k, KP, D0.x, r64_, q_, z_, partials_, sums_, sc_, s);
    dev::launch_fcg_direction((long long)n, k, z_, sc_, p_, s);
    dev::launch_raw_apply_dot(rawA_.runs, rawA_.nRuns, rawA_.coef, rawA_.planeStride, rawA_.bPtr, rawA_.bCol, rawA_.bVal, rawA_.bGlobal,
                              rawA_.nB, p_, q_, k, partials_, sums_, s);
    dev::launch_fcg_alpha(k, sums_, frozen_, sc_, s);
    dev::launch_fcg_update((long long)n, k, KP, sc_, p_, q_, X, r64_, D0.b, partials_, sums_, s);
    if (!check(cudaStreamEndCapture(s, &g), "capture end")) return false;
    StepGraph sg;
    sg.kind = 1;
    sg.k = k;
    sg.x = X;
    sg.kernels = kernel_nodes(g);
    if (!check(cudaGraphInstantiate(&sg.exec, g, 0), "graph instantiate")) { cudaGraphDestroy(g); return false; }
    cudaGraphDestroy(g);
    add_graph(sg);
    krylovGraph = sg.exec;
  }
  if (!true_residual()) return false;
  rm = rel_from(true);
  for (int c = 0; c < k; c++) frozenHost_[c] = 2;  // not a flag value: forces the first upload
  if (!update_frozen()) return false;
  it = 0;
  if (rm <= tol) return true;
  if (!restart()) return false;
  while (it < maxIters) {
    kernelLaunches += graphKernels;
    if (!check(cudaGraphLaunch(krylovGraph, s), "graph launch") || !fetch("krylov step")) return false;
    it++;
    collect_timing(mg);
    rm = rel_from(false);  // recursively updated residual
    if (rm <= tol) {
      if (!true_residual()) return false;  // confirm with b - A x
      rm = rel_from(false);
      if (rm <= tol) break;
      if (!update_frozen() || !restart()) return false;  // drift: restart from the true residual
      continue;
    }
    if (!update_frozen()) return false;
  }
  return true;
}

bool DeviceSystem::autotune(const double* b, int k, double tol, SolverKnobs& best, double& bestSeconds) {
  if (!err_.empty()) return false;
  cudaSetDevice(device_);
  const size_t n = h_.levels[0].numTexels;
  // b and x stay on the device: only the solve itself is timed
  DeviceArena tune;
  double* bDev = tune.upload(std::vector<double>(b, b + n * k));
  double* xDev = static_cast<double*>(tune.alloc(n * k * sizeof(double)));
  if (!check(tune.last, "autotune buffers")) return false;
  const SolverKnobs base = knobs;
  bestSeconds = 1e300;
  best = base;
  // candidates: deep sweeps before / after the coarse correction on the finer
  // levels, and on the levels from `coarseFrom` on (-1: same as the finer
  // ones); the exact boundary solve follows the coarse correction; the outer
  // iteration is plain refinement or flexible CG
  const int fine[][2] = {{1, 1}, {2, 2}, {2, 3}, {3, 3}, {3, 4}, {4, 4}};
  const int coarse[][3] = {{-1, -1, 2}, {0, 1, 2}, {0, 2, 2}, {0, 3, 2}, {1, 1, 2}, {1, 2, 2},
                           {0, 2, 1}, {0, 3, 1}, {1, 2, 1}, {0, 2, 3}};
  for (int kr = 0; kr < 2; kr++)
  for (const auto& f : fine)
    for (const auto& c : coarse) {
      knobs = base;
      knobs.krylov = kr;
      knobs.preSweeps = f[0];
      knobs.postSweeps = f[1];
      knobs.preBoundary = 0;
      knobs.postBoundary = 1;
      knobs.coarsePreSweeps = c[0];
      knobs.coarsePostSweeps = c[1];
      knobs.coarseFrom = c[2];
      invalidate_graph();
      double t = 1e300;
      for (int rep = 0; rep < 3; rep++) {  // the first run captures the graph
        SolveReport r;
        if (!solve_mixed(nullptr, nullptr, bDev, xDev, k, tol, 60, nullptr, r, true)) return false;
        if (r.relMax > tol) { t = 1e300; break; }
        if (rep > 0) t = std::min(t, r.seconds);
      }
      if (t < bestSeconds) { bestSeconds = t; best = knobs; }
    }
  knobs = best;
  invalidate_graph();
  return true;
}

bool DeviceSystem::solve_fp64(const double* b_host, double* x_host, const double* b_dev, double* x_dev, int k, double tol,
                              int maxIters, cudaStream_t userStream, SolveReport& rep) {
  if (!err_.empty()) return false;
  cudaSetDevice(device_);
  if (!updated_) { err_ = "solve before update"; return false; }
  if (k < 1 || k > 64) { err_ = "k must be in [1, 64]"; return false; }
  const int KP = kp_for(k);
  if (!mg64_ || mg64_->KP < KP) {
    invalidate_graph();  // captured FP64 steps use the multigrid being replaced
    mg64_.reset(new Multigrid<double>());
    if (!build_multigrid(*mg64_, KP)) return false;
  }
  if (!ensure_work(k)) return false;
  Multigrid<double>& mg = *mg64_;
  const size_t n = h_.levels[0].numTexels;
  cudaStream_t s = stream_;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  if (userStream) {
    cudaEventRecord(e0, userStream);
    cudaStreamWaitEvent(s, e0, 0);
  }
  cudaEventRecord(e0, s);
  // caller's device buffers (x holds the initial guess), or the work vectors
  // filled from the host
  const double* B = b_dev ? b_dev : b64_;
  double* X = x_dev ? x_dev : x64_;
  if (b_host && !check(cudaMemcpyAsync(b64_, b_host, n * k * 8, cudaMemcpyHostToDevice, s), "h2d b")) return false;
  if (x_host && !check(cudaMemcpyAsync(x64_, x_host, n * k * 8, cudaMemcpyHostToDevice, s), "h2d x")) return false;
  kernelLaunches += 2;  // operator + norm reduction
  if (!raw_apply_dev(rawA_, B, X, r64_, k, 0, s, nullptr) || !read_norms(k, s, "initial residual")) return false;
  rep = SolveReport();
  rep.rel.assign(k, 0.0);
  auto rel_max = [&]() {
    double m = 0;
    for (int c = 0; c < k; c++) {
      rep.rel[c] = std::sqrt(sumsHost_[c] / std::max(sumsHost_[k + c], 1e-300));
      m = std::max(m, rep.rel[c]);
    }
    return m;
  };
  double rm = rel_max();
  int it = 0;
  LevelDev<double>& D0 = mg.levels[0];
  // one refinement step (rhs <- r, V-cycle, x += e, r <- b - A x and norms)
  // as a captured graph, like the mixed-precision path
  cudaGraphExec_t step = find_graph(2, k, B, X);
  if (!step) {
    cudaGraph_t g;
    if (!check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "capture")) return false;
    dev::launch_pack_rhs<double>(r64_, D0.b, (long long)n, k, mg.KP, s);
    cudaMemsetAsync(D0.x, 0, n * mg.KP * sizeof(double), s);
    if (mg.KP == 1) vcycle<double, 1>(mg, s, true); else vcycle<double, 4>(mg, s, true);
    dev::launch_add_correction<double>(X, D0.x, (long long)n, k, mg.KP, s);
    raw_apply_dev(rawA_, B, X, r64_, k, 0, s, nullptr);
    if (!check(cudaStreamEndCapture(s, &g), "capture end")) return false;
    StepGraph sg;
    sg.kind = 2;
    sg.k = k;
    sg.b = B;
    sg.x = X;
    sg.kernels = kernel_nodes(g);
    if (!check(cudaGraphInstantiate(&sg.exec, g, 0), "graph instantiate")) { cudaGraphDestroy(g); return false; }
    cudaGraphDestroy(g);
    add_graph(sg);
    step = sg.exec;
  }
  while (rm > tol && it < maxIters) {
    kernelLaunches += graphKernels;
    if (!check(cudaGraphLaunch(step, s), "graph launch") || !read_norms(k, s, "refinement step")) return false;
    it++;
    rm = rel_max();
  }
  if (x_host && !check(cudaMemcpyAsync(x_host, x64_, n * k * 8, cudaMemcpyDeviceToHost, s), "d2h x")) return false;
  queue_barrier_check(mg, s);
  cudaEventRecord(e1, s);
  if (userStream) cudaStreamWaitEvent(userStream, e1, 0);
  if (!check(cudaEventSynchronize(e1), "solve") || !barrier_ok(mg)) return false;
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  rep.iterations = it;
  rep.vcycles = it;
  rep.relMax = rm;
  rep.seconds = ms * 1e-3;
  return true;
}

}  // namespace gdtp
