// Host-callable launchers of the V-cycle kernels (vcycle_kernels.cu).
#pragma once
#include <atomic>
#include <cstdint>
#include <string>
#include <vector>
#include <cuda_runtime.h>

namespace gdtp {
namespace dev {

constexpr int kMaxDevices = 64;
constexpr int kUnset = -2;


struct ColourRun;
struct RowLine;
struct RestrictRun;
struct ProlongRun;

// Longest j chunk of a boundary dense product (its input vector is staged in
// shared memory): subdomains hold at most this many rows, and the separator
// product is split into at least ceil(nS / kBoundaryChunkMax) chunks.
constexpr int kBoundaryChunkMax = 384;

// Device view of one level's exact boundary solver (setup/bsolve.cpp).  Solver
// positions: interior rows of the subdomains first (subdomain by subdomain),
// then the separator.  Dense inverses are symmetric, stored row-major with rows
// padded to a multiple of 4 entries; a task {matrix, first row quad, -, -} is
// one 128-row group, launched as `chunks` blocks over the j range.
template <typename T>
struct BoundaryDev {
  int nb = 0, nSub = 0, nI = 0, nS = 0;
  const int* subPtr = nullptr;          // subdomain row ranges (positions)
  const int* rowSub = nullptr;          // interior position -> subdomain
  const long long* invOff = nullptr;
  const T* inv = nullptr;
  const int4* subTasks = nullptr;
  int nSubTasks = 0, subChunks = 1;
  const T* sinv = nullptr;              // separator Schur complement inverse (nS x nSp)
  const int4* schurTasks = nullptr;
  int nSchurTasks = 0, schurChunks = 1;
  const int* posGlobal = nullptr;       // position -> global texel
  const T* scale = nullptr;
  const int *bdPtr = nullptr, *bdCol = nullptr;
  const T* bdVal = nullptr;
  const int *asiPtr = nullptr, *asiCol = nullptr;  // separator x interior coupling (scaled)
  const T* asiVal = nullptr;
  const int *touchPtr = nullptr, *touch = nullptr; // per subdomain: separator columns
  const long long* wOff = nullptr;
  const T* wt = nullptr;                // Inv_p A_{I_p,touch}, column-major m x t_p
  T *y = nullptr, *xs = nullptr, *subPart = nullptr, *schurPart = nullptr;  // work
  T* rhat = nullptr;                    // scaled right-hand side s (rhs - BD x) per position (work)
  int *subCount = nullptr, *schurCount = nullptr;                            // chunk arrival counters (zero between launches)
};

// One multigrid level on the device, value type T (plain pointers and counts;
// also read by the cluster kernel from a device-side array).
template <typename T>
struct LevelDev {
  int n = 0, nDeep = 0, nB = 0;
  const ColourRun* runs = nullptr;
  int nRuns = 0, runStart[5] = {0, 0, 0, 0, 0};
  const T* coef = nullptr;      // 10 planes, reciprocal form
  int planeStride = 0;
  const int *bPtr = nullptr, *bCol = nullptr, *bGlobal = nullptr;
  const T* bVal = nullptr;      // boundary rows: BD + BB with global columns
  BoundaryDev<T> B;
  const RestrictRun* rruns = nullptr;  // to the next level
  int nRRuns = 0;
  const int *rbPtr = nullptr, *rbCol = nullptr, *rbOut = nullptr;
  const T* rbVal = nullptr;
  int nRB = 0;
  const ProlongRun* pruns = nullptr;   // from the next level
  int nPRuns = 0;
  T *x = nullptr, *b = nullptr, *r = nullptr;
  const int* groups = nullptr;  // per chart: first run of each colour [4], run counts [4], texel span [2]
  int nGroups = 0, maxGroupDeep = 0, maxGroupSpan = 0;
  int maxGroupColourRuns = 0;   // most runs of one colour in one chart
  // fused tile smoother (launch_tile_smooth): tiles ordered by tile colour
  // (tiles of colour c are [tileStart[c], tileStart[c + 1])), segments, FP32
  // coefficient blocks
  const int4* tiles = nullptr;
  int nTiles = 0, tileStart[5] = {0, 0, 0, 0, 0};
  const int4* tileSegs = nullptr;
  const int* tileNbrs = nullptr;
  const float* tileCoef = nullptr;
  int* tileSync = nullptr;      // per multigrid (its rounds run in its stream order)
  // row smoother (launch_gs_rows): the raster lines of even [0] and odd [1]
  // rows packed into blocks of rowBlock threads; rowLineOf[block * rowBlock +
  // thread] = its line (-1: idle)
  const RowLine* rowLines[2] = {nullptr, nullptr};
  const int* rowLineOf[2] = {nullptr, nullptr};
  int nRowBins[2] = {0, 0};
  int rowBlock = 0, rowSlots = 0;
};

template <typename T, int W>
// skip: bit k set = neighbour slot k (3 (dy + 1) + dx + 1) is known to be zero;
// rhsEarly: the previous launch in the stream does not write rhs (a colour pass
// of the same smoothing step), so rhs is read before waiting for it
void launch_gs_colour(const ColourRun* runs, int nRuns, const T* coef, int planeStride, const T* rhs, T* x, int KP, cudaStream_t s,
                      int skip = 0, bool rhsEarly = false);
// Two colour passes of one row parity in one launch (rows: 0 even rows, colours
// 0 then 1 or, with oddFirst, 1 then 0; 1 odd rows, colours 2 / 3): a block
// per group of whole raster lines, which stages the line's row and the rows
// above and below in shared memory, updates the first colour, then the second
// from the first's new values.  A row's update reads only the other parity's
// rows and its own, so the lines are independent and the result is that of
// the two launch_gs_colour passes, bit for bit.  skip: bit 0 / 1 = the first
// colour's row (above and below) / own-row neighbours are known zeros, bits 2
// / 3 the same for the second colour.
constexpr int kRowBlockMax = 1024;
// shared-memory slots per row-smoother block of bs threads (a line of len
// texels takes len + 2; bs threads hold lines of at most 2 bs texels)
constexpr int row_slot_cap(int bs) { return 2 * bs + 64; }
// false: nothing launched (the level has no row blocks, or their shared memory
// does not fit this device); gs_rows_available tells before any launch
template <typename T, int W>
bool launch_gs_rows(const LevelDev<T>& D, int rows, bool oddFirst, int KP, cudaStream_t s, int skip = 0, bool rhsEarly = false);
template <typename T, int W>
bool gs_rows_available(const LevelDev<T>& D);
template <typename T, int W>
size_t gs_rows_smem(const LevelDev<T>& D);
// `sweeps` 4-colour Gauss-Seidel sweeps (colours 0..3, or 3..0 when reverse)
// in one launch, one block per chart group with the chart's x in shared memory:
// the same updates in the same order as launch_gs_colour per colour.  False
// (nothing launched) when a chart's span does not fit kGroupSmemMax.
constexpr size_t kGroupSmemMax = 200 * 1024;
// rhsEarly: the previous launch does not write the level's right-hand side
template <typename T, int W>
bool launch_gs_groups(const LevelDev<T>& D, int sweeps, bool reverse, int KP, cudaStream_t s, bool rhsEarly = false);
// Fused smoothing round (tile_smoother.cu): tiles of kTileW x kTileH texels of
// one chart, a CTA each, `sweeps` 4-colour sweeps in shared memory, x updated
// in place.  Tiles are ordered by tile colour (tile column parity | tile row
// parity << 1): colour c is [tileStart[c], tileStart[c + 1]).  A tile starts
// once its neighbours of earlier colours (colours 0..3, or 3..0 in reverse)
// are done.  tiles[t] = {first coefficient of the tile, first segment, segment
// count (<= kTileMaxSegs), element count}; coefficients: 10 planes of
// kTileSlots per tile, slot = colour * kTileSlots / 4 + (j / 2) * kTileW / 2 +
// i / 2 for tile-local (i, j) of colour (i & 1) | (j & 1) << 1, zeros where
// the texel is not deep; segs[s] = {global texel of the first element, row r |
// first column u0 << 6 | length << 12, first element of the segment in the
// tile, 0}: runs of consecutive global texels on one row of the tile with its
// one-texel ring (r, u0 in 0 .. size + 1), in row order; nbrs: 8 neighbour
// tiles per tile (-1: none); sync: 2 + nTiles ints, zero (the kernel leaves
// them zero); err: set to 2 when a wait for a neighbour timed out.
// zeroStart: x = 0 on entry.  KP = 1 or 4; false if not launched.
constexpr int kTileW = 32, kTileH = 32, kTileSlots = kTileW * kTileH;
constexpr int kTileMaxSegs = (kTileH + 2) * (kTileW / 2 + 1);  // every other ring texel active
struct TileRound {
  const int4* tiles;
  const int4* segs;
  const int* nbrs;
  const float* coef;
  const float* rhs;
  int* sync;
  unsigned int* err;
  int nTiles, tileStart[5];
  int sweeps, reverse, zeroStart;
};
bool launch_tile_smooth(const TileRound& round, float* x, int KP, cudaStream_t s);
template <typename T, int W>
// rhsEarly: the previous launch in the stream does not write rhs (it only wrote
// x: smoothing or a boundary solve), so rhs is read before waiting for it
void launch_residual(const ColourRun* runs, int nRuns, const T* coef, int planeStride, const int* bPtr, const int* bCol,
                     const T* bVal, const int* bGlobal, int nB, const T* rhs, const T* x, T* res, int KP, cudaStream_t s,
                     bool rhsEarly = false);
// also clears the coarse iterate coarseX (coarseTexels x KP values)
template <typename T, int W>
void launch_restrict(const RestrictRun* runs, int nRuns, const int* rPtr, const int* rCol, const T* rVal, const int* rOut,
                     int nB, const T* res, T* coarseRhs, T* coarseX, long long coarseTexels, int KP, cudaStream_t s);
template <typename T, int W>
void launch_prolong_add(const ProlongRun* runs, int nRuns, const T* coarse, T* fine, int KP, cudaStream_t s);
template <typename T, int W>
// rhsEarly: the previous launch in the stream does not write rhs (the
// prolongation before the solve after the coarse correction)
void launch_boundary_solve(const BoundaryDev<T>& B, const T* rhs, T* x, int KP, cudaStream_t s, bool rhsEarly = false);
template <typename T, int W>
void launch_coarse_solve(int n, const double* ainv, const double* scale, const T* rhs, T* x, int KP, cudaStream_t s);

void launch_raw_operator(const ColourRun* runs, int nRuns, const double* coef, int planeStride, const int* bPtr, const int* bCol,
                         const double* bVal, const int* bGlobal, int nB, const double* b, const double* x, double* out, int K,
                         int mode, double* partials, double* sums, cudaStream_t s);
// Blocks of the FP64 operator's fixed grid on the current device (8 per SM, at
// most kRawMaxBlocks): the partial-sum buffers hold this many blocks x 2K.
constexpr int kRawMaxBlocks = 2048;
int raw_operator_blocks(int nRuns, int nB, int K);
// r = b - A x written as the padded FP32 right-hand side (n x KP), plus norms;
// xZero: x is known to be zero, r = b without reading x or the operator (the
// same bits and norms)
void launch_raw_residual_f32(const ColourRun* runs, int nRuns, const double* coef, int planeStride, const int* bPtr,
                             const int* bCol, const double* bVal, const int* bGlobal, int nB, const double* b, const double* x,
                             float* rhs32, int K, int KP, double* partials, double* sums, cudaStream_t s, bool xZero = false);
template <typename T>
void launch_pack_rhs(const double* r, T* rhs, long long n, int K, int KP, cudaStream_t s);
// n doubles (n <= a few hundred) by one block, e.g. into mapped pinned host memory
void launch_copy_f64(double* dst, const double* src, int n, cudaStream_t s);
// flags[c] = bit c of mask, c < k <= 64
void launch_set_flags(int* flags, unsigned long long mask, int k, cudaStream_t s);
// Flexible preconditioned CG around the FP32 V-cycle (vcycle_kernels.cu).  sc: 4K
// per-RHS scalars {alpha, beta, rho, rho_old}; sums: 2K.
//   precond:   z = e (e cleared), rho = z.r, beta = -alpha_old (z.q_old) / rho_old
//   direction: p = z + beta p
//   apply_dot: q = A p, sums[0..K) = p.q
//   alpha:     alpha = rho / p.q (0 where frozen)
//   update:    x += alpha p, r -= alpha q, rhs32 = r, sums[0..K) = r.r
void launch_fcg_precond(long long n, int K, int KP, float* e, const double* r, const double* q, double* z, double* partials,
                        double* sums, double* sc, cudaStream_t s);
void launch_fcg_direction(long long n, int K, const double* z, const double* sc, double* p, cudaStream_t s);
void launch_raw_apply_dot(const ColourRun* runs, int nRuns, const double* coef, int planeStride, const int* bPtr, const int* bCol,
                          const double* bVal, const int* bGlobal, int nB, const double* x, double* out, int K, double* partials,
                          double* sums, cudaStream_t s);
void launch_fcg_alpha(int K, const double* sums, const int* frozen, double* sc, cudaStream_t s);
void launch_fcg_update(long long n, int K, int KP, const double* sc, const double* p, const double* q, double* x, double* r, float* rhs32,
                       double* partials, double* sums, cudaStream_t s);
// out = a x + b y over n doubles
void launch_axpby(double* out, double a, const double* x, double b, const double* y, long long n, cudaStream_t s);
// x += e (columns c with frozen[c] != 0 unchanged; frozen may be null), then e = 0
template <typename T>
void launch_add_correction(double* x, T* e, long long n, int K, int KP, cudaStream_t s, const int* frozen = nullptr);
// Sweeps per level inside the coarse-level kernel (the host's pre_sweeps /
// post_sweeps rule: levels >= coarseFrom use the coarse counts when >= 0).
struct CoarseSweeps {
  int finePre, finePost, coarsePre, coarsePost, coarseFrom;
  int preBoundary, postBoundary;
  __host__ __device__ int pre(int l) const { return (l >= coarseFrom && coarsePre >= 0) ? coarsePre : finePre; }
  __host__ __device__ int post(int l) const { return (l >= coarseFrom && coarsePost >= 0) ? coarsePost : finePost; }
};
// State of the persistent kernel's grid barrier (device memory, zeroed once;
// error != 0 after a barrier timed out: zero it again before the next launch)
struct GridBarrierState {
  unsigned int count, gen, error, pad;
};
// Coarse levels l0 .. L-1 in one kernel (coarse_cycle.cu): one thread-block
// cluster (barrier == nullptr) or every SM of the device in a cooperative launch
// with grid barriers (barrier: its state).
// leg 0: down leg of levels l0..L-2 (pre-smoothing, residual, restriction);
// leg 1: up leg (prolongation, boundary solve, post-smoothing); leg 2: both with
// the coarsest dense solve in between.  lvDev: device array of all levels.
// timeline (optional, 1024 entries): {phase code, globaltimer ns} pairs after each
// phase, start time in [1022].  Returns false when the launch is not possible.
template <typename T, int W>
bool launch_coarse_cycle(const LevelDev<T>* lvDev, int l0, int L, int leg, const CoarseSweeps& sw, int KP, int coarseN,
                         const double* coarseInv, const double* coarseScale, unsigned long long* timeline,
                         GridBarrierState* barrier, cudaStream_t s);
// CTAs of the coarse-level cluster on this device (0: clusters unavailable)
int coarse_cycle_cluster_ctas(bool fp64, int W);
// CTAs of the persistent whole-GPU variant (0: cooperative launch unavailable)
int coarse_cycle_grid_ctas(bool fp64, int W);
// largest coarsest level the coarse kernels solve inside (leg 2)
constexpr int kCoarseInKernelMax(bool grid) { return grid ? 4096 : 1024; }
// Per-device cache of a value a kernel's launch set-up computes once (an
// attribute set, an occupancy figure): `compute` runs once per device, calls
// from several threads are safe (the server's workers launch concurrently).
template <typename F>
int per_device_once(std::atomic<int> (&slots)[kMaxDevices], F compute) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return compute();
  int v = slots[dev].load(std::memory_order_acquire);
  if (v == kUnset) {
    v = compute();  // a racing thread computes the same value
    slots[dev].store(v, std::memory_order_release);
  }
  return v;
}
// Programmatic dependent launch of the V-cycle kernels (process-wide, default on)
void set_programmatic_launch(bool on);
bool programmatic_launch();

// assembly (assembly_kernels.cu)
void launch_interior_cells(int n, const int* cellPtr, const int* cellTri, const int* cellIJ, const int* cellChart,
                           const double* chartCellSize, const double* triPos, const double* triMetricInv, const double* triScale,
                           double* mass, double* stiff, cudaStream_t s);
void launch_deep_gather(int nDeep, const int* deepCells, const double* cellMass, const double* cellStiff, double* deepMass,
                        double* deepStiff, cudaStream_t s);
void launch_boundary_triangles(int n, const int* btPtr, const int* btTri, const double* btPos, const double* triPos,
                               const double* triMetric, const double* triMetricInv, double* mass, double* stiff, cudaStream_t s);
void launch_gather_cells(int n, const int* idx, const double* src, double* dst, cudaStream_t s);

// Dense FP64 set-up products (kernels/dense_kernels.cu).
// One task of a batched C = alpha op(A) B + beta C (row-major, offsets in
// doubles into the A, B and C buffers of the launch; op(A) = A (M x K) or,
// transA, the transpose of A stored K x M).
struct GemmTask {
  long long a, b, c;
  int M, N, K, lda, ldb, ldc, transA, pad;
  double alpha, beta;
};
void launch_gemm_batch(const GemmTask* dTasks, int nTasks, int maxM, int maxN, const double* A, const double* B, double* C,
                       cudaStream_t s);
// Batched inverse of SPD blocks by blocked Gauss-Jordan elimination: the
// layout (host) of blocks q at offsets[q], sizes[q] x sizes[q] row-major, and
// its device arrays (uploaded by the caller from the layout's vectors).
struct SpdInverseLayout {
  int nMat = 0, steps = 0;
  long long total = 0, elems = 0, wsTotal = 0;
  std::vector<int64_t> offsets, first, ws;
  std::vector<int> sizes, taskStart, stepMax;
  std::vector<GemmTask> tasks;
};
struct SpdInverseDevice {
  const long long* off;
  const int* size;
  const long long* first;
  const long long* ws;
  const GemmTask* tasks;
};
bool spd_inverse_layout(const std::vector<int64_t>& offsets, const std::vector<int>& sizes, SpdInverseLayout& L, std::string& err);
// scratch doubles one launch_spd_inverse needs
size_t spd_inverse_scratch_doubles(const SpdInverseLayout& L);
// A (elems doubles, destroyed) -> out = the exactly symmetric inverses at the
// same offsets; *bad set to 1 on a non-positive pivot (caller zeroes it)
bool launch_spd_inverse(const SpdInverseLayout& L, const SpdInverseDevice& D, double* A, double* out, double* scratch, int* bad,
                        cudaStream_t s);
// per block p: G_p = Inv_p C_p (m x t at cOff[p]) and local_p = C_p^T G_p (t x t at localOff[p])
void schur_product_tasks(const std::vector<int64_t>& invOff, const std::vector<int>& m, const std::vector<int64_t>& cOff,
                         const std::vector<int>& t, const std::vector<int64_t>& localOff, std::vector<GemmTask>& gTasks,
                         std::vector<GemmTask>& lTasks, int& maxM, int& maxT);
// Host-vector forms, synchronous on s: in-place inverses of SPD matrices data[off[q] ..] (size[q] x size[q],
// row-major) by Gauss-Jordan elimination, made exactly symmetric.
bool gpu_spd_inverse_batched(double* data, const std::vector<int64_t>& offsets, const std::vector<int>& sizes, cudaStream_t s,
                             std::string& err);
// Per block p: G_p = Inv_p C_p (m_p x t_p) and local_p = C_p^T G_p (t_p x t_p).
bool gpu_schur_products(const std::vector<double>& inv, const std::vector<int64_t>& invOff, const std::vector<int>& m,
                        const std::vector<double>& C, const std::vector<int64_t>& cOff, const std::vector<int>& t, std::vector<double>& G,
                        std::vector<double>& local, const std::vector<int64_t>& localOff, cudaStream_t s, std::string& err);

}  // namespace dev
}  // namespace gdtp
