// Fused smoothing step on large levels: every Gauss-Seidel sweep of one
// smoothing step inside a tile of a chart's texel grid, one CTA per tile.
//
// A tile is kTileW x kTileH texels of one chart (chart-local origin at
// multiples of the tile size, so tile parity is chart parity).  The CTA stages
// the tile's x with a one-texel ring in shared memory, its right-hand side and
// its 10 reciprocal-form coefficient planes per texel (registers), runs all
// `sweeps` 4-colour sweeps there (the colour order of the colour-run path,
// IterativeSolvers.inl:449-463 arithmetic per texel), and writes the tile's
// deep texels back in place.  Coefficients, rhs and x then cross HBM once per
// smoothing step instead of once per sweep.
//
// Tiles carry a tile colour (tile column parity | tile row parity << 1).
// Tiles of one colour never touch each other (not even at corners).  A
// smoothing round visits the colours in turn (3..0 in reverse): a tile starts
// once every neighbour of an earlier colour has finished, so its ring holds the
// newest values of those tiles and the starting values of the tiles that come
// after it (they wait for this one).  That is a Gauss-Seidel sweep over tiles
// with Gauss-Seidel sweeps inside each tile, and the result does not depend on
// the order the CTAs run in.  One persistent launch runs a whole round: CTAs
// take tiles from a counter in colour order, so every tile a CTA waits for has
// already been taken by a running CTA and every wait ends; waits are bounded
// anyway (a timeout sets an error word the host reads).
//
// Shared memory keeps each colour's texels in their own sub-grid
// (kTileW/2 + 2) x (kTileH/2 + 2), so the 16 texels of one colour on a tile row
// are 16 consecutive vectors: a warp's neighbour reads are conflict-free.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>

#include "vcycle.cuh"
#include "vcycle_kernels.h"

namespace gdtp {
namespace dev {

namespace {

constexpr int kSubW = kTileW / 2 + 2, kSubH = kTileH / 2 + 2, kSub = kSubW * kSubH;  // one colour with its ring
constexpr int kPerColour = kTileSlots / 4;                                        // 256 = threads per CTA
constexpr int kHalfW = kTileW / 2;

// floor(v / 2) for v in [-1, 3]
__host__ __device__ constexpr int half_floor(int v) { return (v + 2) / 2 - 1; }

template <int KP>
struct TileVec;
template <>
struct TileVec<1> {
  float v[1];
};
template <>
struct __align__(16) TileVec<4> {
  float v[4];
};

template <int KP>
__device__ __forceinline__ TileVec<KP> tload(const float* p) {
  return *reinterpret_cast<const TileVec<KP>*>(p);
}
template <int KP>
__device__ __forceinline__ void tstore(float* p, const TileVec<KP>& v) {
  *reinterpret_cast<TileVec<KP>*>(p) = v;
}

// Gauss-Seidel update of this thread's texel of colour CC (tile-local
// i = 2p + (CC & 1), j = 2q + (CC >> 1)): x = b c4 - sum_{k != 4} c_k x_k, the
// eight neighbour reads issued first and the sum in two chains (rows above and
// below the texel, then its row) so that shared-memory latency overlaps.
template <int KP, int CC>
__device__ __forceinline__ void relax_colour(float* xs, const float* bs, const float (&c)[10], int p, int q) {
  if (c[9] == 0.f) return;  // not a deep texel (its coefficients are zero)
  constexpr int bi = CC & 1, bj = CC >> 1;
  TileVec<KP> v[9];
#pragma unroll
  for (int k = 0; k < 9; k++) {
    if (k == 4) continue;
    const int di = k % 3 - 1, dj = k / 3 - 1;  // stencil slot k = 3 (dj + 1) + di + 1
    const int sub = ((bi + di) & 1) | (((bj + dj) & 1) << 1);
    const int su = p + 1 + half_floor(bi + di), sv = q + 1 + half_floor(bj + dj);
    v[k] = tload<KP>(xs + (sub * kSub + sv * kSubW + su) * KP);
  }
  const TileVec<KP> b = tload<KP>(bs + (CC * kPerColour + q * kHalfW + p) * KP);
  TileVec<KP> out;
#pragma unroll
  for (int ch = 0; ch < KP; ch++) {
    const float lo = c[0] * v[0].v[ch] + c[1] * v[1].v[ch] + c[2] * v[2].v[ch];
    const float hi = c[6] * v[6].v[ch] + c[7] * v[7].v[ch] + c[8] * v[8].v[ch];
    const float mid = c[3] * v[3].v[ch] + c[5] * v[5].v[ch];
    out.v[ch] = b.v[ch] * c[4] - ((lo + hi) + mid);
  }
  tstore<KP>(xs + (CC * kSub + (q + 1) * kSubW + (p + 1)) * KP, out);
}

template <int KP, int CC>
__device__ __forceinline__ void pass(float* xs, const float* bs, const float (&c)[4][10], int p, int q) {
  relax_colour<KP, CC>(xs, bs, c[CC], p, q);
  __syncthreads();
}

// global -> shared copies that bypass registers (completion: cp_async_wait_all)
template <int KP>
__device__ __forceinline__ void cp_async(float* smem, const float* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  if constexpr (KP == 4)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// ring-and-tile elements per thread (a tile with its ring has at most
// (kTileW + 2) x (kTileH + 2) active texels)
constexpr int kElemsPerThread = ((kTileW + 2) * (kTileH + 2) + kPerColour - 1) / kPerColour;

// Polls of a neighbour tile's done flag before the wait gives up (about a
// second); a tile takes microseconds.
constexpr long long kTilePolls = 1ll << 20;

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <int KP>
__device__ __forceinline__ TileVec<KP> tload_l2(const float* p);
template <>
__device__ __forceinline__ TileVec<1> tload_l2<1>(const float* p) {
  TileVec<1> r;
  r.v[0] = __ldcg(p);
  return r;
}
template <>
__device__ __forceinline__ TileVec<4> tload_l2<4>(const float* p) {
  const float4 v = __ldcg(reinterpret_cast<const float4*>(p));
  TileVec<4> r;
  r.v[0] = v.x; r.v[1] = v.y; r.v[2] = v.z; r.v[3] = v.w;
  return r;
}

// Position in colour order (the order of the round) of a tile colour.
__device__ __forceinline__ int colour_rank(int colour, int reverse) { return reverse ? 3 - colour : colour; }

// One smoothing round over all tiles of a level.  sync: {tile counter, exit
// counter, done flag per tile}, zero on entry and left zero by the last CTA to
// exit; err: set to 2 when a wait timed out.  x is read (ring and tile) and
// written (the tile's deep texels) in place.
template <int KP>
__global__ void __launch_bounds__(kPerColour, 3) k_tile_smooth(TileRound a, float* x) {
  __shared__ __align__(16) float xs[4 * kSub * KP];
  __shared__ __align__(16) float bs[kTileSlots * KP];
  __shared__ int segOff[kTileMaxSegs], segG[kTileMaxSegs], segP[kTileMaxSegs];
  __shared__ unsigned char deep[kTileSlots];
  __shared__ int sTile, sStart[5];
  grid_dependency_wait();
  const int t = threadIdx.x;
  if (t == 0) {  // indexed by colour below: shared memory, not the parameter
#pragma unroll
    for (int k = 0; k < 5; k++) sStart[k] = a.tileStart[k];
  }
  const int p = t % kHalfW, q = t / kHalfW;
  int* counter = a.sync;
  int* exits = a.sync + 1;
  int* done = a.sync + 2;
  for (;;) {
    if (t == 0) sTile = atomicAdd(counter, 1);
    __syncthreads();
    const int idx = sTile;
    if (idx >= a.nTiles) break;
    // the idx-th tile in colour order
    int tile = idx, rank = 0;
    for (int k = 0, base = 0; k < 4; k++) {
      const int c = a.reverse ? 3 - k : k, n = sStart[c + 1] - sStart[c];
      if (idx < base + n) { tile = sStart[c] + idx - base; rank = k; break; }
      base += n;
    }
    const int4 T = a.tiles[tile];  // {first coefficient, first segment, segments, elements}
    // segment descriptors {first global texel, row | column << 6 | length << 12,
    // first element of the segment within the tile} to shared memory
    for (int i = t; i < T.z; i += kPerColour) {
      const int4 sg = a.segs[T.y + i];
      segG[i] = sg.x;
      segP[i] = sg.y;
      segOff[i] = sg.z;
    }
    // this thread's coefficients, one texel per colour (planes of kTileSlots)
    float c[4][10];
#pragma unroll
    for (int cc = 0; cc < 4; cc++)
#pragma unroll
      for (int k = 0; k < 10; k++) c[cc][k] = __ldg(a.coef + (long long)T.x + k * kTileSlots + cc * kPerColour + t);
#pragma unroll
    for (int cc = 0; cc < 4; cc++) deep[cc * kPerColour + t] = c[cc][9] != 0.f ? 1 : 0;
    // a tile first in its round from a zero iterate sees only zeros
    const bool zero = a.zeroStart && rank == 0;
    if (zero)
      for (int i = t; i < 4 * kSub * KP; i += kPerColour) xs[i] = 0.f;
    __syncthreads();
    // this thread's elements (active texels of the tile and its ring); the
    // right-hand side (fixed during the round) is copied before the wait
    int gE[kElemsPerThread], sE[kElemsPerThread], slotE[kElemsPerThread];
#pragma unroll
    for (int m = 0; m < kElemsPerThread; m++) {
      const int e = t + m * kPerColour;
      int g = -1, so = 0, slot = -1;
      if (e < T.w) {
        int lo = 0;  // last segment with segOff <= e (fixed-step binary search)
#pragma unroll
        for (int step = 512; step >= 1; step >>= 1)
          if (lo + step < T.z && segOff[lo + step] <= e) lo += step;
        const int pk = segP[lo], r = pk & 63, u = ((pk >> 6) & 63) + (e - segOff[lo]);
        const int U = u + 1, V = r + 1;  // tile-local i + 2, j + 2 (same parity as i, j)
        const int sub = (U & 1) | ((V & 1) << 1);
        g = segG[lo] + (e - segOff[lo]);
        so = (sub * kSub + (V >> 1) * kSubW + (U >> 1)) * KP;
        if (u >= 1 && u <= kTileW && r >= 1 && r <= kTileH) {
          slot = sub * kPerColour + ((V >> 1) - 1) * kHalfW + ((U >> 1) - 1);
          cp_async<KP>(bs + slot * KP, a.rhs + (long long)g * KP);
        }
      }
      gE[m] = g;
      sE[m] = so;
      slotE[m] = slot;
    }
    // wait for the neighbours that come earlier in the round (one thread each)
    if (t < 8) {
      const int nb = a.nbrs[8 * tile + t];
      if (nb >= 0) {
        int cn = 0;
        while (cn < 3 && nb >= sStart[cn + 1]) cn++;
        if (colour_rank(cn, a.reverse) < rank) {
          long long polls = 0;
          while (ld_acquire_gpu(done + nb) == 0) {
            if (++polls > kTilePolls) { atomicExch(a.err, 2); break; }
            __nanosleep(32);
          }
        }
      }
    }
    __syncthreads();
    // x of the tile and its ring, read through L2 (other CTAs wrote it during
    // this launch)
    if (!zero) {
#pragma unroll
      for (int m = 0; m < kElemsPerThread; m++)
        if (gE[m] >= 0) tstore<KP>(xs + sE[m], tload_l2<KP>(x + (long long)gE[m] * KP));
    }
    cp_async_wait_all();
    __syncthreads();
    for (int sw = 0; sw < a.sweeps; sw++) {
      if (a.reverse) {
        pass<KP, 3>(xs, bs, c, p, q);
        pass<KP, 2>(xs, bs, c, p, q);
        pass<KP, 1>(xs, bs, c, p, q);
        pass<KP, 0>(xs, bs, c, p, q);
      } else {
        pass<KP, 0>(xs, bs, c, p, q);
        pass<KP, 1>(xs, bs, c, p, q);
        pass<KP, 2>(xs, bs, c, p, q);
        pass<KP, 3>(xs, bs, c, p, q);
      }
    }
    // the deep texels back (the only ones the sweeps change), element by
    // element so that neighbouring threads write neighbouring texels
#pragma unroll
    for (int m = 0; m < kElemsPerThread; m++)
      if (slotE[m] >= 0 && deep[slotE[m]]) tstore<KP>(x + (long long)gE[m] * KP, tload<KP>(xs + sE[m]));
    __syncthreads();
    if (t == 0) {
      __threadfence();  // the tile's texels before its flag
      st_release_gpu(done + tile, 1);
    }
  }
  // the last CTA out (every tile is done by then) leaves the counters and
  // flags zero for the next round
  __shared__ int last;
  if (t == 0) last = atomicAdd(exits, 1) == int(gridDim.x) - 1;
  __syncthreads();
  if (last) {
    __threadfence();
    for (int i = t; i < a.nTiles; i += kPerColour) done[i] = 0;
    __syncthreads();
    if (t == 0) {
      *counter = 0;
      *exits = 0;
      __threadfence();
    }
  }
  grid_launch_dependents();
}

}  // namespace

// CTAs of the round per SM (the kernel's occupancy), per device
static int tile_ctas_per_sm(int KP) {
  static std::atomic<int> slots[2][kMaxDevices];
  static const bool init = [] {
    for (auto& row : slots)
      for (auto& a : row) a.store(kUnset);
    return true;
  }();
  (void)init;
  return per_device_once(slots[KP == 4 ? 1 : 0], [KP] {
    int n = 0;
    const cudaError_t e = KP == 4 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_tile_smooth<4>, kPerColour, 0)
                                  : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_tile_smooth<1>, kPerColour, 0);
    return e == cudaSuccess && n > 0 ? n : 1;
  });
}

bool launch_tile_smooth(const TileRound& round, float* x, int KP, cudaStream_t s) {
  if (round.nTiles == 0 || round.sweeps <= 0) return true;
  if (KP != 1 && KP != 4) return false;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return false;
  const int ctas = std::max(1, std::min(round.nTiles, sms * tile_ctas_per_sm(KP)));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ctas);
  cfg.blockDim = dim3(kPerColour);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = programmatic_launch() ? 1 : 0;
  if (KP == 4) return cudaLaunchKernelEx(&cfg, k_tile_smooth<4>, round, x) == cudaSuccess;
  return cudaLaunchKernelEx(&cfg, k_tile_smooth<1>, round, x) == cudaSuccess;
}

}  // namespace dev
}  // namespace gdtp
