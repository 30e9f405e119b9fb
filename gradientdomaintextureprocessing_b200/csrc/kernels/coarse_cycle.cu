// Coarse levels of the V-cycle in one thread-block cluster.
//
// Below a few hundred thousand texels a level's work is far too small for the
// GPU: each phase (a colour pass, the residual, the restriction, a boundary
// product) costs one dependent launch, and those latencies, not bandwidth, set
// the time of the coarse half of the V-cycle.  Here a single cluster of up to
// 16 CTAs x 1024 threads runs every phase of the coarse levels back to back,
// separated by hardware cluster barriers (barrier.cluster arrive.release /
// wait.acquire).  The work stays in L2, which the phases read through ld.cg
// (LoadL2) because each reads what other CTAs wrote in the previous phase.
//
// The per-item arithmetic is the kernels' own (vcycle_ops.cuh), and the dense
// boundary products reproduce the launch path's partition and summation order
// (row groups of 128, j chunks of the same length, 8 interleaved warps per
// chunk, chunk sums in chunk order), so a V-cycle gives the same bits on
// either path.
//
// The same kernel also runs persistently on the whole GPU (one cooperative
// launch, every CTA resident) with a software grid barrier between phases:
// one barrier (an atomic arrival and a poll of a generation word in L2) costs
// far less than a dependent launch, and the phases get all SMs instead of one
// cluster's.  The barrier's polls are bounded: a block that waits too long
// records an error and every block abandons the remaining phases, so a lost
// block cannot hang the GPU; the host reads the error word after the solve.
#include <cooperative_groups.h>

#include <algorithm>

#include "vcycle.cuh"
#include "vcycle_kernels.h"
#include "vcycle_ops.cuh"

namespace cg = cooperative_groups;

namespace gdtp {
namespace dev {

constexpr int kClusterBlock = 1024;   // threads per CTA
constexpr int kChunkGroups = kClusterBlock / 256;  // chunks processed at once (8 warps each)

template <typename T, int W>
static size_t cluster_smem_bytes() {
  // per-warp partials [32 warps][32 lanes][4W] + chunk inputs [groups][kBoundaryChunkMax]
  return size_t(32) * 32 * 4 * W * sizeof(T) + size_t(kChunkGroups) * kBoundaryChunkMax * sizeof(Vec<T, W>);
}

// One dense boundary product (mode 0: subdomain inverses, mode 1: separator
// Schur inverse) by the CTAs of the cluster, tasks split across CTAs.
template <typename T, int W>
__device__ void cluster_bs_dense(const BoundaryDev<T>& B, int mode, const T* rhs, T* x, int KP, int G, T* red, Vec<T, W>* vin) {
  const int nTasks = mode == 0 ? B.nSubTasks : B.nSchurTasks;
  const int4* tasks = mode == 0 ? B.subTasks : B.schurTasks;
  const int nch = mode == 0 ? B.subChunks : B.schurChunks;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, grp = warp >> 3, lw = warp & 7;
  constexpr int NO = 32 * 4 * W;  // outputs of a row group per channel group
  for (int ti = blockIdx.x; ti < nTasks; ti += gridDim.x) {
    const int4 task = tasks[ti];
    const int r0 = mode == 0 ? B.subPtr[task.x] : 0;
    const int m = mode == 0 ? B.subPtr[task.x + 1] - r0 : B.nS, mp = (m + 3) & ~3;
    const T* M = mode == 0 ? B.inv + B.invOff[task.x] : B.sinv;
    const int clen = (m + nch - 1) / nch;
    const int rq = task.y + lane;
    const bool active = 4 * rq < m;
    for (int q = 0; q < G; q++) {
      const int off = q * W;
      T S = 0;  // running chunk sum of output threadIdx.x (< NO)
      for (int c0 = 0; c0 < nch; c0 += kChunkGroups) {
        // inputs of the (up to) kChunkGroups chunks
        for (int g = 0; g < kChunkGroups && c0 + g < nch; g++) {
          const int j0 = min(m, (c0 + g) * clen), j1 = min(m, j0 + clen);
          if (mode == 0) {
            for (int j = j0 + (int)threadIdx.x; j < j1; j += kClusterBlock)
              vin[g * kBoundaryChunkMax + (j - j0)] = LoadL2::ld<T, W>(B.rhat + (long long)(r0 + j) * KP + off);
          } else {
            const int lane8 = threadIdx.x & 7;
            for (int jb = j0; jb < j1; jb += kClusterBlock / 8) {
              const int j = jb + (int)(threadIdx.x >> 3);
              const Vec<T, W> v = bs_schur_input_group<T, W, LoadL2>(B, j, j < j1, KP, off, lane8);
              if (j < j1 && lane8 == 0) vin[g * kBoundaryChunkMax + (j - j0)] = v;
            }
          }
        }
        __syncthreads();
        T acc[4][W];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int c = 0; c < W; c++) acc[a][c] = 0;
        const int ch = c0 + grp;
        if (ch < nch && active) {
          const int j0 = min(m, ch * clen), j1 = min(m, j0 + clen);
#pragma unroll 4
          for (int j = j0 + lw; j < j1; j += 8) {
            const Quad<T> mq = *reinterpret_cast<const Quad<T>*>(M + (long long)j * mp + 4 * rq);
            const Vec<T, W> v = vin[grp * kBoundaryChunkMax + (j - j0)];
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
              for (int c = 0; c < W; c++) acc[a][c] += mq.v[a] * v.v[c];
          }
        }
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int c = 0; c < W; c++) red[(warp * 32 + lane) * 4 * W + a * W + c] = acc[a][c];
        __syncthreads();
        if ((int)threadIdx.x < NO) {
          const int o = threadIdx.x, ol = o / (4 * W), oi = o - ol * 4 * W;
          for (int g = 0; g < kChunkGroups && c0 + g < nch; g++) {
            T v = 0;
            for (int w = 0; w < 8; w++) v += red[((g * 8 + w) * 32 + ol) * 4 * W + oi];
            S += v;
          }
        }
        __syncthreads();
      }
      if ((int)threadIdx.x < NO) {
        const int o = threadIdx.x, ol = o / (4 * W), oi = o - ol * 4 * W, a = oi / W, c = oi - a * W;
        const int row = 4 * (task.y + ol) + a;
        if (row < m) {
          if (mode == 0) {
            B.y[(long long)(r0 + row) * KP + off + c] = S;
          } else {
            B.xs[(long long)row * KP + off + c] = S;
            x[(long long)B.posGlobal[B.nI + row] * KP + off + c] = S * B.scale[B.nI + row];
          }
        }
      }
    }
  }
}

struct CoarseCycleArgs {
  int l0, L;            // levels l0 .. L-1 of the V-cycle, L-1 the coarsest
  int leg;              // 0: down leg (ends with the restriction into L-1), 1: up leg, 2: both + coarse solve
  CoarseSweeps sw;
  int KP;
  int coarseN;
  const double* coarseInv;
  const double* coarseScale;
  unsigned long long* timeline;  // optional: {phase code, globaltimer ns} after every phase (CTA 0)
  GridBarrierState* barrier;     // persistent whole-GPU variant only
};

// Polls of the barrier's generation word before a block gives up (about a
// second at most); a phase of the coarse levels takes microseconds.
constexpr long long kBarrierPolls = 1ll << 20;

__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier: every block's writes before it are visible to every block
// after it.  The last block to arrive resets the count and advances the
// generation; the others poll the generation (bounded).  Returns false, in
// every thread of the block, once any block has recorded a timeout.
__device__ bool grid_barrier(GridBarrierState* gb, unsigned int& gen) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();  // release this block's writes
    const unsigned int g = gen;
    if (atomicAdd(&gb->count, 1u) == gridDim.x - 1) {
      atomicExch(&gb->count, 0u);
      __threadfence();
      atomicExch(&gb->gen, g + 1);
    } else {
      long long polls = 0;
      while (ld_acquire_gpu(&gb->gen) == g) {
        if (++polls > kBarrierPolls) { atomicExch(&gb->error, 1u); break; }
        __nanosleep(64);
      }
    }
    __threadfence();  // acquire the other blocks' writes
    gen = g + 1;
    ok = ld_acquire_gpu(&gb->error) == 0;
  }
  __syncthreads();
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// kGrid false: one thread-block cluster (cluster barriers); true: every SM,
// cooperative launch, grid barriers.
template <typename T, int W, bool kGrid>
__global__ void __launch_bounds__(kClusterBlock, 1) k_coarse_cycle(const LevelDev<T>* __restrict__ lv, CoarseCycleArgs a) {
  grid_dependency_wait();
  // the persistent variant lets the next kernel launch only when it is done
  // (early dependents would only take SM slots from nothing)
  if constexpr (!kGrid) grid_launch_dependents();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* red = reinterpret_cast<T*>(smem_raw);
  Vec<T, W>* vin = reinterpret_cast<Vec<T, W>*>(red + 32 * 32 * 4 * W);
  const int KP = a.KP, G = KP / W;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  int phase = a.leg == 1 ? 255 : 0;  // the up leg stamps the second half
  unsigned int gen = 0;
  if (kGrid) gen = ld_acquire_gpu(&a.barrier->gen);  // nobody advances it before every block has arrived once
  bool alive = true;
  // barrier between phases; with a timeline, CTA 0 stamps the phase's end.
  // After a barrier timeout (grid variant) the remaining phases are skipped.
  auto sync = [&](int code) {
    if constexpr (kGrid) {
      if (alive) alive = grid_barrier(a.barrier, gen);
    } else {
      cg::this_cluster().sync();
    }
    if (a.timeline && blockIdx.x == 0 && threadIdx.x == 0 && phase < 510) {
      a.timeline[2 * phase] = (unsigned long long)code;
      a.timeline[2 * phase + 1] = global_ns();
    }
    phase++;
  };
  if (a.timeline && blockIdx.x == 0 && threadIdx.x == 0) a.timeline[a.leg == 1 ? 1020 : 1022] = global_ns();  // start
  auto boundary_solve = [&](const LevelDev<T>& D, int code) {
    const BoundaryDev<T>& B = D.B;
    if (B.nb == 0 || !alive) return;
    // 8-lane group items, 4 per warp, warp-uniform loops
    const long long w0 = tid >> 5, nw = nth >> 5;
    const int lane = threadIdx.x & 31;
    for (long long gb = w0 * 4; gb < (long long)B.nb * G; gb += nw * 4)
      bs_prep_group<T, W, LoadL2>(B, D.b, D.x, KP, G, gb + (lane >> 3), lane & 7);
    sync(code + 4);
    if (B.nSubTasks > 0) { cluster_bs_dense<T, W>(B, 0, D.b, D.x, KP, G, red, vin); sync(code + 1); }
    if (B.nS > 0) { cluster_bs_dense<T, W>(B, 1, D.b, D.x, KP, G, red, vin); sync(code + 2); }
    if (B.nI > 0) {
      for (long long gb = w0 * 4; gb < (long long)B.nI * G; gb += nw * 4)
        bs_back_group<T, W, LoadL2>(B, D.x, KP, G, gb + (lane >> 3), lane & 7);
      sync(code + 3);
    }
  };
  auto colour_pass = [&](const LevelDev<T>& D, int c, int code) {
    const int nr = alive ? D.runStart[c + 1] - D.runStart[c] : 0;
    for (long long t = tid; t < (long long)nr * 32 * G; t += nth)
      gs_item<T, W, LoadL2>(D.runs + D.runStart[c], nr, D.coef, D.planeStride, D.b, D.x, KP, G, t);
    sync(code + c);
  };
  if (a.leg != 1) {
    for (int l = a.l0; l + 1 < a.L && alive; l++) {
      const LevelDev<T>& D = lv[l];
      const LevelDev<T>& C = lv[l + 1];
      if (a.sw.preBoundary) boundary_solve(D, 1000 * l);
      for (int sw = 0; sw < a.sw.pre(l); sw++)
        for (int c = 0; c < 4; c++) colour_pass(D, c, 1000 * l + 10);
      for (long long t = alive ? tid : (long long)D.nRuns * 32 * G; t < (long long)D.nRuns * 32 * G; t += nth)
        residual_deep_item<T, W, LoadL2>(D.runs, D.nRuns, D.coef, D.planeStride, D.b, D.x, D.r, KP, G, t);
      for (long long t = tid; t < (long long)D.nB * G; t += nth)
        residual_boundary_item<T, W, LoadL2>(D.bPtr, D.bCol, D.bVal, D.bGlobal, D.nB, D.b, D.x, D.r, KP, G, t);
      sync(1000 * l + 20);
      for (long long i = tid; i < (long long)C.n * KP; i += nth) C.x[i] = T(0);
      for (long long t = tid; t < (long long)D.nRRuns * 32 * G; t += nth)
        restrict_deep_item<T, W, LoadL2>(D.rruns, D.nRRuns, D.r, C.b, KP, G, t);
      for (long long t = tid; t < (long long)D.nRB * G; t += nth)
        restrict_boundary_item<T, W, LoadL2>(D.rbPtr, D.rbCol, D.rbVal, D.rbOut, D.nRB, D.r, C.b, KP, G, t);
      sync(1000 * l + 21);
    }
  }
  if (a.leg == 2 && alive) {
    const LevelDev<T>& C = lv[a.L - 1];
    const int lane = threadIdx.x & 31;
    for (long long w = tid >> 5; w < a.coarseN; w += nth >> 5)
      coarse_row<T, W, LoadL2>(a.coarseN, a.coarseInv, a.coarseScale, C.b, C.x, KP, G, (int)w, lane);
    sync(1000 * (a.L - 1) + 30);
  }
  if (a.leg != 0) {
    for (int l = a.L - 2; l >= a.l0 && alive; l--) {
      const LevelDev<T>& D = lv[l];
      const LevelDev<T>& C = lv[l + 1];
      for (long long t = tid; t < (long long)D.nPRuns * 32 * G; t += nth)
        prolong_item<T, W, LoadL2>(D.pruns, D.nPRuns, C.x, D.x, KP, G, t);
      sync(1000 * l + 40);
      if (a.sw.postBoundary) boundary_solve(D, 1000 * l + 40);
      for (int sw = 0; sw < a.sw.post(l); sw++)
        for (int c = 3; c >= 0; c--) colour_pass(D, c, 1000 * l + 50);
    }
  }
}

template <typename T, int W>
int coarse_cycle_cluster_size_uncached();
template <typename T, int W>
int coarse_cycle_cluster_size() {
  static std::atomic<int> cached[kMaxDevices];
  static const bool init = [] {
    for (auto& a : cached) a.store(kUnset);
    return true;
  }();
  (void)init;
  return per_device_once(cached, [] { return coarse_cycle_cluster_size_uncached<T, W>(); });
}
template <typename T, int W>
int coarse_cycle_cluster_size_uncached() {
  auto k = k_coarse_cycle<T, W, false>;
  const size_t smem = cluster_smem_bytes<T, W>();
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
      cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(16);
  cfg.blockDim = dim3(kClusterBlock);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 16;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int cs = 0;
  if (cudaOccupancyMaxPotentialClusterSize(&cs, k, &cfg) != cudaSuccess) {
    cudaGetLastError();
    cs = 0;
  }
  for (int c : {16, 8, 4}) {  // largest supported size that can run
    if (cs < c) continue;
    attr[0].val.clusterDim.x = c;
    cfg.gridDim = dim3(c);
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, k, &cfg) == cudaSuccess && clusters >= 1) return c;
    cudaGetLastError();
  }
  return 0;
}

// Every SM x the CTAs of this kernel that fit on one (all resident at once, as
// a cooperative launch requires).
template <typename T, int W>
int coarse_cycle_grid_size_uncached();
template <typename T, int W>
int coarse_cycle_grid_size() {
  static std::atomic<int> cached[kMaxDevices];
  static const bool init = [] {
    for (auto& a : cached) a.store(kUnset);
    return true;
  }();
  (void)init;
  return per_device_once(cached, [] { return coarse_cycle_grid_size_uncached<T, W>(); });
}
template <typename T, int W>
int coarse_cycle_grid_size_uncached() {
  auto k = k_coarse_cycle<T, W, true>;
  const size_t smem = cluster_smem_bytes<T, W>();
  int dev = 0, sms = 0, coop = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop ||
      cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, kClusterBlock, smem) != cudaSuccess || per < 1) {
    cudaGetLastError();
    return 0;
  }
  return sms * per;
}

template <typename T, int W>
bool launch_coarse_cycle(const LevelDev<T>* lvDev, int l0, int L, int leg, const CoarseSweeps& sw, int KP, int coarseN,
                         const double* coarseInv, const double* coarseScale, unsigned long long* timeline,
                         GridBarrierState* barrier, cudaStream_t s) {
  CoarseCycleArgs a{l0, L, leg, sw, KP, coarseN, coarseInv, coarseScale, timeline, barrier};
  cudaLaunchConfig_t cfg = {};
  cfg.blockDim = dim3(kClusterBlock);
  cfg.dynamicSmemBytes = cluster_smem_bytes<T, W>();
  cfg.stream = s;
  cudaLaunchAttribute attr[2];
  cfg.attrs = attr;
  if (barrier) {
    // every CTA resident: cooperative launch (no programmatic overlap with the
    // previous kernel, whose CTAs would hold SMs the barrier needs)
    const int ctas = coarse_cycle_grid_size<T, W>();
    if (ctas == 0) return false;
    cfg.gridDim = dim3(ctas);
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_coarse_cycle<T, W, true>, lvDev, a) == cudaSuccess;
  }
  const int cs = coarse_cycle_cluster_size<T, W>();
  if (cs == 0) return false;
  cfg.gridDim = dim3(cs);
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.numAttrs = programmatic_launch() ? 2 : 1;
  return cudaLaunchKernelEx(&cfg, k_coarse_cycle<T, W, false>, lvDev, a) == cudaSuccess;
}

int coarse_cycle_cluster_ctas(bool fp64, int W) {
  if (fp64) return W == 4 ? coarse_cycle_cluster_size<double, 4>() : coarse_cycle_cluster_size<double, 1>();
  return W == 4 ? coarse_cycle_cluster_size<float, 4>() : coarse_cycle_cluster_size<float, 1>();
}
int coarse_cycle_grid_ctas(bool fp64, int W) {
  if (fp64) return W == 4 ? coarse_cycle_grid_size<double, 4>() : coarse_cycle_grid_size<double, 1>();
  return W == 4 ? coarse_cycle_grid_size<float, 4>() : coarse_cycle_grid_size<float, 1>();
}

#define GDTP_COARSE_CYCLE(T, W)                                                                                         \
  template bool launch_coarse_cycle<T, W>(const LevelDev<T>*, int, int, int, const CoarseSweeps&, int, int, const double*, \
                                          const double*, unsigned long long*, GridBarrierState*, cudaStream_t);
GDTP_COARSE_CYCLE(float, 1)
GDTP_COARSE_CYCLE(float, 4)
GDTP_COARSE_CYCLE(double, 1)
GDTP_COARSE_CYCLE(double, 4)

}  // namespace dev
}  // namespace gdtp
