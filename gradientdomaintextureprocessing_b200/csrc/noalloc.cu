// Residual and norms with caller-owned buffers and no device allocation.
//
// Some callers cannot allocate device memory at the moment they need a
// residual check: a render or simulation loop that plans all its memory up
// front, code that runs while a stream-ordered memory pool must not grow, or a
// host that forbids cudaMalloc because it would synchronise the device in the
// middle of its own work.  gdtp_residual_static serves them: the caller passes
// its own device buffers for b, x and the residual, and the per-block partial
// sums of the norm reduction live in the fixed-size device array below instead
// of in memory allocated by the library.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <string>

#include "gdtp.h"
#include "capi_internal.h"
#include "kernels/vcycle_kernels.h"
#include "system.h"

namespace {

// Upper bounds of the static scratch: the operator kernel runs a fixed grid of
// at most kRawMaxBlocks blocks, each writing 2*k partial sums, plus 2*k totals.
constexpr int kStaticMaxRhs = 64;
constexpr int kStaticBlocks = gdtp::dev::kRawMaxBlocks;
constexpr size_t kStaticScratch = size_t(kStaticBlocks) * 2 * kStaticMaxRhs + 2 * kStaticMaxRhs;  // doubles (~2.1 MB)

// Held by every device that loads the library until the process exits.  In
// host code this name is only a stand-in for the symbol: its device address is
// looked up once per device with cudaGetSymbolAddress.
__device__ __align__(256) double g_residual_scratch[kStaticScratch];

// Device address of the array per device ordinal, published atomically: the
// server's workers may make their first call on one device at the same time
// (both resolve and store the same address).
constexpr int kMaxDevices = 64;
std::atomic<double*> g_scratch_address[kMaxDevices];

// Puts the caller's current device back on every return path.
struct DeviceRestore {
  int saved = -1;
  DeviceRestore() {
    if (cudaGetDevice(&saved) != cudaSuccess) saved = -1;
  }
  ~DeviceRestore() {
    if (saved >= 0) cudaSetDevice(saved);
  }
};

}  // namespace

using namespace gdtp;

struct gdtp_system;  // defined in capi_system.cpp; accessed through gdtp_system_device_view
extern "C" __attribute__((visibility("hidden"))) int gdtp_system_device_view(const gdtp_system* s, const void** sys);

extern "C" int gdtp_residual_static(gdtp_system* s, const double* b_dev, const double* x_dev, double* r_dev, int k,
                                    double* rel_host, void* stream) {
  const void* view = nullptr;
  if (gdtp_system_device_view(s, &view) != GDTP_OK || !view) return fail(GDTP_ERR_INVALID, "gdtp_residual_static: null system");
  const DeviceSystem& sys = *static_cast<const DeviceSystem*>(view);
  if (!b_dev || !x_dev || !r_dev || !rel_host) return fail(GDTP_ERR_INVALID, "gdtp_residual_static: null buffer");
  if (k < 1 || k > kStaticMaxRhs)
    return fail(GDTP_ERR_INVALID, "gdtp_residual_static: k=" + std::to_string(k) + " exceeds the static scratch limit of " +
                                      std::to_string(kStaticMaxRhs) + " right-hand sides");
  if (!sys.is_updated()) return fail(GDTP_ERR_STATE, "gdtp_residual_static: system not updated");
  const int dev = sys.device();
  if (dev < 0 || dev >= kMaxDevices) return fail(GDTP_ERR_INVALID, "gdtp_residual_static: device ordinal out of range");
  DeviceRestore restore;
  cudaError_t e = cudaSetDevice(dev);
  if (e != cudaSuccess) return fail(GDTP_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  const RawOperator& op = sys.raw_system_operator();
  if (op.nRuns == 0 && op.nB == 0) {  // no rows: nothing to write, and no norm to report
    for (int c = 0; c < k; c++) rel_host[c] = 0.0;
    return GDTP_OK;
  }
  // first call on this device: resolve the static array's device address (must
  // happen outside stream capture; later calls only launch kernels and copy)
  double* partials = g_scratch_address[dev].load(std::memory_order_acquire);
  if (!partials) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_residual_scratch);
    if (e != cudaSuccess) return fail(GDTP_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    partials = static_cast<double*>(p);
    g_scratch_address[dev].store(partials, std::memory_order_release);
  }
  double* sums = partials + size_t(kStaticBlocks) * 2 * kStaticMaxRhs;
  if (dev::raw_operator_blocks(op.nRuns, op.nB, k) > kStaticBlocks)
    return fail(GDTP_ERR_INVALID, "gdtp_residual_static: operator grid exceeds the static scratch");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // every block overwrites its own partials and the reduction overwrites the
  // totals, so the scratch needs no clearing between calls
  dev::launch_raw_operator(op.runs, op.nRuns, op.coef, op.planeStride, op.bPtr, op.bCol, op.bVal, op.bGlobal, op.nB, b_dev, x_dev,
                           r_dev, k, 0, partials, sums, st);
  double tot[2 * kStaticMaxRhs];
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(tot, sums, 2 * size_t(k) * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(GDTP_ERR_CUDA, std::string("gdtp_residual_static: ") + cudaGetErrorString(e));
  for (int c = 0; c < k; c++) rel_host[c] = std::sqrt(tot[c] / (tot[k + c] > 0 ? tot[k + c] : 1e-300));
  return GDTP_OK;
}
