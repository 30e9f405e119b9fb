// Heat-method geodesic distances on the texel grid (the Geodesics app's
// pipeline, Geodesics/Geodesics.cpp:507-550):
//   (1) smooth an impulse:      (M + t S) u = delta_source
//   (2) integrate the unit field X = -grad u / |grad u| against the basis
//       gradients (VectorFieldIntergration.inl), boundary terms through the
//       fine boundary nodes (prolong u, integrate, restrict back)
//   (3) solve the Poisson problem (eps M + S) d = rhs, shift d(source) = 0.
// All three steps run on the device; k sources are k right-hand sides.
#pragma once
#include <string>

#include "kernels/geodesic_kernels.h"
#include "system.h"

namespace gdtp {

class GeodesicIntegrator {
 public:
  // Samples from the system's hierarchy, boundary elements and metric.
  explicit GeodesicIntegrator(DeviceSystem& sys);
  bool ok() const { return err_.empty(); }
  const std::string& error() const { return err_; }

  // rhs (n x k, FP64) of the potential u (n x k, FP64), device buffers, stream-ordered
  bool rhs_device(const double* u, double* rhs, int k, cudaStream_t s);
  // same on host buffers
  bool rhs_host(const double* u, double* rhs, int k);
  // heat-method distances from k source texels; smooth: M + t S, dist: eps M + S
  // (both updated by the caller); d_host: n x k
  bool distance(DeviceSystem& smooth, DeviceSystem& dist, const int* sources, int k, double tol, int maxIters, double* d_host,
                SolveReport& smoothRep, SolveReport& distRep);

  int cellSlots = 0, hexSlots = 0;
  // host copies for inspection: "cellSamples" (16 per slot), "hexSamples" (20 per
  // slot), "cellPtr", "corners", "slotBt", "btIdx"
  bool download(const std::string& name, std::vector<double>& out);

 private:
  bool ensure_k(int k);
  bool check(cudaError_t e, const char* what);

  DeviceSystem& sys_;
  std::string err_;
  DeviceArena arena_, work_;
  dev::GeoDev G_;
  // distance pipeline buffers (n x dK_), kept so that the solves' captured graphs are reused
  DeviceArena dwork_;
  int dK_ = 0;
  double *b_ = nullptr, *u_ = nullptr, *r_ = nullptr, *d_ = nullptr, *sv_ = nullptr;
  int* src_ = nullptr;
};

}  // namespace gdtp
