// Drop-in forwarding of the reference's solve path to libgdtp (gdtp.h).
//
// The reference is header-only: TextureFiltering, Geodesics and
// LineIntegralConvolution include <Src/Hierarchy.h> and <Src/MassAndStiffness.h>
// and instantiate its templates.  Put this repository's include/ directory
// before the reference's on the include path and link libgdtp: the two
// wrapper headers of the same names include the reference's own headers
// (#include_next) and then this file (Src/Hierarchy.h) or
// gdtp_dropin_assembly.inl (Src/MassAndStiffness.h), and the apps' code
// compiles unchanged:
//
//   g++ -I<repo>/include -I<reference>/include app.cpp -L<repo>/gradientdomaintextureprocessing_b200 -lgdtp
//
// What is forwarded, and how:
//  * UpdateLinearSystem (UpdateCoefficients.inl:463-469), VCycle
//    (IterativeSolvers.inl:1211-1216) and MultiplyBySystemMatrix_NoReciprocals
//    (IterativeSolvers.inl:881) are function templates.  The templates below
//    take the same arguments with the app's Real (REAL_TYPE) fixed, so they are
//    more specialised and C++ overload resolution picks them at every app call.
//  * InitializeHierarchy (HierarchyConstruction.inl:799-800) and
//    InitializeMassAndStiffness (MassAndStiffness.h:490-495) are plain
//    functions: a macro after the reference's definitions sends the apps'
//    calls to wrappers with the same parameters, which run the reference's
//    own set-up (the apps keep using its outputs) and record what the device
//    system is built from: the mesh (keyed by the hierarchy's address) and the
//    parameter metric with the operator's coefficient arrays (keyed by the
//    deep mass and stiffness arrays' addresses).
//  * The first UpdateLinearSystem of an operator builds the device system:
//    the hierarchy from the recorded mesh (bit-exact to the reference's, so
//    texel vectors keep their order) and the FP64 assembly on the GPU with the
//    recorded metric.  Later calls only re-weight it.  The multigrid
//    coefficient vector's address then names the device system for VCycle.
//  * VCycle uploads variables[0].x and .rhs, runs one V-cycle on the device
//    (FP32 when REAL_TYPE is float, FP64 otherwise) and downloads x: the
//    host-visible vectors the apps read and write between cycles stay valid.
//  * MultiplyBySystemMatrix_NoReciprocals on a recorded deep mass or stiffness
//    array applies that operator on the device (FP64); on any other array it
//    is the reference's own template.
//  * The --useDirectSolver factorisation (fineSolver) stays the reference's.
// Errors print "ERROR ..." and return 0, the reference's convention.
#pragma once

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <utility>
#include <vector>

#include "../gdtp.h"

namespace gdtp_dropin {

struct MeshRecord {
  std::vector<double> vertices, uv;
  std::vector<int32_t> triangles;
  int width = 0, height = 0, levels = 0;
  gdtp_hierarchy* hierarchy = nullptr;
};

struct OperatorRecord {
  const void* hierarchy = nullptr;  // key of its MeshRecord
  std::vector<double> metric;       // per mesh triangle: g(0,0) g(0,1) g(1,0) g(1,1)
  gdtp_system* system = nullptr;
};

inline std::map<const void*, MeshRecord>& meshes() {
  static std::map<const void*, MeshRecord> m;
  return m;
}
inline std::map<const void*, OperatorRecord>& operators() {  // keyed by the deep mass array
  static std::map<const void*, OperatorRecord> m;
  return m;
}
inline std::map<const void*, std::pair<const void*, int>>& deep_arrays() {  // deep array -> (operator, 1 mass / 2 stiffness)
  static std::map<const void*, std::pair<const void*, int>> m;
  return m;
}
inline std::map<const void*, gdtp_system*>& coefficient_systems() {  // multigrid coefficients -> system
  static std::map<const void*, gdtp_system*> m;
  return m;
}

inline int device() {
  const char* d = std::getenv("GDTP_DEVICE");
  return d ? std::atoi(d) : 0;
}

inline bool ok(int code, const char* what) {
  if (code != GDTP_OK) std::printf("ERROR : %s: %s\n", what, gdtp_last_error());
  return code == GDTP_OK;
}

// The device system of a recorded operator, built on first use.
inline gdtp_system* system_of(OperatorRecord& op) {
  if (op.system) return op.system;
  auto m = meshes().find(op.hierarchy);
  if (m == meshes().end()) {
    std::printf("ERROR : gdtp drop-in: no InitializeHierarchy recorded for this hierarchy\n");
    return nullptr;
  }
  MeshRecord& r = m->second;
  if (!r.hierarchy &&
      !ok(gdtp_hierarchy_build(r.vertices.data(), int64_t(r.vertices.size() / 3), r.triangles.data(), int64_t(r.triangles.size() / 3),
                               r.uv.data(), r.width, r.height, r.levels, nullptr, &r.hierarchy),
          "gdtp_hierarchy_build"))
    return nullptr;
  const double* metric = op.metric.empty() ? nullptr : op.metric.data();
  if (!ok(gdtp_system_create(r.hierarchy, device(), 0, metric, r.vertices.data(), int64_t(r.vertices.size() / 3), &op.system),
          "gdtp_system_create"))
    return nullptr;
  return op.system;
}

// Channels of a texel value: RGB in a 4-lane vector (lane 3 unused) or a scalar.
inline int channels(const float&) { return 1; }
inline int channels(const double&) { return 1; }
template <class R>
inline void get(const float& v, R* a) { a[0] = R(v); }
template <class R>
inline void get(const double& v, R* a) { a[0] = R(v); }
template <class R>
inline void set(float& v, const R* a) { v = float(a[0]); }
template <class R>
inline void set(double& v, const R* a) { v = double(a[0]); }
#ifdef VECTOR_TYPE
inline int channels(const VECTOR_TYPE&) { return 3; }
template <class R>
inline void get(const VECTOR_TYPE& v, R* a) {
  for (int c = 0; c < 3; c++) a[c] = R(v[c]);
}
template <class R>
inline void set(VECTOR_TYPE& v, const R* a) {
  v = SetData(REAL_TYPE(a[0]), REAL_TYPE(a[1]), REAL_TYPE(a[2]));
}
#endif

template <class Data, class R>
inline int pack(const std::vector<Data>& v, std::vector<R>& out) {
  const int k = v.empty() ? 1 : channels(v[0]);
  out.resize(v.size() * size_t(k));
  for (size_t i = 0; i < v.size(); i++) get<R>(v[i], &out[i * k]);
  return k;
}
template <class Data, class R>
inline void unpack(const std::vector<R>& a, int k, std::vector<Data>& v) {
  for (size_t i = 0; i < v.size(); i++) set<R>(v[i], &a[i * k]);
}

inline void vcycle(gdtp_system* s, std::vector<float>& x, const std::vector<float>& rhs, int k, int& code) {
  code = gdtp_vcycle(s, x.data(), rhs.data(), k);
}
inline void vcycle(gdtp_system* s, std::vector<double>& x, const std::vector<double>& rhs, int k, int& code) {
  code = gdtp_vcycle64(s, x.data(), rhs.data(), k);
}

// InitializeHierarchy (HierarchyConstruction.inl:799-800): the reference's set-up,
// and the mesh recorded for the device system.
inline int InitializeHierarchy(TexturedMesh& mesh, const int width, const int height, const int levels,
                               std::vector<TextureNodeInfo>& textureNodes, std::vector<CellIndex>& cellNodes, HierarchicalSystem& hierarchy,
                               std::vector<AtlasChart>& atlasCharts, const MultigridBlockInfo& multigridBlockInfo, bool verbose = false,
                               bool detailVerbose = false, bool computeProlongation = false) {
  MeshRecord r;
  r.width = width;
  r.height = height;
  r.levels = levels;
  r.vertices.reserve(3 * mesh.vertices.size());
  for (const auto& p : mesh.vertices)
    for (int c = 0; c < 3; c++) r.vertices.push_back(p[c]);
  r.triangles.reserve(3 * mesh.triangles.size());
  for (const auto& t : mesh.triangles)
    for (int c = 0; c < 3; c++) r.triangles.push_back(int32_t(t[c]));
  r.uv.reserve(2 * mesh.textureCoordinates.size());
  for (const auto& q : mesh.textureCoordinates)
    for (int c = 0; c < 2; c++) r.uv.push_back(q[c]);
  const int result = ::InitializeHierarchy(mesh, width, height, levels, textureNodes, cellNodes, hierarchy, atlasCharts, multigridBlockInfo,
                                           verbose, detailVerbose, computeProlongation);
  if (result) {
    MeshRecord& old = meshes()[&hierarchy];
    if (old.hierarchy) gdtp_hierarchy_free(old.hierarchy);
    old = r;
  }
  return result;
}
// the reference's other InitializeHierarchy (from an atlas mesh) unchanged
template <class... A>
inline int InitializeHierarchy(const std::vector<int>& oppositeHalfEdge, A&&... a) {
  return ::InitializeHierarchy(oppositeHalfEdge, std::forward<A>(a)...);
}

}  // namespace gdtp_dropin

// UpdateLinearSystem (UpdateCoefficients.inl:463-469) with the app's Real:
// screenWeight M + stiffnessWeight S and its Galerkin hierarchy on the device
// (built on the first call of this operator).
template <class CoarseSolverType, class BoundarySolverType, class DirectSolverType>
int UpdateLinearSystem(double stiffnessWeight, double screenWeight, const HierarchicalSystem& hierarchy,
                       std::vector<MultigridLevelCoefficients<REAL_TYPE>>& multigridCoefficients,
                       const std::vector<double>& deepMassCoefficients, const std::vector<double>& deepStiffnessCoefficients,
                       const SparseMatrix<double, int>& boundaryBoundaryMassMatrix, const SparseMatrix<double, int>& boundaryBoundaryStiffnessMatrix,
                       const SparseMatrix<double, int>& boundaryDeepMassMatrix, const SparseMatrix<double, int>& boundaryDeepStiffnessMatrix,
                       CoarseSolverType& coarseSolver, std::vector<BoundarySolverType>& boundarySolver, DirectSolverType& fineSolver,
                       const SparseMatrix<double, int>& fineSystemMatrix, bool detailVerbose = false, bool initSolvers = true,
                       bool updateFineSolver = false) {
  auto it = gdtp_dropin::operators().find(&deepMassCoefficients);
  if (it == gdtp_dropin::operators().end()) {
    std::printf("ERROR : gdtp drop-in: UpdateLinearSystem before InitializeMassAndStiffness of this operator\n");
    return 0;
  }
  gdtp_system* s = gdtp_dropin::system_of(it->second);
  if (!s || !gdtp_dropin::ok(gdtp_system_update(s, stiffnessWeight, screenWeight), "gdtp_system_update")) return 0;
  gdtp_dropin::coefficient_systems()[&multigridCoefficients] = s;
  multigridCoefficients.resize(hierarchy.gridAtlases.size());
  if (updateFineSolver) {  // the --useDirectSolver factorisation, as the reference does it
    if (initSolvers) fineSolver.init(fineSystemMatrix);
    fineSolver.update(fineSystemMatrix);
  }
  return 1;
}

// VCycle (IterativeSolvers.inl:1211-1216) with the app's Real: one V-cycle of
// the operator these coefficients name, on the device; variables[0].rhs and .x
// are uploaded at entry and x downloaded at exit.
template <class DataType, class BoundarySolver, class CoarseSolver>
int VCycle(std::vector<MultigridLevelVariables<DataType>>& variables, const std::vector<MultigridLevelCoefficients<REAL_TYPE>>& coefficients,
           const std::vector<MultigridLevelIndices<REAL_TYPE>>& indices, std::vector<BoundarySolver>& boundarySolvers,
           CoarseSolver& coarseSolver, bool verbose, bool detailVerbose) {
  auto it = gdtp_dropin::coefficient_systems().find(&coefficients);
  if (it == gdtp_dropin::coefficient_systems().end() || variables.empty()) {
    std::printf("ERROR : gdtp drop-in: VCycle on coefficients that no UpdateLinearSystem produced\n");
    return 0;
  }
  std::vector<REAL_TYPE> x, rhs;
  const int k = gdtp_dropin::pack(variables[0].x, x);
  gdtp_dropin::pack(variables[0].rhs, rhs);
  int code = GDTP_OK;
  gdtp_dropin::vcycle(it->second, x, rhs, k, code);
  if (!gdtp_dropin::ok(code, "gdtp V-cycle")) return 0;
  gdtp_dropin::unpack(x, k, variables[0].x);
  return 1;
}

// MultiplyBySystemMatrix_NoReciprocals (IterativeSolvers.inl:881) on FP64
// coefficients: a recorded mass or stiffness operator is applied on the device.
template <class Data>
int MultiplyBySystemMatrix_NoReciprocals(const std::vector<double>& deepCoefficients, const SparseMatrix<double, int>& boundaryDeepMatrix,
                                         const SparseMatrix<double, int>& boundaryBoundaryMatrix, const std::vector<int>& boundaryGlobalIndex,
                                         const std::vector<RasterLine>& rasterLines, const std::vector<Data>& in, std::vector<Data>& out,
                                         bool verbose = false) {
  auto d = gdtp_dropin::deep_arrays().find(&deepCoefficients);
  if (d == gdtp_dropin::deep_arrays().end())  // not an operator of this library: the reference's own product
    return MultiplyBySystemMatrix_NoReciprocals<double, Data>(deepCoefficients, boundaryDeepMatrix, boundaryBoundaryMatrix,
                                                              boundaryGlobalIndex, rasterLines, in, out, verbose);
  gdtp_system* s = gdtp_dropin::system_of(gdtp_dropin::operators()[d->second.first]);
  if (!s) return 0;
  std::vector<double> x, y;
  const int k = gdtp_dropin::pack(in, x);
  y.resize(x.size());
  if (!gdtp_dropin::ok(gdtp_apply(s, d->second.second, x.data(), y.data(), k), "gdtp_apply")) return 0;
  out.resize(in.size());
  gdtp_dropin::unpack(y, k, out);
  return 1;
}

// the apps' calls of InitializeHierarchy go to the recording wrapper
// (InitializeMassAndStiffness: gdtp_dropin_assembly.inl, after its definition)
#define InitializeHierarchy gdtp_dropin::InitializeHierarchy
