// Oracle harness: drives the UNMODIFIED reference solve path (compiled from the
// reference's own headers, never copied) and dumps every structure the B200
// implementation must reproduce.  Test infrastructure only: nothing in the
// product links or runs this program.
//
// Call sequence mirrors the TextureFiltering app (TextureFiltering/TextureFiltering.cpp:581-718):
//   InitializeHierarchy            include/Src/HierarchyConstruction.inl:799
//   InitializeBoundaryProlongationData include/Src/BoundaryQuadraticElements.inl:775
//   InitializeMetric (embedding)   include/Src/Metric.inl:448
//   InitializeAnisotropicMetric    include/Src/Metric.inl:468  (with a .vf tangent field, as the LIC app)
//   InitializeMassAndStiffness     include/Src/MassAndStiffness.h:490
//   FullMatrixConstruction         include/Src/UpdateCoefficients.inl:137
//   UpdateLinearSystem             include/Src/UpdateCoefficients.inl:463
//   MultiplyBySystemMatrix_NoReciprocals include/Src/IterativeSolvers.inl:881
//   VCycle                         include/Src/IterativeSolvers.inl:1211
//   solve(EigenCholeskySolver3)    include/Src/Solver.h:191   (the --useDirectSolver FP64 ground truth)
// Mode "geodesic" follows the Geodesics app instead (Geodesics/Geodesics.cpp:257-300, 552-760):
//   (M + stiffness S) u = delta_source, InitializeGridAtladInteriorCellLines /
//   InitializeNormalizedVectorFieldIntegration (VectorFieldIntergration.inl:68-73, 428-437),
//   boundary prolongation, IntergrateNormalizedVectorFieldFromSamples (:453-582), boundary
//   restriction, (1e-6 M + S) d = rhs with exact solves, d shifted to 0 at the source.
//
// Usage: gdtp_ref <mesh.gdm> <out.gdd> [levels] [stiffness] [sharpness] [vcycles] [mode] [tol] [field.vf] [source]
//   mode "dump": everything (small meshes); "solve": counts + rhs + exact solution + V-cycle timing;
//   "time": V-cycles to tol only (no dumps, no direct solve); "vsolve": V-cycles to tol (the FP64
//   reference solution where a direct solve is too large) plus the FP64 operator fine/A;
//   "brush": the sharpening brush's modulated stiffness for a seeded cell mask (brush/mask, brush/out).
//   field.vf may instead be a ".pm" file: the parameter metric itself (nt x 4 float64,
//   g(0,0) g(0,1) g(1,0) g(1,1) per mesh triangle), which InitializeMassAndStiffness then uses.
//   The RHS is  M f + stiffness*sharpness * S f  and the operator  M + stiffness*S.
//   With field.vf (the reference's vector file: int32 count + per-triangle Point2D<double> in the
//   triangle's edge basis, read by its own ReadVector) M and S use the anisotropic metric instead.
#ifndef USE_FLOAT
#define USE_FLOAT 0
#endif
#define PNG_INCLUDED 1
void PNGWriteColor(const char*, const unsigned char*, int, int) {}
unsigned char* PNGReadColor(const char*, int&, int&) { return nullptr; }

#include <Src/VectorPrecisionType.inl>
#include <Misha/CmdLineParser.h>
#include <Src/SimpleMesh.h>
#include <Src/Basis.h>
#include <Misha/FEM.h>
#include <Src/Solver.h>
#include <Src/Hierarchy.h>
#include <Src/MassAndStiffness.h>
#include <Src/VectorIO.h>
#include <Src/VectorFieldIntergration.inl>
#include <Src/InteriorTexelToCellLines.inl>
#include <algorithm>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>
#include <omp.h>

// ---------------------------------------------------------------------------
// named-array container ("GDTPDMP1"): name, dtype code, ndim, dims, raw bytes
// dtype codes: 1=int32 2=float64 3=float32 4=int64
// ---------------------------------------------------------------------------
struct Dump {
  FILE* f = nullptr;
  explicit Dump(const char* path) {
    f = fopen(path, "wb");
    if (!f) { fprintf(stderr, "cannot open %s\n", path); exit(2); }
    fwrite("GDTPDMP1", 1, 8, f);
  }
  ~Dump() { if (f) fclose(f); }
  void put(const std::string& name, int code, const std::vector<int64_t>& dims, const void* data, size_t bytes) {
    uint32_t n = (uint32_t)name.size();
    fwrite(&n, 4, 1, f);
    fwrite(name.data(), 1, n, f);
    uint8_t c = (uint8_t)code;
    fwrite(&c, 1, 1, f);
    uint32_t nd = (uint32_t)dims.size();
    fwrite(&nd, 4, 1, f);
    fwrite(dims.data(), 8, nd, f);
    if (bytes) fwrite(data, 1, bytes, f);
  }
  void i32(const std::string& name, const std::vector<int>& v, int64_t cols = 1) {
    put(name, 1, cols == 1 ? std::vector<int64_t>{(int64_t)v.size()} : std::vector<int64_t>{(int64_t)v.size() / cols, cols}, v.data(), v.size() * 4);
  }
  void f64(const std::string& name, const std::vector<double>& v, int64_t cols = 1) {
    put(name, 2, cols == 1 ? std::vector<int64_t>{(int64_t)v.size()} : std::vector<int64_t>{(int64_t)v.size() / cols, cols}, v.data(), v.size() * 8);
  }
  template <class T>
  void csr(const std::string& name, const SparseMatrix<T, int>& M) {
    std::vector<int> ptr(M.rows + 1, 0), col;
    std::vector<double> val;
    for (size_t i = 0; i < M.rows; i++) {
      ptr[i + 1] = ptr[i] + (int)M.RowSize(i);
      for (size_t j = 0; j < M.RowSize(i); j++) { col.push_back(M[i][j].N); val.push_back((double)M[i][j].Value); }
    }
    i32(name + "/ptr", ptr);
    i32(name + "/col", col);
    f64(name + "/val", val);
  }
};

static bool ReadGDM(const char* path, TexturedMesh& mesh) {
  FILE* f = fopen(path, "rb");
  if (!f) return false;
  char magic[8];
  if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "GDTPMSH1", 8)) { fclose(f); return false; }
  int64_t hdr[5];
  if (fread(hdr, 8, 5, f) != 5) { fclose(f); return false; }
  int64_t nv = hdr[0], nt = hdr[1], w = hdr[2], h = hdr[3], c = hdr[4];
  std::vector<double> v(nv * 3), uv(nt * 6);
  std::vector<int> t(nt * 3);
  std::vector<float> tex(w * h * c);
  size_t ok = fread(v.data(), 8, v.size(), f) + fread(t.data(), 4, t.size(), f) + fread(uv.data(), 8, uv.size(), f) +
              fread(tex.data(), 4, tex.size(), f);
  fclose(f);
  if (ok != v.size() + t.size() + uv.size() + tex.size()) return false;
  mesh.vertices.resize(nv);
  for (int64_t i = 0; i < nv; i++) mesh.vertices[i] = Point3D<double>(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
  mesh.triangles.resize(nt);
  for (int64_t i = 0; i < nt; i++) mesh.triangles[i] = TriangleIndex(t[3 * i], t[3 * i + 1], t[3 * i + 2]);
  mesh.textureCoordinates.resize(nt * 3);
  for (int64_t i = 0; i < nt * 3; i++) mesh.textureCoordinates[i] = Point2D<double>(uv[2 * i], uv[2 * i + 1]);
  mesh.texture.resize((int)w, (int)h);
  for (int64_t j = 0; j < h; j++)
    for (int64_t i = 0; i < w; i++) {
      const float* p = &tex[(j * w + i) * c];
      mesh.texture(i, j) = Point3D<float>(p[0], c > 1 ? p[1] : p[0], c > 2 ? p[2] : p[0]);
    }
  return true;
}

typedef VECTOR_TYPE Vec;
typedef REAL_TYPE Real;

static double ResidualNorm(const std::vector<MultigridLevelCoefficients<Real>>&, const std::vector<double>& deepA,
                           const SparseMatrix<double, int>& BD, const SparseMatrix<double, int>& BB,
                           const GridAtlas& atlas, const std::vector<Vec>& x, const std::vector<Vec>& b,
                           double bnorm2[3], double rnorm2[3]) {
  std::vector<Vec> Ax(x.size());
  MultiplyBySystemMatrix_NoReciprocals(deepA, BD, BB, atlas.boundaryGlobalIndex, atlas.rasterLines, x, Ax);
  double worst = 0;
  for (int c = 0; c < 3; c++) { bnorm2[c] = 0; rnorm2[c] = 0; }
  for (size_t i = 0; i < x.size(); i++)
    for (int c = 0; c < 3; c++) {
      double r = (double)b[i][c] - (double)Ax[i][c];
      rnorm2[c] += r * r;
      bnorm2[c] += (double)b[i][c] * (double)b[i][c];
    }
  for (int c = 0; c < 3; c++) worst = std::max(worst, sqrt(rnorm2[c] / std::max(bnorm2[c], 1e-300)));
  return worst;
}

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s mesh.gdm out.gdd [levels] [stiffness] [sharpness] [vcycles] [dump|solve]\n", argv[0]);
    return 2;
  }
  const int levels = argc > 3 ? atoi(argv[3]) : 4;
  const double stiffnessWeight = argc > 4 ? atof(argv[4]) : 1e-3;
  const double sharpnessWeight = argc > 5 ? atof(argv[5]) : 2.0;
  const int vcycles = argc > 6 ? atoi(argv[6]) : 12;
  const std::string mode = argc > 7 ? argv[7] : "dump";
  const bool full = (mode == "dump");
  // V-cycles to `tol` (argv[8]) only: no dumps, no direct solve ("vsolve" also dumps fine/A)
  const bool timeOnly = (mode == "time" || mode == "vsolve");
  const double tol = argc > 8 ? atof(argv[8]) : 1e-6;

  TexturedMesh mesh;
  if (!ReadGDM(argv[1], mesh)) { fprintf(stderr, "cannot read %s\n", argv[1]); return 2; }
  const int width = mesh.texture.width(), height = mesh.texture.height();
  Dump out(argv[2]);

  auto T0 = std::chrono::steady_clock::now();
  auto secs = [](std::chrono::steady_clock::time_point a) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
  };

  // ---------------- hierarchy -------------------------------------------------------------
  MultigridBlockInfo blockInfo(128, 16, 2, 0, 0);  // app defaults TextureFiltering.cpp:25-28
  std::vector<TextureNodeInfo> textureNodes;
  std::vector<CellIndex> cellIndices;
  HierarchicalSystem hierarchy;
  std::vector<AtlasChart> atlasCharts;
  if (!InitializeHierarchy(mesh, width, height, levels, textureNodes, cellIndices, hierarchy, atlasCharts, blockInfo, false, false)) {
    fprintf(stderr, "InitializeHierarchy failed\n");
    return 3;
  }
  double tHierarchy = secs(T0);
  auto T1 = std::chrono::steady_clock::now();
  BoundaryProlongationData boundaryProlongation;
  if (!InitializeBoundaryProlongationData(hierarchy.gridAtlases[0], boundaryProlongation)) return 3;
  std::vector<std::vector<SquareMatrix<double, 2>>> parameterMetric;
  const char* vfPath = argc > 9 ? argv[9] : nullptr;
  const std::string vfName = vfPath ? vfPath : "";
  if (vfName.size() > 3 && vfName.compare(vfName.size() - 3, 3, ".pm") == 0) {
    std::vector<double> pm(4 * mesh.triangles.size());
    FILE* fp = fopen(vfPath, "rb");
    const bool okRead = fp && fread(pm.data(), sizeof(double), pm.size(), fp) == pm.size();
    if (fp) fclose(fp);
    if (!okRead) { fprintf(stderr, "bad parameter metric %s\n", vfPath); return 2; }
    parameterMetric.resize(atlasCharts.size());
    for (size_t c = 0; c < atlasCharts.size(); c++) {
      parameterMetric[c].resize(atlasCharts[c].meshTriangleIndices.size());
      for (size_t k = 0; k < atlasCharts[c].meshTriangleIndices.size(); k++) {
        const int t = atlasCharts[c].meshTriangleIndices[k];
        SquareMatrix<double, 2>& g = parameterMetric[c][k];
        g(0, 0) = pm[4 * t]; g(0, 1) = pm[4 * t + 1]; g(1, 0) = pm[4 * t + 2]; g(1, 1) = pm[4 * t + 3];
      }
    }
  } else if (vfPath && *vfPath) {
    std::vector<Point2D<double>> vf;
    if (!ReadVector(vf, vfPath) || vf.size() != mesh.triangles.size()) { fprintf(stderr, "bad vector field %s\n", vfPath); return 2; }
    if (!InitializeAnisotropicMetric(mesh, atlasCharts, parameterMetric, vf, false)) return 3;
  } else if (!InitializeMetric(mesh, EMBEDDING_METRIC, atlasCharts, parameterMetric)) {
    return 3;
  }
  if (full) {  // parameter metric in mesh triangle order, entries g(0,0) g(0,1) g(1,0) g(1,1)
    std::vector<double> pm(4 * mesh.triangles.size(), 0.0);
    for (size_t c = 0; c < atlasCharts.size(); c++)
      for (size_t k = 0; k < atlasCharts[c].meshTriangleIndices.size(); k++) {
        const int t = atlasCharts[c].meshTriangleIndices[k];
        const SquareMatrix<double, 2>& g = parameterMetric[c][k];
        pm[4 * t] = g(0, 0); pm[4 * t + 1] = g(0, 1); pm[4 * t + 2] = g(1, 0); pm[4 * t + 3] = g(1, 1);
      }
    out.f64("metric/parameter", pm, 4);
  }

  const GridAtlas& fine = hierarchy.gridAtlases[0];
  std::vector<Point3D<double>> inputSignal(textureNodes.size());
  std::vector<Vec> f0(textureNodes.size());
  for (size_t i = 0; i < textureNodes.size(); i++) {
    Point3D<float> t = mesh.texture(textureNodes[i].ci, textureNodes[i].cj);
    inputSignal[i] = Point3D<double>(t[0], t[1], t[2]);
    f0[i] = SetData(t[0], t[1], t[2]);
  }

  std::vector<double> deepMass, deepStiffness, texelToCell;
  SparseMatrix<double, int> bbM, bbS, bdM, bdS, cellRHS[3];
  const bool brush = (mode == "brush");  // the sharpening brush's cell-based stiffness (TextureFiltering.cpp:569)
  if (!InitializeMassAndStiffness(deepMass, deepStiffness, bbM, bbS, bdM, bdS, hierarchy, parameterMetric, atlasCharts,
                                  boundaryProlongation, brush, inputSignal, texelToCell, cellRHS)) {
    fprintf(stderr, "InitializeMassAndStiffness failed\n");
    return 3;
  }
  double tAssembly = secs(T1);
  if (brush) {
#if USE_FLOAT  // the brush's cell matrices are FP64 (SparseMatrix<double>); the FP32 build has no brush mode
    fprintf(stderr, "brush mode needs the FP64 build (gdtp_ref)\n");
    return 2;
#else
    // CellStiffnessToTexelStiffness (IterativeSolvers.inl:1170-1208) for a seeded
    // cell mask m_c = ((c * 2654435761) mod 2^32 mod 1000) / 1000, in FP64 (Vec4d),
    // the texel-to-cell coefficients converted as the app does (TextureFiltering.cpp:641-642)
    std::vector<InteriorTexelToCellLine> lines;
    InitializeInteriorTexelToCellLines(lines, fine);
    std::vector<Vec> coeffs(4 * size_t(fine.numDeepTexels));
    for (size_t i = 0; i < coeffs.size(); i++) coeffs[i] = SetData(texelToCell[3 * i], texelToCell[3 * i + 1], texelToCell[3 * i + 2]);
    std::vector<Real> mask(fine.numCells), boundaryValues[3];
    for (int c = 0; c < fine.numCells; c++) mask[c] = Real(double((uint32_t(c) * 2654435761u) % 1000u) / 1000.0);
    for (int c = 0; c < 3; c++) boundaryValues[c].resize(fine.boundaryGlobalIndex.size());
    std::vector<Vec> modulated(fine.numTexels, ZeroData());
    auto flat = [&] {
      std::vector<double> o(3 * size_t(fine.numTexels));
      for (size_t i = 0; i < modulated.size(); i++)
        for (int c = 0; c < 3; c++) o[3 * i + c] = double(modulated[i][c]);
      return o;
    };
    CellStiffnessToTexelStiffness(mask, lines, coeffs, cellRHS, boundaryValues, fine.boundaryGlobalIndex, modulated);
    out.f64("brush/mask", std::vector<double>(mask.begin(), mask.end()));
    out.f64("brush/out", flat(), 3);
    std::vector<Real> ones(fine.numCells, Real(1));  // a uniform brush: the stiffness applied to the signal
    CellStiffnessToTexelStiffness(ones, lines, coeffs, cellRHS, boundaryValues, fine.boundaryGlobalIndex, modulated);
    out.f64("brush/out_ones", flat(), 3);
    std::vector<Vec> sf(fine.numTexels);
    MultiplyBySystemMatrix_NoReciprocals(deepStiffness, bdS, bbS, fine.boundaryGlobalIndex, fine.rasterLines, f0, sf);
    out.f64("brush/stiffness_f", [&] {
      std::vector<double> o(3 * sf.size());
      for (size_t i = 0; i < sf.size(); i++)
        for (int c = 0; c < 3; c++) o[3 * i + c] = double(sf[i][c]);
      return o;
    }(), 3);
    out.f64("solve/f", [&] {
      std::vector<double> f(3 * inputSignal.size());
      for (size_t i = 0; i < inputSignal.size(); i++)
        for (int c = 0; c < 3; c++) f[3 * i + c] = inputSignal[i][c];
      return f;
    }(), 3);
    out.i32("L0/counts", {fine.numTexels, fine.numDeepTexels, (int)fine.boundaryGlobalIndex.size(), fine.numCells});
    fprintf(stderr, "ok: brush, %d texels, %d cells\n", fine.numTexels, fine.numCells);
    return 0;
#endif
  }

  // ---------------- system ---------------------------------------------------------------
  auto T2 = std::chrono::steady_clock::now();
  SparseMatrix<double, int> mass, stiffness, A;
  FullMatrixConstruction(fine, deepMass, bbM, bdM, mass);
  FullMatrixConstruction(fine, deepStiffness, bbS, bdS, stiffness);
  A = mass + stiffness * stiffnessWeight;

  std::vector<MultigridLevelCoefficients<Real>> coeffs;
  EigenCholeskySolver3<Real> coarseSolver;
  std::vector<EigenCholeskySolver3<Real>> boundarySolvers;
  EigenCholeskySolver3<Real> directSolver;
  if (!UpdateLinearSystem(stiffnessWeight, 1.0, hierarchy, coeffs, deepMass, deepStiffness, bbM, bbS, bdM, bdS, coarseSolver,
                          boundarySolvers, directSolver, A, false, true, false)) {
    fprintf(stderr, "UpdateLinearSystem failed\n");
    return 3;
  }
  double tSystem = secs(T2);

  std::vector<Vec> mf(f0.size()), sf(f0.size()), rhs(f0.size());
  MultiplyBySystemMatrix_NoReciprocals(deepMass, bdM, bbM, fine.boundaryGlobalIndex, fine.rasterLines, f0, mf);
  MultiplyBySystemMatrix_NoReciprocals(deepStiffness, bdS, bbS, fine.boundaryGlobalIndex, fine.rasterLines, f0, sf);
  for (size_t i = 0; i < f0.size(); i++) rhs[i] = mf[i] + sf[i] * (Real)(sharpnessWeight * stiffnessWeight);

  // combined FP64 operator (no reciprocals) for residual checks
  std::vector<double> deepA(deepMass.size());
  for (size_t i = 0; i < deepA.size(); i++) deepA[i] = deepMass[i] + stiffnessWeight * deepStiffness[i];
  SparseMatrix<double, int> BBA = bbM + bbS * stiffnessWeight;
  SparseMatrix<double, int> BDA = bdM + bdS * stiffnessWeight;

  // ---------------- FP64 direct solve (the accuracy oracle) ------------------------------
  auto T3 = std::chrono::steady_clock::now();
  std::vector<Vec> exact(f0.size(), ZeroData());
  if (!timeOnly) {
#if !USE_FLOAT  // the FP32 build only reproduces the shipped V-cycle; ground truth needs FP64
  directSolver.init(A);
  directSolver.update(A);
  solve(directSolver, exact, rhs);
#endif
  }
  double tDirect = secs(T3);

  // ---------------- V-cycles ------------------------------------------------------------
  std::vector<MultigridLevelIndices<Real>> indices(levels);
  for (int l = 0; l < levels; l++) {
    const GridAtlas& g = hierarchy.gridAtlases[l];
    indices[l].threadTasks = g.threadTasks;
    indices[l].boundaryGlobalIndex = g.boundaryGlobalIndex;
    indices[l].segmentedLines = g.segmentedLines;
    indices[l].rasterLines = g.rasterLines;
    indices[l].restrictionLines = g.restrictionLines;
    indices[l].prolongationLines = g.prolongationLines;
    if (l < levels - 1) indices[l].boundaryRestriction = hierarchy.boundaryRestriction[l];
  }
  std::vector<MultigridLevelVariables<Vec>> vars(levels);
  for (int l = 0; l < levels; l++) {
    const GridAtlas& g = hierarchy.gridAtlases[l];
    vars[l].x.assign(g.numTexels, ZeroData());
    vars[l].rhs.assign(g.numTexels, ZeroData());
    vars[l].residual.assign(g.numTexels, ZeroData());
    vars[l].boundary_rhs.assign(g.boundaryGlobalIndex.size(), ZeroData());
    vars[l].boundary_value.assign(g.boundaryGlobalIndex.size(), ZeroData());
    vars[l].variable_boundary_value.assign(g.boundaryGlobalIndex.size(), ZeroData());
  }
  for (size_t i = 0; i < f0.size(); i++) vars[0].rhs[i] = rhs[i];
  std::vector<double> history, cycleTimes;
  double bn[3], rn[3];
  history.push_back(ResidualNorm(coeffs, deepA, BDA, BBA, fine, vars[0].x, rhs, bn, rn));
  std::vector<double> firstIterate;
  for (int it = 0; it < vcycles; it++) {
    if (timeOnly && history.back() <= tol) break;
    auto Tc = std::chrono::steady_clock::now();
    VCycle(vars, coeffs, indices, boundarySolvers, coarseSolver, false, false);
    cycleTimes.push_back(secs(Tc));
    history.push_back(ResidualNorm(coeffs, deepA, BDA, BBA, fine, vars[0].x, rhs, bn, rn));
    if (it == 0 && full)
      for (size_t i = 0; i < f0.size(); i++)
        for (int c = 0; c < 3; c++) firstIterate.push_back((double)vars[0].x[i][c]);
  }

  // ---------------- heat-method geodesics (mode "geodesic", FP64 build) -------------------
#if !USE_FLOAT
  if (mode == "geodesic") {
    const int n = (int)textureNodes.size();
    const int src = argc > 10 ? atoi(argv[10]) : n / 3;
    EigenCholeskySolver1<double> smoothSolver, distSolver;
    smoothSolver.init(A);
    smoothSolver.update(A);
    std::vector<double> delta(n, 0.0), u(n, 0.0), d(n, 0.0);
    delta[src] = 1.0;
    solve(smoothSolver, u, delta);
    std::vector<InteriorCellLine> lines;
    std::vector<std::pair<int, int>> lineIndex;
    InitializeGridAtladInteriorCellLines(atlasCharts, fine.gridCharts, lines, lineIndex);
    std::vector<std::vector<CellLineSampleInfo<double>>> cellSamples(lines.size());
    std::vector<HexagonalSampleInfo<double>> hexSamples;
    if (!InitializeNormalizedVectorFieldIntegration<double>(parameterMetric, atlasCharts, fine.gridCharts, lineIndex,
                                                            boundaryProlongation.fineBoundaryIndex, cellSamples, hexSamples)) {
      fprintf(stderr, "InitializeNormalizedVectorFieldIntegration failed\n");
      return 3;
    }
    for (auto& v : cellSamples) std::sort(v.begin(), v.end(), CellLineSampleCompare<double>);
    const std::vector<int>& bgi = fine.boundaryGlobalIndex;
    const int nf = boundaryProlongation.numFineBoundarNodes;
    std::vector<double> cbv(bgi.size()), cbr(bgi.size()), fbv(nf), fbr(nf), grhs(n, 0.0);
    for (size_t i = 0; i < bgi.size(); i++) cbv[i] = u[bgi[i]];
    boundaryProlongation.coarseBoundaryFineBoundaryProlongation.Multiply(&cbv[0], &fbv[0]);
    omp_set_num_threads(1);  // its line-parallel scatter races at range boundaries
    IntergrateNormalizedVectorFieldFromSamples<double>(double(width), double(height), lines, cellSamples, hexSamples, u, grhs, fbv, fbr);
    std::vector<double> interiorRhs = grhs;
    boundaryProlongation.fineBoundaryCoarseBoundaryRestriction.Multiply(&fbr[0], &cbr[0]);
    for (size_t i = 0; i < bgi.size(); i++) grhs[bgi[i]] += cbr[i];
    SparseMatrix<double, int> G = mass * 1e-6 + stiffness;
    distSolver.init(G);
    distSolver.update(G);
    solve(distSolver, d, grhs);
    const double d0 = d[src];
    for (auto& v : d) v -= d0;
    size_t nCellSamples = 0;
    for (auto& v : cellSamples) nCellSamples += v.size();
    // samples: hex {pos(2), tensor(4: (0,0) (0,1) (1,0) (1,1)), v(12), fine nodes(6)}; cell {line, cellOffset, pos, tensor, v(8)}
    std::vector<double> hx, cl;
    for (const auto& h : hexSamples) {
      hx.insert(hx.end(), {h.pos[0], h.pos[1], h.tensor(0, 0), h.tensor(0, 1), h.tensor(1, 0), h.tensor(1, 1)});
      for (int k = 0; k < 6; k++) { hx.push_back(h.v[k][0]); hx.push_back(h.v[k][1]); }
      for (int k = 0; k < 6; k++) hx.push_back(h.fineNodes[k]);
    }
    for (size_t r = 0; r < cellSamples.size(); r++)
      for (const auto& c : cellSamples[r]) {
        cl.insert(cl.end(), {double(r), double(c.cellOffset), c.pos[0], c.pos[1], c.tensor(0, 0), c.tensor(0, 1), c.tensor(1, 0), c.tensor(1, 1)});
        for (int k = 0; k < 4; k++) { cl.push_back(c.v[k][0]); cl.push_back(c.v[k][1]); }
      }
    out.f64("geo/hex_samples", hx, 24);
    out.csr("geo/prolongation", boundaryProlongation.coarseBoundaryFineBoundaryProlongation);
    out.f64("geo/cell_samples", cl, 16);
    std::vector<int> li;
    for (const auto& l : lines) li.insert(li.end(), {l.prevLineIndex, l.nextLineIndex, l.length});
    out.i32("geo/cell_lines", li, 3);
    out.i32("geo/source", {src, (int)lines.size(), (int)nCellSamples, (int)hexSamples.size(), nf});
    out.f64("geo/weights", {stiffnessWeight, 1e-6});
    out.f64("geo/u", u);
    out.f64("geo/fine_boundary_u", fbv);
    out.f64("geo/rhs_interior", interiorRhs);
    out.f64("geo/fine_boundary_rhs", fbr);
    out.f64("geo/rhs", grhs);
    out.f64("geo/dist", d);
  }
#endif

  // ---------------- output --------------------------------------------------------------
  out.i32("meta/size", {width, height, levels, (int)atlasCharts.size(), omp_get_max_threads()});
  out.f64("meta/weights", {stiffnessWeight, sharpnessWeight});
  out.f64("time/setup", {tHierarchy, tAssembly, tSystem, tDirect});
  out.f64("time/vcycle", cycleTimes);
  out.f64("vcycle/history", history);
  auto vec3 = [&](const std::vector<Vec>& v) {
    std::vector<double> o(v.size() * 3);
    for (size_t i = 0; i < v.size(); i++)
      for (int c = 0; c < 3; c++) o[3 * i + c] = (double)v[i][c];
    return o;
  };
  out.f64("solve/f", vec3(f0), 3);
  out.f64("solve/rhs", vec3(rhs), 3);
  out.f64("solve/exact", vec3(exact), 3);
  out.f64("solve/vcycle_x", vec3(vars[0].x), 3);
  if (mode == "vsolve") out.csr("fine/A", A);
  if (full) out.f64("solve/vcycle_x1", firstIterate, 3);

  for (int l = 0; l < levels; l++) {
    const GridAtlas& g = hierarchy.gridAtlases[l];
    std::string p = "L" + std::to_string(l) + "/";
    out.i32(p + "counts", {g.numTexels, g.numDeepTexels, g.numBoundaryTexels, g.numCells, g.numBoundaryCells, g.numInteriorCells,
                           g.numInteriorTexels});
    if (!full) continue;
    std::vector<int> ni;
    for (auto& n : g.nodeInfo) { ni.push_back(n.chartId); ni.push_back(n.ci); ni.push_back(n.cj); ni.push_back(n.nodeType); }
    out.i32(p + "nodeinfo", ni, 4);
    out.i32(p + "boundaryGlobalIndex", g.boundaryGlobalIndex);
    out.i32(p + "deepGlobalIndex", g.deepGlobalIndex);
    out.i32(p + "boundaryAndDeepIndex", g.boundaryAndDeepIndex);
    std::vector<int> rl;
    for (auto& r : g.rasterLines) { rl.insert(rl.end(), {r.lineStartIndex, r.lineEndIndex, r.prevLineIndex, r.nextLineIndex, r.coeffStartIndex}); }
    out.i32(p + "rasterLines", rl, 5);
    rl.clear();
    for (auto& r : g.restrictionLines) { rl.insert(rl.end(), {r.lineStartIndex, r.lineEndIndex, r.prevLineIndex, r.nextLineIndex, r.coeffStartIndex}); }
    out.i32(p + "restrictionLines", rl, 5);
    rl.clear();
    for (auto& r : g.deepLines) { rl.insert(rl.end(), {r.coarseLineStartIndex, r.coarseLineEndIndex, r.finePrevLineIndex, r.fineCurrentLineIndex, r.fineNextLineIndex}); }
    out.i32(p + "deepLines", rl, 5);
    rl.clear();
    for (auto& r : g.prolongationLines) { rl.insert(rl.end(), {r.startIndex, r.length, r.centerLineIndex, r.prevLineIndex, r.nextLineIndex, (int)r.alignedStart}); }
    out.i32(p + "prolongationLines", rl, 6);
    std::vector<int> ci;
    std::vector<double> cd;
    std::vector<int> ctype, ntype;
    for (auto& c : g.gridCharts) {
      ci.insert(ci.end(), {c.cornerCoords[0], c.cornerCoords[1], c.centerOffset[0], c.centerOffset[1], c.width, c.height,
                           c.globalIndexTexelOffset, c.globalTexelDeepOffset, c.globalTexelBoundaryOffset, c.globalIndexCellOffset,
                           c.numInteriorCells, c.numBoundaryCells});
      cd.insert(cd.end(), {c.corner[0], c.corner[1], c.cellSizeW, c.cellSizeH});
      for (int k = 0; k < c.cellType.size(); k++) ctype.push_back(c.cellType[k]);
      for (int k = 0; k < c.nodeType.size(); k++) ntype.push_back(c.nodeType[k]);
    }
    out.i32(p + "charts_i", ci, 12);
    out.f64(p + "charts_d", cd, 4);
    out.i32(p + "cellType", ctype);
    out.i32(p + "nodeType", ntype);
    std::vector<int> cc;  // every active cell's corners, in global cell order
    for (auto& c : g.gridCharts)
      for (const CellIndex& q : c.cellIndices)
        for (int k = 0; k < 4; k++) cc.push_back(int(q[k]));
    out.i32(p + "cellIndices", cc, 4);
    if (l == 0) {  // InitializeInteriorTexelToCellLines (InteriorTexelToCellLines.inl:3-29)
      std::vector<InteriorTexelToCellLine> tl;
      InitializeInteriorTexelToCellLines(tl, g);
      std::vector<int> t5;
      for (const auto& t : tl)
        t5.insert(t5.end(), {t.texelStartIndex, t.texelEndIndex, t.coeffOffset, t.previousCellStartIndex, t.nextCellStartIndex});
      out.i32(p + "interiorTexelToCellLines", t5, 5);
    }
    // multigrid coefficients (reciprocal form for l < levels-1)
    std::vector<double> dc(coeffs[l].deepCoefficients.begin(), coeffs[l].deepCoefficients.end());
    out.f64(p + "coef/deep", dc, 10);
    out.csr(p + "coef/BB", coeffs[l].boundaryBoundaryMatrix);
    out.csr(p + "coef/BD", coeffs[l].boundaryDeepMatrix);
    if (l < levels - 1) out.csr(p + "boundaryRestriction", hierarchy.boundaryRestriction[l]);
  }
  if (full) {
    std::vector<int> tn;
    std::vector<double> tb;
    for (auto& n : textureNodes) {
      tn.insert(tn.end(), {n.ci, n.cj, n.chartId, n.tId, (int)n.isInterior});
      tb.insert(tb.end(), {n.baricentricCoords[0], n.baricentricCoords[1]});
    }
    out.i32("fine/textureNodes", tn, 5);
    out.f64("fine/textureBary", tb, 2);
    out.f64("fine/deepMass", deepMass, 10);
    out.f64("fine/deepStiffness", deepStiffness, 10);
    out.csr("fine/BBmass", bbM);
    out.csr("fine/BBstiffness", bbS);
    out.csr("fine/BDmass", bdM);
    out.csr("fine/BDstiffness", bdS);
    out.csr("fine/A", A);
    out.i32("fine/boundaryNodes", {fine.numBoundaryNodes, fine.numMidPoints, fine.numFineNodes, boundaryProlongation.numFineBoundarNodes});
    out.csr("fine/boundaryProlongation", boundaryProlongation.coarseBoundaryFineBoundaryProlongation);
    std::vector<int> ac;
    std::vector<double> ad;
    for (auto& c : atlasCharts) {
      ac.insert(ac.end(), {c.originCoords[0], c.originCoords[1], (int)c.triangles.size(), (int)c.vertices.size(), (int)c.boundaryHalfEdges.size()});
      ad.insert(ad.end(), {c.minCorner[0], c.minCorner[1], c.maxCorner[0], c.maxCorner[1], c.gridOrigin[0], c.gridOrigin[1]});
    }
    out.i32("atlas/charts_i", ac, 5);
    // boundary-cell triangulation: per triangle chart, cell, corner node indices, corner positions
    std::vector<int> bti;
    std::vector<double> btd;
    for (size_t c = 0; c < fine.gridCharts.size(); c++) {
      const GridChart& g = fine.gridCharts[c];
      for (size_t cell = 0; cell < g.boundaryTriangles.size(); cell++)
        for (const BoundaryIndexedTriangle& t : g.boundaryTriangles[cell]) {
          bti.insert(bti.end(), {(int)c, (int)cell, (int)t.indices[0], (int)t.indices[1], (int)t.indices[2]});
          for (int k = 0; k < 3; k++) { btd.push_back(t.vertices[k][0]); btd.push_back(t.vertices[k][1]); }
        }
    }
    out.i32("fine/boundaryTriangles", bti, 5);
    out.f64("fine/boundaryTrianglePos", btd, 6);
    out.f64("atlas/charts_d", ad, 6);
    for (int l = 1; l < levels; l++) {
      std::string p = "L" + std::to_string(l) + "/";
      out.csr(p + "boundaryCoarseFineProlongation", hierarchy.boundaryCoarseFineProlongation[l]);
    }
  }
  fprintf(stderr, "ok: %d texels, %d levels, hierarchy %.3fs assembly %.3fs system %.3fs direct %.3fs, vcycle %.4fs, resid %g -> %g\n",
          fine.numTexels, levels, tHierarchy, tAssembly, tSystem, tDirect,
          cycleTimes.empty() ? 0.0 : cycleTimes.back(), history.front(), history.back());
  return 0;
}
