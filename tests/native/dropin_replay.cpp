// Headless replay of the TextureFiltering app's solve path, written against the
// reference's own headers and types, call for call as TextureFilter::InitializeSystem
// and TextureFilter::UpdateSolution make them (TextureFiltering/TextureFiltering.cpp:
// 581-718 and 562-579), without the window and the texture files.
//
// The same source is compiled twice (oracle/Makefile):
//   dropin_replay_ref   -I<reference>/include            the reference itself (CPU)
//   dropin_replay_gdtp  -I<repo>/include -I<reference>/include, linked to libgdtp:
//                       the drop-in headers forward the solve path to the device
// so the test compares an unchanged app against itself with and without the
// drop-in.  Test infrastructure only.
//
// Usage: dropin_replay <mesh.gdm> <out.bin> [levels] [stiffness] [sharpness] [vcycles]
// out.bin: int64 n, then float64 n x 3 arrays: rhs, x after the first V-cycle,
// x after the last.
#define USE_FLOAT 1
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
#include <Src/InteriorTexelToCellLines.inl>
#include <Src/Padding.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

typedef float Real;

// the repository's binary mesh container (meshgen.write_gdm): magic, five int64
// counts (vertices, triangles, texture width, height, channels), then vertices
// (float64 x 3), triangles (int32 x 3), per-corner uv (float64 x 6 per
// triangle) and the texture (float32, rows of width x channels)
static bool read_mesh(const char* path, TexturedMesh& mesh) {
  FILE* f = fopen(path, "rb");
  if (!f) return false;
  char magic[8];
  int64_t hdr[5];
  bool ok = fread(magic, 1, 8, f) == 8 && !memcmp(magic, "GDTPMSH1", 8) && fread(hdr, 8, 5, f) == 5;
  std::vector<double> v, uv;
  std::vector<int32_t> t;
  std::vector<float> tex;
  if (ok) {
    v.resize(size_t(hdr[0]) * 3);
    t.resize(size_t(hdr[1]) * 3);
    uv.resize(size_t(hdr[1]) * 6);
    tex.resize(size_t(hdr[2] * hdr[3] * hdr[4]));
    ok = fread(v.data(), 8, v.size(), f) == v.size() && fread(t.data(), 4, t.size(), f) == t.size() &&
         fread(uv.data(), 8, uv.size(), f) == uv.size() && fread(tex.data(), 4, tex.size(), f) == tex.size();
  }
  fclose(f);
  if (!ok) return false;
  const int w = int(hdr[2]), h = int(hdr[3]), c = int(hdr[4]);
  mesh.vertices.resize(hdr[0]);
  for (size_t i = 0; i < mesh.vertices.size(); i++) mesh.vertices[i] = Point3D<double>(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
  mesh.triangles.resize(hdr[1]);
  for (size_t i = 0; i < mesh.triangles.size(); i++) mesh.triangles[i] = TriangleIndex(t[3 * i], t[3 * i + 1], t[3 * i + 2]);
  mesh.textureCoordinates.resize(size_t(hdr[1]) * 3);
  for (size_t i = 0; i < mesh.textureCoordinates.size(); i++) mesh.textureCoordinates[i] = Point2D<double>(uv[2 * i], uv[2 * i + 1]);
  mesh.texture.resize(w, h);
  for (int j = 0; j < h; j++)
    for (int i = 0; i < w; i++) {
      const float* p = &tex[(size_t(j) * w + i) * c];
      mesh.texture(i, j) = Point3D<float>(p[0], c > 1 ? p[1] : p[0], c > 2 ? p[2] : p[0]);
    }
  return true;
}

static void put(FILE* f, const std::vector<VECTOR_TYPE>& v) {
  std::vector<double> a(v.size() * 3);
  for (size_t i = 0; i < v.size(); i++)
    for (int c = 0; c < 3; c++) a[3 * i + c] = double(v[i][c]);
  fwrite(a.data(), 8, a.size(), f);
}

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s mesh.gdm out.bin [levels] [stiffness] [sharpness] [vcycles]\n", argv[0]);
    return 2;
  }
  const int levels = argc > 3 ? atoi(argv[3]) : 4;
  const double stiffnessWeight = argc > 4 ? atof(argv[4]) : 1e-3;
  const double sharpnessWeight = argc > 5 ? atof(argv[5]) : 2.0;
  const int vcycles = argc > 6 ? atoi(argv[6]) : 6;

  TexturedMesh mesh;
  if (!read_mesh(argv[1], mesh)) {
    fprintf(stderr, "cannot read %s\n", argv[1]);
    return 2;
  }
  const int width = mesh.texture.width(), height = mesh.texture.height();

  // the app's state (TextureFilter<Real>'s static members)
  std::vector<TextureNodeInfo> textureNodes;
  std::vector<CellIndex> cellIndices;
  HierarchicalSystem hierarchy;
  std::vector<AtlasChart> atlasCharts;
  std::vector<double> deepMassCoefficients, deepStiffnessCoefficients;
  SparseMatrix<double, int> boundaryBoundaryMassMatrix, boundaryBoundaryStiffnessMatrix, boundaryDeepMassMatrix,
      boundaryDeepStiffnessMatrix, boundaryCellBasedStiffnessRHSMatrix[3], filteringMatrix;
  std::vector<VECTOR_TYPE> interiorTexelToCellCoeffs, mass_x0, stiffness_x0;
  std::vector<InteriorTexelToCellLine> interiorTexelToCellLines;
  std::vector<Real> boundaryTexelStiffness[3];
  std::vector<VECTOR_TYPE> texelModulatedStiffness;
  std::vector<MultigridLevelCoefficients<Real>> multigridFilteringCoefficients;
  std::vector<MultigridLevelVariables<VECTOR_TYPE>> multigridFilteringVariables;
  std::vector<MultigridLevelIndices<Real>> multigridIndices;
  std::vector<EigenCholeskySolver3<Real>> boundarySolver;
  EigenCholeskySolver3<Real> coarseSolver, directSolver;

  // ---- TextureFilter::InitializeSystem (TextureFiltering.cpp:581-718), no direct solver
  MultigridBlockInfo multigridBlockInfo(128, 16, 2, 0, 0);  // the app's defaults (TextureFiltering.cpp:25-28)
  if (!InitializeHierarchy(mesh, width, height, levels, textureNodes, cellIndices, hierarchy, atlasCharts, multigridBlockInfo, true,
                           false)) {
    printf("ERROR : Failed intialization! \n");
    return 3;
  }
  BoundaryProlongationData boundaryProlongation;
  if (!InitializeBoundaryProlongationData(hierarchy.gridAtlases[0], boundaryProlongation)) return 3;
  std::vector<VECTOR_TYPE> _x0(textureNodes.size());
  for (size_t i = 0; i < textureNodes.size(); i++) {
    const Point3D<float> texelValue = mesh.texture(textureNodes[i].ci, textureNodes[i].cj);
    _x0[i] = SetData(texelValue[0], texelValue[1], texelValue[2]);
  }
  std::vector<Point3D<double>> inputSignal(textureNodes.size());
  for (size_t i = 0; i < textureNodes.size(); i++) inputSignal[i] = mesh.texture(textureNodes[i].ci, textureNodes[i].cj);
  std::vector<double> texelToCellCoeffs;
  std::vector<std::vector<SquareMatrix<double, 2>>> parameterMetric;
  if (!InitializeMetric(mesh, EMBEDDING_METRIC, atlasCharts, parameterMetric)) return 3;
  SparseMatrix<double, int> _boundaryCellBasedStiffnessRHSMatrix[3];
  if (!InitializeMassAndStiffness(deepMassCoefficients, deepStiffnessCoefficients, boundaryBoundaryMassMatrix,
                                  boundaryBoundaryStiffnessMatrix, boundaryDeepMassMatrix, boundaryDeepStiffnessMatrix, hierarchy,
                                  parameterMetric, atlasCharts, boundaryProlongation, true, inputSignal, texelToCellCoeffs,
                                  _boundaryCellBasedStiffnessRHSMatrix)) {
    printf("ERROR : Failed intialization! \n");
    return 3;
  }
  for (int c = 0; c < 3; c++) boundaryCellBasedStiffnessRHSMatrix[c] = _boundaryCellBasedStiffnessRHSMatrix[c];
  interiorTexelToCellCoeffs.resize(4 * hierarchy.gridAtlases[0].numDeepTexels);
  for (int i = 0; i < 4 * hierarchy.gridAtlases[0].numDeepTexels; i++)
    interiorTexelToCellCoeffs[i] = SetData(Real(texelToCellCoeffs[3 * i + 0]), Real(texelToCellCoeffs[3 * i + 1]), Real(texelToCellCoeffs[3 * i + 2]));
  if (!InitializeInteriorTexelToCellLines(interiorTexelToCellLines, hierarchy.gridAtlases[0])) return 3;
  for (int c = 0; c < 3; c++) boundaryTexelStiffness[c].resize(hierarchy.gridAtlases[0].boundaryGlobalIndex.size());
  texelModulatedStiffness.resize(hierarchy.gridAtlases[0].numTexels);
  multigridIndices.resize(levels);
  for (int i = 0; i < levels; i++) {
    const GridAtlas& gridAtlas = hierarchy.gridAtlases[i];
    multigridIndices[i].threadTasks = gridAtlas.threadTasks;
    multigridIndices[i].boundaryGlobalIndex = gridAtlas.boundaryGlobalIndex;
    multigridIndices[i].segmentedLines = gridAtlas.segmentedLines;
    multigridIndices[i].rasterLines = gridAtlas.rasterLines;
    multigridIndices[i].restrictionLines = gridAtlas.restrictionLines;
    multigridIndices[i].prolongationLines = gridAtlas.prolongationLines;
    if (i < levels - 1) multigridIndices[i].boundaryRestriction = hierarchy.boundaryRestriction[i];
  }
  if (!UpdateLinearSystem(stiffnessWeight, 1.0, hierarchy, multigridFilteringCoefficients, deepMassCoefficients, deepStiffnessCoefficients,
                          boundaryBoundaryMassMatrix, boundaryBoundaryStiffnessMatrix, boundaryDeepMassMatrix, boundaryDeepStiffnessMatrix,
                          coarseSolver, boundarySolver, directSolver, filteringMatrix, false, true, false)) {
    printf("ERROR : Failed system update! \n");
    return 3;
  }
  multigridFilteringVariables.resize(levels);
  for (int i = 0; i < levels; i++) {
    MultigridLevelVariables<VECTOR_TYPE>& variables = multigridFilteringVariables[i];
    variables.x.resize(hierarchy.gridAtlases[i].numTexels);
    variables.rhs.resize(hierarchy.gridAtlases[i].numTexels);
    variables.residual.resize(hierarchy.gridAtlases[i].numTexels);
    variables.boundary_rhs.resize(hierarchy.gridAtlases[i].boundaryGlobalIndex.size());
    variables.boundary_value.resize(hierarchy.gridAtlases[i].boundaryGlobalIndex.size());
    variables.variable_boundary_value.resize(hierarchy.gridAtlases[i].boundaryGlobalIndex.size());
  }
  mass_x0.resize(textureNodes.size());
  MultiplyBySystemMatrix_NoReciprocals(deepMassCoefficients, boundaryDeepMassMatrix, boundaryBoundaryMassMatrix,
                                       hierarchy.gridAtlases[0].boundaryGlobalIndex, hierarchy.gridAtlases[0].rasterLines, _x0, mass_x0);
  stiffness_x0.resize(textureNodes.size());
  MultiplyBySystemMatrix_NoReciprocals(deepStiffnessCoefficients, boundaryDeepStiffnessMatrix, boundaryBoundaryStiffnessMatrix,
                                       hierarchy.gridAtlases[0].boundaryGlobalIndex, hierarchy.gridAtlases[0].rasterLines, _x0, stiffness_x0);
  for (size_t i = 0; i < _x0.size(); i++) {
    multigridFilteringVariables[0].x[i] = _x0[i];
    multigridFilteringVariables[0].rhs[i] = mass_x0[i] + stiffness_x0[i] * sharpnessWeight * stiffnessWeight;
  }

  // ---- TextureFilter::UpdateSolution (TextureFiltering.cpp:562-579), vcycles times
  FILE* out = fopen(argv[2], "wb");
  if (!out) return 2;
  const int64_t n = int64_t(_x0.size());
  fwrite(&n, 8, 1, out);
  put(out, multigridFilteringVariables[0].rhs);
  for (int it = 0; it < vcycles; it++) {
    if (!VCycle(multigridFilteringVariables, multigridFilteringCoefficients, multigridIndices, boundarySolver, coarseSolver, false,
                false))
      return 4;
    if (it == 0) put(out, multigridFilteringVariables[0].x);
  }
  put(out, multigridFilteringVariables[0].x);
  fclose(out);
  printf("replay ok: %lld texels, %d V-cycles\n", (long long)n, vcycles);
  return 0;
}
