// Host-side set-up of the texel-FEM system: atlas, texel-grid hierarchy,
// boundary elements and the Galerkin coefficient hierarchy.
//
// Index conventions are the reference's (they are the interface the apps and
// the vectors they pass in rely on):
//   * texels of one level are numbered chart by chart, raster order (j outer,
//     i inner), over active grid nodes;
//   * node types: -1 inactive, 0 exterior, 1 interior boundary, 2 deep
//     (HierarchyConstruction.inl:37-38);
//   * boundaryAndDeepIndex: boundary texels +1-based, deep texels -1-based
//     (HierarchyConstruction.inl:3-35);
//   * deep coefficients: 10 per deep texel, stencil offset (dj+1)*3+(di+1),
//     slot 9 free (holds the diagonal once reciprocals are taken,
//     UpdateCoefficients.inl:374-397).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace gdtp {

struct V2 {
  double x = 0, y = 0;
  V2() = default;
  V2(double a, double b) : x(a), y(b) {}
  V2 operator+(const V2& o) const { return V2(x + o.x, y + o.y); }
  V2 operator-(const V2& o) const { return V2(x - o.x, y - o.y); }
  V2 operator*(double s) const { return V2(x * s, y * s); }
  V2 operator/(double s) const { return V2(x / s, y / s); }
  double operator[](int i) const { return i ? y : x; }
  double& operator[](int i) { return i ? y : x; }
};
inline double dot(const V2& a, const V2& b) { return a.x * b.x + a.y * b.y; }

// 2x2 matrix stored column-major as c[col][row] (the layout the reference's
// FP64 formulas are written against; keeping it makes classification bit-exact).
struct M2 {
  double c[2][2] = {{0, 0}, {0, 0}};
  V2 operator*(const V2& v) const { return V2(c[0][0] * v.x + c[1][0] * v.y, c[0][1] * v.x + c[1][1] * v.y); }
  double det() const { return c[0][0] * c[1][1] - c[0][1] * c[1][0]; }
  M2 inverse() const {
    M2 r;
    double d = 1. / (c[0][0] * c[1][1] - c[0][1] * c[1][0]);
    r.c[0][0] = c[1][1] * d;
    r.c[1][1] = c[0][0] * d;
    r.c[0][1] = -c[0][1] * d;
    r.c[1][0] = -c[1][0] * d;
    return r;
  }
  M2 transpose() const {
    M2 r;
    r.c[0][0] = c[0][0]; r.c[1][1] = c[1][1]; r.c[0][1] = c[1][0]; r.c[1][0] = c[0][1];
    return r;
  }
  // (this * o)(col j,row i) = sum_k this(k,i) * o(j,k)
  M2 operator*(const M2& o) const {
    M2 r;
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 2; j++) r.c[j][i] = c[0][i] * o.c[j][0] + c[1][i] * o.c[j][1];
    return r;
  }
};

struct I3 { int v[3]; int& operator[](int i) { return v[i]; } int operator[](int i) const { return v[i]; } };

// ----------------------------------------------------------------------------
// input mesh
// ----------------------------------------------------------------------------
struct Mesh {
  std::vector<double> vertices;   // nv*3
  std::vector<int> triangles;     // nt*3
  std::vector<double> uv;         // nt*3*2 per-corner texture coordinates
  int nv() const { return (int)vertices.size() / 3; }
  int nt() const { return (int)triangles.size() / 3; }
  V2 corner(int t, int k) const { return V2(uv[6 * t + 2 * k], uv[6 * t + 2 * k + 1]); }
};

struct AtlasChart {
  V2 minCorner, maxCorner, gridOrigin;
  int originCoords[2] = {0, 0};
  std::vector<I3> triangles;            // chart-local vertex ids
  std::vector<V2> vertices;             // chart vertices (texture space)
  std::vector<int> boundaryHalfEdges;   // 3*chartTriangle + k
  std::vector<int> atlasEdgeIndices;    // per chart corner 3*t+k
  std::vector<int> meshVertexIndices;
  std::vector<int> meshTriangleIndices;
};

struct Atlas {
  int width = 0, height = 0;
  std::vector<V2> vertices;             // atlas vertices (unique (uv, mesh vertex) pairs)
  std::vector<I3> triangles;
  std::vector<int> vertexMap;           // atlas vertex -> mesh vertex
  std::vector<int> triangleChart;
  std::vector<int> halfEdgeToEdgeIndex;
  std::vector<int> oppositeHalfEdge;    // on the input mesh, -1 open
  std::vector<char> isBoundaryHalfEdge;
  std::vector<int> boundaryVertexIndex; // mesh vertex -> boundary vertex id or -1
  int numBoundaryVertices = 0;
  bool isClosed = true;
  int numCharts = 0;
  int gridJitterCount = 0;              // vertices moved off texel-centre lines
  std::vector<AtlasChart> charts;
};

// ----------------------------------------------------------------------------
// texel grid per chart and level
// ----------------------------------------------------------------------------
struct GridChart {
  V2 corner;
  int cornerCoords[2] = {0, 0};
  int centerOffset[2] = {0, 0};
  double cellSizeW = 0, cellSizeH = 0;
  int width = 0, height = 0;
  int texelOffset = 0, deepOffset = 0, boundaryOffset = 0, interiorTexelOffset = 0, cellOffset = 0;
  int gridIndexOffset = 0;
  std::vector<int> nodeType;            // width*height
  std::vector<int> cellType;            // (width-1)*(height-1): -1 inactive, 0 boundary, 1 interior
  std::vector<int> texel;               // global texel index or -1
  std::vector<int> interiorTexel;       // global interior texel index or -1
  std::vector<int> deepTexel;           // global deep index or -1
  std::vector<int> boundaryTexel;       // global boundary index or -1
  std::vector<int> localCell, localInteriorCell, localBoundaryCell;  // (width-1)*(height-1)
  std::vector<int> cellCorners;         // 4 global texels per active cell (local cell order)
  std::vector<int> interiorCellCorners; // 4 global texels per interior cell
  std::vector<int> interiorCellToCell, boundaryCellToCell;
  int numInteriorCells = 0, numBoundaryCells = 0;
  std::vector<int> triangleId;          // width*height, mesh triangle or -1
  std::vector<V2> bary;                 // width*height
  int at(int i, int j) const { return j * width + i; }
  int cat(int i, int j) const { return j * (width - 1) + i; }
};

struct Line { int start, end, prev, next, coeff; };                 // RasterLine / RestrictionLine
struct DeepLine { int coarseStart, coarseEnd, finePrev, fineCurrent, fineNext; };
struct ProlongationLine { int start, length, center, prev, next, aligned; };

struct Csr {                                                          // CSR, sorted columns
  int rows = 0, cols = 0;
  std::vector<int> ptr{0}, col;
  std::vector<double> val;
  int nnz() const { return (int)col.size(); }
};
struct Triplet { int r, c; double v; };
Csr csr_from_triplets(int rows, int cols, std::vector<Triplet>& t);    // sums duplicates
// two value sets on one list of (row, column) entries: m1 from v1, m2 from v2,
// each as csr_from_triplets would build it
void csr_from_pairs(int rows, int cols, const std::vector<int>& r, const std::vector<int>& c, const std::vector<double>& v1,
                    const std::vector<double>& v2, Csr& m1, Csr& m2);
// c1 = a b and c2 = a' b' on one pattern, a' = a with values *a2 (or a's own
// when null), b' likewise; each as csr_multiply would compute it
void csr_multiply2(const Csr& a, const std::vector<double>* a2, const Csr& b, const std::vector<double>* b2, Csr& c1, Csr& c2);
Csr csr_transpose(const Csr& a);
Csr csr_multiply(const Csr& a, const Csr& b);
Csr csr_axpby(double a, const Csr& A, double b, const Csr& B);

struct NodeInfo { int chart, ci, cj, type; };

struct GridLevel {
  int numTexels = 0, numInteriorTexels = 0, numDeep = 0, numBoundary = 0;
  int numCells = 0, numBoundaryCells = 0, numInteriorCells = 0;
  std::vector<GridChart> charts;
  std::vector<NodeInfo> nodes;
  std::vector<int> boundaryAndDeep, boundaryGlobal, deepGlobal;
  std::vector<Line> rasterLines;
  std::vector<Line> restrictionLines;   // this level is the coarse side
  std::vector<DeepLine> deepLines;      // this level is the coarse side
  std::vector<ProlongationLine> prolongationLines;  // this level is the fine side
  Csr boundaryRestriction;              // (coarse boundary) x (this level's texels), for levels < L-1
  // boundary elements (finest level only)
  int numBoundaryNodes = 0, numMidPoints = 0, numFineNodes = 0;
};

struct Hierarchy {
  int requestedLevels = 0;              // levels asked for; more may be built for the coarse direct solve
  Atlas atlas;
  std::vector<GridLevel> levels;
  std::string error;
};

struct BlockInfo { int blockWidth = 128, blockHeight = 16, paddingWidth = 2, paddingHeight = 0, boundaryDilation = 0; };

// atlas.cpp
bool build_atlas(const Mesh& mesh, int width, int height, Atlas& atlas, std::string& err);
// grid.cpp
// Builds `levels` levels, then keeps coarsening while the coarsest level holds
// more than extendToTexels texels (0: never), up to maxLevels.
bool build_hierarchy(const Mesh& mesh, int width, int height, int levels, const BlockInfo& info, Hierarchy& h,
                     int extendToTexels = 0, int maxLevels = 12);

// ----------------------------------------------------------------------------
// boundary elements and assembly
// ----------------------------------------------------------------------------
struct AuxNode { V2 pos; int index; };
struct BoundaryTriangle {              // quadratic element inside one boundary cell
  V2 v[3];
  int idx[6];                           // 3 corner nodes + 3 mid-edge nodes (fine node ids)
  int atlasVertex[3], atlasEdge[3], parentEdge[3];
};
struct ChartBoundary {
  std::vector<std::vector<BoundaryTriangle>> cellTriangles;  // per boundary cell
  std::vector<AuxNode> aux;
};
struct BoundaryElements {
  std::vector<ChartBoundary> charts;
  int numBoundaryNodes = 0, numMidPoints = 0, numFineNodes = 0, numBoundaryVertices = 0;
  int numFineBoundary = 0;
  std::vector<int> fineBoundaryIndex;   // fine node -> fine boundary index or -1
  Csr prolongation;                     // fine boundary nodes x coarse boundary texels
  int degenerateTriangulations = 0;
};
bool build_boundary_elements(const Hierarchy& h, BoundaryElements& be, std::string& err);

// per chart, per chart triangle: 2x2 parameter metric g (column-major c[col][row])
typedef std::vector<std::vector<M2>> ChartMetrics;
bool embedding_metric(const Mesh& mesh, const Atlas& atlas, ChartMetrics& g);
// Per mesh triangle metrics (metric.cpp), in the basis of the triangle's edges:
// mode 0 = embedding (edges in space), 1 = uniform (edges in texture space);
// optionally divided by the total area they measure.
bool surface_metric(const Mesh& mesh, int mode, bool normalizeArea, std::vector<M2>& G);
// Tangent-field metric: g B diag(0, across) B^-1 + isotropic g, with B the
// g-orthonormal frame (field, field rotated); vf = nt x 2 edge-basis vectors.
bool vector_field_metric(const std::vector<M2>& G, const double* vf, double across, double isotropic, bool normalizeArea,
                         std::vector<M2>& out);
// Pull-back to texture coordinates: J^-T G J^-1 with J the texture-space edges.
bool parameter_metric(const Mesh& mesh, const std::vector<M2>& G, std::vector<M2>& out);

// Work lists of the device assembly.  Interior cells: for every interior cell
// (chart order, then interior-cell order) the chart triangles overlapping it,
// in increasing chart-triangle order (the reference's accumulation order).
// Boundary triangles: the same for every quadratic boundary element.
struct AssemblyWork {
  int numTriangles = 0, numInteriorCells = 0, numBoundaryTriangles = 0;
  std::vector<double> triPos;           // 6 per chart triangle (chart-major): grid-corner-relative corners
  std::vector<double> triMetric;        // 4 per triangle: g (c00,c01,c10,c11)
  std::vector<double> triMetricInv;     // 4 per triangle: g^-1
  std::vector<double> triScale;         // sqrt(det g)
  std::vector<int> cellPtr, cellTri;    // interior cell -> triangles
  std::vector<int> cellIJ, cellChart;   // chart-local cell coordinates, chart
  std::vector<double> chartCellSize;    // 2 per chart
  std::vector<int> deepCells;           // 4 per deep texel: surrounding interior cells, raster order
  std::vector<int> boundaryAdjacentCells;  // interior cells with a non-deep corner
  std::vector<double> btPos;            // 6 per boundary triangle
  std::vector<int> btIdx;               // 6 per boundary triangle: fine boundary indices
  std::vector<int> btPtr, btTri;        // boundary triangle -> chart triangles
};
void build_assembly_work(const Hierarchy& h, const BoundaryElements& be, const ChartMetrics& g, AssemblyWork& w);

struct FineSystem {
  std::vector<double> deepMass, deepStiffness;   // 10 per deep texel
  Csr bbMass, bbStiffness;                       // boundary x boundary (texel boundary indices)
  Csr bdMass, bdStiffness;                       // boundary x global texel
};
// Boundary rows: interior-cell element matrices of the boundary-adjacent cells
// (16 per cell, [4k+l]) and boundary-triangle element matrices (36 per triangle,
// [6l+k]), both computed on the device, become the BB and BD blocks.
bool assemble_boundary_blocks(const Hierarchy& h, const BoundaryElements& be, const AssemblyWork& w,
                              const std::vector<double>& adjCellMass, const std::vector<double>& adjCellStiffness,
                              const std::vector<double>& btMass, const std::vector<double>& btStiffness, FineSystem& fs,
                              std::string& err);

struct LevelCoefficients {
  std::vector<double> deep;             // 10 per deep texel, raw (no reciprocals)
  Csr bb, bd;                           // boundary x boundary, boundary x global
};
// Galerkin hierarchy A_{l+1} = P^T A_l P; coarsest also as a dense matrix.
bool galerkin_hierarchy(const Hierarchy& h, int levels, const std::vector<double>& deep0, const Csr& bb0, const Csr& bd0,
                        std::vector<LevelCoefficients>& out, std::string& err);
void full_matrix(const GridLevel& g, const LevelCoefficients& c, Csr& full);

// Exact boundary-block solve by subdomain inverses + separator Schur complement
// (bsolve.cpp).  Positions k index `order` (interiors by subdomain, then separators).
struct BoundarySolverSetup {
  int nb = 0, nSub = 0, nI = 0, nS = 0;
  std::vector<int> order;               // position -> boundary index
  std::vector<int> subPtr;              // subdomain -> [subPtr[p], subPtr[p+1]) positions
  std::vector<double> scale;            // per position: 1/sqrt(BB_ii)
  std::vector<int64_t> invOff;          // per subdomain offset into inv
  std::vector<double> inv;              // scaled dense inverses, row-major m x m
  Csr AIS, ASI;                         // scaled couplings: interior positions x separator, and transpose
  std::vector<int> touchPtr, touch;     // per subdomain: the separator columns its rows couple to
  std::vector<int64_t> wOff;            // per subdomain offset into W
  std::vector<double> W;                // Inv_p A_{I_p,touch}, m x t column-major (scaled)
  std::vector<double> Sinv;             // scaled nS x nS inverse Schur complement
  Csr BD;                               // positions x global texels (unscaled boundary-deep rows)
  // ms spent: partition and sparse assembly, subdomain inverses, Schur
  // products and assembly, Schur complement inverse
  double ms[4] = {0, 0, 0, 0};
};
// Subdomains and separator of a boundary block from its pattern alone:
// order (position -> row; interiors grouped by subdomain, then the separator),
// subPtr (subdomain -> position range), nI (interior positions).
void partition_boundary(const Csr& BB, int maxBlock, int denseMax, std::vector<int>& order, std::vector<int>& subPtr, int& nI);

// The weight-independent structure of the boundary solver: the partition, and
// for each of its values the boundary-block entry it is made from, so that the
// values can be recomputed on the device for new weights.  A BB entry k of rows
// i, j gives the scaled value BB_k s_pos(i) s_pos(j), s = 1 / sqrt(diag).
struct BoundarySymbolic {
  int nb = 0, nSub = 0, nI = 0, nS = 0;
  std::vector<int> order, pos, subPtr;
  std::vector<int> bbRow;                   // BB entry -> its row
  std::vector<int> diagEntry;               // row -> its diagonal BB entry
  std::vector<int64_t> invOff;              // subdomain -> offset of its m x m block (nSub + 1)
  std::vector<int> fillEntry;               // BB entries inside a subdomain block ...
  std::vector<int64_t> fillDest;            // ... and their position in the blocks
  std::vector<int> ssEntry;                 // BB entries between separator rows ...
  std::vector<int64_t> ssDest;              // ... and their position in the nS x nS Schur block
  Csr AIS, ASI;                             // interior x separator coupling and transpose; val = BB entry
  std::vector<int64_t> aisDest;             // AIS entry -> position in the C_p blocks (m x t row-major at wOff[p])
  std::vector<int> touchPtr, touch;         // per subdomain: the separator columns its rows couple to
  std::vector<int64_t> wOff, lOff;          // per subdomain: m x t block offset, t x t block offset (nSub + 1)
  Csr BD;                                   // boundary-deep rows in solver order; val = BD entry
};
bool build_boundary_symbolic(const Csr& BB, const Csr& BD, int maxBlock, int denseMax, BoundarySymbolic& sym, std::string& err);

// Where the dense FP64 products of the set-up run: the host (nullptr) or a
// device backend (system.cu: kernels/dense_kernels.cu).
struct DenseBackend {
  virtual ~DenseBackend() = default;
  // in-place inverses of SPD matrices data[off[q] ..], size[q] x size[q] row-major
  virtual bool spd_inverse_batched(double* data, const std::vector<int64_t>& off, const std::vector<int>& size, std::string& err) = 0;
  // per subdomain p: G_p = Inv_p C_p (m_p x t_p, C_p row-major at cOff[p]) and
  // local_p = C_p^T G_p (t_p x t_p at localOff[p])
  virtual bool schur_products(const std::vector<double>& inv, const std::vector<int64_t>& invOff, const std::vector<int>& m,
                              const std::vector<double>& C, const std::vector<int64_t>& cOff, const std::vector<int>& t,
                              std::vector<double>& G, std::vector<double>& local, const std::vector<int64_t>& localOff,
                              std::string& err) = 0;
};
// denseMax: blocks of at most this many rows are inverted whole (no subdomains)
bool build_boundary_solver(const Csr& BB, const Csr& BD, int maxBlock, int denseMax, BoundarySolverSetup& bs, std::string& err,
                           DenseBackend* dense = nullptr);
bool dense_spd_inverse(double* A, int n, bool parallel);

}  // namespace gdtp
