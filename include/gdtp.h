/*
 * gdtp.h -- C ABI of the B200 texel-FEM solve path (gradient-domain texture
 * processing: atlas-clipped texel grid, multigrid V-cycle, coarse direct solve).
 *
 * Plain pointers and sizes only.  Every function returns a gdtp status (0 = ok,
 * negative = error); gdtp_last_error() returns the message of the calling
 * thread's last failure.  Arrays are row-major; "host" pointers are ordinary
 * CPU memory, "device" pointers are CUDA device memory of the handle's device.
 *
 * Texel vectors use the reference's layout: one entry per active texel in the
 * reference's global texel order (chart by chart, raster order), k channels
 * interleaved (x[texel * k + channel]).
 *
 * Each entry point names the reference interface it replaces (path:line in
 * fabianprada/GradientDomainTextureProcessing).
 */
#ifndef GDTP_H
#define GDTP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GDTP_OK 0
#define GDTP_ERR_INVALID (-1)       /* bad argument */
#define GDTP_ERR_SETUP (-2)         /* mesh / atlas / hierarchy construction failed */
#define GDTP_ERR_CUDA (-3)          /* CUDA runtime error or no usable device */
#define GDTP_ERR_NOT_CONVERGED (-4) /* solve stopped at max_iters above tolerance */
#define GDTP_ERR_BUDGET (-5)        /* HBM admission budget exceeded */
#define GDTP_ERR_STATE (-6)         /* call out of order (e.g. solve before update) */
#define GDTP_ERR_NUMERIC (-7)       /* coarse factorisation not positive definite */

typedef struct gdtp_hierarchy gdtp_hierarchy;
typedef struct gdtp_system gdtp_system;

const char* gdtp_last_error(void);
int gdtp_version(void);

/* ---------------------------------------------------------------------------
 * Hierarchy (host).  Replaces InitializeHierarchy
 * (include/Src/HierarchyConstruction.inl:799-849) and, for the finest level,
 * InitializeBoundaryTriangulation (include/Src/BoundaryQuadraticElements.inl:619)
 * and InitializeBoundaryProlongationData (BoundaryQuadraticElements.inl:775).
 * vertices: nv*3, triangles: nt*3, uv: nt*3*2 per-corner coordinates.
 * block_info: {blockWidth, blockHeight, paddingWidth, paddingHeight,
 * boundaryDilation} as MultigridBlockInfo (include/Src/Hierarchy.h:61-76), or NULL.
 * ------------------------------------------------------------------------- */
int gdtp_hierarchy_build(const double* vertices, int64_t nv, const int32_t* triangles, int64_t nt, const double* uv,
                         int width, int height, int levels, const int32_t* block_info, gdtp_hierarchy** out);
void gdtp_hierarchy_free(gdtp_hierarchy* h);
int gdtp_hierarchy_levels(const gdtp_hierarchy* h);
int gdtp_hierarchy_charts(const gdtp_hierarchy* h);
/* counts[8] = {texels, deep, boundary, cells, boundaryCells, interiorCells, interiorTexels, charts}
 * (GridAtlas counters, include/Src/Hierarchy.h:241-252) */
int gdtp_hierarchy_counts(const gdtp_hierarchy* h, int level, int64_t* counts);
/* Named host arrays of one level (int32 unless noted).  With out == NULL only
 * *count (elements) is written.  Names and row widths:
 *   "nodeinfo"(4: chart,ci,cj,type)  GridAtlas::nodeInfo           Hierarchy.h:236
 *   "boundaryAndDeep" "boundaryGlobal" "deepGlobal"                Hierarchy.h:233-235
 *   "rasterLines"(5) "restrictionLines"(5) "deepLines"(5)          Hierarchy.h:239-241
 *   "prolongationLines"(6)                                         Hierarchy.h:242
 *   "charts"(12) chart grid ints, "chartsd"(4, float64) corner+cell size   Hierarchy.h:146-161
 *   "nodeType" "cellType" concatenated per-chart images
 *   "interiorTexelToCellLines"(5: texel start, texel end, coefficient offset, first
 *   cell of the row above, of the row below) per raster line, level 0 only
 *   (InitializeInteriorTexelToCellLines, InteriorTexelToCellLines.inl:3-29)
 *   "cellCorners"(4) global texels of every active cell, chart by chart in raster
 *   order: the global cell index (InitializeCellNodes, HierarchyConstruction.inl:557-566)
 *   "textureNodes"(5: ci,cj,chart,tId,isInterior) level 0 only     Basis.h:4-28
 *   "textureBary"(2, float64) level 0 only
 *   "boundaryRestriction.ptr/.col/.val(float64)"  HierarchicalSystem::boundaryRestriction
 *   "boundaryNodes"(4: boundaryNodes, midPoints, fineNodes, fineBoundaryNodes) level 0
 *   "boundaryProlongation.ptr/.col/.val(float64)" level 0 (coarseBoundaryFineBoundaryProlongation) */
int gdtp_hierarchy_array(const gdtp_hierarchy* h, const char* name, int level, void* out, int64_t* count);
/* The texture value of every level-0 texel, in texel order: out[t * channels
 * + c] = the texture's channel c at the texel's pixel (x, y)
 * (TextureFiltering.cpp:603-608).  texture: height x width x channels values,
 * float32 (bytes_per_value 4) or float64 (8), at byte offset y * row_stride +
 * x * pixel_stride + c * channel_stride (any layout, no copy); out: float64
 * numTexels * channels.  GDTP_ERR_INVALID when a texel lies outside the image. */
int gdtp_texel_signal(const gdtp_hierarchy* h, const void* texture, int width, int height, int channels, int bytes_per_value,
                      int64_t row_stride, int64_t pixel_stride, int64_t channel_stride, double* out);

/* ---------------------------------------------------------------------------
 * Metrics (host).  Per mesh triangle parameter metric (nt*4, the layout of
 * gdtp_system_create's parameter_metric), area-normalised as the reference's.
 * gdtp_surface_metric: mode 0 = embedding (InitializeEmbeddingMetric,
 * Metric.inl:248-275), 1 = uniform (InitializeUniformMetric, :277-303), pulled
 * back to texture space (InitializeParameterMetric, :415-446).
 * gdtp_anisotropic_metric: tangent-field metric for line-integral convolution
 * (InitializeVectorFieldMetric, Metric.inl:12-67, as InitializeAnisotropicMetric
 * :468-486 applies it to a given field): g B diag(0, across) B^-1 + isotropic*g
 * with B the g-orthonormal frame {field, field rotated by 90 degrees}.  vf: nt*2,
 * the field on each triangle in the basis of its edges (p1 - p0, p2 - p0), the
 * per-triangle layout of the reference's vector-field files.  The reference uses
 * across = 0.1 and isotropic = 1e-5 (Metric.inl:45-55).
 * ------------------------------------------------------------------------- */
int gdtp_surface_metric(const double* vertices, int64_t nv, const int32_t* triangles, int64_t nt, const double* uv, int mode,
                        double* metric_out);
int gdtp_anisotropic_metric(const double* vertices, int64_t nv, const int32_t* triangles, int64_t nt, const double* uv,
                            const double* vf, double across, double isotropic, double* metric_out);

/* ---------------------------------------------------------------------------
 * System (device).  gdtp_system_create binds a hierarchy to a CUDA device and
 * assembles the FP64 mass and stiffness matrices: replaces InitializeMetric
 * (include/Src/Metric.inl:448; metric_mode 0 = embedding) and
 * InitializeMassAndStiffness (include/Src/MassAndStiffness.h:490-549).
 * parameter_metric: optional per mesh triangle 2x2 metric (nt*4, column-major
 * g(0,0),g(0,1),g(1,0),g(1,1) in texture coordinates, as InitializeParameterMetric
 * produces, Metric.inl:415-446); NULL selects metric_mode (0 = embedding,
 * 1 = uniform: InitializeMetric, Metric.inl:448-466).
 * ------------------------------------------------------------------------- */
int gdtp_system_create(gdtp_hierarchy* h, int device, int metric_mode, const double* parameter_metric,
                       const double* vertices, int64_t nv, gdtp_system** out);
void gdtp_system_free(gdtp_system* s);
/* Named host copies of the assembled FP64 system (level 0 unless noted):
 *   "deepMass" "deepStiffness" (10 per deep texel)
 *   "bbMass.ptr/.col/.val" "bbStiffness.*" "bdMass.*" "bdStiffness.*"
 *   after gdtp_system_update: "coef.deep"(level l, raw, 10 per deep texel), "coef.bb.*", "coef.bd.*"
 *   "profile": {timed level-0 sweep groups, their total ms, deep texels per group,
 *   kernels per step graph, kernels launched by solves, the timed group's smoother:
 *   1 one fused tile-smoother launch, 2 a sweep of two row-smoother launches, 0 a
 *   sweep of four colour passes}; "profile.reset" clears the counts
 *   "profile.setup": ms of the last set-up {update, boundary solver factorisations,
 *   coarsest inverse, other multigrid set-up, then the factorisations split into
 *   partition and sparse assembly, subdomain inverses, Schur products, Schur
 *   complement inverse; then the assembly {work lists, device assembly with its
 *   transfers, boundary blocks, level-0 operators}, the Galerkin coarsening of M
 *   and S and the numeric set-up's layout}: 14 values.  With the numeric set-up
 *   (device_factor 1) an update of a built system refills its multigrid in
 *   place and reports that in the first eight; otherwise the multigrid values
 *   are spent by the first solve after an update (or after a new
 *   right-hand-side width) */
int gdtp_system_array(const gdtp_system* s, const char* name, int level, void* out, int64_t* count);

/* Combine and coarsen: A = screen*M + stiffness*S and its Galerkin hierarchy
 * (M and S are coarsened once per level count; an update combines them).  With
 * device_factor 1 (the default) every weight-dependent value -- smoother planes,
 * boundary rows, boundary-block and coarsest-level inverses -- is recomputed on
 * the device, in place in a multigrid already built; otherwise the next solve
 * rebuilds the multigrid from host-combined coefficients.
 * Replaces UpdateLinearSystem (include/Src/UpdateCoefficients.inl:463-513),
 * UpdateMultigridCoefficients (:285-399) and UpdateMultigridSolvers (:402-439). */
int gdtp_system_update(gdtp_system* s, double stiffness_weight, double screen_weight);

/* y = A x with the raw FP64 operator (which: 0 = A, 1 = M, 2 = S).  Replaces
 * MultiplyBySystemMatrix_NoReciprocals (include/Src/IterativeSolvers.inl:881-950).
 * Host float64 buffers of numTexels*k. */
int gdtp_apply(gdtp_system* s, int which, const double* x, double* y, int k);
/* y = mass_weight M x + stiffness_weight S x (host float64 numTexels*k, one
 * upload and one download): the filtering right-hand side M f + w s S f of
 * TextureFiltering.cpp:693-700, which the reference forms with two
 * MultiplyBySystemMatrix_NoReciprocals calls (IterativeSolvers.inl:881-950). */
int gdtp_apply_mass_stiffness(gdtp_system* s, double mass_weight, double stiffness_weight, const double* x, double* y, int k);

/* One FP32 V-cycle on level-0 vectors (host float32, numTexels*k), x updated in
 * place.  Replaces VCycle (include/Src/IterativeSolvers.inl:1211-1333). */
int gdtp_vcycle(gdtp_system* s, float* x, const float* rhs, int k);
/* The same V-cycle in FP64 (host float64 numTexels*k): VCycle of the
 * reference's FP64 build (USE_FLOAT 0, IterativeSolvers.inl:1211-1333). */
int gdtp_vcycle64(gdtp_system* s, double* x, const double* rhs, int k);

/* `sweeps` Gauss-Seidel sweeps over the level-0 deep texels (host float32,
 * numTexels*k, x updated in place; boundary texels unchanged), colours in
 * order 0..3 (reverse: 3..0), with the smoother the V-cycle uses on level 0:
 * one launch per colour pass, or, when the "tile_texels" knob selects level 0,
 * the fused tile smoother (Gauss-Seidel inside 32 x 32 tiles of a chart,
 * Jacobi across tile borders).  Replaces Relaxation
 * (include/Src/IterativeSolvers.inl:174-395). */
int gdtp_relax(gdtp_system* s, float* x, const float* rhs, int k, int sweeps, int reverse);

typedef struct gdtp_report {
  int iterations;          /* outer FP64 refinement steps (or V-cycles for the plain FP64 path) */
  int vcycles;             /* total V-cycles */
  double rel_residual_max; /* max over RHS of ||b - A x||_2 / ||b||_2 with the FP64 operator */
  double seconds;          /* device time of the solve */
} gdtp_report;

/* Mixed-precision solve A x = b: FP32 V-cycles (all k right-hand sides at once)
 * inside FP64 iterative refinement, until every RHS reaches tol.  x holds the
 * initial guess on entry.  Host float64 numTexels*k.  Replaces the app loop of
 * VCycle calls (TextureFiltering.cpp:562-579) and, for accuracy, the
 * --useDirectSolver path (TextureFiltering.cpp:651-655, 704-707). */
int gdtp_solve(gdtp_system* s, const double* b, double* x, int k, double tol, int max_iters, gdtp_report* report);
/* As gdtp_solve with flags: GDTP_ZERO_GUESS starts from x = 0 and treats x as
 * output only (no host-to-device copy of x). */
#define GDTP_ZERO_GUESS 1
int gdtp_solve_ex(gdtp_system* s, const double* b, double* x, int k, double tol, int max_iters, int flags, gdtp_report* report);
/* count independent problems, each solved as gdtp_solve_ex with GDTP_ZERO_GUESS:
 * b[i] (input) and x[i] (output) host float64 numTexels*k, all k the same.
 * The upload of b[i+1] and the download of x[i-1] run on two copy streams
 * while problem i is solved, so a sequence of problems (frames of a filtering
 * session, a queue of requests) costs about the solves alone.  Pinned host
 * buffers (cudaMallocHost / cudaHostRegister) give the overlap; pageable ones
 * give the same results with the copies serialised.  No x[i] may overlap a
 * b[j].  reports: count entries, or NULL.  Returns after every x[i] is
 * written; GDTP_ERR_NOT_CONVERGED if any problem stopped above tol (its x is
 * still written).  No counterpart in the reference, which solves one problem
 * per call (TextureFiltering.cpp:562-579). */
int gdtp_solve_stream(gdtp_system* s, const double* const* b, double* const* x, int count, int k, double tol, int max_iters,
                      gdtp_report* reports);
/* Same on device float64 buffers (no host copies); stream = cudaStream_t or NULL. */
int gdtp_solve_device(gdtp_system* s, const double* b_dev, double* x_dev, int k, double tol, int max_iters,
                      void* stream, gdtp_report* report);
/* Plain FP64 V-cycles (no mixed precision) until tol: the comparator path, the
 * app loop of VCycle calls in the reference's FP64 build (USE_FLOAT 0,
 * TextureFiltering.cpp:562-579 with IterativeSolvers.inl:1211-1333) on the
 * device.  Host float64 numTexels*k; x holds the initial guess. */
int gdtp_solve_fp64(gdtp_system* s, const double* b, double* x, int k, double tol, int max_iters, gdtp_report* report);
/* Same on device float64 buffers (x_dev holds the initial guess; no host
 * copies), ordered after `stream` (cudaStream_t or NULL) like gdtp_solve_device. */
int gdtp_solve_fp64_device(gdtp_system* s, const double* b_dev, double* x_dev, int k, double tol, int max_iters, void* stream,
                           gdtp_report* report);

/* Relative residuals ||b - A x|| / ||b|| per RHS (FP64 operator), host buffers. */
int gdtp_residual(gdtp_system* s, const double* b, const double* x, int k, double* rel);

/* Residual check that allocates nothing, for callers that may not allocate
 * device memory when they need it (pre-planned render/simulation loops,
 * stream-ordered pools that must not grow, hosts where cudaMalloc would stall
 * their own work).  No counterpart in the reference.  Device buffers b_dev,
 * x_dev (inputs) and r_dev (output residual b - A x), float64 numTexels*k;
 * rel_host receives ||b - A x|| / ||b|| per right-hand side.  k <= 64: the
 * norm reduction's scratch is a fixed ~2.1 MB static device array that every
 * device loading the library holds until exit.  The first call on a device
 * resolves that array's address (cudaGetSymbolAddress) and must come before any
 * stream capture.  All calls share the array: calls that overlap on the GPU
 * race; the call waits on `stream` before returning.  The caller's current
 * device is left as it was.  Calls no cudaMalloc or cudaFree. */
int gdtp_residual_static(gdtp_system* s, const double* b_dev, const double* x_dev, double* r_dev, int k, double* rel_host,
                         void* stream);

/* Solver knobs (value as double): "pre_sweeps", "post_sweeps" (deep colour sweeps
 * per smoothing, default 3/3), "coarse_pre_sweeps", "coarse_post_sweeps" (the
 * same on levels >= "coarse_from", -1 = as the finer levels; defaults 0/3 from
 * level 1), "pre_boundary", "post_boundary" (exact boundary solve before the
 * pre / post sweeps, default 0/1), "max_block" (boundary subdomain size, 16..384,
 * next update), "max_coarse" (coarsest level size, next update),
 * "bs_blocks_per_sm" (boundary products chunked for this many blocks per SM,
 * 1..16, default 2, next update), "dense_boundary_max" (boundary blocks of at most this many
 * texels are inverted whole instead of by subdomains, 0..8192, default 0 = off,
 * next update),
 * "programmatic_launch" (0/1, default 1: V-cycle kernels overlap their launch
 * with the previous kernel's tail; process-wide), "cluster_texels" (levels up to
 * this many texels run in one thread-block cluster; default 0 = off),
 * "grid_texels" (levels up to this many texels run in one persistent kernel on
 * every SM, phases separated by grid barriers; same results as the launch
 * path; takes precedence over "cluster_texels"; 0 = off), "chart_texels"
 * (levels whose largest chart has at most this many deep texels run all sweeps
 * of a smoothing step in one launch, one block per chart with the chart's
 * texels in shared memory; same results; default 1000, 0 = off),
 * "trace_levels" (0/1: time every level's legs, arrays "profile.levels" and
 * "profile.cluster"), "krylov" (0/1, default 0: flexible preconditioned
 * conjugate gradients in FP64 around the FP32 V-cycle instead of plain
 * iterative refinement; for slowly contracting V-cycles, e.g. strongly
 * anisotropic metrics), "zero_start_skip" (0/1, default 1: the first level-0
 * sweep of a V-cycle on a zero correction reads only the neighbours it has
 * already updated, and a level entered with a zero iterate and no
 * pre-smoothing restricts its right-hand side as its residual; same results),
 * "tile_texels" (levels with at least this many deep texels smooth with the
 * fused tile smoother: 32 x 32 texel tiles of a chart, each running all sweeps
 * of a step in shared memory, tiles in four tile colours so that every tile
 * sees its neighbours' newest values; 0 = off, the default),
 * "tile_pre_sweeps", "tile_post_sweeps" (sweeps per smoothing step on tiled
 * levels, default 2/2), "tile_rounds"
 * (passes over the tiles per smoothing step, the sweeps split between them,
 * default 1), "row_sweeps" (0/1, default 1: each 4-colour sweep of an FP32
 * multigrid level of up to 4 channels whose raster lines fit a block runs as
 * two launches, both colours of a row parity per launch, the same updates bit
 * for bit; FP64 multigrids and wider batches keep the colour passes),
 * "tile_finish" (0/1: one
 * global colour sweep closes each tiled
 * smoothing step), "device_factor" (0/1, default 1: the dense FP64 inverses
 * and products of the set-up -- boundary subdomain blocks, separator Schur
 * complement, coarsest level -- run on the device by blocked Gauss-Jordan
 * elimination; 0 = host Cholesky).  "max_block", "max_coarse",
 * "dense_boundary_max", "device_factor" and "tile_texels" drop the built
 * multigrids; the next solve builds them again.  The autotuner leaves the tile smoother off: with host
 * copies running beside the solve (gdtp_solve_stream) its rounds slow down
 * more than the sweeps they replace. */
int gdtp_system_set(gdtp_system* s, const char* knob, double value);
int gdtp_system_get(const gdtp_system* s, const char* knob, double* value);
/* Autotuner: times complete solves of b (host float64 numTexels*k, uploaded
 * once; device time only) to tol for a grid of smoother settings (sweeps on the
 * finer and on the coarser levels), keeps the fastest that converges (read the
 * choice back with gdtp_system_get).  knobs_out (optional, 5 doubles): pre sweeps, post
 * sweeps, pre boundary, post boundary, best solve seconds. */
int gdtp_system_autotune(gdtp_system* s, const double* b, int k, double tol, double* knobs_out);
/* ---------------------------------------------------------------------------
 * Sharpening brush (device): the filtering app's right-hand side
 * M f + lambda sum_cells m_c S_c f for a per-cell mask m (TextureFiltering.cpp:
 * 562-570).  gdtp_brush_create keeps, for the signal f (host float64
 * numTexels*k, 1 <= k <= 4), every cell's stiffness applied to f: the four
 * cells around each deep texel, and for the boundary texels a boundary x cells
 * matrix per channel (the fine boundary rows restricted to the boundary
 * texels) -- what InitializeMassAndStiffness computes with
 * computeCellBasedStiffness (MassAndStiffness.h:490-546).
 * gdtp_brush_apply: out (numTexels*k) = sum_cells mask[cell] S_cell f, the
 * modulated stiffness; replaces CellStiffnessToTexelStiffness
 * (IterativeSolvers.inl:1170-1208).  mask: one float64 per cell in the global
 * cell order (the hierarchy's "cellCorners" rows; counts[3] cells); host
 * buffers, or device buffers ordered on `stream` for _device.  The system must
 * outlive the brush.
 * ------------------------------------------------------------------------- */
typedef struct gdtp_brush gdtp_brush;
int gdtp_brush_create(gdtp_system* s, const double* signal, int k, gdtp_brush** out);
void gdtp_brush_free(gdtp_brush* b);
int gdtp_brush_apply(gdtp_brush* b, const double* cell_mask, double* out);
int gdtp_brush_apply_device(gdtp_brush* b, const double* mask_dev, double* out_dev, void* stream);

/* ---------------------------------------------------------------------------
 * Heat-method geodesics (device).  gdtp_geodesics_create builds, for the
 * system's mesh, atlas and metric, the integration samples of the Geodesics
 * app: replaces InitializeGridAtladInteriorCellLines and
 * InitializeNormalizedVectorFieldIntegration (include/Src/VectorFieldIntergration.inl:68-73,
 * 428-437; samples per interior cell / boundary element and chart triangle,
 * computed in FP64, stored in FP32).
 * gdtp_geodesic_rhs: rhs = integral of X . grad(phi_i), X = -grad u / |grad u|
 * in the metric, boundary terms through the fine boundary nodes (prolong u,
 * integrate, restrict): replaces IntergrateNormalizedVectorFieldFromSamples
 * (VectorFieldIntergration.inl:453-582) with the boundary prolongation and
 * restriction around it (Geodesics/Geodesics.cpp:519-532).  Host float64
 * numTexels*k in and out (or device buffers, stream-ordered, for _device).
 * gdtp_geodesic_distance: the whole pipeline for k source texels (k right-hand
 * sides): (M + t S) u = delta on `smooth`, rhs, (eps M + S) d = rhs on
 * `distance` (both systems updated by the caller; the app uses eps = 1e-6,
 * Geodesics.cpp:642), d shifted to 0 at each source (Geodesics.cpp:536-547).
 * report: iterations and V-cycles of both solves summed, worst residual.
 * ------------------------------------------------------------------------- */
typedef struct gdtp_geodesics gdtp_geodesics;
int gdtp_geodesics_create(gdtp_system* s, gdtp_geodesics** out);
void gdtp_geodesics_free(gdtp_geodesics* g);
/* counts[2] = {interior-cell samples, boundary-element samples} */
int gdtp_geodesics_counts(const gdtp_geodesics* g, int64_t* counts);
/* Host copies of the samples (as float64; with out == NULL only *count):
 * "cellSamples" 16 per (interior cell, chart triangle) slot: pos(2), tensor(4),
 * v_0..v_3(8), 0, 0; "hexSamples" 20 per (boundary element, chart triangle)
 * slot: pos(2), tensor(4), v_0..v_5(12), 0, 0; "cellPtr", "corners", "slotBt", "btIdx". */
int gdtp_geodesics_array(gdtp_geodesics* g, const char* name, double* out, int64_t* count);
int gdtp_geodesic_rhs(gdtp_geodesics* g, const double* potential, double* rhs, int k);
int gdtp_geodesic_rhs_device(gdtp_geodesics* g, const double* potential_dev, double* rhs_dev, int k, void* stream);
int gdtp_geodesic_distance(gdtp_geodesics* g, gdtp_system* smooth, gdtp_system* distance, const int32_t* sources, int k, double tol,
                           int max_iters, double* distance_out, gdtp_report* report);

/* ---------------------------------------------------------------------------
 * Solve server (device).  Holds many meshes / resolutions, admits them to the
 * device under an HBM budget (idle models evicted least recently used first;
 * GDTP_ERR_BUDGET when a model cannot fit) and runs requests with `slots`
 * worker threads: queued requests of one model (same tol and max_iters, up to 16
 * right-hand sides) are solved as one batch on that model's stream while other
 * models' batches run on theirs.  Converged right-hand sides are frozen inside a
 * batch, so each result is the one the request gets alone.  Kinds:
 *   GDTP_KIND_FILTER   M + weight S, request signal f (n x k) -> solve of
 *                      M f + weight * second * S f   (TextureFiltering.cpp:693-700)
 *   GDTP_KIND_GEODESIC smoothing weight t = weight, eps = second; request = k source
 *                      texels -> distances (n x k)   (Geodesics.cpp)
 *   GDTP_KIND_LIC      parameter_metric (nt*4) required, M + weight S, request
 *                      signal f (n x 1..k) -> solve of M f  (LineIntegralConvolution.cpp:698-706)
 * The hierarchy is built by gdtp_server_add_model (host); gdtp_server_warm makes
 * a model resident now.  gdtp_server_wait blocks, copies the result (n x k) and
 * forgets the request; timing (optional, 3): {latency ms, queued ms, batch size}.
 * stats[14]: completed, failed, p50 ms, p99 ms, mean ms, texel x RHS per second,
 * batches, requests in batches, evictions, builds, resident bytes, peak bytes,
 * budget, 0.  Not a counterpart of a reference interface: the reference apps
 * solve one mesh at a time.
 * ------------------------------------------------------------------------- */
#define GDTP_KIND_FILTER 0
#define GDTP_KIND_GEODESIC 1
#define GDTP_KIND_LIC 2
typedef struct gdtp_server gdtp_server;
int gdtp_server_create(int device, int64_t hbm_budget_bytes, int slots, gdtp_server** out);
void gdtp_server_free(gdtp_server* s);
int gdtp_server_add_model(gdtp_server* s, const double* vertices, int64_t nv, const int32_t* triangles, int64_t nt, const double* uv,
                          int width, int height, int levels, int kind, double weight, double second, const double* parameter_metric,
                          int* model_out);
int gdtp_server_model_texels(gdtp_server* s, int model, int64_t* texels);
/* measured device bytes of a resident model, else the admission estimate */
int gdtp_server_model_bytes(gdtp_server* s, int model, int64_t* bytes);
int gdtp_server_warm(gdtp_server* s, int model);
int gdtp_server_submit(gdtp_server* s, int model, const double* signal, const int32_t* sources, int k, double tol, int max_iters,
                       int64_t* request_out);
int gdtp_server_poll(gdtp_server* s, int64_t request, int* done);
int gdtp_server_wait(gdtp_server* s, int64_t request, double* out, gdtp_report* report, double* timing);
int gdtp_server_stats(gdtp_server* s, double* stats);

/* Device bytes held by the system (coefficients, vectors, coarse factor). */
int gdtp_system_device_bytes(const gdtp_system* s, int64_t* bytes);

/* ---------------------------------------------------------------------------
 * Texture I/O (host; no device needed).  The apps' inputs and outputs: a
 * textured mesh (PLY), a colour or normal texture, a tangent field, and the
 * atlas padding applied before the texel grid is built
 * (TextureFiltering.cpp:807-837, LineIntegralConvolution.cpp:579-586).
 * Errors (unreadable or malformed files) return GDTP_ERR_INVALID with the
 * reason in gdtp_last_error(); the reference exits or reads garbage instead.
 * ------------------------------------------------------------------------- */
/* ReadTexturedMesh without a texture (include/Src/SimpleMesh.h:118-146): the
 * "vertex" element's x, y, z and the "face" element's vertex_indices and
 * texcoord lists, ASCII or binary (either endianness), items converted as the
 * reference's PLY library does (include/Misha/PlyFile.inl:2342-2480).  Faces
 * keep their first three corners.  With all outputs NULL only *nv and *nt are
 * written; otherwise *nv, *nt give the capacities of vertices (nv*3),
 * triangles (nt*3) and uv (nt*3*2, per corner) and receive the counts. */
int gdtp_read_textured_mesh(const char* path, int64_t* nv, int64_t* nt, double* vertices, int32_t* triangles, double* uv);
/* The name of a "comment TextureFile <name>" header line ("" if none), as
 * WriteTexturedMesh records the atlas; name NULL: *size = bytes needed. */
int gdtp_textured_mesh_texture_file(const char* path, char* name, int64_t* size);
/* WriteTexturedMesh (SimpleMesh.h:93-116): ASCII PLY with double vertices and
 * texcoords, written with 17 significant digits so that they read back
 * bit-exact (the reference prints fewer); texture_file (or NULL) goes into the
 * TextureFile comment. */
int gdtp_write_textured_mesh(const char* path, const double* vertices, int64_t nv, const int32_t* triangles, int64_t nt,
                             const double* uv, const char* texture_file);
/* Image<Point3D<float>>::read (include/Misha/Image.h:90-110) by extension:
 * ".png" through the reference's PNGReadColor transforms (PNG.inl:10-72:
 * 16-bit samples keep their high byte, 1/2/4-bit samples are unpacked without
 * rescaling, palette indices are looked up, alpha is dropped; grey is copied to
 * all three channels), each byte / 255; ".normap" as ReadBinaryImage
 * (include/Src/VectorIO.h:47-58: int32 width, int32 height, float RGB).  rgb:
 * width*height*3 floats, row 0 first (the first PNG row), pixel (i, j) at
 * 3*(j*width + i).  rgb NULL: only *width, *height; otherwise they must match
 * the file. */
int gdtp_read_image(const char* path, int* width, int* height, float* rgb);
/* Image<Point3D<float>>::write (Image.h:152-163): ".png" 8-bit RGB with each
 * value v stored as min(255, max(0, (int)(v*255 + 0.5))) in float arithmetic
 * (values beyond the int range, undefined in the reference, saturate);
 * ".normap" as WriteBinaryImage (VectorIO.h:34-45). */
int gdtp_write_image(const char* path, const float* rgb, int width, int height);
/* ReadVector / WriteVector (VectorIO.h:9-32): int32 count, then count raw
 * elements of elem_bytes each (16 for the Point2D<double> tangent fields of
 * ".vf" files).  data NULL: *count = the file's count; otherwise *count is the
 * capacity and receives the count. */
int gdtp_read_vector(const char* path, int64_t elem_bytes, int64_t* count, void* data);
int gdtp_write_vector(const char* path, int64_t elem_bytes, int64_t count, const void* data);
/* ComputePadding (include/Src/Padding.h:16-46) over n_uv (u, v) pairs:
 * padding = {left, bottom, right, top}; texture coordinates closer than half a
 * texel to the image edge grow the grid, which is then rounded up to multiples
 * of 8 by growing left and bottom (a no-op padding is all zeros).
 * GDTP_ERR_INVALID for width or height above 2^24, coordinates that are not
 * finite or beyond 1e6, or a padding beyond 2^24 texels. */
int gdtp_compute_padding(int width, int height, const double* uv, int64_t n_uv, int32_t* padding);
/* PaddTextureCoordinates / UnpaddTextureCoordinates (Padding.h:76-94) in
 * place; width, height: the unpadded image size. */
int gdtp_pad_texture_coordinates(const int32_t* padding, int width, int height, double* uv, int64_t n_uv, int unpad);
/* PaddImage (Padding.h:48-60, edge texels repeated) into out of
 * (width+left+right) x (height+bottom+top), or with unpad UnpaddImage
 * (:62-73, a crop) into out of (width-left-right) x (height-bottom-top);
 * width, height: the size of `in`. */
int gdtp_pad_image(const int32_t* padding, const float* in, int width, int height, float* out, int unpad);

#ifdef __cplusplus
}
#endif
#endif /* GDTP_H */
