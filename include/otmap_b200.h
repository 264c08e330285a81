/* otmap_b200 -- C ABI of the B200 (sm_100a) grid optimal-transport solver.
 *
 * One shared library (libotmap_b200.so) holds the CUDA kernels and these entry
 * points. They take plain pointers and sizes only; every pointer argument may be
 * host memory or device memory of the context's GPU (the library checks which and
 * copies host buffers through the context's stream). There is no CPU fallback: a
 * context cannot be created without a CUDA device.
 *
 * Each entry point replaces one piece of the reference otmap library
 * (ggael/otmap, otlib/), cited as file:line:
 *
 *   otm_init              GridBasedTransportSolver::init           otsolver_2dgrid.h:55, otsolver_2dgrid.cpp:75-104
 *   otm_solve             GridBasedTransportSolver::solve          otsolver_2dgrid.h:58, otsolver_2dgrid.cpp:106-245
 *   otm_solve_batch       (many independent solve() calls)         apps/common/generic_tasks.cpp:57-68
 *   otm_map_create        TransportMap::TransportMap               transport_map.h:33-35, transport_map.cpp:30-34
 *   otm_map_init_inverse  TransportMap::init_inverse               transport_map.h:41, transport_map.cpp:36-43
 *   otm_map_inverse       apply_inverse_map / TransportMap::inv    transport_map.h:44,66-68, transport_map.cpp:50-128
 *   otm_map_inverse_mode  TransportMap::inv / inv_fast             transport_map.h:44-45, transport_map.cpp:50-102
 *   otm_rasterize         rasterize_image (both overloads)         utils/rasterizer.h:21-22, utils/rasterizer.cpp:188-308
 *   otm_rasterize_mode    rasterize_image with RasterImageOption   utils/rasterizer.h:16-22, utils/rasterizer.cpp:188-302
 *   otm_rasterize_mesh    rasterize_image on any tri/quad mesh     utils/rasterizer.cpp:36-185, 188-302
 *   otm_transport_cost    transport_cost                           transport_map.h:70, transport_map.cpp:131-215
 *   otm_grid_transport_cost  GridBasedTransportSolver::compute_transport_cost  otsolver_2dgrid.cpp:608-640
 *   otm_mesh_blend        interpolate (bilinear / linear blend)    apps/barycenters.cpp:127-139, 250-276
 *   otm_barycenter        interpolate + synthetize_and_save_image  apps/barycenters.cpp:250-290
 *   otm_barycenter_loss   the barycenters demo as one differentiable loss apps/barycenters.cpp:184-198, 250-290
 *   otm_sample_image      sample_transportmap_to_image             utils/stochastic_rasterizer.cpp:19-88
 *   otm_grid_faces        generate_quad_mesh's faces               utils/mesh_utils.cpp:90-122
 *   otm_write_off         Surface_mesh::write (.off)               surface_mesh/IO_off.cpp:312-380
 *   otm_read_off          Surface_mesh::read (.off)                surface_mesh/IO_off.cpp:45-300
 *   otm_prune_empty_faces prune_empty_faces                        utils/mesh_utils.cpp:124-141
 *
 * Buffer conventions (identical to the reference's in-memory layouts):
 *   n        grid size, N = n*n cells, V = (n+1)*(n+1) vertices
 *   cells    double[N], face index f = j + i*n with i the x cell index and j the
 *            y cell index (otsolver_2dgrid.h:90); a column-major n x n image
 *            (rows = y) flattened, as generic_tasks.cpp:67 passes vec(MatrixXd)
 *   vertices double[2*V] AoS (x, y), vertex v = j + i*(n+1) at (i/n, j/n) on the
 *            origin grid (otsolver_2dgrid.h:91, utils/mesh_utils.cpp:90-122);
 *            face f's corners are (i,j), (i+1,j), (i+1,j+1), (i,j+1)
 *   points   double[2*P] AoS
 *   images   double[rows*cols] row-major [y][x]
 *
 * Errors: every entry point returns an otm_status; negative values are errors
 * (nothing written to outputs), zero is success. otm_last_error() describes the
 * most recent error of the calling thread.
 */
#ifndef OTMAP_B200_H
#define OTMAP_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OTM_ABI_VERSION 1

typedef enum {
  OTM_OK = 0,
  OTM_ERR_BAD_ARG = -1,     /* invalid size, null pointer, unknown option */
  OTM_ERR_CUDA = -2,        /* a CUDA runtime call failed */
  OTM_ERR_NO_DEVICE = -3,   /* no usable CUDA device */
  OTM_ERR_TIMEOUT = -4,     /* a bounded device-side wait gave up */
  OTM_ERR_NOT_INIT = -5     /* otm_solve before otm_init for that size */
} otm_status;

/* Per-solve outcome codes reported in otm_solve_stats.outcome. The reference has
 * no error channel: solve() returns a map whatever happens (otsolver_2dgrid.cpp:244). */
typedef enum {
  OTM_CONVERGED = 0,      /* residual <= threshold */
  OTM_MAX_ITER = 1,       /* stopped at max_iter with residual > threshold */
  OTM_SMALL_STEP = 2,     /* stopped because |d_hat| <= 2*DBL_MIN (otsolver_2dgrid.cpp:182) */
  OTM_NONFINITE = 3       /* residual became NaN/Inf (the loop condition then fails, as in the reference) */
} otm_outcome;

/* otmap::BetaOpt (otsolver_2dgrid.h:33-35) */
typedef enum { OTM_BETA_ZERO = 0, OTM_BETA_CONJUGATE_JACOBIAN = 1 } otm_beta;

/* otmap::SolverOptions (otsolver_2dgrid.h:37-43). otm_default_options() fills the
 * reference defaults: ConjugateJacobian, 1000, 1e-7, DBL_MAX. */
typedef struct {
  int beta;          /* otm_beta */
  int max_iter;
  double threshold;  /* stop when sum(r^2)/e^2 <= threshold */
  double max_ratio;  /* density max/min clamp (otsolver_2dgrid.cpp:57-63) */
} otm_solver_options;

/* What one solve did. */
typedef struct {
  int iterations;
  int outcome;           /* otm_outcome */
  double residual;       /* final sum(r^2)/e^2 as the reference reports it (line-search value) */
  double linf;           /* max(r)/e^2 of the final residual vector (otsolver_2dgrid.cpp:236) */
  double initial_residual;
} otm_solve_stats;

typedef struct otm_context otm_context; /* one GPU, one CUDA stream, cached per-size tables */
typedef struct otm_map otm_map;         /* a transport map resident on the GPU */

const char* otm_last_error(void);
int otm_abi_version(void);
void otm_default_options(otm_solver_options* opt);

/* Creates a context on CUDA device `device` (its own non-blocking stream). */
int otm_create(int device, otm_context** ctx);
/* Frees the context. Every otm_map created on it must be destroyed first: a map keeps
 * using its context's device and stream, and destroying it afterwards is undefined. */
int otm_destroy(otm_context* ctx);

/* GridBasedTransportSolver::init (otsolver_2dgrid.cpp:75-104): prepares the size-n
 * tables (cosine basis, eigenvalues) and checks on the GPU that the reference's
 * assembled pseudo-Laplacian (otsolver_2dgrid.cpp:284-311) is diagonalised by that
 * basis before the cosine-transform Poisson solve is used. Cached per n. */
int otm_init(otm_context* ctx, int n);

/* GridBasedTransportSolver::solve (otsolver_2dgrid.cpp:106-245).
 *   density   cells, the raw input density (normalised here as the reference does)
 *   opt       NULL = reference defaults
 *   fwd_xy    vertices out: the forward mesh (origin grid + vertex gradients)
 *   adjusted  cells out, optional: the adjusted density the map carries
 *   stats     optional */
int otm_solve(otm_context* ctx, int n, const double* density, const otm_solver_options* opt,
              double* fwd_xy, double* adjusted, otm_solve_stats* stats);

/* `count` independent solves of possibly different sizes, run together on the GPU
 * (each with its own convergence test). Arrays of `count` entries; entries of
 * `adjusted` and `stats` may be NULL as a whole. With host output buffers, the
 * outputs of an instance that has stopped are written (on a second stream of the
 * context) while the others still iterate; the call returns once all are written. */
int otm_solve_batch(otm_context* ctx, int count, const int* n, const double* const* density,
                    const otm_solver_options* opt, double* const* fwd_xy, double* const* adjusted,
                    otm_solve_stats* stats);

/* TransportMap(origin, fwd, density) (transport_map.cpp:30-34): copies the forward
 * mesh vertices and the per-cell density to the GPU. The origin mesh is the regular
 * (n+1)^2 grid. */
int otm_map_create(otm_context* ctx, int n, const double* fwd_xy, const double* density, otm_map** map);
int otm_map_destroy(otm_map* map);
/* Builds the point-location structure (done lazily by otm_map_inverse otherwise). */
int otm_map_init_inverse(otm_map* map);

/* apply_inverse_map (transport_map.cpp:105-128): each point, clamped to [0,1]^2, is
 * located in the forward mesh; the result is the bilinear interpolation of the
 * origin grid at the located face (transport_map.cpp:50-102, same hit-selection
 * rule). points are overwritten in place.
 *   face   optional int[P]: the chosen face index, -1 where no face contains the point
 *          (the point is then set to NaN; the reference reads an empty hit list there)
 *   nhits  optional int[P]: how many faces contain the point
 *   missing optional: number of points with no face */
int otm_map_inverse(otm_map* map, double* points, long count, int* face, int* nhits, long* missing);

/* otm_map_inverse with the face choice of TransportMap::inv (OTM_INV_DENSEST, the rule
 * above) or of TransportMap::inv_fast (OTM_INV_FIRST: the first containing face and its
 * own weights, transport_map.cpp:94-98). The reference's "first" is the first in its
 * BVH traversal; here it is the lowest face index. Both agree wherever one face
 * contains the point. */
#define OTM_INV_DENSEST 0
#define OTM_INV_FIRST 1
int otm_map_inverse_mode(otm_map* map, double* points, long count, int mode, int* face, int* nhits, long* missing);

/* rasterize_image (utils/rasterizer.cpp:188-308), PerFace mode on the quad mesh of
 * an (n+1)^2 grid whose vertex positions are `xy`: each pixel whose centre lies in a
 * face (bilinear coordinates in [0,1]) gets float(1/N) * density[f] / |area f|, the
 * highest face index winning as in the reference's sequential loop. density NULL =
 * unit density (rasterizer.cpp:305-308). img receives rows*cols doubles. */
int otm_rasterize(otm_context* ctx, int n, const double* xy, const double* density, int rows, int cols,
                  double* img);
/* The face each pixel of the PerFace raster of the (n+1)^2 grid mesh xy takes its value
 * from (rows x cols ints, [y][x]; -1 where no face covers the pixel centre): the highest
 * face index accepting the pixel, as rasterize_image's sequential loop leaves it
 * (rasterizer.cpp:162-236). No counterpart in the reference; the differentiable
 * barycenter loss holds this ownership fixed. */
int otm_rasterize_faces(otm_context* ctx, int n, const double* xy, int rows, int cols, int* face);

/* rasterize_image's RasterImageOption (utils/rasterizer.h:16-19). */
#define OTM_RIO_PER_VERTEX 0
#define OTM_RIO_PER_FACE 1

/* rasterize_image (utils/rasterizer.cpp:188-302) of the (n+1)^2 grid mesh `xy` with
 * either option. OTM_RIO_PER_FACE is otm_rasterize. OTM_RIO_PER_VERTEX gives each
 * vertex float(1/N) * (float sum of 1/|area| over its faces, in face order) / (its
 * face count), and each covered pixel of the winning face the float sum over the
 * face's corners of (vertex 0's value * float(weight)) -- the reference's
 * interpolation reads vertex 0 for every corner (rasterizer.cpp:177). The density
 * values are not used by that option; only their count sets the scale. */
int otm_rasterize_mode(otm_context* ctx, int n, const double* xy, const double* density, int rows, int cols,
                       int mode, double* img);

/* rasterize_image on an indexed face set of triangles and quads (the reference's
 * Surface_mesh overload for meshes other than the grid, e.g. after
 * prune_empty_faces): nv vertices xy[2*nv]; face f has corners
 * face_vertices[face_start[f] .. face_start[f+1]) (3 or 4, face_start[0] = 0) in
 * circulation order. density[cells] per face (cells >= nf; its length sets the
 * scale float(1/cells)), NULL = unit density over the nf faces. Triangles use the
 * barycentric transform of rasterizer.cpp:36-58, quads the bilinear coordinates. */
int otm_rasterize_mesh(otm_context* ctx, int nv, const double* xy, int nf, const int* face_start,
                       const int* face_vertices, const double* density, int cells, int rows, int cols, int mode,
                       double* img);

/* transport_cost (transport_map.cpp:131-215) between the (n+1)^2 grid meshes src_xy
 * and dst_xy with per-cell density (a quad mesh with as many faces as cells, so the
 * reference takes its per-triangle branch on each face's circulation (v3, v0, v1)).
 *   per_face  optional double[N]: density*area*cost of each face / the integral
 *   cost      out: sum(per-face costs) / integral(density*area)
 * Per-face terms are computed as the reference computes them; the two sums are
 * fixed-order tree reductions (the reference sums sequentially), so cost and the
 * normalised per-face values agree to a few ulps. */
int otm_transport_cost(otm_context* ctx, int n, const double* src_xy, const double* dst_xy, const double* density,
                       double* per_face, double* cost);

/* GridBasedTransportSolver::compute_transport_cost (otsolver_2dgrid.cpp:608-640), the
 * cost the solver reports at verbose level 3: per face, density * e^2 * the mean over
 * the 2x2 Gauss points of |bilinear interpolation of the corner displacements|^2.
 *   grads_xy  vertices: displacement of each grid vertex (the solver's vertex
 *             gradients; fwd_xy - origin recovers them to one rounding)
 *   per_face  optional double[N] out; total out: their sum (fixed-order tree sum;
 *             the reference's Eigen sum orders its additions differently) */
int otm_grid_transport_cost(otm_context* ctx, int n, const double* grads_xy, const double* density,
                            double* per_face, double* total);

/* interpolate (apps/barycenters.cpp:250-276): out = sum_k weights[k] * meshes[k],
 * accumulated left to right per coordinate, as bilerp/lerp (barycenters.cpp:127-139)
 * evaluate it. Bilinear barycenters of four maps at (alpha, beta) use weights
 * ((1-a)(1-b), a(1-b), a b, (1-a) b); linear ones of two maps (1-a, a).
 * count <= 64 meshes of 2*(n+1)^2 doubles each. */
int otm_mesh_blend(otm_context* ctx, int n, int count, const double* const* meshes, const double* weights,
                   double* out);

/* One barycenter image (apps/barycenters.cpp:250-290): blends the inverse meshes as
 * otm_mesh_blend, rasterizes the blend with unit density (PerFace, rows x cols) and
 * rescales it by expected_mean / mean(image) (synthetize_and_save_image,
 * barycenters.cpp:280-290). mesh_out (optional) receives the blended mesh,
 * raster_mean (optional) the mean of the image before rescaling. */
int otm_barycenter(otm_context* ctx, int n, int count, const double* const* inv_meshes, const double* weights,
                   double expected_mean, int rows, int cols, double* mesh_out, double* img, double* raster_mean);

/* sample_transportmap_to_image (utils/stochastic_rasterizer.cpp:19-88): draws
 * samples_per_face[f] random points in each face f -- uniform bilinear coordinates
 * (u, v) in a quad, uniform barycentric coordinates (1-sqrt(r1), sqrt(r1)(1-r2),
 * sqrt(r1) r2) in a triangle, mapped through the face's corners as the reference maps
 * them -- and counts them in img[rows*cols] (row-major [y][x]; pixel (int(y/dy),
 * int(x/dx))); points off the unit square are dropped. The mesh is the (grid_n+1)^2
 * grid (grid_n > 0: nv, nf must match, the face arrays are ignored) or an indexed
 * triangle/quad mesh (grid_n = 0). The random numbers come from a counter-based
 * generator keyed by (seed, face, sample), so an image is reproducible from its seed;
 * the reference draws from the process-wide std::rand() stream instead, so its images
 * agree with these in distribution, not sample by sample. */
int otm_sample_image(otm_context* ctx, int nv, const double* xy, int nf, const int* face_start,
                     const int* face_vertices, int grid_n, const int* samples_per_face, unsigned long long seed,
                     int rows, int cols, double* img);

/* ---- meshes as indexed face sets, OFF files (host-side; no device needed) ----
 *
 * A mesh other than the grid is nv vertices xy[2*nv] and nf faces; face f's corners
 * are face_vertices[face_start[f] .. face_start[f+1]) (face_start[0] = 0) in the
 * order the reference's face circulator visits them. */

/* The faces of the (n+1)^2 grid mesh (utils/mesh_utils.cpp:110-121): face_start[N+1],
 * face_vertices[4N], face f = j + i*n with corners (i,j), (i+1,j), (i+1,j+1), (i,j+1). */
int otm_grid_faces(int n, int* face_start, int* face_vertices);

/* Writes an ASCII OFF file byte for byte as Surface_mesh::write does for these meshes
 * (surface_mesh/IO_off.cpp:312-380): "OFF", "nv nf 0", one "%.10f %.10f %.10f" line
 * per vertex (z = 0, surface_mesh/types.h:50), one "valence i0 i1 ..." line per face. */
int otm_write_off(const char* path, int nv, const double* xy, int nf, const int* face_start,
                  const int* face_vertices);

/* Reads an OFF file as Surface_mesh::read does (surface_mesh/IO_off.cpp:45-300):
 * [ST][C][N]OFF headers, ASCII or BINARY; z and per-vertex normals, colours and
 * texture coordinates are dropped. Call with xy == NULL to get *nv, *nf and *nidx (the
 * total corner count); call again with arrays of at least those sizes (*nv, *nf,
 * *nidx hold the capacities on input). Faces are taken as listed (the reference's
 * add_face also rejects non-manifold faces; such files are not supported). */
int otm_read_off(const char* path, int* nv, int* nf, int* nidx, double* xy, int* face_start, int* face_vertices);

/* prune_empty_faces (utils/mesh_utils.cpp:124-141): removes the faces whose density is
 * 0 (a mesh with nf = 2*cells is a triangulated grid: face f reads cell f/2), then the
 * vertices left without a face, and renumbers both in the order
 * Surface_mesh::garbage_collection leaves them (surface_mesh/Surface_mesh.cpp:1975-2110:
 * each hole, front to back, takes the last survivor). Outputs are sized like the
 * inputs (start_out nf+1); *nv_out and *nf_out receive the kept counts. */
int otm_prune_empty_faces(int nv, const double* xy, int nf, const int* face_start, const int* face_vertices,
                          const double* density, int cells, int* nv_out, double* xy_out, int* nf_out,
                          int* start_out, int* idx_out);

/* ---- implicit adjoint (no counterpart in the reference, which has no derivatives) ----
 *
 * Gradient of a loss of the forward mesh with respect to the raw input density, for a
 * map produced by otm_solve on that density. With F(psi, rho~) = A(psi) - e^2 rho~ the
 * converged residual (otsolver_2dgrid.cpp:449-465), dL/drho~ = e^2 lambda where
 * J^T lambda = G^T dL/dfwd (J = dA/dpsi, G the vertex-gradient operator, both applied
 * matrix-free on the GPU), chained through the normalisation of
 * otsolver_2dgrid.cpp:53-55 (the max_ratio clamp must be inactive).
 *   OTM_ADJOINT_ONE_STEP  lambda = -M^+ G^T dL/dfwd: one cosine-transform Poisson solve
 *                         (M the reference's pseudo-Laplacian, J = -M at psi = 0)
 *   OTM_ADJOINT_KRYLOV    restarted GMRES on J^T, right-preconditioned by M^+, until the
 *                         relative residual is <= tol (or max_iter Poisson solves); each
 *                         restart cycle runs on the device (one graph launch under
 *                         OTM_LOOP_GRAPH, the same kernels step by step under
 *                         OTM_LOOP_HOST, with identical results) */
#define OTM_ADJOINT_ONE_STEP 0
#define OTM_ADJOINT_KRYLOV 1
typedef struct {
  int mode;
  double tol;
  int max_iter;  /* Poisson solves at most */
  int restart;   /* Krylov basis size before a restart */
} otm_adjoint_options;
typedef struct {
  int iterations;            /* Poisson solves used */
  double relative_residual;  /* |G^T q - J^T lambda| / |G^T q| (Krylov mode; -1 in one-step mode) */
} otm_adjoint_stats;
void otm_default_adjoint_options(otm_adjoint_options* opt); /* Krylov, tol 1e-10, 2000 solves, restart 40 */
/*   density    cells: the raw density given to otm_solve
 *   fwd_xy     vertices: the forward mesh otm_solve returned
 *   grad_fwd   vertices: dL/dfwd (x, y per vertex)
 *   grad_density cells out: dL/ddensity */
int otm_adjoint(otm_context* ctx, int n, const double* density, const double* fwd_xy, const double* grad_fwd,
                const otm_adjoint_options* opt, double* grad_density, otm_adjoint_stats* stats);

/* ---- differentiable barycenter image (no counterpart in the reference for the gradient;
 * the forward pass is apps/barycenters.cpp:184-198 and 250-290) ----
 *
 * The pipeline of the barycenters demo for `count` (<= 8) densities of one grid size n:
 * their transport maps in one batched solve, each map's inverse at the (n+1)^2 origin grid
 * vertices (apply_inverse_map of the origin mesh, barycenters.cpp:190), the blend of the
 * inverse meshes with `weights` (bilerp / lerp: otm_mesh_blend), its PerFace raster with
 * unit density at res x res, rescaled to expected = sum_k w_k mean(density_k)
 * (synthetize_and_save_image) -> image ([y][x], optional), and the loss
 * L = sum_pixels (image - target)^2 (target [y][x], res x res).
 * With grad_density non-null, also dL/ddensity_k (cells) for every k: through the image
 * rescale, each face's area in the raster (pixel ownership held fixed: it is piecewise
 * constant in the mesh), the blend, the bilinear inversion (the origin point held fixed in
 * the located face) and otm_adjoint of each map (aopt; NULL = defaults), plus the
 * expected-mean term. Buffers may be host or device memory. The maps' adjoints run
 * concurrently: map 0 on ctx, the others on helper contexts of the same device that ctx
 * creates on first use (count - 1 of them, each with its own stream, adjoint workspace and
 * size tables) and keeps until otm_destroy, one host thread per map for the call's
 * duration. */
typedef struct {
  int iterations[8];
  int outcome[8];
  double residual[8];
  long inverse_missing;  /* origin vertices located in no face, over all maps */
  double expected_mean;  /* sum_k w_k mean(density_k) */
  double raster_mean;    /* mean of the raster before rescaling */
  int adjoint_solves[8]; /* Poisson solves of each map's adjoint (gradient only) */
  double adjoint_residual[8]; /* final relative residual of each map's Krylov adjoint (-1: one-step) */
} otm_barycenter_stats;
int otm_barycenter_loss(otm_context* ctx, int n, int count, const double* const* density, const double* weights,
                        int res, const double* target, const otm_solver_options* opt, const otm_adjoint_options* aopt,
                        double* image, double* loss, double* const* grad_density, otm_barycenter_stats* stats);

/* Context options (no counterpart in the reference).
 *   OTM_OPT_POISSON: how d_hat = M^+ r is computed.
 *     OTM_POISSON_AUTO  (default) fast cosine transform for power-of-two n in [8, 4096],
 *                       dense products otherwise
 *     OTM_POISSON_DENSE C.X.C^T products with the cosine basis, any n
 *     OTM_POISSON_FFT   fast transform where possible (same as AUTO)
 *     OTM_POISSON_TENSOR split-precision instances of n in {128, 256, 512, 1024}: the
 *                       four products C.R.C^T and C^T.Y.C on the tensor cores (tcgen05,
 *                       3xTF32 with FP32 accumulation); other instances as AUTO */
#define OTM_OPT_POISSON 1
#define OTM_POISSON_AUTO 0
#define OTM_POISSON_DENSE 1
#define OTM_POISSON_FFT 2
#define OTM_POISSON_TENSOR 3
/*   OTM_OPT_LOOP: how the iteration loop is driven.
 *     OTM_LOOP_GRAPH (default) one CUDA graph launch per solve: the iteration kernels sit
 *                    in the body of a device-side WHILE node that stops when no instance
 *                    is active (no host round trip between iterations)
 *     OTM_LOOP_HOST  kernels launched from the host, loop test read back every 4
 *                    iterations (used while per-kernel profiling is on) */
#define OTM_OPT_LOOP 2
#define OTM_LOOP_GRAPH 0
#define OTM_LOOP_HOST 1
/*   OTM_OPT_WAIT_TEST: exercises the bounded device-side waits (for tests). Every wait
 *     of the row transforms (a bulk copy completing on an mbarrier) is bounded; when one
 *     runs out, the instance is flagged and stopped and the call returns OTM_ERR_TIMEOUT,
 *     leaving the context usable. With value 1 those waits expect 16 bytes more than
 *     their copy brings and give up after about 1 ms, so the path runs on demand;
 *     0 (default) restores normal operation. */
#define OTM_OPT_WAIT_TEST 3
/*   OTM_OPT_PRECISION: the arithmetic of the iteration.
 *     OTM_PRECISION_FP64  (default) every per-cell array and operation in FP64: the
 *                         reference's arithmetic (same iteration counts, positions within
 *                         1e-6 of the reference's)
 *     OTM_PRECISION_SPLIT for n a power of two in [64, 1024] (other sizes stay FP64):
 *                         r, d_hat, d and the cosine transforms in FP32; the potential,
 *                         every product entering the line-search sums, the sums, beta,
 *                         the quartic and its root, the residual and the mean-zero
 *                         projection in FP64. Positions within 1e-5 of the reference's,
 *                         same stopping threshold on the same tracked residual. */
#define OTM_OPT_PRECISION 4
#define OTM_PRECISION_FP64 0
#define OTM_PRECISION_SPLIT 1
/* Strip height of the two stencil sweeps of a batch configuration (its list of sizes,
 * Poisson mode and precision): OTM_AUTOTUNE_OFF (default) takes it from a fixed rule (64
 * rows when the batch has many 32-row blocks per SM, 16 when it has fewer than the SMs,
 * else 32); OTM_AUTOTUNE_ON times a few iterations of the first call's own densities at
 * each of 16, 32 and 64 rows (host-driven loop, CUDA events) and keeps the fastest for
 * that configuration (the real solve then starts from the same initial state). The strip
 * height changes the order of the partial sums, so results can differ from the untuned
 * configuration's at the last bits. */
#define OTM_OPT_AUTOTUNE 5
#define OTM_AUTOTUNE_OFF 0
#define OTM_AUTOTUNE_ON 1
/* Read-only: the strip height used by the context's last solve call. */
#define OTM_INFO_STRIP_ROWS 6
int otm_set_option(otm_context* ctx, int key, int value);
/* Current value of an option, or OTM_INFO_STRIP_ROWS. */
int otm_get_option(otm_context* ctx, int key, int* value);

/* ---- allocation-free solve (no counterpart in the reference) ----
 *
 * For callers that cannot let a library call cudaMalloc: hosts whose own allocator has
 * reserved all device memory up front (a framework's caching pool, an inference server
 * that partitions HBM at start-up) and processes under a hard device-memory budget, where
 * a cudaMalloc in the middle of a run can fail or evict something the host owns.
 * otm_solve_noalloc does what otm_solve does for one density but allocates nothing: its
 * working memory is a fixed 8 MiB array in the library's device data, which every GPU
 * that loads the library holds until the process exits. Hence the size limit:
 * n <= OTM_NOALLOC_MAX_N (larger n is rejected with OTM_ERR_BAD_ARG).
 *   - It runs the dense-product Poisson solve (C.X.C^T with the cosine basis, O(n^3) work
 *     per iteration) and the one-tile-per-block stencil kernels, not the fast transforms
 *     and fused sweeps of otm_solve; results agree with otm_solve to the solver's
 *     tolerance (same iteration count, positions within 1e-6), not bit for bit.
 *   - Runs on the calling thread's current device, on `stream` (a cudaStream_t;
 *     NULL = the legacy default stream), and returns when the result is written.
 *   - Buffers may be host or device memory, as for otm_solve; no context needed.
 *   - It is not for use while `stream` is being captured into a CUDA graph: it copies
 *     from host memory, synchronises the stream and reads the loop state back to the
 *     host every 4 iterations, none of which a capture allows.
 *   - The first call on each device looks up the array's device address and checks
 *     the cosine basis against the assembled matrix for that n.
 *   - All calls on a device share the one array (it keeps the last call's contents;
 *     each call re-initialises what must start at zero): calls that overlap on the
 *     GPU -- from two threads, or on two streams -- race and give wrong results.
 *     Serialise them. */
#define OTM_NOALLOC_MAX_N 256
int otm_solve_noalloc(int n, const double* density, const otm_solver_options* opt, double* fwd_xy,
                      double* adjusted, otm_solve_stats* stats, void* stream);

/* ---- instrumentation (no counterpart in the reference, which times its phases
 * with BenchTimer, otsolver_2dgrid.cpp:153-217) ---- */

/* The context's CUDA stream (a cudaStream_t), for callers that record their own
 * events around otm_* calls; every otm_* call has finished on it when it returns. */
int otm_stream(otm_context* ctx, void** stream);
/* Kernels this context has launched since it was created. */
long otm_launch_count(otm_context* ctx);
/* enable = 1 / 0 turns per-kernel CUDA-event timing on / off; -1 resets the totals. */
int otm_profile(otm_context* ctx, int enable);
/* Reads entry `index` of the per-kernel totals: kernel name, total ms, launches.
 * Returns 0 past the last entry. */
int otm_profile_entry(otm_context* ctx, int index, const char** name, double* ms, long* launches);

#ifdef __cplusplus
}
#endif
#endif
