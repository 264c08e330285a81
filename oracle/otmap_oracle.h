/* Test infrastructure only: a plain-C restatement of the reference otmap solver,
 * inversion and rasterizer (ggael/otmap, otlib/), used by the tests and by
 * __graft_entry__.smoke() as the checker of the CUDA library. Never linked into
 * the product.
 *
 * Conventions (same as the product C ABI, include/otmap_b200.h):
 *   n      grid size; N = n*n cells; V = (n+1)^2 vertices; e = 1/n
 *   cells  face index f = j + i*n, i = x cell index, j = y cell index
 *   verts  vertex index v = j + i*(n+1) at (i/n, j/n); xy arrays are AoS (V x 2)
 *   images row-major [y][x]
 */
#ifndef OTMAP_ORACLE_H
#define OTMAP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int beta_cj;      /* 1: BetaOpt::ConjugateJacobian, 0: BetaOpt::Zero */
  int max_iter;     /* SolverOptions::max_iter (default 1000) */
  double threshold; /* SolverOptions::threshold (default 1e-7) */
  double max_ratio; /* SolverOptions::max_ratio (default DBL_MAX) */
} oro_options;

/* otsolver_2dgrid.cpp:47-63 */
void oro_adjust_density(int n, double* density, double max_ratio);
/* otsolver_2dgrid.cpp:362-423; g is V x 2 AoS */
void oro_vertex_gradients(int n, const double* psi, double* g);
/* otsolver_2dgrid.cpp:425-447 */
void oro_face_areas(int n, const double* g, double* area);
/* otsolver_2dgrid.cpp:449-465; returns sum(r^2)/e^2 */
double oro_residual(int n, const double* psi, const double* density, double* r);
/* otsolver_2dgrid.cpp:467-539 from cached gradients g0 and direction gradients gd */
void oro_line_params(int n, const double* g0, const double* gd, double* a, double* b);
/* otsolver_2dgrid.cpp:563-595: step from the quartic coefficients z[5];
 * returns 1 if a real root in [-10,10] was picked, 0 for the 0.5 fallback */
int oro_pick_step(const double z[5], double* alpha, double* emin);
/* y = M x with M the assembled pseudo-Laplacian (otsolver_2dgrid.cpp:284-311), no pin */
void oro_laplacian_apply(int n, const double* x, double* y);
/* pseudo-inverse of M by the orthonormal 2-D DCT-II (eigenvalues 2-2cos(pi k/n)cos(pi l/n),
 * (0,0) mode dropped) followed by the mean projection of otsolver_2dgrid.cpp:179 */
void oro_poisson_dct(int n, const double* r, double* d);
/* pinned-matrix solve + mean projection exactly as otsolver_2dgrid.cpp:175-179 and :321,
 * by a dense banded Cholesky factorisation (small n only: O(n^4)) */
int oro_poisson_pinned(int n, const double* r, double* d);

/* The whole solve (otsolver_2dgrid.cpp:106-245). Outputs (any may be NULL):
 *   psi[N], fwd_xy[V*2], density_out[N] (adjusted density),
 *   trace[iters*5] = {alpha, beta, norm(d), res^2, Linf} per iteration (otsolver_2dgrid.cpp:653-659)
 * returns the iteration count; *residual gets the final residual. */
int oro_solve(int n, const double* density_in, const oro_options* opt, double* psi, double* fwd_xy,
              double* density_out, double* trace, int trace_cap, double* residual);

/* ---- inversion: BVH2D (utils/bvh2d.cpp) + TransportMap::inv_impl (transport_map.cpp:50-102) ---- */
typedef struct oro_bvh oro_bvh;
oro_bvh* oro_bvh_build(int n, const double* fwd_xy); /* bvh2d.cpp:29-64 with (4, 24) */
void oro_bvh_free(oro_bvh* b);
/* the build's final face array and, per face, the enlarged box of its leaf */
void oro_bvh_order(int n, const double* fwd_xy, int* faces_out, double* leaf_box);
/* all hits for one point (already clamped by the caller as inv_impl does); returns count,
 * writes up to cap faces / 4 weights in traversal order */
int oro_bvh_query_all(const oro_bvh* b, const double q[2], int cap, int* faces, double* bary);
/* apply_inverse_map (transport_map.cpp:105-128) on P AoS points, in place; density is the
 * map's adjusted density. face_out (optional) gets the chosen face (-1 if none). Returns the
 * number of points that had no face (the reference reads hits[0] of an empty list there). */
long oro_apply_inverse(int n, const double* fwd_xy, const double* density, double* pts, long P,
                       int* face_out, int* nhits_out);

/* ---- geometry helpers (utils/mesh_utils.cpp, utils/eigen_addons.h) ---- */
int oro_bilinear_in_quad(const double q[2], const double p[8], double* u, double* v);
int oro_bilinear_weights(const double q[2], const double p[8], double w[4]);
int oro_inside_quad(const double q[2], const double p[8]);

/* ---- rasterize_image PerFace mode (utils/rasterizer.cpp:188-236, quad faces) ----
 * density NULL = unit density (rasterizer.cpp:305-308). img row-major [rows][cols].
 * Where the bilinear solve fails (D < 0) the reference tests weights it never wrote
 * (rasterizer.cpp:193-195). stale_weights = 0 treats such pixels as outside;
 * stale_weights = 1 reuses the weights of the most recent successful solve, which
 * is what the reference's optimised build ends up reading. */
void oro_rasterize(int n, const double* xy, const double* density, int rows, int cols, int stale_weights,
                   double* img);

/* ---- rasterize_image on an indexed triangle/quad mesh, both options ----
 * (utils/rasterizer.cpp:36-58, 86-185, 188-302). mode 0 = RIO_PerVertexDensity,
 * 1 = RIO_PerFaceDensity. Face f's corners are idx[start[f] .. start[f+1]). density
 * NULL = unit density over nf faces; otherwise cells = its length (sets the scale). */
void oro_rasterize_mesh(int nv, const double* xy, int nf, const int* start, const int* idx, const double* density,
                        int cells, int rows, int cols, int mode, int stale_weights, double* img);
/* The (n+1)^2 grid's faces as an indexed face set (start[N+1], idx[4N]). */
void oro_grid_faces(int n, int* start, int* idx);
/* interpolate (apps/barycenters.cpp:250-276): out[t] = sum_k w[k] meshes[k][t]. */
void oro_mesh_blend(long V2, int count, const double* const* meshes, const double* w, double* out);
/* prune_empty_faces (utils/mesh_utils.cpp:124-141) + Surface_mesh::garbage_collection. */
int oro_prune_empty_faces(int nv, const double* xy, int nf, const int* start, const int* idx, const double* density,
                          int cells, int* nv_out, double* xy_out, int* nf_out, int* start_out, int* idx_out);

/* sample_transportmap_to_image (utils/stochastic_rasterizer.cpp:19-88) with the
 * library's counter-based generator; img row-major [rows][cols]. */
void oro_sample_image(int nv, const double* xy, int nf, const int* start, const int* idx, const int* spf,
                      unsigned long long seed, int rows, int cols, double* img);

/* GridBasedTransportSolver::compute_transport_cost (otsolver_2dgrid.cpp:608-640) of
 * vertex displacements g (V x 2 AoS); returns the sum of per_face (optional). */
double oro_grid_transport_cost(int n, const double* g, const double* density, double* per_face);

/* ---- transport_cost for an (n+1)^2 quad grid (transport_map.cpp:131-215, quad branch) ---- */
double oro_transport_cost(int n, const double* src_xy, const double* dst_xy, const double* density,
                          double* per_face);

#ifdef __cplusplus
}
#endif
#endif
