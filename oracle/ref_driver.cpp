// Test infrastructure only: a C ABI around the reference otmap library, compiled
// from the reference's own sources by oracle/Makefile into oracle/_ref/libotref.so.
//
// Nothing in the product links or loads this file. The parity tests, the golden
// fixture generator (tests/golden/make_golden.py) and the CPU arm of bench.py call
// it through ctypes to run the unmodified reference code path:
//   GridBasedTransportSolver::init/solve      otlib/otsolver_2dgrid.cpp:75-245
//   apply_inverse_map / BVH2D::query_all      otlib/transport_map.cpp:105-128, otlib/utils/bvh2d.cpp:84-92
//   rasterize_image                           otlib/utils/rasterizer.cpp:188-308
//   transport_cost                            otlib/transport_map.cpp:131-215
//   rasterize_image on indexed meshes, prune_empty_faces, Surface_mesh OFF read/write,
//   and the barycenter image of apps/barycenters.cpp:250-290
// plus unit probes of the solver's protected steps through a derived class.
//
// Buffer conventions (shared with the product C ABI):
//   per-cell arrays: face index f = j + i*n, i = x cell index, j = y cell index
//   per-vertex xy:   AoS doubles, vertex v = j + i*(n+1) at (i/n, j/n) on the origin grid
//   images:          row-major [y][x]

#include "otsolver_2dgrid.h"
#include "transport_map.h"
#include "utils/bvh2d.h"
#include "utils/mesh_utils.h"
#include "utils/rasterizer.h"
#include "utils/stochastic_rasterizer.h"

#include <xmmintrin.h>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

using namespace Eigen;
using surface_mesh::Surface_mesh;

namespace {

// Restores the caller's MXCSR: the reference solver's constructor turns on FTZ/DAZ
// for the calling thread (otsolver_2dgrid.cpp:34-39); that must not leak into the
// Python harness.
struct CsrGuard {
  unsigned int saved;
  CsrGuard() : saved(_mm_getcsr()) {}
  ~CsrGuard() { _mm_setcsr(saved); }
};

// Captures std::cout for the duration of a call.
struct CoutCapture {
  std::stringstream ss;
  std::streambuf* old;
  std::streamsize old_prec;
  CoutCapture() : old(std::cout.rdbuf(ss.rdbuf())), old_prec(std::cout.precision(17)) {}
  ~CoutCapture() {
    std::cout.rdbuf(old);
    std::cout.precision(old_prec);
  }
};

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Gives the harness access to the solver's protected steps.
struct Probe : public otmap::GridBasedTransportSolver {
  using GridBasedTransportSolver::compute_1D_problem_parameters;
  using GridBasedTransportSolver::compute_residual;
  using GridBasedTransportSolver::compute_transport_cost;
  using GridBasedTransportSolver::compute_vertex_gradients;
  using GridBasedTransportSolver::solve_1D_problem;
  void set_density(const VectorXd* d) { m_input_density = d; }
  VectorXd laplacian_solve(const VectorXd& r) {
    VectorXd d = m_laplacian_solver.solve(r);
    d.array() -= d.mean();
    return d;
  }
  void set_g0(const MatrixX2d& g) { m_cache_1D_g0 = g; }
  const MatrixX2d& g0() const { return m_cache_1D_g0; }
};

struct Solver {
  std::unique_ptr<Probe> s;
  int n = -1;
};

struct RefMap {
  std::unique_ptr<otmap::TransportMap> tmap;
  int n = 0;
};

void parse_trace(const std::string& out, double* trace, int cap, int* iters) {
  std::istringstream in(out);
  std::string line;
  int k = 0;
  while (std::getline(in, line)) {
    auto pa = line.find("alpha=");
    if (pa != std::string::npos && line.find("beta=") != std::string::npos) {
      double v[5] = {0, 0, 0, 0, 0};
      const char* keys[5] = {"alpha=", "beta=", "norm(d)=", "res^2=", "Linf="};
      for (int q = 0; q < 5; ++q) {
        auto p = line.find(keys[q]);
        if (p != std::string::npos) v[q] = std::strtod(line.c_str() + p + std::strlen(keys[q]), nullptr);
      }
      if (trace && k < cap)
        for (int q = 0; q < 5; ++q) trace[5 * k + q] = v[q];
      ++k;
    }
    auto pi = line.find("iters(");
    if (pi != std::string::npos && iters) *iters = std::atoi(line.c_str() + pi + 6);
  }
  if (trace && iters) *iters = k;
}

void load_grid_mesh(Surface_mesh& mesh, int n, const double* xy) {
  otmap::generate_quad_mesh(n + 1, n + 1, mesh);
  if (xy) {
    auto& pts = mesh.points();
    for (size_t v = 0; v < pts.size(); ++v) pts[v] = Vector2d(xy[2 * v], xy[2 * v + 1]);
  }
}

}  // namespace

extern "C" {

void* otref_solver_new() {
  CsrGuard g;
  auto* h = new Solver;
  // value-initialisation zeroes the members the reference constructor leaves unset
  h->s.reset(new Probe());
  h->s->set_verbose_level(0);
  return h;
}

void otref_solver_free(void* h) { delete static_cast<Solver*>(h); }

// GridBasedTransportSolver::init (otsolver_2dgrid.cpp:75-104). Returns wall seconds.
double otref_solver_init(void* hp, int n) {
  CsrGuard g;
  auto* h = static_cast<Solver*>(hp);
  double t0 = now_s();
  if (h->n != n) {
    // the reference's constructor leaves m_gridSize uninitialised (otsolver_2dgrid.cpp:30-40)
    // and init() returns early when it happens to equal n (:79); a value-initialised
    // (zeroed) solver per size keeps that check well defined
    h->s.reset(new Probe());
    h->s->set_verbose_level(0);
    h->s->init(n);
    h->n = n;
  }
  return now_s() - t0;
}

// GridBasedTransportSolver::solve (otsolver_2dgrid.cpp:106-245).
// trace (optional): per iteration {alpha, beta, norm(d), res^2, Linf}, as the reference
// prints them at verbose level 5 (otsolver_2dgrid.cpp:653-659), at 17 digits.
// Returns a map handle; *seconds gets the wall time of solve().
void* otref_solve(void* hp, const double* density, int beta_cj, int max_iter, double threshold,
                  double max_ratio, double* trace, int trace_cap, int* iters, double* residual,
                  double* seconds) {
  CsrGuard g;
  auto* h = static_cast<Solver*>(hp);
  int n = h->n;
  RefMap* m = new RefMap;
  m->n = n;
  otmap::SolverOptions opt;
  opt.beta = beta_cj ? otmap::BetaOpt::ConjugateJacobian : otmap::BetaOpt::Zero;
  opt.max_iter = max_iter;
  opt.threshold = threshold;
  opt.max_ratio = max_ratio;
  VectorXd dens = Map<const VectorXd>(density, (Index)n * n);
  std::string out;
  double t0, t1;
  {
    CoutCapture cap;
    h->s->set_verbose_level(trace ? 5 : 1);
    t0 = now_s();
    m->tmap.reset(new otmap::TransportMap(h->s->solve(dens, opt)));
    t1 = now_s();
    h->s->set_verbose_level(0);
    out = cap.ss.str();
  }
  if (seconds) *seconds = t1 - t0;
  int it = 0;
  parse_trace(out, trace, trace_cap, &it);
  if (iters) *iters = it;
  if (residual) {
    // " - error L2=<value>   Linf=..." (otsolver_2dgrid.cpp:235-236)
    auto p = out.rfind("error L2=");
    *residual = p == std::string::npos ? -1.0 : std::strtod(out.c_str() + p + 9, nullptr);
  }
  return m;
}

void otref_map_free(void* m) { delete static_cast<RefMap*>(m); }

// Forward mesh vertex positions, AoS (V x 2).
void otref_map_fwd(void* mp, double* xy) {
  auto* m = static_cast<RefMap*>(mp);
  const Surface_mesh& mesh = m->tmap->fwd_mesh();
  for (unsigned int v = 0; v < mesh.vertices_size(); ++v) {
    const auto& p = mesh.position(Surface_mesh::Vertex(v));
    xy[2 * v] = p[0];
    xy[2 * v + 1] = p[1];
  }
}

// The adjusted density copy the map owns (otsolver_2dgrid.cpp:121-123).
void otref_map_density(void* mp, double* d) {
  auto* m = static_cast<RefMap*>(mp);
  const VectorXd& v = m->tmap->density();
  for (Index i = 0; i < v.size(); ++i) d[i] = v[i];
}

// apply_inverse_map (transport_map.cpp:105-128) on P points, in place (AoS).
// Returns wall seconds (BVH build + queries).
double otref_apply_inverse(void* mp, double* pts, long P) {
  CsrGuard g;
  auto* m = static_cast<RefMap*>(mp);
  std::vector<Vector2d> p((size_t)P);
  for (long i = 0; i < P; ++i) p[i] = Vector2d(pts[2 * i], pts[2 * i + 1]);
  double t0 = now_s();
  {
    CoutCapture cap;
    otmap::apply_inverse_map(*m->tmap, p, 0);
  }
  double t1 = now_s();
  for (long i = 0; i < P; ++i) {
    pts[2 * i] = p[i][0];
    pts[2 * i + 1] = p[i][1];
  }
  return t1 - t0;
}

// BVH2D::query_all on the forward mesh, with the BVH built exactly as
// TransportMap::init_inverse builds it (transport_map.cpp:36-43: leaf size 4, depth 24),
// after the same clamp to [0,1]^2 (transport_map.cpp:53).
// Per point: nhits (all of them), and the first `cap` hits' faces and 4 weights in hit order.
void otref_query_all(const double* fwd_xy, int n, const double* pts, long P, int cap, int* nhits,
                     int* faces, double* bary) {
  CsrGuard g;
  Surface_mesh mesh;
  load_grid_mesh(mesh, n, fwd_xy);
  otmap::BVH2D bvh;
  bvh.build(&mesh, 4, 24);
  std::vector<otmap::BVH2D::Hit> hits;
  for (long i = 0; i < P; ++i) {
    Vector2d p = Vector2d(pts[2 * i], pts[2 * i + 1]).array().max(0.).min(1.);
    hits.clear();
    {
      CoutCapture cap_out;
      bvh.query_all(p, hits);
    }
    nhits[i] = (int)hits.size();
    for (int k = 0; k < cap; ++k) {
      faces[i * cap + k] = k < (int)hits.size() ? hits[k].face_id.idx() : -1;
      for (int q = 0; q < 4; ++q) bary[(i * cap + k) * 4 + q] = k < (int)hits.size() ? hits[k].bary_coord[q] : 0.0;
    }
  }
}

// rasterize_image (rasterizer.cpp:188-303) of a deformed (n+1)^2 grid mesh.
// density == nullptr selects the overload with unit density (rasterizer.cpp:305-308).
// img is row-major [rows][cols]. Returns wall seconds.
double otref_rasterize(const double* xy, int n, const double* density, int rows, int cols,
                       int per_vertex, double* img) {
  CsrGuard g;
  Surface_mesh mesh;
  load_grid_mesh(mesh, n, xy);
  MatrixXd im(rows, cols);
  auto opt = per_vertex ? otmap::RIO_PerVertexDensity : otmap::RIO_PerFaceDensity;
  double t0 = now_s();
  if (density) {
    VectorXd d = Map<const VectorXd>(density, (Index)n * n);
    otmap::rasterize_image(mesh, d, im, opt);
  } else {
    otmap::rasterize_image(mesh, im, opt);
  }
  double t1 = now_s();
  for (int y = 0; y < rows; ++y)
    for (int x = 0; x < cols; ++x) img[(size_t)y * cols + x] = im(y, x);
  return t1 - t0;
}

// transport_cost (transport_map.cpp:131-215) between two (n+1)^2 grid meshes.
double otref_transport_cost(const double* src_xy, const double* dst_xy, int n, const double* density,
                            double* per_face) {
  CsrGuard g;
  Surface_mesh src, dst;
  load_grid_mesh(src, n, src_xy);
  load_grid_mesh(dst, n, dst_xy);
  VectorXd d = Map<const VectorXd>(density, (Index)n * n);
  VectorXd cost;
  double c = otmap::transport_cost(src, dst, d, per_face ? &cost : nullptr);
  if (per_face)
    for (Index i = 0; i < cost.size(); ++i) per_face[i] = cost[i];
  return c;
}

// ---- unit probes of protected solver steps (solver must be init'ed to n) ----

// compute_vertex_gradients (otsolver_2dgrid.cpp:362-423). g is V x 2 AoS.
void otref_vertex_gradients(void* hp, const double* psi, double* g) {
  CsrGuard cg;
  auto* h = static_cast<Solver*>(hp);
  int n = h->n;
  VectorXd p = Map<const VectorXd>(psi, (Index)n * n);
  MatrixX2d G;
  h->s->compute_vertex_gradients(p, G);
  for (Index v = 0; v < G.rows(); ++v) {
    g[2 * v] = G(v, 0);
    g[2 * v + 1] = G(v, 1);
  }
}

// compute_residual (otsolver_2dgrid.cpp:449-465) against an (already adjusted) density.
double otref_residual(void* hp, const double* psi, const double* density, double* r) {
  CsrGuard cg;
  auto* h = static_cast<Solver*>(hp);
  int n = h->n;
  VectorXd d = Map<const VectorXd>(density, (Index)n * n);
  VectorXd p = Map<const VectorXd>(psi, (Index)n * n);
  VectorXd out((Index)n * n);
  h->s->set_density(&d);
  double res = h->s->compute_residual(p, out);
  h->s->set_density(nullptr);
  for (Index i = 0; i < out.size(); ++i) r[i] = out[i];
  return res;
}

// Pinned-Laplacian Cholesky solve plus mean projection (otsolver_2dgrid.cpp:175-179).
void otref_laplacian_solve(void* hp, const double* r, double* d) {
  CsrGuard cg;
  auto* h = static_cast<Solver*>(hp);
  int n = h->n;
  VectorXd rr = Map<const VectorXd>(r, (Index)n * n);
  VectorXd out = h->s->laplacian_solve(rr);
  for (Index i = 0; i < out.size(); ++i) d[i] = out[i];
}

// compute_1D_problem_parameters (otsolver_2dgrid.cpp:467-539) with the cached
// vertex gradients g0 taken as the exact gradients of psi.
void otref_1d_params(void* hp, const double* psi, const double* dir, double* a, double* b) {
  CsrGuard cg;
  auto* h = static_cast<Solver*>(hp);
  int n = h->n;
  VectorXd p = Map<const VectorXd>(psi, (Index)n * n);
  VectorXd dd = Map<const VectorXd>(dir, (Index)n * n);
  MatrixX2d G;
  h->s->compute_vertex_gradients(p, G);
  h->s->set_g0(G);
  VectorXd A((Index)n * n), B((Index)n * n);
  h->s->compute_1D_problem_parameters(p, dd, A, B);
  for (Index i = 0; i < A.size(); ++i) {
    a[i] = A[i];
    b[i] = B[i];
  }
}

// solve_1D_problem (otsolver_2dgrid.cpp:541-606), g0 = exact gradients of psi.
// Writes psi1, r1 and alpha; returns the new residual (rmin / e^2).
double otref_line_search(void* hp, const double* psi, const double* dir, const double* r, double ek,
                         double* psi1, double* r1, double* alpha) {
  CsrGuard cg;
  auto* h = static_cast<Solver*>(hp);
  int n = h->n;
  Index N = (Index)n * n;
  VectorXd p = Map<const VectorXd>(psi, N);
  VectorXd dd = Map<const VectorXd>(dir, N);
  VectorXd rk = Map<const VectorXd>(r, N);
  MatrixX2d G;
  h->s->compute_vertex_gradients(p, G);
  h->s->set_g0(G);
  VectorXd x1(N), rr1(N);
  double res = h->s->solve_1D_problem(p, dd, rk, ek, x1, rr1, alpha);
  for (Index i = 0; i < N; ++i) {
    psi1[i] = x1[i];
    r1[i] = rr1[i];
  }
  return res;
}

// ---- meshes other than the grid, barycenters, mesh IO ----

// Indexed face set -> Surface_mesh (add_face keeps the given circulation order).
static void load_indexed_mesh(Surface_mesh& mesh, int nv, const double* xy, int nf, const int* start,
                              const int* idx) {
  std::vector<Surface_mesh::Vertex> vs(nv);
  for (int v = 0; v < nv; ++v) vs[v] = mesh.add_vertex(surface_mesh::Point(xy[2 * v], xy[2 * v + 1]));
  std::vector<Surface_mesh::Vertex> fv;
  for (int f = 0; f < nf; ++f) {
    fv.clear();
    for (int k = start[f]; k < start[f + 1]; ++k) fv.push_back(vs[idx[k]]);
    mesh.add_face(fv);
  }
}

// rasterize_image (rasterizer.cpp:188-302) of an indexed triangle/quad mesh.
double otref_rasterize_mesh(int nv, const double* xy, int nf, const int* start, const int* idx,
                            const double* density, int cells, int rows, int cols, int per_vertex, double* img) {
  CsrGuard g;
  Surface_mesh mesh;
  load_indexed_mesh(mesh, nv, xy, nf, start, idx);
  MatrixXd im(rows, cols);
  auto opt = per_vertex ? otmap::RIO_PerVertexDensity : otmap::RIO_PerFaceDensity;
  double t0 = now_s();
  if (density) {
    VectorXd d = Map<const VectorXd>(density, (Index)cells);
    otmap::rasterize_image(mesh, d, im, opt);
  } else {
    otmap::rasterize_image(mesh, im, opt);
  }
  double t1 = now_s();
  for (int y = 0; y < rows; ++y)
    for (int x = 0; x < cols; ++x) img[(size_t)y * cols + x] = im(y, x);
  return t1 - t0;
}

// One barycenter image as apps/barycenters.cpp:250-290 forms it: the inverse meshes
// (count 4: bilinear at (alpha, beta); count 2: linear at alpha) blended vertex by
// vertex with the bilerp/lerp expressions of barycenters.cpp:127-139 (written out
// here: the app is not part of otlib), rasterized with unit density, rescaled to the
// blended density mean. Returns the expected mean.
double otref_barycenter(int n, int count, const double* const* inv, double alpha, double beta,
                        const double* means, int rows, int cols, double* mesh_out, double* img) {
  CsrGuard g;
  Surface_mesh res;
  load_grid_mesh(res, n, inv[0]);
  auto& pts = res.points();
  const double u = alpha, v = beta;
  for (size_t k = 0; k < pts.size(); ++k) {
    Vector2d a0(inv[0][2 * k], inv[0][2 * k + 1]), a1(inv[1][2 * k], inv[1][2 * k + 1]);
    if (count == 4) {
      Vector2d a2(inv[2][2 * k], inv[2][2 * k + 1]), a3(inv[3][2 * k], inv[3][2 * k + 1]);
      pts[k] = (1. - u) * (1. - v) * a0 + (u) * (1. - v) * a1 + (u) * (v)*a2 + (1. - u) * (v)*a3;
    } else {
      pts[k] = (1. - u) * a0 + u * a1;
    }
  }
  double expected = count == 4 ? (1. - u) * (1. - v) * means[0] + (u) * (1. - v) * means[1] +
                                     (u) * (v)*means[2] + (1. - u) * (v)*means[3]
                               : (1. - u) * means[0] + u * means[1];
  MatrixXd im(rows, cols);
  otmap::rasterize_image(res, im);
  im = im * (expected / im.mean());
  for (size_t k = 0; k < pts.size(); ++k) {
    mesh_out[2 * k] = pts[k][0];
    mesh_out[2 * k + 1] = pts[k][1];
  }
  for (int y = 0; y < rows; ++y)
    for (int x = 0; x < cols; ++x) img[(size_t)y * cols + x] = im(y, x);
  return expected;
}

// Mean of a rows x cols image as Eigen's MatrixXd::mean() forms it.
double otref_image_mean(const double* img, int rows, int cols) {
  MatrixXd im(rows, cols);
  for (int y = 0; y < rows; ++y)
    for (int x = 0; x < cols; ++x) im(y, x) = img[(size_t)y * cols + x];
  return im.mean();
}

// prune_empty_faces (mesh_utils.cpp:124-141) of an indexed mesh; the result is read
// back in the garbage-collected order. Outputs sized by the input (nv, nf, start[nf]).
void otref_prune(int nv, const double* xy, int nf, const int* start, const int* idx, const double* density,
                 int cells, int* nv_out, double* xy_out, int* nf_out, int* start_out, int* idx_out) {
  CsrGuard g;
  Surface_mesh mesh;
  load_indexed_mesh(mesh, nv, xy, nf, start, idx);
  VectorXd d = Map<const VectorXd>(density, (Index)cells);
  otmap::prune_empty_faces(mesh, d);
  *nv_out = (int)mesh.n_vertices();
  *nf_out = (int)mesh.n_faces();
  for (int v = 0; v < *nv_out; ++v) {
    auto p = mesh.position(Surface_mesh::Vertex(v));
    xy_out[2 * v] = p[0];
    xy_out[2 * v + 1] = p[1];
  }
  int k = 0;
  start_out[0] = 0;
  for (int f = 0; f < *nf_out; ++f) {
    for (auto v : mesh.vertices(Surface_mesh::Face(f))) idx_out[k++] = v.idx();
    start_out[f + 1] = k;
  }
}

// Surface_mesh::write (IO_off.cpp:312-380) of an indexed mesh; 1 on success.
int otref_write_off(int nv, const double* xy, int nf, const int* start, const int* idx, const char* path) {
  Surface_mesh mesh;
  load_indexed_mesh(mesh, nv, xy, nf, start, idx);
  return mesh.write(path) ? 1 : 0;
}

// Surface_mesh::read (IO_off.cpp:255-300) -> indexed arrays (capacities given).
int otref_read_off(const char* path, int cap_v, int cap_f, int cap_i, int* nv, double* xy, int* nf, int* start,
                   int* idx) {
  Surface_mesh mesh;
  if (!mesh.read(path)) return 0;
  *nv = (int)mesh.n_vertices();
  *nf = (int)mesh.n_faces();
  if (*nv > cap_v || *nf > cap_f) return -1;
  for (int v = 0; v < *nv; ++v) {
    auto p = mesh.position(Surface_mesh::Vertex(v));
    xy[2 * v] = p[0];
    xy[2 * v + 1] = p[1];
  }
  int k = 0;
  start[0] = 0;
  for (int f = 0; f < *nf; ++f) {
    for (auto v : mesh.vertices(Surface_mesh::Face(f))) {
      if (k >= cap_i) return -1;
      idx[k++] = v.idx();
    }
    start[f + 1] = k;
  }
  return 1;
}

// sample_transportmap_to_image (stochastic_rasterizer.cpp:19-88) after srand(seed).
void otref_sample_image(int nv, const double* xy, int nf, const int* start, const int* idx, const int* spf,
                        unsigned int seed, int rows, int cols, double* img) {
  CsrGuard g;
  Surface_mesh mesh;
  load_indexed_mesh(mesh, nv, xy, nf, start, idx);
  VectorXi s = Map<const VectorXi>(spf, nf);
  MatrixXd im(rows, cols);
  std::srand(seed);
  {
    CoutCapture cap;
    otmap::sample_transportmap_to_image(mesh, s, im);
  }
  for (int y = 0; y < rows; ++y)
    for (int x = 0; x < cols; ++x) img[(size_t)y * cols + x] = im(y, x);
}

// compute_transport_cost (otsolver_2dgrid.cpp:608-640) of vertex displacements g
// (V x 2 AoS) against a density; returns the sum the solver prints at verbose >= 3.
double otref_grid_transport_cost(void* hp, const double* g, const double* density, double* per_face) {
  CsrGuard cg;
  auto* h = static_cast<Solver*>(hp);
  int n = h->n;
  Index V = (Index)(n + 1) * (n + 1);
  MatrixX2d G(V, 2);
  for (Index v = 0; v < V; ++v) {
    G(v, 0) = g[2 * v];
    G(v, 1) = g[2 * v + 1];
  }
  VectorXd d = Map<const VectorXd>(density, (Index)n * n);
  VectorXd cost;
  h->s->set_density(&d);
  h->s->compute_transport_cost(G, cost);
  h->s->set_density(nullptr);
  for (Index i = 0; i < cost.size(); ++i) per_face[i] = cost[i];
  return cost.sum();
}

}  // extern "C"
