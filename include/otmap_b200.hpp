// otmap_b200.hpp -- C++ drop-in for the public API of the reference otmap library
// (namespace otmap: otlib/otsolver_2dgrid.h, otlib/transport_map.h,
// otlib/utils/rasterizer.h, otlib/utils/mesh_utils.h), header-only, over the C ABI of
// otmap_b200.h. Link with -lotmap_b200.
//
// Same names, argument meaning and results as the reference, with these differences:
//   * Types. When <Eigen/Core> is on the include path (and OTMAP_B200_NO_EIGEN is not
//     defined) densities are Eigen::VectorXd, images Eigen::MatrixXd (rows = y) and
//     points Eigen::Vector2d, as in the reference. Otherwise they are the plain
//     containers otmap::Vector, otmap::Image (column-major, rows = y) and
//     std::array<double, 2>. Either way a point is two contiguous doubles.
//   * Meshes. otmap::Mesh stands in for surface_mesh::Surface_mesh: vertex positions
//     (points(), position(v)) and faces as corner lists in circulation order, with the
//     OFF read/write of the reference (write(), read()). Solver meshes are the
//     (n+1)^2 grid, vertex v = j + i*(n+1).
//   * Errors. The reference has no error channel; solve() always returns a map and so
//     does this one, whatever the outcome (last_stats() tells which). Invalid
//     arguments and CUDA failures, which the reference would turn into undefined
//     behaviour, throw std::runtime_error with the library's message.
//   * The solver does not change the calling thread's floating-point control state
//     (the reference sets FTZ/DAZ in its constructor, otsolver_2dgrid.cpp:34-39).
//   * Copies of a TransportMap share its device point-location structure (the
//     reference's copies share a raw BVH pointer and double-free it).
#pragma once

#include <array>
#include <cstdio>
#include <iostream>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "otmap_b200.h"

#if !defined(OTMAP_B200_NO_EIGEN) && defined(__has_include)
#if __has_include(<Eigen/Core>)
#include <Eigen/Core>
#define OTMAP_B200_EIGEN 1
#endif
#endif

namespace otmap {

#ifdef OTMAP_B200_EIGEN
using Point = Eigen::Vector2d;
using Vector = Eigen::VectorXd;
using IndexVector = Eigen::VectorXi;
using Image = Eigen::MatrixXd;
inline Vector make_vector(long n, double value = 0.0) { return Vector::Constant(n, value); }
#else
using Point = std::array<double, 2>;
using Vector = std::vector<double>;
using IndexVector = std::vector<int>;
// Column-major image with rows = y, like the reference's Eigen::MatrixXd.
class Image {
 public:
  Image() = default;
  Image(long rows, long cols) : rows_(rows), cols_(cols), data_((size_t)(rows * cols), 0.0) {}
  long rows() const { return rows_; }
  long cols() const { return cols_; }
  long size() const { return rows_ * cols_; }
  double& operator()(long y, long x) { return data_[(size_t)(x * rows_ + y)]; }
  double operator()(long y, long x) const { return data_[(size_t)(x * rows_ + y)]; }
  double* data() { return data_.data(); }
  const double* data() const { return data_.data(); }
  double mean() const {
    double s = 0;
    for (double v : data_) s += v;
    return s / (double)data_.size();
  }

 private:
  long rows_ = 0, cols_ = 0;
  std::vector<double> data_;
};
inline Vector make_vector(long n, double value = 0.0) { return Vector((size_t)n, value); }
#endif
static_assert(sizeof(Point) == 2 * sizeof(double), "a point must be two contiguous doubles");

namespace detail {

inline void check(int status, const char* what) {
  if (status < 0) throw std::runtime_error(std::string(what) + ": " + otm_last_error());
}

// One GPU context (device, stream, cached per-size tables).
class Context {
 public:
  explicit Context(int device) { check(otm_create(device, &h_), "otm_create"); }
  ~Context() {
    if (h_) otm_destroy(h_);
  }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  otm_context* get() const { return h_; }

 private:
  otm_context* h_ = nullptr;
};

inline std::shared_ptr<Context> default_context() {
  static std::shared_ptr<Context> ctx = std::make_shared<Context>(0);
  return ctx;
}

// Copies a row-major [y][x] buffer into an image (rows = y).
inline void from_row_major(const std::vector<double>& buf, Image& img) {
  const long rows = img.rows(), cols = img.cols();
  for (long y = 0; y < rows; ++y)
    for (long x = 0; x < cols; ++x) img(y, x) = buf[(size_t)(y * cols + x)];
}

}  // namespace detail

// otsolver_2dgrid.h:33-43
enum struct BetaOpt { Zero, ConjugateJacobian };

struct SolverOptions {
  BetaOpt beta = BetaOpt::ConjugateJacobian;
  int max_iter = 1000;
  double threshold = 1e-7;
  double max_ratio = std::numeric_limits<double>::max();
};

// utils/rasterizer.h:16-19
enum RasterImageOption { RIO_PerVertexDensity = OTM_RIO_PER_VERTEX, RIO_PerFaceDensity = OTM_RIO_PER_FACE };

// Stand-in for surface_mesh::Surface_mesh: vertex positions and faces (3 or 4 corners
// for the rasterizer; any valence for file IO) in circulation order.
class Mesh {
 public:
  Mesh() = default;

  // generate_quad_mesh(n+1, n+1) (utils/mesh_utils.cpp:90-122): the (n+1)^2 grid.
  static Mesh grid(int n) {
    Mesh m;
    m.grid_n_ = n;
    m.pts_.resize((size_t)(n + 1) * (n + 1));
    const double dx = 1. / double(n);
    for (int i = 0; i <= n; ++i)
      for (int j = 0; j <= n; ++j) m.pts_[(size_t)(j + i * (n + 1))] = Point{double(i) * dx, double(j) * dx};
    m.start_.assign((size_t)n * n + 1, 0);
    m.idx_.resize((size_t)4 * n * n);
    detail::check(otm_grid_faces(n, m.start_.data(), m.idx_.data()), "otm_grid_faces");
    return m;
  }

  std::vector<Point>& points() { return pts_; }
  const std::vector<Point>& points() const { return pts_; }
  Point& position(int v) { return pts_[(size_t)v]; }
  const Point& position(int v) const { return pts_[(size_t)v]; }
  int n_vertices() const { return (int)pts_.size(); }
  int vertices_size() const { return n_vertices(); }
  int n_faces() const { return (int)start_.size() - 1; }
  int faces_size() const { return n_faces(); }
  int valence(int f) const { return start_[(size_t)f + 1] - start_[(size_t)f]; }
  const int* face_vertices(int f) const { return idx_.data() + start_[(size_t)f]; }
  const std::vector<int>& face_start() const { return start_; }
  const std::vector<int>& face_indices() const { return idx_; }
  // n for the solver's (n+1)^2 grid mesh (whatever the positions), 0 otherwise.
  int grid_size() const { return grid_n_; }

  int add_vertex(const Point& p) {
    grid_n_ = 0;
    pts_.push_back(p);
    return (int)pts_.size() - 1;
  }
  int add_face(const std::vector<int>& corners) {
    grid_n_ = 0;
    idx_.insert(idx_.end(), corners.begin(), corners.end());
    start_.push_back((int)idx_.size());
    return n_faces() - 1;
  }
  void clear() { *this = Mesh(); }

  // Surface_mesh::write / read for .off (surface_mesh/IO_off.cpp).
  bool write(const std::string& path) const {
    return otm_write_off(path.c_str(), n_vertices(), raw(), n_faces(), start_.data(), idx_.data()) == OTM_OK;
  }
  bool read(const std::string& path) {
    int nv = 0, nf = 0, ni = 0;
    if (otm_read_off(path.c_str(), &nv, &nf, &ni, nullptr, nullptr, nullptr) != OTM_OK) return false;
    Mesh m;
    m.pts_.resize((size_t)nv);
    m.start_.assign((size_t)nf + 1, 0);
    m.idx_.resize((size_t)(ni > 0 ? ni : 1));
    if (otm_read_off(path.c_str(), &nv, &nf, &ni, reinterpret_cast<double*>(m.pts_.data()), m.start_.data(),
                     m.idx_.data()) != OTM_OK)
      return false;
    m.idx_.resize((size_t)ni);
    *this = std::move(m);
    return true;
  }

  const double* raw() const { return reinterpret_cast<const double*>(pts_.data()); }
  double* raw() { return reinterpret_cast<double*>(pts_.data()); }

 private:
  friend void prune_empty_faces(Mesh& mesh, const Vector& density);
  std::vector<Point> pts_;
  std::vector<int> start_{0};
  std::vector<int> idx_;
  int grid_n_ = 0;
};

// transport_map.h:29-63
class TransportMap {
 public:
  TransportMap(std::shared_ptr<Mesh> origin_mesh, std::shared_ptr<Mesh> fwd_mesh, std::shared_ptr<Vector> density,
               std::shared_ptr<detail::Context> ctx = nullptr)
      : origin_(std::move(origin_mesh)),
        fwd_(std::move(fwd_mesh)),
        density_(std::move(density)),
        ctx_(ctx ? std::move(ctx) : detail::default_context()),
        loc_(std::make_shared<Locator>()) {}

  // Must be called once before inv / inv_fast (transport_map.cpp:36-43).
  void init_inverse() const {
    ensure_map();
    detail::check(otm_map_init_inverse(loc_->m), "init_inverse");
  }
  Point inv(const Point& p) const { return inv_impl(p, false); }
  Point inv_fast(const Point& p) const { return inv_impl(p, true); }

  // All points at once, in place; returns how many had no face.
  long inverse(Point* points, long count, bool fast = false) const {
    ensure_map();
    long missing = 0;
    detail::check(otm_map_inverse_mode(loc_->m, reinterpret_cast<double*>(points), count,
                                       fast ? OTM_INV_FIRST : OTM_INV_DENSEST, nullptr, nullptr, &missing),
                  "apply_inverse_map");
    return missing;
  }

  std::shared_ptr<Mesh> fwd_mesh_ptr() { return fwd_; }
  std::shared_ptr<Vector> density_ptr() { return density_; }
  const Mesh& origin_mesh() const { return *origin_; }
  const Mesh& fwd_mesh() const { return *fwd_; }
  const Vector& density() const { return *density_; }
  const std::shared_ptr<detail::Context>& context() const { return ctx_; }

 private:
  struct Locator {
    otm_map* m = nullptr;
    ~Locator() {
      if (m) otm_map_destroy(m);
    }
  };
  void ensure_map() const {
    if (loc_->m) return;
    const int n = fwd_->grid_size();
    if (n < 1) throw std::runtime_error("TransportMap: the forward mesh is not the solver's grid mesh");
    detail::check(otm_map_create(ctx_->get(), n, fwd_->raw(), density_->data(), &loc_->m), "TransportMap");
  }
  Point inv_impl(const Point& p, bool fast) const {
    Point q = p;
    inverse(&q, 1, fast);
    return q;
  }

  std::shared_ptr<Mesh> origin_, fwd_;
  std::shared_ptr<Vector> density_;
  std::shared_ptr<detail::Context> ctx_;
  std::shared_ptr<Locator> loc_;  // shared by copies, freed with the last one
};

// otsolver_2dgrid.h:45-125
class GridBasedTransportSolver {
 public:
  explicit GridBasedTransportSolver(int device = 0)
      : ctx_(device == 0 ? detail::default_context() : std::make_shared<detail::Context>(device)) {}

  // adjust the amount of information sent to std::cout
  void set_verbose_level(int v) { verbose_ = v; }

  // Prepares the size-n tables (otsolver_2dgrid.cpp:75-104); cached per n.
  void init(int n) {
    if (verbose_ >= 1) std::cout << "Init solver...\n";
    detail::check(otm_init(ctx_->get(), n), "init");
    n_ = n;
    origin_ = std::make_shared<Mesh>(Mesh::grid(n));
  }

  // otsolver_2dgrid.cpp:106-245: density has n*n cells in face order (vec of a
  // column-major n x n image).
  TransportMap solve(const Vector& density, SolverOptions opt = SolverOptions()) {
    if (n_ < 1) throw std::runtime_error("solve: init(n) must come first");
    if ((long)density.size() != (long)n_ * n_) throw std::runtime_error("solve: density size does not match init(n)");
    if (verbose_ >= 1)
      std::cout << " Solve transport map using beta=" << (opt.beta == BetaOpt::Zero ? "0" : "Conjugate-Jacobian")
                << " ;  max_iter=" << opt.max_iter << " ;  threshold=" << opt.threshold;
    auto fwd = std::make_shared<Mesh>(*origin_);
    auto adjusted = std::make_shared<Vector>(make_vector((long)n_ * n_));
    otm_solver_options o = to_c(opt);
    detail::check(otm_solve(ctx_->get(), n_, density.data(), &o, fwd->raw(), adjusted->data(), &stats_), "solve");
    if (verbose_ >= 1) {
      std::cout << "  ; initial L2=" << stats_.initial_residual << "\n";
      std::cout << " Solution:\n  - iters(" << stats_.iterations << ")\n  - error L2=" << stats_.residual
                << "   Linf=" << stats_.linf << "\n";
    }
    return TransportMap(origin_, fwd, adjusted, ctx_);
  }

  // Many independent solves (any sizes) in one GPU run; each density is square.
  std::vector<TransportMap> solve_batch(const std::vector<Vector>& densities, SolverOptions opt = SolverOptions()) {
    const int count = (int)densities.size();
    std::vector<int> ns(count);
    std::vector<const double*> dp(count);
    std::vector<double*> fp(count), ap(count);
    std::vector<std::shared_ptr<Mesh>> fwd(count);
    std::vector<std::shared_ptr<Vector>> adj(count);
    std::vector<std::shared_ptr<Mesh>> origin(count);
    for (int k = 0; k < count; ++k) {
      long cells = (long)densities[(size_t)k].size();
      int n = 1;
      while ((long)n * n < cells) ++n;
      if ((long)n * n != cells) throw std::runtime_error("solve_batch: densities must be square");
      ns[(size_t)k] = n;
      origin[(size_t)k] = std::make_shared<Mesh>(Mesh::grid(n));
      fwd[(size_t)k] = std::make_shared<Mesh>(*origin[(size_t)k]);
      adj[(size_t)k] = std::make_shared<Vector>(make_vector(cells));
      dp[(size_t)k] = densities[(size_t)k].data();
      fp[(size_t)k] = fwd[(size_t)k]->raw();
      ap[(size_t)k] = adj[(size_t)k]->data();
    }
    batch_stats_.assign((size_t)count, otm_solve_stats{});
    otm_solver_options o = to_c(opt);
    detail::check(otm_solve_batch(ctx_->get(), count, ns.data(), dp.data(), &o, fp.data(), ap.data(),
                                  batch_stats_.data()),
                  "solve_batch");
    std::vector<TransportMap> maps;
    for (int k = 0; k < count; ++k)
      maps.emplace_back(origin[(size_t)k], fwd[(size_t)k], adj[(size_t)k], ctx_);
    return maps;
  }

  // What the last solve() did (iterations, outcome, residuals).
  const otm_solve_stats& last_stats() const { return stats_; }
  const std::vector<otm_solve_stats>& last_batch_stats() const { return batch_stats_; }

 private:
  static otm_solver_options to_c(const SolverOptions& opt) {
    otm_solver_options o;
    o.beta = opt.beta == BetaOpt::Zero ? OTM_BETA_ZERO : OTM_BETA_CONJUGATE_JACOBIAN;
    o.max_iter = opt.max_iter;
    o.threshold = opt.threshold;
    o.max_ratio = opt.max_ratio;
    return o;
  }

  std::shared_ptr<detail::Context> ctx_;
  int verbose_ = 1;
  int n_ = 0;
  std::shared_ptr<Mesh> origin_;
  otm_solve_stats stats_{};
  std::vector<otm_solve_stats> batch_stats_;
};

// transport_map.h:66-68: inverts points (in-out) through the map.
inline void apply_inverse_map(const TransportMap& tmap, std::vector<Point>& points, int verbose_level = 2) {
  tmap.init_inverse();
  const long missing = tmap.inverse(points.data(), (long)points.size());
  if (missing && verbose_level >= 1) std::cerr << "Error: no face found for " << missing << " point(s).\n";
}

// transport_map.h:70, between two (n+1)^2 grid meshes.
inline double transport_cost(const Mesh& src_mesh, const Mesh& dst_mesh, const Vector& density_per_face,
                             Vector* cost_per_face = nullptr) {
  const int n = src_mesh.grid_size();
  if (n < 1 || dst_mesh.n_vertices() != src_mesh.n_vertices() || (long)density_per_face.size() != (long)n * n)
    throw std::runtime_error("transport_cost: meshes must be the same (n+1)^2 grid with n*n densities");
  if (cost_per_face) *cost_per_face = make_vector((long)n * n);
  double c = 0;
  detail::check(otm_transport_cost(detail::default_context()->get(), n, src_mesh.raw(), dst_mesh.raw(),
                                   density_per_face.data(), cost_per_face ? cost_per_face->data() : nullptr, &c),
                "transport_cost");
  return c;
}

// rasterizer.h:21-22: img must be sized (rows = y) beforehand.
inline void rasterize_image(const Mesh& mesh, const Vector& density_per_face, Image& img,
                            RasterImageOption opt = RIO_PerFaceDensity) {
  const long rows = img.rows(), cols = img.cols();
  std::vector<double> buf((size_t)(rows * cols));
  otm_context* ctx = detail::default_context()->get();
  const double* d = density_per_face.size() ? density_per_face.data() : nullptr;
  if (mesh.grid_size() > 0) {
    detail::check(otm_rasterize_mode(ctx, mesh.grid_size(), mesh.raw(), d, (int)rows, (int)cols, (int)opt,
                                     buf.data()),
                  "rasterize_image");
  } else {
    detail::check(otm_rasterize_mesh(ctx, mesh.n_vertices(), mesh.raw(), mesh.n_faces(), mesh.face_start().data(),
                                     mesh.face_indices().data(), d, (int)density_per_face.size(), (int)rows,
                                     (int)cols, (int)opt, buf.data()),
                  "rasterize_image");
  }
  detail::from_row_major(buf, img);
}

inline void rasterize_image(const Mesh& mesh, Image& img, RasterImageOption opt = RIO_PerFaceDensity) {
  rasterize_image(mesh, make_vector(0), img, opt);
}

// stochastic_rasterizer.h: sample_transportmap_to_image (stochastic_rasterizer.cpp:19-88).
// img must be sized beforehand; counts of random points per pixel. The points come from
// a counter-based generator keyed by `seed` (the reference uses std::rand()).
inline void sample_transportmap_to_image(const Mesh& mesh, const IndexVector& sample_per_face, Image& img,
                                         unsigned long long seed = 0) {
  if ((long)sample_per_face.size() != (long)mesh.n_faces())
    throw std::runtime_error("sample_transportmap_to_image: one sample count per face");
  const long rows = img.rows(), cols = img.cols();
  std::vector<double> buf((size_t)(rows * cols));
  const int g = mesh.grid_size();
  detail::check(otm_sample_image(detail::default_context()->get(), mesh.n_vertices(), mesh.raw(), mesh.n_faces(),
                                 g > 0 ? nullptr : mesh.face_start().data(),
                                 g > 0 ? nullptr : mesh.face_indices().data(), g, sample_per_face.data(), seed,
                                 (int)rows, (int)cols, buf.data()),
                "sample_transportmap_to_image");
  detail::from_row_major(buf, img);
}

inline void sample_transportmap_to_image(const Mesh& mesh, Image& img, int sample_per_face,
                                         unsigned long long seed = 0) {
  IndexVector spf(mesh.n_faces());
  for (int f = 0; f < mesh.n_faces(); ++f) spf[f] = sample_per_face;
  sample_transportmap_to_image(mesh, spf, img, seed);
}

// mesh_utils.h: prune_empty_faces (mesh_utils.cpp:124-141), in place.
inline void prune_empty_faces(Mesh& mesh, const Vector& density) {
  std::vector<Point> xy(mesh.pts_.size());
  std::vector<int> st(mesh.start_.size()), ix(mesh.idx_.size() > 0 ? mesh.idx_.size() : 1);
  int nv = 0, nf = 0;
  detail::check(otm_prune_empty_faces(mesh.n_vertices(), mesh.raw(), mesh.n_faces(), mesh.start_.data(),
                                      mesh.idx_.data(), density.data(), (int)density.size(), &nv,
                                      reinterpret_cast<double*>(xy.data()), &nf, st.data(), ix.data()),
                "prune_empty_faces");
  xy.resize((size_t)nv);
  st.resize((size_t)nf + 1);
  ix.resize((size_t)st[(size_t)nf]);
  mesh.pts_ = std::move(xy);
  mesh.start_ = std::move(st);
  mesh.idx_ = std::move(ix);
  mesh.grid_n_ = 0;
}

// The blends of apps/barycenters.cpp:250-276 (application code in the reference):
// bilinear of four inverse meshes at (alpha, beta), linear of two at alpha.
inline void interpolate(const std::vector<Mesh>& inv_maps, double alpha, double beta, Mesh& result) {
  if (inv_maps.size() != 4) throw std::runtime_error("interpolate: bilinear barycenters take 4 maps");
  const double u = alpha, v = beta;
  const double w[4] = {(1. - u) * (1. - v), u * (1. - v), u * v, (1. - u) * v};
  const double* m[4] = {inv_maps[0].raw(), inv_maps[1].raw(), inv_maps[2].raw(), inv_maps[3].raw()};
  result = inv_maps[0];
  detail::check(otm_mesh_blend(detail::default_context()->get(), result.grid_size(), 4, m, w, result.raw()),
                "interpolate");
}

inline void interpolate(const std::vector<Mesh>& inv_maps, double alpha, Mesh& result) {
  if (inv_maps.size() != 2) throw std::runtime_error("interpolate: linear barycenters take 2 maps");
  const double w[2] = {1. - alpha, alpha};
  const double* m[2] = {inv_maps[0].raw(), inv_maps[1].raw()};
  result = inv_maps[0];
  detail::check(otm_mesh_blend(detail::default_context()->get(), result.grid_size(), 2, m, w, result.raw()),
                "interpolate");
}

}  // namespace otmap
