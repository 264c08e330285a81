// Test driver for the C++ facade (include/otmap_b200.hpp): the calls of the reference's
// demo apps/otmap.cpp:95-140, made through namespace otmap, with outputs written to a
// folder for the Python tests to compare.
//
//   facade_demo mesh <dir>                    host-only: grid mesh, OFF write/read, prune
//   facade_demo pipeline <dir> <u.bin> <v.bin> solve two densities and derive everything
//
// A density file is int32 n followed by n*n float64 cells in face order. Outputs are
// OFF files and raw float64 dumps (*.f64); results.txt lists scalars as "key value".

#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <string>
#include <vector>

#include "otmap_b200.hpp"

using namespace otmap;

static Vector read_density(const std::string& path, int& n) {
  std::ifstream in(path, std::ios::binary);
  int32_t nn = 0;
  in.read(reinterpret_cast<char*>(&nn), 4);
  n = nn;
  Vector d = make_vector((long)n * n);
  in.read(reinterpret_cast<char*>(d.data()), sizeof(double) * (size_t)n * n);
  if (!in) throw std::runtime_error("cannot read " + path);
  return d;
}

static void dump(const std::string& path, const double* p, size_t count) {
  std::ofstream out(path, std::ios::binary);
  out.write(reinterpret_cast<const char*>(p), sizeof(double) * count);
}

static void dump_image(const std::string& path, const Image& img) {
  std::vector<double> rm((size_t)(img.rows() * img.cols()));
  for (long y = 0; y < img.rows(); ++y)
    for (long x = 0; x < img.cols(); ++x) rm[(size_t)(y * img.cols() + x)] = img(y, x);
  dump(path, rm.data(), rm.size());
}

static int mesh_mode(const std::string& dir) {
  Mesh g = Mesh::grid(8);
  g.position(10) = Point{0.3, 0.2};
  if (!g.write(dir + "/grid8.off")) return 2;
  Mesh r;
  if (!r.read(dir + "/grid8.off")) return 3;
  if (r.n_vertices() != g.n_vertices() || r.n_faces() != g.n_faces()) return 4;
  Vector d = make_vector(64, 1.0);
  for (int f = 0; f < 64; f += 3) d[f] = 0.0;
  Mesh p = g;
  prune_empty_faces(p, d);
  if (!p.write(dir + "/grid8_pruned.off")) return 5;
  std::ofstream res(dir + "/results.txt");
  res << "pruned_vertices " << p.n_vertices() << "\npruned_faces " << p.n_faces() << "\n";
  return 0;
}

static int pipeline_mode(const std::string& dir, const std::string& fu, const std::string& fv) {
  int nu = 0, nv = 0;
  Vector du = read_density(fu, nu), dv = read_density(fv, nv);
  GridBasedTransportSolver solver;
  solver.set_verbose_level(0);
  std::vector<TransportMap> tmaps;
  solver.init(nu);
  tmaps.push_back(solver.solve(du));
  const int it_u = solver.last_stats().iterations;
  solver.init(nv);
  tmaps.push_back(solver.solve(dv));
  const int it_v = solver.last_stats().iterations;
  std::ofstream res(dir + "/results.txt");
  res << std::setprecision(17) << "iterations_u " << it_u << "\niterations_v " << it_v << "\n";
  const char* tag[2] = {"u", "v"};
  for (int k = 0; k < 2; ++k) {
    const TransportMap& t = tmaps[(size_t)k];
    t.fwd_mesh().write(dir + "/" + tag[k] + "_fwd.off");
    dump(dir + "/" + tag[k] + "_fwd.f64", t.fwd_mesh().raw(), 2 * (size_t)t.fwd_mesh().n_vertices());
    dump(dir + "/" + tag[k] + "_density.f64", t.density().data(), (size_t)t.density().size());
    res << "cost_" << tag[k] << " " << transport_cost(t.origin_mesh(), t.fwd_mesh(), t.density()) << "\n";
    Mesh inv = t.origin_mesh();
    apply_inverse_map(t, inv.points(), 0);
    inv.write(dir + "/" + tag[k] + "_inv.off");
    dump(dir + "/" + tag[k] + "_inv.f64", inv.raw(), 2 * (size_t)inv.n_vertices());
  }
  // composite maps u->v and v->u (apps/otmap.cpp:120-137)
  Mesh map_uv = tmaps[0].fwd_mesh();
  apply_inverse_map(tmaps[1], map_uv.points(), 0);
  res << "cost_uv " << transport_cost(tmaps[0].origin_mesh(), map_uv, tmaps[0].density()) << "\n";
  dump(dir + "/map_uv.f64", map_uv.raw(), 2 * (size_t)map_uv.n_vertices());
  Image img(nu, nu);
  rasterize_image(map_uv, img);
  dump_image(dir + "/map_uv_raster.f64", img);
  Image pv(nu, nu);
  rasterize_image(map_uv, tmaps[0].density(), pv, RIO_PerVertexDensity);
  dump_image(dir + "/map_uv_pervertex.f64", pv);
  prune_empty_faces(map_uv, tmaps[0].density());
  map_uv.write(dir + "/map_uv.off");
  Image pr(nu + 3, nu);
  rasterize_image(map_uv, pr);
  dump_image(dir + "/map_uv_pruned_raster.f64", pr);
  // copies share the point locator
  TransportMap copy = tmaps[1];
  Point q = copy.inv(Point{0.37, 0.61});
  Point qf = copy.inv_fast(Point{0.37, 0.61});
  res << "inv_x " << q[0] << "\ninv_y " << q[1] << "\ninvfast_x " << qf[0] << "\ninvfast_y " << qf[1] << "\n";
  // linear barycenter halfway between the two inverse maps when the sizes agree
  if (nu == nv) {
    std::vector<Mesh> inv(2, tmaps[0].origin_mesh());
    for (int k = 0; k < 2; ++k) apply_inverse_map(tmaps[(size_t)k], inv[(size_t)k].points(), 0);
    Mesh mid;
    interpolate(inv, 0.5, mid);
    dump(dir + "/mid.f64", mid.raw(), 2 * (size_t)mid.n_vertices());
  }
  // stochastic splat of the composite map, 50 samples per face
  Image sp(nu, nu);
  sample_transportmap_to_image(tmaps[0].fwd_mesh(), sp, 50, 7);
  dump_image(dir + "/u_fwd_samples.f64", sp);
  // many solves in one run
  std::vector<Vector> both = {du, dv};
  std::vector<TransportMap> batch = solver.solve_batch(both);
  for (int k = 0; k < 2; ++k)
    dump(dir + "/batch_" + tag[k] + "_fwd.f64", batch[(size_t)k].fwd_mesh().raw(),
         2 * (size_t)batch[(size_t)k].fwd_mesh().n_vertices());
  return 0;
}

int main(int argc, char** argv) {
  try {
    std::string mode = argc > 1 ? argv[1] : "";
    if (mode == "mesh" && argc == 3) return mesh_mode(argv[2]);
    if (mode == "pipeline" && argc == 5) return pipeline_mode(argv[2], argv[3], argv[4]);
    std::fprintf(stderr, "usage: facade_demo mesh <dir> | pipeline <dir> <u.bin> <v.bin>\n");
    return 1;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "facade_demo: %s\n", e.what());
    return 10;
  }
}
