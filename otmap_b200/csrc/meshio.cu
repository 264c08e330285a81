// Host-side mesh formats around the solver: the grid's indexed face set, OFF files as
// the reference's Surface_mesh reads and writes them (otlib/surface_mesh/IO_off.cpp),
// and prune_empty_faces (otlib/utils/mesh_utils.cpp:124-141) with the element order
// Surface_mesh::garbage_collection leaves (otlib/surface_mesh/Surface_mesh.cpp:1975-2110).
// These are file and topology operations on a few million integers at most; they run
// on the host and need no device.

#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "common.cuh"
#include "otmap_b200.h"

namespace otm {
namespace {

template <class F>
int guarded_host(F&& f) {
  try {
    return f();
  } catch (const BadArg& e) {
    set_error(e.what);
    return OTM_ERR_BAD_ARG;
  } catch (const std::exception& e) {
    set_error(e.what());
    return OTM_ERR_BAD_ARG;
  }
}

void check_topology(const char* who, int nv, int nf, const int* start, const int* idx) {
  if (nv < 0 || nf < 0) throw BadArg{std::string(who) + ": negative size"};
  if (nf > 0 && (!start || !idx)) throw BadArg{std::string(who) + ": null face arrays"};
  if (nf > 0 && start[0] != 0) throw BadArg{std::string(who) + ": face_start[0] must be 0"};
  for (int f = 0; f < nf; ++f)
    if (start[f + 1] - start[f] < 3) throw BadArg{std::string(who) + ": a face has fewer than 3 corners"};
  const int total = nf > 0 ? start[nf] : 0;
  for (int k = 0; k < total; ++k)
    if (idx[k] < 0 || idx[k] >= nv) throw BadArg{std::string(who) + ": vertex index out of range"};
}

// Compacts `count` elements flagged in `dead` the way garbage_collection does: a
// front cursor stops at each hole, a back cursor at the last survivor, and the two
// trade places until the cursors meet. newpos[i] = new index of element i, -1 if
// removed. Returns the number kept.
int compact(int count, const std::vector<char>& dead_in, std::vector<int>& newpos) {
  std::vector<char> dead(dead_in);
  std::vector<int> at(count);
  for (int i = 0; i < count; ++i) at[i] = i;
  newpos.assign(count, -1);
  if (count == 0) return 0;
  int front = 0, back = count - 1;
  for (;;) {
    while (!dead[front] && front < back) ++front;
    while (dead[back] && front < back) --back;
    if (front >= back) break;
    std::swap(dead[front], dead[back]);
    std::swap(at[front], at[back]);
  }
  const int kept = dead[front] ? front : front + 1;
  for (int pos = 0; pos < kept; ++pos) newpos[at[pos]] = pos;
  return kept;
}

// Reads one record line into a 200-byte buffer, as IO_off.cpp reads vertex and face records.
bool read_line(FILE* in, char* line) { return std::fgets(line, 200, in) != nullptr; }

}  // namespace
}  // namespace otm

using namespace otm;

extern "C" int otm_grid_faces(int n, int* face_start, int* face_vertices) {
  return guarded_host([&] {
    if (n < 1 || n > 16384 || !face_start || !face_vertices) throw BadArg{"otm_grid_faces: bad arguments"};
    const long N = (long)n * n;
    for (long f = 0; f < N; ++f) {
      const int i = (int)(f / n), j = (int)(f % n);
      face_start[f] = (int)(4 * f);
      face_vertices[4 * f] = j + i * (n + 1);
      face_vertices[4 * f + 1] = j + (i + 1) * (n + 1);
      face_vertices[4 * f + 2] = (j + 1) + (i + 1) * (n + 1);
      face_vertices[4 * f + 3] = (j + 1) + i * (n + 1);
    }
    face_start[N] = (int)(4 * N);
    return (int)OTM_OK;
  });
}

extern "C" int otm_write_off(const char* path, int nv, const double* xy, int nf, const int* face_start,
                             const int* face_vertices) {
  return guarded_host([&] {
    if (!path || (nv > 0 && !xy)) throw BadArg{"otm_write_off: null argument"};
    check_topology("otm_write_off", nv, nf, face_start, face_vertices);
    FILE* out = std::fopen(path, "w");
    if (!out) throw BadArg{std::string("otm_write_off: cannot open ") + path};
    // header, then "x y 0" per vertex and "valence i0 i1 ..." per face (IO_off.cpp:336-375)
    std::fprintf(out, "OFF\n%d %d 0\n", nv, nf);
    for (int v = 0; v < nv; ++v) std::fprintf(out, "%.10f %.10f %.10f\n", xy[2 * v], xy[2 * v + 1], 0.0);
    for (int f = 0; f < nf; ++f) {
      std::fprintf(out, "%d", face_start[f + 1] - face_start[f]);
      for (int k = face_start[f]; k < face_start[f + 1]; ++k) std::fprintf(out, " %d", face_vertices[k]);
      std::fprintf(out, "\n");
    }
    const bool ok = std::ferror(out) == 0;
    std::fclose(out);
    if (!ok) throw BadArg{std::string("otm_write_off: write failed: ") + path};
    return (int)OTM_OK;
  });
}

extern "C" int otm_read_off(const char* path, int* nv, int* nf, int* nidx, double* xy, int* face_start,
                            int* face_vertices) {
  return guarded_host([&] {
    if (!path || !nv || !nf || !nidx) throw BadArg{"otm_read_off: null argument"};
    FILE* in = std::fopen(path, "r");
    if (!in) throw BadArg{std::string("otm_read_off: cannot open ") + path};
    struct Closer {
      FILE* f;
      ~Closer() {
        if (f) std::fclose(f);
      }
    } closer{in};
    // header [ST][C][N]OFF [BINARY] (IO_off.cpp:262-283)
    char line[200];
    if (!read_line(in, line)) throw BadArg{"otm_read_off: empty file"};
    const char* c = line;
    bool tex = false, col = false, nrm = false;
    if (c[0] == 'S' && c[1] == 'T') {
      tex = true;
      c += 2;
    }
    if (c[0] == 'C') {
      col = true;
      ++c;
    }
    if (c[0] == 'N') {
      nrm = true;
      ++c;
    }
    if (c[0] == '4' || c[0] == 'n' || std::strncmp(c, "OFF", 3) != 0)
      throw BadArg{"otm_read_off: not an OFF file this reader handles"};
    const bool binary = std::strncmp(c + 4, "BINARY", 6) == 0;
    std::vector<double> pts;
    std::vector<int> starts(1, 0), idx;
    unsigned int V = 0, F = 0, E = 0;
    if (!binary) {
      if (std::fscanf(in, "%d %d %d\n", (int*)&V, (int*)&F, (int*)&E) != 3) throw BadArg{"otm_read_off: bad counts"};
      if (V > (1u << 28) || F > (1u << 28)) throw BadArg{"otm_read_off: counts too large"};
      pts.reserve(2 * (size_t)V);
      // positions lead each vertex line; normals, colours and texture coordinates
      // that follow on the line are not kept
      for (unsigned int i = 0; i < V; ++i) {
        if (!read_line(in, line)) throw BadArg{"otm_read_off: truncated vertex list"};
        double p[3];
        int nc = 0;
        if (std::sscanf(line, "%lf %lf %lf%n", &p[0], &p[1], &p[2], &nc) != 3)
          throw BadArg{"otm_read_off: bad vertex record"};
        pts.push_back(p[0]);  // a Surface_mesh point is 2-D: z is dropped (types.h:42-49)
        pts.push_back(p[1]);
      }
      for (unsigned int i = 0; i < F; ++i) {
        if (!read_line(in, line)) throw BadArg{"otm_read_off: truncated face list"};
        const char* lp = line;
        int k = 0, nc = 0;
        if (std::sscanf(lp, "%d%n", &k, &nc) != 1 || k < 3) throw BadArg{"otm_read_off: bad face record"};
        lp += nc;
        for (int j = 0; j < k; ++j) {
          int v = 0;
          if (std::sscanf(lp, "%d%n", &v, &nc) != 1) throw BadArg{"otm_read_off: bad face record"};
          lp += nc;
          idx.push_back(v);
        }
        starts.push_back((int)idx.size());
      }
    } else {
      // binary layout (IO_off.cpp:170-240): counts, then per vertex three doubles
      // [+ normal] [+ texcoord], then per face its valence and indices (uint32)
      if (col) throw BadArg{"otm_read_off: binary OFF with colours is not readable"};
      std::fclose(in);
      closer.f = in = std::fopen(path, "rb");
      if (!in || !read_line(in, line)) throw BadArg{"otm_read_off: cannot reopen"};
      auto rd = [&](void* p, size_t b) {
        if (std::fread(p, 1, b, in) != b) throw BadArg{"otm_read_off: truncated binary file"};
      };
      rd(&V, 4);
      rd(&F, 4);
      rd(&E, 4);
      if (V > (1u << 28) || F > (1u << 28)) throw BadArg{"otm_read_off: counts too large"};
      for (unsigned int i = 0; i < V; ++i) {
        double p[3];
        rd(p, sizeof p);
        pts.push_back(p[0]);
        pts.push_back(p[1]);
        if (nrm) rd(p, sizeof p);
        if (tex) rd(p, 2 * sizeof(double));
      }
      for (unsigned int i = 0; i < F; ++i) {
        unsigned int k = 0;
        rd(&k, 4);
        if (k < 3 || k > 1024) throw BadArg{"otm_read_off: bad face record"};
        for (unsigned int j = 0; j < k; ++j) {
          unsigned int v = 0;
          rd(&v, 4);
          idx.push_back((int)v);
        }
        starts.push_back((int)idx.size());
      }
    }
    for (int v : idx)
      if (v < 0 || v >= (int)V) throw BadArg{"otm_read_off: vertex index out of range"};
    const bool fill = xy != nullptr;
    if (fill && (*nv < (int)V || *nf < (int)F || *nidx < (int)idx.size()))
      throw BadArg{"otm_read_off: output arrays too small"};
    *nv = (int)V;
    *nf = (int)F;
    *nidx = (int)idx.size();
    if (fill) {
      if (!face_start || (!face_vertices && !idx.empty())) throw BadArg{"otm_read_off: null face arrays"};
      std::memcpy(xy, pts.data(), sizeof(double) * pts.size());
      std::memcpy(face_start, starts.data(), sizeof(int) * starts.size());
      if (!idx.empty()) std::memcpy(face_vertices, idx.data(), sizeof(int) * idx.size());
    }
    return (int)OTM_OK;
  });
}

extern "C" int otm_prune_empty_faces(int nv, const double* xy, int nf, const int* face_start,
                                     const int* face_vertices, const double* density, int cells, int* nv_out,
                                     double* xy_out, int* nf_out, int* start_out, int* idx_out) {
  return guarded_host([&] {
    if (!density || !nv_out || !nf_out || (nv > 0 && (!xy || !xy_out)) || !start_out || (nf > 0 && !idx_out))
      throw BadArg{"otm_prune_empty_faces: null argument"};
    check_topology("otm_prune_empty_faces", nv, nf, face_start, face_vertices);
    // a triangulated grid (two faces per cell) reads cell f/2 for face f (mesh_utils.cpp:128-133)
    const bool pairs = nf == 2 * cells;
    if (!pairs && cells < nf) throw BadArg{"otm_prune_empty_faces: density shorter than the face count"};
    std::vector<char> fdead(nf), touched(nv, 0), live(nv, 0), vdead(nv);
    for (int f = 0; f < nf; ++f) {
      fdead[f] = density[pairs ? f / 2 : f] == 0;
      for (int k = face_start[f]; k < face_start[f + 1]; ++k) (fdead[f] ? touched : live)[face_vertices[k]] = 1;
    }
    // delete_face removes a vertex once its last face is gone (Surface_mesh.cpp:1787-1880)
    for (int v = 0; v < nv; ++v) vdead[v] = touched[v] && !live[v];
    std::vector<int> vpos, fpos;
    const int kv = compact(nv, vdead, vpos);
    const int kf = compact(nf, fdead, fpos);
    for (int v = 0; v < nv; ++v)
      if (vpos[v] >= 0) {
        xy_out[2 * vpos[v]] = xy[2 * v];
        xy_out[2 * vpos[v] + 1] = xy[2 * v + 1];
      }
    std::vector<int> from(kf);
    for (int f = 0; f < nf; ++f)
      if (fpos[f] >= 0) from[fpos[f]] = f;
    int k = 0;
    start_out[0] = 0;
    for (int q = 0; q < kf; ++q) {
      const int f = from[q];
      for (int t = face_start[f]; t < face_start[f + 1]; ++t) idx_out[k++] = vpos[face_vertices[t]];
      start_out[q + 1] = k;
    }
    *nv_out = kv;
    *nf_out = kf;
    return (int)OTM_OK;
  });
}
