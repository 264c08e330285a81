// Point location in the forward mesh (TransportMap inversion) and rasterization of
// a deformed grid mesh, for sm_100a.
//
// Both run on a uniform bin grid built on the GPU: faces are binned by their
// bounding boxes (count, exclusive scan, scatter) and each query -- a point to
// invert, or a pixel centre to shade -- tests only the faces of its bin. The query
// kernels are atomics-free gathers; the only atomics are the integer bin counters
// of the build. This file is compiled without FMA contraction: the geometric
// predicates (utils/mesh_utils.cpp:18-88) then round exactly as the reference's
// scalar x86-64 build does, which makes the located faces, weights, inverse
// positions and pixel values bit-identical to the reference wherever the
// reference's own result does not depend on the order of its BVH traversal.

#include <cfloat>
#include <cmath>
#include <vector>

#include "context.h"

namespace otm {

// ---- geometry (utils/eigen_addons.h:15-22, utils/mesh_utils.h:18-25, mesh_utils.cpp:18-88) ----

__device__ __forceinline__ double cross2(double ax, double ay, double bx, double by) { return ax * by - ay * bx; }

__device__ __forceinline__ double signed_area3(double ax, double ay, double bx, double by, double cx, double cy) {
  return 0.5 * cross2(bx - ax, by - ay, cx - ax, cy - ay);
}

struct Quad {
  double x[4], y[4];
};

__device__ __forceinline__ bool inside_tri(double qx, double qy, double p0x, double p0y, double p1x, double p1y,
                                           double p2x, double p2y) {
  double q2x = qx - p2x, q2y = qy - p2y;
  double eux = p1x - p2x, euy = p1y - p2y;
  double evx = p0x - p2x, evy = p0y - p2y;
  double area2 = cross2(evx, evy, eux, euy);
  double u = cross2(q2x, q2y, eux, euy) / area2;
  double v = cross2(evx, evy, q2x, q2y) / area2;
  const double eps = 1e-8;
  return u >= -eps && v >= -eps && u + v <= 1. + eps;
}

// inside_quad (mesh_utils.cpp:62-74)
__device__ __forceinline__ bool inside_quad(double qx, double qy, const Quad& p) {
  return inside_tri(qx, qy, p.x[0], p.y[0], p.x[1], p.y[1], p.x[2], p.y[2]) ||
         inside_tri(qx, qy, p.x[0], p.y[0], p.x[2], p.y[2], p.x[3], p.y[3]);
}

// bilinear_coordinates_in_quad, weights form (mesh_utils.cpp:18-59, 76-88).
__device__ bool bilinear_weights(double qx, double qy, const Quad& p, double w[4]) {
  double A0 = signed_area3(qx, qy, p.x[0], p.y[0], p.x[1], p.y[1]);
  double A1 = signed_area3(qx, qy, p.x[1], p.y[1], p.x[2], p.y[2]);
  double A2 = signed_area3(qx, qy, p.x[2], p.y[2], p.x[3], p.y[3]);
  double A3 = signed_area3(qx, qy, p.x[3], p.y[3], p.x[0], p.y[0]);
  double B0 = signed_area3(qx, qy, p.x[3], p.y[3], p.x[1], p.y[1]);
  double B1 = signed_area3(qx, qy, p.x[0], p.y[0], p.x[2], p.y[2]);
  double B3 = signed_area3(qx, qy, p.x[2], p.y[2], p.x[0], p.y[0]);
  double D = B0 * B0 + B1 * B1 + 2 * A0 * A2 + 2 * A1 * A3;
  if (D < 0) return false;
  double sD = sqrt(D);
  double E0 = 2 * A0 - B0 - B1 + sD;
  double E3 = 2 * A3 - B3 - B0 + sD;
  const double zero = 4 * DBL_MIN;
  double v = fabs(A0) <= zero ? 0 : 2 * A0 / E0;
  double u = fabs(A3) <= zero ? 0 : 2 * A3 / E3;
  double E0p = 2 * A0 - B0 - B1 - sD;
  double E3p = 2 * A3 - B3 - B0 - sD;
  double v_alt = fabs(A0) <= zero ? 0 : 2 * A0 / E0p;
  double u_alt = fabs(A3) <= zero ? 0 : 2 * A3 / E3p;
  const double eps = 1.4901161193847656e-08;  // sqrt(DBL_EPSILON), exact
  if (fabs(u) < eps) u = 0;
  if (fabs(v) < eps) v = 0;
  if (fabs(u - 1.) < eps) u = 1;
  if (fabs(v - 1.) < eps) v = 1;
  if (fabs(u_alt) < eps) u_alt = 0;
  if (fabs(v_alt) < eps) v_alt = 0;
  if (fabs(u_alt - 1.) < eps) u_alt = 1;
  if (fabs(v_alt - 1.) < eps) v_alt = 1;
  if ((u < 0 || v < 0 || u > 1 || v > 1) && (u_alt >= 0 && v_alt >= 0 && u_alt <= 1 && v_alt <= 1)) {
    u = u_alt;
    v = v_alt;
  }
  const double weps = 4 * DBL_EPSILON;
  w[0] = (1. - u) * (1 - v);
  w[1] = (u) * (1. - v);
  w[2] = (u) * (v);
  w[3] = (1. - u) * (v);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (fabs(w[k]) <= weps)
      w[k] = 0;
    else if (fabs(w[k] - 1.) <= weps)
      w[k] = 1;
  }
  return true;
}

__device__ __forceinline__ bool weights_inside(const double w[4]) {
  return w[0] <= 1.0f && w[1] <= 1.0f && w[2] <= 1.0f && w[3] <= 1.0f && w[0] >= 0.0f && w[1] >= 0.0f &&
         w[2] >= 0.0f && w[3] >= 0.0f;
}

// Corners of face f = j + i*n of an (n+1)^2 grid mesh: (i,j), (i+1,j), (i+1,j+1), (i,j+1).
__device__ __forceinline__ void load_quad(const double* xy, int n, int f, Quad& p, int vid[4]) {
  int i = f / n, j = f - (f / n) * n;
  vid[0] = j + i * (n + 1);
  vid[1] = j + (i + 1) * (n + 1);
  vid[2] = (j + 1) + (i + 1) * (n + 1);
  vid[3] = (j + 1) + i * (n + 1);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    p.x[k] = xy[2 * (size_t)vid[k]];
    p.y[k] = xy[2 * (size_t)vid[k] + 1];
  }
}

// ---- exclusive scan of int counts (three passes) ----

constexpr int SCAN_B = 1024;

__global__ void k_scan_local(const int* in, int* out, int* block_sums, int count) {
  __shared__ int s[SCAN_B];
  int g = blockIdx.x * SCAN_B + threadIdx.x;
  int v = g < count ? in[g] : 0;
  s[threadIdx.x] = v;
  __syncthreads();
  for (int off = 1; off < SCAN_B; off <<= 1) {
    int t = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
    __syncthreads();
    s[threadIdx.x] += t;
    __syncthreads();
  }
  if (g < count) out[g] = s[threadIdx.x] - v;
  if (threadIdx.x == SCAN_B - 1) block_sums[blockIdx.x] = s[threadIdx.x];
}

// Scans the block sums in place (sequential over at most a few thousand values) and
// writes the grand total to out[count].
__global__ void k_scan_sums(int* block_sums, int nblocks, int* out, int count) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int acc = 0;
  for (int b = 0; b < nblocks; ++b) {
    int v = block_sums[b];
    block_sums[b] = acc;
    acc += v;
  }
  out[count] = acc;
}

__global__ void k_scan_add(int* out, const int* block_sums, int count) {
  int g = blockIdx.x * SCAN_B + threadIdx.x;
  if (g < count) out[g] += block_sums[blockIdx.x];
}

static void exclusive_scan(cudaStream_t st, const int* counts, int* starts, int* block_sums, int count) {
  int nb = (count + SCAN_B - 1) / SCAN_B;
  k_scan_local<<<nb, SCAN_B, 0, st>>>(counts, starts, block_sums, count);
  k_scan_sums<<<1, 32, 0, st>>>(block_sums, nb, starts, count);
  k_scan_add<<<nb, SCAN_B, 0, st>>>(starts, block_sums, count);
}

// ---- point location (TransportMap::init_inverse / inv_impl) ----

// Bin range of face f's bounding box, enlarged so that every point the reference's
// tolerant tests can accept (inside_quad eps 1e-8, weight snapping) lands inside it.
__device__ __forceinline__ void face_bins(const Quad& p, int B, int& bx0, int& bx1, int& by0, int& by1,
                                          double4& box) {
  double mnx = fmin(fmin(p.x[0], p.x[1]), fmin(p.x[2], p.x[3]));
  double mxx = fmax(fmax(p.x[0], p.x[1]), fmax(p.x[2], p.x[3]));
  double mny = fmin(fmin(p.y[0], p.y[1]), fmin(p.y[2], p.y[3]));
  double mxy = fmax(fmax(p.y[0], p.y[1]), fmax(p.y[2], p.y[3]));
  double m = 1e-6 * fmax(mxx - mnx, mxy - mny) + 1e-12;
  box = make_double4(mnx - m, mny - m, mxx + m, mxy + m);
  auto cl = [B](double v) {
    double t = floor(v * (double)B);
    return t < 0 ? 0 : (t >= B ? B - 1 : (int)t);
  };
  bx0 = cl(box.x);
  bx1 = cl(box.z);
  by0 = cl(box.y);
  by1 = cl(box.w);
}

__global__ void k_bin_count(const double* xy, int n, int B, int* counts, double4* boxes) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n * n) return;
  Quad p;
  int vid[4];
  load_quad(xy, n, f, p, vid);
  int bx0, bx1, by0, by1;
  double4 box;
  face_bins(p, B, bx0, bx1, by0, by1, box);
  boxes[f] = box;
  for (int by = by0; by <= by1; ++by)
    for (int bx = bx0; bx <= bx1; ++bx) atomicAdd(&counts[by * B + bx], 1);
}

__global__ void k_bin_fill(const double* xy, int n, int B, const int* starts, int* cursor, int* faces) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n * n) return;
  Quad p;
  int vid[4];
  load_quad(xy, n, f, p, vid);
  int bx0, bx1, by0, by1;
  double4 box;
  face_bins(p, B, bx0, bx1, by0, by1, box);
  for (int by = by0; by <= by1; ++by)
    for (int bx = bx0; bx <= bx1; ++bx) {
      int b = by * B + bx;
      faces[starts[b] + atomicAdd(&cursor[b], 1)] = f;
    }
}

constexpr int MAXHITS = 8;

// inv_impl (transport_map.cpp:50-102) per point. Hits are taken in increasing face
// order; with several hits the reference keeps the weights of its first hit and the
// face of the densest later one (transport_map.cpp:70-85), which is reproduced.
__global__ void k_inverse(const double* xy, const double* density, int n, int B, const int* starts,
                          const int* faces, const double4* boxes, double* pts, long P, int* face_out,
                          int* nhits_out, unsigned long long* missing) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  double qx = fmin(fmax(pts[2 * i], 0.), 1.);
  double qy = fmin(fmax(pts[2 * i + 1], 0.), 1.);
  if (!(qx == qx)) qx = 0.;  // NaN input: clamp like Eigen's max/min would not; keep it finite
  if (!(qy == qy)) qy = 0.;
  int bx = (int)fmin(floor(qx * (double)B), (double)(B - 1));
  int by = (int)fmin(floor(qy * (double)B), (double)(B - 1));
  int b = by * B + bx;
  int hf[MAXHITS];
  double hw[MAXHITS][4];
  int nh = 0;
  for (int k = starts[b]; k < starts[b + 1]; ++k) {
    int f = faces[k];
    double4 bb = boxes[f];
    if (qx < bb.x || qx > bb.z || qy < bb.y || qy > bb.w) continue;
    Quad p;
    int vid[4];
    load_quad(xy, n, f, p, vid);
    double w[4];
    if (!inside_quad(qx, qy, p)) continue;
    if (!bilinear_weights(qx, qy, p, w)) continue;
    if (!weights_inside(w)) continue;
    // insertion in increasing face order
    int pos = nh < MAXHITS ? nh : MAXHITS - 1;
    if (nh >= MAXHITS && f > hf[MAXHITS - 1]) {
      ++nh;
      continue;
    }
    while (pos > 0 && hf[pos - 1] > f) {
      hf[pos] = hf[pos - 1];
#pragma unroll
      for (int c = 0; c < 4; ++c) hw[pos][c] = hw[pos - 1][c];
      --pos;
    }
    hf[pos] = f;
#pragma unroll
    for (int c = 0; c < 4; ++c) hw[pos][c] = w[c];
    ++nh;
  }
  if (nhits_out) nhits_out[i] = nh;
  if (nh == 0) {
    pts[2 * i] = NAN;
    pts[2 * i + 1] = NAN;
    if (face_out) face_out[i] = -1;
    atomicAdd(missing, 1ull);
    return;
  }
  int f = hf[0];
  int kmax = nh < MAXHITS ? nh : MAXHITS;
  if (nh > 1) {
    double best = density[f];
    for (int k = 1; k < kmax; ++k) {
      double dk = density[hf[k]];
      if (dk > best) {
        f = hf[k];
        best = dk > best;  // the reference stores the comparison's bool here (transport_map.cpp:82)
      }
    }
  }
  Quad p;
  int vid[4];
  load_quad(xy, n, f, p, vid);
  const double dx = 1.0 / (double)n;
  double rx = 0, ry = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    int vi = vid[k] / (n + 1), vj = vid[k] - (vid[k] / (n + 1)) * (n + 1);
    double ox = (double)vi * dx, oy = (double)vj * dx;
    if (k == 0) {
      rx = hw[0][0] * ox;
      ry = hw[0][0] * oy;
    } else {
      rx += hw[0][k] * ox;
      ry += hw[0][k] * oy;
    }
  }
  pts[2 * i] = rx;
  pts[2 * i + 1] = ry;
  if (face_out) face_out[i] = f;
}

// ---- rasterization (utils/rasterizer.cpp:162-236) ----

constexpr int RT = 16;  // pixel tile edge for face binning

struct FaceRaster {
  int x0, x1, y0, y1;  // pixel box [x0,x1) x [y0,y1), as rasterize_face computes it
  double value;        // float(1/N) * density / |area|
};

__device__ __forceinline__ FaceRaster face_raster(const double* xy, const double* density, int n, float scale,
                                                  int rows, int cols, int f) {
  Quad p;
  int vid[4];
  load_quad(xy, n, f, p, vid);
  FaceRaster r;
  double in_mass = scale * (density ? density[f] : 1.0);
  double area = fabs(signed_area3(p.x[0], p.y[0], p.x[1], p.y[1], p.x[2], p.y[2]) +
                     signed_area3(p.x[0], p.y[0], p.x[2], p.y[2], p.x[3], p.y[3]));
  r.value = in_mass / area;
  double ulx = fmin(fmin(fmin(p.x[0], p.x[1]), p.x[2]), p.x[3]);
  double uly = fmin(fmin(fmin(p.y[0], p.y[1]), p.y[2]), p.y[3]);
  double lrx = fmax(fmax(fmax(p.x[0], p.x[1]), p.x[2]), p.x[3]);
  double lry = fmax(fmax(fmax(p.y[0], p.y[1]), p.y[2]), p.y[3]);
  // Eigen cast<int> truncates toward zero; the boxes are clamped to the image
  double fx0 = ulx * (double)cols, fy0 = uly * (double)rows;
  double fx1 = lrx * (double)cols, fy1 = lry * (double)rows;
  auto trunc_int = [](double v) {
    if (!(v == v)) return 0;
    if (v > 2.0e9) return 2000000000;
    if (v < -2.0e9) return -2000000000;
    return (int)v;
  };
  r.x0 = max(trunc_int(fx0), 0);
  r.y0 = max(trunc_int(fy0), 0);
  r.x1 = min(trunc_int(fx1) + 1, cols);
  r.y1 = min(trunc_int(fy1) + 1, rows);
  return r;
}

__global__ void k_raster_count(const double* xy, const double* density, int n, float scale, int rows, int cols,
                               int TX, FaceRaster* fr, int* counts) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n * n) return;
  FaceRaster r = face_raster(xy, density, n, scale, rows, cols, f);
  fr[f] = r;
  if (r.x0 >= r.x1 || r.y0 >= r.y1) return;
  for (int ty = r.y0 / RT; ty <= (r.y1 - 1) / RT; ++ty)
    for (int tx = r.x0 / RT; tx <= (r.x1 - 1) / RT; ++tx) atomicAdd(&counts[ty * TX + tx], 1);
}

__global__ void k_raster_fill(const FaceRaster* fr, int n, int TX, const int* starts, int* cursor, int* faces) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n * n) return;
  FaceRaster r = fr[f];
  if (r.x0 >= r.x1 || r.y0 >= r.y1) return;
  for (int ty = r.y0 / RT; ty <= (r.y1 - 1) / RT; ++ty)
    for (int tx = r.x0 / RT; tx <= (r.x1 - 1) / RT; ++tx) {
      int b = ty * TX + tx;
      faces[starts[b] + atomicAdd(&cursor[b], 1)] = f;
    }
}

// Weights the reference's sequential loop would test at (f, x, y) when its bilinear
// solve fails there (D < 0): its Vector4d is never written, and the optimised build
// then reads the weights of the most recent successful solve. Walk back through the
// loop order -- earlier pixels of face f's box row by row, then earlier faces -- to
// the most recent pixel whose solve succeeds. Bounded; gives zeros (the start state)
// when it runs out, as the sequential emulation does before any solve.
__device__ void stale_weights(const double* xy, int n, int rows, int cols, const FaceRaster* fr, int f, int x,
                              int y, double w[4]) {
  int steps = 0;
  const int limit = 1 << 22;
  while (steps < limit) {
    FaceRaster r = fr[f];
    // previous pixel in face f's scan
    if (x > r.x0) {
      --x;
    } else if (y > r.y0) {
      --y;
      x = r.x1 - 1;
    } else {
      // last pixel of the previous face with a non-empty box
      int g = f - 1;
      while (g >= 0 && (fr[g].x0 >= fr[g].x1 || fr[g].y0 >= fr[g].y1) && steps < limit) {
        --g;
        ++steps;
      }
      if (g < 0 || steps >= limit) break;
      f = g;
      x = fr[g].x1 - 1;
      y = fr[g].y1 - 1;
    }
    ++steps;
    Quad p;
    int vid[4];
    load_quad(xy, n, f, p, vid);
    double qx = ((double)x + 0.5) / (double)cols, qy = ((double)y + 0.5) / (double)rows;
    if (bilinear_weights(qx, qy, p, w)) return;
  }
  w[0] = w[1] = w[2] = w[3] = 0.0;
}

__global__ void k_raster(const double* xy, int n, int rows, int cols, int TX, const FaceRaster* fr,
                         const int* starts, const int* faces, double* img) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= cols || y >= rows) return;
  int b = (y / RT) * TX + (x / RT);
  double qx = ((double)x + 0.5) / (double)cols, qy = ((double)y + 0.5) / (double)rows;
  int best = -1;
  for (int k = starts[b]; k < starts[b + 1]; ++k) {
    int f = faces[k];
    if (f <= best) continue;
    FaceRaster r = fr[f];
    if (x < r.x0 || x >= r.x1 || y < r.y0 || y >= r.y1) continue;
    Quad p;
    int vid[4];
    load_quad(xy, n, f, p, vid);
    double w[4];
    if (!bilinear_weights(qx, qy, p, w)) stale_weights(xy, n, rows, cols, fr, f, x, y, w);
    if (weights_inside(w)) best = f;
  }
  img[(size_t)y * cols + x] = best >= 0 ? fr[best].value : 0.0;
}

// ---- host ----

static void build_locator(otm_map* m) {
  otm_context* ctx = m->ctx;
  cudaStream_t st = ctx->stream;
  const int n = m->n, N = n * n;
  const int B = n;
  const int nb = B * B;
  m->bins = B;
  m->bin_start.reserve(sizeof(int) * (nb + 1));
  m->face_box.reserve(sizeof(double4) * N);
  DevBuf counts, sums;
  counts.reserve(sizeof(int) * nb);
  sums.reserve(sizeof(int) * ((nb + SCAN_B - 1) / SCAN_B + 1));
  OTM_CUDA(cudaMemsetAsync(counts.p, 0, sizeof(int) * nb, st));
  const double* xy = m->fwd.as<double>();
  launch(ctx, "bin_count", k_bin_count, (N + 255) / 256, 256, xy, n, B, counts.as<int>(), m->face_box.as<double4>());
  exclusive_scan(st, counts.as<int>(), m->bin_start.as<int>(), sums.as<int>(), nb);
  int total = 0;
  OTM_CUDA(cudaMemcpyAsync(&total, m->bin_start.as<int>() + nb, sizeof(int), cudaMemcpyDeviceToHost, st));
  OTM_CUDA(cudaStreamSynchronize(st));
  m->bin_faces.reserve(sizeof(int) * (size_t)(total > 0 ? total : 1));
  OTM_CUDA(cudaMemsetAsync(counts.p, 0, sizeof(int) * nb, st));
  launch(ctx, "bin_fill", k_bin_fill, (N + 255) / 256, 256, xy, n, B, (const int*)m->bin_start.as<int>(),
         counts.as<int>(), m->bin_faces.as<int>());
  OTM_CUDA(cudaGetLastError());
  OTM_CUDA(cudaStreamSynchronize(st));
  m->located = true;
}

}  // namespace otm

using namespace otm;

extern "C" int otm_map_create(otm_context* ctx, int n, const double* fwd_xy, const double* density, otm_map** out) {
  return guarded([&] {
    if (!ctx || !fwd_xy || !density || !out) throw BadArg{"otm_map_create: null argument"};
    if (n < 1 || n > 16384) throw BadArg{"otm_map_create: grid size out of range"};
    make_current(ctx);
    auto* m = new otm_map;
    m->ctx = ctx;
    m->n = n;
    try {
      size_t V = (size_t)(n + 1) * (n + 1), N = (size_t)n * n;
      m->fwd.reserve(sizeof(double) * 2 * V);
      m->density.reserve(sizeof(double) * N);
      copy_in(ctx, m->fwd.p, fwd_xy, sizeof(double) * 2 * V);
      copy_in(ctx, m->density.p, density, sizeof(double) * N);
      OTM_CUDA(cudaStreamSynchronize(ctx->stream));
    } catch (...) {
      delete m;
      throw;
    }
    *out = m;
    return (int)OTM_OK;
  });
}

extern "C" int otm_map_destroy(otm_map* m) {
  if (!m) return OTM_OK;
  cudaSetDevice(m->ctx->device);
  cudaStreamSynchronize(m->ctx->stream);
  delete m;
  return OTM_OK;
}

extern "C" int otm_map_init_inverse(otm_map* m) {
  return guarded([&] {
    if (!m) throw BadArg{"otm_map_init_inverse: null map"};
    make_current(m->ctx);
    if (!m->located) build_locator(m);
    return (int)OTM_OK;
  });
}

extern "C" int otm_map_inverse(otm_map* m, double* points, long count, int* face, int* nhits, long* missing) {
  return guarded([&] {
    if (!m) throw BadArg{"otm_map_inverse: null map"};
    if (count < 0 || (count > 0 && !points)) throw BadArg{"otm_map_inverse: bad points"};
    otm_context* ctx = m->ctx;
    make_current(ctx);
    if (!m->located) build_locator(m);
    cudaStream_t st = ctx->stream;
    if (count == 0) {
      if (missing) *missing = 0;
      return (int)OTM_OK;
    }
    // device staging: points (2P doubles), faces, nhits, missing counter
    bool pdev = is_device_ptr(points), fdev = face && is_device_ptr(face), hdev = nhits && is_device_ptr(nhits);
    size_t bp = pdev ? 0 : sizeof(double) * 2 * (size_t)count;
    size_t bf = (face && !fdev) ? sizeof(int) * (size_t)count : 0;
    size_t bh = (nhits && !hdev) ? sizeof(int) * (size_t)count : 0;
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    m->scratch.reserve(al(bp) + al(bf) + al(bh) + 256);
    char* base = m->scratch.as<char>();
    double* dp = pdev ? points : reinterpret_cast<double*>(base);
    int* df = face ? (fdev ? face : reinterpret_cast<int*>(base + al(bp))) : nullptr;
    int* dh = nhits ? (hdev ? nhits : reinterpret_cast<int*>(base + al(bp) + al(bf))) : nullptr;
    unsigned long long* dm = reinterpret_cast<unsigned long long*>(base + al(bp) + al(bf) + al(bh));
    if (!pdev) OTM_CUDA(cudaMemcpyAsync(dp, points, bp, cudaMemcpyHostToDevice, st));
    OTM_CUDA(cudaMemsetAsync(dm, 0, sizeof(unsigned long long), st));
    unsigned grid = (unsigned)((count + 255) / 256);
    launch(ctx, "inverse", k_inverse, grid, 256, (const double*)m->fwd.as<double>(),
           (const double*)m->density.as<double>(), m->n, m->bins, (const int*)m->bin_start.as<int>(),
           (const int*)m->bin_faces.as<int>(), (const double4*)m->face_box.as<double4>(), dp, (long)count, df, dh,
           dm);
    OTM_CUDA(cudaGetLastError());
    if (!pdev) OTM_CUDA(cudaMemcpyAsync(points, dp, bp, cudaMemcpyDeviceToHost, st));
    if (face && !fdev) OTM_CUDA(cudaMemcpyAsync(face, df, bf, cudaMemcpyDeviceToHost, st));
    if (nhits && !hdev) OTM_CUDA(cudaMemcpyAsync(nhits, dh, bh, cudaMemcpyDeviceToHost, st));
    unsigned long long miss = 0;
    OTM_CUDA(cudaMemcpyAsync(&miss, dm, sizeof(miss), cudaMemcpyDeviceToHost, st));
    OTM_CUDA(cudaStreamSynchronize(st));
    ctx->prof.flush();
    if (missing) *missing = (long)miss;
    return (int)OTM_OK;
  });
}

extern "C" int otm_rasterize(otm_context* ctx, int n, const double* xy, const double* density, int rows, int cols,
                             double* img) {
  return guarded([&] {
    if (!ctx || !xy || !img) throw BadArg{"otm_rasterize: null argument"};
    if (n < 1 || n > 16384 || rows < 1 || cols < 1 || rows > 65536 || cols > 65536)
      throw BadArg{"otm_rasterize: size out of range"};
    make_current(ctx);
    cudaStream_t st = ctx->stream;
    const int N = n * n;
    size_t V = (size_t)(n + 1) * (n + 1);
    const int TX = (cols + RT - 1) / RT, TY = (rows + RT - 1) / RT, nb = TX * TY;
    size_t pix = (size_t)rows * cols;
    DevBuf dxy, dden, dimg, fr, counts, starts, sums, faces;
    const double* pxy = xy;
    if (!is_device_ptr(xy)) {
      dxy.reserve(sizeof(double) * 2 * V);
      OTM_CUDA(cudaMemcpyAsync(dxy.p, xy, sizeof(double) * 2 * V, cudaMemcpyHostToDevice, st));
      pxy = dxy.as<double>();
    }
    const double* pden = density;
    if (density && !is_device_ptr(density)) {
      dden.reserve(sizeof(double) * N);
      OTM_CUDA(cudaMemcpyAsync(dden.p, density, sizeof(double) * N, cudaMemcpyHostToDevice, st));
      pden = dden.as<double>();
    }
    bool idev = is_device_ptr(img);
    double* pimg = img;
    if (!idev) {
      dimg.reserve(sizeof(double) * pix);
      pimg = dimg.as<double>();
    }
    fr.reserve(sizeof(FaceRaster) * N);
    counts.reserve(sizeof(int) * nb);
    starts.reserve(sizeof(int) * (nb + 1));
    sums.reserve(sizeof(int) * ((nb + SCAN_B - 1) / SCAN_B + 1));
    OTM_CUDA(cudaMemsetAsync(counts.p, 0, sizeof(int) * nb, st));
    float scale = (float)(1. / (double)N);  // rasterizer.cpp:193 keeps this in a float
    launch(ctx, "raster_count", k_raster_count, (N + 255) / 256, 256, pxy, pden, n, scale, rows, cols, TX,
           fr.as<FaceRaster>(), counts.as<int>());
    exclusive_scan(st, counts.as<int>(), starts.as<int>(), sums.as<int>(), nb);
    int total = 0;
    OTM_CUDA(cudaMemcpyAsync(&total, starts.as<int>() + nb, sizeof(int), cudaMemcpyDeviceToHost, st));
    OTM_CUDA(cudaStreamSynchronize(st));
    faces.reserve(sizeof(int) * (size_t)(total > 0 ? total : 1));
    OTM_CUDA(cudaMemsetAsync(counts.p, 0, sizeof(int) * nb, st));
    launch(ctx, "raster_fill", k_raster_fill, (N + 255) / 256, 256, (const FaceRaster*)fr.as<FaceRaster>(), n, TX,
           (const int*)starts.as<int>(), counts.as<int>(), faces.as<int>());
    dim3 blk(32, 8), grd((cols + 31) / 32, (rows + 7) / 8);
    launch(ctx, "raster", k_raster, grd, blk, pxy, n, rows, cols, TX, (const FaceRaster*)fr.as<FaceRaster>(),
           (const int*)starts.as<int>(), (const int*)faces.as<int>(), pimg);
    OTM_CUDA(cudaGetLastError());
    if (!idev) OTM_CUDA(cudaMemcpyAsync(img, pimg, sizeof(double) * pix, cudaMemcpyDeviceToHost, st));
    OTM_CUDA(cudaStreamSynchronize(st));
    ctx->prof.flush();
    return (int)OTM_OK;
  });
}
