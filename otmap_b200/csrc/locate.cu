// Point location in the forward mesh (TransportMap inversion) and rasterization of
// the deformed grid mesh or of any triangle/quad mesh, for sm_100a.
//
// Inversion runs on a uniform bin grid built on the GPU: faces are binned by their
// bounding boxes (count, exclusive scan, scatter) and each query point tests only the
// faces of its bin. Rasterization is face-parallel: each face tests the pixel centres
// of its box and keeps the highest accepting face index per pixel with an integer
// atomicMax; a per-pixel pass then writes the values. This file is compiled without FMA contraction: the geometric
// predicates (utils/mesh_utils.cpp:18-88) then round exactly as the reference's
// scalar x86-64 build does, and the reference's BVH face order and leaf boxes are
// rebuilt on the GPU (build_bvh_order), which makes the located faces, hit counts,
// weights, inverse positions and pixel values bit-identical to the reference.

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
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

// Scans the block sums in place (one block of SCAN_B threads, chunks of SCAN_B values
// with a running carry) and writes the grand total to out[count].
__global__ void k_scan_sums(int* block_sums, int nblocks, int* out, int count) {
  __shared__ int s[SCAN_B];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  for (int c0 = 0; c0 < nblocks; c0 += SCAN_B) {
    const int g = c0 + threadIdx.x;
    const int v = g < nblocks ? block_sums[g] : 0;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < SCAN_B; off <<= 1) {
      int t = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
      __syncthreads();
      s[threadIdx.x] += t;
      __syncthreads();
    }
    if (g < nblocks) block_sums[g] = carry + s[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == SCAN_B - 1) carry += s[threadIdx.x];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[count] = carry;
}

__global__ void k_scan_add(int* out, const int* block_sums, int count) {
  int g = blockIdx.x * SCAN_B + threadIdx.x;
  if (g < count) out[g] += block_sums[blockIdx.x];
}

static void exclusive_scan(cudaStream_t st, const int* counts, int* starts, int* block_sums, int count) {
  int nb = (count + SCAN_B - 1) / SCAN_B;
  k_scan_local<<<nb, SCAN_B, 0, st>>>(counts, starts, block_sums, count);
  k_scan_sums<<<1, SCAN_B, 0, st>>>(block_sums, nb, starts, count);
  k_scan_add<<<nb, SCAN_B, 0, st>>>(starts, block_sums, count);
}

// ---- the reference's BVH face order (utils/bvh2d.cpp:29-64, 165-242) ----
//
// The reference's locator is a BVH over face centroids (leaves of <= 4 faces, depth <= 24,
// TransportMap::init_inverse, transport_map.cpp:36-43). Two of its properties are visible in
// results: the order of the hits of a point (increasing position in its permuted face
// array, the order of the depth-first traversal, bvh2d.cpp:94-162), and that a face is
// only tested where the point lies in the (slightly enlarged) box of the face's leaf.
// Both follow from the permutation the build leaves in its face array, which is
// computed here level by level, all nodes of a level at once:
//   * node box: min / max over its faces' vertices (order-free, exact), enlarged by
//     2 eps diag + eps; split dimension = the first largest extent, split value =
//     float(0.5 (max + min)) of the enlarged box (bvh2d.cpp:178-212);
//   * split() (bvh2d.cpp:167-176) is a two-ended partition. With S the number of
//     "small" centroids (c < split value) in [start, end), the k-th "big" element from
//     the left among the first S positions trades places with the k-th small element
//     from the right among the others -- exactly the pairs its loop swaps -- so prefix
//     counts give every element's final position. Its return value is start + S, plus
//     one when the element then at start + S equals the split value, except in the one
//     loop exit that skips the final scan (last swap at start + S - 2 and start + S);
//   * leaves: <= 4 faces, level >= 24, or a split that leaves one side empty.
// Result per face: rank (position in the final face array) and the box of its leaf.

constexpr int BVH_LEAF = 4, BVH_DEPTH = 24;

struct BvhNode {
  int start, end;
  int leaf, dim;
  float sv;
  int mid, lo, hi;
  unsigned long long kmin[2], kmax[2];  // order-preserving keys of the box (atomics)
  double box[4];                        // enlarged box: min x, min y, max x, max y
};

__device__ __forceinline__ unsigned long long dkey(double x) {
  unsigned long long u = (unsigned long long)__double_as_longlong(x);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double dkey_inv(unsigned long long k) {
  unsigned long long u = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
  return __longlong_as_double((long long)u);
}

__device__ __forceinline__ void bvh_node_init(BvhNode& b, int start, int end) {
  b.start = start;
  b.end = end;
  b.leaf = 0;
  b.lo = b.hi = -1;
  b.kmin[0] = b.kmin[1] = ~0ull;
  b.kmax[0] = b.kmax[1] = 0ull;
}

// Face centroids (bvh2d.cpp:44-58: zero + the corners in circulator order, / 4), face
// boxes, identity permutation, every position in the root node.
__global__ void k_bvh_init(const double* xy, int n, int* fac, double2* cen, double4* fbox, int* node_of,
                           BvhNode* root, int* counts) {
  const int N = n * n;
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f == 0) {
    bvh_node_init(*root, 0, N);
    counts[0] = 1;  // one node in the first level's list
    counts[1] = 0;
  }
  if (f >= N) return;
  Quad p;
  int vid[4];
  load_quad(xy, n, f, p, vid);
  double cx = 0.0, cy = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    cx += p.x[k];
    cy += p.y[k];
  }
  cen[f] = make_double2(cx / 4, cy / 4);
  fbox[f] = make_double4(fmin(fmin(p.x[0], p.x[1]), fmin(p.x[2], p.x[3])),
                         fmin(fmin(p.y[0], p.y[1]), fmin(p.y[2], p.y[3])),
                         fmax(fmax(p.x[0], p.x[1]), fmax(p.x[2], p.x[3])),
                         fmax(fmax(p.y[0], p.y[1]), fmax(p.y[2], p.y[3])));
  fac[f] = f;
  node_of[f] = 0;
}

// Node boxes: per position its face box folded into its node's with 64-bit atomics on
// order-preserving keys. A node's positions are contiguous, so a block whose 256
// positions all belong to one node (the upper levels) reduces them first and issues one
// set of atomics; otherwise every warp reduces each run of equal nodes with a segmented
// shuffle scan and the last lane of a run issues its atomics.
__device__ __forceinline__ double4 box_join(double4 a, double4 b) {
  return make_double4(fmin(a.x, b.x), fmin(a.y, b.y), fmax(a.z, b.z), fmax(a.w, b.w));
}
__device__ __forceinline__ double4 box_shfl_up(double4 b, int o) {
  return make_double4(__shfl_up_sync(0xffffffffu, b.x, o), __shfl_up_sync(0xffffffffu, b.y, o),
                      __shfl_up_sync(0xffffffffu, b.z, o), __shfl_up_sync(0xffffffffu, b.w, o));
}
__device__ __forceinline__ void box_atomic(BvhNode& nd, const double4& b) {
  atomicMin(&nd.kmin[0], dkey(b.x));
  atomicMin(&nd.kmin[1], dkey(b.y));
  atomicMax(&nd.kmax[0], dkey(b.z));
  atomicMax(&nd.kmax[1], dkey(b.w));
}

constexpr int BBOX_T = 256;

__global__ __launch_bounds__(BBOX_T) void k_bvh_bbox(int N, const int* node_of, const double4* fbox, BvhNode* nodes) {
  __shared__ int s_first;
  __shared__ double4 s_box[BBOX_T / 32];
  const int p = blockIdx.x * BBOX_T + threadIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int k = p < N ? node_of[p] : -1;
  double4 b = k >= 0 ? fbox[p] : make_double4(0, 0, 0, 0);
  if (threadIdx.x == 0) s_first = k;
  __syncthreads();
  const int first = s_first;
  if (__syncthreads_and(k == first)) {  // one node (or only finished positions) in the block
    if (first < 0) return;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      b.x = fmin(b.x, __shfl_xor_sync(0xffffffffu, b.x, o));
      b.y = fmin(b.y, __shfl_xor_sync(0xffffffffu, b.y, o));
      b.z = fmax(b.z, __shfl_xor_sync(0xffffffffu, b.z, o));
      b.w = fmax(b.w, __shfl_xor_sync(0xffffffffu, b.w, o));
    }
    if (lane == 0) s_box[warp] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
      double4 t = s_box[0];
#pragma unroll
      for (int w = 1; w < BBOX_T / 32; ++w) t = box_join(t, s_box[w]);
      box_atomic(nodes[first], t);
    }
    return;
  }
  // runs of equal node ids are contiguous: inclusive segmented scan over each run
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double4 u = box_shfl_up(b, o);
    const int ku = __shfl_up_sync(0xffffffffu, k, o);
    if (lane >= o && ku == k) b = box_join(b, u);
  }
  const int kn = __shfl_down_sync(0xffffffffu, k, 1);
  if (k >= 0 && (lane == 31 || kn != k)) box_atomic(nodes[k], b);
}

// Enlarged box, leaf test by size and depth, split dimension and value (bvh2d.cpp:178-212).
__global__ void k_bvh_decide(BvhNode* nodes, const int* count, int level) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= *count) return;
  BvhNode& nd = nodes[k];
  const double mn[2] = {dkey_inv(nd.kmin[0]), dkey_inv(nd.kmin[1])};
  const double mx[2] = {dkey_inv(nd.kmax[0]), dkey_inv(nd.kmax[1])};
  double diag[2];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    diag[c] = mx[c] - mn[c];
    const double en = diag[c] * (2. * DBL_EPSILON) + DBL_EPSILON;
    nd.box[c] = mn[c] - en;
    nd.box[2 + c] = mx[c] + en;
  }
  if (nd.end - nd.start <= BVH_LEAF || level >= BVH_DEPTH) {
    nd.leaf = 1;
    return;
  }
  nd.dim = diag[1] > diag[0] ? 1 : 0;  // Eigen's maxCoeff: the first of equal maxima
  nd.sv = (float)(0.5 * (nd.box[2 + nd.dim] + nd.box[nd.dim]));
}

// small[p] = 1 when position p's centroid lies below its (splitting) node's value.
__global__ void k_bvh_classify(int N, const int* node_of, const double2* cen, const BvhNode* nodes, int* small) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const int k = node_of[p];
  int s = 0;
  if (k >= 0 && !nodes[k].leaf) {
    const double2 c = cen[p];
    s = (nodes[k].dim ? c.y : c.x) < (double)nodes[k].sv ? 1 : 0;
  }
  small[p] = s;
}

// The partition's pairs: big elements among the first S positions (rank from the left)
// and small elements after them (rank from the right) record their positions by rank.
__global__ void k_bvh_slots(int N, const int* node_of, const BvhNode* nodes, const int* small, const int* spre,
                            int* slot_big, int* slot_small) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const int k = node_of[p];
  if (k < 0 || nodes[k].leaf) return;
  const int start = nodes[k].start, end = nodes[k].end;
  const int S = spre[end] - spre[start], q = start + S;
  if (!small[p] && p < q) {
    slot_big[start + (p - start) - (spre[p] - spre[start])] = p;
  } else if (small[p] && p >= q) {
    slot_small[start + spre[end] - spre[p + 1]] = p;
  }
}

// Each big element among the first S positions swaps with its partner (one thread per
// pair, so the swap is race-free).
__global__ void k_bvh_swap(int N, const int* node_of, const BvhNode* nodes, const int* small, const int* spre,
                           const int* slot_small, int* fac, double2* cen, double4* fbox) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const int k = node_of[p];
  if (k < 0 || nodes[k].leaf || small[p]) return;
  const int start = nodes[k].start, end = nodes[k].end;
  const int S = spre[end] - spre[start];
  if (p >= start + S) return;
  const int r = slot_small[start + (p - start) - (spre[p] - spre[start])];
  const int tf = fac[p];
  fac[p] = fac[r];
  fac[r] = tf;
  const double2 tc = cen[p];
  cen[p] = cen[r];
  cen[r] = tc;
  const double4 tb = fbox[p];
  fbox[p] = fbox[r];
  fbox[r] = tb;
}

// split()'s return value (bvh2d.cpp:175), the no-improvement leaf test (:214-221) and
// the children, appended to the next level's list.
__global__ void k_bvh_children(BvhNode* nodes, const int* count, const int* spre, const int* slot_big,
                               const int* slot_small, const double2* cen, BvhNode* next, int* next_count) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= *count) return;
  BvhNode& nd = nodes[k];
  if (nd.leaf) return;
  const int start = nd.start, end = nd.end, len = end - start;
  const int S = spre[end] - spre[start];
  int mid;
  if (S == len) {
    mid = end;  // no big element: the loop runs to `end` and both branches give end
  } else {
    const int q = start + S;
    const int m = S - (spre[q] - spre[start]);  // swapped pairs
    const double2 c = cen[q];
    int eq = (nd.dim ? c.y : c.x) == (double)nd.sv ? 1 : 0;
    // the loop exits right after its last swap (at q - 2 and q) without the final scan:
    // it then tests the small element at q - 1 and returns q
    if (eq && m >= 1 && slot_big[start + m - 1] == q - 2 && slot_small[start + m - 1] == q) eq = 0;
    mid = q + eq;
  }
  nd.mid = mid;
  if (mid == start || mid == end) {
    nd.leaf = 1;
    return;
  }
  const int c0 = atomicAdd(next_count, 2);
  bvh_node_init(next[c0], start, mid);
  bvh_node_init(next[c0 + 1], mid, end);
  nd.lo = c0;
  nd.hi = c0 + 1;
}

// Positions of leaves are final: record rank and leaf box per face; the others move to
// their child node.
__global__ void k_bvh_assign(int N, int* node_of, const BvhNode* nodes, const int* fac, int* rank, double4* lbox) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const int k = node_of[p];
  if (k < 0) return;
  const BvhNode& nd = nodes[k];
  if (nd.leaf) {
    const int f = fac[p];
    rank[f] = p;
    lbox[f] = make_double4(nd.box[0], nd.box[1], nd.box[2], nd.box[3]);
    node_of[p] = -1;
  } else {
    node_of[p] = p < nd.mid ? nd.lo : nd.hi;
  }
}

// rank[f] and the leaf box of f for the n^2 quads of the forward mesh xy (device). The
// levels are a fixed sequence of ~250 small launches for a given n: they run as one CUDA
// graph per size (captured on first use, kept in the context), on the context's grow-only
// scratch, with the mesh copied in and the results copied out around it -- a host that
// enqueues launches slowly then costs one launch instead of ~250. With profiling on, the
// same launches are issued one by one so that each is timed.
static void build_bvh_order(otm_context* ctx, const double* xy, int n, int* rank, double4* lbox) {
  cudaStream_t st = ctx->stream;
  const int N = n * n;
  const int cap = std::min(1 << BVH_DEPTH, 2 * (N / (BVH_LEAF + 1)) + 2);
  auto al = [](size_t b) { return (b + 255) / 256 * 256; };
  const int nsums = (N + 1 + SCAN_B - 1) / SCAN_B + 1;
  const size_t b_fac = al(sizeof(int) * N), b_cen = al(sizeof(double2) * N), b_box = al(sizeof(double4) * N);
  const size_t b_int = al(sizeof(int) * (N + 1)), b_nodes = al(sizeof(BvhNode) * cap), b_sums = al(sizeof(int) * nsums);
  const size_t b_xy = al(sizeof(double) * 2 * (size_t)(n + 1) * (n + 1));
  DevBuf& buf = ctx->bvh_scratch;  // grow-only: no allocation once a size has been built
  buf.reserve(b_fac + b_cen + 2 * b_box + 5 * b_int + 2 * b_nodes + b_sums + b_xy + b_fac + 256);
  char* q = buf.as<char>();
  auto take = [&](size_t b) {
    char* r = q;
    q += b;
    return r;
  };
  int* fac = reinterpret_cast<int*>(take(b_fac));
  double2* cen = reinterpret_cast<double2*>(take(b_cen));
  double4* fbox = reinterpret_cast<double4*>(take(b_box));
  int* node_of = reinterpret_cast<int*>(take(b_int));
  int* small = reinterpret_cast<int*>(take(b_int));
  int* spre = reinterpret_cast<int*>(take(b_int));
  int* slot_big = reinterpret_cast<int*>(take(b_int));
  int* slot_small = reinterpret_cast<int*>(take(b_int));
  BvhNode* lists[2] = {reinterpret_cast<BvhNode*>(take(b_nodes)), reinterpret_cast<BvhNode*>(take(b_nodes))};
  int* sums = reinterpret_cast<int*>(take(b_sums));
  int* counts = reinterpret_cast<int*>(take(256));  // node count of the current and next list
  double* sxy = reinterpret_cast<double*>(take(b_xy));
  int* srank = reinterpret_cast<int*>(take(b_fac));
  double4* slbox = reinterpret_cast<double4*>(take(b_box));
  auto levels = [&]() {
    const unsigned ge = (unsigned)((N + 255) / 256);
    launch(ctx, "bvh_init", k_bvh_init, ge, 256, (const double*)sxy, n, fac, cen, fbox, node_of, lists[0], counts);
    for (int level = 0; level <= BVH_DEPTH; ++level) {
      BvhNode* cur = lists[level & 1];
      BvhNode* nxt = lists[(level + 1) & 1];
      int* ccount = counts + (level & 1);
      int* ncount = counts + ((level + 1) & 1);
      const int ncap = std::min(level < 30 ? (1 << level) : cap, cap);
      const unsigned gn = (unsigned)((ncap + 255) / 256);
      OTM_CUDA(cudaMemsetAsync(ncount, 0, sizeof(int), st));
      launch(ctx, "bvh_bbox", k_bvh_bbox, (unsigned)((N + BBOX_T - 1) / BBOX_T), BBOX_T, N, (const int*)node_of,
             (const double4*)fbox, cur);
      launch(ctx, "bvh_decide", k_bvh_decide, gn, 256, cur, (const int*)ccount, level);
      launch(ctx, "bvh_classify", k_bvh_classify, ge, 256, N, (const int*)node_of, (const double2*)cen,
             (const BvhNode*)cur, small);
      exclusive_scan(st, small, spre, sums, N);
      ctx->launches += 3;
      launch(ctx, "bvh_slots", k_bvh_slots, ge, 256, N, (const int*)node_of, (const BvhNode*)cur, (const int*)small,
             (const int*)spre, slot_big, slot_small);
      launch(ctx, "bvh_swap", k_bvh_swap, ge, 256, N, (const int*)node_of, (const BvhNode*)cur, (const int*)small,
             (const int*)spre, (const int*)slot_small, fac, cen, fbox);
      launch(ctx, "bvh_children", k_bvh_children, gn, 256, cur, (const int*)ccount, (const int*)spre,
             (const int*)slot_big, (const int*)slot_small, (const double2*)cen, nxt, ncount);
      launch(ctx, "bvh_assign", k_bvh_assign, ge, 256, N, node_of, (const BvhNode*)cur, (const int*)fac, srank,
             slbox);
    }
  };
  OTM_CUDA(cudaMemcpyAsync(sxy, xy, sizeof(double) * 2 * (size_t)(n + 1) * (n + 1), cudaMemcpyDeviceToDevice, st));
  if (ctx->prof.on) {
    levels();
  } else {
    auto& slot = ctx->bvh_graphs[n];
    if (!slot || slot->base != buf.p) {
      slot.reset(new otm_context::GraphExec());
      slot->base = buf.p;
      cudaGraph_t g = nullptr;
      const long before = ctx->launches;
      OTM_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      try {
        levels();
      } catch (...) {
        cudaGraph_t dummy;
        cudaStreamEndCapture(st, &dummy);
        if (dummy) cudaGraphDestroy(dummy);
        throw;
      }
      OTM_CUDA(cudaStreamEndCapture(st, &g));
      slot->kernels = ctx->launches - before;
      ctx->launches = before;  // captured, not executed
      const cudaError_t e = cudaGraphInstantiate(&slot->exec, g, 0);
      cudaGraphDestroy(g);
      OTM_CUDA(e);
    }
    OTM_CUDA(cudaGraphLaunch(slot->exec, st));
    ctx->launches += slot->kernels;
  }
  OTM_CUDA(cudaMemcpyAsync(rank, srank, sizeof(int) * N, cudaMemcpyDeviceToDevice, st));
  OTM_CUDA(cudaMemcpyAsync(lbox, slbox, sizeof(double4) * N, cudaMemcpyDeviceToDevice, st));
  OTM_CUDA(cudaGetLastError());
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

// inv_impl (transport_map.cpp:50-102) per point. A face of the point's bin is a hit
// when the point lies in the box of the face's BVH leaf (the reference only reaches
// faces through their leaf, bvh2d.cpp:148-161) and passes the face tests of
// bvh2d.cpp:117-142; hits are ordered by the face's position in the reference's BVH face
// array, its traversal order. With several hits the reference keeps the weights of its
// first hit and the face of the densest later one (transport_map.cpp:70-85); the
// first-hit mode (inv_fast, bvh2d.cpp:66-81) keeps the first.
__global__ void k_inverse(const double* xy, const double* density, int n, int B, const int* starts,
                          const int* faces, const double4* boxes, const int* rank, const double4* lbox, double* pts,
                          long P, int first_hit, int* face_out, int* hit0_out, int* nhits_out,
                          unsigned long long* missing) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  double qx = fmin(fmax(pts[2 * i], 0.), 1.);
  double qy = fmin(fmax(pts[2 * i + 1], 0.), 1.);
  if (!(qx == qx)) qx = 0.;  // NaN input: clamp like Eigen's max/min would not; keep it finite
  if (!(qy == qy)) qy = 0.;
  int bx = (int)fmin(floor(qx * (double)B), (double)(B - 1));
  int by = (int)fmin(floor(qy * (double)B), (double)(B - 1));
  int b = by * B + bx;
  int hf[MAXHITS], hr[MAXHITS];
  double hw[MAXHITS][4];
  int nh = 0;
  for (int k = starts[b]; k < starts[b + 1]; ++k) {
    int f = faces[k];
    double4 bb = boxes[f];
    if (qx < bb.x || qx > bb.z || qy < bb.y || qy > bb.w) continue;
    const double4 lb = lbox[f];
    if (!(lb.x <= qx && lb.y <= qy && qx <= lb.z && qy <= lb.w)) continue;  // AlignedBox::contains
    Quad p;
    int vid[4];
    load_quad(xy, n, f, p, vid);
    double w[4];
    if (!inside_quad(qx, qy, p)) continue;
    if (!bilinear_weights(qx, qy, p, w)) continue;
    if (!weights_inside(w)) continue;
    // insertion in increasing BVH position
    const int rk = rank[f];
    int pos = nh < MAXHITS ? nh : MAXHITS - 1;
    if (nh >= MAXHITS && rk > hr[MAXHITS - 1]) {
      ++nh;
      continue;
    }
    while (pos > 0 && hr[pos - 1] > rk) {
      hf[pos] = hf[pos - 1];
      hr[pos] = hr[pos - 1];
#pragma unroll
      for (int c = 0; c < 4; ++c) hw[pos][c] = hw[pos - 1][c];
      --pos;
    }
    hf[pos] = f;
    hr[pos] = rk;
#pragma unroll
    for (int c = 0; c < 4; ++c) hw[pos][c] = w[c];
    ++nh;
  }
  if (nhits_out) nhits_out[i] = nh;
  if (hit0_out) hit0_out[i] = nh > 0 ? hf[0] : -1;
  if (nh == 0) {
    pts[2 * i] = NAN;
    pts[2 * i + 1] = NAN;
    if (face_out) face_out[i] = -1;
    atomicAdd(missing, 1ull);
    return;
  }
  int f = hf[0];
  int kmax = nh < MAXHITS ? nh : MAXHITS;
  if (nh > 1 && !first_hit) {
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

// ---- rasterization (utils/rasterizer.cpp:36-58, 86-185, 188-302) ----

// A mesh to rasterize: the quads of the (n+1)^2 grid (start == nullptr), or an indexed
// face set of triangles and quads whose face f lists vertices idx[start[f] .. start[f+1])
// in the order the reference's face circulator visits them.
struct MeshRef {
  const double* xy;
  int n;       // grid size (grid meshes only)
  int nf;      // faces
  int nv;      // vertices
  const int* start;
  const int* idx;
};

// Loads face f's corners; returns its valence (3 or 4). Triangles repeat their last
// corner in slot 3, which leaves their bounding box unchanged.
__device__ __forceinline__ int load_face(const MeshRef& m, int f, Quad& p, int vid[4]) {
  if (!m.start) {
    load_quad(m.xy, m.n, f, p, vid);
    return 4;
  }
  const int s = m.start[f];
  const int c = m.start[f + 1] - s;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    vid[k] = m.idx[s + (k < c ? k : c - 1)];
    p.x[k] = m.xy[2 * (size_t)vid[k]];
    p.y[k] = m.xy[2 * (size_t)vid[k] + 1];
  }
  return c;
}

// |area| of a face as rasterize_image takes it (eigen_addons.h:18-23).
__device__ __forceinline__ double face_abs_area(const Quad& p, int c) {
  if (c == 3) return fabs(signed_area3(p.x[0], p.y[0], p.x[1], p.y[1], p.x[2], p.y[2]));
  return fabs(signed_area3(p.x[0], p.y[0], p.x[1], p.y[1], p.x[2], p.y[2]) +
              signed_area3(p.x[0], p.y[0], p.x[2], p.y[2], p.x[3], p.y[3]));
}

// BarycentricTransform (rasterizer.cpp:36-58): T = [s1-s3 | s2-s3], inverted as Eigen
// inverts a 2x2 matrix (adjugate times 1/det), b = T^-1 (q - s3), bary = (b0, b1, 1-b0-b1).
__device__ __forceinline__ void tri_weights(double qx, double qy, const Quad& p, double w[4]) {
  const double m00 = p.x[0] - p.x[2], m10 = p.y[0] - p.y[2];
  const double m01 = p.x[1] - p.x[2], m11 = p.y[1] - p.y[2];
  const double invdet = 1.0 / (m00 * m11 - m10 * m01);
  const double t00 = m11 * invdet, t10 = -m10 * invdet, t01 = -m01 * invdet, t11 = m00 * invdet;
  const double vx = qx - p.x[2], vy = qy - p.y[2];
  const double b0 = t00 * vx + t01 * vy;
  const double b1 = t10 * vx + t11 * vy;
  w[0] = b0;
  w[1] = b1;
  w[2] = 1.0 - b0 - b1;
  w[3] = 0.0;
}

struct FaceRaster {
  int x0, x1, y0, y1;  // pixel box [x0,x1) x [y0,y1), as rasterize_face computes it
  double value;        // PerFace value: float(1/N) * density / |area|
};

__device__ __forceinline__ FaceRaster face_raster(const MeshRef& m, const double* density, float scale, int rows,
                                                  int cols, int f) {
  Quad p;
  int vid[4];
  const int c = load_face(m, f, p, vid);
  FaceRaster r;
  double in_mass = scale * (density ? density[f] : 1.0);
  r.value = in_mass / face_abs_area(p, c);
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

__global__ void k_face_boxes(MeshRef m, const double* density, float scale, int rows, int cols, FaceRaster* fr) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= m.nf) return;
  fr[f] = face_raster(m, density, scale, rows, cols, f);
}

// Weights the reference's sequential loop would test at (f, x, y) when its bilinear
// solve fails there (D < 0): its Vector4d is never written, and the optimised build
// then reads the weights of the most recent successful solve. Walk back through the
// loop order -- earlier pixels of face f's box row by row, then earlier quads -- to
// the most recent pixel whose solve succeeds. Bounded; gives zeros (the start state)
// when it runs out, as the sequential emulation does before any solve. Triangles
// never touch that Vector4d and are passed over.
__device__ void stale_weights(const MeshRef& m, int rows, int cols, const FaceRaster* fr, int f, int x, int y,
                              double w[4]) {
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
      // last pixel of the previous quad with a non-empty box
      int g = f - 1;
      while (g >= 0 && steps < limit) {
        const bool empty = fr[g].x0 >= fr[g].x1 || fr[g].y0 >= fr[g].y1;
        const bool tri = m.start && (m.start[g + 1] - m.start[g] == 3);
        if (!empty && !tri) break;
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
    load_face(m, f, p, vid);
    double qx = ((double)x + 0.5) / (double)cols, qy = ((double)y + 0.5) / (double)rows;
    if (bilinear_weights(qx, qy, p, w)) return;
  }
  w[0] = w[1] = w[2] = w[3] = 0.0;
}

// Weights of face f at the centre of pixel (x, y) as the reference's loop forms them
// (triangles: the barycentric transform; quads: bilinear coordinates, or the stale
// weights where that solve fails). Returns the face's valence; vid gets its corners.
__device__ __forceinline__ int pixel_weights(const MeshRef& m, int rows, int cols, const FaceRaster* fr, int f,
                                             int x, int y, double w[4], int vid[4]) {
  Quad p;
  const int c = load_face(m, f, p, vid);
  const double qx = ((double)x + 0.5) / (double)cols, qy = ((double)y + 0.5) / (double)rows;
  if (c == 3) {
    tri_weights(qx, qy, p, w);
  } else if (!bilinear_weights(qx, qy, p, w)) {
    stale_weights(m, rows, cols, fr, f, x, y, w);
  }
  return c;
}

// Box rows per face (0 for an empty box): the work list of k_raster_owner_rows.
__global__ void k_box_rows(int nf, const FaceRaster* fr, int* rows_of) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  const FaceRaster r = fr[f];
  rows_of[f] = (r.x0 < r.x1 && r.y0 < r.y1) ? r.y1 - r.y0 : 0;
}

// The owner pass: every pixel centre of a face's box that the face accepts records the
// face index with atomicMax, so each pixel ends with the highest accepting index -- the
// face the reference's sequential loop writes last (rasterizer.cpp:162-236). One thread
// per (face, box row) rather than per face: a stretched face
// (the inverse maps of sharp densities have some that span much of the image) spreads over
// as many threads as its box has rows, instead of holding one thread for its whole box
// while the rest of the grid idles. Work item t belongs to the last face f with
// row_start[f] <= t (row_start: exclusive prefix of the box rows, total at [nf]); grid-
// stride over the total, which is read on the device. Same atomicMax of the face index,
// so the owners are those of the per-face pass.
__global__ void k_raster_owner_rows(MeshRef m, int rows, int cols, const FaceRaster* fr, const int* row_start,
                                    int* owner) {
  const int nf = m.nf;
  const int total = row_start[nf];
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    int lo = 0, hi = nf;  // row_start[lo] <= t < row_start[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (row_start[mid] <= t) lo = mid; else hi = mid;
    }
    const int f = lo;
    const FaceRaster r = fr[f];
    const int y = r.y0 + (t - row_start[f]);
    Quad p;
    int vid[4];
    const int c = load_face(m, f, p, vid);
    const double qy = ((double)y + 0.5) / (double)rows;
    for (int x = r.x0; x < r.x1; ++x) {
      const double qx = ((double)x + 0.5) / (double)cols;
      double w[4];
      if (c == 3) {
        tri_weights(qx, qy, p, w);
      } else if (!bilinear_weights(qx, qy, p, w)) {
        stale_weights(m, rows, cols, fr, f, x, y, w);
      }
      if (weights_inside(w)) atomicMax(&owner[(size_t)y * cols + x], f);
    }
  }
}

// One thread per pixel: the owner's PerFace value, or for PerVertex (vval != nullptr)
// the float interpolation of rasterize_face's loop, which scales vertex 0's value by
// each weight (rasterizer.cpp:123-130, 174-181) and sums in float.
__global__ void k_raster_resolve(MeshRef m, int rows, int cols, const FaceRaster* fr, const int* owner,
                                 const float* vval, double* img) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= cols || y >= rows) return;
  const int f = owner[(size_t)y * cols + x];
  double out = 0.0;
  if (f >= 0) {
    if (vval) {
      double w[4];
      int vid[4];
      const int c = pixel_weights(m, rows, cols, fr, f, x, y, w, vid);
      const float v0 = vval[vid[0]];
      float acc = 0.0f;
      for (int q = 0; q < c; ++q) acc = acc + v0 * (float)w[q];
      out = (double)acc;
    } else {
      out = fr[f].value;
    }
  }
  img[(size_t)y * cols + x] = out;
}

// PerVertex values (rasterizer.cpp:240-271) on the grid mesh: each vertex sums, in
// float and in face order, 1/|area| over its faces, then takes float(scale) * value /
// (number of faces) with the reference's float and double steps.
__global__ void k_vertex_values_grid(const double* xy, int n, float scale, float* value) {
  const long v = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long V = (long)(n + 1) * (n + 1);
  if (v >= V) return;
  const int vi = (int)(v / (n + 1)), vj = (int)(v % (n + 1));
  float acc = 0.0f;
  double div = 0.0;
  // faces around vertex (vi, vj) in increasing index j + i*n
  const int ci[4] = {vi - 1, vi - 1, vi, vi}, cj[4] = {vj - 1, vj, vj - 1, vj};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (ci[k] < 0 || cj[k] < 0 || ci[k] >= n || cj[k] >= n) continue;
    Quad p;
    int vid[4];
    load_quad(xy, n, cj[k] + ci[k] * n, p, vid);
    acc = (float)((double)acc + 1. / face_abs_area(p, 4));
    div += 1.;
  }
  value[v] = (float)((double)(scale * acc) / div);
}

// Indexed meshes: vertex -> face lists (count, scan, scatter, then each list sorted by
// face index so the float sums run in the reference's face order).
__global__ void k_vf_count(MeshRef m, int* counts) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= m.nf) return;
  for (int k = m.start[f]; k < m.start[f + 1]; ++k) atomicAdd(&counts[m.idx[k]], 1);
}

__global__ void k_vf_fill(MeshRef m, const int* vstart, int* cursor, int* vfaces, double* inv_area) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= m.nf) return;
  Quad p;
  int vid[4];
  const int c = load_face(m, f, p, vid);
  inv_area[f] = 1. / face_abs_area(p, c);
  for (int k = m.start[f]; k < m.start[f + 1]; ++k) {
    const int v = m.idx[k];
    vfaces[vstart[v] + atomicAdd(&cursor[v], 1)] = f;
  }
}

__global__ void k_vertex_values_mesh(int nv, const int* vstart, int* vfaces, const double* inv_area, float scale,
                                     float* value) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const int s = vstart[v], e = vstart[v + 1];
  for (int a = s + 1; a < e; ++a) {  // insertion sort: lists are short
    int f = vfaces[a], b = a;
    while (b > s && vfaces[b - 1] > f) {
      vfaces[b] = vfaces[b - 1];
      --b;
    }
    vfaces[b] = f;
  }
  float acc = 0.0f;
  double div = 0.0;
  for (int a = s; a < e; ++a) {
    acc = (float)((double)acc + inv_area[vfaces[a]]);
    div += 1.;
  }
  value[v] = (float)((double)(scale * acc) / div);
}

// ---- backward of the grid raster and of the grid inversion (differentiable barycenters) ----

// dL/dA_f per face of a grid mesh from the pixels it owns in the last raster: an owned
// pixel's PerFace value is scale / |A_f| with A_f the signed fan area of face_abs_area,
// so d value / d A_f = -value / A_f.
__global__ void k_raster_area_grad(MeshRef m, int rows, int cols, const FaceRaster* fr, const int* owner,
                                   const double* dL_dpix, double* dL_dA) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= m.nf) return;
  const FaceRaster r = fr[f];
  double acc = 0.0;
  for (int y = r.y0; y < r.y1; ++y)
    for (int x = r.x0; x < r.x1; ++x) {
      const size_t q = (size_t)y * cols + x;
      if (owner[q] == f) acc += dL_dpix[q];
    }
  Quad p;
  int vid[4];
  load_face(m, f, p, vid);
  const double A = signed_area3(p.x[0], p.y[0], p.x[1], p.y[1], p.x[2], p.y[2]) +
                   signed_area3(p.x[0], p.y[0], p.x[2], p.y[2], p.x[3], p.y[3]);
  dL_dA[f] = (acc != 0.0 && A != 0.0) ? -acc * r.value / A : 0.0;
}

// Per vertex (i, j) of the grid mesh, in a fixed order over the faces around it (face
// (i,j) corner 0, (i-1,j) corner 1, (i-1,j-1) corner 2, (i,j-1) corner 3): with dL_dA,
// sum_f dL/dA_f times the shoelace gradient dA/dx_c = (y_{c+1} - y_{c-1}) / 2,
// dA/dy_c = (x_{c-1} - x_{c+1}) / 2; with cs, the per-face corner sums cs[f][c] as they are.
__global__ void k_grid_vertex_gather(const double* xy, int n, const double* dL_dA, const double2* cs, double* out) {
  const long v = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long V = (long)(n + 1) * (n + 1);
  if (v >= V) return;
  const int i = (int)(v / (n + 1)), j = (int)(v % (n + 1));
  double gx = 0.0, gy = 0.0;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int a = i - ((c == 1 || c == 2) ? 1 : 0), b = j - ((c == 2 || c == 3) ? 1 : 0);
    if (a < 0 || b < 0 || a >= n || b >= n) continue;
    const int f = b + a * n;
    if (cs) {
      const double2 t = cs[4 * (size_t)f + c];
      gx += t.x;
      gy += t.y;
    } else {
      const double g = dL_dA[f];
      if (g == 0.0) continue;
      Quad p;
      int vid[4];
      load_quad(xy, n, f, p, vid);
      const int nx = (c + 1) & 3, pv = (c + 3) & 3;
      gx += g * (0.5 * (p.y[nx] - p.y[pv]));
      gy += g * (0.5 * (p.x[pv] - p.x[nx]));
    }
  }
  out[2 * v] = gx;
  out[2 * v + 1] = gy;
}

struct InvGrad {  // per located origin vertex: q = -e J^-T dL/dI and the weights of its first hit
  double qx, qy, w[4];
};

// Origin vertex v = (i * (1/n), j * (1/n)) (mesh_utils.cpp:100-108) located in face
// h = hit0[v] of the forward mesh with weights w of the bilinear coordinates
// (u, v) = (w1 + w2, w2 + w3): its inverse position is I = sum_c w_c O_c with O the
// origin corners (a square of side e, so dI/d(u,v) = e Id), and x = sum_c w_c P_c with P
// the forward corners. Holding x fixed, d(u,v) = -J^-1 sum_c w_c dP_c with
// J = [dx/du | dx/dv], hence dL/dP_c = -e w_c J^-T dL/dI.
__global__ void k_inv_point_grad(const double* fwd, int n, const int* hit0, const double* dL_dI, InvGrad* pg,
                                 int* count) {
  const long v = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long V = (long)(n + 1) * (n + 1);
  if (v >= V) return;
  InvGrad g;
  g.qx = g.qy = 0.0;
  g.w[0] = g.w[1] = g.w[2] = g.w[3] = 0.0;
  const int h = hit0[v];
  if (h >= 0) {
    const double dx = 1.0 / (double)n;
    const double qx = (double)(v / (n + 1)) * dx, qy = (double)(v % (n + 1)) * dx;
    Quad P;
    int vid[4];
    load_quad(fwd, n, h, P, vid);
    double w[4];
    if (bilinear_weights(qx, qy, P, w)) {
      const double u = w[1] + w[2], t = w[2] + w[3];
      const double jux = (1.0 - t) * (P.x[1] - P.x[0]) + t * (P.x[2] - P.x[3]);
      const double juy = (1.0 - t) * (P.y[1] - P.y[0]) + t * (P.y[2] - P.y[3]);
      const double jvx = (1.0 - u) * (P.x[3] - P.x[0]) + u * (P.x[2] - P.x[1]);
      const double jvy = (1.0 - u) * (P.y[3] - P.y[0]) + u * (P.y[2] - P.y[1]);
      const double det = jux * jvy - juy * jvx;
      if (det != 0.0 && isfinite(det)) {
        const double gx = dL_dI[2 * v], gy = dL_dI[2 * v + 1];
        const double s = -dx / det;
        g.qx = s * (jvy * gx - juy * gy);
        g.qy = s * (-jvx * gx + jux * gy);
#pragma unroll
        for (int c = 0; c < 4; ++c) g.w[c] = w[c];
      }
    }
    atomicAdd(&count[h], 1);
  }
  pg[v] = g;
}

__global__ void k_inv_fill(long V, const int* hit0, const int* start, int* cursor, int* list) {
  const long v = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V) return;
  const int h = hit0[v];
  if (h >= 0) list[start[h] + atomicAdd(&cursor[h], 1)] = (int)v;
}

// Per face: its points in increasing index order (the fill order is arbitrary), then the
// corner sums cs[f][c] = sum_points w_c q in that order.
__global__ void k_inv_face_sums(int N, const int* start, int* list, const InvGrad* pg, double2* cs) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= N) return;
  const int b = start[f], e = start[f + 1];
  for (int a = b + 1; a < e; ++a) {  // insertion sort: lists hold a few points
    const int key = list[a];
    int k = a - 1;
    while (k >= b && list[k] > key) {
      list[k + 1] = list[k];
      --k;
    }
    list[k + 1] = key;
  }
  double2 acc[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) acc[c] = make_double2(0.0, 0.0);
  for (int a = b; a < e; ++a) {
    const InvGrad g = pg[list[a]];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      acc[c].x += g.w[c] * g.qx;
      acc[c].y += g.w[c] * g.qy;
    }
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) cs[4 * (size_t)f + c] = acc[c];
}

// ---- host ----

static void build_locator(otm_map* m) {
  otm_context* ctx = m->ctx;
  cudaStream_t st = ctx->stream;
  const int n = m->n, N = n * n;
  const int B = n;
  const int nb = B * B;
  m->bins = B;
  m->bin_start.reserve(sizeof(int) * (nb + 1), ctx->stream, ctx->pool);
  m->face_box.reserve(sizeof(double4) * N, ctx->stream, ctx->pool);
  // bin counts and scan sums in the context's grow-only scratch
  const size_t b_counts = (sizeof(int) * nb + 255) / 256 * 256;
  ctx->locate_scratch.reserve(b_counts + sizeof(int) * ((nb + SCAN_B - 1) / SCAN_B + 1));
  int* counts = ctx->locate_scratch.as<int>();
  int* sums = reinterpret_cast<int*>(ctx->locate_scratch.as<char>() + b_counts);
  OTM_CUDA(cudaMemsetAsync(counts, 0, sizeof(int) * nb, st));
  const double* xy = m->fwd.as<double>();
  launch(ctx, "bin_count", k_bin_count, (N + 255) / 256, 256, xy, n, B, counts, m->face_box.as<double4>());
  exclusive_scan(st, counts, m->bin_start.as<int>(), sums, nb);
  int total = 0;
  OTM_CUDA(cudaMemcpyAsync(&total, m->bin_start.as<int>() + nb, sizeof(int), cudaMemcpyDeviceToHost, st));
  OTM_CUDA(cudaStreamSynchronize(st));
  m->bin_faces.reserve(sizeof(int) * (size_t)(total > 0 ? total : 1), ctx->stream, ctx->pool);
  OTM_CUDA(cudaMemsetAsync(counts, 0, sizeof(int) * nb, st));
  launch(ctx, "bin_fill", k_bin_fill, (N + 255) / 256, 256, xy, n, B, (const int*)m->bin_start.as<int>(), counts,
         m->bin_faces.as<int>());
  OTM_CUDA(cudaGetLastError());
  m->bvh_rank.reserve(sizeof(int) * N, ctx->stream, ctx->pool);
  m->leaf_box.reserve(sizeof(double4) * N, ctx->stream, ctx->pool);
  build_bvh_order(ctx, xy, n, m->bvh_rank.as<int>(), m->leaf_box.as<double4>());
  m->located = true;
}

}  // namespace otm

namespace otm {

// Inversion of `count` points (device buffers) through map m, in place; face / hit0 (the
// first hit in the reference's order) / nhits may be null; missing is added to.
void map_inverse_dev(otm_map* m, double* pts, long count, int mode, int* face, int* hit0, int* nhits,
                     unsigned long long* missing) {
  otm_context* ctx = m->ctx;
  if (!m->located) build_locator(m);
  if (count <= 0) return;
  const unsigned grid = (unsigned)((count + 255) / 256);
  launch(ctx, "inverse", k_inverse, grid, 256, (const double*)m->fwd.as<double>(),
         (const double*)m->density.as<double>(), m->n, m->bins, (const int*)m->bin_start.as<int>(),
         (const int*)m->bin_faces.as<int>(), (const double4*)m->face_box.as<double4>(),
         (const int*)m->bvh_rank.as<int>(), (const double4*)m->leaf_box.as<double4>(), pts, count,
         mode == OTM_INV_FIRST ? 1 : 0, face, hit0, nhits, missing);
  OTM_CUDA(cudaGetLastError());
}

void raster_grid_backward(otm_context* ctx, int n, const double* xy, int rows, int cols, const double* dL_dpix,
                          double* dL_dxy) {
  const int N = n * n;
  auto al = [](size_t b) { return (b + 255) / 256 * 256; };
  // the layout raster_mesh leaves in the scratch: face boxes, then pixel owners
  const char* base = ctx->raster_scratch.as<char>();
  const FaceRaster* fr = reinterpret_cast<const FaceRaster*>(base);
  const int* owner = reinterpret_cast<const int*>(base + al(sizeof(FaceRaster) * (size_t)(N > 0 ? N : 1)));
  DevBuf dA;
  dA.reserve(sizeof(double) * N);
  MeshRef m{xy, n, N, (n + 1) * (n + 1), nullptr, nullptr};
  launch(ctx, "raster_area_grad", k_raster_area_grad, (N + 255) / 256, 256, m, rows, cols, fr, owner, dL_dpix,
         dA.as<double>());
  const long V = (long)(n + 1) * (n + 1);
  launch(ctx, "area_vertex_grad", k_grid_vertex_gather, (unsigned)((V + 255) / 256), 256, xy, n,
         (const double*)dA.as<double>(), (const double2*)nullptr, dL_dxy);
  OTM_CUDA(cudaGetLastError());
  OTM_CUDA(cudaStreamSynchronize(ctx->stream));  // dA is released on return
}

void inverse_grid_backward(otm_context* ctx, int n, const double* fwd, const int* hit0, const double* dL_dI,
                           double* dL_dfwd) {
  cudaStream_t st = ctx->stream;
  const int N = n * n;
  const long V = (long)(n + 1) * (n + 1);
  auto al = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t b_pg = al(sizeof(InvGrad) * V), b_cnt = al(sizeof(int) * (N + 1)), b_list = al(sizeof(int) * V);
  const size_t b_cs = al(sizeof(double2) * 4 * (size_t)N), b_sums = al(sizeof(int) * ((N + SCAN_B - 1) / SCAN_B + 1));
  DevBuf buf;
  buf.reserve(b_pg + 3 * b_cnt + b_list + b_cs + b_sums);
  char* q = buf.as<char>();
  InvGrad* pg = reinterpret_cast<InvGrad*>(q);
  int* count = reinterpret_cast<int*>(q + b_pg);
  int* start = reinterpret_cast<int*>(q + b_pg + b_cnt);
  int* cursor = reinterpret_cast<int*>(q + b_pg + 2 * b_cnt);
  int* list = reinterpret_cast<int*>(q + b_pg + 3 * b_cnt);
  double2* cs = reinterpret_cast<double2*>(q + b_pg + 3 * b_cnt + b_list);
  int* sums = reinterpret_cast<int*>(q + b_pg + 3 * b_cnt + b_list + b_cs);
  OTM_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * N, st));
  OTM_CUDA(cudaMemsetAsync(cursor, 0, sizeof(int) * N, st));
  const unsigned gv = (unsigned)((V + 255) / 256), gf = (unsigned)((N + 255) / 256);
  launch(ctx, "inv_point_grad", k_inv_point_grad, gv, 256, fwd, n, hit0, dL_dI, pg, count);
  exclusive_scan(st, count, start, sums, N);
  launch(ctx, "inv_fill", k_inv_fill, gv, 256, V, hit0, (const int*)start, cursor, list);
  launch(ctx, "inv_face_sums", k_inv_face_sums, gf, 256, N, (const int*)start, list, (const InvGrad*)pg, cs);
  launch(ctx, "inv_vertex_grad", k_grid_vertex_gather, gv, 256, fwd, n, (const double*)nullptr, (const double2*)cs,
         dL_dfwd);
  OTM_CUDA(cudaGetLastError());
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
      m->fwd.reserve(sizeof(double) * 2 * V, ctx->stream, ctx->pool);
      m->density.reserve(sizeof(double) * N, ctx->stream, ctx->pool);
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
  delete m;  // the buffers are freed in stream order, after the work queued on them
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

extern "C" int otm_map_inverse_mode(otm_map* m, double* points, long count, int mode, int* face, int* nhits,
                                   long* missing) {
  return guarded([&] {
    if (!m) throw BadArg{"otm_map_inverse: null map"};
    if (mode != OTM_INV_DENSEST && mode != OTM_INV_FIRST) throw BadArg{"otm_map_inverse: unknown mode"};
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
    m->scratch.reserve(al(bp) + al(bf) + al(bh) + 256, ctx->stream, ctx->pool);
    char* base = m->scratch.as<char>();
    double* dp = pdev ? points : reinterpret_cast<double*>(base);
    int* df = face ? (fdev ? face : reinterpret_cast<int*>(base + al(bp))) : nullptr;
    int* dh = nhits ? (hdev ? nhits : reinterpret_cast<int*>(base + al(bp) + al(bf))) : nullptr;
    unsigned long long* dm = reinterpret_cast<unsigned long long*>(base + al(bp) + al(bf) + al(bh));
    if (!pdev) OTM_CUDA(cudaMemcpyAsync(dp, points, bp, cudaMemcpyHostToDevice, st));
    OTM_CUDA(cudaMemsetAsync(dm, 0, sizeof(unsigned long long), st));
    map_inverse_dev(m, dp, (long)count, mode, df, nullptr, dh, dm);
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

extern "C" int otm_map_inverse(otm_map* m, double* points, long count, int* face, int* nhits, long* missing) {
  return otm_map_inverse_mode(m, points, count, OTM_INV_DENSEST, face, nhits, missing);
}

// ---- stochastic splatting (utils/stochastic_rasterizer.cpp:19-88) ----

// Counter-based uniform doubles in [0, 1): the splitmix64 output function (Steele, Lea
// and Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014) applied to
// a key made of (seed, face, sample, draw), so any sample can be drawn independently.
__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

__device__ __forceinline__ double splat_uniform(unsigned long long face_key, long sample, int draw) {
  const unsigned long long x = mix64(face_key + (unsigned long long)(2 * sample + draw + 1) * 0x9e3779b97f4a7c15ULL);
  return (double)(x >> 11) * 0x1.0p-53;
}

// One warp per face: each of the face's samples is a random point of the face (uniform
// bilinear coordinates for a quad, uniform barycentric ones for a triangle), counted in
// the pixel that contains it. Counts are integers, so the atomic additions are exact and
// the image does not depend on their order.
__global__ void k_splat(MeshRef m, const int* spf, unsigned long long seed, int rows, int cols, double* img) {
  const int lane = threadIdx.x & 31;
  const long f = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (f >= m.nf) return;
  const int ns = spf[f];
  if (ns <= 0) return;
  Quad p;
  int vid[4];
  const int c = load_face(m, (int)f, p, vid);
  const unsigned long long key = mix64(seed ^ mix64((unsigned long long)(f + 1) * 0xd1b54a32d192ed03ULL));
  const double dx = 1. / double(cols), dy = 1. / double(rows);
  for (long s = lane; s < ns; s += 32) {
    double px, py;
    if (c == 3) {
      const double r1 = sqrt(splat_uniform(key, s, 0)), r2 = splat_uniform(key, s, 1);
      const double b0 = 1. - r1, b1 = r1 * (1. - r2), b2 = r1 * r2;
      px = b0 * p.x[0] + b1 * p.x[1] + b2 * p.x[2];
      py = b0 * p.y[0] + b1 * p.y[1] + b2 * p.y[2];
    } else {
      const double u = splat_uniform(key, s, 0), v = splat_uniform(key, s, 1);
      const double w0 = (1. - u) * (1 - v), w1 = (u) * (1 - v), w2 = (u) * (v), w3 = (1. - u) * (v);
      px = w0 * p.x[0] + w1 * p.x[1] + w2 * p.x[2] + w3 * p.x[3];
      py = w0 * p.y[0] + w1 * p.y[1] + w2 * p.y[2] + w3 * p.y[3];
    }
    // stochastic_rasterizer.cpp:71-83: points off the unit square (or not finite) are dropped
    if (!(px >= 0 && py >= 0 && px <= 1 && py <= 1)) continue;
    const int pi = (int)(py / dy), pj = (int)(px / dx);
    if (pi < rows && pj < cols) atomicAdd(&img[(size_t)pi * cols + pj], 1.0);
  }
}

namespace otm {

// Rasterizes mesh m (all pointers on the device) into img (device, rows*cols).
static void raster_mesh(otm_context* ctx, const MeshRef& m, const double* density, int cells, int rows, int cols,
                        int mode, double* img) {
  cudaStream_t st = ctx->stream;
  const int nf = m.nf;
  const size_t pix = (size_t)rows * cols;
  auto al = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t b_fr = al(sizeof(FaceRaster) * (size_t)(nf > 0 ? nf : 1)), b_own = al(sizeof(int) * pix);
  const size_t b_vv = al(sizeof(float) * (size_t)(m.nv > 0 ? m.nv : 1));
  const size_t b_rows = al(sizeof(int) * (size_t)(nf + 1)), b_rs = al(sizeof(int) * ((nf + SCAN_B) / SCAN_B + 1));
  ctx->raster_scratch.reserve(b_fr + b_own + b_vv + 2 * b_rows + b_rs);  // grows, kept for the next call
  char* base = ctx->raster_scratch.as<char>();
  FaceRaster* fr = reinterpret_cast<FaceRaster*>(base);
  int* owner = reinterpret_cast<int*>(base + b_fr);
  float* vval = reinterpret_cast<float*>(base + b_fr + b_own);
  int* rows_of = reinterpret_cast<int*>(base + b_fr + b_own + b_vv);
  int* row_start = reinterpret_cast<int*>(base + b_fr + b_own + b_vv + b_rows);
  int* row_sums = reinterpret_cast<int*>(base + b_fr + b_own + b_vv + 2 * b_rows);
  OTM_CUDA(cudaMemsetAsync(owner, 0xff, sizeof(int) * pix, st));  // -1: no face
  // rasterizer.cpp:193 keeps 1/density.size() in a float
  const float scale = (float)(1. / (double)(density ? cells : nf));
  const int fblocks = nf > 0 ? (nf + 255) / 256 : 1;
  launch(ctx, "face_boxes", k_face_boxes, fblocks, 256, m, density, scale, rows, cols, fr);
  if (nf > 0) {
    launch(ctx, "box_rows", k_box_rows, fblocks, 256, nf, (const FaceRaster*)fr, rows_of);
    exclusive_scan(st, rows_of, row_start, row_sums, nf);
    ctx->launches += 3;
    launch(ctx, "raster_owner", k_raster_owner_rows, ctx->num_sms * 8, 256, m, rows, cols, (const FaceRaster*)fr,
           (const int*)row_start, owner);
  }
  const float* pv = nullptr;
  DevBuf vcount, vstart, vsums, vfaces, inv_area;  // indexed PerVertex temporaries
  if (mode == OTM_RIO_PER_VERTEX) {
    const unsigned vb = (unsigned)((m.nv + 255) / 256);
    if (!m.start) {
      launch(ctx, "vertex_values", k_vertex_values_grid, vb, 256, m.xy, m.n, scale, vval);
    } else {
      int nref = 0;
      OTM_CUDA(cudaMemcpyAsync(&nref, m.start + nf, sizeof(int), cudaMemcpyDeviceToHost, st));
      vcount.reserve(sizeof(int) * m.nv);
      vstart.reserve(sizeof(int) * (m.nv + 1));
      vsums.reserve(sizeof(int) * ((m.nv + SCAN_B - 1) / SCAN_B + 1));
      inv_area.reserve(sizeof(double) * (size_t)(nf > 0 ? nf : 1));
      OTM_CUDA(cudaMemsetAsync(vcount.p, 0, sizeof(int) * m.nv, st));
      launch(ctx, "vf_count", k_vf_count, fblocks, 256, m, vcount.as<int>());
      exclusive_scan(st, vcount.as<int>(), vstart.as<int>(), vsums.as<int>(), m.nv);
      OTM_CUDA(cudaStreamSynchronize(st));
      vfaces.reserve(sizeof(int) * (size_t)(nref > 0 ? nref : 1));
      OTM_CUDA(cudaMemsetAsync(vcount.p, 0, sizeof(int) * m.nv, st));
      launch(ctx, "vf_fill", k_vf_fill, fblocks, 256, m, (const int*)vstart.as<int>(), vcount.as<int>(),
             vfaces.as<int>(), inv_area.as<double>());
      launch(ctx, "vertex_values", k_vertex_values_mesh, vb, 256, m.nv, (const int*)vstart.as<int>(),
             vfaces.as<int>(), (const double*)inv_area.as<double>(), scale, vval);
    }
    pv = vval;
  }
  dim3 blk(32, 8), grd((cols + 31) / 32, (rows + 7) / 8);
  launch(ctx, "raster_resolve", k_raster_resolve, grd, blk, m, rows, cols, (const FaceRaster*)fr,
         (const int*)owner, pv, img);
  OTM_CUDA(cudaGetLastError());
  if (m.start && mode == OTM_RIO_PER_VERTEX) OTM_CUDA(cudaStreamSynchronize(st));  // temporaries freed on return
}

void raster_grid(otm_context* ctx, int n, const double* xy, const double* density, int rows, int cols, int mode,
                 double* img) {
  MeshRef m{xy, n, n * n, (n + 1) * (n + 1), nullptr, nullptr};
  raster_mesh(ctx, m, density, n * n, rows, cols, mode, img);
}

// Host-side check of an indexed face set (the kernels index with it unchecked).
static void check_faces(int nv, int nf, const int* start, const int* idx) {
  if (start[0] != 0) throw BadArg{"otm_rasterize_mesh: face_start[0] must be 0"};
  for (int f = 0; f < nf; ++f) {
    const int c = start[f + 1] - start[f];
    if (c != 3 && c != 4) throw BadArg{"otm_rasterize_mesh: faces must be triangles or quads"};
  }
  const int total = start[nf];
  for (int k = 0; k < total; ++k)
    if (idx[k] < 0 || idx[k] >= nv) throw BadArg{"otm_rasterize_mesh: vertex index out of range"};
}

}  // namespace otm

extern "C" int otm_rasterize_mode(otm_context* ctx, int n, const double* xy, const double* density, int rows,
                                  int cols, int mode, double* img) {
  return guarded([&] {
    if (!ctx || !xy || !img) throw BadArg{"otm_rasterize: null argument"};
    if (n < 1 || n > 16384 || rows < 1 || cols < 1 || rows > 65536 || cols > 65536)
      throw BadArg{"otm_rasterize: size out of range"};
    if (mode != OTM_RIO_PER_VERTEX && mode != OTM_RIO_PER_FACE) throw BadArg{"otm_rasterize: unknown mode"};
    make_current(ctx);
    cudaStream_t st = ctx->stream;
    const int N = n * n;
    size_t V = (size_t)(n + 1) * (n + 1);
    size_t pix = (size_t)rows * cols;
    DevBuf dxy, dden, dimg;
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
    raster_grid(ctx, n, pxy, pden, rows, cols, mode, pimg);
    if (!idev) OTM_CUDA(cudaMemcpyAsync(img, pimg, sizeof(double) * pix, cudaMemcpyDeviceToHost, st));
    OTM_CUDA(cudaStreamSynchronize(st));
    ctx->prof.flush();
    return (int)OTM_OK;
  });
}

extern "C" int otm_rasterize_faces(otm_context* ctx, int n, const double* xy, int rows, int cols, int* face) {
  return guarded([&] {
    if (!ctx || !xy || !face) throw BadArg{"otm_rasterize_faces: null argument"};
    if (n < 1 || n > 16384 || rows < 1 || cols < 1 || rows > 65536 || cols > 65536)
      throw BadArg{"otm_rasterize_faces: size out of range"};
    make_current(ctx);
    cudaStream_t st = ctx->stream;
    const size_t V2 = 2 * (size_t)(n + 1) * (n + 1), pix = (size_t)rows * cols;
    DevBuf buf;
    buf.reserve(sizeof(double) * (V2 + pix) + 256);
    const double* pxy = xy;
    if (!is_device_ptr(xy)) {
      OTM_CUDA(cudaMemcpyAsync(buf.p, xy, sizeof(double) * V2, cudaMemcpyHostToDevice, st));
      pxy = buf.as<double>();
    }
    double* img = buf.as<double>() + V2;
    raster_grid(ctx, n, pxy, nullptr, rows, cols, OTM_RIO_PER_FACE, img);
    const int N = n * n;
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    const int* owner =
        reinterpret_cast<const int*>(ctx->raster_scratch.as<char>() + al(sizeof(FaceRaster) * (size_t)N));
    OTM_CUDA(cudaMemcpyAsync(face, owner, sizeof(int) * pix, cudaMemcpyDefault, st));
    OTM_CUDA(cudaStreamSynchronize(st));
    ctx->prof.flush();
    return (int)OTM_OK;
  });
}

extern "C" int otm_rasterize(otm_context* ctx, int n, const double* xy, const double* density, int rows, int cols,
                             double* img) {
  return otm_rasterize_mode(ctx, n, xy, density, rows, cols, OTM_RIO_PER_FACE, img);
}

extern "C" int otm_rasterize_mesh(otm_context* ctx, int nv, const double* xy, int nf, const int* face_start,
                                  const int* face_vertices, const double* density, int cells, int rows, int cols,
                                  int mode, double* img) {
  return guarded([&] {
    if (!ctx || !img || nv < 0 || nf < 0 || (nv > 0 && !xy) || (nf > 0 && (!face_start || !face_vertices)))
      throw BadArg{"otm_rasterize_mesh: null argument"};
    if (rows < 1 || cols < 1 || rows > 65536 || cols > 65536) throw BadArg{"otm_rasterize_mesh: size out of range"};
    if (mode != OTM_RIO_PER_VERTEX && mode != OTM_RIO_PER_FACE) throw BadArg{"otm_rasterize_mesh: unknown mode"};
    if (density && cells < nf) throw BadArg{"otm_rasterize_mesh: density shorter than the face count"};
    make_current(ctx);
    cudaStream_t st = ctx->stream;
    // host copies of the topology (from host or device memory), validated before any
    // kernel indexes with it
    auto to_host = [&](int* dst, const int* src, size_t count) {
      if (is_device_ptr(src)) {
        OTM_CUDA(cudaMemcpyAsync(dst, src, sizeof(int) * count, cudaMemcpyDeviceToHost, st));
        OTM_CUDA(cudaStreamSynchronize(st));
      } else {
        std::memcpy(dst, src, sizeof(int) * count);
      }
    };
    std::vector<int> hstart((size_t)nf + 1, 0);
    if (nf > 0) to_host(hstart.data(), face_start, (size_t)nf + 1);
    const int total = nf > 0 ? hstart[nf] : 0;
    if (total < 0 || total > 4 * nf) throw BadArg{"otm_rasterize_mesh: bad face_start"};
    std::vector<int> hidx((size_t)(total > 0 ? total : 1));
    if (total > 0) to_host(hidx.data(), face_vertices, (size_t)total);
    if (nf > 0) check_faces(nv, nf, hstart.data(), hidx.data());
    const size_t pix = (size_t)rows * cols;
    DevBuf dxy, dden, dimg, dstart, didx;
    const double* pxy = xy;
    if (nv > 0 && !is_device_ptr(xy)) {
      dxy.reserve(sizeof(double) * 2 * (size_t)nv);
      OTM_CUDA(cudaMemcpyAsync(dxy.p, xy, sizeof(double) * 2 * (size_t)nv, cudaMemcpyHostToDevice, st));
      pxy = dxy.as<double>();
    }
    const double* pden = density;
    if (density && !is_device_ptr(density)) {
      dden.reserve(sizeof(double) * (size_t)cells);
      OTM_CUDA(cudaMemcpyAsync(dden.p, density, sizeof(double) * (size_t)cells, cudaMemcpyHostToDevice, st));
      pden = dden.as<double>();
    }
    bool idev = is_device_ptr(img);
    double* pimg = img;
    if (!idev) {
      dimg.reserve(sizeof(double) * pix);
      pimg = dimg.as<double>();
    }
    if (nf == 0) {
      OTM_CUDA(cudaMemsetAsync(pimg, 0, sizeof(double) * pix, st));
    } else {
      dstart.reserve(sizeof(int) * ((size_t)nf + 1));
      didx.reserve(sizeof(int) * (size_t)total);
      OTM_CUDA(cudaMemcpyAsync(dstart.p, hstart.data(), sizeof(int) * ((size_t)nf + 1), cudaMemcpyHostToDevice, st));
      OTM_CUDA(cudaMemcpyAsync(didx.p, hidx.data(), sizeof(int) * (size_t)total, cudaMemcpyHostToDevice, st));
      MeshRef m{pxy, 0, nf, nv, dstart.as<int>(), didx.as<int>()};
      raster_mesh(ctx, m, pden, cells, rows, cols, mode, pimg);
    }
    if (!idev) OTM_CUDA(cudaMemcpyAsync(img, pimg, sizeof(double) * pix, cudaMemcpyDeviceToHost, st));
    OTM_CUDA(cudaStreamSynchronize(st));
    ctx->prof.flush();
    return (int)OTM_OK;
  });
}

namespace otm {
static void splat(otm_context* ctx, const MeshRef& m, const int* spf_dev, unsigned long long seed, int rows, int cols,
                  double* img_dev) {
  OTM_CUDA(cudaMemsetAsync(img_dev, 0, sizeof(double) * (size_t)rows * cols, ctx->stream));
  if (m.nf == 0) return;
  const unsigned blocks = (unsigned)(((long)m.nf * 32 + 255) / 256);
  launch(ctx, "splat", k_splat, blocks, 256, m, spf_dev, seed, rows, cols, img_dev);
  OTM_CUDA(cudaGetLastError());
}
}  // namespace otm

extern "C" int otm_sample_image(otm_context* ctx, int nv, const double* xy, int nf, const int* face_start,
                                const int* face_vertices, int grid_n, const int* samples_per_face,
                                unsigned long long seed, int rows, int cols, double* img) {
  return guarded([&] {
    if (!ctx || !img || !samples_per_face || nf < 0 || nv < 0 || (nv > 0 && !xy))
      throw BadArg{"otm_sample_image: null argument"};
    if (rows < 1 || cols < 1 || rows > 65536 || cols > 65536) throw BadArg{"otm_sample_image: size out of range"};
    const bool grid = grid_n > 0;
    if (grid && (grid_n > 16384 || nf != grid_n * grid_n || nv != (grid_n + 1) * (grid_n + 1)))
      throw BadArg{"otm_sample_image: grid_n does not match nv and nf"};
    if (!grid && nf > 0 && (!face_start || !face_vertices)) throw BadArg{"otm_sample_image: null face arrays"};
    make_current(ctx);
    cudaStream_t st = ctx->stream;
    std::vector<int> hstart, hidx;
    if (!grid && nf > 0) {
      auto to_host = [&](std::vector<int>& dst, const int* src, size_t count) {
        dst.resize(count);
        if (is_device_ptr(src)) {
          OTM_CUDA(cudaMemcpyAsync(dst.data(), src, sizeof(int) * count, cudaMemcpyDeviceToHost, st));
          OTM_CUDA(cudaStreamSynchronize(st));
        } else {
          std::memcpy(dst.data(), src, sizeof(int) * count);
        }
      };
      to_host(hstart, face_start, (size_t)nf + 1);
      if (hstart[nf] < 0 || hstart[nf] > 4 * nf) throw BadArg{"otm_sample_image: bad face_start"};
      to_host(hidx, face_vertices, (size_t)(hstart[nf] > 0 ? hstart[nf] : 1));
      check_faces(nv, nf, hstart.data(), hidx.data());
    }
    const size_t pix = (size_t)rows * cols;
    DevBuf dxy, dspf, dimg, dstart, didx;
    const double* pxy = xy;
    if (nv > 0 && !is_device_ptr(xy)) {
      dxy.reserve(sizeof(double) * 2 * (size_t)nv);
      OTM_CUDA(cudaMemcpyAsync(dxy.p, xy, sizeof(double) * 2 * (size_t)nv, cudaMemcpyHostToDevice, st));
      pxy = dxy.as<double>();
    }
    const int* pspf = samples_per_face;
    if (nf > 0 && !is_device_ptr(samples_per_face)) {
      dspf.reserve(sizeof(int) * (size_t)nf);
      OTM_CUDA(cudaMemcpyAsync(dspf.p, samples_per_face, sizeof(int) * (size_t)nf, cudaMemcpyHostToDevice, st));
      pspf = dspf.as<int>();
    }
    const bool idev = is_device_ptr(img);
    double* pimg = img;
    if (!idev) {
      dimg.reserve(sizeof(double) * pix);
      pimg = dimg.as<double>();
    }
    MeshRef m{pxy, grid ? grid_n : 0, nf, nv, nullptr, nullptr};
    if (!grid && nf > 0) {
      dstart.reserve(sizeof(int) * ((size_t)nf + 1));
      didx.reserve(sizeof(int) * hidx.size());
      OTM_CUDA(cudaMemcpyAsync(dstart.p, hstart.data(), sizeof(int) * hstart.size(), cudaMemcpyHostToDevice, st));
      OTM_CUDA(cudaMemcpyAsync(didx.p, hidx.data(), sizeof(int) * hidx.size(), cudaMemcpyHostToDevice, st));
      m.start = dstart.as<int>();
      m.idx = didx.as<int>();
    }
    splat(ctx, m, pspf, seed, rows, cols, pimg);
    if (!idev) OTM_CUDA(cudaMemcpyAsync(img, pimg, sizeof(double) * pix, cudaMemcpyDeviceToHost, st));
    OTM_CUDA(cudaStreamSynchronize(st));
    ctx->prof.flush();
    return (int)OTM_OK;
  });
}
