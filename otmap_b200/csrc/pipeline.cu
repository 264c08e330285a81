// Operations around the solve that the reference's callers use: blending inverse maps
// and rendering the blend (bilinear barycenters, apps/barycenters.cpp:127-139, 250-290)
// and the transport cost of a mesh map (otlib/transport_map.cpp:131-215). Compiled
// without FMA contraction so the per-element arithmetic rounds as the reference's does.

#include <algorithm>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "context.h"

namespace otm {

void dct_reg_attrs(int device);      // dct_reg.cu
void poisson_fft_attrs(int device);  // poisson.cu

// out = sum_k w_k mesh_k, left to right (bilerp / lerp of apps/barycenters.cpp:127-139).
__global__ void k_blend(long V2, int count, const double* const* meshes, const double* w, double* out) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= V2) return;
  double acc = w[0] * meshes[0][t];
  for (int k = 1; k < count; ++k) acc = acc + w[k] * meshes[k][t];
  out[t] = acc;
}

__device__ __forceinline__ double sarea3(double ax, double ay, double bx, double by, double cx, double cy) {
  return 0.5 * ((bx - ax) * (cy - ay) - (by - ay) * (cx - ax));
}

// transport_cost, quad grid mesh: per face the triangle (v3, v0, v1) of its circulation
// (transport_map.cpp:184-199), with partial sums of density*area and of the costs.
__global__ void k_cost_faces(int n, const double* src, const double* dst, const double* density, double* per_face,
                             double* partial) {
  __shared__ double red[64];
  const long N = (long)n * n;
  double v[2] = {0.0, 0.0};
  for (long f = (long)blockIdx.x * blockDim.x + threadIdx.x; f < N; f += (long)gridDim.x * blockDim.x) {
    const int i = (int)(f / n), j = (int)(f % n);
    const long t[3] = {(long)(j + 1) + (long)i * (n + 1), (long)j + (long)i * (n + 1),
                       (long)j + (long)(i + 1) * (n + 1)};
    const double area = sarea3(src[2 * t[0]], src[2 * t[0] + 1], src[2 * t[1]], src[2 * t[1] + 1], src[2 * t[2]],
                               src[2 * t[2] + 1]);
    double dx[3], dy[3];
    for (int k = 0; k < 3; ++k) {
      dx[k] = dst[2 * t[k]] - src[2 * t[k]];
      dy[k] = dst[2 * t[k] + 1] - src[2 * t[k] + 1];
    }
    auto dist2 = [&](double l1, double l2, double l3) {
      double x = l1 * dx[0] + l2 * dx[1] + l3 * dx[2];
      double y = l1 * dy[0] + l2 * dy[1] + l3 * dy[2];
      return x * x + y * y;
    };
    double cost = (dist2(0.5, 0.5, 0) + dist2(0, 0.5, 0.5) + dist2(0.5, 0, 0.5)) / 3.0;
    const double da = density[f] * area;
    cost = da * cost;
    if (per_face) per_face[f] = cost;
    v[0] += da;
    v[1] += cost;
  }
  block_sum<2>(v, red);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = v[0];
    partial[2 * blockIdx.x + 1] = v[1];
  }
}

// integral and total from the partials (fixed order), per_face /= integral.
__global__ void k_cost_finish(long N, int nblocks, const double* partial, double* per_face, double* result) {
  __shared__ double red[64];
  __shared__ double s_int;
  double v[2] = {0.0, 0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    v[0] += partial[2 * b];
    v[1] += partial[2 * b + 1];
  }
  block_sum<2>(v, red);
  if (threadIdx.x == 0) {
    s_int = v[0];
    result[0] = v[1] / v[0];
    result[1] = v[0];
  }
  __syncthreads();
  if (per_face)
    for (long f = threadIdx.x; f < N; f += blockDim.x) per_face[f] /= s_int;
}

// compute_transport_cost (otsolver_2dgrid.cpp:608-640): per face, density * e^2 times
// the mean over the 2x2 Gauss points (z1, z2 = 1/2 +- sqrt(1/3)/2) of the squared
// bilinear interpolation of the corner displacements g; partial sums per block.
__global__ void k_grid_cost(int n, const double* g, const double* density, double e2, double* per_face,
                            double* partial) {
  __shared__ double red[32];
  const long N = (long)n * n;
  const double z1 = sqrt(1. / 3.) / 2. + 0.5, z2 = -sqrt(1. / 3.) / 2. + 0.5;
  double v[1] = {0.0};
  for (long f = (long)blockIdx.x * blockDim.x + threadIdx.x; f < N; f += (long)gridDim.x * blockDim.x) {
    const int i = (int)(f / n), j = (int)(f % n);
    const long c[4] = {(long)j + (long)i * (n + 1), (long)j + (long)(i + 1) * (n + 1),
                       (long)(j + 1) + (long)(i + 1) * (n + 1), (long)(j + 1) + (long)i * (n + 1)};
    auto dist2 = [&](double u, double w) {
      const double a0 = (1 - u) * (1 - w), a1 = u * (1 - w), a2 = u * w, a3 = (1 - u) * w;
      const double x = a0 * g[2 * c[0]] + a1 * g[2 * c[1]] + a2 * g[2 * c[2]] + a3 * g[2 * c[3]];
      const double y = a0 * g[2 * c[0] + 1] + a1 * g[2 * c[1] + 1] + a2 * g[2 * c[2] + 1] + a3 * g[2 * c[3] + 1];
      return x * x + y * y;
    };
    const double cost =
        density[f] * e2 * (dist2(z1, z1) + dist2(z1, z2) + dist2(z2, z2) + dist2(z2, z1)) / 4.;
    if (per_face) per_face[f] = cost;
    v[0] += cost;
  }
  block_sum<1>(v, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = v[0];
}

__global__ void k_sum_partials(int nparts, const double* partial, double* out) {
  __shared__ double red[32];
  double v[1] = {0.0};
  for (int b = threadIdx.x; b < nparts; b += blockDim.x) v[0] += partial[b];
  block_sum<1>(v, red);
  if (threadIdx.x == 0) *out = v[0];
}

// Sum of img in a fixed order: per-block partials over a grid-stride loop.
__global__ void k_img_partials(long count, const double* img, double* partial) {
  __shared__ double red[32];
  double v[1] = {0.0};
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < count; t += (long)gridDim.x * blockDim.x)
    v[0] += img[t];
  block_sum<1>(v, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = v[0];
}

// img *= expected_mean / mean(img) (apps/barycenters.cpp:284); every block forms the
// same total from the partials in the same order.
__global__ void k_img_rescale(long count, int nparts, const double* partial, double expected_mean, double* img,
                              double* mean_out) {
  __shared__ double red[32];
  __shared__ double s_factor;
  double v[1] = {0.0};
  for (int b = threadIdx.x; b < nparts; b += blockDim.x) v[0] += partial[b];
  block_sum<1>(v, red);
  if (threadIdx.x == 0) {
    const double mean = v[0] / (double)count;
    s_factor = expected_mean / mean;
    if (blockIdx.x == 0 && mean_out) *mean_out = mean;
  }
  __syncthreads();
  const double factor = s_factor;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < count; t += (long)gridDim.x * blockDim.x)
    img[t] = img[t] * factor;
}

// Device copies of `count` meshes of V2 doubles: device pointers are used in place,
// host ones are staged into `stage`.
static std::vector<const double*> stage_meshes(otm_context* ctx, const double* const* meshes, int count, size_t V2,
                                               double* stage) {
  std::vector<const double*> ptrs(count);
  for (int k = 0; k < count; ++k) {
    if (!meshes[k]) throw BadArg{"null mesh"};
    if (is_device_ptr(meshes[k])) {
      ptrs[k] = meshes[k];
    } else {
      double* d = stage + V2 * k;
      OTM_CUDA(cudaMemcpyAsync(d, meshes[k], sizeof(double) * V2, cudaMemcpyHostToDevice, ctx->stream));
      ptrs[k] = d;
    }
  }
  return ptrs;
}

}  // namespace otm

using namespace otm;

extern "C" int otm_mesh_blend(otm_context* ctx, int n, int count, const double* const* meshes, const double* weights,
                              double* out) {
  return guarded([&] {
    if (!ctx || !meshes || !weights || !out || count < 1 || count > 64) throw BadArg{"otm_mesh_blend: bad arguments"};
    if (n < 1 || n > 16384) throw BadArg{"otm_mesh_blend: grid size out of range"};
    make_current(ctx);
    cudaStream_t st = ctx->stream;
    const size_t V2 = 2 * (size_t)(n + 1) * (n + 1);
    DevBuf buf;
    buf.reserve(sizeof(double) * (V2 * (count + 1) + count + 8) + sizeof(double*) * count);
    double* base = buf.as<double>();
    std::vector<const double*> ptrs = stage_meshes(ctx, meshes, count, V2, base);
    double* d_out = base + V2 * count;
    double* d_w = d_out + V2;
    const double** d_ptrs = reinterpret_cast<const double**>(d_w + count + (count & 1));
    OTM_CUDA(cudaMemcpyAsync(d_w, weights, sizeof(double) * count, cudaMemcpyHostToDevice, st));
    OTM_CUDA(cudaMemcpyAsync(d_ptrs, ptrs.data(), sizeof(double*) * count, cudaMemcpyHostToDevice, st));
    const bool odev = is_device_ptr(out);
    double* dst = odev ? out : d_out;
    launch(ctx, "blend", k_blend, (unsigned)((V2 + 255) / 256), 256, (long)V2, count, (const double* const*)d_ptrs,
           (const double*)d_w, dst);
    OTM_CUDA(cudaGetLastError());
    if (!odev) OTM_CUDA(cudaMemcpyAsync(out, dst, sizeof(double) * V2, cudaMemcpyDeviceToHost, st));
    OTM_CUDA(cudaStreamSynchronize(st));
    ctx->prof.flush();
    return (int)OTM_OK;
  });
}

extern "C" int otm_transport_cost(otm_context* ctx, int n, const double* src_xy, const double* dst_xy,
                                  const double* density, double* per_face, double* cost) {
  return guarded([&] {
    if (!ctx || !src_xy || !dst_xy || !density || !cost) throw BadArg{"otm_transport_cost: null argument"};
    if (n < 1 || n > 16384) throw BadArg{"otm_transport_cost: grid size out of range"};
    make_current(ctx);
    cudaStream_t st = ctx->stream;
    const size_t V2 = 2 * (size_t)(n + 1) * (n + 1), N = (size_t)n * n;
    const int nb = 512;
    DevBuf buf;
    buf.reserve(sizeof(double) * (2 * V2 + 2 * N + 2 * nb + 8));
    double* p = buf.as<double>();
    auto in = [&](const double* src, double* tmp, size_t words) -> const double* {
      if (is_device_ptr(src)) return src;
      OTM_CUDA(cudaMemcpyAsync(tmp, src, sizeof(double) * words, cudaMemcpyHostToDevice, st));
      return tmp;
    };
    const double* d_src = in(src_xy, p, V2);
    const double* d_dst = in(dst_xy, p + V2, V2);
    const double* d_den = in(density, p + 2 * V2, N);
    double* d_pf = per_face ? (is_device_ptr(per_face) ? per_face : p + 2 * V2 + N) : nullptr;
    double* d_part = p + 2 * V2 + 2 * N;
    double* d_res = d_part + 2 * nb;
    launch(ctx, "cost_faces", k_cost_faces, nb, 256, n, d_src, d_dst, d_den, d_pf, d_part);
    launch(ctx, "cost_finish", k_cost_finish, 1, 1024, (long)N, nb, (const double*)d_part, d_pf, d_res);
    OTM_CUDA(cudaGetLastError());
    double res[2];
    OTM_CUDA(cudaMemcpyAsync(res, d_res, sizeof(res), cudaMemcpyDeviceToHost, st));
    if (per_face && !is_device_ptr(per_face))
      OTM_CUDA(cudaMemcpyAsync(per_face, d_pf, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
    OTM_CUDA(cudaStreamSynchronize(st));
    ctx->prof.flush();
    *cost = res[0];
    return (int)OTM_OK;
  });
}

extern "C" int otm_barycenter(otm_context* ctx, int n, int count, const double* const* inv_meshes,
                              const double* weights, double expected_mean, int rows, int cols, double* mesh_out,
                              double* img, double* raster_mean) {
  return guarded([&] {
    if (!ctx || !inv_meshes || !weights || !img || count < 1 || count > 64)
      throw BadArg{"otm_barycenter: bad arguments"};
    if (n < 1 || n > 16384 || rows < 1 || cols < 1 || rows > 65536 || cols > 65536)
      throw BadArg{"otm_barycenter: size out of range"};
    make_current(ctx);
    cudaStream_t st = ctx->stream;
    const size_t V2 = 2 * (size_t)(n + 1) * (n + 1), pix = (size_t)rows * cols;
    const int nparts = 512;
    DevBuf buf;
    buf.reserve(sizeof(double) * (V2 * (count + 1) + count + pix + nparts + 16) + sizeof(double*) * count);
    double* base = buf.as<double>();
    std::vector<const double*> ptrs = stage_meshes(ctx, inv_meshes, count, V2, base);
    double* d_mesh = base + V2 * count;
    double* d_w = d_mesh + V2;
    double* d_img = d_w + count + (count & 1);
    double* d_part = d_img + pix;
    double* d_mean = d_part + nparts;
    const double** d_ptrs = reinterpret_cast<const double**>(d_mean + 8);
    OTM_CUDA(cudaMemcpyAsync(d_w, weights, sizeof(double) * count, cudaMemcpyHostToDevice, st));
    OTM_CUDA(cudaMemcpyAsync(d_ptrs, ptrs.data(), sizeof(double*) * count, cudaMemcpyHostToDevice, st));
    const bool mdev = mesh_out && is_device_ptr(mesh_out);
    double* pm = mdev ? mesh_out : d_mesh;
    launch(ctx, "blend", k_blend, (unsigned)((V2 + 255) / 256), 256, (long)V2, count, (const double* const*)d_ptrs,
           (const double*)d_w, pm);
    const bool idev = is_device_ptr(img);
    double* pi = idev ? img : d_img;
    raster_grid(ctx, n, pm, nullptr, rows, cols, OTM_RIO_PER_FACE, pi);
    launch(ctx, "img_partials", k_img_partials, nparts, 256, (long)pix, (const double*)pi, d_part);
    const unsigned sb = (unsigned)std::min<size_t>((pix + 255) / 256, (size_t)4 * ctx->num_sms);
    launch(ctx, "img_rescale", k_img_rescale, sb, 256, (long)pix, nparts, (const double*)d_part, expected_mean, pi,
           d_mean);
    OTM_CUDA(cudaGetLastError());
    if (mesh_out && !mdev) OTM_CUDA(cudaMemcpyAsync(mesh_out, pm, sizeof(double) * V2, cudaMemcpyDeviceToHost, st));
    if (!idev) OTM_CUDA(cudaMemcpyAsync(img, pi, sizeof(double) * pix, cudaMemcpyDeviceToHost, st));
    double mean = 0;
    OTM_CUDA(cudaMemcpyAsync(&mean, d_mean, sizeof(double), cudaMemcpyDeviceToHost, st));
    OTM_CUDA(cudaStreamSynchronize(st));
    ctx->prof.flush();
    if (raster_mean) *raster_mean = mean;
    return (int)OTM_OK;
  });
}

extern "C" int otm_grid_transport_cost(otm_context* ctx, int n, const double* grads_xy, const double* density,
                                       double* per_face, double* total) {
  return guarded([&] {
    if (!ctx || !grads_xy || !density || !total) throw BadArg{"otm_grid_transport_cost: null argument"};
    if (n < 1 || n > 16384) throw BadArg{"otm_grid_transport_cost: grid size out of range"};
    make_current(ctx);
    cudaStream_t st = ctx->stream;
    const size_t V2 = 2 * (size_t)(n + 1) * (n + 1), N = (size_t)n * n;
    const int nb = 512;
    DevBuf buf;
    buf.reserve(sizeof(double) * (V2 + 2 * N + nb + 8));
    double* p = buf.as<double>();
    const double* d_g = grads_xy;
    if (!is_device_ptr(grads_xy)) {
      OTM_CUDA(cudaMemcpyAsync(p, grads_xy, sizeof(double) * V2, cudaMemcpyHostToDevice, st));
      d_g = p;
    }
    const double* d_den = density;
    if (!is_device_ptr(density)) {
      OTM_CUDA(cudaMemcpyAsync(p + V2, density, sizeof(double) * N, cudaMemcpyHostToDevice, st));
      d_den = p + V2;
    }
    double* d_pf = per_face ? (is_device_ptr(per_face) ? per_face : p + V2 + N) : nullptr;
    double* d_part = p + V2 + 2 * N;
    double* d_res = d_part + nb;
    const double e2 = 1.0 / (double(n) * double(n));  // otsolver_2dgrid.cpp:97
    launch(ctx, "grid_cost", k_grid_cost, nb, 256, n, d_g, d_den, e2, d_pf, d_part);
    launch(ctx, "sum_partials", k_sum_partials, 1, 512, nb, (const double*)d_part, d_res);
    OTM_CUDA(cudaGetLastError());
    double res = 0;
    OTM_CUDA(cudaMemcpyAsync(&res, d_res, sizeof(double), cudaMemcpyDeviceToHost, st));
    if (per_face && !is_device_ptr(per_face))
      OTM_CUDA(cudaMemcpyAsync(per_face, d_pf, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
    OTM_CUDA(cudaStreamSynchronize(st));
    ctx->prof.flush();
    *total = res;
    return (int)OTM_OK;
  });
}

// ---- differentiable barycenter image (apps/barycenters.cpp:184-198, 250-290) ----

namespace otm {

// The origin grid vertices, vertex v = j + i (n+1) at (i * (1/n), j * (1/n))
// (utils/mesh_utils.cpp:100-108).
__global__ void k_origin_grid(int n, double* xy) {
  const long v = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long V = (long)(n + 1) * (n + 1);
  if (v >= V) return;
  const double dx = 1.0 / (double)n;
  xy[2 * v] = (double)(v / (n + 1)) * dx;
  xy[2 * v + 1] = (double)(v % (n + 1)) * dx;
}

// Per-block partial sums of (img - t)^2 and of g R (g = 2 (img - t), R = img / s the
// raster before rescaling), and g itself.
__global__ void k_bary_loss(long count, const double* img, const double* target, double inv_s, double* g,
                            double* partial) {
  __shared__ double red[64];
  double v[2] = {0.0, 0.0};
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < count; t += (long)gridDim.x * blockDim.x) {
    const double d = img[t] - target[t];
    const double gt = 2.0 * d;
    g[t] = gt;
    v[0] += d * d;
    v[1] += gt * (img[t] * inv_s);
  }
  block_sum<2>(v, red);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = v[0];
    partial[2 * blockIdx.x + 1] = v[1];
  }
}

__global__ void k_sum_partials2(int nparts, const double* partial, double* out) {
  __shared__ double red[64];
  double v[2] = {0.0, 0.0};
  for (int b = threadIdx.x; b < nparts; b += blockDim.x) {
    v[0] += partial[2 * b];
    v[1] += partial[2 * b + 1];
  }
  block_sum<2>(v, red);
  if (threadIdx.x == 0) {
    out[0] = v[0];
    out[1] = v[1];
  }
}

// dL/dR = s (g - c2) in place of g.
__global__ void k_bary_dR(long count, double s, double c2, double* g) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < count) g[t] = s * (g[t] - c2);
}

__global__ void k_scale(long count, double a, const double* x, double* y) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < count) y[t] = a * x[t];
}

__global__ void k_add_const(long count, double c, double* y) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < count) y[t] = y[t] + c;
}

}  // namespace otm

extern "C" int otm_barycenter_loss(otm_context* ctx, int n, int count, const double* const* density,
                                   const double* weights, int res, const double* target,
                                   const otm_solver_options* opt, const otm_adjoint_options* aopt, double* image,
                                   double* loss, double* const* grad_density, otm_barycenter_stats* stats) {
  return guarded([&] {
    if (!ctx || !density || !weights || !target || count < 1 || count > 8)
      throw BadArg{"otm_barycenter_loss: bad arguments"};
    if (n < 1 || n > 16384 || res < 1 || res > 65536) throw BadArg{"otm_barycenter_loss: size out of range"};
    for (int k = 0; k < count; ++k)
      if (!density[k] || (grad_density && !grad_density[k])) throw BadArg{"otm_barycenter_loss: null buffer"};
    make_current(ctx);
    cudaStream_t st = ctx->stream;
    const size_t N = (size_t)n * n, V = (size_t)(n + 1) * (n + 1), V2 = 2 * V, pix = (size_t)res * res;
    const int nparts = 512;
    auto al = [](size_t w) { return (w + 31) / 32 * 32; };  // in doubles
    // device layout: per map raw density, adjusted density, gradient, forward mesh, inverse
    // mesh (later dL/dI), dL/dF, first hits; then the blend, its gradient, image, target,
    // g, partials, scalars, blend pointers and weights
    const size_t per = al(N) * 3 + al(V2) * 3 + al((V + 1) / 2);
    DevBuf buf;
    buf.reserve(sizeof(double) * (per * count + al(V2) * 2 + al(pix) * 3 + al(2 * nparts) + al(64) + al(8) * 2));
    double* p = buf.as<double>();
    auto take = [&](size_t w) {
      double* r = p;
      p += al(w);
      return r;
    };
    std::vector<double*> rho(count), adj(count), fwd(count), inv(count), dF(count), grad(count);
    std::vector<int*> hit0(count);
    for (int k = 0; k < count; ++k) {
      rho[k] = take(N);
      adj[k] = take(N);
      grad[k] = take(N);
      fwd[k] = take(V2);
      inv[k] = take(V2);
      dF[k] = take(V2);
      hit0[k] = reinterpret_cast<int*>(take((V + 1) / 2));
    }
    double* blend = take(V2);
    double* dB = take(V2);
    double* img = take(pix);
    double* tgt = take(pix);
    double* g = take(pix);
    double* part = take(2 * nparts);
    double* scal = take(64);  // reduction results and the missing counter
    const double** d_ptrs = reinterpret_cast<const double**>(take(8));
    double* d_w = take(8);

    // inputs and the expected mean sum_k w_k mean(density_k) (barycenters.cpp:193, 283)
    for (int k = 0; k < count; ++k) copy_in(ctx, rho[k], density[k], sizeof(double) * N);
    copy_in(ctx, tgt, target, sizeof(double) * pix);
    for (int k = 0; k < count; ++k) {
      launch(ctx, "img_partials", k_img_partials, nparts, 256, (long)N, (const double*)rho[k], part);
      launch(ctx, "sum_partials", k_sum_partials, 1, 256, nparts, (const double*)part, scal + k);
    }
    std::vector<double> hs(count);
    OTM_CUDA(cudaMemcpyAsync(hs.data(), scal, sizeof(double) * count, cudaMemcpyDeviceToHost, st));
    OTM_CUDA(cudaStreamSynchronize(st));
    double expected = 0.0;
    for (int k = 0; k < count; ++k) {
      const double mean = hs[k] / (double)N;
      expected = k == 0 ? weights[0] * mean : expected + weights[k] * mean;
    }

    // forward maps (one batch), inverse meshes of the origin grid
    std::vector<int> ns(count, n);
    std::vector<const double*> rin(rho.begin(), rho.end());
    std::vector<otm_solve_stats> sst(count);
    int rc = otm_solve_batch(ctx, count, ns.data(), rin.data(), opt, fwd.data(), adj.data(), sst.data());
    if (rc != OTM_OK) return rc;
    unsigned long long* d_missing = reinterpret_cast<unsigned long long*>(scal + 16);
    OTM_CUDA(cudaMemsetAsync(d_missing, 0, sizeof(unsigned long long), st));
    const unsigned gv = (unsigned)((V + 255) / 256), gv2 = (unsigned)((V2 + 255) / 256);
    for (int k = 0; k < count; ++k) {
      otm_map* m = nullptr;
      rc = otm_map_create(ctx, n, fwd[k], adj[k], &m);
      if (rc != OTM_OK) return rc;
      try {
        launch(ctx, "origin_grid", k_origin_grid, gv, 256, n, inv[k]);
        map_inverse_dev(m, inv[k], (long)V, OTM_INV_DENSEST, nullptr, hit0[k], nullptr, d_missing);
        OTM_CUDA(cudaStreamSynchronize(st));
      } catch (...) {
        otm_map_destroy(m);
        throw;
      }
      otm_map_destroy(m);
    }

    // blend, raster, rescale, loss
    OTM_CUDA(cudaMemcpyAsync(d_w, weights, sizeof(double) * count, cudaMemcpyHostToDevice, st));
    OTM_CUDA(cudaMemcpyAsync(d_ptrs, inv.data(), sizeof(double*) * count, cudaMemcpyHostToDevice, st));
    launch(ctx, "blend", k_blend, gv2, 256, (long)V2, count, (const double* const*)d_ptrs, (const double*)d_w,
           blend);
    raster_grid(ctx, n, blend, nullptr, res, res, OTM_RIO_PER_FACE, img);
    launch(ctx, "img_partials", k_img_partials, nparts, 256, (long)pix, (const double*)img, part);
    const unsigned sb = (unsigned)std::min<size_t>((pix + 255) / 256, (size_t)4 * ctx->num_sms);
    launch(ctx, "img_rescale", k_img_rescale, sb, 256, (long)pix, nparts, (const double*)part, expected, img,
           scal + 8);
    double rmean = 0.0;
    OTM_CUDA(cudaMemcpyAsync(&rmean, scal + 8, sizeof(double), cudaMemcpyDeviceToHost, st));
    OTM_CUDA(cudaStreamSynchronize(st));
    const double s = expected / rmean;  // image = s R
    launch(ctx, "bary_loss", k_bary_loss, nparts, 256, (long)pix, (const double*)img, (const double*)tgt, 1.0 / s, g,
           part);
    launch(ctx, "sum_partials2", k_sum_partials2, 1, 256, nparts, (const double*)part, scal + 10);
    double red2[2];
    unsigned long long miss = 0;
    OTM_CUDA(cudaMemcpyAsync(red2, scal + 10, sizeof(red2), cudaMemcpyDeviceToHost, st));
    OTM_CUDA(cudaMemcpyAsync(&miss, d_missing, sizeof(miss), cudaMemcpyDeviceToHost, st));
    OTM_CUDA(cudaStreamSynchronize(st));
    const double L = red2[0], sgR = red2[1];
    std::vector<int> solves(count, 0);
    std::vector<double> ares(count, 0.0);

    if (grad_density) {
      // dL/dR = s (g - sum(g R) / sum(R)); dL/dexpected = sum(g R) / mean(R)
      const double sumR = rmean * (double)pix;
      const double c2 = sgR / sumR, dL_dexp = sgR / rmean;
      const unsigned gp = (unsigned)((pix + 255) / 256);
      launch(ctx, "bary_dR", k_bary_dR, gp, 256, (long)pix, s, c2, g);
      raster_grid_backward(ctx, n, blend, res, res, g, dB);
      otm_adjoint_options ao;
      otm_default_adjoint_options(&ao);
      if (aopt) ao = *aopt;
      for (int k = 0; k < count; ++k) {
        double* dI = inv[k];  // the inverse mesh is no longer needed: its buffer holds dL/dI
        launch(ctx, "scale", k_scale, gv2, 256, (long)V2, weights[k], (const double*)dB, dI);
        inverse_grid_backward(ctx, n, fwd[k], hit0[k], dI, dF[k]);
      }
      // the maps' adjoints are independent: each runs on its own context (this one for map
      // 0, cached helpers of the same device for the others) from its own host thread, so
      // their kernels -- a 512^2 Poisson solve fills a fraction of the GPU -- overlap
      OTM_CUDA(cudaStreamSynchronize(st));
      dct_reg_attrs(ctx->device);  // device-wide set-up done once, before the threads
      poisson_fft_attrs(ctx->device);
      while ((int)ctx->helpers.size() < count - 1) {
        otm_context* h = nullptr;
        const int hrc = otm_create(ctx->device, &h);
        if (hrc != OTM_OK) return hrc;
        ctx->helpers.push_back(h);
      }
      std::vector<int> rcs(count, OTM_OK);
      std::vector<otm_adjoint_stats> asts(count);
      std::vector<std::string> errs(count);
      std::vector<long> launches0(count, 0);
      auto run = [&](int k) {
        otm_context* c = k == 0 ? ctx : ctx->helpers[k - 1];
        if (k > 0) {
          c->poisson_mode = ctx->poisson_mode;
          c->loop_mode = ctx->loop_mode;
          c->wait_test = ctx->wait_test;
          launches0[k] = c->launches;
        }
        rcs[k] = otm_adjoint(c, n, rho[k], fwd[k], dF[k], &ao, grad[k], &asts[k]);
        if (rcs[k] != OTM_OK) errs[k] = otm_last_error();
      };
      {
        std::vector<std::thread> threads;
        try {
          for (int k = 1; k < count; ++k) threads.emplace_back(run, k);
        } catch (...) {  // a thread could not start: join those that did, then report
          for (auto& t : threads) t.join();
          throw;
        }
        run(0);
        for (auto& t : threads) t.join();
      }
      make_current(ctx);
      for (int k = 0; k < count; ++k)
        if (rcs[k] != OTM_OK) {
          set_error(errs[k]);
          return rcs[k];
        }
      for (int k = 0; k < count; ++k) {
        if (k > 0) ctx->launches += ctx->helpers[k - 1]->launches - launches0[k];
        solves[k] = asts[k].iterations;
        ares[k] = asts[k].relative_residual;
        // expected = ... + w_k mean(density_k): d/ddensity_k = w_k / N per cell
        launch(ctx, "add_const", k_add_const, (unsigned)((N + 255) / 256), 256, (long)N,
               weights[k] * dL_dexp / (double)N, grad[k]);
        copy_out(ctx, grad_density[k], grad[k], sizeof(double) * N);
      }
    }
    if (image) copy_out(ctx, image, img, sizeof(double) * pix);
    OTM_CUDA(cudaGetLastError());
    OTM_CUDA(cudaStreamSynchronize(st));
    ctx->prof.flush();
    if (loss) *loss = L;
    if (stats) {
      std::memset(stats, 0, sizeof(*stats));
      for (int k = 0; k < count; ++k) {
        stats->iterations[k] = sst[k].iterations;
        stats->outcome[k] = sst[k].outcome;
        stats->residual[k] = sst[k].residual;
        stats->adjoint_solves[k] = solves[k];
        stats->adjoint_residual[k] = ares[k];
      }
      stats->inverse_missing = (long)miss;
      stats->expected_mean = expected;
      stats->raster_mean = rmean;
    }
    return (int)OTM_OK;
  });
}
