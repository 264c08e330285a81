// The grid transport solver on the GPU: GridBasedTransportSolver::init/solve of the
// reference (otlib/otsolver_2dgrid.cpp) as CUDA kernels for sm_100a.
//
// One engine serves single and batched solves: every kernel walks a flat list of
// (instance, tile) work items, reads its instance's state from a device record
// (Inst) and returns at once when that instance has stopped, so instances of
// different sizes converge independently inside the same launches.
//
// Per iteration (otsolver_2dgrid.cpp:160-220), for every active instance:
//   d_hat = M^+ r_k    the cosine-transform Poisson solve (:175-179): register FFT
//                      transforms (dct_reg.cu) for power-of-two n in 64..1024, shared-
//                      memory FFTs (poisson.cu) for other powers of two, dense products
//                      with the cosine basis (k_dct_gemm here) for any other n
//   k_sweep_sums       |d_hat| (early exit, :182), beta (:248-261) and the quartic of the
//                      line search; its last block solves the cubic (:541-595)
//   k_sweep_update     d = d_hat + beta d_prev, psi += alpha d, r += alpha b + alpha^2 a
//                      (:599-605); its last block advances the iteration and tests the
//                      loop condition (:160)
// (stencil.cu). By default the iteration is the body of a device-side WHILE loop in one
// CUDA graph launch. Set-up (density normalisation, initial residual) and the forward
// mesh are tile kernels below. k_beta / k_coeffs / k_update are the earlier one-tile-per-
// block form of the two sweeps, kept for the allocation-free solve at the end of this
// file. Every reduction is fixed-order (per-block partials, reduced in block order by the
// last block of the instance), so results are run-to-run identical. All arithmetic is
// FP64, compiled without FMA contraction so each cell's operations round as the
// reference's scalar code does.

#include <cfloat>
#include <cmath>
#include <algorithm>
#include <chrono>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <random>
#include <vector>

#include "engine.cuh"

namespace otm {

__device__ __forceinline__ int clampi(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }

// s[(HI) x (HJ)] <- f(cell) over cells (i0-1 .. i0+TI) x (j0-1 .. j0+TJ), indices
// clamped to the grid. With clamped indices the interior vertex-gradient formula
// reproduces the reference's boundary rules exactly (otsolver_2dgrid.cpp:405-422):
// tangential one-sided differences, zero normal component, zero at the corners.
template <class F>
__device__ __forceinline__ void load_halo(double* s, int n, int i0, int j0, F f) {
  for (int idx = threadIdx.x; idx < HI * HJ; idx += NT) {
    int li = idx / HJ, lj = idx - li * HJ;
    int gi = clampi(i0 + li - 1, n), gj = clampi(j0 + lj - 1, n);
    s[idx] = f((size_t)gi * n + gj);
  }
}

// Vertex gradients (otsolver_2dgrid.cpp:379-391): vertex (i0+vi, j0+vj) from the
// four cells around it, 0.5 n ((p10 + p11) - (p00 + p01)) and 0.5 n ((p01 + p11) - (p00 + p10)).
__device__ __forceinline__ void vertex_grads(const double* s, double* gx, double* gy, double hw) {
  for (int idx = threadIdx.x; idx < VI * VJ; idx += NT) {
    int vi = idx / VJ, vj = idx - vi * VJ;
    double p00 = s[vi * HJ + vj], p01 = s[vi * HJ + vj + 1];
    double p10 = s[(vi + 1) * HJ + vj], p11 = s[(vi + 1) * HJ + vj + 1];
    gx[idx] = hw * ((p10 + p11) - (p00 + p01));
    gy[idx] = hw * ((p01 + p11) - (p00 + p10));
  }
}

// Quad area from its corner displacements (otsolver_2dgrid.cpp:425-447).
__device__ __forceinline__ double cell_area(const double* gx, const double* gy, int ci, int cj, double e) {
  int v00 = ci * VJ + cj, v10 = (ci + 1) * VJ + cj, v01 = ci * VJ + cj + 1, v11 = (ci + 1) * VJ + cj + 1;
  return 0.5 * ((gx[v11] - gx[v00] + e) * (gy[v01] - gy[v10] + e) -
                (gy[v11] - gy[v00] + e) * (gx[v01] - gx[v10] - e));
}

// r(psi + t dir) = r(psi) + b t + a t^2 (otsolver_2dgrid.cpp:516-537): g = gradients at
// psi, h = gradients of dir.
__device__ __forceinline__ void cell_ab(const double* gx, const double* gy, const double* hx, const double* hy,
                                        int ci, int cj, double e, double& a, double& b) {
  int v00 = ci * VJ + cj, v10 = (ci + 1) * VJ + cj, v01 = ci * VJ + cj + 1, v11 = (ci + 1) * VJ + cj + 1;
  double diag0a_x = gx[v11] - gx[v00] + e;
  double diag0a_y = gy[v11] - gy[v00] + e;
  double diag0b_x = gx[v01] - gx[v10] - e;
  double diag0b_y = gy[v01] - gy[v10] + e;
  double dda_x = hx[v11] - hx[v00];
  double dda_y = hy[v11] - hy[v00];
  double ddb_x = hx[v01] - hx[v10];
  double ddb_y = hy[v01] - hy[v10];
  a = 0.5 * (dda_x * ddb_y - dda_y * ddb_x);
  b = 0.5 * (dda_x * diag0b_y - dda_y * diag0b_x + diag0a_x * ddb_y - diag0a_y * ddb_x);
}

struct TileCoord {
  int i0, j0, ci, cj, gi, gj;
  bool inside;
  size_t f;
};

__device__ __forceinline__ TileCoord tile_coord(const Inst& I, int block) {
  TileCoord t;
  int n = I.n, tl = block - I.tile0, tjn = (n + TJ - 1) / TJ;
  t.i0 = (tl / tjn) * TI;
  t.j0 = (tl % tjn) * TJ;
  t.ci = threadIdx.x / TJ;
  t.cj = threadIdx.x % TJ;
  t.gi = t.i0 + t.ci;
  t.gj = t.j0 + t.cj;
  t.inside = t.gi < n && t.gj < n;
  t.f = (size_t)t.gi * n + t.gj;
  return t;
}

// Sums partials[tile0 .. tile0+ntiles) (K values each) in tile order.
template <int K>
__device__ __forceinline__ void reduce_partials(const double* partials, int tile0, int ntiles, double (&v)[K],
                                                double* red) {
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = 0.0;
  for (int t = threadIdx.x; t < ntiles; t += NT)
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] += __ldcg(&partials[(size_t)(tile0 + t) * KP + k]);
  block_sum<K>(v, red);
}

__device__ __forceinline__ double reduce_partials_max(const double* partials, int tile0, int ntiles, int k,
                                                      double* red) {
  double m = -INFINITY;
  for (int t = threadIdx.x; t < ntiles; t += NT) m = fmax(m, __ldcg(&partials[(size_t)(tile0 + t) * KP + k]));
  return block_max(m, red);
}

__device__ __forceinline__ double reduce_partials_min(const double* partials, int tile0, int ntiles, int k,
                                                      double* red) {
  double m = INFINITY;
  for (int t = threadIdx.x; t < ntiles; t += NT) m = fmin(m, __ldcg(&partials[(size_t)(tile0 + t) * KP + k]));
  return -block_max(-m, red);
}

__device__ __forceinline__ double elem_area(int n) { return 1.0 / ((double)n * (double)n); }

// ---------------------------------------------------------------------------
// Density normalisation (otsolver_2dgrid.cpp:47-63), three passes.

__global__ __launch_bounds__(NT) void k_density_sum(Inst* insts, const int* tile_inst, double* partials) {
  __shared__ double red[32 * 2];
  Inst& I = insts[tile_inst[blockIdx.x]];
  TileCoord t = tile_coord(I, blockIdx.x);
  double v[1] = {t.inside ? I.rho[t.f] : 0.0};
  block_sum<1>(v, red);
  if (threadIdx.x == 0) partials[(size_t)blockIdx.x * KP] = v[0];
  if (last_block(&I.counter, I.ntiles)) {
    double s[1];
    reduce_partials<1>(partials, I.tile0, I.ntiles, s, red);
    if (threadIdx.x == 0) I.dens_scale = s[0] * elem_area(I.n);
  }
}

__global__ __launch_bounds__(NT) void k_density_scale(Inst* insts, const int* tile_inst, double* partials) {
  __shared__ double red[32 * 2];
  Inst& I = insts[tile_inst[blockIdx.x]];
  TileCoord t = tile_coord(I, blockIdx.x);
  double mn = INFINITY, mx = -INFINITY;
  if (t.inside) {
    double x = I.rho[t.f] / I.dens_scale;
    I.rho[t.f] = x;
    mn = x;
    mx = x;
  }
  mx = block_max(mx, red);
  mn = -block_max(-mn, red);
  if (threadIdx.x == 0) {
    partials[(size_t)blockIdx.x * KP + 0] = mn;
    partials[(size_t)blockIdx.x * KP + 1] = mx;
  }
  if (last_block(&I.counter, I.ntiles)) {
    double gmn = reduce_partials_min(partials, I.tile0, I.ntiles, 0, red);
    double gmx = reduce_partials_max(partials, I.tile0, I.ntiles, 1, red);
    if (threadIdx.x == 0) {
      double ratio = std_min(I.max_ratio, gmx / gmn);
      I.dens_beta = std_max(0.0, (ratio * gmn - gmx) / (1.0 - ratio));
    }
  }
}

__global__ __launch_bounds__(NT) void k_density_apply(Inst* insts, const int* tile_inst) {
  Inst& I = insts[tile_inst[blockIdx.x]];
  TileCoord t = tile_coord(I, blockIdx.x);
  if (t.inside) I.rho[t.f] = (I.rho[t.f] + I.dens_beta) / (1.0 + I.dens_beta);
}

// ---------------------------------------------------------------------------
// Initial residual at psi = 0 (otsolver_2dgrid.cpp:146).

// At psi = 0 every vertex gradient is zero and the quad-area formula (cell_area) reduces
// exactly to 0.5 * (e*e - e*(-e)) = e*e, so the kernel streams rho without the stencil.
__global__ __launch_bounds__(NT) void k_residual_init(Inst* insts, const int* tile_inst, double* partials) {
  __shared__ double red[32 * 2];
  Inst& I = insts[tile_inst[blockIdx.x]];
  const int n = I.n;
  const double e = 1.0 / (double)n, ea = elem_area(n);
  TileCoord t = tile_coord(I, blockIdx.x);
  double v[1] = {0.0};
  double mx = -INFINITY;
  if (t.inside) {
    double r = e * e - ea * I.rho[t.f];
    if (I.split) {
      // FP32 residual: the sums below start from the stored (rounded) values
      const float rf = (float)r;
      reinterpret_cast<float*>(I.r[0])[t.f] = rf;
      r = rf;
    } else {
      I.r[0][t.f] = r;
    }
    v[0] = r * r;
    mx = r;
  }
  block_sum<1>(v, red);
  mx = block_max(mx, red);
  if (threadIdx.x == 0) {
    partials[(size_t)blockIdx.x * KP + 0] = v[0];
    partials[(size_t)blockIdx.x * KP + 1] = mx;
  }
  if (last_block(&I.counter, I.ntiles)) {
    double sum[1];
    reduce_partials<1>(partials, I.tile0, I.ntiles, sum, red);
    double gmx = reduce_partials_max(partials, I.tile0, I.ntiles, 1, red);
    if (threadIdx.x == 0) {
      I.residual = sum[0] / ea;
      I.residual0 = I.residual;
      I.linf = gmx / ea;
      I.it = 0;
      I.alpha = 0.0;
      I.beta = 0.0;
      I.use_beta = 0;
      I.active = (0 < I.max_iter && I.residual > I.threshold) ? 1 : 0;
      if (!I.active) stop_outcome(I);
    }
  }
}

// ---------------------------------------------------------------------------
// Poisson solve as dense products with the cosine basis C (n x n, C[k][i]):
//   t1 = C r ; t2 = (t1 C^T) / lambda ; t1 = C^T t2 ; d_hat = t1 C
// lambda_kl = 2 - 2 cos(pi k/n) cos(pi l/n) are the eigenvalues of the reference's
// assembled matrix (otsolver_2dgrid.cpp:284-311); dropping the (0,0) mode is the
// mean-zero projection of :179. epi = 2 multiplies by lambda instead (the
// diagonalisation check at init).

__global__ __launch_bounds__(256) void k_dct_gemm(const Inst* insts, const int* gemm_inst, int stage, int epi) {
  const Inst& I = insts[gemm_inst[blockIdx.x]];
  if (!I.active) return;
  const int n = I.n;
  const int tl = blockIdx.x - I.gemm0, tn = (n + GB - 1) / GB;
  const int m0 = (tl / tn) * GB, n0 = (tl % tn) * GB;
  const double *A, *B;
  double* D;
  bool ta, tb;
  int ep = 0;
  switch (stage) {
    case 0: A = I.C; ta = false; B = I.r[I.it % 3]; tb = false; D = I.t1; break;
    case 1: A = I.t1; ta = false; B = I.C; tb = true; D = I.t2; ep = epi; break;
    case 2: A = I.C; ta = true; B = I.t2; tb = false; D = I.t1; break;
    default: A = I.t1; ta = false; B = I.C; tb = false; D = I.dhat; break;
  }
  __shared__ double As[GK][GB + 1];
  __shared__ double Bs[GK][GB + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  for (int k0 = 0; k0 < n; k0 += GK) {
    for (int e = threadIdx.x; e < GB * GK; e += 256) {
      int mm, kk;
      if (!ta) {
        mm = e / GK;
        kk = e - mm * GK;
      } else {
        kk = e / GB;
        mm = e - kk * GB;
      }
      int gm = m0 + mm, gk = k0 + kk;
      double v = 0.0;
      if (gm < n && gk < n) v = ta ? A[(size_t)gk * n + gm] : A[(size_t)gm * n + gk];
      As[kk][mm] = v;
    }
    for (int e = threadIdx.x; e < GB * GK; e += 256) {
      int nn, kk;
      if (!tb) {
        kk = e / GB;
        nn = e - kk * GB;
      } else {
        nn = e / GK;
        kk = e - nn * GK;
      }
      int gn = n0 + nn, gk = k0 + kk;
      double v = 0.0;
      if (gn < n && gk < n) v = tb ? B[(size_t)gn * n + gk] : B[(size_t)gk * n + gn];
      Bs[kk][nn] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GK; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int gm = m0 + ty * 4 + i;
    if (gm >= n) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int gn = n0 + tx * 4 + j;
      if (gn >= n) continue;
      double v = acc[i][j];
      if (ep) {
        double lam = 2.0 - 2.0 * I.cosk[gm] * I.cosk[gn];
        if (ep == 1)
          v = (gm == 0 && gn == 0) ? 0.0 : v / lam;
        else
          v = v * lam;
      }
      D[(size_t)gm * n + gn] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// |d_hat|, early exit and the conjugate-Jacobian beta (otsolver_2dgrid.cpp:179-200, 248-261).

__global__ __launch_bounds__(NT) void k_beta(Inst* insts, const int* tile_inst, double* partials) {
  __shared__ double s[HI * HJ];
  __shared__ double gx[VI * VJ], gy[VI * VJ];
  __shared__ double red[32 * 3];
  Inst& I = insts[tile_inst[blockIdx.x]];
  if (!I.active) return;
  const int n = I.n, it = I.it;
  const double e = 1.0 / (double)n, ea = elem_area(n);
  const bool use_beta = it >= 1 && I.beta_cj;
  TileCoord t = tile_coord(I, blockIdx.x);
  double v[3] = {0.0, 0.0, 0.0};
  if (t.inside) {
    double dh = I.dhat[t.f];
    v[0] = dh * dh;
  }
  if (use_beta) {
    const double eps = I.alpha / 2.0;
    const double* psi = I.psi[it & 1];
    const double* dh = I.dhat;
    load_halo(s, n, t.i0, t.j0, [&](size_t g) { return psi[g] - eps * dh[g]; });
    __syncthreads();
    vertex_grads(s, gx, gy, 0.5 * (double)n);
    __syncthreads();
    if (t.inside) {
      double reps = cell_area(gx, gy, t.ci, t.cj, e) - ea * I.rho[t.f];
      double rk = I.r[it % 3][t.f], rkm1 = I.r[(it + 2) % 3][t.f];
      double jd = rk - rkm1;
      v[1] = jd * (reps - rk);
      v[2] = jd * jd;
    }
  }
  block_sum<3>(v, red);
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) partials[(size_t)blockIdx.x * KP + k] = v[k];
  if (last_block(&I.counter, I.ntiles)) {
    double sum[3];
    reduce_partials<3>(partials, I.tile0, I.ntiles, sum, red);
    if (threadIdx.x == 0) {
      if (sqrt(sum[0]) <= 2.0 * DBL_MIN) {
        I.active = 0;
        I.outcome = OTM_SMALL_STEP;
      } else {
        I.use_beta = use_beta ? 1 : 0;
        if (use_beta) {
          double eps = I.alpha / 2.0;
          I.beta = std_max(-1.0, sum[1] / sum[2] / eps * I.alpha);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Exact line search (otsolver_2dgrid.cpp:541-606).

// d = d_hat + beta d_prev (written), a and b per cell, the quartic's sums; the last
// block picks the step.
__global__ __launch_bounds__(NT) void k_coeffs(Inst* insts, const int* tile_inst, double* partials) {
  __shared__ double sp[HI * HJ], sd[HI * HJ];
  __shared__ double gx[VI * VJ], gy[VI * VJ], hx[VI * VJ], hy[VI * VJ];
  __shared__ double red[32 * 6];
  Inst& I = insts[tile_inst[blockIdx.x]];
  if (!I.active) return;
  const int n = I.n, it = I.it;
  const double e = 1.0 / (double)n, hw = 0.5 * (double)n;
  TileCoord t = tile_coord(I, blockIdx.x);
  const bool use_beta = I.use_beta;
  const double beta = I.beta;
  const double* dh = I.dhat;
  const double* dprev = I.d[(it + 1) & 1];
  double* dnew = I.d[it & 1];
  const double* psi = I.psi[it & 1];
  load_halo(sd, n, t.i0, t.j0, [&](size_t g) { return use_beta ? dh[g] + beta * dprev[g] : dh[g]; });
  load_halo(sp, n, t.i0, t.j0, [&](size_t g) { return psi[g]; });
  __syncthreads();
  vertex_grads(sp, gx, gy, hw);
  vertex_grads(sd, hx, hy, hw);
  __syncthreads();
  double v[6] = {0, 0, 0, 0, 0, 0};
  if (t.inside) {
    double dv = sd[(t.ci + 1) * HJ + t.cj + 1];
    dnew[t.f] = dv;
    double a, b;
    cell_ab(gx, gy, hx, hy, t.ci, t.cj, e, a, b);
    double rk = I.r[it % 3][t.f];
    v[0] = b * rk;
    v[1] = b * b;
    v[2] = a * rk;
    v[3] = a * b;
    v[4] = a * a;
    v[5] = dv * dv;
  }
  block_sum<6>(v, red);
  if (threadIdx.x == 0)
    for (int k = 0; k < 6; ++k) partials[(size_t)blockIdx.x * KP + k] = v[k];
  if (last_block(&I.counter, I.ntiles)) {
    double sum[6];
    reduce_partials<6>(partials, I.tile0, I.ntiles, sum, red);
    if (threadIdx.x == 0) {
      const double ea = elem_area(n);
      double z[5] = {I.residual * ea, 2.0 * sum[0], sum[1] + 2 * sum[2], 2.0 * sum[3], sum[4]};
      double alpha, rmin;
      pick_step(z, &alpha, &rmin);
      I.alpha = alpha;
      I.residual = rmin / ea;
      I.dnorm = sqrt(sum[5]);
    }
  }
}

// psi_{k+1} = psi_k + alpha d and r_{k+1} = a alpha^2 + b alpha + r_k; the last block
// advances the iteration and evaluates the loop condition.
__global__ __launch_bounds__(NT) void k_update(Inst* insts, const int* tile_inst, double* partials) {
  __shared__ double sp[HI * HJ], sd[HI * HJ];
  __shared__ double gx[VI * VJ], gy[VI * VJ], hx[VI * VJ], hy[VI * VJ];
  __shared__ double red[32 * 2];
  Inst& I = insts[tile_inst[blockIdx.x]];
  if (!I.active) return;
  const int n = I.n, it = I.it;
  const double e = 1.0 / (double)n, hw = 0.5 * (double)n, alpha = I.alpha;
  TileCoord t = tile_coord(I, blockIdx.x);
  const double* d = I.d[it & 1];
  const double* psi = I.psi[it & 1];
  load_halo(sd, n, t.i0, t.j0, [&](size_t g) { return d[g]; });
  load_halo(sp, n, t.i0, t.j0, [&](size_t g) { return psi[g]; });
  __syncthreads();
  vertex_grads(sp, gx, gy, hw);
  vertex_grads(sd, hx, hy, hw);
  __syncthreads();
  double mx = -INFINITY;
  if (t.inside) {
    double a, b;
    cell_ab(gx, gy, hx, hy, t.ci, t.cj, e, a, b);
    double p = sp[(t.ci + 1) * HJ + t.cj + 1], dv = sd[(t.ci + 1) * HJ + t.cj + 1];
    I.psi[(it + 1) & 1][t.f] = p + alpha * dv;
    double rn = a * (alpha * alpha) + b * alpha + I.r[it % 3][t.f];
    I.r[(it + 1) % 3][t.f] = rn;
    mx = rn;
  }
  mx = block_max(mx, red);
  if (threadIdx.x == 0) partials[(size_t)blockIdx.x * KP] = mx;
  if (last_block(&I.counter, I.ntiles)) {
    double gmx = reduce_partials_max(partials, I.tile0, I.ntiles, 0, red);
    if (threadIdx.x == 0) {
      I.linf = gmx / elem_area(n);
      I.it = it + 1;
      I.active = (I.it < I.max_iter && I.residual > I.threshold) ? 1 : 0;
      if (!I.active) stop_outcome(I);
    }
  }
}

// Forward mesh: origin grid + exact vertex gradients of the final potential
// (otsolver_2dgrid.cpp:222-227). One thread per vertex.
__global__ void k_forward_mesh(const Inst* insts, int q, double* xy) {
  const Inst& I = insts[q];
  const int n = I.n;
  long v = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long V = (long)(n + 1) * (n + 1);
  if (v >= V) return;
  int i = (int)(v / (n + 1)), j = (int)(v % (n + 1));
  const double* psi = I.psi[I.it & 1];
  auto P = [&](int a, int b) { return psi[(size_t)clampi(a, n) * n + clampi(b, n)]; };
  double p00 = P(i - 1, j - 1), p01 = P(i - 1, j), p10 = P(i, j - 1), p11 = P(i, j);
  double hw = 0.5 * (double)n;
  double gx = hw * ((p10 + p11) - (p00 + p01));
  double gy = hw * ((p01 + p11) - (p00 + p10));
  double dx = 1.0 / (double)n;
  xy[2 * v] = (double)i * dx + gx;
  xy[2 * v + 1] = (double)j * dx + gy;
}

// y = M x, the reference's assembled matrix (otsolver_2dgrid.cpp:284-311), for the
// diagonalisation check.
__global__ void k_laplacian_apply(int n, const double* x, double* y) {
  long f = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= (long)n * n) return;
  int i = (int)(f / n), j = (int)(f % n);
  int i1 = i == 0 ? i : i - 1, j1 = j == 0 ? j : j - 1;
  int i2 = i == n - 1 ? i : i + 1, j2 = j == n - 1 ? j : j + 1;
  y[f] = 2.0 * x[f] - 0.5 * (x[(size_t)i1 * n + j1] + x[(size_t)i1 * n + j2] + x[(size_t)i2 * n + j1] +
                             x[(size_t)i2 * n + j2]);
}

// ---------------------------------------------------------------------------
// Host side.

void DevBuf::reserve(size_t b) {
  if (b <= bytes) return;
  release();
  OTM_CUDA(cudaMalloc(&p, b));
  bytes = b;
}

void AsyncBuf::reserve(size_t b, cudaStream_t s, cudaMemPool_t pool) {
  if (b <= bytes) return;
  release();
  st = s;
  OTM_CUDA(cudaMallocFromPoolAsync(&p, b, pool, s));
  bytes = b;
}

static int tiles_of(int n) { return ((n + TI - 1) / TI) * ((n + TJ - 1) / TJ); }
static int gemm_tiles_of(int n) {
  int t = (n + GB - 1) / GB;
  return t * t;
}

// Strip height srows for every instance of h: its sweep blocks and their place in the
// work list (FP64 instances first, then the split-precision ones: two launches of each
// sweep when a batch has both). Returns the list length; *split0 = first split block.
static int assign_strips(std::vector<Inst>& h, int srows, int* split0 = nullptr) {
  int strips = 0;
  for (auto& I : h) {
    I.srows = srows;
    I.nstrip = strip_blocks(I.n, srows);
  }
  for (int pass = 0; pass < 2; ++pass) {
    if (pass == 1 && split0) *split0 = strips;
    for (auto& I : h)
      if (I.split == pass) {
        I.strip0 = strips;
        strips += I.nstrip;
      }
  }
  return strips;
}

// assign_strips, then the workspace's sweep work list (block -> instance) on the device
// and its partial-sum slots.
static void set_strips(otm_context* ctx, Workspace& ws, std::vector<Inst>& h, int srows) {
  int split0 = 0;
  const int strips = assign_strips(h, srows, &split0);
  std::vector<int> si(strips);
  for (size_t q = 0; q < h.size(); ++q)
    for (int k = 0; k < h[q].nstrip; ++k) si[h[q].strip0 + k] = (int)q;
  ws.strip_inst.reserve(sizeof(int) * strips);
  ws.sweep_partials.reserve(sizeof(double) * SWEEP_SLOTS * (size_t)strips);
  OTM_CUDA(cudaMemcpyAsync(ws.strip_inst.p, si.data(), sizeof(int) * strips, cudaMemcpyHostToDevice, ctx->stream));
  OTM_CUDA(cudaStreamSynchronize(ctx->stream));  // the host list is released on return
  ws.split_strip0 = split0;
  ws.total_strips = strips;
  ws.srows = srows;
}

// Lays out (or reuses) the workspace for a list of sizes and returns host copies of
// the instance records with buffer pointers filled in.
static std::vector<Inst> layout_workspace(otm_context* ctx, const std::vector<int>& sizes) {
  const int count = (int)sizes.size();
  std::vector<Inst> h(count);
  size_t cells = 0;
  int tiles = 0, gemm = 0, rows = 0, cols = 0, tcitems = 0;
  // Taller sweep strips halve the per-strip overhead (ring prologue, block reduction) when
  // the batch has blocks to spare; a batch that does not fill the GPU twice over keeps
  // 32-row strips for parallelism, and one with fewer 32-row blocks than SMs takes 16-row
  // strips (a lone 512^2 solve: sums 28 -> 24.5 us, update 21 -> 16.4 us).
  int srows = 32;
  {
    long blocks32 = 0;
    for (int q = 0; q < count; ++q) blocks32 += strip_blocks(sizes[q], 32);
    if (blocks32 >= 6L * ctx->num_sms)
      srows = 64;
    else if (blocks32 < ctx->num_sms)
      srows = 16;
  }
  for (int q = 0; q < count; ++q) {
    int n = sizes[q];
    Inst& I = h[q];
    std::memset(&I, 0, sizeof(Inst));
    I.n = n;
    I.tile0 = tiles;
    I.ntiles = tiles_of(n);
    tiles += I.ntiles;
    I.fft = (ctx->poisson_mode != OTM_POISSON_DENSE && fft_eligible(n)) ? 1 : 0;
    I.split = (ctx->precision == OTM_PRECISION_SPLIT && I.fft && dct_reg_supported(n)) ? 1 : 0;
    if (ctx->poisson_mode == OTM_POISSON_TENSOR && I.split && dct_tc_supported(n)) {
      I.fft = 0;  // the tensor-core products instead of the FFT passes
      I.tc0 = tcitems;
      I.ntc = dct_tc_tiles(n);
      I.tcn = dct_tc_tn(n);
      tcitems += I.ntc;
    } else if (I.fft) {
      int lg = 0;
      while ((1 << lg) < n) ++lg;
      I.logn = lg;
    } else {
      I.gemm0 = gemm;
      I.ngemm = gemm_tiles_of(n);
      gemm += I.ngemm;
    }
    // 11 cell arrays per instance (12 on the tensor-core transform: the residual's TF32
    // planes), each padded to 32 doubles (256 bytes)
    cells += (11 + (I.ntc > 0 ? 1 : 0)) * (((size_t)n * n + 31) / 32 * 32);
  }
  // fast-transform work lists, grouped into one segment per (kernel family, size)
  std::vector<Workspace::Segment> segs;
  {
    std::vector<int> order;
    for (int q = 0; q < count; ++q)
      if (h[q].fft) order.push_back(q);
    auto key = [&](int q) { return std::make_pair(dct_reg_supported(h[q].n) ? 1 : 0, h[q].n); };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key(a) < key(b); });
    for (size_t k = 0; k < order.size(); ++k) {
      Inst& I = h[order[k]];
      const int reg = dct_reg_supported(I.n) ? 1 : 0;
      const int per = reg ? dct_reg_lines_per_block(I.n) : fft_lines(I.n);
      const int cper = reg ? dct_reg_cols_per_block(I.n) : fft_lines(I.n);
      if (segs.empty() || segs.back().n != I.n || segs.back().reg != reg)
        segs.push_back({I.n, reg, I.split, rows, 0, cols, 0});
      I.row0 = rows;
      I.nrow = I.n / per;
      I.col0 = cols;
      I.ncol = I.n / cper;
      rows += I.nrow;
      cols += I.ncol;
      segs.back().rcnt += I.nrow;
      segs.back().ccnt += I.ncol;
    }
  }
  // the workspace of this configuration: a cached one, else a new one (evicting the least
  // recently used)
  bool same = false;
  {
    auto& W = ctx->workspaces;
    size_t hit = W.size();
    for (size_t k = 0; k < W.size(); ++k)
      if (W[k]->sizes == sizes && W[k]->mode == ctx->poisson_mode && W[k]->precision == ctx->precision) hit = k;
    if (hit < W.size()) {
      std::rotate(W.begin(), W.begin() + hit, W.begin() + hit + 1);
      same = true;
    } else {
      if ((int)W.size() >= otm_context::kWorkspaces) W.pop_back();
      W.insert(W.begin(), std::make_unique<Workspace>());
    }
    ctx->wsp = W.front().get();
  }
  Workspace& ws = ctx->ws();
  if (!same) {
    ws.drop_graph();
    ws.insts.reserve(sizeof(Inst) * count);
    ws.tile_inst.reserve(sizeof(int) * tiles);
    ws.gemm_inst.reserve(sizeof(int) * (gemm > 0 ? gemm : 1));
    ws.tc_inst.reserve(sizeof(int) * (tcitems > 0 ? tcitems : 1));
    ws.row_inst.reserve(sizeof(int) * (rows > 0 ? rows : 1));
    ws.col_inst.reserve(sizeof(int) * (cols > 0 ? cols : 1));
    ws.partials.reserve(sizeof(double) * KP * (size_t)tiles);
    ws.arena.reserve(sizeof(double) * cells);
    std::vector<int> ti(tiles), gi(gemm), ri(rows), ci(cols), tci(tcitems);
    for (int q = 0; q < count; ++q) {
      for (int k = 0; k < h[q].ntc; ++k) tci[h[q].tc0 + k] = q;
      for (int k = 0; k < h[q].ntiles; ++k) ti[h[q].tile0 + k] = q;
      for (int k = 0; k < h[q].ngemm; ++k) gi[h[q].gemm0 + k] = q;
      for (int k = 0; k < h[q].nrow; ++k) ri[h[q].row0 + k] = q;
      for (int k = 0; k < h[q].ncol; ++k) ci[h[q].col0 + k] = q;
    }
    cudaStream_t st = ctx->stream;
    OTM_CUDA(cudaMemcpyAsync(ws.tile_inst.p, ti.data(), sizeof(int) * tiles, cudaMemcpyHostToDevice, st));
    if (gemm) OTM_CUDA(cudaMemcpyAsync(ws.gemm_inst.p, gi.data(), sizeof(int) * gemm, cudaMemcpyHostToDevice, st));
    if (tcitems)
      OTM_CUDA(cudaMemcpyAsync(ws.tc_inst.p, tci.data(), sizeof(int) * tcitems, cudaMemcpyHostToDevice, st));
    if (rows) OTM_CUDA(cudaMemcpyAsync(ws.row_inst.p, ri.data(), sizeof(int) * rows, cudaMemcpyHostToDevice, st));
    if (cols) OTM_CUDA(cudaMemcpyAsync(ws.col_inst.p, ci.data(), sizeof(int) * cols, cudaMemcpyHostToDevice, st));
    OTM_CUDA(cudaStreamSynchronize(st));
    ws.sizes = sizes;
    ws.mode = ctx->poisson_mode;
    ws.precision = ctx->precision;
    ws.total_tiles = tiles;
    ws.total_gemm = gemm;
    ws.total_tc = tcitems;
    ws.total_rows = rows;
    ws.total_cols = cols;
    ws.segments = segs;
    size_t need = sizeof(Inst) * count;
    if (ws.h_pinned_bytes < need) {
      if (ws.h_pinned) cudaFreeHost(ws.h_pinned);
      ws.h_pinned = nullptr;
      OTM_CUDA(cudaMallocHost(&ws.h_pinned, need));
      ws.h_pinned_bytes = need;
    }
  }
  // sweep strips: a new layout takes the rule's height, a cached one keeps its own
  // (possibly autotuned) height and work list
  if (!same)
    set_strips(ctx, ws, h, srows);
  else
    assign_strips(h, ws.srows);
  double* base = ws.arena.as<double>();
  for (int q = 0; q < count; ++q) {
    Inst& I = h[q];
    size_t N = (((size_t)I.n * I.n + 31) / 32) * 32;
    double* arr[12] = {};
    for (int k = 0; k < 11 + (I.ntc > 0 ? 1 : 0); ++k) {
      arr[k] = base;
      base += N;
    }
    I.psi[0] = arr[0];
    I.psi[1] = arr[1];
    I.r[0] = arr[2];
    I.r[1] = arr[3];
    I.r[2] = arr[4];
    I.dhat = arr[5];
    I.d[0] = arr[6];
    I.d[1] = arr[7];
    I.rho = arr[8];
    I.t1 = arr[9];
    I.t2 = arr[10];
    SizeTables* T = ctx->tables.at(I.n).get();
    I.C = T->C.as<double>();
    I.cosk = T->cosk.as<double>();
    I.tw = T->tw.as<double2>();
    I.pt = T->pt.as<double2>();
    I.Cf = T->Cf.as<float>();
    I.CTf = T->CTf.as<float>();
    I.rs = reinterpret_cast<float*>(arr[11]);
  }
  if (tcitems > 0) {
    // tensor maps of the tensor-core instances, encoded again only when their buffers moved
    std::vector<const void*> key;
    for (const Inst& I : h)
      if (I.ntc > 0) key.insert(key.end(), {(const void*)I.rs, I.t1, I.t2, I.Cf, I.CTf, (const void*)(size_t)I.n});
    const size_t mb = dct_tc_map_bytes();
    if (key != ws.tmap_key) {
      ws.tmap_key.clear();
      std::vector<unsigned char> maps;
      for (const Inst& I : h)
        if (I.ntc > 0) {
          maps.resize(maps.size() + mb);
          dct_tc_encode(I, maps.data() + maps.size() - mb);
        }
      ws.tmaps.reserve(maps.size());
      OTM_CUDA(cudaMemcpyAsync(ws.tmaps.p, maps.data(), maps.size(), cudaMemcpyHostToDevice, ctx->stream));
      OTM_CUDA(cudaStreamSynchronize(ctx->stream));
      ws.tmap_key = key;
    }
    size_t k = 0;
    for (Inst& I : h)
      if (I.ntc > 0) I.tmaps = ws.tmaps.as<unsigned char>() + mb * k++;
  }
  return h;
}

static SizeTables* init_size(otm_context* ctx, int n);

// The dense-product Poisson solve for one record (used by the adjoint).
void dense_poisson(otm_context* ctx, Inst* d_inst, const int* gemm_inst, int G) {
  for (int s = 0; s < 4; ++s) launch(ctx, "dct_gemm", k_dct_gemm, G, 256, (const Inst*)d_inst, gemm_inst, s, 1);
}

// Bound on the device-side loop: the WHILE node stops after `cap` bodies whatever the
// instances report, and flags it.
struct LoopCtl {
  unsigned int count, cap;
  int error, pad;
};

// Body tail of the graph loop: continue while any instance is active.
__global__ void k_loop_check(const Inst* insts, int count, LoopCtl* ctl, cudaGraphConditionalHandle h) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int q = threadIdx.x; q < count; q += blockDim.x)
    if (insts[q].active) any = 1;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int c = ++ctl->count;
    unsigned int go = any && c < ctl->cap;
    if (any && !(c < ctl->cap)) ctl->error = 1;
    cudaGraphSetConditional(h, go);
  }
}

// Launches one iteration of every active instance (Poisson solve + the two sweeps).
static void launch_iteration(otm_context* ctx, Inst* d_insts) {
  Workspace& ws = ctx->ws();
  const int G = ws.total_gemm;
  if (G > 0)
    for (int s = 0; s < 4; ++s)
      launch(ctx, "dct_gemm", k_dct_gemm, G, 256, (const Inst*)d_insts, ws.gemm_inst.as<int>(), s, 1);
  for (const auto& sg : ws.segments) {
    if (sg.reg)
      dct_reg_run(ctx, sg.n, sg.split != 0, d_insts, ws.row_inst.as<int>(), sg.roff, sg.rcnt, ws.col_inst.as<int>(), sg.coff,
                  sg.ccnt);
    else
      poisson_fft(ctx, d_insts, ws.row_inst.as<int>(), sg.roff, sg.rcnt, ws.col_inst.as<int>(), sg.coff, sg.ccnt);
  }
  if (ws.total_tc > 0) dct_tc_run(ctx, d_insts, ws.tc_inst.as<int>(), 0, ws.total_tc);
  const int* si = ws.strip_inst.as<int>();
  double* sp = ws.sweep_partials.as<double>();
  const int s64 = ws.split_strip0, s32 = ws.total_strips - ws.split_strip0;
  sweep_sums(ctx, d_insts, si, 0, s64, false, sp);
  sweep_sums(ctx, d_insts, si, s64, s32, true, sp);
  sweep_update(ctx, d_insts, si, 0, s64, false, sp);
  sweep_update(ctx, d_insts, si, s64, s32, true, sp);
}

// Captures the iteration loop of the current workspace into a graph with a WHILE node.
static void build_loop_graph(otm_context* ctx, int count) {
  Workspace& ws = ctx->ws();
  cudaStream_t st = ctx->stream;
  sweep_attrs(ctx->device);
  dct_reg_attrs(ctx->device);
  dct_tc_attrs(ctx->device);
  poisson_fft_attrs(ctx->device);
  ws.loopctl.reserve(sizeof(LoopCtl));
  cudaGraph_t g = nullptr;
  OTM_CUDA(cudaGraphCreate(&g, 0));
  try {
    cudaGraphConditionalHandle handle;
    OTM_CUDA(cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams params = {};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = handle;
    params.conditional.type = cudaGraphCondTypeWhile;
    params.conditional.size = 1;
    cudaGraphNode_t node;
    OTM_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &params));
    cudaGraph_t body = params.conditional.phGraph_out[0];
    const long before = ctx->launches;
    OTM_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    try {
      launch_iteration(ctx, ws.insts.as<Inst>());
      launch(ctx, "loop_check", k_loop_check, 1, 256, (const Inst*)ws.insts.as<Inst>(), count,
             ws.loopctl.as<LoopCtl>(), handle);
    } catch (...) {
      cudaGraph_t dummy;
      cudaStreamEndCapture(st, &dummy);
      throw;
    }
    OTM_CUDA(cudaStreamEndCapture(st, &body));
    ws.graph_body_kernels = ctx->launches - before;
    ctx->launches = before;  // captured, not executed
    OTM_CUDA(cudaGraphInstantiate(&ws.graph_exec, g, 0));
  } catch (...) {
    cudaGraphDestroy(g);
    throw;
  }
  cudaGraphDestroy(g);
}

// Runs the whole solve for `count` instances whose raw densities have been copied
// into their rho buffers. Host-side copies of the final records are returned. With
// `stopped` (device loop only), the host watches the records while the loop runs and
// calls stopped(q) once for each instance that is no longer active -- its potential and
// density are final from then on -- so that its outputs can be produced on the side
// stream while the rest of the batch iterates; `done` marks those instances.
static std::vector<Inst> run_solver(otm_context* ctx, std::vector<Inst>& h, const otm_solver_options& o,
                                    const std::function<void(int)>* stopped = nullptr,
                                    std::vector<char>* done = nullptr) {
  Workspace& ws = ctx->ws();
  cudaStream_t st = ctx->stream;
  const int count = (int)h.size();
  for (auto& I : h) {
    I.max_iter = o.max_iter;
    I.beta_cj = o.beta == OTM_BETA_CONJUGATE_JACOBIAN ? 1 : 0;
    I.threshold = o.threshold;
    I.max_ratio = o.max_ratio;
    size_t N = (size_t)I.n * I.n;
    OTM_CUDA(cudaMemsetAsync(I.psi[0], 0, N * sizeof(double), st));
    OTM_CUDA(cudaMemsetAsync(I.d[0], 0, N * sizeof(double), st));
    OTM_CUDA(cudaMemsetAsync(I.d[1], 0, N * sizeof(double), st));
    OTM_CUDA(cudaMemsetAsync(I.r[2], 0, N * sizeof(double), st));
  }
  Inst* d_insts = ws.insts.as<Inst>();
  OTM_CUDA(cudaMemcpyAsync(d_insts, h.data(), sizeof(Inst) * count, cudaMemcpyHostToDevice, st));
  const int* ti = ws.tile_inst.as<int>();
  double* part = ws.partials.as<double>();
  const int T = ws.total_tiles;

  launch(ctx, "density_sum", k_density_sum, T, NT, d_insts, ti, part);
  launch(ctx, "density_scale", k_density_scale, T, NT, d_insts, ti, part);
  launch(ctx, "density_apply", k_density_apply, T, NT, d_insts, ti);
  launch(ctx, "residual_init", k_residual_init, T, NT, d_insts, ti, part);
  OTM_CUDA(cudaGetLastError());
  if (stopped) OTM_CUDA(cudaEventRecord(ctx->side_ready, st));

  Inst* hp = static_cast<Inst*>(ws.h_pinned);
  if (ctx->loop_mode == OTM_LOOP_GRAPH && !ctx->prof.on) {
    if (!ws.graph_exec) build_loop_graph(ctx, count);
    LoopCtl c = {0u, (unsigned int)o.max_iter + 2u, 0, 0};
    OTM_CUDA(cudaMemcpyAsync(ws.loopctl.p, &c, sizeof(c), cudaMemcpyHostToDevice, st));
    OTM_CUDA(cudaGraphLaunch(ws.graph_exec, st));
    if (stopped && done) {
      Inst* poll = static_cast<Inst*>(ctx->h_poll);
      // the records start inactive on the host side: watch them only once the set-up
      // kernels (queued before the graph) have initialised them
      OTM_CUDA(cudaStreamWaitEvent(ctx->side, ctx->side_ready, 0));
      while (true) {
        const cudaError_t q = cudaStreamQuery(st);
        if (q == cudaSuccess) break;
        if (q != cudaErrorNotReady) OTM_CUDA(q);
        // a racy but harmless read: `active` only ever goes from 1 to 0, and the last
        // block that clears it has made the instance's arrays final before doing so
        OTM_CUDA(cudaMemcpyAsync(poll, d_insts, sizeof(Inst) * count, cudaMemcpyDeviceToHost, ctx->side));
        OTM_CUDA(cudaStreamSynchronize(ctx->side));
        for (int k = 0; k < count; ++k)
          if (!(*done)[k] && !poll[k].active && !poll[k].fault) {
            (*stopped)(k);
            (*done)[k] = 1;
          }
        std::this_thread::sleep_for(std::chrono::microseconds(200));
      }
      OTM_CUDA(cudaStreamSynchronize(ctx->side));
    }
    OTM_CUDA(cudaMemcpyAsync(hp, d_insts, sizeof(Inst) * count, cudaMemcpyDeviceToHost, st));
    OTM_CUDA(cudaMemcpyAsync(&c, ws.loopctl.p, sizeof(c), cudaMemcpyDeviceToHost, st));
    OTM_CUDA(cudaStreamSynchronize(st));
    ctx->launches += ws.graph_body_kernels * (long)c.count;
    if (c.error) throw CudaError{cudaErrorLaunchTimeout, "device loop exceeded its iteration bound"};
  } else {
    int launched = 0;
    const int chunk = 4;
    while (true) {
      OTM_CUDA(cudaMemcpyAsync(hp, d_insts, sizeof(Inst) * count, cudaMemcpyDeviceToHost, st));
      OTM_CUDA(cudaStreamSynchronize(st));
      ctx->prof.flush();
      bool any = false;
      for (int q = 0; q < count; ++q) any |= hp[q].active != 0;
      if (!any || launched >= o.max_iter) break;
      for (int c = 0; c < chunk && launched < o.max_iter; ++c, ++launched) launch_iteration(ctx, d_insts);
      OTM_CUDA(cudaGetLastError());
    }
  }
  for (int q = 0; q < count; ++q)
    if (hp[q].fault) throw DeviceTimeout{"a bounded device-side wait gave up"};
  std::vector<Inst> out(hp, hp + count);
  return out;
}

// OTM_AUTOTUNE_ON, first call of a batch configuration: K iterations of the call's own
// densities at each candidate strip height (host-driven loop, CUDA events on the context
// stream, the second of two runs), the fastest kept for the configuration. Every run
// starts from the raw densities (the set-up normalises them in place), and so does the
// real solve afterwards.
static void tune_strips(otm_context* ctx, std::vector<Inst>& h, const otm_solver_options& o,
                        const double* const* density) {
  Workspace& ws = ctx->ws();
  const int K = 4;
  ws.tuned = true;
  if (o.max_iter < K) return;  // nothing worth timing
  auto reload = [&] {
    for (size_t q = 0; q < h.size(); ++q)
      copy_in(ctx, h[q].rho, density[q], sizeof(double) * (size_t)h[q].n * h[q].n);
  };
  otm_solver_options t = o;
  t.max_iter = K;
  const int loop = ctx->loop_mode, rule = ws.srows;
  cudaEvent_t a = nullptr, b = nullptr;
  int best = rule;
  double best_ms = 0.0;
  try {
    ctx->loop_mode = OTM_LOOP_HOST;
    OTM_CUDA(cudaEventCreate(&a));
    OTM_CUDA(cudaEventCreate(&b));
    for (int c : {16, 32, 64}) {
      set_strips(ctx, ws, h, c);
      float ms = 0.f;
      for (int rep = 0; rep < 2; ++rep) {
        reload();
        OTM_CUDA(cudaEventRecord(a, ctx->stream));
        run_solver(ctx, h, t);
        OTM_CUDA(cudaEventRecord(b, ctx->stream));
        OTM_CUDA(cudaEventSynchronize(b));
        OTM_CUDA(cudaEventElapsedTime(&ms, a, b));
      }
      if (best_ms == 0.0 || ms < best_ms) {
        best_ms = ms;
        best = c;
      }
    }
  } catch (...) {
    ctx->loop_mode = loop;
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    throw;
  }
  ctx->loop_mode = loop;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  set_strips(ctx, ws, h, best);
  ws.drop_graph();  // captured with another work list
  reload();
}

static void fill_stats(const Inst& I, otm_solve_stats* s) {
  if (!s) return;
  s->iterations = I.it;
  s->outcome = I.outcome;
  s->residual = I.residual;
  s->linf = I.linf;
  s->initial_residual = I.residual0;
}

// Builds the size-n cosine tables and runs the diagonalisation check on the GPU.
static SizeTables* init_size(otm_context* ctx, int n) {
  auto it = ctx->tables.find(n);
  if (it != ctx->tables.end()) return it->second.get();
  auto T = std::make_unique<SizeTables>();
  T->n = n;
  std::vector<double> C((size_t)n * n), ck(n);
  for (int k = 0; k < n; ++k) {
    double s = k == 0 ? std::sqrt(1.0 / n) : std::sqrt(2.0 / n);
    for (int i = 0; i < n; ++i) C[(size_t)k * n + i] = s * std::cos(M_PI * (i + 0.5) * k / n);
    ck[k] = std::cos(M_PI * k / n);
  }
  T->C.reserve(sizeof(double) * C.size());
  T->cosk.reserve(sizeof(double) * n);
  cudaStream_t st = ctx->stream;
  if (fft_eligible(n)) {
    std::vector<double2> tw(n / 2), pt(n);
    for (int k = 0; k < n / 2; ++k) tw[k] = make_double2(std::cos(2.0 * M_PI * k / n), -std::sin(2.0 * M_PI * k / n));
    for (int k = 0; k < n; ++k) pt[k] = make_double2(std::cos(M_PI * k / (2.0 * n)), std::sin(M_PI * k / (2.0 * n)));
    std::vector<double2> tw2;
    dct_reg_step2_table(n, tw, tw2);
    tw.insert(tw.end(), tw2.begin(), tw2.end());
    T->tw.reserve(sizeof(double2) * tw.size());
    T->pt.reserve(sizeof(double2) * n);
    OTM_CUDA(cudaMemcpyAsync(T->tw.p, tw.data(), sizeof(double2) * tw.size(), cudaMemcpyHostToDevice, st));
    OTM_CUDA(cudaMemcpyAsync(T->pt.p, pt.data(), sizeof(double2) * n, cudaMemcpyHostToDevice, st));
    OTM_CUDA(cudaStreamSynchronize(st));
  }
  OTM_CUDA(cudaMemcpyAsync(T->C.p, C.data(), sizeof(double) * C.size(), cudaMemcpyHostToDevice, st));
  if (dct_tc_supported(n)) {  // TF32 planes of the basis and its transpose (tensor-core transform)
    std::vector<float> cf, ctf;
    dct_tc_split_basis(C.data(), n, cf, ctf);
    T->Cf.reserve(sizeof(float) * cf.size());
    T->CTf.reserve(sizeof(float) * ctf.size());
    OTM_CUDA(cudaMemcpyAsync(T->Cf.p, cf.data(), sizeof(float) * cf.size(), cudaMemcpyHostToDevice, st));
    OTM_CUDA(cudaMemcpyAsync(T->CTf.p, ctf.data(), sizeof(float) * ctf.size(), cudaMemcpyHostToDevice, st));
    OTM_CUDA(cudaStreamSynchronize(st));  // the host vectors are released on return
  }
  OTM_CUDA(cudaMemcpyAsync(T->cosk.p, ck.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));

  // Check M x == C^T (lambda o (C X C^T)) C on a random probe (otsolver_2dgrid.cpp:284-311).
  size_t N = (size_t)n * n;
  DevBuf buf;
  buf.reserve(sizeof(double) * N * 5);
  double* x = buf.as<double>();
  double* y1 = x + N;
  double* y2 = x + 2 * N;
  double* t1 = x + 3 * N;
  double* t2 = x + 4 * N;
  std::vector<double> hx(N);
  std::mt19937_64 rng(12345 + n);
  std::uniform_real_distribution<double> U(-1.0, 1.0);
  for (auto& v : hx) v = U(rng);
  OTM_CUDA(cudaMemcpyAsync(x, hx.data(), sizeof(double) * N, cudaMemcpyHostToDevice, st));
  k_laplacian_apply<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(n, x, y1);
  Inst I;
  std::memset(&I, 0, sizeof(I));
  I.n = n;
  I.ngemm = gemm_tiles_of(n);
  I.r[0] = x;
  I.dhat = y2;
  I.t1 = t1;
  I.t2 = t2;
  I.C = T->C.as<double>();
  I.cosk = T->cosk.as<double>();
  I.active = 1;
  DevBuf dI, dG;
  dI.reserve(sizeof(Inst));
  dG.reserve(sizeof(int) * I.ngemm);
  std::vector<int> zeros(I.ngemm, 0);
  OTM_CUDA(cudaMemcpyAsync(dI.p, &I, sizeof(Inst), cudaMemcpyHostToDevice, st));
  OTM_CUDA(cudaMemcpyAsync(dG.p, zeros.data(), sizeof(int) * I.ngemm, cudaMemcpyHostToDevice, st));
  for (int s = 0; s < 4; ++s) k_dct_gemm<<<I.ngemm, 256, 0, st>>>(dI.as<Inst>(), dG.as<int>(), s, 2);
  OTM_CUDA(cudaGetLastError());
  std::vector<double> h1(N), h2(N);
  OTM_CUDA(cudaMemcpyAsync(h1.data(), y1, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  OTM_CUDA(cudaMemcpyAsync(h2.data(), y2, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  OTM_CUDA(cudaStreamSynchronize(st));
  double err = 0, scale = 0;
  for (size_t f = 0; f < N; ++f) {
    err = std::max(err, std::fabs(h1[f] - h2[f]));
    scale = std::max(scale, std::fabs(h1[f]));
  }
  T->dct_check_err = scale > 0 ? err / scale : err;
  T->dct_ok = T->dct_check_err <= 1e-10;
  SizeTables* raw = T.get();
  ctx->tables[n] = std::move(T);
  return raw;
}

}  // namespace otm

using namespace otm;

extern "C" int otm_init(otm_context* ctx, int n) {
  return guarded([&] {
    if (!ctx) throw BadArg{"otm_init: null context"};
    if (n < 1 || n > 16384) throw BadArg{"otm_init: grid size must be in [1, 16384]"};
    make_current(ctx);
    SizeTables* T = init_size(ctx, n);
    if (!T->dct_ok)
      throw BadArg{"otm_init: the cosine basis does not diagonalise the assembled matrix (relative error " +
                   std::to_string(T->dct_check_err) + ")"};
    return (int)OTM_OK;
  });
}

static void check_opts(const otm_solver_options& o) {
  if (o.beta != OTM_BETA_ZERO && o.beta != OTM_BETA_CONJUGATE_JACOBIAN) throw BadArg{"unknown beta option"};
  if (o.max_iter < 0) throw BadArg{"max_iter must be >= 0"};
}

extern "C" int otm_solve_batch(otm_context* ctx, int count, const int* ns, const double* const* density,
                               const otm_solver_options* opt, double* const* fwd_xy, double* const* adjusted,
                               otm_solve_stats* stats) {
  return guarded([&] {
    if (!ctx) throw BadArg{"otm_solve_batch: null context"};
    if (count < 1 || !ns || !density || !fwd_xy) throw BadArg{"otm_solve_batch: bad arguments"};
    otm_solver_options o;
    otm_default_options(&o);
    if (opt) o = *opt;
    check_opts(o);
    make_current(ctx);
    std::vector<int> sizes(ns, ns + count);
    for (int q = 0; q < count; ++q) {
      if (sizes[q] < 1 || sizes[q] > 16384) throw BadArg{"otm_solve_batch: grid size out of range"};
      if (!density[q] || !fwd_xy[q]) throw BadArg{"otm_solve_batch: null buffer"};
      auto it = ctx->tables.find(sizes[q]);
      if (it == ctx->tables.end()) {
        SizeTables* T = init_size(ctx, sizes[q]);
        if (!T->dct_ok) throw BadArg{"otm_solve_batch: diagonalisation check failed"};
      }
    }
    std::vector<Inst> h = layout_workspace(ctx, sizes);
    for (int q = 0; q < count; ++q)
      copy_in(ctx, h[q].rho, density[q], sizeof(double) * (size_t)sizes[q] * sizes[q]);
    if (ctx->autotune == OTM_AUTOTUNE_ON && !ctx->ws().tuned && !ctx->prof.on) tune_strips(ctx, h, o, density);
    ctx->last_srows = ctx->ws().srows;
    Inst* d_insts = ctx->ws().insts.as<Inst>();
    // Host outputs of a batch on the device loop: the mesh of an instance that has stopped
    // is formed and copied out on a second stream while the others still iterate.
    bool early = count > 1 && ctx->loop_mode == OTM_LOOP_GRAPH && !ctx->prof.on;
    bool any_host = false;
    size_t vmax = 0;
    for (int q = 0; q < count; ++q) {
      any_host |= !is_device_ptr(fwd_xy[q]);
      vmax = std::max(vmax, (size_t)(sizes[q] + 1) * (sizes[q] + 1));
    }
    early = early && any_host;
    std::vector<char> done(count, 0);
    std::function<void(int)> stopped = [&](int q) {
      const int n = sizes[q];
      const size_t V = (size_t)(n + 1) * (n + 1);
      const bool dev = is_device_ptr(fwd_xy[q]);
      double* dst = dev ? fwd_xy[q] : ctx->staging_side.as<double>();
      ctx->launches++;
      k_forward_mesh<<<(unsigned)((V + 255) / 256), 256, 0, ctx->side>>>((const Inst*)d_insts, q, dst);
      OTM_CUDA(cudaGetLastError());
      if (!dev) OTM_CUDA(cudaMemcpyAsync(fwd_xy[q], dst, sizeof(double) * 2 * V, cudaMemcpyDefault, ctx->side));
      if (adjusted && adjusted[q])
        OTM_CUDA(cudaMemcpyAsync(adjusted[q], h[q].rho, sizeof(double) * (size_t)n * n, cudaMemcpyDefault,
                                 ctx->side));
    };
    if (early) {
      if (!ctx->side) OTM_CUDA(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
      if (!ctx->side_ready) OTM_CUDA(cudaEventCreateWithFlags(&ctx->side_ready, cudaEventDisableTiming));
      ctx->staging_side.reserve(sizeof(double) * 2 * vmax);  // before the loop: no allocation inside it
      const size_t pb = sizeof(Inst) * (size_t)count;
      if (ctx->h_poll_bytes < pb) {
        if (ctx->h_poll) cudaFreeHost(ctx->h_poll);
        ctx->h_poll = nullptr;
        OTM_CUDA(cudaMallocHost(&ctx->h_poll, pb));
        ctx->h_poll_bytes = pb;
      }
    }
    std::vector<Inst> fin = early ? run_solver(ctx, h, o, &stopped, &done) : run_solver(ctx, h, o);
    for (int q = 0; q < count; ++q) {
      if (done[q]) {
        if (stats) fill_stats(fin[q], &stats[q]);
        continue;
      }
      int n = sizes[q];
      size_t V = (size_t)(n + 1) * (n + 1);
      bool dev = is_device_ptr(fwd_xy[q]);
      double* dst = fwd_xy[q];
      if (!dev) {
        ctx->staging.reserve(sizeof(double) * 2 * V);
        dst = ctx->staging.as<double>();
      }
      launch(ctx, "forward_mesh", k_forward_mesh, (unsigned)((V + 255) / 256), 256, (const Inst*)d_insts, q, dst);
      OTM_CUDA(cudaGetLastError());
      if (!dev) copy_out(ctx, fwd_xy[q], dst, sizeof(double) * 2 * V);
      if (adjusted && adjusted[q]) copy_out(ctx, adjusted[q], h[q].rho, sizeof(double) * (size_t)n * n);
      if (stats) fill_stats(fin[q], &stats[q]);
    }
    OTM_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->prof.flush();
    return (int)OTM_OK;
  });
}

extern "C" int otm_solve(otm_context* ctx, int n, const double* density, const otm_solver_options* opt,
                         double* fwd_xy, double* adjusted, otm_solve_stats* stats) {
  double* adj[1] = {adjusted};
  double* fwd[1] = {fwd_xy};
  const double* dens[1] = {density};
  return otm_solve_batch(ctx, 1, &n, dens, opt, fwd, adjusted ? adj : nullptr, stats);
}

// ---------------------------------------------------------------------------
// Allocation-free solve.
//
// Some callers cannot let a library call cudaMalloc: hosts whose own allocator has
// reserved all device memory at start-up, and processes under a hard device-memory
// budget where an allocation in mid-run can fail. otm_solve_noalloc serves them: its
// working memory -- instance record, work lists, partial sums, cosine tables and the
// per-cell arrays -- lives in one file-scope device array of fixed size, so the call
// allocates nothing. That array is held by every GPU that loads the library until the
// process exits, which is why it is kept modest: it bounds the grid size to
// OTM_NOALLOC_MAX_N. The solve runs the dense-product Poisson solve (k_dct_gemm, O(n^3)
// per iteration) and the one-tile-per-block stencil kernels k_beta / k_coeffs /
// k_update, whose work lists fit the array for any n up to that bound; it matches
// otm_solve to the solver's tolerance, not bit for bit. It synchronises the stream and
// reads the loop state back every 4 iterations, so it cannot run inside a stream capture.

namespace otm {

constexpr size_t kNoallocWords = size_t(1) << 20;  // 8 MiB of doubles
static __device__ __align__(256) double g_noalloc_scratch[kNoallocWords];

constexpr int kMaxDevices = 64;
static std::mutex g_noalloc_mu;
static double* g_noalloc_ptr[kMaxDevices];                        // device address of the array, per device
static unsigned char g_noalloc_checked[kMaxDevices][OTM_NOALLOC_MAX_N + 1];  // diagonalisation verified

// Cosine tables for size n, built on the device (no host staging buffer).
__global__ void k_noalloc_tables(int n, double* C, double* cosk) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < (long)n * n) {
    int k = (int)(t / n), i = (int)(t % n);
    double s = k == 0 ? sqrt(1.0 / n) : sqrt(2.0 / n);
    C[t] = s * cos(M_PI * (i + 0.5) * k / n);
  }
  if (t < n) cosk[t] = cos(M_PI * (double)t / n);
}

// Deterministic probe vector in [-1, 1) for the diagonalisation check.
__global__ void k_noalloc_probe(long N, double* x) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= N) return;
  unsigned long long h = (unsigned long long)(t + 1) * 0x9E3779B97F4A7C15ull;
  h ^= h >> 31;
  h *= 0xBF58476D1CE4E5B9ull;
  h ^= h >> 29;
  x[t] = (double)(h >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}

// out[0] = max |a - b|, out[1] = max |a| (one block).
__global__ void k_noalloc_maxdiff(long N, const double* a, const double* b, double* out) {
  __shared__ double red[32];
  double d = 0.0, m = 0.0;
  for (long t = threadIdx.x; t < N; t += blockDim.x) {
    d = fmax(d, fabs(a[t] - b[t]));
    m = fmax(m, fabs(a[t]));
  }
  d = block_max(d, red);
  m = block_max(m, red);
  if (threadIdx.x == 0) {
    out[0] = d;
    out[1] = m;
  }
}

// Word offsets of everything the solve keeps in the array, for grid size n.
struct NoallocLayout {
  size_t inst, tiles, gemm, partials, C, cosk, cells, fwd, check, end;
  size_t npad;
};

static size_t up32(size_t w) { return (w + 31) / 32 * 32; }

static NoallocLayout noalloc_layout(int n) {
  NoallocLayout L;
  size_t w = 0;
  L.inst = w;
  w += up32((sizeof(Inst) + 7) / 8);
  L.tiles = w;
  w += up32(((size_t)tiles_of(n) + 1) / 2);
  L.gemm = w;
  w += up32(((size_t)gemm_tiles_of(n) + 1) / 2);
  L.partials = w;
  w += up32((size_t)tiles_of(n) * KP);
  L.C = w;
  w += up32((size_t)n * n);
  L.cosk = w;
  w += up32((size_t)n);
  L.npad = up32((size_t)n * n);
  L.cells = w;
  w += 11 * L.npad;
  L.fwd = w;
  w += up32(2 * (size_t)(n + 1) * (n + 1));
  L.check = w;
  w += 2 * 32;
  L.end = w;
  return L;
}

static double* noalloc_scratch(int dev) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    double* p = nullptr;
    // with `dev` current: the symbol's address on that device
    OTM_CUDA(cudaGetSymbolAddress((void**)&p, g_noalloc_scratch));
    g_noalloc_ptr[dev] = p;
  }
  return g_noalloc_ptr[dev];
}

}  // namespace otm

extern "C" int otm_solve_noalloc(int n, const double* density, const otm_solver_options* opt, double* fwd_xy,
                                 double* adjusted, otm_solve_stats* stats, void* stream_handle) {
  return guarded([&] {
    if (n < 1 || n > OTM_NOALLOC_MAX_N)
      throw BadArg{"otm_solve_noalloc: grid size " + std::to_string(n) + " exceeds the allocation-free limit of " +
                   std::to_string(OTM_NOALLOC_MAX_N) + " (use otm_solve)"};
    if (!density || !fwd_xy) throw BadArg{"otm_solve_noalloc: null buffer"};
    otm_solver_options o;
    otm_default_options(&o);
    if (opt) o = *opt;
    check_opts(o);
    int dev = 0;
    OTM_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw BadArg{"otm_solve_noalloc: device ordinal out of range"};
    cudaStream_t st = static_cast<cudaStream_t>(stream_handle);
    double* base = noalloc_scratch(dev);
    const NoallocLayout L = noalloc_layout(n);
    if (L.end > kNoallocWords) throw BadArg{"otm_solve_noalloc: scratch layout exceeds the static array"};

    const size_t N = (size_t)n * n, V = (size_t)(n + 1) * (n + 1);
    Inst* d_inst = reinterpret_cast<Inst*>(base + L.inst);
    int* d_tiles = reinterpret_cast<int*>(base + L.tiles);
    int* d_gemm = reinterpret_cast<int*>(base + L.gemm);
    double* part = base + L.partials;
    double* C = base + L.C;
    double* cosk = base + L.cosk;
    double* cells = base + L.cells;
    const int T = tiles_of(n), G = gemm_tiles_of(n);

    // work lists: every tile belongs to instance 0 (T, G <= 256 for n <= 256)
    int zeros[256];
    for (int k = 0; k < 256; ++k) zeros[k] = 0;
    OTM_CUDA(cudaMemcpyAsync(d_tiles, zeros, sizeof(int) * T, cudaMemcpyHostToDevice, st));
    OTM_CUDA(cudaMemcpyAsync(d_gemm, zeros, sizeof(int) * G, cudaMemcpyHostToDevice, st));
    k_noalloc_tables<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(n, C, cosk);

    Inst I;
    std::memset(&I, 0, sizeof(I));
    I.n = n;
    I.tile0 = 0;
    I.ntiles = T;
    I.gemm0 = 0;
    I.ngemm = G;
    double* arr[11];
    for (int k = 0; k < 11; ++k) arr[k] = cells + k * L.npad;
    I.psi[0] = arr[0];
    I.psi[1] = arr[1];
    I.r[0] = arr[2];
    I.r[1] = arr[3];
    I.r[2] = arr[4];
    I.dhat = arr[5];
    I.d[0] = arr[6];
    I.d[1] = arr[7];
    I.rho = arr[8];
    I.t1 = arr[9];
    I.t2 = arr[10];
    I.C = C;
    I.cosk = cosk;

    // the diagonalisation check, once per device and size, in the same array
    bool checked;
    {
      std::lock_guard<std::mutex> lock(g_noalloc_mu);
      checked = g_noalloc_checked[dev][n] != 0;
    }
    if (!checked) {
      Inst P = I;
      P.active = 1;
      P.r[0] = arr[0];   // probe x
      P.dhat = arr[2];   // C^T (lambda o (C X C^T)) C
      k_noalloc_probe<<<(unsigned)((N + 255) / 256), 256, 0, st>>>((long)N, arr[0]);
      k_laplacian_apply<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(n, arr[0], arr[1]);
      OTM_CUDA(cudaMemcpyAsync(d_inst, &P, sizeof(Inst), cudaMemcpyHostToDevice, st));
      for (int s = 0; s < 4; ++s) k_dct_gemm<<<G, 256, 0, st>>>(d_inst, d_gemm, s, 2);
      k_noalloc_maxdiff<<<1, 256, 0, st>>>((long)N, arr[1], arr[2], base + L.check);
      double res[2] = {0, 0};
      OTM_CUDA(cudaMemcpyAsync(res, base + L.check, sizeof(res), cudaMemcpyDeviceToHost, st));
      OTM_CUDA(cudaStreamSynchronize(st));
      double rel = res[1] > 0 ? res[0] / res[1] : res[0];
      if (!(rel <= 1e-10))
        throw BadArg{"otm_solve_noalloc: the cosine basis does not diagonalise the assembled matrix"};
      std::lock_guard<std::mutex> lock(g_noalloc_mu);
      g_noalloc_checked[dev][n] = 1;
    }

    // state that must start at zero: the initial potential, the directions and the
    // residual buffer read as r_{k-1} in the first iteration (the record is rewritten)
    I.max_iter = o.max_iter;
    I.beta_cj = o.beta == OTM_BETA_CONJUGATE_JACOBIAN ? 1 : 0;
    I.threshold = o.threshold;
    I.max_ratio = o.max_ratio;
    OTM_CUDA(cudaMemsetAsync(I.psi[0], 0, N * sizeof(double), st));
    OTM_CUDA(cudaMemsetAsync(I.d[0], 0, N * sizeof(double), st));
    OTM_CUDA(cudaMemsetAsync(I.d[1], 0, N * sizeof(double), st));
    OTM_CUDA(cudaMemsetAsync(I.r[2], 0, N * sizeof(double), st));
    OTM_CUDA(cudaMemcpyAsync(d_inst, &I, sizeof(Inst), cudaMemcpyHostToDevice, st));
    OTM_CUDA(cudaMemcpyAsync(I.rho, density, N * sizeof(double),
                             is_device_ptr(density) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));

    k_density_sum<<<T, NT, 0, st>>>(d_inst, d_tiles, part);
    k_density_scale<<<T, NT, 0, st>>>(d_inst, d_tiles, part);
    k_density_apply<<<T, NT, 0, st>>>(d_inst, d_tiles);
    k_residual_init<<<T, NT, 0, st>>>(d_inst, d_tiles, part);
    OTM_CUDA(cudaGetLastError());
    Inst h;
    int launched = 0;
    while (true) {
      OTM_CUDA(cudaMemcpyAsync(&h, d_inst, sizeof(Inst), cudaMemcpyDeviceToHost, st));
      OTM_CUDA(cudaStreamSynchronize(st));
      if (!h.active || launched >= o.max_iter) break;
      for (int c = 0; c < 4 && launched < o.max_iter; ++c, ++launched) {
        for (int s = 0; s < 4; ++s) k_dct_gemm<<<G, 256, 0, st>>>(d_inst, d_gemm, s, 1);
        k_beta<<<T, NT, 0, st>>>(d_inst, d_tiles, part);
        k_coeffs<<<T, NT, 0, st>>>(d_inst, d_tiles, part);
        k_update<<<T, NT, 0, st>>>(d_inst, d_tiles, part);
      }
      OTM_CUDA(cudaGetLastError());
    }
    bool fdev = is_device_ptr(fwd_xy);
    double* dst = fdev ? fwd_xy : base + L.fwd;
    k_forward_mesh<<<(unsigned)((V + 255) / 256), 256, 0, st>>>(d_inst, 0, dst);
    OTM_CUDA(cudaGetLastError());
    if (!fdev) OTM_CUDA(cudaMemcpyAsync(fwd_xy, dst, sizeof(double) * 2 * V, cudaMemcpyDeviceToHost, st));
    if (adjusted)
      OTM_CUDA(cudaMemcpyAsync(adjusted, I.rho, sizeof(double) * N,
                               is_device_ptr(adjusted) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    OTM_CUDA(cudaStreamSynchronize(st));
    fill_stats(h, stats);
    return (int)OTM_OK;
  });
}
