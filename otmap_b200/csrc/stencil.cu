// The per-iteration stencil work of the solve in two passes over the grid
// (otlib/otsolver_2dgrid.cpp:179-220, 248-261, 467-606):
//
//   k_sweep_sums   reads psi, d_hat, d_prev, r_k, r_{k-1}; per cell the line
//                  coefficients of d_hat (b1, a11) and of d_prev (b2, a22) and their
//                  cross term a12, and 26 partial sums. The last block of an instance
//                  turns them into |d_hat| (early exit, :182), beta (:248-261, with
//                  r(psi - eps d_hat) - r_k = -eps b1 + eps^2 a11, exact for the
//                  quadratic area) and the quartic of the line search for
//                  d = d_hat + beta d_prev (its five sums are polynomials in beta of the
//                  cross sums), then solves the cubic for alpha (:556-595).
//   k_sweep_update reads psi, d_hat, d_prev, r_k; writes d = d_hat + beta d_prev,
//                  psi + alpha d and r_k + alpha b + alpha^2 a (:599-604); the last
//                  block advances the iteration and tests the loop condition (:160).
//
// Geometry: one warp owns a strip of 32 consecutive columns (j, contiguous in memory)
// and SR rows; it walks down the rows keeping two rows of the fields and of their
// vertex gradients in registers. Left/right neighbours come from warp shuffles, the
// strip's two halo columns from two extra loads. A block is 8 strips side by side.
// Per cell the arithmetic is the reference's, in FP64, without FMA contraction.

#include "engine.cuh"

namespace otm {

constexpr int SW = 32;        // strip width (one warp)
constexpr int SR = 16;        // strip height (rows per warp)
constexpr int SWARPS = 8;     // strips per block
constexpr int ST = SW * SWARPS;
constexpr int KA = SWEEP_SLOTS;  // partial-sum slots per block

struct Row {   // one field on one grid row around the lane's column j
  double c;    // column j
  double l;    // column j - 1
  double rh;   // lane 31: column j0 + 32
};

struct VG {    // vertex gradients (v, j) and (v, j + 1)
  double gx, gy, gxr, gyr;
};

__device__ __forceinline__ int clampn(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }

template <class F>
__device__ __forceinline__ Row load_row(F f, int row, int j0, int lane, int n) {
  Row r;
  const size_t base = (size_t)clampn(row, n) * n;
  r.c = f(base + clampn(j0 + lane, n));
  double halo = 0.0;
  if (lane == 0) halo = f(base + clampn(j0 - 1, n));
  if (lane == 31) halo = f(base + clampn(j0 + 32, n));
  double up = __shfl_up_sync(0xffffffffu, r.c, 1);
  r.l = lane == 0 ? halo : up;
  r.rh = halo;
  return r;
}

// Vertex gradients of vertex row v from cell rows a = v-1 and b = v
// (otsolver_2dgrid.cpp:379-391 with clamped cells = boundary rules :405-422).
__device__ __forceinline__ VG vgrad(const Row& a, const Row& b, double hw, int lane) {
  VG g;
  g.gx = hw * ((b.l + b.c) - (a.l + a.c));
  g.gy = hw * ((a.c + b.c) - (a.l + b.l));
  double gxr = __shfl_down_sync(0xffffffffu, g.gx, 1);
  double gyr = __shfl_down_sync(0xffffffffu, g.gy, 1);
  if (lane == 31) {
    gxr = hw * ((b.c + b.rh) - (a.c + a.rh));
    gyr = hw * ((a.rh + b.rh) - (a.c + b.c));
  }
  g.gxr = gxr;
  g.gyr = gyr;
  return g;
}

// Diagonals of the cell between vertex rows p (row c) and q (row c + 1):
// v00 = p.g, v01 = p.gr, v10 = q.g, v11 = q.gr.
struct Diag {
  double ax, ay, bx, by;  // v11 - v00, v01 - v10
};

__device__ __forceinline__ Diag diag(const VG& p, const VG& q) {
  Diag d;
  d.ax = q.gxr - p.gx;
  d.ay = q.gyr - p.gy;
  d.bx = p.gxr - q.gx;
  d.by = p.gyr - q.gy;
  return d;
}

// a(dir) and b(dir; psi) of otsolver_2dgrid.cpp:523-536 from the direction's diagonal
// differences h and the potential's g.
__device__ __forceinline__ void line_ab(const Diag& g, const Diag& h, double e, double& a, double& b) {
  double diag0a_x = g.ax + e;
  double diag0a_y = g.ay + e;
  double diag0b_x = g.bx - e;
  double diag0b_y = g.by + e;
  a = 0.5 * (h.ax * h.by - h.ay * h.bx);
  b = 0.5 * (h.ax * diag0b_y - h.ay * diag0b_x + diag0a_x * h.by - diag0a_y * h.bx);
}

struct StripCoord {
  int i0, j0, lane, warp;
};

__device__ __forceinline__ StripCoord strip_coord(const Inst& I, int block) {
  StripCoord s;
  s.lane = threadIdx.x & 31;
  s.warp = threadIdx.x >> 5;
  const int n = I.n;
  const int cols = (n + SW - 1) / SW;
  const int strip = (block - I.strip0) * SWARPS + s.warp;
  s.i0 = (strip / cols) * SR;
  s.j0 = (strip % cols) * SW;
  return s;
}

template <int K>
__device__ __forceinline__ void write_partials(double (&v)[K], double* red, double* partials, int block) {
  block_sum<K>(v, red);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) partials[(size_t)block * KA + k] = v[k];
}

template <int K>
__device__ __forceinline__ void reduce_block_partials(const double* partials, int b0, int nb, double (&v)[K],
                                                      double* red) {
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = 0.0;
  for (int t = threadIdx.x; t < nb; t += blockDim.x)
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] += __ldcg(&partials[(size_t)(b0 + t) * KA + k]);
  block_sum<K>(v, red);
}

// Sum slots of k_sweep_sums.
enum {
  S_HH, S_HQ, S_QQ,            // |d_hat|^2, d_hat.d_prev, |d_prev|^2
  S_JB, S_JA, S_JJ,            // Jd.b1, Jd.a11, |Jd|^2 with Jd = r_k - r_{k-1}
  S_B1R, S_B2R, S_B1B1, S_B1B2, S_B2B2,
  S_A11R, S_A12R, S_A22R,
  S_A11B1, S_A11B2, S_A12B1, S_A12B2, S_A22B1, S_A22B2,
  S_A11A11, S_A11A12, S_A12A12, S_A11A22, S_A12A22, S_A22A22,
  S_COUNT
};

__global__ __launch_bounds__(ST) void k_sweep_sums(Inst* insts, const int* strip_inst, double* partials) {
  __shared__ double red[32 * S_COUNT];
  Inst& I = insts[strip_inst[blockIdx.x]];
  if (!I.active) return;
  const int n = I.n, it = I.it;
  const double e = 1.0 / (double)n, hw = 0.5 * (double)n;
  const StripCoord sc = strip_coord(I, blockIdx.x);
  const int j = sc.j0 + sc.lane;
  const double* psi = I.psi[it & 1];
  const double* dh = I.dhat;
  const double* dp = I.d[(it + 1) & 1];
  const double* rk = I.r[it % 3];
  const double* rkm1 = I.r[(it + 2) % 3];
  double acc[S_COUNT];
#pragma unroll
  for (int k = 0; k < S_COUNT; ++k) acc[k] = 0.0;
  const bool active_strip = sc.i0 < n;
  if (active_strip) {
    auto P = [&](size_t g) { return psi[g]; };
    auto H = [&](size_t g) { return dh[g]; };
    auto Q = [&](size_t g) { return dp[g]; };
    Row pa = load_row(P, sc.i0 - 1, sc.j0, sc.lane, n), ha = load_row(H, sc.i0 - 1, sc.j0, sc.lane, n),
        qa = load_row(Q, sc.i0 - 1, sc.j0, sc.lane, n);
    Row pb = load_row(P, sc.i0, sc.j0, sc.lane, n), hb = load_row(H, sc.i0, sc.j0, sc.lane, n),
        qb = load_row(Q, sc.i0, sc.j0, sc.lane, n);
    VG gp = vgrad(pa, pb, hw, sc.lane), gh = vgrad(ha, hb, hw, sc.lane), gq = vgrad(qa, qb, hw, sc.lane);
    for (int c = sc.i0; c < sc.i0 + SR && c < n; ++c) {
      // vertex row c + 1 from cell rows c and c + 1
      Row pn = load_row(P, c + 1, sc.j0, sc.lane, n), hn = load_row(H, c + 1, sc.j0, sc.lane, n),
          qn = load_row(Q, c + 1, sc.j0, sc.lane, n);
      VG gp2 = vgrad(pb, pn, hw, sc.lane), gh2 = vgrad(hb, hn, hw, sc.lane), gq2 = vgrad(qb, qn, hw, sc.lane);
      if (j < n) {
        const size_t f = (size_t)c * n + j;
        Diag G = diag(gp, gp2), Hd = diag(gh, gh2), Qd = diag(gq, gq2);
        double a11, b1, a22, b2;
        line_ab(G, Hd, e, a11, b1);
        line_ab(G, Qd, e, a22, b2);
        double a12 = 0.5 * (Hd.ax * Qd.by - Hd.ay * Qd.bx + Qd.ax * Hd.by - Qd.ay * Hd.bx);
        double r = rk[f], jd = r - rkm1[f];
        double hv = hb.c, qv = qb.c;
        acc[S_HH] += hv * hv;
        acc[S_HQ] += hv * qv;
        acc[S_QQ] += qv * qv;
        acc[S_JB] += jd * b1;
        acc[S_JA] += jd * a11;
        acc[S_JJ] += jd * jd;
        acc[S_B1R] += b1 * r;
        acc[S_B2R] += b2 * r;
        acc[S_B1B1] += b1 * b1;
        acc[S_B1B2] += b1 * b2;
        acc[S_B2B2] += b2 * b2;
        acc[S_A11R] += a11 * r;
        acc[S_A12R] += a12 * r;
        acc[S_A22R] += a22 * r;
        acc[S_A11B1] += a11 * b1;
        acc[S_A11B2] += a11 * b2;
        acc[S_A12B1] += a12 * b1;
        acc[S_A12B2] += a12 * b2;
        acc[S_A22B1] += a22 * b1;
        acc[S_A22B2] += a22 * b2;
        acc[S_A11A11] += a11 * a11;
        acc[S_A11A12] += a11 * a12;
        acc[S_A12A12] += a12 * a12;
        acc[S_A11A22] += a11 * a22;
        acc[S_A12A22] += a12 * a22;
        acc[S_A22A22] += a22 * a22;
      }
      pb = pn;
      hb = hn;
      qb = qn;
      gp = gp2;
      gh = gh2;
      gq = gq2;
    }
  }
  write_partials<S_COUNT>(acc, red, partials, blockIdx.x);
  if (last_block(&I.counter, I.nstrip)) {
    double S[S_COUNT];
    reduce_block_partials<S_COUNT>(partials, I.strip0, I.nstrip, S, red);
    if (threadIdx.x == 0) {
      if (sqrt(S[S_HH]) <= 2.0 * DBL_MIN) {  // otsolver_2dgrid.cpp:182
        I.active = 0;
        I.outcome = OTM_SMALL_STEP;
      } else {
        const bool use_beta = it >= 1 && I.beta_cj;
        I.use_beta = use_beta ? 1 : 0;
        if (use_beta) {
          const double alpha = I.alpha, eps = alpha / 2.0;
          const double num = -eps * S[S_JB] + eps * eps * S[S_JA];
          I.beta = std_max(-1.0, num / S[S_JJ] / eps * alpha);
        }
        const double B = use_beta ? I.beta : 0.0, B2 = B * B, B3 = B2 * B, B4 = B2 * B2;
        const double sbr = S[S_B1R] + B * S[S_B2R];
        const double sbb = S[S_B1B1] + 2.0 * B * S[S_B1B2] + B2 * S[S_B2B2];
        const double sar = S[S_A11R] + B * S[S_A12R] + B2 * S[S_A22R];
        const double sab = S[S_A11B1] + B * (S[S_A11B2] + S[S_A12B1]) + B2 * (S[S_A12B2] + S[S_A22B1]) +
                           B3 * S[S_A22B2];
        const double saa = S[S_A11A11] + 2.0 * B * S[S_A11A12] + B2 * (S[S_A12A12] + 2.0 * S[S_A11A22]) +
                           2.0 * B3 * S[S_A12A22] + B4 * S[S_A22A22];
        const double ea = 1.0 / ((double)n * (double)n);
        double z[5] = {I.residual * ea, 2.0 * sbr, sbb + 2 * sar, 2.0 * sab, saa};
        double alpha, rmin;
        pick_step(z, &alpha, &rmin);
        I.alpha = alpha;
        I.residual = rmin / ea;
        I.dnorm = sqrt(std_max(0.0, S[S_HH] + 2.0 * B * S[S_HQ] + B2 * S[S_QQ]));
      }
    }
  }
}

__global__ __launch_bounds__(ST) void k_sweep_update(Inst* insts, const int* strip_inst, double* partials) {
  __shared__ double red[32];
  Inst& I = insts[strip_inst[blockIdx.x]];
  if (!I.active) return;
  const int n = I.n, it = I.it;
  const double e = 1.0 / (double)n, hw = 0.5 * (double)n, alpha = I.alpha;
  const bool use_beta = I.use_beta;
  const double beta = I.beta;
  const StripCoord sc = strip_coord(I, blockIdx.x);
  const int j = sc.j0 + sc.lane;
  const double* psi = I.psi[it & 1];
  const double* dh = I.dhat;
  const double* dp = I.d[(it + 1) & 1];
  const double* rk = I.r[it % 3];
  double* dnew = I.d[it & 1];
  double* psin = I.psi[(it + 1) & 1];
  double* rn = I.r[(it + 1) % 3];
  double mx = -INFINITY;
  if (sc.i0 < n) {
    auto P = [&](size_t g) { return psi[g]; };
    auto D = [&](size_t g) { return use_beta ? dh[g] + beta * dp[g] : dh[g]; };
    Row pa = load_row(P, sc.i0 - 1, sc.j0, sc.lane, n), da = load_row(D, sc.i0 - 1, sc.j0, sc.lane, n);
    Row pb = load_row(P, sc.i0, sc.j0, sc.lane, n), db = load_row(D, sc.i0, sc.j0, sc.lane, n);
    VG gp = vgrad(pa, pb, hw, sc.lane), gd = vgrad(da, db, hw, sc.lane);
    for (int c = sc.i0; c < sc.i0 + SR && c < n; ++c) {
      Row pn = load_row(P, c + 1, sc.j0, sc.lane, n), dn = load_row(D, c + 1, sc.j0, sc.lane, n);
      VG gp2 = vgrad(pb, pn, hw, sc.lane), gd2 = vgrad(db, dn, hw, sc.lane);
      if (j < n) {
        const size_t f = (size_t)c * n + j;
        double a, b;
        line_ab(diag(gp, gp2), diag(gd, gd2), e, a, b);
        dnew[f] = db.c;
        psin[f] = pb.c + alpha * db.c;
        double r = a * (alpha * alpha) + b * alpha + rk[f];
        rn[f] = r;
        mx = fmax(mx, r);
      }
      pb = pn;
      db = dn;
      gp = gp2;
      gd = gd2;
    }
  }
  mx = block_max(mx, red);
  if (threadIdx.x == 0) partials[(size_t)blockIdx.x * KA] = mx;
  if (last_block(&I.counter, I.nstrip)) {
    double m = -INFINITY;
    for (int t = threadIdx.x; t < I.nstrip; t += blockDim.x)
      m = fmax(m, __ldcg(&partials[(size_t)(I.strip0 + t) * KA]));
    m = block_max(m, red);
    if (threadIdx.x == 0) {
      I.linf = m / (1.0 / ((double)n * (double)n));
      I.it = it + 1;
      I.active = (I.it < I.max_iter && I.residual > I.threshold) ? 1 : 0;
      if (!I.active) stop_outcome(I);
    }
  }
}

int strip_blocks(int n) {
  const int strips = ((n + SR - 1) / SR) * ((n + SW - 1) / SW);
  return (strips + SWARPS - 1) / SWARPS;
}

void sweep_sums(otm_context* ctx, Inst* d_insts, const int* strip_inst, int nblocks, double* partials) {
  launch(ctx, "sweep_sums", k_sweep_sums, nblocks, ST, d_insts, strip_inst, partials);
}

void sweep_update(otm_context* ctx, Inst* d_insts, const int* strip_inst, int nblocks, double* partials) {
  launch(ctx, "sweep_update", k_sweep_update, nblocks, ST, d_insts, strip_inst, partials);
}

}  // namespace otm
