// The per-iteration stencil work of the solve in two passes over the grid
// (otlib/otsolver_2dgrid.cpp:179-220, 248-261, 467-606):
//
//   k_sweep_sums   reads psi, d_hat, d_prev, r_k, r_{k-1}; per cell the line
//                  coefficients of d_hat (b1, a11) and of d_prev (b2, a22) and their
//                  cross term a12, and 23 partial sums. The last block of an instance
//                  turns them into |d_hat| (early exit, :182), beta (:248-261, with
//                  r(psi - eps d_hat) - r_k = -eps b1 + eps^2 a11, exact for the
//                  quadratic area) and the quartic of the line search for
//                  d = d_hat + beta d_prev (its five sums are polynomials in beta of the
//                  cross sums), then solves the cubic for alpha (:556-595).
//   k_sweep_update reads psi, d_hat, d_prev, r_k; writes d = d_hat + beta d_prev,
//                  psi + alpha d and r_k + alpha b + alpha^2 a (:599-604); the last
//                  block advances the iteration and tests the loop condition (:160).
//
// Geometry: one warp owns a strip of 32 consecutive columns (j, contiguous in memory) and
// Inst::srows rows (32; 64 when the batch has strips to spare, 16 when it has too few to
// fill the SMs) and walks down it. Grid rows are prefetched asynchronously (cp.async) into
// a per-warp ring of RD rows in shared memory, so RD-2 rows per warp are in flight while
// it computes; the previous vertex-gradient row is kept in registers. The strip's two halo
// columns are staged with the row; neighbours come from the ring. A block is SWARPS strips
// side by side.
// Per cell the arithmetic is the reference's, in FP64, without FMA contraction.

#include "engine.cuh"

namespace otm {

constexpr int SW = 32;        // strip width (one warp)
// strip height (rows per warp): Inst::srows, 16, 32 or 64 per batch (layout_workspace)
constexpr int SWARPS = 4;     // strips per block
constexpr int ST = SW * SWARPS;
constexpr int KA = SWEEP_SLOTS;  // partial-sum slots per block
constexpr int RD = 8;         // rows in the per-warp prefetch ring (RD - 3 in flight beyond the two in use)
static_assert((RD & (RD - 1)) == 0, "the ring depth is a power of two");

__device__ __forceinline__ int clampn(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }

struct Row {   // one field on one grid row around the lane's column j
  double c;    // column j
  double l;    // column j - 1
  double r;    // column j + 1
};

// ---- per-warp asynchronous row prefetch (cp.async) ----
// A stage holds one grid row of the strip for every field: stencil fields take 36
// slots (columns j0-2 .. j0+33; slot 1 + lane is column j - 1), pointwise fields 32
// (columns j0 .. j0+31). Interior strips (j0 >= 2, j0 + 34 <= n, n even) copy a stencil
// row with one 16-byte cp.async on 18 lanes (16 column pairs and the two halo pairs) and
// a pointwise row on 16 lanes; edge strips and odd n use 8-byte copies with clamped
// columns (the reference's boundary cells).

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(double* dst, const double* src) {
  unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int NS, int NP>
struct Ring {
  static constexpr int SS = 36;  // slots of a stencil field row
  static constexpr int STAGE = NS * SS + NP * 32;
  static constexpr int STAGE_BYTES = STAGE * 8;
  double* buf;  // RD * STAGE doubles (this warp's)
  const double* sf[NS > 0 ? NS : 1];
  const double* pf[NP > 0 ? NP : 1];
  int n, j0, lane, rows_end;  // rows beyond rows_end are not fetched
  bool interior;              // 16-byte copies (warp-uniform)
  int soff, gcol;             // this lane's stencil slot and global column (interior copies)

  // the sweeps' fields: psi, d_hat, d_prev; r_k (, r_{k-1})
  __device__ __forceinline__ void bind(const Inst& I, int it) {
    sf[0] = I.psi[it & 1];
    sf[1] = I.dhat;
    sf[2] = I.d[(it + 1) & 1];
    pf[0] = I.r[it % 3];
    if constexpr (NP > 1) pf[1] = I.r[(it + 2) % 3];
  }
  __device__ __forceinline__ void setup() {
    interior = (j0 >= 2) && (j0 + 34 <= n) && ((n & 1) == 0);
    soff = lane < 16 ? 2 + 2 * lane : (lane == 16 ? 0 : 34);
    gcol = lane < 16 ? j0 + 2 * lane : (lane == 16 ? j0 - 2 : j0 + 32);
  }

  // RD is a power of two and row >= -1, so the stage index is a mask of row + RD
  __device__ __forceinline__ double* stage(int row) { return buf + ((unsigned)(row + RD) & (RD - 1u)) * STAGE; }

  // Queues the copies of grid row `row` (clamped) and commits them as one group.
  __device__ __forceinline__ void issue(int row) {
    if (row <= rows_end) {
      double* st = stage(row);
      const size_t base = (size_t)clampn(row, n) * n;
      if (interior) {
        if (lane < 18) {
#pragma unroll
          for (int k = 0; k < NS; ++k) cp_async16(st + k * SS + soff, sf[k] + base + gcol);
        }
        if (lane < 16) {
#pragma unroll
          for (int k = 0; k < NP; ++k) cp_async16(st + NS * SS + k * 32 + 2 * lane, pf[k] + base + j0 + 2 * lane);
        }
      } else {
        const size_t cj = base + clampn(j0 + lane, n);
#pragma unroll
        for (int k = 0; k < NS; ++k) {
          double* d = st + k * SS;
          cp_async8(d + 2 + lane, sf[k] + cj);
          if (lane == 0) cp_async8(d + 1, sf[k] + base + clampn(j0 - 1, n));
          if (lane == 31) cp_async8(d + 34, sf[k] + base + clampn(j0 + 32, n));
        }
#pragma unroll
        for (int k = 0; k < NP; ++k) cp_async8(st + NS * SS + k * 32 + lane, pf[k] + cj);
      }
    }
    cp_async_commit();
  }
  __device__ __forceinline__ Row row_of(int row, int k) {
    const double* d = stage(row) + k * SS;
    Row r;
    r.c = d[2 + lane];
    r.l = d[1 + lane];
    r.r = d[3 + lane];
    return r;
  }
  __device__ __forceinline__ double point(int row, int k) { return stage(row)[NS * SS + k * 32 + lane]; }
};

struct VG {    // vertex gradients (v, j) and (v, j + 1)
  double gx, gy, gxr, gyr;
};

// Vertex gradients of vertex row v at columns j and j+1 from cell rows a = v-1 and
// b = v (otsolver_2dgrid.cpp:379-391 with clamped cells = boundary rules :405-422),
// divided by the reference's factor n/2: the sweeps carry that factor into the line
// coefficients (a, b scale by (n/2)^2) and apply it to the sums and the residual
// update. For power-of-two n the factor is a power of two and every result is
// bit-identical to scaling each gradient. The gradient at j+1 is the expression lane j+1
// evaluates for its own vertex, formed here from the staged column j+1.
__device__ __forceinline__ VG vgrad(const Row& a, const Row& b) {
  VG g;
  const double sc = a.c + b.c;
  g.gx = (b.l + b.c) - (a.l + a.c);
  g.gy = sc - (a.l + b.l);
  g.gxr = (b.c + b.r) - (a.c + a.r);
  g.gyr = (a.r + b.r) - sc;
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

// 2a(dir) and 2b(dir; psi) of otsolver_2dgrid.cpp:523-536 from the direction's diagonal
// differences h and the potential's g (the reference's factor 1/2 is applied, exactly,
// with the (n/2)^2 scale).
__device__ __forceinline__ void line_ab(const Diag& g, const Diag& h, double e, double& a, double& b) {
  double diag0a_x = g.ax + e;
  double diag0a_y = g.ay + e;
  double diag0b_x = g.bx - e;
  double diag0b_y = g.by + e;
  a = h.ax * h.by - h.ay * h.bx;
  b = h.ax * diag0b_y - h.ay * diag0b_x + diag0a_x * h.by - diag0a_y * h.bx;
}

// The split form's line coefficients with fused multiply-adds (no reference rounding to
// retrace there): g0 holds the potential's shifted diagonals (g.ax + e, g.ay + e,
// g.bx - e, g.by + e), h the direction's diagonals.
__device__ __forceinline__ Diag shift_diag(const Diag& g, double e) {
  Diag d;
  d.ax = g.ax + e;
  d.ay = g.ay + e;
  d.bx = g.bx - e;
  d.by = g.by + e;
  return d;
}
__device__ __forceinline__ void line_ab_fma(const Diag& g0, const Diag& h, double& a, double& b) {
  a = fma(h.ax, h.by, -(h.ay * h.bx));
  b = fma(h.ax, g0.by, fma(-h.ay, g0.bx, fma(g0.ax, h.by, -(g0.ay * h.bx))));
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
  s.i0 = (strip / cols) * I.srows;
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
  S_AB0, S_AB1, S_AB2, S_AB3,  // sum a(beta) b(beta) by powers of beta: a11b1, a11b2+a12b1, a12b2+a22b1, a22b2
  S_AA0, S_AA1, S_AA2, S_AA3, S_AA4,  // a11^2, a11a12, a12^2+2a11a22, a12a22, a22^2
  S_COUNT
};

// Last block of an instance in the sum sweep (thread 0): restores the factor (n/2)^2 / 2
// of the line coefficients in the sums, then the early exit (otsolver_2dgrid.cpp:182),
// beta (:248-261) and the step alpha of the quartic for d = d_hat + beta d_prev (:541-606).
__device__ __forceinline__ void sums_step(Inst& I, double (&S)[S_COUNT], int n, int it) {
  const double hw = 0.5 * (double)n;
  const double h2 = 0.5 * hw * hw, h4 = h2 * h2;
  S[S_JB] *= h2;
  S[S_JA] *= h2;
  S[S_B1R] *= h2;
  S[S_B2R] *= h2;
  S[S_A11R] *= h2;
  S[S_A12R] *= h2;
  S[S_A22R] *= h2;
#pragma unroll
  for (int k = S_B1B1; k <= S_B2B2; ++k) S[k] *= h4;
#pragma unroll
  for (int k = S_AB0; k < S_COUNT; ++k) S[k] *= h4;
  if (sqrt(S[S_HH]) <= 2.0 * DBL_MIN) {  // otsolver_2dgrid.cpp:182
    I.active = 0;
    I.outcome = OTM_SMALL_STEP;
    return;
  }
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
  const double sab = S[S_AB0] + B * S[S_AB1] + B2 * S[S_AB2] + B3 * S[S_AB3];
  const double saa = S[S_AA0] + 2.0 * B * S[S_AA1] + B2 * S[S_AA2] + 2.0 * B3 * S[S_AA3] + B4 * S[S_AA4];
  const double ea = 1.0 / ((double)n * (double)n);
  double z[5] = {I.residual * ea, 2.0 * sbr, sbb + 2 * sar, 2.0 * sab, saa};
  double alpha, rmin;
  pick_step(z, &alpha, &rmin);
  I.alpha = alpha;
  I.residual = rmin / ea;
  I.dnorm = sqrt(std_max(0.0, S[S_HH] + 2.0 * B * S[S_HQ] + B2 * S[S_QQ]));
}

// Last block of an instance in the update sweep (thread 0): the max residual, the
// iteration count and the loop test (otsolver_2dgrid.cpp:160).
__device__ __forceinline__ void update_step(Inst& I, double rmax, int n, int it) {
  I.linf = rmax / (1.0 / ((double)n * (double)n));
  I.it = it + 1;
  I.active = (I.it < I.max_iter && I.residual > I.threshold) ? 1 : 0;
  if (!I.active) stop_outcome(I);
}

// ---- split precision (OTM_PRECISION_SPLIT) ----
//
// r_k, r_{k-1}, d_hat and d are stored in FP32 (psi stays FP64): the sweeps move 24 and
// 36 bytes per cell instead of 40 and 56. The per-cell arithmetic stays FP64: the staged
// FP32 values are converted exactly when read, so the line coefficients a, b are exact
// for the directions the update applies and the line search's tracked residual stays
// that of the stored residual. (Forming the directions' vertex gradients and diagonals in
// FP32 is not enough: they are second differences of smooth fields, and the cancellation
// left about 1e-4 relative error in a and b; at 1024^2 the tracked residual then drifted
// away from the mesh's, solves stopped 5e-3 away from the reference's map or ran to
// max_iter.) d and r' are rounded to FP32 when stored; psi' = psi + alpha d uses the
// unrounded d, as do a and b of the update. Having no reference rounding to retrace, the
// split form fuses its multiply-adds (line coefficients, d, psi', r').

__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16v(void* dst, const void* src) {
  unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(src) : "memory");
}

// Prefetch ring of the split form: the FP64 potential (36 doubles as in Ring), two FP32
// stencil fields d_hat, d_prev (40 floats: columns j0-4 .. j0+35, slot 4 + lane is column
// j) and NP FP32 pointwise fields r_k (, r_{k-1}) (32 floats). Interior strips (j0 >= 4,
// j0 + 36 <= n, n a multiple of 4) copy with 16-byte cp.async (18 lanes for the FP64 row,
// 10 per FP32 stencil row, 8 per pointwise row); edge strips copy element-wise with
// clamped columns. Reads return FP64 rows and values, as Ring's do.
template <int NP>
struct RingS {
  static constexpr int NS = 2, PD = 36, FS = 40, FP = 32;
  static constexpr int STAGE_BYTES = PD * 8 + NS * FS * 4 + NP * FP * 4;
  static_assert(STAGE_BYTES % 16 == 0, "stages stay 16-byte aligned");
  unsigned char* buf;  // RD * STAGE_BYTES (this warp's)
  const double* psi;
  const float* sf[NS];
  const float* pf[NP];
  int n, j0, lane, rows_end;
  bool interior;
  int soff, gcol;  // this lane's FP64 slot and column (interior copies)

  __device__ __forceinline__ void bind(const Inst& I, int it) {
    psi = I.psi[it & 1];
    sf[0] = reinterpret_cast<const float*>(I.dhat);
    sf[1] = reinterpret_cast<const float*>(I.d[(it + 1) & 1]);
    pf[0] = reinterpret_cast<const float*>(I.r[it % 3]);
    if constexpr (NP > 1) pf[1] = reinterpret_cast<const float*>(I.r[(it + 2) % 3]);
  }
  __device__ __forceinline__ void setup() {
    interior = (j0 >= 4) && (j0 + 36 <= n) && ((n & 3) == 0);
    soff = lane < 16 ? 2 + 2 * lane : (lane == 16 ? 0 : 34);
    gcol = lane < 16 ? j0 + 2 * lane : (lane == 16 ? j0 - 2 : j0 + 32);
  }
  __device__ __forceinline__ unsigned char* stage(int row) {
    return buf + ((unsigned)(row + RD) & (RD - 1u)) * STAGE_BYTES;
  }
  __device__ __forceinline__ double* pstage(int row) { return reinterpret_cast<double*>(stage(row)); }
  __device__ __forceinline__ float* fstage(int row, int k) {
    return reinterpret_cast<float*>(stage(row) + PD * 8) + k * FS;
  }
  __device__ __forceinline__ float* ptstage(int row, int k) {
    return reinterpret_cast<float*>(stage(row) + PD * 8 + NS * FS * 4) + k * FP;
  }
  __device__ __forceinline__ void issue(int row) {
    if (row <= rows_end) {
      double* sp = pstage(row);
      const size_t base = (size_t)clampn(row, n) * n;
      if (interior) {
        if (lane < 18) cp_async16v(sp + soff, psi + base + gcol);
        if (lane < 10) {
#pragma unroll
          for (int k = 0; k < NS; ++k) cp_async16v(fstage(row, k) + 4 * lane, sf[k] + base + j0 - 4 + 4 * lane);
        }
        if (lane < 8) {
#pragma unroll
          for (int k = 0; k < NP; ++k) cp_async16v(ptstage(row, k) + 4 * lane, pf[k] + base + j0 + 4 * lane);
        }
      } else {
        const size_t cj = base + clampn(j0 + lane, n);
        cp_async8(sp + 2 + lane, psi + cj);
        if (lane == 0) cp_async8(sp + 1, psi + base + clampn(j0 - 1, n));
        if (lane == 31) cp_async8(sp + 34, psi + base + clampn(j0 + 32, n));
#pragma unroll
        for (int k = 0; k < NS; ++k) {
          float* d = fstage(row, k);
          cp_async4(d + 4 + lane, sf[k] + cj);
          if (lane == 0) cp_async4(d + 3, sf[k] + base + clampn(j0 - 1, n));
          if (lane == 31) cp_async4(d + 36, sf[k] + base + clampn(j0 + 32, n));
        }
#pragma unroll
        for (int k = 0; k < NP; ++k) cp_async4(ptstage(row, k) + lane, pf[k] + cj);
      }
    }
    cp_async_commit();
  }
  // field 0: the potential; fields 1, 2: d_hat, d_prev (converted to FP64, exactly)
  __device__ __forceinline__ Row row_of(int row, int k) {
    Row r;
    if (k == 0) {
      const double* d = pstage(row);
      r.c = d[2 + lane];
      r.l = d[1 + lane];
      r.r = d[3 + lane];
    } else {
      const float* d = fstage(row, k - 1);
      r.c = (double)d[4 + lane];
      r.l = (double)d[3 + lane];
      r.r = (double)d[5 + lane];
    }
    return r;
  }
  __device__ __forceinline__ double point(int row, int k) { return (double)ptstage(row, k)[lane]; }
};

// The two sweeps over a ring type: Ring<3, NP> (every field FP64) or RingS<NP> (split
// precision: FP32 storage of r, d_hat, d; FP64 arithmetic).
template <class RT, bool SPLIT>
__global__ __launch_bounds__(ST) void k_sweep_sums_t(Inst* insts, const int* strip_inst, int base, double* partials) {
  extern __shared__ __align__(16) unsigned char ring_raw[];
  __shared__ double red[32 * S_COUNT];
  const int blk = base + blockIdx.x;
  Inst& I = insts[strip_inst[blk]];
  if (!I.active) return;
  const int n = I.n, it = I.it;
  // gradients are unscaled (vgrad): the shift e of the diagonals becomes e / (n/2)
  const double hw = 0.5 * (double)n, es = (1.0 / (double)n) / hw;
  const StripCoord sc = strip_coord(I, blk);
  const int j = sc.j0 + sc.lane;
  double acc[S_COUNT];
#pragma unroll
  for (int k = 0; k < S_COUNT; ++k) acc[k] = 0.0;
  if (sc.i0 < n) {
    RT R;
    R.buf = reinterpret_cast<decltype(R.buf)>(ring_raw + (size_t)sc.warp * RD * RT::STAGE_BYTES);
    R.bind(I, it);
    R.n = n;
    R.j0 = sc.j0;
    R.lane = sc.lane;
    const int last = min(sc.i0 + I.srows, n);  // cell rows i0 .. last-1; grid rows i0-1 .. last
    R.rows_end = last;
    R.setup();
#pragma unroll
    for (int k = 0; k < RD - 1; ++k) R.issue(sc.i0 - 1 + k);
    VG gp, gh, gq;
#pragma unroll 2
    for (int row = sc.i0; row <= last; ++row) {
      cp_async_wait<RD - 3>();
      __syncwarp();
      // grid row row-1 is still in the ring: read again rather than carried in registers
      const Row ap = R.row_of(row - 1, 0), ah = R.row_of(row - 1, 1), aq = R.row_of(row - 1, 2);
      const Row bp = R.row_of(row, 0), bh = R.row_of(row, 1), bq = R.row_of(row, 2);
      // vertex row `row` from grid rows row-1 and row
      VG np = vgrad(ap, bp);
      VG nh = vgrad(ah, bh);
      VG nq = vgrad(aq, bq);
      if (row > sc.i0 && j < n) {
        const int c = row - 1;
        Diag G = diag(gp, np), Hd = diag(gh, nh), Qd = diag(gq, nq);
        double a11, b1, a22, b2, a12;
        if constexpr (SPLIT) {
          const Diag G0 = shift_diag(G, es);
          line_ab_fma(G0, Hd, a11, b1);
          line_ab_fma(G0, Qd, a22, b2);
          a12 = fma(Hd.ax, Qd.by, fma(-Hd.ay, Qd.bx, fma(Qd.ax, Hd.by, -(Qd.ay * Hd.bx))));
        } else {
          line_ab(G, Hd, es, a11, b1);
          line_ab(G, Qd, es, a22, b2);
          a12 = Hd.ax * Qd.by - Hd.ay * Qd.bx + Qd.ax * Hd.by - Qd.ay * Hd.bx;
        }
        double r = R.point(c, 0), jd = r - R.point(c, 1);
        double hv = ah.c, qv = aq.c;
        acc[S_HH] = fma(hv, hv, acc[S_HH]);
        acc[S_HQ] = fma(hv, qv, acc[S_HQ]);
        acc[S_QQ] = fma(qv, qv, acc[S_QQ]);
        acc[S_JB] = fma(jd, b1, acc[S_JB]);
        acc[S_JA] = fma(jd, a11, acc[S_JA]);
        acc[S_JJ] = fma(jd, jd, acc[S_JJ]);
        acc[S_B1R] = fma(b1, r, acc[S_B1R]);
        acc[S_B2R] = fma(b2, r, acc[S_B2R]);
        acc[S_B1B1] = fma(b1, b1, acc[S_B1B1]);
        acc[S_B1B2] = fma(b1, b2, acc[S_B1B2]);
        acc[S_B2B2] = fma(b2, b2, acc[S_B2B2]);
        acc[S_A11R] = fma(a11, r, acc[S_A11R]);
        acc[S_A12R] = fma(a12, r, acc[S_A12R]);
        acc[S_A22R] = fma(a22, r, acc[S_A22R]);
        acc[S_AB0] = fma(a11, b1, acc[S_AB0]);
        acc[S_AB1] = fma(a11, b2, fma(a12, b1, acc[S_AB1]));
        acc[S_AB2] = fma(a12, b2, fma(a22, b1, acc[S_AB2]));
        acc[S_AB3] = fma(a22, b2, acc[S_AB3]);
        acc[S_AA0] = fma(a11, a11, acc[S_AA0]);
        acc[S_AA1] = fma(a11, a12, acc[S_AA1]);
        acc[S_AA2] = fma(a12, a12, fma(a11 + a11, a22, acc[S_AA2]));
        acc[S_AA3] = fma(a12, a22, acc[S_AA3]);
        acc[S_AA4] = fma(a22, a22, acc[S_AA4]);
      }
      gp = np;
      gh = nh;
      gq = nq;
      __syncwarp();
      R.issue(row - 2 + RD);  // refill the stage of grid row row-2, no longer needed
    }
    cp_async_wait<0>();
  }
  write_partials<S_COUNT>(acc, red, partials, blk);
  if (last_block(&I.counter, I.nstrip)) {
    double S[S_COUNT];
    reduce_block_partials<S_COUNT>(partials, I.strip0, I.nstrip, S, red);
    if (threadIdx.x == 0) sums_step(I, S, n, it);
  }
}

template <class RT, bool SPLIT>
__global__ __launch_bounds__(ST) void k_sweep_update_t(Inst* insts, const int* strip_inst, int base,
                                                       double* partials) {
  extern __shared__ __align__(16) unsigned char ring_raw[];
  __shared__ double red[32];
  const int blk = base + blockIdx.x;
  Inst& I = insts[strip_inst[blk]];
  if (!I.active) return;
  const int n = I.n, it = I.it;
  const double hw = 0.5 * (double)n, es = (1.0 / (double)n) / hw, h2 = 0.5 * hw * hw, alpha = I.alpha;
  const bool use_beta = I.use_beta;
  const double beta = I.beta;
  const StripCoord sc = strip_coord(I, blk);
  const int j = sc.j0 + sc.lane;
  double* psin = I.psi[(it + 1) & 1];
  double mx = -INFINITY;
  if (sc.i0 < n) {
    RT R;
    R.buf = reinterpret_cast<decltype(R.buf)>(ring_raw + (size_t)sc.warp * RD * RT::STAGE_BYTES);
    R.bind(I, it);
    R.n = n;
    R.j0 = sc.j0;
    R.lane = sc.lane;
    const int last = min(sc.i0 + I.srows, n);
    R.rows_end = last;
    R.setup();
#pragma unroll
    for (int k = 0; k < RD - 1; ++k) R.issue(sc.i0 - 1 + k);
    // d = d_hat + beta d_prev, formed from the staged rows exactly as the reference
    // forms the vector d before its gradients (otsolver_2dgrid.cpp:199)
    auto drow = [&](int row) {
      Row h = R.row_of(row, 1);
      if (!use_beta) return h;
      Row q = R.row_of(row, 2);
      Row d;
      if constexpr (SPLIT) {
        d.c = fma(beta, q.c, h.c);
        d.l = fma(beta, q.l, h.l);
        d.r = fma(beta, q.r, h.r);
      } else {
        d.c = h.c + beta * q.c;
        d.l = h.l + beta * q.l;
        d.r = h.r + beta * q.r;
      }
      return d;
    };
    // cell row c between vertex rows with gradients (pp, pd) and (qp, qd); pr, dr: grid
    // row c of psi and of d
    auto cell = [&](const VG& pp, const VG& pd, const VG& qp, const VG& qd, const Row& pr, const Row& dr, int c) {
      const size_t f = (size_t)c * n + j;
      double a, b, r;
      if constexpr (SPLIT) {
        line_ab_fma(shift_diag(diag(pp, qp), es), diag(pd, qd), a, b);
        psin[f] = fma(alpha, dr.c, pr.c);
        r = fma(h2, fma(a, alpha * alpha, b * alpha), R.point(c, 0));
      } else {
        line_ab(diag(pp, qp), diag(pd, qd), es, a, b);
        psin[f] = pr.c + alpha * dr.c;
        // (n/2)^2 / 2 (a alpha^2 + b alpha) = a_ref alpha^2 + b_ref alpha, exactly for power-of-two n
        r = h2 * (a * (alpha * alpha) + b * alpha) + R.point(c, 0);
      }
      if constexpr (SPLIT) {
        reinterpret_cast<float*>(I.d[it & 1])[f] = (float)dr.c;
        const float rf = (float)r;
        reinterpret_cast<float*>(I.r[(it + 1) % 3])[f] = rf;
        r = (double)rf;
      } else {
        I.d[it & 1][f] = dr.c;
        I.r[(it + 1) % 3][f] = r;
      }
      mx = fmax(mx, r);
    };
    VG gp, gd;
    Row pc, dc;  // grid row row-1 of psi and of d, carried from the previous step
    int row = sc.i0;
    // split form: two vertex rows per step, their gradients and cells independent chains
    // issued after one wait (grid rows row-1 .. row+1 staged); 128 registers, four blocks
    // per SM (one row per step with the loop unrolled: 142, three blocks; 102 -> 85 us at
    // 8 x 1024^2). The FP64 form keeps one row per step (its two-row form measured slower).
#pragma unroll 1
    for (; SPLIT && row + 1 <= last; row += 2) {
      cp_async_wait<RD - 4>();
      __syncwarp();
      if (row == sc.i0) {
        pc = R.row_of(row - 1, 0);
        dc = drow(row - 1);
      }
      const Row pb = R.row_of(row, 0), db = drow(row);
      const Row pn = R.row_of(row + 1, 0), dn = drow(row + 1);
      const VG mp = vgrad(pc, pb), md = vgrad(dc, db);
      const VG np = vgrad(pb, pn), nd = vgrad(db, dn);
      if (j < n) {
        if (row > sc.i0) cell(gp, gd, mp, md, pc, dc, row - 1);
        cell(mp, md, np, nd, pb, db, row);
      }
      gp = np;
      gd = nd;
      pc = pn;
      dc = dn;
      __syncwarp();
      R.issue(row - 2 + RD);
      R.issue(row - 1 + RD);
    }
    // one row per step: every row of the FP64 form, the odd last row of the split form
    auto one_row = [&](int row) {
      cp_async_wait<RD - 3>();
      __syncwarp();
      if (row == sc.i0) {
        pc = R.row_of(row - 1, 0);
        dc = drow(row - 1);
      }
      const Row pb = R.row_of(row, 0), db = drow(row);
      const VG np = vgrad(pc, pb), nd = vgrad(dc, db);
      if (row > sc.i0 && j < n) cell(gp, gd, np, nd, pc, dc, row - 1);
      gp = np;
      gd = nd;
      pc = pb;
      dc = db;
      __syncwarp();
      R.issue(row - 2 + RD);
    };
    if constexpr (SPLIT) {
      if (row <= last) one_row(row);
    } else {
#pragma unroll 4
      for (; row <= last; ++row) one_row(row);
    }
    cp_async_wait<0>();
  }
  mx = block_max(mx, red);
  if (threadIdx.x == 0) partials[(size_t)blk * KA] = mx;
  if (last_block(&I.counter, I.nstrip)) {
    double m = -INFINITY;
    for (int t = threadIdx.x; t < I.nstrip; t += blockDim.x)
      m = fmax(m, __ldcg(&partials[(size_t)(I.strip0 + t) * KA]));
    m = block_max(m, red);
    if (threadIdx.x == 0) update_step(I, m, n, it);
  }
}

int strip_blocks(int n, int srows) {
  const int strips = ((n + srows - 1) / srows) * ((n + SW - 1) / SW);
  return (strips + SWARPS - 1) / SWARPS;
}

using SumsF64 = Ring<3, 2>;
using UpdF64 = Ring<3, 1>;
using SumsSplit = RingS<2>;
using UpdSplit = RingS<1>;

void sweep_attrs(int device) {
  static bool done[64] = {};
  if (device < 64 && done[device]) return;
  OTM_CUDA(cudaFuncSetAttribute(k_sweep_sums_t<SumsF64, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                SWARPS * RD * SumsF64::STAGE_BYTES));
  OTM_CUDA(cudaFuncSetAttribute(k_sweep_update_t<UpdF64, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                SWARPS * RD * UpdF64::STAGE_BYTES));
  OTM_CUDA(cudaFuncSetAttribute(k_sweep_sums_t<SumsSplit, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                SWARPS * RD * SumsSplit::STAGE_BYTES));
  OTM_CUDA(cudaFuncSetAttribute(k_sweep_update_t<UpdSplit, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                SWARPS * RD * UpdSplit::STAGE_BYTES));
  if (device < 64) done[device] = true;
}

void sweep_sums(otm_context* ctx, Inst* d_insts, const int* strip_inst, int base, int nblocks, bool split,
                double* partials) {
  sweep_attrs(ctx->device);
  if (nblocks <= 0) return;
  if (split)
    launch_smem(ctx, "sweep32_sums", k_sweep_sums_t<SumsSplit, true>, nblocks, ST, SWARPS * RD * SumsSplit::STAGE_BYTES,
                d_insts, strip_inst, base, partials);
  else
    launch_smem(ctx, "sweep_sums", k_sweep_sums_t<SumsF64, false>, nblocks, ST, SWARPS * RD * SumsF64::STAGE_BYTES,
                d_insts, strip_inst, base, partials);
}

void sweep_update(otm_context* ctx, Inst* d_insts, const int* strip_inst, int base, int nblocks, bool split,
                  double* partials) {
  sweep_attrs(ctx->device);
  if (nblocks <= 0) return;
  if (split)
    launch_smem(ctx, "sweep32_update", k_sweep_update_t<UpdSplit, true>, nblocks, ST,
                SWARPS * RD * UpdSplit::STAGE_BYTES, d_insts, strip_inst, base, partials);
  else
    launch_smem(ctx, "sweep_update", k_sweep_update_t<UpdF64, false>, nblocks, ST, SWARPS * RD * UpdF64::STAGE_BYTES,
                d_insts, strip_inst, base, partials);
}

}  // namespace otm
