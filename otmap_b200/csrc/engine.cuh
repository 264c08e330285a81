// Device-side records shared by the solver kernels (solver.cu) and the cosine-
// transform kernels (poisson.cu).
#pragma once

#include <cfloat>

#include "context.h"

namespace otm {

constexpr int TI = 8, TJ = 32, NT = 256;  // stencil tile: TI cells along x (i), TJ along y (j)
constexpr int HI = TI + 2, HJ = TJ + 2;   // halo tile of cells
constexpr int VI = TI + 1, VJ = TJ + 1;   // vertex tile
constexpr int KP = 8;                     // partial sums per tile
constexpr int GB = 64, GK = 16;           // DCT GEMM tile (GB x GB outputs, GK deep)

// Device record of one solve instance. Buffer pointers are fixed for the life of
// the workspace; everything below `it` is loop state updated by the kernels.
struct Inst {
  int n, tile0, ntiles, gemm0, ngemm;
  int max_iter, beta_cj;
  int fault;  // set on the device when a bounded wait gave up (the instance is stopped)
  double threshold, max_ratio;
  double* psi[2];
  double* r[3];
  double* dhat;
  double* d[2];
  double* rho;
  double* t1;
  double* t2;
  const double* C;
  const double* cosk;
  const double2* tw;  // exp(-2 pi i k / n), k < n/2 (fast transform); then the step-2 table
  const double2* pt;  // (cos, sin)(pi k / (2n)), k < n (fast transform)
  int fft, logn;      // fast transform used (n a power of two) / log2 n
  int split;          // split precision: r, d_hat, d, t1 hold FP32 values (psi, rho FP64)
  int tc0, ntc;       // tensor-core transform (dct_tc.cu): first item and item count of its work list
  int tcn;            // its output tile width (256, or 128 for n = 128)
  const float* Cf;    // C[k][i] and C^T as TF32 planes: hi (n^2 floats) then lo (n^2 floats)
  const float* CTf;
  float* rs;          // the residual's TF32 planes (hi, lo) for the first product
  const void* tmaps;  // 16 TMA tensor maps of the four products (device memory)
  int row0, nrow, col0, ncol;  // first item and item count in the row / column work lists
  int strip0, nstrip;          // first block and block count in the strip work list
  // loop state
  int it, active, outcome, use_beta;
  unsigned int counter;
  int srows;  // strip height of the sweeps for this batch (16, 32 or 64 rows)
  double residual, residual0, alpha, beta, linf, dnorm;
  double dens_scale, dens_beta;
};


// Sets `outcome` for an instance whose loop condition (otsolver_2dgrid.cpp:160) failed.
__device__ __forceinline__ void stop_outcome(Inst& I) {
  if (I.residual <= I.threshold)
    I.outcome = OTM_CONVERGED;
  else if (!isfinite(I.residual))
    I.outcome = OTM_NONFINITE;
  else
    I.outcome = OTM_MAX_ITER;
}

// ---------------------------------------------------------------------------
// Exact line search (otsolver_2dgrid.cpp:541-606).

__device__ __forceinline__ double cubic_eval(const double c[4], double t) { return ((c[3] * t + c[2]) * t + c[1]) * t + c[0]; }
__device__ __forceinline__ double cubic_deriv(const double c[4], double t) { return (3.0 * c[3] * t + 2.0 * c[2]) * t + c[1]; }

// Real roots of w3 t^3 + w2 t^2 + w1 t + w0: closed form of the depressed cubic
// (Cardano for one real root, the trigonometric form for three) and two Newton
// steps; replaces the companion-matrix eigensolver of otsolver_2dgrid.cpp:568-572.
__device__ __forceinline__ int cubic_real_roots(const double w[4], double roots[3]) {
  double a = w[2] / w[3], b = w[1] / w[3], c = w[0] / w[3];
  if (!isfinite(a) || !isfinite(b) || !isfinite(c)) return 0;
  double p = b - a * a / 3.0;
  double q = 2.0 * a * a * a / 27.0 - a * b / 3.0 + c;
  double disc = 0.25 * q * q + p * p * p / 27.0;
  int m;
  if (disc > 0.0) {
    double sq = sqrt(disc);
    double u = cbrt(-0.5 * q + (q <= 0.0 ? sq : -sq));
    double y = (u != 0.0) ? u - p / (3.0 * u) : 0.0;
    roots[0] = y - a / 3.0;
    m = 1;
  } else {
    double r = sqrt(std_max(0.0, -p / 3.0));
    if (r == 0.0) {
      roots[0] = roots[1] = roots[2] = -a / 3.0;
    } else {
      double arg = std_max(-1.0, std_min(1.0, -0.5 * q / (r * r * r)));
      double phi = acos(arg) / 3.0;
      for (int k = 0; k < 3; ++k) roots[k] = 2.0 * r * cos(phi - 2.0943951023931954923 * k) - a / 3.0;
    }
    m = 3;
  }
  double cc[4] = {c, b, a, 1.0};
  for (int k = 0; k < m; ++k)
    for (int s = 0; s < 2; ++s) {
      double f = cubic_eval(cc, roots[k]), df = cubic_deriv(cc, roots[k]);
      if (df != 0.0 && isfinite(f / df)) roots[k] -= f / df;
    }
  return m;
}

// Among the real stationary points of e(t) = z0 + z1 t + ... + z4 t^4 in [-10, 10] the
// one with least e(t); else t = 0.5 (otsolver_2dgrid.cpp:575-595).
__device__ __forceinline__ void pick_step(const double z[5], double* alpha, double* emin) {
  double w[4] = {z[1], 2.0 * z[2], 3.0 * z[3], 4.0 * z[4]};
  double roots[3];
  int m = cubic_real_roots(w, roots);
  bool found = false;
  double best = 0.0, rmin = 0.0;
  for (int k = 0; k < m; ++k) {
    double t = roots[k];
    if (t >= -10.0 && t <= 10.0) {
      double r = z[0] + t * (z[1] + t * (z[2] + t * (z[3] + t * z[4])));
      if (!found || r < rmin) {
        found = true;
        best = t;
        rmin = r;
      }
    }
  }
  if (!found) {
    best = 0.5;
    rmin = z[0] + best * (z[1] + best * (z[2] + best * (z[3] + best * z[4])));
  }
  *alpha = best;
  *emin = rmin;
}


// Host launcher of the fast cosine-transform Poisson solve (poisson.cu): d_hat = M^+ r_k
// for every active instance with fft != 0.
void poisson_fft(otm_context* ctx, Inst* d_insts, const int* row_inst, int roff, int nrow_items,
                 const int* col_inst, int coff, int ncol_items);
// Register-resident variant for n in {64, ..., 1024} (dct_reg.cu).
bool dct_reg_supported(int n);
// The register transforms' step-2 twiddles W_n^(t k1) in [register][lane] order (n entries),
// appended to the half table tw of the size.
void dct_reg_step2_table(int n, const std::vector<double2>& tw, std::vector<double2>& out);
int dct_reg_lines_per_block(int n);
int dct_reg_cols_per_block(int n);
// fp32: the FP32 kernels (r_k, the transform temporary t1 and d_hat are FP32 arrays).
void dct_reg_run(otm_context* ctx, int n, bool fp32, Inst* d_insts, const int* row_inst, int roff, int rcnt, const int* col_inst,
                 int coff, int ccnt);
// Tensor-core transform (dct_tc.cu) for split-precision instances of n in {128, ..., 1024}:
// d_hat = C^T ((C r C^T) / lambda) C as four tcgen05 products, 3xTF32 in FP32.
// The TF32 planes (hi then lo, n^2 floats each) of t1, t2 and rs hold every operand; the
// 16 tensor maps of an instance are encoded on the host (dct_tc_encode) once its buffers
// are laid out.
bool dct_tc_supported(int n);
int dct_tc_tn(int n);     // output tile width
int dct_tc_tiles(int n);  // 128 x dct_tc_tn(n) output tiles of one product
size_t dct_tc_map_bytes();  // bytes of one instance's tensor maps
void dct_tc_encode(const Inst& I, void* host_maps);
void dct_tc_split_basis(const double* C, int n, std::vector<float>& cs, std::vector<float>& cts);
void dct_tc_attrs(int device);
void dct_tc_run(otm_context* ctx, Inst* d_insts, const int* tc_inst, int base, int count);
// Dynamic shared-memory limits of the kernels of each family (set once per device,
// before any stream capture).
void sweep_attrs(int device);
void dct_reg_attrs(int device);
void poisson_fft_attrs(int device);

// Two-pass stencil sweep of an iteration (stencil.cu).
int strip_blocks(int n, int srows);
// Blocks base .. base + nblocks - 1 of the strip work list; split = the split-precision
// kernels (FP32 r, d_hat, d arrays).
void sweep_sums(otm_context* ctx, Inst* d_insts, const int* strip_inst, int base, int nblocks, bool split,
                double* partials);
void sweep_update(otm_context* ctx, Inst* d_insts, const int* strip_inst, int base, int nblocks, bool split,
                  double* partials);
constexpr int SWEEP_SLOTS = 32;  // partial-sum slots per sweep block

// Elements staged in shared memory per block of the transform kernels.
constexpr int FFT_ELEMS = 4096;
inline int fft_lines(int n) { return n < FFT_ELEMS / n ? n : FFT_ELEMS / n; }
inline bool fft_eligible(int n) { return n >= 8 && n <= FFT_ELEMS && (n & (n - 1)) == 0; }

}  // namespace otm
