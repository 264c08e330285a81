// Device-side records shared by the solver kernels (solver.cu) and the cosine-
// transform kernels (poisson.cu).
#pragma once

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
  int max_iter, beta_cj, pad0;
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
  const double2* tw;  // exp(-2 pi i k / n), k < n/2 (fast transform)
  const double2* pt;  // (cos, sin)(pi k / (2n)), k < n (fast transform)
  int fft, logn;      // fast transform used (n a power of two) / log2 n
  int row0, nrow, col0, ncol;  // first item and item count in the row / column work lists
  // loop state
  int it, active, outcome, use_beta;
  unsigned int counter, pad1;
  double residual, residual0, alpha, beta, linf, dnorm;
  double dens_scale, dens_beta;
};


// Host launcher of the fast cosine-transform Poisson solve (poisson.cu): d_hat = M^+ r_k
// for every active instance with fft != 0.
void poisson_fft(otm_context* ctx, Inst* d_insts, const int* row_inst, int nrow_items, const int* col_inst,
                 int ncol_items);
// Elements staged in shared memory per block of the transform kernels.
constexpr int FFT_ELEMS = 4096;
inline int fft_lines(int n) { return n < FFT_ELEMS / n ? n : FFT_ELEMS / n; }
inline bool fft_eligible(int n) { return n >= 8 && n <= FFT_ELEMS && (n & (n - 1)) == 0; }

}  // namespace otm
