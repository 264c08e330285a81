// Register-resident cosine transforms for n = N1 * N2 in {64, ..., 1024}.
//
// Same three passes and the same DCT-II / DCT-III formulation as poisson.cu (Makhoul
// reordering + one n-point complex FFT per line), but each n-point FFT is done as a
// four-step Cooley-Tukey split n = N1 * N2 held in registers:
//   step 1  lane t (of N2 lanes per line) holds v[N2*m1 + t], m1 < N1, and runs an
//           N1-point FFT on them in registers;
//   step 2  multiplies by the twiddles exp(-+2 pi i t k1 / n);
//   step 3  transposes through a padded shared-memory buffer (one per line,
//           synchronised by __syncwarp only);
//   step 4  lane k1 (< N1) runs an N2-point FFT on its N2 values in registers, giving
//           X[k1 + N1*k2].
// Shared memory then carries each element twice per transform instead of once per
// radix stage. The column pass stages a tile of CB full columns in shared memory so
// its global reads and writes are row-contiguous.

#include "engine.cuh"

namespace otm {
namespace {

constexpr int RW = 4;  // warps per block

__device__ __forceinline__ double2 cmul(double2 a, double2 w) {
  return make_double2(fma(a.x, w.x, -a.y * w.y), fma(a.x, w.y, a.y * w.x));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

template <int N>
__host__ __device__ constexpr int rbrev(int r) {
  int out = 0;
  for (int b = 1, o = N >> 1; b < N; b <<= 1, o >>= 1)
    if (r & b) out |= o;
  return out;
}

// W_n^e with tw[k] = exp(-2 pi i k / n), k < n/2; conj for the inverse kernel.
__device__ __forceinline__ double2 twid(const double2* __restrict__ tw, int e, int n, bool conj) {
  e &= n - 1;
  double2 w;
  if (e < (n >> 1)) {
    w = __ldg(&tw[e]);
  } else {
    w = __ldg(&tw[e - (n >> 1)]);
    w.x = -w.x;
    w.y = -w.y;
  }
  if (conj) w.y = -w.y;
  return w;
}

// In-register radix-2 decimation-in-frequency FFT of N values, natural order in,
// bit-reversed order out (v[r] = X[rbrev<N>(r)]). Twiddles W_N^k = tw[k * (n / N)].
template <int N>
__device__ __forceinline__ void fft_reg(double2 (&v)[N], const double2* __restrict__ tw, int n, bool conj) {
#pragma unroll
  for (int span = N / 2; span >= 1; span >>= 1) {
#pragma unroll
    for (int start = 0; start < N; start += 2 * span) {
#pragma unroll
      for (int k = 0; k < span; ++k) {
        const double2 a = v[start + k], b = v[start + k + span];
        v[start + k] = cadd(a, b);
        const double2 d = csub(a, b);
        const int e = k * (N / (2 * span));
        if (e == 0) {
          v[start + k + span] = d;
        } else {
          double2 w = __ldg(&tw[e * (n / N)]);
          if (conj) w.y = -w.y;
          v[start + k + span] = cmul(d, w);
        }
      }
    }
  }
}

// Steps 1-4 for one line. `in(m1)` gives lane t's input sample m = N2*m1 + t; `out(k, X)`
// receives X_k on lane k1 = k % N1 (only lanes t < N1 call it). buf is this line's
// N1 x (N2 + 1) shared buffer of doubles (the transpose moves real and imaginary
// parts in two rounds).
template <int N1, int N2, class In, class Out>
__device__ __forceinline__ void fft_line(int t, double* buf, const double2* __restrict__ tw, bool conj, In in,
                                         Out out) {
  constexpr int n = N1 * N2;
  double2 v[N1];
#pragma unroll
  for (int m1 = 0; m1 < N1; ++m1) v[m1] = in(m1);
  fft_reg<N1>(v, tw, n, conj);
#pragma unroll
  for (int r = 0; r < N1; ++r) {
    const int k1 = rbrev<N1>(r);
    if (k1 != 0) v[r] = cmul(v[r], twid(tw, t * k1, n, conj));
  }
  // transpose through shared memory, real parts then imaginary parts
  double2 u[N2];
#pragma unroll
  for (int part = 0; part < 2; ++part) {
#pragma unroll
    for (int r = 0; r < N1; ++r) buf[rbrev<N1>(r) * (N2 + 1) + t] = part ? v[r].y : v[r].x;
    __syncwarp();
    if (t < N1) {
#pragma unroll
      for (int m2 = 0; m2 < N2; ++m2) {
        const double x = buf[t * (N2 + 1) + m2];
        if (part)
          u[m2].y = x;
        else
          u[m2].x = x;
      }
    }
    __syncwarp();
  }
  if (t < N1) {
    fft_reg<N2>(u, tw, n, conj);
#pragma unroll
    for (int r = 0; r < N2; ++r) out(t + N1 * rbrev<N2>(r), u[r]);
  }
  __syncwarp();
}

__device__ __forceinline__ double dct_s(int k, int n) { return k == 0 ? sqrt(1.0 / n) : sqrt(2.0 / n); }
__device__ __forceinline__ int makhoul_src(int m, int n) { return m < (n >> 1) ? 2 * m : 2 * (n - 1 - m) + 1; }
// DCT-II coefficient from V_k: s_k Re(e^{-i pi k / 2n} V_k)
__device__ __forceinline__ double post2(double2 V, double2 pt, double sk) { return sk * fma(V.x, pt.x, V.y * pt.y); }
// DCT-III input W_k from Y_k (a) and Y_{n-k} (b)
__device__ __forceinline__ double2 pre3(int k, double a, double b, double2 pt) {
  if (k == 0) return make_double2(a, 0.0);
  return make_double2(0.5 * fma(a, pt.x, b * pt.y), 0.5 * fma(a, pt.y, -b * pt.x));
}

template <int N1, int N2>
__global__ __launch_bounds__(RW * 32, 3) void k_dct_rows_fwd(const Inst* insts, const int* row_inst, int seg) {
  constexpr int n = N1 * N2, LPW = 32 / N2, LPB = RW * LPW;
  extern __shared__ double sbuf[];
  const int item = seg + blockIdx.x;
  const Inst& I = insts[row_inst[item]];
  if (!I.active) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, sub = lane / N2, t = lane % N2;
  const int row = (item - I.row0) * LPB + warp * LPW + sub;
  double* buf = sbuf + (warp * LPW + sub) * N1 * (N2 + 1);
  const double* x = I.r[I.it % 3] + (size_t)row * n;
  double* y = I.t1 + (size_t)row * n;
  const double2* tw = I.tw;
  const double2* pt = I.pt;
  fft_line<N1, N2>(
      t, buf, tw, false, [&](int m1) { return make_double2(x[makhoul_src(N2 * m1 + t, n)], 0.0); },
      [&](int k, double2 V) { y[k] = post2(V, __ldg(&pt[k]), dct_s(k, n)); });
}

template <int N1, int N2>
__global__ __launch_bounds__(RW * 32, 3) void k_dct_rows_inv(const Inst* insts, const int* row_inst, int seg) {
  constexpr int n = N1 * N2, LPW = 32 / N2, LPB = RW * LPW;
  extern __shared__ double sbuf[];
  const int item = seg + blockIdx.x;
  const Inst& I = insts[row_inst[item]];
  if (!I.active) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, sub = lane / N2, t = lane % N2;
  const int row = (item - I.row0) * LPB + warp * LPW + sub;
  double* buf = sbuf + (warp * LPW + sub) * N1 * (N2 + 1);
  const double* X = I.t1 + (size_t)row * n;
  double* x = I.dhat + (size_t)row * n;
  const double2* tw = I.tw;
  const double2* pt = I.pt;
  fft_line<N1, N2>(
      t, buf, tw, true,
      [&](int m1) {
        const int k = N2 * m1 + t;
        double a = dct_s(k, n) * X[k];
        double b = k == 0 ? 0.0 : dct_s(n - k, n) * X[n - k];
        return pre3(k, a, b, __ldg(&pt[k]));
      },
      [&](int m, double2 v) { x[makhoul_src(m, n)] = v.x; });
}

// Column pass, lanes across columns: a block owns CB consecutive columns. Thread
// (c = tid % CB, s = tid / CB) holds, for column l0 + c, the samples N2*m1 + s (s < N2) of
// step 1 -- loaded straight from global memory, CB consecutive doubles per row -- and the
// outputs k1 = s (s < N1) of step 4. One shared region (n x CB doubles plus a pad per k1
// row) serves in turn as the step-3 transpose buffer, the exchange tile for the DCT-III
// pairs (k, n - k) and the staging tile of the coalesced store.
template <int N1, int N2>
struct ColGeom {
  static constexpr int n = N1 * N2;
  static constexpr int CB = 256 / N2;  // columns per block (256 threads)
  static constexpr int KS = N2 * CB + 1;  // padded stride of a k1 row of the transpose buffer
  static constexpr int SMEM = (N1 * KS > n * CB ? N1 * KS : n * CB);  // doubles
};

template <int N1, int N2>
__device__ __forceinline__ void col_fft_transpose(double2 (&v)[N1], double2 (&u)[N2], double* sh, int c, int s,
                                                  const double2* __restrict__ tw, bool conj) {
  using GG = ColGeom<N1, N2>;
  constexpr int n = GG::n, CB = GG::CB, KS = GG::KS;
  fft_reg<N1>(v, tw, n, conj);
#pragma unroll
  for (int r = 0; r < N1; ++r) {
    const int k1 = rbrev<N1>(r);
    if (k1 != 0) v[r] = cmul(v[r], twid(tw, s * k1, n, conj));
  }
#pragma unroll
  for (int part = 0; part < 2; ++part) {
    __syncthreads();
#pragma unroll
    for (int r = 0; r < N1; ++r) sh[rbrev<N1>(r) * KS + s * CB + c] = part ? v[r].y : v[r].x;
    __syncthreads();
    if (s < N1) {
#pragma unroll
      for (int m2 = 0; m2 < N2; ++m2) {
        const double x = sh[s * KS + m2 * CB + c];
        if (part)
          u[m2].y = x;
        else
          u[m2].x = x;
      }
    }
  }
  if (s < N1) fft_reg<N2>(u, tw, n, conj);
}

template <int N1, int N2>
__global__ __launch_bounds__(256, 1) void k_dct_cols(const Inst* insts, const int* col_inst, int seg) {
  using GG = ColGeom<N1, N2>;
  constexpr int n = GG::n, CB = GG::CB;
  extern __shared__ double sbuf[];
  const int item = seg + blockIdx.x;
  const Inst& I = insts[col_inst[item]];
  if (!I.active) return;
  const int c = threadIdx.x % CB, s = threadIdx.x / CB;
  const int l0 = (item - I.col0) * CB, l = l0 + c;
  double* T = I.t1;
  const double2* tw = I.tw;
  const double2* pt = I.pt;
  const double cl = I.cosk[l];
  double2 v[N1];
  double2 u[N2];
  // forward DCT-II along the column
#pragma unroll
  for (int m1 = 0; m1 < N1; ++m1) v[m1] = make_double2(T[(size_t)makhoul_src(N2 * m1 + s, n) * n + l], 0.0);
  col_fft_transpose<N1, N2>(v, u, sbuf, c, s, tw, false);
  __syncthreads();
  if (s < N1) {
    // coefficient k = s + N1 k2: divide by lambda_kl, keep s_k U_k in the exchange tile [k][c]
#pragma unroll
    for (int r = 0; r < N2; ++r) {
      const int k = s + N1 * rbrev<N2>(r);
      const double sk = dct_s(k, n);
      const double X = post2(u[r], __ldg(&pt[k]), sk);
      const double lam = 2.0 - 2.0 * I.cosk[k] * cl;
      const double U = (k == 0 && l == 0) ? 0.0 : X / lam;
      sbuf[k * CB + c] = sk * U;
    }
  }
  __syncthreads();
  // inverse DCT-III along the column
#pragma unroll
  for (int m1 = 0; m1 < N1; ++m1) {
    const int k = N2 * m1 + s;
    const double a = sbuf[k * CB + c], b = k == 0 ? 0.0 : sbuf[(n - k) * CB + c];
    v[m1] = pre3(k, a, b, __ldg(&pt[k]));
  }
  col_fft_transpose<N1, N2>(v, u, sbuf, c, s, tw, true);
  __syncthreads();
  if (s < N1) {
#pragma unroll
    for (int r = 0; r < N2; ++r) {
      const int m = s + N1 * rbrev<N2>(r);
      sbuf[makhoul_src(m, n) * CB + c] = u[r].x;
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < n * CB; e += 256) {
    const int i = e / CB, cc = e - i * CB;
    T[(size_t)i * n + l0 + cc] = sbuf[i * CB + cc];
  }
}

template <int N1, int N2>
struct RegDct {
  static constexpr int n = N1 * N2, LPW = 32 / N2, LPB = RW * LPW;
  static size_t rows_smem() { return sizeof(double) * LPB * N1 * (N2 + 1); }
  static size_t cols_smem() { return sizeof(double) * ColGeom<N1, N2>::SMEM; }
  static constexpr int CB = ColGeom<N1, N2>::CB;
  static void attrs() {
    OTM_CUDA(cudaFuncSetAttribute(k_dct_rows_fwd<N1, N2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)rows_smem()));
    OTM_CUDA(cudaFuncSetAttribute(k_dct_rows_inv<N1, N2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)rows_smem()));
    OTM_CUDA(cudaFuncSetAttribute(k_dct_cols<N1, N2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)cols_smem()));
  }
  static void run(otm_context* ctx, Inst* d, const int* ri, int roff, int rcnt, const int* ci, int coff, int ccnt) {
    launch_smem(ctx, "dct_rows_fwd", k_dct_rows_fwd<N1, N2>, rcnt, RW * 32, rows_smem(), (const Inst*)d, ri, roff);
    launch_smem(ctx, "dct_cols", k_dct_cols<N1, N2>, ccnt, 256, cols_smem(), (const Inst*)d, ci, coff);
    launch_smem(ctx, "dct_rows_inv", k_dct_rows_inv<N1, N2>, rcnt, RW * 32, rows_smem(), (const Inst*)d, ri, roff);
  }
};

}  // namespace

bool dct_reg_supported(int n) { return n == 64 || n == 128 || n == 256 || n == 512 || n == 1024; }

int dct_reg_lines_per_block(int n) {
  switch (n) {
    case 64: return RegDct<8, 8>::LPB;
    case 128: return RegDct<8, 16>::LPB;
    case 256: return RegDct<16, 16>::LPB;
    case 512: return RegDct<16, 32>::LPB;
    default: return RegDct<32, 32>::LPB;
  }
}

int dct_reg_cols_per_block(int n) {
  switch (n) {
    case 64: return RegDct<8, 8>::CB;
    case 128: return RegDct<8, 16>::CB;
    case 256: return RegDct<16, 16>::CB;
    case 512: return RegDct<16, 32>::CB;
    default: return RegDct<32, 32>::CB;
  }
}

void dct_reg_attrs(int device) {
  static bool done[64] = {};
  if (device < 64 && done[device]) return;
  RegDct<8, 8>::attrs();
  RegDct<8, 16>::attrs();
  RegDct<16, 16>::attrs();
  RegDct<16, 32>::attrs();
  RegDct<32, 32>::attrs();
  if (device < 64) done[device] = true;
}

void dct_reg_run(otm_context* ctx, int n, Inst* d_insts, const int* row_inst, int roff, int rcnt, const int* col_inst,
                 int coff, int ccnt) {
  dct_reg_attrs(ctx->device);
  switch (n) {
    case 64: RegDct<8, 8>::run(ctx, d_insts, row_inst, roff, rcnt, col_inst, coff, ccnt); break;
    case 128: RegDct<8, 16>::run(ctx, d_insts, row_inst, roff, rcnt, col_inst, coff, ccnt); break;
    case 256: RegDct<16, 16>::run(ctx, d_insts, row_inst, roff, rcnt, col_inst, coff, ccnt); break;
    case 512: RegDct<16, 32>::run(ctx, d_insts, row_inst, roff, rcnt, col_inst, coff, ccnt); break;
    case 1024: RegDct<32, 32>::run(ctx, d_insts, row_inst, roff, rcnt, col_inst, coff, ccnt); break;
    default: throw BadArg{"dct_reg_run: unsupported size"};
  }
}

}  // namespace otm
