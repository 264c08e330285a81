// Fast cosine-transform Poisson solve, FP64, for power-of-two grid sizes.
//
// d_hat = M^+ r with M the reference's pseudo-Laplacian (otlib/otsolver_2dgrid.cpp:284-311):
// with C the orthonormal DCT-II, M^+ r = C^T ((C R C^T) / lambda) C where
// lambda_kl = 2 - 2 cos(pi k/n) cos(pi l/n) and the (0,0) mode is dropped (the
// mean-zero projection of :179). Three passes over the n x n array, each staging
// whole lines in shared memory:
//   k_fft_rows_fwd   T[i][l] = DCT-II of r[i][.]                  (rows, contiguous)
//   k_fft_cols       for a block of columns l: DCT-II along i, divide by lambda,
//                    DCT-III back along k                         (in place)
//   k_fft_rows_inv   d_hat[i][j] = DCT-III of T[i][.]
// Each length-n cosine transform is one n-point complex FFT (radix-2, in place,
// bit-reversed input) with Makhoul's even/odd reordering and a quarter-wave twiddle:
//   DCT-II : v_m = x_2m, v_{n-1-m} = x_{2m+1}; V = FFT(v); X_k = s_k Re(e^{-i pi k/2n} V_k)
//   DCT-III: W_0 = Y_0, W_k = e^{i pi k/2n} (Y_k - i Y_{n-k}) / 2, Y = s X; v = IFFT(W) (no 1/n);
//            x_2m = Re v_m, x_{2m+1} = Re v_{n-1-m}
// with s_0 = sqrt(1/n), s_k = sqrt(2/n). The work is memory-bound (3 reads + 3 writes of
// the array) where the dense C.X.C^T form costs 8 n^3 flops.

#include "engine.cuh"

namespace otm {

constexpr int FT = 256;  // threads per block

__device__ __forceinline__ int brev(int m, int logn) { return (int)(__brev((unsigned)m) >> (32 - logn)); }

// Shared-memory slot of element `idx` of a line-major staging buffer: one double2 of
// padding after every 32 keeps bit-reversed scatters and short-stride butterflies
// free of bank conflicts.
__device__ __forceinline__ int slot(int idx) { return idx + (idx >> 5); }
__host__ __device__ constexpr int padded(int elems) { return elems + elems / 32; }

__device__ __forceinline__ double2 cmul(double2 a, double2 w) {
  return make_double2(fma(a.x, w.x, -a.y * w.y), fma(a.x, w.y, a.y * w.x));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

// In-place decimation-in-time FFT of `lines` sequences of length n = 2^logn stored
// line-major in s (padded slots), input in bit-reversed order; forward uses
// exp(-2 pi i k/n), conj the inverse kernel (unnormalised). Two radix-2 stages are
// fused per pass (radix 4, in registers), plus one radix-2 pass when logn is odd.
__device__ void fft_lines_inplace(double2* s, int logn, int lines, const double2* __restrict__ tw, bool conj) {
  const int n = 1 << logn;
  int st = 0;
  if (logn & 1) {  // first stage alone: half = 1, twiddle 1
    const int nb = lines * (n >> 1);
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
      const int i0 = 2 * b;
      const double2 a = s[slot(i0)], c = s[slot(i0 + 1)];
      s[slot(i0)] = cadd(a, c);
      s[slot(i0 + 1)] = csub(a, c);
    }
    __syncthreads();
    st = 1;
  }
  for (; st < logn; st += 2) {
    const int half = 1 << st;
    const int nq = lines * (n >> 2);  // radix-4 butterflies
    for (int b = threadIdx.x; b < nq; b += blockDim.x) {
      const int line = b >> (logn - 2);
      const int bb = b & ((n >> 2) - 1);
      const int pos = bb & (half - 1);
      const int i0 = line * n + ((bb >> st) << (st + 2)) + pos;
      double2 w1 = __ldg(&tw[pos << (logn - 1 - st)]);
      double2 w2 = __ldg(&tw[pos << (logn - 2 - st)]);
      double2 w3 = __ldg(&tw[(pos + half) << (logn - 2 - st)]);
      if (conj) {
        w1.y = -w1.y;
        w2.y = -w2.y;
        w3.y = -w3.y;
      }
      double2 e0 = s[slot(i0)], e1 = s[slot(i0 + half)], e2 = s[slot(i0 + 2 * half)], e3 = s[slot(i0 + 3 * half)];
      // stage st: (e0, e1) and (e2, e3) with w1
      double2 t1 = cmul(e1, w1), t3 = cmul(e3, w1);
      double2 f0 = cadd(e0, t1), f1 = csub(e0, t1), f2 = cadd(e2, t3), f3 = csub(e2, t3);
      // stage st + 1: (f0, f2) with w2, (f1, f3) with w3
      double2 u2 = cmul(f2, w2), u3 = cmul(f3, w3);
      s[slot(i0)] = cadd(f0, u2);
      s[slot(i0 + 2 * half)] = csub(f0, u2);
      s[slot(i0 + half)] = cadd(f1, u3);
      s[slot(i0 + 3 * half)] = csub(f1, u3);
    }
    __syncthreads();
  }
}

// Makhoul position of input sample j in the reordered sequence.
__device__ __forceinline__ int makhoul_pos(int j, int n) { return (j & 1) ? n - 1 - (j >> 1) : (j >> 1); }

__device__ __forceinline__ double dct_scale(int k, int n) { return k == 0 ? sqrt(1.0 / n) : sqrt(2.0 / n); }

// X_k = s_k Re(e^{-i pi k / 2n} V_k)
__device__ __forceinline__ double dct2_post(double2 V, double2 pt, double sk) {
  return sk * fma(V.x, pt.x, V.y * pt.y);
}

// W_k = e^{i pi k / 2n} (a - i b) / 2 with a = Y_k, b = Y_{n-k}; W_0 = Y_0
__device__ __forceinline__ double2 dct3_pre(int k, double a, double b, double2 pt) {
  if (k == 0) return make_double2(a, 0.0);
  return make_double2(0.5 * fma(a, pt.x, b * pt.y), 0.5 * fma(a, pt.y, -b * pt.x));
}

__global__ __launch_bounds__(FT) void k_fft_rows_fwd(const Inst* insts, const int* row_inst, int seg) {
  extern __shared__ double2 sm[];
  const int item = seg + blockIdx.x;
  const Inst& I = insts[row_inst[item]];
  if (!I.active) return;
  const int n = I.n, logn = I.logn, R = n < FFT_ELEMS / n ? n : FFT_ELEMS / n;
  const int i0 = (item - I.row0) * R;
  const double* src = I.r[I.it % 3];
  double* dst = I.t1;
  for (int e = threadIdx.x; e < R * n; e += FT) {
    int line = e >> logn, j = e & (n - 1);
    double x = src[(size_t)(i0 + line) * n + j];
    sm[slot(line * n + brev(makhoul_pos(j, n), logn))] = make_double2(x, 0.0);
  }
  __syncthreads();
  fft_lines_inplace(sm, logn, R, I.tw, false);
  for (int e = threadIdx.x; e < R * n; e += FT) {
    int line = e >> logn, k = e & (n - 1);
    dst[(size_t)(i0 + line) * n + k] = dct2_post(sm[slot(e)], __ldg(&I.pt[k]), dct_scale(k, n));
  }
}

// In place on t1: a block of CB = FFT_ELEMS / n columns (all n rows).
__global__ __launch_bounds__(FT) void k_fft_cols(const Inst* insts, const int* col_inst, int seg) {
  extern __shared__ double2 sm[];
  const int item = seg + blockIdx.x;
  const Inst& I = insts[col_inst[item]];
  if (!I.active) return;
  const int n = I.n, logn = I.logn, CB = n < FFT_ELEMS / n ? n : FFT_ELEMS / n;
  double* ybuf = reinterpret_cast<double*>(sm + padded(CB * n));  // CB * n doubles
  const int l0 = (item - I.col0) * CB;
  double* T = I.t1;
  // load: line c = column l0 + c, sample i = row
  for (int e = threadIdx.x; e < CB * n; e += FT) {
    int i = e / CB, c = e - i * CB;
    double x = T[(size_t)i * n + l0 + c];
    sm[slot(c * n + brev(makhoul_pos(i, n), logn))] = make_double2(x, 0.0);
  }
  __syncthreads();
  fft_lines_inplace(sm, logn, CB, I.tw, false);
  // DCT-II coefficient, divided by lambda_kl, times s_k for the inverse
  for (int e = threadIdx.x; e < CB * n; e += FT) {
    int c = e >> logn, k = e & (n - 1);
    int l = l0 + c;
    double sk = dct_scale(k, n);
    double X = dct2_post(sm[slot(e)], __ldg(&I.pt[k]), sk);
    double lam = 2.0 - 2.0 * I.cosk[k] * I.cosk[l];
    double U = (k == 0 && l == 0) ? 0.0 : X / lam;
    ybuf[e] = sk * U;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < CB * n; e += FT) {
    int c = e >> logn, k = e & (n - 1);
    double a = ybuf[e], b = k == 0 ? 0.0 : ybuf[c * n + (n - k)];
    sm[slot(c * n + brev(k, logn))] = dct3_pre(k, a, b, __ldg(&I.pt[k]));
  }
  __syncthreads();
  fft_lines_inplace(sm, logn, CB, I.tw, true);
  for (int e = threadIdx.x; e < CB * n; e += FT) {
    int i = e / CB, c = e - i * CB;
    int m = (i & 1) ? n - 1 - (i >> 1) : (i >> 1);
    T[(size_t)i * n + l0 + c] = sm[slot(c * n + m)].x;
  }
}

__global__ __launch_bounds__(FT) void k_fft_rows_inv(const Inst* insts, const int* row_inst, int seg) {
  extern __shared__ double2 sm[];
  const int item = seg + blockIdx.x;
  const Inst& I = insts[row_inst[item]];
  if (!I.active) return;
  const int n = I.n, logn = I.logn, R = n < FFT_ELEMS / n ? n : FFT_ELEMS / n;
  const int i0 = (item - I.row0) * R;
  const double* src = I.t1;
  double* dst = I.dhat;
  for (int e = threadIdx.x; e < R * n; e += FT) {
    int line = e >> logn, k = e & (n - 1);
    const double* row = src + (size_t)(i0 + line) * n;
    double a = dct_scale(k, n) * row[k];
    double b = k == 0 ? 0.0 : dct_scale(n - k, n) * row[n - k];
    sm[slot(line * n + brev(k, logn))] = dct3_pre(k, a, b, __ldg(&I.pt[k]));
  }
  __syncthreads();
  fft_lines_inplace(sm, logn, R, I.tw, true);
  for (int e = threadIdx.x; e < R * n; e += FT) {
    int line = e >> logn, i = e & (n - 1);
    int m = (i & 1) ? n - 1 - (i >> 1) : (i >> 1);
    dst[(size_t)(i0 + line) * n + i] = sm[slot(line * n + m)].x;
  }
}

static const int smem_rows = padded(FFT_ELEMS) * sizeof(double2);
static const int smem_cols = padded(FFT_ELEMS) * sizeof(double2) + FFT_ELEMS * sizeof(double);

void poisson_fft_attrs(int device) {
  static bool attr[64] = {};  // per device ordinal
  if (device < 64 && attr[device]) return;
  OTM_CUDA(cudaFuncSetAttribute(k_fft_rows_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_rows));
  OTM_CUDA(cudaFuncSetAttribute(k_fft_rows_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_rows));
  OTM_CUDA(cudaFuncSetAttribute(k_fft_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_cols));
  if (device < 64) attr[device] = true;
}

void poisson_fft(otm_context* ctx, Inst* d_insts, const int* row_inst, int roff, int nrow_items,
                 const int* col_inst, int coff, int ncol_items) {
  poisson_fft_attrs(ctx->device);
  if (nrow_items <= 0) return;
  launch_smem(ctx, "fft_rows_fwd", k_fft_rows_fwd, nrow_items, FT, smem_rows, (const Inst*)d_insts, row_inst, roff);
  launch_smem(ctx, "fft_cols", k_fft_cols, ncol_items, FT, smem_cols, (const Inst*)d_insts, col_inst, coff);
  launch_smem(ctx, "fft_rows_inv", k_fft_rows_inv, nrow_items, FT, smem_rows, (const Inst*)d_insts, row_inst, roff);
}

}  // namespace otm
