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
// radix stage. Every transform here is of real data, so each complex FFT carries two
// lines at once: two rows (or two columns) as its real and imaginary parts. For the
// DCT-II the two spectra are separated afterwards, A_k = (Z_k + conj Z_{n-k}) / 2 and
// B_k = (Z_k - conj Z_{n-k}) / 2i; for the DCT-III both inputs are Hermitian, so the
// real and imaginary parts of the one inverse FFT are the two output lines. The column
// pass stages a tile of full column pairs in shared memory so its global reads and
// writes are row-contiguous. All three kernels are persistent; each block copies the
// size's tables (step-2 twiddles in [register][lane] order, post-twiddles, cosines) into
// shared memory once, so no table read waits on L1 or L2 inside a transform.
//
// Every kernel is instantiated for FP64 (the default precision) and FP32 (the split
// precision mode, OTM_PRECISION_SPLIT: r, the transform temporaries and d_hat are FP32
// arrays). The FP32 forms hold half the registers per line, so their row passes run 16
// warps per block instead of 8; the tables are the same FP64 tables, rounded to FP32
// when a block copies them into shared memory.

#include <algorithm>
#include <cmath>
#include <vector>

#include "engine.cuh"

namespace otm {
namespace {

// Per precision: the complex type, the row passes' warps per block (one block per SM at
// n = 1024) and the spectrum coefficients sharing one division in the column pass.
template <class R>
struct RT;
template <>
struct RT<double> {
  using V = double2;
  static constexpr int RW = 8;
  static constexpr int DIV_GROUP = 4;
  static constexpr int COL_BLOCKS = 1;  // column blocks per SM the kernel is compiled for
};
template <>
struct RT<float> {
  using V = float2;
  static constexpr int RW = 16;
  // products of 2 DIV_GROUP eigenvalues must stay normal in FP32 (lambda >= ~1e-5 at n = 1024)
  static constexpr int DIV_GROUP = 2;
  static constexpr int COL_BLOCKS = 2;
};

__device__ __forceinline__ double2 mk2(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ float2 mk2(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ double rfma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float rfma(float a, float b, float c) { return fmaf(a, b, c); }

// exp(-2 pi i k / 1024), k < 512, in constant memory. A radix-2 stage of an N-point
// sub-FFT needs W_N^e = entry e * (1024 / N), an index known at compile time, so the
// arithmetic reads the twiddle as a constant operand instead of waiting on a load. The
// entries equal those of the per-size tables (same host formula; the index scaling by a
// power of two is exact); the FP32 table is the FP64 one rounded.
constexpr int CTW = 1024;
__constant__ double2 c_tw[CTW / 2];
__constant__ float2 c_twf[CTW / 2];
__device__ __forceinline__ double2 ctw(double2*, int e) { return c_tw[e]; }
__device__ __forceinline__ float2 ctw(float2*, int e) { return c_twf[e]; }

__device__ __forceinline__ double2 cmul(double2 a, double2 w) {
  return make_double2(fma(a.x, w.x, -a.y * w.y), fma(a.x, w.y, a.y * w.x));
}
__device__ __forceinline__ float2 cmul(float2 a, float2 w) {
  return make_float2(fmaf(a.x, w.x, -a.y * w.y), fmaf(a.x, w.y, a.y * w.x));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

template <int N>
__host__ __device__ constexpr int rbrev(int r) {
  int out = 0;
  for (int b = 1, o = N >> 1; b < N; b <<= 1, o >>= 1)
    if (r & b) out |= o;
  return out;
}

// Step-2 twiddle of register r on lane t, W_n^(t * rbrev<N1>(r)), from the per-size table
// tw2[r * N2 + t] (laid out so that a warp's 32 lanes read consecutive entries: one
// conflict-free shared-memory or coalesced global request per register instead of a
// gather); conj for the inverse kernel.
template <class V>
__device__ __forceinline__ V twid2(const V* tw2, int idx, bool conj) {
  V w = tw2[idx];
  if (conj) w.y = -w.y;
  return w;
}

// In-register radix-2 decimation-in-frequency FFT of N values, natural order in,
// bit-reversed order out (v[r] = X[rbrev<N>(r)]). Twiddles from the constant table.
template <int N, class V>
__device__ __forceinline__ void fft_reg(V (&v)[N], bool conj) {
#pragma unroll
  for (int span = N / 2; span >= 1; span >>= 1) {
#pragma unroll
    for (int start = 0; start < N; start += 2 * span) {
#pragma unroll
      for (int k = 0; k < span; ++k) {
        const V a = v[start + k], b = v[start + k + span];
        v[start + k] = cadd(a, b);
        const V d = csub(a, b);
        const int e = k * (N / (2 * span));
        if (e == 0) {
          v[start + k + span] = d;
        } else if (4 * e == N) {
          // W_N^(N/4) = -i (forward) or +i (inverse): a swap instead of a product
          v[start + k + span] = conj ? mk2(-d.y, d.x) : mk2(d.y, -d.x);
        } else {
          V w = ctw((V*)nullptr, e * (CTW / N));
          if (conj) w.y = -w.y;
          v[start + k + span] = cmul(d, w);
        }
      }
    }
  }
}

// Steps 1-4 for one line. On entry lane t (< N2) holds in v[m1] the input sample
// m = N2*m1 + t; on return lanes t < N1 hold u[r] = X_k for k = t + N1 * rbrev<N2>(r).
// Lanes t >= N2 of a wider lane group take no part. buf is this line's N1 x (N2 + 1)
// shared buffer of reals (the transpose moves real and imaginary parts in two rounds).
template <int N1, int N2, class R, class V>
__device__ __forceinline__ void fft_line(int t, R* buf, const V* tw2, bool conj, V (&v)[N1], V (&u)[N2]) {
  const int tt = t < N2 ? t : 0;
  fft_reg<N1>(v, conj);
#pragma unroll
  for (int r = 0; r < N1; ++r) {
    const int k1 = rbrev<N1>(r);
    if (k1 != 0) v[r] = cmul(v[r], twid2(tw2, r * N2 + tt, conj));
  }
  // transpose through shared memory, real parts then imaginary parts
#pragma unroll
  for (int part = 0; part < 2; ++part) {
    if (t < N2) {
#pragma unroll
      for (int r = 0; r < N1; ++r) buf[rbrev<N1>(r) * (N2 + 1) + t] = part ? v[r].y : v[r].x;
    }
    __syncwarp();
    if (t < N1) {
#pragma unroll
      for (int m2 = 0; m2 < N2; ++m2) {
        const R x = buf[t * (N2 + 1) + m2];
        if (part)
          u[m2].y = x;
        else
          u[m2].x = x;
      }
    }
    __syncwarp();
  }
  if (t < N1) fft_reg<N2>(u, conj);
}

// Register index holding X_{n-k} on the partner lane, for the X_k held in u[r]:
// lane t != 0 pairs with lane N1 - t and k2 -> N2 - 1 - k2; lane 0 with itself and
// k2 -> (N2 - k2) mod N2.
template <int N2>
__host__ __device__ constexpr int partner_reg(int r, bool lane0) {
  const int k2 = rbrev<N2>(r);
  const int k2p = lane0 ? (N2 - k2) % N2 : N2 - 1 - k2;
  return rbrev<N2>(k2p);  // rbrev is its own inverse
}

// Orthonormal DCT scale s_k = sqrt(1/n) (k = 0) or sqrt(2/n), the two roots formed once per thread.
template <class R>
struct DctScale {
  R s0, s1;
  __device__ __forceinline__ explicit DctScale(int n) : s0((R)sqrt(1.0 / n)), s1((R)sqrt(2.0 / n)) {}
  __device__ __forceinline__ R operator()(int k) const { return k == 0 ? s0 : s1; }
};
// DCT-II coefficient from V_k: s_k Re(e^{-i pi k / 2n} V_k)
template <class R, class V>
__device__ __forceinline__ R post2(V X, V pt, R sk) {
  return sk * rfma(X.x, pt.x, X.y * pt.y);
}
// DCT-III input W_k from Y_k (a) and Y_{n-k} (b)
template <class R, class V>
__device__ __forceinline__ V pre3(int k, R a, R b, V pt) {
  if (k == 0) return mk2(a, (R)0);
  return mk2((R)0.5 * rfma(a, pt.x, b * pt.y), (R)0.5 * rfma(a, pt.y, -b * pt.x));
}

// ---- row passes: software-pipelined over the warp's work items ----
//
// A work item is LPW consecutive row pairs (one per FFT line of the warp), 2*LPW whole
// rows that are contiguous in global memory; items are numbered within the segment
// (seg + item indexes the work list, whose entries Inst::row0 counts from). The grid is persistent (as many blocks as
// fit on the GPU); each warp takes items item, item + stride, ... and keeps one item in
// flight: as soon as an item's rows are in registers, one lane starts the bulk copy
// (cp.async.bulk, completion on the warp's mbarrier) of the next item into the warp's
// shared buffer, and the copy proceeds while the warp computes the FFTs of the current
// item. Waits are bounded: if one runs out the instance is flagged (Inst::fault) and
// stopped, and the warp returns after a second bounded wait for its copy.

template <class R, int N1, int N2>
struct RowGeom {
  using V = typename RT<R>::V;
  static constexpr int RW = RT<R>::RW;               // warps per block
  static constexpr int n = N1 * N2, LPW = 32 / N2;
  static constexpr int DATA = 2 * LPW * n;           // reals: the item's rows
  static constexpr int TRANS = LPW * N1 * (N2 + 1);  // reals: step-3 transpose buffers
  static constexpr int WARP = DATA + TRANS;          // reals per warp
  static_assert((WARP * sizeof(R)) % 16 == 0, "each warp's buffer starts 16-byte aligned");
  static constexpr int TABLES = 2 * n;               // complex: the step-2 twiddles, then pt
  static constexpr size_t SMEM = sizeof(R) * RW * WARP + sizeof(V) * TABLES + 16 * RW;  // + mbarriers
};

// The block's copy of the size's step-2 twiddles (n entries) and post-twiddles pt (n entries),
// read by every item of the persistent kernel: shared-memory latency instead of L1's.
template <class R, int N1, int N2>
__device__ __forceinline__ typename RT<R>::V* load_row_tables(R* sbuf, const Inst& I) {
  using G = RowGeom<R, N1, N2>;
  using V = typename G::V;
  constexpr int n = G::n;
  V* tab = reinterpret_cast<V*>(sbuf + G::RW * G::WARP);
  const double2* tw2 = I.tw + (n >> 1);
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    const double2 a = __ldg(&tw2[e]), b = __ldg(&I.pt[e]);
    tab[e] = mk2((R)a.x, (R)a.y);
    tab[n + e] = mk2((R)b.x, (R)b.y);
  }
  __syncthreads();
  return tab;
}

constexpr long long kWaitCycles = 2000000000LL;   // ~1 s at the B200's clock
constexpr long long kTestWaitCycles = 2000000LL;  // ~1 ms (OTM_OPT_WAIT_TEST)

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// One lane: expect `bytes` (+ `extra`, which never arrive: OTM_OPT_WAIT_TEST) on the
// barrier and start the bulk copy global -> shared. The proxy fence orders the warp's
// earlier generic reads of the buffer before the copy's writes.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned extra,
                                          unsigned long long* bar) {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes + extra)
               : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Waits until the barrier's phase of parity `parity` has completed; false when the
// bound ran out first.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, long long limit) {
  const unsigned a = smem_u32(bar);
  const long long t0 = clock64();
  while (true) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > limit) return false;
  }
}

// A wait ran out: flag and stop the instance, give the copy in flight one more bounded
// wait, and leave.
__device__ __forceinline__ void wait_fault(Inst& I, unsigned long long* bar, unsigned parity, int lane,
                                           long long limit) {
  if (lane == 0) {
    atomicExch(&I.fault, 1);
    I.active = 0;
  }
  mbar_wait(bar, parity, limit);
}

// Forward DCT-II of rows 2p and 2p+1 of r_k (one complex FFT per row pair) -> T.
template <class R, int N1, int N2>
__global__ __launch_bounds__(RT<R>::RW * 32, 1) void k_dct_rows_fwd(Inst* insts, const int* row_inst, int seg,
                                                                     int items, unsigned extra, long long limit) {
  using G = RowGeom<R, N1, N2>;
  using V = typename G::V;
  constexpr int n = G::n, LPW = G::LPW, RW = G::RW;
  const DctScale<R> ds(n);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sbuf = reinterpret_cast<R*>(smem_raw);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, sub = lane / N2, t = lane % N2;
  R* data = sbuf + warp * G::WARP;
  R* buf = data + G::DATA + sub * N1 * (N2 + 1);
  if (items <= 0) return;
  const V* tab = load_row_tables<R, N1, N2>(sbuf, insts[row_inst[seg]]);
  const V* spt = tab + n;
  unsigned long long* bar =
      reinterpret_cast<unsigned long long*>(smem_raw + sizeof(R) * RW * G::WARP + sizeof(V) * G::TABLES) + warp;
  const int stride = gridDim.x * RW;
  if (lane == 0) mbar_init(bar);
  __syncwarp();
  auto issue = [&](int it) -> bool {
    if (it >= items) return false;
    const Inst& J = insts[row_inst[seg + it]];
    if (!J.active) return false;
    if (lane == 0)
      bulk_load(data, reinterpret_cast<const R*>(J.r[J.it % 3]) + (size_t)(seg + it - J.row0) * G::DATA,
                sizeof(R) * G::DATA, extra, bar);
    return true;
  };
  unsigned phase = 0;
  // consecutive items go to consecutive blocks, so that a short list (a batch's last few
  // active instances) still spreads over every SM
  int item = warp * gridDim.x + blockIdx.x;
  bool pending = issue(item);
  const int mirror = (lane - t) + (N2 - 1 - t);
  const int src_lane = (lane - t) + (t < N1 ? (N1 - t) % N1 : 0);
  while (item < items) {
    const int next = item + stride;
    if (!pending) {
      pending = issue(next);
      item = next;
      continue;
    }
    Inst& I = insts[row_inst[seg + item]];
    if (!mbar_wait(bar, phase, limit)) {
      wait_fault(I, bar, phase, lane, limit);
      return;
    }
    phase ^= 1;
    // Makhoul order: sample m < n/2 is x[2m], sample m >= n/2 is x[2(n-1-m)+1]. Lane t
    // reads the pairs x[2(N2 m1 + t)], x[2(N2 m1 + t) + 1] (m1 < N1/2): the first is its
    // own sample m = N2 m1 + t, the second is sample n-1-m, which belongs to lane
    // N2-1-t at m1' = N1-1-m1 and is passed there by a shuffle.
    const R* xa = data + sub * 2 * n;
    const R* xb = xa + n;
    V v[N1];
    V u[N2];
#pragma unroll
    for (int m1 = 0; m1 < N1 / 2; ++m1) {
      const V pa = *reinterpret_cast<const V*>(xa + 2 * (N2 * m1 + t));
      const V pb = *reinterpret_cast<const V*>(xb + 2 * (N2 * m1 + t));
      v[m1] = mk2(pa.x, pb.x);
      v[N1 - 1 - m1] = mk2(__shfl_sync(0xffffffffu, pa.y, mirror), __shfl_sync(0xffffffffu, pb.y, mirror));
    }
    __syncwarp();
    pending = issue(next);  // the next item's rows arrive while this one is transformed
    const int row = (seg + item - I.row0) * 2 * LPW + 2 * sub;
    R* ya = reinterpret_cast<R*>(I.t1) + (size_t)row * n;
    R* yb = ya + n;
    fft_line<N1, N2>(t, buf, tab, false, v, u);
#pragma unroll
    for (int r = 0; r < N2; ++r) {
      const V send = (t == 0) ? u[partner_reg<N2>(r, true)] : u[partner_reg<N2>(r, false)];
      const R px = __shfl_sync(0xffffffffu, send.x, src_lane);
      const R py = __shfl_sync(0xffffffffu, send.y, src_lane);
      if (t < N1) {
        const int k = t + N1 * rbrev<N2>(r);
        const V Z = u[r];
        const V A = mk2((R)0.5 * (Z.x + px), (R)0.5 * (Z.y - py));
        const V B = mk2((R)0.5 * (Z.y + py), (R)0.5 * (px - Z.x));
        const V w = spt[k];
        const R sk = ds(k);
        ya[k] = post2(A, w, sk);
        yb[k] = post2(B, w, sk);
      }
    }
    item = next;
  }
}

// Inverse DCT-III of rows 2p and 2p+1 of T -> d_hat: the inputs W^a + i W^b of the two
// rows go through one inverse FFT; its real and imaginary parts are the two rows.
template <class R, int N1, int N2>
__global__ __launch_bounds__(RT<R>::RW * 32, 1) void k_dct_rows_inv(Inst* insts, const int* row_inst, int seg,
                                                                     int items, unsigned extra, long long limit) {
  using G = RowGeom<R, N1, N2>;
  using V = typename G::V;
  constexpr int n = G::n, LPW = G::LPW, RW = G::RW;
  const DctScale<R> ds(n);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sbuf = reinterpret_cast<R*>(smem_raw);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, sub = lane / N2, t = lane % N2;
  R* data = sbuf + warp * G::WARP;
  R* buf = data + G::DATA + sub * N1 * (N2 + 1);
  if (items <= 0) return;
  const V* tab = load_row_tables<R, N1, N2>(sbuf, insts[row_inst[seg]]);
  const V* spt = tab + n;
  unsigned long long* bar =
      reinterpret_cast<unsigned long long*>(smem_raw + sizeof(R) * RW * G::WARP + sizeof(V) * G::TABLES) + warp;
  const int stride = gridDim.x * RW;
  if (lane == 0) mbar_init(bar);
  __syncwarp();
  auto issue = [&](int it) -> bool {
    if (it >= items) return false;
    const Inst& J = insts[row_inst[seg + it]];
    if (!J.active) return false;
    if (lane == 0)
      bulk_load(data, reinterpret_cast<const R*>(J.t1) + (size_t)(seg + it - J.row0) * G::DATA, sizeof(R) * G::DATA,
                extra, bar);
    return true;
  };
  unsigned phase = 0;
  // consecutive items go to consecutive blocks, so that a short list (a batch's last few
  // active instances) still spreads over every SM
  int item = warp * gridDim.x + blockIdx.x;
  bool pending = issue(item);
  const int mirror = (lane - t) + (t < N1 ? N1 - 1 - t : 0);
  while (item < items) {
    const int next = item + stride;
    if (!pending) {
      pending = issue(next);
      item = next;
      continue;
    }
    Inst& I = insts[row_inst[seg + item]];
    if (!mbar_wait(bar, phase, limit)) {
      wait_fault(I, bar, phase, lane, limit);
      return;
    }
    phase ^= 1;
    const R* Xa = data + sub * 2 * n;
    const R* Xb = Xa + n;
    V v[N1];
    V u[N2];
#pragma unroll
    for (int m1 = 0; m1 < N1; ++m1) {
      const int k = N2 * m1 + t;
      const V w = spt[k];
      const R sk = ds(k), snk = k == 0 ? (R)0 : ds(n - k);
      const V Wa = pre3(k, sk * Xa[k], k == 0 ? (R)0 : snk * Xa[n - k], w);
      const V Wb = pre3(k, sk * Xb[k], k == 0 ? (R)0 : snk * Xb[n - k], w);
      v[m1] = mk2(Wa.x - Wb.y, Wa.y + Wb.x);
    }
    __syncwarp();
    pending = issue(next);
    const int row = (seg + item - I.row0) * 2 * LPW + 2 * sub;
    R* xa = reinterpret_cast<R*>(I.dhat) + (size_t)row * n;
    R* xb = xa + n;
    fft_line<N1, N2>(t, buf, tab, true, v, u);
    // Output m = t + N1 k2 goes to x[2m] for m < n/2; its neighbour x[2m+1] is output
    // n-1-m, held by lane N1-1-t in the register of k2' = N2-1-k2: one shuffle and a
    // 16-byte store per pair.
#pragma unroll
    for (int r = 0; r < N2; ++r) {
      if (rbrev<N2>(r) >= N2 / 2) continue;
      const V other = u[rbrev<N2>(N2 - 1 - rbrev<N2>(r))];
      const R qa = __shfl_sync(0xffffffffu, other.x, mirror);
      const R qb = __shfl_sync(0xffffffffu, other.y, mirror);
      if (t < N1) {
        const int m = t + N1 * rbrev<N2>(r);
        *reinterpret_cast<V*>(xa + 2 * m) = mk2(u[r].x, qa);
        *reinterpret_cast<V*>(xb + 2 * m) = mk2(u[r].y, qb);
      }
    }
    item = next;
  }
}

// Column pass, one warp per column pair (LPW pairs per warp when a line takes fewer than 32
// lanes), so that the two FFTs and the exchanges between them stay inside the warp. A block
// of 8 warps owns CPB = 8 LPW consecutive column pairs: it copies their tile of n rows into
// shared memory with coalesced 16-byte cp.async (rows stored in Makhoul order, row m holding
// global row 2m for m < n/2 and 2(n-1-m)+1 above, so that the lanes of a line read
// consecutive rows), each warp transforms its pairs -- DCT-II (split N1 x N2), division by
// lambda, DCT-III (split N2 x N1, which takes the forward output in the lanes where it
// already lies) -- and the block writes the tile back in global row order. While the warps transform, the tile's
// space holds, per line, a 2n-double region: the step-3 transpose buffer, and the line's
// spectrum for the exchanges of X_k with X_{n-k}.
template <class R, int N1, int N2>
struct ColGeom {
  using V = typename RT<R>::V;
  static constexpr int n = N1 * N2, LPW = 32 / N2;
  static constexpr int CT = 256;                // threads per block
  static constexpr int CPB = (CT / 32) * LPW;   // column pairs per block
  static constexpr int CB = 2 * CPB;            // columns per block
  static constexpr int RS = CPB + 1;            // complex per tile row (odd: conflict-free line reads)
  static constexpr int TILE = 2 * n * RS;       // reals
  static constexpr int LINE = 2 * n;            // reals: a line's region (spectrum, transpose)
  static_assert(LINE >= N1 * (N2 + 1) && LINE >= N2 * (N1 + 1), "the transposes fit in a line's region");
  static_assert((CT / 32) * LPW * LINE <= TILE, "the lines' regions fit in the tile");
  static constexpr int TABLES = 7 * n;          // reals: step-2 twiddles (N1 x N2, N2 x N1), pt, cos
  static constexpr int SMEM = TILE + TABLES;    // reals
};

__device__ __forceinline__ int makhoul_inv(int i, int n) { return (i & 1) ? n - 1 - (i >> 1) : (i >> 1); }

// Persistent: each block copies the size's tables into shared memory once and then takes
// the column tiles blockIdx.x, blockIdx.x + gridDim.x, ... of the segment.
template <class R, int N1, int N2>
__global__ __launch_bounds__(ColGeom<R, N1, N2>::CT, RT<R>::COL_BLOCKS) void k_dct_cols(const Inst* insts, const int* col_inst,
                                                                        int seg, int items) {
  using GG = ColGeom<R, N1, N2>;
  using V = typename GG::V;
  constexpr int n = GG::n, CPB = GG::CPB, CB = GG::CB, RS = GG::RS, LPW = GG::LPW;
  const DctScale<R> ds(n);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sbuf = reinterpret_cast<R*>(smem_raw);
  V* tile = reinterpret_cast<V*>(sbuf);  // [m][pair], rows in Makhoul order
  if (items <= 0) return;
  V* stw = reinterpret_cast<V*>(sbuf + GG::TILE);  // step-2 twiddles, N1 x N2 split
  V* stw_sw = stw + n;                             // the same for the N2 x N1 split
  V* spt = stw_sw + n;                             // (cos, sin)(pi k / 2n)
  R* scos = reinterpret_cast<R*>(spt + n);         // cos(pi k / n)
  {
    const Inst& I0 = insts[col_inst[seg]];
    const double2* tw2 = I0.tw + (n >> 1);
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      const double2 a = __ldg(&tw2[e]), b = __ldg(&tw2[n + e]), c = __ldg(&I0.pt[e]);
      stw[e] = mk2((R)a.x, (R)a.y);
      stw_sw[e] = mk2((R)b.x, (R)b.y);
      spt[e] = mk2((R)c.x, (R)c.y);
      scos[e] = (R)__ldg(&I0.cosk[e]);
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, sub = lane / N2, t = lane % N2;
  const int cp = warp * LPW + sub;  // this lane group's column pair within the block
  R* buf = sbuf + (warp * LPW + sub) * GG::LINE;  // this line's region of the tile space
  V* zl = reinterpret_cast<V*>(buf);
  for (int b = blockIdx.x; b < items; b += gridDim.x) {
    const int item = seg + b;
    const Inst& I = insts[col_inst[item]];
    if (!I.active) continue;  // uniform over the block
    const int l0 = (item - I.col0) * CB, la = l0 + 2 * cp;
    R* T = reinterpret_cast<R*>(I.t1);
    // the previous tile's store has read the tile (and the tables are in place)
    __syncthreads();
    for (int e = threadIdx.x; e < n * CPB; e += GG::CT) {
      const int i = e / CPB, cc = e - i * CPB;
      const unsigned dst = smem_u32(&tile[makhoul_inv(i, n) * RS + cc]);
      if (sizeof(V) == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(T + (size_t)i * n + l0 + 2 * cc)
                     : "memory");
      else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(T + (size_t)i * n + l0 + 2 * cc)
                     : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    V v[N1];
    V u[N2];
    // forward DCT-II of the two columns (one complex line; samples in Makhoul order)
#pragma unroll
    for (int m1 = 0; m1 < N1; ++m1) v[m1] = tile[(N2 * m1 + t) * RS + cp];
    __syncthreads();  // the tile's space now holds the lines' regions
    fft_line<N1, N2>(t, buf, stw, false, v, u);
    // Z_k (k = t + N1 rbrev(r)) into the line's region, then each lane separates the two
    // spectra with Z_{n-k}, divides by lambda_kl (the (0,0) mode is dropped) and keeps
    // s_k U_k, which goes back to the region for the partner's DCT-III input
    __syncwarp();
    if (t < N1) {
#pragma unroll
      for (int r = 0; r < N2; ++r) zl[t + N1 * rbrev<N2>(r)] = u[r];
    }
    __syncwarp();
    if (t < N1) {
      // U = X / lambda for the 2 LG values of a group of LG coefficients with one division:
      // each lambda's reciprocal is the product of the other lambdas over the product of all
      // (every lambda lies in (0, 4], so the products neither overflow nor underflow; the
      // result is within about ten ulps of separate divisions, which cost several times the
      // time and instruction footprint: 95 -> 74 us per column pass at 8 x 1024^2)
      constexpr int LG = RT<R>::DIV_GROUP;
      const R cla = scos[la], clb = scos[la + 1];
#pragma unroll
      for (int r0 = 0; r0 < N2; r0 += LG) {
        R Xa[LG], Xb[LG], lam[2 * LG], sk[LG];
        bool zero[LG];
#pragma unroll
        for (int g = 0; g < LG; ++g) {
          const int r = r0 + g;
          const int k = t + N1 * rbrev<N2>(r);
          const V Z = u[r], P = zl[(n - k) & (n - 1)];
          const V A = mk2((R)0.5 * (Z.x + P.x), (R)0.5 * (Z.y - P.y));
          const V B = mk2((R)0.5 * (Z.y + P.y), (R)0.5 * (P.x - Z.x));
          const V w = spt[k];
          sk[g] = ds(k);
          Xa[g] = post2(A, w, sk[g]);
          Xb[g] = post2(B, w, sk[g]);
          const R ck = scos[k];
          zero[g] = (k == 0 && la == 0);  // the (0,0) mode is dropped
          lam[2 * g] = zero[g] ? (R)1 : (R)2 - (R)2 * ck * cla;
          lam[2 * g + 1] = (R)2 - (R)2 * ck * clb;
        }
        R pre[2 * LG + 1], suf[2 * LG + 1];
        pre[0] = (R)1;
        suf[2 * LG] = (R)1;
#pragma unroll
        for (int j = 0; j < 2 * LG; ++j) pre[j + 1] = pre[j] * lam[j];
#pragma unroll
        for (int j = 2 * LG - 1; j >= 0; --j) suf[j] = suf[j + 1] * lam[j];
        const R inv = (R)1 / pre[2 * LG];
#pragma unroll
        for (int g = 0; g < LG; ++g) {
          const R ia = (pre[2 * g] * suf[2 * g + 1]) * inv;
          const R ib = (pre[2 * g + 1] * suf[2 * g + 2]) * inv;
          const R Ua = zero[g] ? (R)0 : Xa[g] * ia;
          const R Ub = Xb[g] * ib;
          u[r0 + g] = mk2(sk[g] * Ua, sk[g] * Ub);
        }
      }
    }
    __syncwarp();
    if (t < N1) {
#pragma unroll
      for (int r = 0; r < N2; ++r) zl[t + N1 * rbrev<N2>(r)] = u[r];
    }
    __syncwarp();
    // inverse DCT-III of the two columns, split N2 x N1: lane t (< N1) takes the samples
    // k = t + N1 m1 it holds; U_{n-k} comes from the region
    V w2[N2];
    V x2[N1];
#pragma unroll
    for (int m1 = 0; m1 < N2; ++m1) {
      const int k = t < N1 ? t + N1 * m1 : 0;
      const V a = u[rbrev<N2>(m1)];
      const V bb = zl[(n - k) & (n - 1)];
      const V w = spt[k];
      const V Wa = pre3(k, a.x, bb.x, w), Wb = pre3(k, a.y, bb.y, w);
      w2[m1] = mk2(Wa.x - Wb.y, Wa.y + Wb.x);
    }
    __syncwarp();  // the region's spectrum is read: it becomes the transpose buffer
    fft_line<N2, N1>(t, buf, stw_sw, true, w2, x2);
    __syncthreads();  // every warp is done with its transpose buffer: the space is the tile again
    // output sample m = t + N2 rbrev<N1>(r) (Makhoul order) of both columns
#pragma unroll
    for (int r = 0; r < N1; ++r) tile[(t + N2 * rbrev<N1>(r)) * RS + cp] = x2[r];
    __syncthreads();
    for (int e = threadIdx.x; e < n * CPB; e += GG::CT) {
      const int i = e / CPB, cc = e - i * CPB;
      *reinterpret_cast<V*>(T + (size_t)i * n + l0 + 2 * cc) = tile[makhoul_inv(i, n) * RS + cc];
    }
  }
}

template <class R, int N1, int N2>
struct RegDct {
  static constexpr int LPW = 32 / N2, RW = RT<R>::RW;
  static size_t rows_smem() { return RowGeom<R, N1, N2>::SMEM; }
  static size_t cols_smem() { return sizeof(R) * ColGeom<R, N1, N2>::SMEM; }
  static constexpr int CB = ColGeom<R, N1, N2>::CB;
  static int rows_blocks_per_sm;  // occupancy of the row kernels (set by attrs)
  static int cols_blocks_per_sm;  // occupancy of the column kernel
  static void attrs() {
    OTM_CUDA(cudaFuncSetAttribute(k_dct_rows_fwd<R, N1, N2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)rows_smem()));
    OTM_CUDA(cudaFuncSetAttribute(k_dct_rows_inv<R, N1, N2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)rows_smem()));
    OTM_CUDA(cudaFuncSetAttribute(k_dct_cols<R, N1, N2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)cols_smem()));
    int a = 0, b = 0;
    OTM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_dct_rows_fwd<R, N1, N2>, RW * 32, rows_smem()));
    OTM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_dct_rows_inv<R, N1, N2>, RW * 32, rows_smem()));
    rows_blocks_per_sm = std::max(1, std::min(a, b));
    OTM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_dct_cols<R, N1, N2>, 256, cols_smem()));
    cols_blocks_per_sm = std::max(1, a);
  }
  static void run(otm_context* ctx, Inst* d, const int* ri, int roff, int rcnt, const int* ci, int coff, int ccnt) {
    const int grid = std::max(1, std::min((rcnt + RW - 1) / RW, rows_blocks_per_sm * ctx->num_sms));
    const unsigned extra = ctx->wait_test ? 16u : 0u;
    const long long limit = ctx->wait_test ? kTestWaitCycles : kWaitCycles;
    constexpr bool f = sizeof(R) == 4;
    launch_smem(ctx, f ? "dct32_rows_fwd" : "dct_rows_fwd", k_dct_rows_fwd<R, N1, N2>, grid, RW * 32, rows_smem(), d, ri, roff, rcnt, extra,
                limit);
    const int cgrid = std::max(1, std::min(ccnt, cols_blocks_per_sm * ctx->num_sms));
    launch_smem(ctx, f ? "dct32_cols" : "dct_cols", k_dct_cols<R, N1, N2>, cgrid, 256, cols_smem(), (const Inst*)d, ci, coff, ccnt);
    launch_smem(ctx, f ? "dct32_rows_inv" : "dct_rows_inv", k_dct_rows_inv<R, N1, N2>, grid, RW * 32, rows_smem(), d, ri, roff, rcnt, extra,
                limit);
  }
};
template <class R, int N1, int N2>
int RegDct<R, N1, N2>::rows_blocks_per_sm = 1;
template <class R, int N1, int N2>
int RegDct<R, N1, N2>::cols_blocks_per_sm = 1;

}  // namespace

bool dct_reg_supported(int n) { return n == 64 || n == 128 || n == 256 || n == 512 || n == 1024; }

namespace {
template <int N1, int N2>
void step2_table(const std::vector<double2>& tw, std::vector<double2>& out) {
  constexpr int n = N1 * N2;
  out.resize(n);
  for (int r = 0; r < N1; ++r)
    for (int t = 0; t < N2; ++t) {
      // the entry of the half table tw (k < n/2), negated in the upper half: the same
      // value the transform would form from tw itself
      const int e = (t * rbrev<N1>(r)) & (n - 1);
      double2 w = e < n / 2 ? tw[e] : make_double2(-tw[e - n / 2].x, -tw[e - n / 2].y);
      out[(size_t)r * N2 + t] = w;
    }
}
}  // namespace

void dct_reg_step2_table(int n, const std::vector<double2>& tw, std::vector<double2>& out) {
  std::vector<double2> sw;
  switch (n) {
    case 64: step2_table<8, 8>(tw, out); step2_table<8, 8>(tw, sw); break;
    case 128: step2_table<8, 16>(tw, out); step2_table<16, 8>(tw, sw); break;
    case 256: step2_table<16, 16>(tw, out); step2_table<16, 16>(tw, sw); break;
    case 512: step2_table<16, 32>(tw, out); step2_table<32, 16>(tw, sw); break;
    case 1024: step2_table<32, 32>(tw, out); step2_table<32, 32>(tw, sw); break;
    default: out.clear();
  }
  out.insert(out.end(), sw.begin(), sw.end());
}

int dct_reg_lines_per_block(int n) {  // rows per row-pass work item: two per FFT line of a warp
  switch (n) {
    case 64: return 2 * RegDct<double, 8, 8>::LPW;
    case 128: return 2 * RegDct<double, 8, 16>::LPW;
    case 256: return 2 * RegDct<double, 16, 16>::LPW;
    case 512: return 2 * RegDct<double, 16, 32>::LPW;
    default: return 2 * RegDct<double, 32, 32>::LPW;
  }
}

int dct_reg_cols_per_block(int n) {
  switch (n) {
    case 64: return RegDct<double, 8, 8>::CB;
    case 128: return RegDct<double, 8, 16>::CB;
    case 256: return RegDct<double, 16, 16>::CB;
    case 512: return RegDct<double, 16, 32>::CB;
    default: return RegDct<double, 32, 32>::CB;
  }
}

void dct_reg_attrs(int device) {
  static bool done[64] = {};
  if (device < 64 && done[device]) return;
  {
    std::vector<double2> tw(CTW / 2);
    std::vector<float2> twf(CTW / 2);
    for (int k = 0; k < CTW / 2; ++k) {
      tw[k] = make_double2(std::cos(2.0 * M_PI * k / CTW), -std::sin(2.0 * M_PI * k / CTW));
      twf[k] = make_float2((float)tw[k].x, (float)tw[k].y);
    }
    OTM_CUDA(cudaMemcpyToSymbol(c_tw, tw.data(), sizeof(double2) * (CTW / 2)));
    OTM_CUDA(cudaMemcpyToSymbol(c_twf, twf.data(), sizeof(float2) * (CTW / 2)));
  }
  RegDct<double, 8, 8>::attrs();
  RegDct<double, 8, 16>::attrs();
  RegDct<double, 16, 16>::attrs();
  RegDct<double, 16, 32>::attrs();
  RegDct<double, 32, 32>::attrs();
  RegDct<float, 8, 8>::attrs();
  RegDct<float, 8, 16>::attrs();
  RegDct<float, 16, 16>::attrs();
  RegDct<float, 16, 32>::attrs();
  RegDct<float, 32, 32>::attrs();
  if (device < 64) done[device] = true;
}

template <class R>
static void dct_reg_run_t(otm_context* ctx, int n, Inst* d, const int* ri, int roff, int rcnt, const int* ci, int coff,
                          int ccnt) {
  switch (n) {
    case 64: RegDct<R, 8, 8>::run(ctx, d, ri, roff, rcnt, ci, coff, ccnt); break;
    case 128: RegDct<R, 8, 16>::run(ctx, d, ri, roff, rcnt, ci, coff, ccnt); break;
    case 256: RegDct<R, 16, 16>::run(ctx, d, ri, roff, rcnt, ci, coff, ccnt); break;
    case 512: RegDct<R, 16, 32>::run(ctx, d, ri, roff, rcnt, ci, coff, ccnt); break;
    case 1024: RegDct<R, 32, 32>::run(ctx, d, ri, roff, rcnt, ci, coff, ccnt); break;
    default: throw BadArg{"dct_reg_run: unsupported size"};
  }
}

void dct_reg_run(otm_context* ctx, int n, bool fp32, Inst* d_insts, const int* row_inst, int roff, int rcnt,
                 const int* col_inst, int coff, int ccnt) {
  dct_reg_attrs(ctx->device);
  if (fp32)
    dct_reg_run_t<float>(ctx, n, d_insts, row_inst, roff, rcnt, col_inst, coff, ccnt);
  else
    dct_reg_run_t<double>(ctx, n, d_insts, row_inst, roff, rcnt, col_inst, coff, ccnt);
}

}  // namespace otm
