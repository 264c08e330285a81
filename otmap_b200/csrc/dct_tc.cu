// The cosine-transform Poisson solve on the tensor cores (tcgen05, sm_100a), for the
// split-precision mode (FP32 arrays): d_hat = C^T ((C R C^T) / lambda) C with C the
// orthonormal DCT-II matrix (otsolver_2dgrid.cpp:175-179; the (0,0) mode dropped = the
// mean-zero projection of :179), as four dense products per solve:
//   stage 0  U  = R C^T        A = R      B = C     stored transposed (T1[l][i] = U[i][l])
//   stage 1  X  = C U          A = C      B = T1    Y = X / lambda, stored transposed (T2)
//   stage 2  W  = C^T Y        A = C^T    B = T2    stored as is (T1)
//   stage 3  d  = W C          A = T1     B = C^T   stored as is (d_hat, FP32)
// Every product is D[m][n] = sum_k A[m][k] B[n][k] with both operands K-major (row m of A
// and row n of B hold their k values contiguously), which is why the first two products
// store their results transposed.
//
// 3xTF32: every operand value x is held as two TF32 planes, hi = x rounded to TF32 and
// lo = (x - hi) rounded to TF32 (|x - hi - lo| <= 2^-22 |x|), and a product is
// hi*hi + hi*lo + lo*hi accumulated in FP32. The planes are written once per value: the
// basis C and C^T at init, R by k_tc_split before stage 0, the intermediates by the
// epilogue of the stage that produces them. The tensor core rounds each accumulation into
// its FP32 accumulator with a bias (the error of the first-step transform grows linearly
// with the number of accumulations), so the two small correction products go to a second
// accumulator and the large one takes one accumulation per K = 8 only; the epilogue adds
// the two.
//
// A CTA of 128 threads computes one 128 x TN output tile (TN = 256, or 128 for n = 128) in
// tensor memory: main accumulator in columns [0, TN), correction in [256, 256 + TN).
// Thread 0 is the producer: it streams 128 x 32 slices of A and TN x 32 slices of B (hi
// and lo planes) into a two-stage shared-memory ring with TMA (2-D tiled loads, 128-byte
// rows, 128-byte swizzle, no multicast), each stage completing an mbarrier with its
// transaction bytes. Thread 32 issues tcgen05.mma kind::tf32 (M = 128, N = TN, K = 8) on
// the swizzled K-major layout (8-row groups 1024 bytes apart; the K offset within the
// 128-byte row advances the start address by 32 bytes) and frees each stage with
// tcgen05.commit on its "empty" mbarrier, then commits the last products to "done". All
// four warps run the epilogue: tcgen05.ld of 32 lanes x 32 columns per warp and step.
// Every wait is bounded; a wait that runs out flags the instance (Inst::fault) and stops
// it, the CTA waits (again bounded) for the loads and products in flight, frees the
// tensor memory and returns. OTM_OPT_WAIT_TEST makes the stage barriers expect bytes that
// never arrive, so that this path runs without any fault.

#include <cuda.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "engine.cuh"

namespace otm {
namespace {

constexpr int TM = 128, TK = 32, TN_MAX = 256;   // CTA tile (TN runtime: 256 or 128), K slice
constexpr int STAGES = 2;
constexpr int A_BYTES = TM * TK * 4;             // one plane of an A slice (16 KB)
constexpr int B_BYTES = TN_MAX * TK * 4;         // one plane of a B slice (32 KB)
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
constexpr int CTL_BYTES = 128;                   // mbarriers and control words
constexpr int SMEM = 1024 + STAGES * STAGE_BYTES + CTL_BYTES;  // + alignment slack
constexpr int TMEM_COLS = 512, CORR_COL = 256;
constexpr long long kTcWait = 2000000000LL;      // ~1 s at the B200's clock
constexpr long long kTcTestWait = 2000000LL;     // ~1 ms (OTM_OPT_WAIT_TEST)

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor of a K-major operand in the 128-byte swizzled layout:
// start address, leading offset 16 bytes (unused for this layout), stride offset 1024
// bytes between 8-row groups, descriptor version 1, layout type SWIZZLE_128B (2).
__device__ __forceinline__ unsigned long long smem_desc_sw128(unsigned addr) {
  return (unsigned long long)((addr >> 4) & 0x3FFFu) | (1ull << 16) | ((unsigned long long)(1024 >> 4) << 32) |
         (1ull << 46) | (2ull << 61);
}

// Instruction descriptor: FP32 accumulator, TF32 A and B, both K-major, M = 128, N = tn.
__device__ __forceinline__ unsigned idesc_tf32(int tn) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(tn >> 3) << 17) | ((unsigned)(TM >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(unsigned tmem_d, unsigned long long da, unsigned long long db, unsigned idesc,
                                         unsigned acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void mma_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool bar_wait(unsigned long long* bar, unsigned parity, long long limit) {
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

__device__ __forceinline__ void bar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// 2-D tiled TMA load of the box at (x, y) = (column, row) of the map into shared memory,
// completing its bytes on the mbarrier's transaction count.
__device__ __forceinline__ void tma_load_2d(unsigned dst, const CUtensorMap* map, int x, int y, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// 32 consecutive FP32 columns of this thread's accumulator row (warp w reads lanes
// 32w .. 32w+31).
__device__ __forceinline__ void tmem_ld32(unsigned addr, float (&v)[32]) {
  unsigned r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}

// Nearest TF32 value of x (10 mantissa bits), as an FP32 bit pattern.
__device__ __forceinline__ float to_tf32(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// The hi and lo TF32 planes of the residual R (FP32, from the sweep) for stage 0. Work
// item t of an instance splits cells [t E, (t+1) E), E = n^2 / items.
// Each work item is split by SPLIT_PARTS blocks; the loop keeps four loads in flight per
// thread.
constexpr int SPLIT_PARTS = 2;
__global__ __launch_bounds__(256) void k_tc_split(Inst* insts, const int* tc_inst, int base) {
  const int item = base + blockIdx.x / SPLIT_PARTS, part = blockIdx.x % SPLIT_PARTS;
  const Inst& I = insts[tc_inst[item]];
  if (!I.active) return;
  const size_t nn = (size_t)I.n * I.n, E = nn / I.ntc / SPLIT_PARTS;
  const size_t e0 = (size_t)(item - I.tc0) * E * SPLIT_PARTS + (size_t)part * E;
  const float4* r = reinterpret_cast<const float4*>(reinterpret_cast<const float*>(I.r[I.it % 3]) + e0);
  float4* hi = reinterpret_cast<float4*>(I.rs + e0);
  float4* lo = reinterpret_cast<float4*>(I.rs + nn + e0);
#pragma unroll 4
  for (size_t k = threadIdx.x; k < E / 4; k += blockDim.x) {
    const float4 x = r[k];
    float4 h, l;
    h.x = to_tf32(x.x);
    h.y = to_tf32(x.y);
    h.z = to_tf32(x.z);
    h.w = to_tf32(x.w);
    l.x = to_tf32(x.x - h.x);
    l.y = to_tf32(x.y - h.y);
    l.z = to_tf32(x.z - h.z);
    l.w = to_tf32(x.w - h.w);
    hi[k] = h;
    lo[k] = l;
  }
}

// One 128 x TN output tile of stage `stage` for the instance owning work item blockIdx.x.
// extra: bytes added to every stage's expected transaction count (0; 16 under
// OTM_OPT_WAIT_TEST, so that no stage ever completes and every wait runs out after
// `limit`, by which time the real copies have landed: nothing is in flight at exit).
__global__ __launch_bounds__(128, 1) void k_dct_tc(Inst* insts, const int* tc_inst, int base, int stage,
                                                   unsigned extra, long long limit) {
  extern __shared__ unsigned char sm_raw[];
  const int item = base + blockIdx.x;
  Inst& I = insts[tc_inst[item]];
  if (!I.active) return;
  const int n = I.n, TN = I.tcn, tiles_n = n / TN;
  const int t = item - I.tc0, tm = t / tiles_n, tn = t - tm * tiles_n;
  const size_t nn = (size_t)n * n;
  // 1024-byte aligned stages (the 128-byte swizzle repeats every 8 rows of 128 bytes)
  const unsigned raw = smem_u32(sm_raw), sbase = (raw + 1023u) & ~1023u;
  unsigned char* ctl_p = sm_raw + (sbase - raw) + STAGES * STAGE_BYTES;
  unsigned long long* full = reinterpret_cast<unsigned long long*>(ctl_p);
  unsigned long long* empty = full + STAGES;
  unsigned long long* done = empty + STAGES;
  volatile int* ctl = reinterpret_cast<volatile int*>(done + 1);  // tmem, fault, issued, consumed
  const CUtensorMap* maps = reinterpret_cast<const CUtensorMap*>(I.tmaps) + 4 * stage;  // A hi, A lo, B hi, B lo
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32((const void*)ctl)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 32) {
    for (int s = 0; s < STAGES; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(full + s)) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(empty + s)) : "memory");
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(done)) : "memory");
    ctl[1] = 0;
    ctl[2] = 0;
    ctl[3] = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = (unsigned)ctl[0], tmem_corr = tmem + (unsigned)CORR_COL;
  const int slices = n / TK;

  if (warp == 0) {
    if (lane == 0) {  // producer
      const unsigned tx = 2u * (unsigned)(A_BYTES + TN * TK * 4) + extra;
      int i = 0;
      for (; i < slices; ++i) {
        const int s = i % STAGES;
        if (i >= STAGES && !bar_wait(empty + s, (unsigned)((i / STAGES - 1) & 1), limit)) {
          ctl[1] = 1;
          break;
        }
        const unsigned st = sbase + (unsigned)(s * STAGE_BYTES);
        bar_expect_tx(full + s, tx);
        tma_load_2d(st, maps + 0, i * TK, tm * TM, full + s);
        tma_load_2d(st + A_BYTES, maps + 1, i * TK, tm * TM, full + s);
        tma_load_2d(st + 2 * A_BYTES, maps + 2, i * TK, tn * TN, full + s);
        tma_load_2d(st + 2 * A_BYTES + B_BYTES, maps + 3, i * TK, tn * TN, full + s);
      }
      ctl[2] = i;
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      const unsigned idesc = idesc_tf32(TN);
      int i = 0;
      for (; i < slices; ++i) {
        const int s = i % STAGES;
        if (!bar_wait(full + s, (unsigned)((i / STAGES) & 1), limit)) {
          ctl[1] = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const unsigned st = sbase + (unsigned)(s * STAGE_BYTES);
#pragma unroll
        for (int q = 0; q < TK / 8; ++q) {  // K = 8 TF32 = 32 bytes of each 128-byte row
          const unsigned off = (unsigned)(q * 32);
          const unsigned long long ah = smem_desc_sw128(st + off), al = smem_desc_sw128(st + A_BYTES + off);
          const unsigned long long bh = smem_desc_sw128(st + 2 * A_BYTES + off);
          const unsigned long long bl = smem_desc_sw128(st + 2 * A_BYTES + B_BYTES + off);
          const unsigned acc = (i > 0 || q > 0) ? 1u : 0u;
          mma_tf32(tmem, ah, bh, idesc, acc);
          mma_tf32(tmem_corr, ah, bl, idesc, acc);
          mma_tf32(tmem_corr, al, bh, idesc, 1u);
        }
        mma_commit(empty + s);  // the stage is free once these products have read it
      }
      ctl[3] = i;
      mma_commit(done);  // completes once every product issued above has
    }
    __syncwarp();
  }
  __syncthreads();
  // loads issued but not consumed (after a timeout): wait for them before the CTA exits
  if (threadIdx.x == 0)
    for (int i = ctl[3]; i < ctl[2]; ++i)
      if (!bar_wait(full + (i % STAGES), (unsigned)((i / STAGES) & 1), limit)) ctl[1] = 1;
  const bool fin = bar_wait(done, 0u, limit);
  const bool ok = __syncthreads_and(fin && ctl[1] == 0) != 0;
  if (!ok) {
    if (threadIdx.x == 0) {
      atomicExch(&I.fault, 1);
      I.active = 0;
    }
  } else {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int m = tm * TM + warp * 32 + lane;  // this thread's output row
    const unsigned lane_off = (unsigned)(warp * 32) << 16;
    float* T1 = reinterpret_cast<float*>(I.t1);
    float* T2 = reinterpret_cast<float*>(I.t2);
    const float ck = stage == 1 ? (float)I.cosk[m] : 0.f;
#pragma unroll 1
    for (int c0 = 0; c0 < TN; c0 += 32) {
      float v[32], w[32];
      tmem_ld32(tmem + lane_off + (unsigned)c0, v);
      tmem_ld32(tmem_corr + lane_off + (unsigned)c0, w);
#pragma unroll
      for (int q = 0; q < 32; ++q) v[q] += w[q];
      const int n0 = tn * TN + c0;
      if (stage == 0 || stage == 1) {
        float* hi = stage == 0 ? T1 : T2;
        float* lo = hi + nn;
#pragma unroll
        for (int q = 0; q < 32; ++q) {
          float x = v[q];
          if (stage == 1) {
            const int l = n0 + q;
            const float lam = 2.0f - 2.0f * ck * (float)I.cosk[l];
            x = (m == 0 && l == 0) ? 0.0f : x / lam;
          }
          const float h = to_tf32(x);
          // transposed: the warp's 32 rows are 32 consecutive floats of row n0 + q
          hi[(size_t)(n0 + q) * n + m] = h;
          lo[(size_t)(n0 + q) * n + m] = to_tf32(x - h);
        }
      } else if (stage == 2) {
        float* hi = T1 + (size_t)m * n + n0;
        float* lo = hi + nn;
#pragma unroll
        for (int q = 0; q < 32; q += 4) {
          float4 h, l;
          h.x = to_tf32(v[q]);
          h.y = to_tf32(v[q + 1]);
          h.z = to_tf32(v[q + 2]);
          h.w = to_tf32(v[q + 3]);
          l.x = to_tf32(v[q] - h.x);
          l.y = to_tf32(v[q + 1] - h.y);
          l.z = to_tf32(v[q + 2] - h.z);
          l.w = to_tf32(v[q + 3] - h.w);
          *reinterpret_cast<float4*>(hi + q) = h;
          *reinterpret_cast<float4*>(lo + q) = l;
        }
      } else {
        float* out = reinterpret_cast<float*>(I.dhat) + (size_t)m * n + n0;
#pragma unroll
        for (int q = 0; q < 32; q += 4)
          *reinterpret_cast<float4*>(out + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

// The driver's tensor-map encoder, looked up once (a thread-safe static initialisation;
// a failed lookup throws and is retried on the next call).
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    OTM_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !p) throw std::runtime_error("cuTensorMapEncodeTiled is not available");
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// Map of one n x n FP32 plane (row-major) read in boxes of 32 columns (128 bytes) x rows.
void encode_plane(CUtensorMap* m, const float* plane, int n, int rows) {
  const cuuint64_t dim[2] = {(cuuint64_t)n, (cuuint64_t)n};
  const cuuint64_t stride[1] = {(cuuint64_t)n * sizeof(float)};
  const cuuint32_t box[2] = {(cuuint32_t)TK, (cuuint32_t)rows};
  const cuuint32_t es[2] = {1, 1};
  const CUresult r = encode_fn()(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(plane), dim, stride, box, es,
                                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw std::runtime_error("cuTensorMapEncodeTiled failed for a transform plane");
}

}  // namespace

bool dct_tc_supported(int n) { return n == 128 || n == 256 || n == 512 || n == 1024; }

int dct_tc_tn(int n) { return n >= TN_MAX ? TN_MAX : 128; }

int dct_tc_tiles(int n) { return (n / TM) * (n / dct_tc_tn(n)); }

size_t dct_tc_map_bytes() { return 16 * sizeof(CUtensorMap); }

void dct_tc_encode(const Inst& I, void* host_maps) {
  CUtensorMap m[16];  // 64-byte aligned for the encoder; copied out below
  const int n = I.n, TN = I.tcn;
  const size_t nn = (size_t)n * n;
  const float* T1 = reinterpret_cast<const float*>(I.t1);
  const float* T2 = reinterpret_cast<const float*>(I.t2);
  const float* A[4] = {I.rs, I.Cf, I.CTf, T1};  // hi planes; the lo plane follows at + n^2
  const float* B[4] = {I.Cf, T1, T2, I.CTf};
  for (int s = 0; s < 4; ++s) {
    encode_plane(m + 4 * s + 0, A[s], n, TM);
    encode_plane(m + 4 * s + 1, A[s] + nn, n, TM);
    encode_plane(m + 4 * s + 2, B[s], n, TN);
    encode_plane(m + 4 * s + 3, B[s] + nn, n, TN);
  }
  std::memcpy(host_maps, m, sizeof(m));
}

void dct_tc_split_basis(const double* C, int n, std::vector<float>& cs, std::vector<float>& cts) {
  // nearest TF32 value, ties away from zero (as cvt.rna), of a finite float below 2^127
  auto tf32 = [](float x) {
    unsigned u;
    std::memcpy(&u, &x, 4);
    u = (u + 0x1000u) & 0xFFFFE000u;
    float y;
    std::memcpy(&y, &u, 4);
    return y;
  };
  const size_t nn = (size_t)n * n;
  cs.assign(2 * nn, 0.f);
  cts.assign(2 * nn, 0.f);
  for (int k = 0; k < n; ++k)
    for (int i = 0; i < n; ++i) {
      const double c = C[(size_t)k * n + i];
      const float h = tf32((float)c);
      const float l = tf32((float)(c - (double)h));
      cs[(size_t)k * n + i] = h;
      cs[nn + (size_t)k * n + i] = l;
      cts[(size_t)i * n + k] = h;
      cts[nn + (size_t)i * n + k] = l;
    }
}

void dct_tc_attrs(int device) {
  static bool done[64] = {};
  if (device < 64 && done[device]) return;
  OTM_CUDA(cudaFuncSetAttribute(k_dct_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
  if (device < 64) done[device] = true;
}

void dct_tc_run(otm_context* ctx, Inst* d_insts, const int* tc_inst, int base, int count) {
  dct_tc_attrs(ctx->device);
  if (count <= 0) return;
  launch(ctx, "dct_tc_split", k_tc_split, count * SPLIT_PARTS, 256, d_insts, tc_inst, base);
  const unsigned extra = ctx->wait_test ? 16u : 0u;
  const long long limit = ctx->wait_test ? kTcTestWait : kTcWait;
  for (int s = 0; s < 4; ++s)
    launch_smem(ctx, "dct_tc", k_dct_tc, count, 128, SMEM, d_insts, tc_inst, base, s, extra, limit);
}

}  // namespace otm
