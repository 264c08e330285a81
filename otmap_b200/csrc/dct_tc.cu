// The cosine-transform Poisson solve on the tensor cores (tcgen05, sm_100a), for the
// split-precision mode (FP32 arrays): d_hat = C^T ((C R C^T) / lambda) C with C the
// orthonormal DCT-II matrix (otsolver_2dgrid.cpp:175-179; the (0,0) mode dropped = the
// mean-zero projection of :179), as four dense products per solve:
//   stage 0  U  = R C^T        A = R      B = C     stored transposed (T1[l][i] = U[i][l])
//   stage 1  X  = C U          A = C      B = T1    Y = X / lambda, stored transposed (T2)
//   stage 2  W  = C^T Y        A = C^T    B = T2    stored as is (T1)
//   stage 3  d  = W C          A = T1     B = C^T   stored as is (d_hat)
// Every product is D[m][n] = sum_k A[m][k] B[n][k] with both operands K-major (row m of A
// and row n of B hold their k values contiguously), which is why the first two products
// store their results transposed. A CTA of 128 threads computes one 128 x 128 tile of D
// in tensor memory (128 lanes x 128 FP32 columns): it stages 128 x 32 slices of A and B in
// shared memory in the canonical no-swizzle K-major layout (8-row x 16-byte core
// matrices), each value split into its nearest TF32 value and the TF32-rounded remainder,
// and one thread issues tcgen05.mma kind::tf32 (M = 128, N = 128, K = 8) for the products
// hi*hi + hi*lo + lo*hi ("3xTF32": about FP32 accuracy). The tensor core rounds each
// accumulation into its FP32 accumulator with a bias (the error of the first-step
// transform grows linearly with the number of accumulations), so the two small correction
// products go to a second accumulator (columns 128..255) and the large one takes one
// accumulation per K = 8 only; the epilogue adds the two. Slices are double-buffered: the
// threads stage slice s+1 while the products of slice s run. Completion is signalled by
// tcgen05.commit on one mbarrier per buffer; every wait is bounded and a wait that runs
// out (block-uniformly) flags the instance (Inst::fault) and stops it, waits for the
// products in flight, frees the tensor memory and returns. The epilogue reads the
// accumulators with tcgen05.ld (32 lanes x 32 columns per warp and step).

#include <cmath>

#include "engine.cuh"

namespace otm {
namespace {

constexpr int TCM = 128, TCN = 128, TCK = 32;   // CTA tile and K slice
constexpr int CORE = 128;                        // bytes of a core matrix (8 rows x 16 bytes)
constexpr int LBO = CORE;                        // next core matrix along K
constexpr int SBO = (TCK / 4) * CORE;            // next 8-row group
constexpr int SLICE = TCM * TCK * 4;             // bytes of one operand slice (16 KB)
constexpr int STAGES = 2;                        // slice buffers (A hi/lo, B hi/lo each)
constexpr int BUF = 4 * SLICE;
constexpr int SMEM = STAGES * BUF + 64;          // buffers, one mbarrier per buffer, tmem address
constexpr int TMEM_COLS = 2 * TCN;               // main and correction accumulators
constexpr long long kTcWait = 2000000000LL;      // ~1 s at the B200's clock

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: start address, leading (K) and stride (M/N) byte
// offsets in 16-byte units, descriptor version 1, no swizzle.
__device__ __forceinline__ unsigned long long smem_desc(unsigned addr) {
  return (unsigned long long)((addr >> 4) & 0x3FFFu) | ((unsigned long long)((LBO >> 4) & 0x3FFF) << 16) |
         ((unsigned long long)((SBO >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Instruction descriptor: FP32 accumulator, TF32 A and B, both K-major, N = 128, M = 128.
constexpr unsigned kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(TCN >> 3) << 17) | ((unsigned)(TCM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(unsigned tmem_d, unsigned long long da, unsigned long long db, unsigned acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdesc), "r"(acc)
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

// Offset of (row r, K chunk c of 4 values) in a staged slice.
__device__ __forceinline__ int core_off(int r, int c) { return (r >> 3) * SBO + c * LBO + (r & 7) * 16; }

// Nearest TF32 value of x (10 mantissa bits), as an FP32 bit pattern.
__device__ __forceinline__ float to_tf32(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Stages a 128 x 32 slice of the K-major operand M (row stride n) starting at (row0, k0):
// high part = x rounded to TF32, low part = the remainder rounded to TF32 (|x - hi - lo|
// <= 2^-22 |x|). Thread e of a pass takes row (e>>6)*8 + (e&7), chunk (e>>3)&7: the 8
// threads of a quarter-warp write 8 consecutive rows of one core matrix (128 contiguous
// bytes, no bank conflict) and read 16 bytes each from 8 rows, 64 bytes per row per warp.
__device__ __forceinline__ void stage_slice(const float* M, int n, int row0, int k0, unsigned char* hi,
                                            unsigned char* lo) {
  for (int e = threadIdx.x; e < TCM * (TCK / 4); e += blockDim.x) {
    const int r = ((e >> 6) << 3) | (e & 7), c = (e >> 3) & 7;
    const float4 x = *reinterpret_cast<const float4*>(M + (size_t)(row0 + r) * n + k0 + 4 * c);
    float4 h, l;
    h.x = to_tf32(x.x);
    h.y = to_tf32(x.y);
    h.z = to_tf32(x.z);
    h.w = to_tf32(x.w);
    l.x = to_tf32(x.x - h.x);
    l.y = to_tf32(x.y - h.y);
    l.z = to_tf32(x.z - h.z);
    l.w = to_tf32(x.w - h.w);
    const int o = core_off(r, c);
    *reinterpret_cast<float4*>(hi + o) = h;
    *reinterpret_cast<float4*>(lo + o) = l;
  }
}

// One 128 x 128 output tile of stage `stage` for the instance owning work item blockIdx.x.
__global__ __launch_bounds__(128, 1) void k_dct_tc(Inst* insts, const int* tc_inst, int base, int stage,
                                                   long long limit) {
  extern __shared__ __align__(128) unsigned char sm[];
  const int item = base + blockIdx.x;
  Inst& I = insts[tc_inst[item]];
  if (!I.active) return;
  const int n = I.n, tiles = n / TCM;
  const int t = item - I.tc0, tm = t / tiles, tn = t - (t / tiles) * tiles;
  const float* R = reinterpret_cast<const float*>(I.r[I.it % 3]);
  float* T1 = reinterpret_cast<float*>(I.t1);
  float* T2 = reinterpret_cast<float*>(I.t2);
  const float* A;
  const float* B;
  switch (stage) {
    case 0: A = R; B = I.Cf; break;
    case 1: A = I.Cf; B = T1; break;
    case 2: A = I.CTf; B = T2; break;
    default: A = T1; B = I.CTf; break;
  }
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(sm + STAGES * BUF);
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(sm + STAGES * BUF + 8 * STAGES);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    for (int b = 0; b < STAGES; ++b)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar + b)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = *tmem_slot, tmem_corr = tmem + (unsigned)TCN;
  bool ok = true;
  unsigned phase[STAGES] = {};
  bool pending[STAGES] = {};
  for (int s = 0, k0 = 0; k0 < n; ++s, k0 += TCK) {
    const int b = s % STAGES;
    unsigned char* a_hi = sm + b * BUF;
    unsigned char* a_lo = a_hi + SLICE;
    unsigned char* b_hi = a_hi + 2 * SLICE;
    unsigned char* b_lo = a_hi + 3 * SLICE;
    if (pending[b]) {  // the buffer is reused: wait for the products that read it
      ok = __syncthreads_and(bar_wait(bar + b, phase[b], limit) ? 1 : 0) != 0;
      if (!ok) break;  // still pending: waited for once more below
      phase[b] ^= 1u;
      pending[b] = false;
    }
    stage_slice(A, n, tm * TCM, k0, a_hi, a_lo);
    stage_slice(B, n, tn * TCN, k0, b_hi, b_lo);
    // generic-proxy writes to shared memory become visible to the tensor core's reads
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int q = 0; q < TCK / 8; ++q) {  // K = 8 per instruction: two core matrices along K
        const unsigned off = (unsigned)(q * 2 * LBO);
        const unsigned long long ah = smem_desc(smem_u32(a_hi) + off), al = smem_desc(smem_u32(a_lo) + off);
        const unsigned long long bh = smem_desc(smem_u32(b_hi) + off), bl = smem_desc(smem_u32(b_lo) + off);
        const unsigned first = (k0 > 0 || q > 0) ? 1u : 0u;
        mma_tf32(tmem, ah, bh, first);
        mma_tf32(tmem_corr, ah, bl, first);
        mma_tf32(tmem_corr, al, bh, 1u);
      }
      mma_commit(bar + b);
    }
    pending[b] = true;
  }
  // the products in flight (all of them once ok; after a timeout, one more bounded wait each)
  for (int b = 0; b < STAGES; ++b)
    if (pending[b]) {
      const bool w = __syncthreads_and(bar_wait(bar + b, phase[b], limit) ? 1 : 0) != 0;
      ok = ok && w;
    }
  if (!ok) {
    if (threadIdx.x == 0) {
      atomicExch(&I.fault, 1);
      I.active = 0;
    }
  } else {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int m = tm * TCM + warp * 32 + lane;  // this thread's output row
    const unsigned lane_off = (unsigned)(warp * 32) << 16;
    float ck = 0.f;
    if (stage == 1) ck = (float)I.cosk[m];
#pragma unroll 1
    for (int c0 = 0; c0 < TCN; c0 += 32) {
      float v[32], w[32];
      tmem_ld32(tmem + lane_off + (unsigned)c0, v);
      tmem_ld32(tmem_corr + lane_off + (unsigned)c0, w);
#pragma unroll
      for (int q = 0; q < 32; ++q) v[q] += w[q];
      const int n0 = tn * TCN + c0;
      if (stage == 0 || stage == 1) {
        float* out = stage == 0 ? T1 : T2;
#pragma unroll
        for (int q = 0; q < 32; ++q) {
          float x = v[q];
          if (stage == 1) {
            const int l = n0 + q;
            const float lam = 2.0f - 2.0f * ck * (float)I.cosk[l];
            x = (m == 0 && l == 0) ? 0.0f : x / lam;
          }
          out[(size_t)(n0 + q) * n + m] = x;  // transposed: the warp's 32 rows are 32 consecutive floats
        }
      } else {
        float* out = stage == 2 ? T1 : reinterpret_cast<float*>(I.dhat);
#pragma unroll
        for (int q = 0; q < 32; q += 4)
          *reinterpret_cast<float4*>(out + (size_t)m * n + n0 + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

}  // namespace

bool dct_tc_supported(int n) { return n == 128 || n == 256 || n == 512 || n == 1024; }

int dct_tc_tiles(int n) { return (n / TCM) * (n / TCM); }

void dct_tc_attrs(int device) {
  static bool done[64] = {};
  if (device < 64 && done[device]) return;
  OTM_CUDA(cudaFuncSetAttribute(k_dct_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
  if (device < 64) done[device] = true;
}

void dct_tc_run(otm_context* ctx, Inst* d_insts, const int* tc_inst, int base, int count) {
  dct_tc_attrs(ctx->device);
  if (count <= 0) return;
  for (int s = 0; s < 4; ++s)
    launch_smem(ctx, "dct_tc", k_dct_tc, count, 128, SMEM, d_insts, tc_inst, base, s, kTcWait);
}

}  // namespace otm
