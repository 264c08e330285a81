// Shared device/host helpers for the otmap_b200 CUDA library.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <string>

namespace otm {

// Thread-local message behind otm_last_error().
void set_error(const std::string& msg);

struct CudaError {
  cudaError_t code;
  std::string where;
};

#define OTM_CUDA(call)                                                                  \
  do {                                                                                  \
    cudaError_t _e = (call);                                                            \
    if (_e != cudaSuccess)                                                              \
      throw ::otm::CudaError{_e, std::string(#call) + " at " + __FILE__ + ":" +         \
                                     std::to_string(__LINE__)};                         \
  } while (0)

struct BadArg {
  std::string what;
};

// A bounded device-side wait gave up (reported as OTM_ERR_TIMEOUT).
struct DeviceTimeout {
  std::string what;
};

// True when p points into device (or managed) memory; host pointers, registered
// or not, report false.
inline bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// ---- device-side reductions (fixed order: results are run-to-run identical) ----

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide sums of K values per thread; result valid in thread 0. `red` is
// shared scratch of K * 32 doubles. Blocks are multiples of 32 threads.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) red[k * 32 + warp] = v[k];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double x = lane < nw ? red[k * 32 + lane] : 0.0;
      v[k] = warp_sum(x);
    }
  }
  __syncthreads();
}

__device__ __forceinline__ double block_max(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) v = warp_max(lane < nw ? red[lane] : -INFINITY);
  __syncthreads();
  return v;
}

// "Last block" election for a reduction spread over `total` blocks that share
// `counter`: every block calls it once after thread 0 has written the block's
// partials; it returns true (in all threads) in exactly one block, the last to
// arrive, which may then read every block's partials. The counter is reset for
// the next kernel by the last block.
__device__ __forceinline__ bool last_block(unsigned int* counter, unsigned int total) {
  __shared__ bool s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int prev = atomicAdd(counter, 1u);
    s_last = (prev == total - 1u);
    if (s_last) *counter = 0u;
  }
  __syncthreads();
  if (s_last) __threadfence();
  return s_last;
}

// std::max / std::min semantics (NaN in the second argument yields the first).
__host__ __device__ __forceinline__ double std_max(double a, double b) { return a < b ? b : a; }
__host__ __device__ __forceinline__ double std_min(double a, double b) { return b < a ? b : a; }

}  // namespace otm
