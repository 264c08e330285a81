// Host-side state behind the opaque otm_context / otm_map handles.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <vector>

#include "common.cuh"
#include "otmap_b200.h"

namespace otm {

// Owning device buffer.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  // Grows (never shrinks) to at least `b` bytes; contents are not preserved.
  void reserve(size_t b);
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// Device buffer from the stream-ordered allocator (cudaMallocFromPoolAsync / cudaFreeAsync
// on the stream it was reserved on, from the context's memory pool): freeing it does not
// synchronise the device, and the pool hands the memory to the next allocation. Used for
// the per-map buffers, which live and die with each TransportMap.
struct AsyncBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaStream_t st = nullptr;
  AsyncBuf() = default;
  AsyncBuf(const AsyncBuf&) = delete;
  AsyncBuf& operator=(const AsyncBuf&) = delete;
  ~AsyncBuf() { release(); }
  void release() {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    bytes = 0;
  }
  // Grows (never shrinks) to at least `b` bytes on stream s from `pool`; contents are not
  // preserved.
  void reserve(size_t b, cudaStream_t s, cudaMemPool_t pool);
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// Per grid size: the orthonormal DCT-II basis and cos(pi k / n), built by otm_init.
struct SizeTables {
  int n = 0;
  DevBuf C;     // n*n doubles, C[k*n + i]
  DevBuf cosk;  // n doubles
  DevBuf tw;    // n/2 double2, exp(-2 pi i k / n) (power-of-two n)
  DevBuf pt;    // n double2, (cos, sin)(pi k / 2n) (power-of-two n)
  DevBuf Cf;    // C[k][i] as TF32 planes, hi then lo (2 n*n floats; tensor-core transform sizes)
  DevBuf CTf;   // C^T, likewise
  bool dct_ok = false;      // the assembled matrix is diagonalised by C (checked on the GPU)
  double dct_check_err = 0;  // relative error of that check
};

struct Inst;  // device instance record (solver.cu)

// Buffers of one batch configuration (the list of grid sizes), reused across calls.
struct Workspace {
  std::vector<int> sizes;
  DevBuf insts;      // Inst[count]
  DevBuf tile_inst;  // int per stencil tile
  DevBuf gemm_inst;  // int per GEMM tile (instances on the dense-product transform)
  DevBuf tc_inst;    // int per output tile of the tensor-core transform
  DevBuf strip_inst;  // int per sweep block
  DevBuf sweep_partials;  // double[sweep blocks * SWEEP_SLOTS]
  DevBuf row_inst;   // int per row block of the fast transform
  DevBuf col_inst;   // int per column block of the fast transform
  DevBuf partials;   // double[total_tiles * 8]
  DevBuf arena;      // per-instance cell arrays
  DevBuf tmaps;      // tensor maps of the tensor-core transform instances
  std::vector<const void*> tmap_key;  // the buffers those maps were encoded for
  std::vector<unsigned char> h_insts;  // host mirror of Inst[count]
  void* h_pinned = nullptr;            // pinned staging for Inst readback
  size_t h_pinned_bytes = 0;
  int total_tiles = 0, total_gemm = 0, total_rows = 0, total_cols = 0, total_strips = 0, total_tc = 0;
  int mode = -1;       // poisson mode the layout was built for
  int precision = -1;  // precision the layout was built for
  int srows = 0;       // strip height of the sweeps (rule or autotuned)
  bool tuned = false;  // srows was chosen by timing (OTM_OPT_AUTOTUNE)
  int split_strip0 = 0;  // strips of split-precision instances start here (FP64 ones before)
  struct Segment {  // instances of one size on one transform kernel family
    int n, reg, split, roff, rcnt, coff, ccnt;
  };
  std::vector<Segment> segments;
  // the iteration loop captured as a CUDA graph with a device-side WHILE node
  cudaGraphExec_t graph_exec = nullptr;
  long graph_body_kernels = 0;
  DevBuf loopctl;  // LoopCtl (solver.cu)
  void drop_graph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    graph_exec = nullptr;
  }
  ~Workspace() {
    drop_graph();
    if (h_pinned) cudaFreeHost(h_pinned);
  }
};

}  // namespace otm

namespace otm {
// Per-kernel CUDA-event timing on the context stream (enabled by otm_profile).
struct Profiler {
  struct Rec {
    int name;
    cudaEvent_t a, b;
  };
  bool on = false;
  std::vector<const char*> names;
  std::vector<double> ms;
  std::vector<long> count;
  std::vector<Rec> pending;
  std::vector<cudaEvent_t> pool;
  int id(const char* name);
  cudaEvent_t get();
  void flush();  // after a stream sync: fold pending pairs into the totals
  ~Profiler();
};
}  // namespace otm

struct otm_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;  // stream-ordered allocations of the per-map buffers
  int num_sms = 0;
  long launches = 0;  // kernels launched by this context since creation
  int poisson_mode = 0;  // OTM_POISSON_AUTO / _DENSE / _FFT
  int loop_mode = 0;     // OTM_LOOP_GRAPH (0) / OTM_LOOP_HOST (1)
  int wait_test = 0;     // OTM_OPT_WAIT_TEST: bounded waits made to run out
  int precision = 0;     // OTM_PRECISION_FP64 / _SPLIT
  int autotune = 0;      // OTM_AUTOTUNE_OFF / _ON (sweep strip height per batch configuration)
  int last_srows = 0;    // strip height of the last solve call (OTM_INFO_STRIP_ROWS)
  otm::Profiler prof;
  std::map<int, std::unique_ptr<otm::SizeTables>> tables;
  // Workspaces of the most recent batch configurations (size list + Poisson mode), most
  // recently used first; a call with a configuration seen before reuses its buffers and
  // its captured loop graph. At most kWorkspaces are kept.
  static constexpr int kWorkspaces = 6;
  std::vector<std::unique_ptr<otm::Workspace>> workspaces;
  otm::Workspace* wsp = nullptr;  // the workspace of the current call
  otm::Workspace& ws() { return *wsp; }
  otm::DevBuf staging;  // device staging for host inputs/outputs
  // second stream of a batched solve: outputs of instances that stopped while the rest of
  // the batch iterates (created on first use), its staging and a pinned copy of the records
  cudaStream_t side = nullptr;
  cudaEvent_t side_ready = nullptr;  // the batch's records are initialised (set-up kernels done)
  otm::DevBuf staging_side;
  void* h_poll = nullptr;
  size_t h_poll_bytes = 0;
  otm::DevBuf raster_scratch;  // rasterizer face boxes, pixel owners, vertex values (grow-only)
  // point-locator builds (locate.cu, grow-only): bin counts and scan sums; the BVH-order
  // build's per-position arrays and node lists. Builds are ordered on the context stream.
  otm::DevBuf locate_scratch, bvh_scratch;
  // the BVH-order build of a grid size as a graph over bvh_scratch (rebuilt when the
  // scratch moves)
  struct GraphExec {
    cudaGraphExec_t exec = nullptr;
    void* base = nullptr;
    long kernels = 0;
    GraphExec() = default;
    GraphExec(const GraphExec&) = delete;
    GraphExec& operator=(const GraphExec&) = delete;
    ~GraphExec() {
      if (exec) cudaGraphExecDestroy(exec);
    }
  };
  std::map<int, std::unique_ptr<GraphExec>> bvh_graphs;
  // adjoint workspaces per grid size (adjoint.cu); type-erased to keep this header small
  struct Erased {
    virtual ~Erased() = default;
  };
  std::map<int, std::unique_ptr<Erased>> adjoint;
  // contexts of the same device on which otm_barycenter_loss runs the adjoints of its maps
  // concurrently, one host thread each (created on first use, destroyed by otm_destroy)
  std::vector<otm_context*> helpers;
};

struct otm_map {
  otm_context* ctx = nullptr;
  int n = 0;
  // buffers on the context stream's stream-ordered allocator (destroying a map does not
  // synchronise the device)
  otm::AsyncBuf fwd;      // V*2 doubles
  otm::AsyncBuf density;  // N doubles
  // point-location structure (built lazily)
  bool located = false;
  int bins = 0;
  otm::AsyncBuf bin_start;  // int[bins*bins + 1]
  otm::AsyncBuf bin_faces;  // int[entries]
  otm::AsyncBuf face_box;   // double4 per face (min x, min y, max x, max y)
  otm::AsyncBuf bvh_rank;   // int per face: its position in the reference's BVH face array
  otm::AsyncBuf leaf_box;   // double4 per face: the enlarged box of its BVH leaf
  otm::AsyncBuf scratch;
};

namespace otm {
// Makes the context's device current; defined in capi.cu.
void make_current(otm_context* ctx);
// Copies `bytes` from src (host or device) into dst (device), on the context stream.
void copy_in(otm_context* ctx, void* dst, const void* src, size_t bytes);
// Copies `bytes` from src (device) into dst (host or device), on the context stream.
void copy_out(otm_context* ctx, void* dst, const void* src, size_t bytes);

// Rasterizes the (n+1)^2 grid mesh xy (device) into img (device, rows*cols), in
// OTM_RIO_PER_FACE or OTM_RIO_PER_VERTEX mode; density (device) NULL = unit density.
void raster_grid(otm_context* ctx, int n, const double* xy, const double* density, int rows, int cols, int mode,
                 double* img);

// Inversion of `count` device points through map m (locator built on demand), in place;
// face, hit0 (the first hit in the reference's order), nhits (device, may be null) and
// missing (device counter, added to) as otm_map_inverse_mode reports them.
void map_inverse_dev(otm_map* m, double* pts, long count, int mode, int* face, int* hit0, int* nhits,
                     unsigned long long* missing);

// Backward of the PerFace unit-density raster of the (n+1)^2 grid mesh xy that
// raster_grid just drew (its face boxes and pixel owners are still in the context's
// raster scratch): dL/dxy (V x 2, overwritten) from dL/dpixel (rows x cols), through each
// face's |area| (the value of an owned pixel is scale / |area|); pixel ownership is held
// fixed (it is piecewise constant in the mesh).
void raster_grid_backward(otm_context* ctx, int n, const double* xy, int rows, int cols, const double* dL_dpix,
                          double* dL_dxy);

// Backward of the inversion of the (n+1)^2 origin grid vertices through the forward mesh
// fwd (apps/barycenters.cpp:190): for each vertex located with first hit hit0[v],
// inverse position I_v = sum_i w_i(x_v; fwd corners of hit0) O_i, dL/dfwd (V x 2,
// overwritten) from dL/dI (V x 2). Deterministic: per-face point lists in index order.
void inverse_grid_backward(otm_context* ctx, int n, const double* fwd, const int* hit0, const double* dL_dI,
                           double* dL_dfwd);

// Launches `kernel` on the context stream, counting it and (when profiling) bracketing
// it with CUDA events.
template <class K, class... Args>
void launch(otm_context* ctx, const char* name, K kernel, dim3 grid, dim3 block, Args... args) {
  ctx->launches++;
  if (ctx->prof.on) {
    int id = ctx->prof.id(name);
    cudaEvent_t a = ctx->prof.get(), b = ctx->prof.get();
    cudaEventRecord(a, ctx->stream);
    kernel<<<grid, block, 0, ctx->stream>>>(args...);
    cudaEventRecord(b, ctx->stream);
    ctx->prof.pending.push_back({id, a, b});
  } else {
    kernel<<<grid, block, 0, ctx->stream>>>(args...);
  }
}

// As launch(), with dynamic shared memory.
template <class K, class... Args>
void launch_smem(otm_context* ctx, const char* name, K kernel, dim3 grid, dim3 block, size_t smem, Args... args) {
  ctx->launches++;
  if (ctx->prof.on) {
    int id = ctx->prof.id(name);
    cudaEvent_t a = ctx->prof.get(), b = ctx->prof.get();
    cudaEventRecord(a, ctx->stream);
    kernel<<<grid, block, smem, ctx->stream>>>(args...);
    cudaEventRecord(b, ctx->stream);
    ctx->prof.pending.push_back({id, a, b});
  } else {
    kernel<<<grid, block, smem, ctx->stream>>>(args...);
  }
}

// Runs an entry point body, mapping exceptions to otm_status codes.
template <class F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const BadArg& e) {
    set_error(e.what);
    return OTM_ERR_BAD_ARG;
  } catch (const DeviceTimeout& e) {
    set_error(e.what);
    return OTM_ERR_TIMEOUT;
  } catch (const CudaError& e) {
    set_error(std::string(cudaGetErrorString(e.code)) + " (" + e.where + ")");
    cudaGetLastError();  // a non-sticky error must not resurface in the next call's check
    return OTM_ERR_CUDA;
  } catch (const std::exception& e) {
    set_error(e.what());
    return OTM_ERR_CUDA;
  }
}
}  // namespace otm
