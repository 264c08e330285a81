// Context management, host/device copies and error reporting of the C ABI.

#include <cfloat>
#include <cstring>
#include <string>

#include "context.h"

namespace otm {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

void make_current(otm_context* ctx) { OTM_CUDA(cudaSetDevice(ctx->device)); }

void copy_in(otm_context* ctx, void* dst, const void* src, size_t bytes) {
  if (!bytes) return;
  OTM_CUDA(cudaMemcpyAsync(dst, src, bytes, is_device_ptr(src) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                           ctx->stream));
}

void copy_out(otm_context* ctx, void* dst, const void* src, size_t bytes) {
  if (!bytes) return;
  OTM_CUDA(cudaMemcpyAsync(dst, src, bytes, is_device_ptr(dst) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                           ctx->stream));
}

int Profiler::id(const char* name) {
  for (size_t k = 0; k < names.size(); ++k)
    if (std::strcmp(names[k], name) == 0) return (int)k;
  names.push_back(name);
  ms.push_back(0.0);
  count.push_back(0);
  return (int)names.size() - 1;
}

cudaEvent_t Profiler::get() {
  if (!pool.empty()) {
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  OTM_CUDA(cudaEventCreate(&e));
  return e;
}

void Profiler::flush() {
  for (auto& r : pending) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, r.a, r.b) == cudaSuccess) {
      ms[r.name] += t;
      count[r.name] += 1;
    } else {
      cudaGetLastError();
    }
    pool.push_back(r.a);
    pool.push_back(r.b);
  }
  pending.clear();
}

Profiler::~Profiler() {
  for (auto& r : pending) {
    pool.push_back(r.a);
    pool.push_back(r.b);
  }
  for (auto e : pool) cudaEventDestroy(e);
}

}  // namespace otm

using namespace otm;

extern "C" const char* otm_last_error(void) { return g_last_error.c_str(); }

extern "C" int otm_abi_version(void) { return OTM_ABI_VERSION; }

extern "C" void otm_default_options(otm_solver_options* opt) {
  if (!opt) return;
  opt->beta = OTM_BETA_CONJUGATE_JACOBIAN;
  opt->max_iter = 1000;
  opt->threshold = 1e-7;
  opt->max_ratio = DBL_MAX;
}

extern "C" int otm_create(int device, otm_context** out) {
  if (!out) {
    set_error("otm_create: null output pointer");
    return OTM_ERR_BAD_ARG;
  }
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("otm_create: no CUDA device");
    return OTM_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) {
    set_error("otm_create: device index out of range");
    return OTM_ERR_BAD_ARG;
  }
  return guarded([&] {
    auto* ctx = new otm_context;
    ctx->device = device;
    try {
      OTM_CUDA(cudaSetDevice(device));
      OTM_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
      OTM_CUDA(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device));
      // the per-map buffers come from this context's own memory pool (stream-ordered
      // allocation), which keeps freed memory for the next map instead of returning it to
      // the driver at every synchronisation; the device's default pool is left as it is
      cudaMemPoolProps props = {};
      props.allocType = cudaMemAllocationTypePinned;
      props.handleTypes = cudaMemHandleTypeNone;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = device;
      OTM_CUDA(cudaMemPoolCreate(&ctx->pool, &props));
      uint64_t keep = UINT64_MAX;
      OTM_CUDA(cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    } catch (...) {
      delete ctx;
      throw;
    }
    *out = ctx;
    return (int)OTM_OK;
  });
}

extern "C" int otm_destroy(otm_context* ctx) {
  if (!ctx) return OTM_OK;
  for (otm_context* h : ctx->helpers) otm_destroy(h);
  ctx->helpers.clear();
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->side) cudaStreamSynchronize(ctx->side);
  cudaStream_t st = ctx->stream, side = ctx->side;
  cudaEvent_t ready = ctx->side_ready;
  void* poll = ctx->h_poll;
  cudaMemPool_t pool = ctx->pool;
  delete ctx;
  if (st) cudaStreamDestroy(st);
  // maps are destroyed before their context; memory a map still held would go back to
  // the driver when that map frees it
  if (pool) cudaMemPoolDestroy(pool);
  if (side) cudaStreamDestroy(side);
  if (ready) cudaEventDestroy(ready);
  if (poll) cudaFreeHost(poll);
  return OTM_OK;
}

extern "C" int otm_stream(otm_context* ctx, void** stream) {
  if (!ctx || !stream) {
    set_error("otm_stream: null argument");
    return OTM_ERR_BAD_ARG;
  }
  *stream = (void*)ctx->stream;
  return OTM_OK;
}

extern "C" long otm_launch_count(otm_context* ctx) { return ctx ? ctx->launches : 0; }

extern "C" int otm_profile(otm_context* ctx, int enable) {
  if (!ctx) {
    set_error("otm_profile: null context");
    return OTM_ERR_BAD_ARG;
  }
  return guarded([&] {
    make_current(ctx);
    OTM_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->prof.flush();
    if (enable < 0) {  // reset the totals
      for (auto& m : ctx->prof.ms) m = 0.0;
      for (auto& c : ctx->prof.count) c = 0;
    } else {
      ctx->prof.on = enable != 0;
    }
    return (int)OTM_OK;
  });
}

extern "C" int otm_profile_entry(otm_context* ctx, int index, const char** name, double* ms, long* launches) {
  if (!ctx) return 0;
  if (index < 0 || index >= (int)ctx->prof.names.size()) return 0;
  if (name) *name = ctx->prof.names[index];
  if (ms) *ms = ctx->prof.ms[index];
  if (launches) *launches = ctx->prof.count[index];
  return 1;
}

extern "C" int otm_set_option(otm_context* ctx, int key, int value) {
  if (!ctx) {
    set_error("otm_set_option: null context");
    return OTM_ERR_BAD_ARG;
  }
  if (key == OTM_OPT_POISSON) {
    if (value < OTM_POISSON_AUTO || value > OTM_POISSON_TENSOR) {
      set_error("otm_set_option: unknown Poisson mode");
      return OTM_ERR_BAD_ARG;
    }
    ctx->poisson_mode = value;
    return OTM_OK;
  }
  if (key == OTM_OPT_LOOP) {
    if (value != OTM_LOOP_GRAPH && value != OTM_LOOP_HOST) {
      set_error("otm_set_option: unknown loop mode");
      return OTM_ERR_BAD_ARG;
    }
    ctx->loop_mode = value;
    return OTM_OK;
  }
  if (key == OTM_OPT_WAIT_TEST) {
    if (value != 0 && value != 1) {
      set_error("otm_set_option: OTM_OPT_WAIT_TEST takes 0 or 1");
      return OTM_ERR_BAD_ARG;
    }
    if (ctx->wait_test != value) {
      cudaSetDevice(ctx->device);
      cudaStreamSynchronize(ctx->stream);
      for (auto& w : ctx->workspaces) w->drop_graph();  // the captured launches carry the wait parameters
    }
    ctx->wait_test = value;
    return OTM_OK;
  }
  if (key == OTM_OPT_PRECISION) {
    if (value != OTM_PRECISION_FP64 && value != OTM_PRECISION_SPLIT) {
      set_error("otm_set_option: unknown precision");
      return OTM_ERR_BAD_ARG;
    }
    ctx->precision = value;
    return OTM_OK;
  }
  if (key == OTM_OPT_AUTOTUNE) {
    if (value != OTM_AUTOTUNE_OFF && value != OTM_AUTOTUNE_ON) {
      set_error("otm_set_option: OTM_OPT_AUTOTUNE takes 0 or 1");
      return OTM_ERR_BAD_ARG;
    }
    ctx->autotune = value;
    return OTM_OK;
  }
  set_error("otm_set_option: unknown option");
  return OTM_ERR_BAD_ARG;
}

extern "C" int otm_get_option(otm_context* ctx, int key, int* value) {
  if (!ctx || !value) {
    set_error("otm_get_option: null argument");
    return OTM_ERR_BAD_ARG;
  }
  switch (key) {
    case OTM_OPT_POISSON: *value = ctx->poisson_mode; return OTM_OK;
    case OTM_OPT_LOOP: *value = ctx->loop_mode; return OTM_OK;
    case OTM_OPT_WAIT_TEST: *value = ctx->wait_test; return OTM_OK;
    case OTM_OPT_PRECISION: *value = ctx->precision; return OTM_OK;
    case OTM_OPT_AUTOTUNE: *value = ctx->autotune; return OTM_OK;
    case OTM_INFO_STRIP_ROWS: *value = ctx->last_srows; return OTM_OK;
    default: set_error("otm_get_option: unknown key"); return OTM_ERR_BAD_ARG;
  }
}
