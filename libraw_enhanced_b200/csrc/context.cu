// context.cu -- context, workspace arena, errors and pinned host memory.
#include <cstdio>
#include <cstring>

#include "lre_internal.h"

namespace lre {

Workspace::~Workspace() {
  if (base_) cudaFree(base_);
}

cudaError_t Workspace::reserve(size_t bytes, cudaStream_t s) {
  bytes = (bytes + 255) & ~size_t(255);
  if (bytes <= cap_) return cudaSuccess;
  if (base_) {
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    cudaFree(base_);
    base_ = nullptr;
    cap_ = 0;
  }
  cudaError_t e = cudaMalloc(&base_, bytes);
  if (e != cudaSuccess) {
    base_ = nullptr;
    return e;
  }
  cap_ = bytes;
  used_ = 0;
  return cudaSuccess;
}

void Workspace::release() {
  if (base_) cudaFree(base_);
  base_ = nullptr;
  cap_ = used_ = 0;
}

void* Workspace::take(size_t bytes) {
  bytes = (bytes + 255) & ~size_t(255);
  if (used_ + bytes > cap_) return nullptr;
  void* p = base_ + used_;
  used_ += bytes;
  return p;
}

lre_status fail(Context* c, lre_status st, const std::string& msg) {
  if (c) c->last_error = msg;
  return st;
}

lre_status cuda_fail(Context* c, cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  return fail(c, e == cudaErrorMemoryAllocation ? LRE_ERR_OUT_OF_MEMORY : LRE_ERR_CUDA, m);
}

lre_status check_launch(Context* c, const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(c, e, what);
  return LRE_OK;
}

lre_status check_injection(Context* c) {
  if (c->inject_countdown > 0) {
    if (--c->inject_countdown == 0) return fail(c, LRE_ERR_INJECTED, "injected fault (host side, before any device work)");
  }
  return LRE_OK;
}

lre_status ensure_buffer(Context* c, void** p, size_t* cap, size_t bytes) {
  if (bytes <= *cap && *p) return LRE_OK;
  if (*p) {
    LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    cudaFree(*p);
    *p = nullptr;
    *cap = 0;
  }
  size_t b = (bytes + 4095) & ~size_t(4095);
  cudaError_t e = cudaMalloc(p, b);
  if (e != cudaSuccess) {
    *p = nullptr;
    return cuda_fail(c, e, "cudaMalloc(staging)");
  }
  *cap = b;
  return LRE_OK;
}

}  // namespace lre

using lre::Context;

extern "C" {

int lre_abi_version(void) { return LRE_ABI_VERSION; }

int lre_is_available(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return 0;
  }
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, 0) != cudaSuccess) return 0;
  return p.major >= 10 ? 1 : 0;
}

lre_status lre_create(int device, lre_ctx** out) {
  if (!out) return LRE_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return LRE_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= n) return LRE_ERR_INVALID_ARGUMENT;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return LRE_ERR_NO_DEVICE;
  if (prop.major < 10) return LRE_ERR_NO_DEVICE;  // this build carries sm_100a code only
  if (cudaSetDevice(device) != cudaSuccess) return LRE_ERR_CUDA;
  Context* c = new Context();
  c->device = device;
  c->sm_count = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return LRE_ERR_CUDA;
  }
  c->stream = c->own_stream;
  if (cudaMalloc(&c->d_scalars, 64 * sizeof(float)) != cudaSuccess) {
    cudaStreamDestroy(c->own_stream);
    delete c;
    return LRE_ERR_OUT_OF_MEMORY;
  }
  if (lre::aahd_upload_gamma(c) != LRE_OK) {
    cudaFree(c->d_scalars);
    cudaStreamDestroy(c->own_stream);
    delete c;
    return LRE_ERR_CUDA;
  }
  *out = reinterpret_cast<lre_ctx*>(c);
  return LRE_OK;
}

void lre_destroy(lre_ctx* ctx) {
  Context* c = reinterpret_cast<Context*>(ctx);
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
  lre::destroy_stager(c);
  if (c->d_in) cudaFree(c->d_in);
  if (c->d_out) cudaFree(c->d_out);
  if (c->d_aux) cudaFree(c->d_aux);
  if (c->d_scalars) cudaFree(c->d_scalars);
  for (cudaEvent_t& e : c->band_ev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t& e : c->tail_ev)
    if (e) cudaEventDestroy(e);
  if (c->copy_stream) {
    cudaStreamSynchronize(c->copy_stream);
    cudaStreamDestroy(c->copy_stream);
  }
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
}

const char* lre_last_error(const lre_ctx* ctx) {
  const Context* c = reinterpret_cast<const Context*>(ctx);
  return c ? c->last_error.c_str() : "null context";
}

lre_status lre_device_info(lre_ctx* ctx, char* buf, size_t buflen) {
  Context* c = reinterpret_cast<Context*>(ctx);
  if (!c || !buf || buflen == 0) return LRE_ERR_INVALID_ARGUMENT;
  cudaDeviceProp p;
  LRE_CUDA_TRY(c, cudaGetDeviceProperties(&p, c->device));
  snprintf(buf, buflen, "%s (sm_%d%d, %d SMs, %.1f GiB HBM, L2 %d MiB)", p.name, p.major, p.minor,
           p.multiProcessorCount, p.totalGlobalMem / 1073741824.0, p.l2CacheSize >> 20);
  return LRE_OK;
}

lre_status lre_set_stream(lre_ctx* ctx, void* stream) {
  Context* c = reinterpret_cast<Context*>(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  c->stream = stream ? reinterpret_cast<cudaStream_t>(stream) : c->own_stream;
  return LRE_OK;
}

void* lre_get_stream(lre_ctx* ctx) {
  Context* c = reinterpret_cast<Context*>(ctx);
  return c ? reinterpret_cast<void*>(c->stream) : nullptr;
}

lre_status lre_synchronize(lre_ctx* ctx) {
  Context* c = reinterpret_cast<Context*>(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  LRE_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return LRE_OK;
}

lre_status lre_reserve_workspace(lre_ctx* ctx, size_t bytes) {
  Context* c = reinterpret_cast<Context*>(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  LRE_CUDA_TRY(c, c->ws.reserve(bytes, c->stream));
  return LRE_OK;
}

size_t lre_workspace_bytes(const lre_ctx* ctx) {
  const Context* c = reinterpret_cast<const Context*>(ctx);
  return c ? c->ws.capacity() : 0;
}

uint64_t lre_launch_count(const lre_ctx* ctx) {
  const Context* c = reinterpret_cast<const Context*>(ctx);
  return c ? c->launches.load() : 0;
}

lre_status lre_host_alloc(lre_ctx* ctx, size_t bytes, void** out) {
  Context* c = reinterpret_cast<Context*>(ctx);
  if (!c || !out) return LRE_ERR_INVALID_ARGUMENT;
  cudaSetDevice(c->device);
  LRE_CUDA_TRY(c, cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocPortable));
  return LRE_OK;
}

lre_status lre_host_free(lre_ctx* ctx, void* p) {
  Context* c = reinterpret_cast<Context*>(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  if (p) LRE_CUDA_TRY(c, cudaFreeHost(p));
  return LRE_OK;
}

void lre_inject_fault(lre_ctx* ctx, int countdown) {
  Context* c = reinterpret_cast<Context*>(ctx);
  if (c) c->inject_countdown = countdown > 0 ? countdown : 0;
}

lre_status lre_set_wait_limit(lre_ctx* ctx, long long cycles) {
  Context* c = reinterpret_cast<Context*>(ctx);
  if (!c) return LRE_ERR_INVALID_ARGUMENT;
  c->sweep_wait_cycles = cycles > 0 ? cycles : 0;
  return LRE_OK;
}

void lre_inject_sweep_stall(lre_ctx* ctx, int band) {
  Context* c = reinterpret_cast<Context*>(ctx);
  if (c) c->sweep_hold_band = band >= 0 ? band : -1;
}

}  // extern "C"
