// Context: device binding, stream, and the device-memory budget every
// allocation of the engine is charged against.
#include <cstdio>

#include "hm_device.h"

namespace {
// Failure injection for tests: after this many further successful
// allocations on any context, dev_alloc reports HM_ERR_NOMEM (-1 = off).
std::atomic<long long> g_fail_after{-1};
}  // namespace

namespace hm {

int charge(hm_ctx* ctx, size_t bytes) {
  long long f = g_fail_after.load();
  if (f >= 0) {
    if (f == 0) return set_error(HM_ERR_NOMEM, "injected allocation failure (%zu bytes)", bytes);
    g_fail_after.fetch_sub(1);
  }
  size_t now = ctx->used.load();
  if (ctx->budget && now + bytes > ctx->budget)
    return set_error(HM_ERR_NOMEM, "device budget exceeded: %zu used + %zu requested > %zu", now, bytes,
                     ctx->budget);
  ctx->used.fetch_add(bytes);
  return HM_OK;
}

void uncharge(hm_ctx* ctx, size_t bytes) { ctx->used.fetch_sub(bytes); }

int dev_alloc(hm_ctx* ctx, void** p, size_t bytes) {
  *p = nullptr;
  HM_TRY(charge(ctx, bytes));
  // Stream-ordered allocation from the context's pool: no device-wide
  // synchronisation, and freed blocks are reused by the next call. When the
  // pool cannot grow, its cached free blocks are returned and the request is
  // retried once.
  cudaError_t e = cudaMallocFromPoolAsync(p, bytes, ctx->pool, ctx->stream);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    cudaStreamSynchronize(ctx->stream);
    cudaMemPoolTrimTo(ctx->pool, 0);
    e = cudaMallocFromPoolAsync(p, bytes, ctx->pool, ctx->stream);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    uncharge(ctx, bytes);
    return set_error(HM_ERR_NOMEM, "device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
  }
  return HM_OK;
}

void dev_free(hm_ctx* ctx, void* p, size_t bytes) {
  if (!p) return;
  cudaFreeAsync(p, ctx->stream);
  ctx->used.fetch_sub(bytes);
}

void trim_pool(hm_ctx* ctx) {
  cudaStreamSynchronize(ctx->stream);
  cudaMemPoolTrimTo(ctx->pool, 0);
}

}  // namespace hm

extern "C" int hm_ctx_create(int device, size_t mem_budget_bytes, hm_ctx** out) {
  if (!out) return hm::set_error(HM_ERR_INVALID, "hm_ctx_create: out is NULL");
  *out = nullptr;
  int n = 0;
  HM_CUDA(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return hm::set_error(HM_ERR_INVALID, "hm_ctx_create: device %d of %d", device, n);
  HM_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  HM_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10)
    return hm::set_error(HM_ERR_INVALID, "hm_ctx_create: device %d is sm_%d%d; this build targets sm_100a", device,
                         prop.major, prop.minor);
  auto* c = new hm_ctx();
  c->device = device;
  c->n_sms = prop.multiProcessorCount;
  size_t free_b = 0, total_b = 0;
  cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
  if (e != cudaSuccess) {
    delete c;
    return hm::set_error(HM_ERR_CUDA, "cudaMemGetInfo: %s", cudaGetErrorString(e));
  }
  c->budget = mem_budget_bytes ? mem_budget_bytes : free_b;
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return hm::set_error(HM_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
  }
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  e = cudaMemPoolCreate(&c->pool, &props);
  if (e != cudaSuccess) {
    cudaStreamDestroy(c->stream);
    delete c;
    return hm::set_error(HM_ERR_CUDA, "cudaMemPoolCreate: %s", cudaGetErrorString(e));
  }
  uint64_t keep = UINT64_MAX;  // freed blocks stay cached for the next batch
  cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  *out = c;
  return HM_OK;
}

extern "C" int hm_ctx_destroy(hm_ctx* ctx) {
  if (!ctx) return HM_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
  delete ctx;
  return HM_OK;
}

extern "C" int hm_ctx_memory(const hm_ctx* ctx, size_t* used_bytes, size_t* budget_bytes) {
  if (!ctx) return hm::set_error(HM_ERR_INVALID, "hm_ctx_memory: NULL context");
  if (used_bytes) *used_bytes = ctx->used.load();
  if (budget_bytes) *budget_bytes = ctx->budget;
  return HM_OK;
}

extern "C" void* hm_ctx_stream(const hm_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

extern "C" int hm_debug_fail_allocations_after(long long n) {
  g_fail_after.store(n);
  return HM_OK;
}
