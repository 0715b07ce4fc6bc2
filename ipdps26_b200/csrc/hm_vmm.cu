// Growable device memory on CUDA virtual memory management (GrowSpace).
// The driver's VMM calls are looked up through the runtime's entry-point
// query, so the library does not link the driver library directly.
#include <cuda.h>

#include <algorithm>
#include <mutex>

#include "hm_device.h"

namespace {

using FnCreate = CUresult (*)(CUmemGenericAllocationHandle*, size_t, const CUmemAllocationProp*, unsigned long long);
using FnRelease = CUresult (*)(CUmemGenericAllocationHandle);
using FnReserve = CUresult (*)(CUdeviceptr*, size_t, size_t, CUdeviceptr, unsigned long long);
using FnFree = CUresult (*)(CUdeviceptr, size_t);
using FnMap = CUresult (*)(CUdeviceptr, size_t, size_t, CUmemGenericAllocationHandle, unsigned long long);
using FnUnmap = CUresult (*)(CUdeviceptr, size_t);
using FnAccess = CUresult (*)(CUdeviceptr, size_t, const CUmemAccessDesc*, size_t);
using FnGran = CUresult (*)(size_t*, const CUmemAllocationProp*, CUmemAllocationGranularity_flags);
using FnAttr = CUresult (*)(int*, CUdevice_attribute, CUdevice);

struct Vmm {
  bool ok = false;
  FnCreate create = nullptr;
  FnRelease release = nullptr;
  FnReserve reserve = nullptr;
  FnFree free = nullptr;
  FnMap map = nullptr;
  FnUnmap unmap = nullptr;
  FnAccess access = nullptr;
  FnGran gran = nullptr;
  FnAttr attr = nullptr;
};

template <class F>
bool lookup(const char* name, F* fn) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q{};
  if (cudaGetDriverEntryPointByVersion(name, &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !p) {
    cudaGetLastError();
    return false;
  }
  *fn = reinterpret_cast<F>(p);
  return true;
}

const Vmm& vmm_api() {
  static Vmm v;
  static std::once_flag once;
  std::call_once(once, [] {
    v.ok = lookup("cuMemCreate", &v.create) && lookup("cuMemRelease", &v.release) &&
           lookup("cuMemAddressReserve", &v.reserve) && lookup("cuMemAddressFree", &v.free) &&
           lookup("cuMemMap", &v.map) && lookup("cuMemUnmap", &v.unmap) && lookup("cuMemSetAccess", &v.access) &&
           lookup("cuMemGetAllocationGranularity", &v.gran) && lookup("cuDeviceGetAttribute", &v.attr);
  });
  return v;
}

CUmemAllocationProp prop_of(int device) {
  CUmemAllocationProp p = {};
  p.type = CU_MEM_ALLOCATION_TYPE_PINNED;
  p.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
  p.location.id = device;
  return p;
}

size_t round_up(size_t x, size_t g) { return (x + g - 1) / g * g; }

}  // namespace

namespace hm {

// Maps one chunk at va and opens it to the device.
static int map_one(const Vmm& v, int device, CUdeviceptr va, size_t size, unsigned long long handle) {
  if (v.map(va, size, 0, handle, 0) != CUDA_SUCCESS) return set_error(HM_ERR_CUDA, "cuMemMap of %zu bytes failed", size);
  CUmemAccessDesc d = {};
  d.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
  d.location.id = device;
  d.flags = CU_MEM_ACCESS_FLAGS_PROT_READWRITE;
  if (v.access(va, size, &d, 1) != CUDA_SUCCESS) {
    v.unmap(va, size);
    return set_error(HM_ERR_CUDA, "cuMemSetAccess failed");
  }
  return HM_OK;
}

// Unmaps chunks [i0, i1) of a reservation at va, one mapping at a time.
static void unmap_chunks(const Vmm& v, CUdeviceptr va, const std::vector<size_t>& sizes, size_t i0, size_t i1) {
  size_t at = 0;
  for (size_t i = 0; i < i0; ++i) at += sizes[i];
  for (size_t i = i0; i < i1; ++i) {
    v.unmap(va + at, sizes[i]);
    at += sizes[i];
  }
}

// Physical memory is taken in chunks of at most kChunk bytes, so that shrink
// can give back all but the chunk the kept bytes end in.
constexpr size_t kChunk = size_t(1) << 30;

int GrowSpace::grow(hm_ctx* c, size_t bytes) {
  if (bytes <= mapped) return HM_OK;
  if (!ctx) {
    ctx = c;
    int ok = 0;
    const Vmm& v = vmm_api();
    vmm = v.ok && v.attr(&ok, CU_DEVICE_ATTRIBUTE_VIRTUAL_MEMORY_MANAGEMENT_SUPPORTED, c->device) == CUDA_SUCCESS &&
          ok;
  }
  HM_CUDA(cudaSetDevice(ctx->device));
  if (!vmm) {  // allocate, copy, free
    void* q = nullptr;
    HM_TRY(dev_alloc(ctx, &q, bytes));
    if (mapped) {
      HM_CUDA(cudaMemcpyAsync(q, base, mapped, cudaMemcpyDeviceToDevice, ctx->stream));
      dev_free(ctx, base, mapped);
    }
    base = static_cast<char*>(q);
    mapped = reserved = bytes;
    return HM_OK;
  }
  const Vmm& v = vmm_api();
  const CUmemAllocationProp prop = prop_of(ctx->device);
  size_t g = 0;
  if (v.gran(&g, &prop, CU_MEM_ALLOC_GRANULARITY_RECOMMENDED) != CUDA_SUCCESS || !g) g = 2u << 20;
  const size_t target = mapped + round_up(bytes - mapped, g);
  HM_TRY(charge(ctx, target - mapped));
  // the new chunks
  const size_t first = handles.size();
  int status = HM_OK;
  for (size_t at = mapped; at < target;) {
    const size_t sz = std::min(kChunk, target - at);
    CUmemGenericAllocationHandle h = 0;
    CUresult r = v.create(&h, sz, &prop, 0);
    if (r == CUDA_ERROR_OUT_OF_MEMORY) {  // the stream-ordered pool may hold freed blocks
      trim_pool(ctx);
      r = v.create(&h, sz, &prop, 0);
    }
    if (r != CUDA_SUCCESS) {
      status = set_error(r == CUDA_ERROR_OUT_OF_MEMORY ? HM_ERR_NOMEM : HM_ERR_CUDA,
                         "cuMemCreate of %zu bytes failed (%d)", sz, (int)r);
      break;
    }
    handles.push_back(h);
    sizes.push_back(sz);
    at += sz;
  }
  CUdeviceptr va = (CUdeviceptr)base;
  size_t va_size = reserved;
  const bool moved = target > reserved;
  if (status == HM_OK && moved) {
    // a new, larger reservation holding every chunk; the old one is dropped
    // once no kernel can still use it
    va_size = round_up(std::max(2 * reserved, 2 * target), g);
    va = 0;
    if (v.reserve(&va, va_size, g, 0, 0) != CUDA_SUCCESS) {
      va = 0;
      status = set_error(HM_ERR_NOMEM, "cuMemAddressReserve of %zu bytes failed", va_size);
    }
  }
  size_t n_mapped = 0;  // chunks mapped into va by this call, from index `from`
  const size_t from = moved ? 0 : first;
  if (status == HM_OK) {
    size_t at = 0;
    for (size_t i = 0; i < from; ++i) at += sizes[i];
    for (size_t i = from; i < handles.size(); ++i) {
      status = map_one(v, ctx->device, va + at, sizes[i], handles[i]);
      if (status != HM_OK) break;
      ++n_mapped;
      at += sizes[i];
    }
  }
  if (status != HM_OK) {
    unmap_chunks(v, va, sizes, from, from + n_mapped);
    if (moved && va) v.free(va, va_size);
    for (size_t i = first; i < handles.size(); ++i) v.release(handles[i]);
    handles.resize(first);
    sizes.resize(first);
    uncharge(ctx, target - mapped);
    return status;
  }
  if (moved) {
    if (base) {
      HM_CUDA(cudaDeviceSynchronize());
      unmap_chunks(v, (CUdeviceptr)base, sizes, 0, first);
      v.free((CUdeviceptr)base, reserved);
    }
    base = reinterpret_cast<char*>(va);
    reserved = va_size;
  }
  mapped = target;
  return HM_OK;
}

void GrowSpace::shrink(size_t bytes) {
  if (!base || !vmm || bytes >= mapped) return;
  const Vmm& v = vmm_api();
  size_t at = mapped;
  size_t k = handles.size();
  while (k > 0 && at - sizes[k - 1] >= bytes && at - sizes[k - 1] > 0) {
    at -= sizes[k - 1];
    --k;
  }
  if (k == handles.size()) return;
  cudaSetDevice(ctx->device);
  cudaDeviceSynchronize();
  unmap_chunks(v, (CUdeviceptr)base, sizes, k, handles.size());
  for (size_t i = k; i < handles.size(); ++i) v.release(handles[i]);
  uncharge(ctx, mapped - at);
  handles.resize(k);
  sizes.resize(k);
  mapped = at;
}

void GrowSpace::release() {
  if (!base) return;
  if (!vmm) {
    dev_free(ctx, base, mapped);
  } else {
    const Vmm& v = vmm_api();
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    unmap_chunks(v, (CUdeviceptr)base, sizes, 0, handles.size());
    v.free((CUdeviceptr)base, reserved);
    for (auto h : handles) v.release(h);
    uncharge(ctx, mapped);
  }
  handles.clear();
  sizes.clear();
  base = nullptr;
  mapped = reserved = 0;
  ctx = nullptr;
}

bool vmm_available() { return vmm_api().ok; }

}  // namespace hm
