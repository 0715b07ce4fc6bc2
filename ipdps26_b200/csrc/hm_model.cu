// Traffic model of the static count: the algorithmic bytes a launch must move,
// computed exactly from the stored graph. Used for the roofline figures.
//
// B_static follows the reference-equivalent merge algorithm (MoCHy's loop,
// MoCHy-master/main_exact.cpp:91-129, with neighbour lists intersected by
// merge): store read once, every id-oriented pair (a < b) merges N+(a) and
// N+(b) (ids larger than the owner), and every pair closing a triangle
// materialises I_ab from the two member lists:
//   B_static = 4 nnz(H2V) + 8 nnz(H2H) + sum_{(a,b), a<b} 8 (d+(a) + d+(b))
//            + sum_{(a,b), a<b, closed} 4 (|a| + |b|)
// The kernel model is what this engine's two kernels read: H2H once in the
// open phase (id + overlap + size lookup), each oriented row once, and one id
// per probe of N+(b), plus overlap/node on hits.
#include <vector>

#include "hm_device.h"

namespace hm {
namespace {

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint64_t global_warp() { return ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ uint64_t n_warps() { return ((uint64_t)gridDim.x * blockDim.x) >> 5; }

__device__ __forceinline__ uint64_t warp_sum(uint64_t v) {
  for (int d = 16; d; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  return v;
}

// d+_id(a): neighbours with a larger id (rows are sorted by id).
__global__ void k_dplus_id(const uint64_t* off, const uint32_t* len, const uint32_t* nbr, uint32_t n, uint32_t* dp) {
  for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < n; a += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t* row = nbr + off[a];
    uint32_t lo = 0, hi = len[a];
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (row[mid] <= (uint32_t)a) lo = mid + 1;
      else hi = mid;
    }
    dp[a] = len[a] - lo;
  }
}

__global__ void k_merge_bytes(const uint64_t* off, const uint32_t* len, const uint32_t* nbr, const uint32_t* dp,
                              uint32_t n, unsigned long long* out) {
  uint64_t acc = 0;
  for (uint64_t a = global_warp(); a < n; a += n_warps()) {
    const uint64_t s = off[a];
    const uint32_t l = len[a];
    const uint32_t da = dp[a];
    for (uint32_t i = l - da + lane_id(); i < l; i += 32) acc += 8ull * (da + dp[nbr[s + i]]);
  }
  acc = warp_sum(acc);
  if (lane_id() == 0 && acc) atomicAdd(out, (unsigned long long)acc);
}

// Closed pairs (flagged by a diagnostic triangle pass over the oriented
// rows): 4 (|a| + |b|) each. Kernel model: probes and row reads.
__global__ void k_oriented_bytes(const uint64_t* poff, const uint32_t* plen, const uint32_t* pnbr,
                                 const uint8_t* flags, const uint8_t* esize, uint32_t n, unsigned long long* out) {
  uint64_t closed = 0, probes = 0, rows = 0;
  for (uint64_t a = global_warp(); a < n; a += n_warps()) {
    const uint64_t s = poff[a];
    const uint32_t l = plen[a];
    if (l >= 2 && lane_id() == 0) rows += l;
    for (uint32_t i = lane_id(); i < l; i += 32) {
      const uint32_t b = pnbr[s + i];
      if (flags[s + i]) closed += 4ull * (esize[a] + esize[b]);
      if (l >= 2) probes += plen[b];
    }
  }
  closed = warp_sum(closed);
  probes = warp_sum(probes);
  rows = warp_sum(rows);
  if (lane_id() == 0) {
    if (closed) atomicAdd(&out[0], (unsigned long long)closed);
    if (probes) atomicAdd(&out[1], (unsigned long long)probes);
    if (rows) atomicAdd(&out[2], (unsigned long long)rows);
  }
}

}  // namespace
}  // namespace hm

extern "C" int hm_graph_traffic(hm_graph* g, hm_traffic_t* t) {
  if (!g || !t) return hm::set_error(HM_ERR_INVALID, "hm_graph_traffic: NULL argument");
  if (g->temporal) return hm::set_error(HM_ERR_STATE, "hm_graph_traffic: the graph is temporal");
  std::lock_guard<std::mutex> lock(g->ctx->mu);
  cudaSetDevice(g->ctx->device);
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  const uint32_t E = g->n_slots;
  HM_TRY(hm::prepare_static(g));
  hm::DArr<uint32_t> dp;
  hm::DArr<unsigned long long> acc;
  hm::DArr<uint8_t> flags;
  HM_TRY(dp.alloc(ctx, E));
  HM_TRY(acc.alloc(ctx, 4));
  HM_TRY(flags.alloc(ctx, g->plus_nnz));
  HM_CUDA(cudaMemsetAsync(acc.p, 0, 4 * sizeof(unsigned long long), st));
  HM_CUDA(cudaMemsetAsync(flags.p, 0, g->plus_nnz ? g->plus_nnz : 1, st));
  if (E) {
    hm::k_dplus_id<<<hm::grid_for(E, 256), 256, 0, st>>>(g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p, E, dp.p);
    HM_LAUNCH_CHECK();
    hm::k_merge_bytes<<<hm::grid_for((uint64_t)E * 32, 256), 256, 0, st>>>(g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p,
                                                                          dp.p, E, acc.p);
    HM_LAUNCH_CHECK();
  }
  // diagnostic triangle pass: flags every oriented entry that closes a triangle
  HM_TRY(hm::launch_static(g, 0, 1, flags.p));
  uint64_t dummy[30];
  HM_TRY(hm::finish_static(g, dummy));
  if (E) {
    hm::k_oriented_bytes<<<hm::grid_for((uint64_t)E * 32, 256), 256, 0, st>>>(
        g->plus_off.p, g->plus_len.p, g->plus_nbr.p, flags.p, g->esize.p, E, acc.p + 1);
    HM_LAUNCH_CHECK();
  }
  unsigned long long h[4];
  HM_CUDA(cudaMemcpyAsync(h, acc.p, sizeof(h), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  t->store_bytes = 4ull * g->h2v_nnz + 8ull * g->h2h_nnz;
  t->merge_bytes = h[0];
  t->closed_pair_bytes = h[1];
  t->b_static = t->store_bytes + t->merge_bytes + t->closed_pair_bytes;
  t->probes = h[2];
  // open phase: id (4) + overlap (1) per H2H entry; closed phase: each
  // oriented row of a work centre (id 4 + overlap/size 2 + mask 8) and one id
  // per probe
  t->kernel_bytes = 5ull * g->h2h_nnz + 14ull * h[3] + 4ull * h[2];
  t->closed_triangles = g->times.closed_triangles;
  return HM_OK;
}
