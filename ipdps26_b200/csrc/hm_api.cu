// C ABI entry points for graphs: build, destroy, info, query, static counts.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <vector>

#include "hm_classes.h"
#include "hm_device.h"

namespace {

constexpr unsigned kBlock = 256;

__global__ void k_query_sizes(const uint32_t* ids, uint32_t n, uint32_t n_slots, const uint32_t* live_bits,
                              const uint32_t* h2v_len, uint32_t* sizes, int* bad) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t id = ids[i];
    const bool live = id < n_slots && ((live_bits[id >> 5] >> (id & 31)) & 1u);
    if (!live) atomicExch(bad, 1);
    if (sizes) sizes[i] = live ? h2v_len[id] : 0;
  }
}

__global__ void k_query_gather(const uint32_t* ids, uint32_t n, const uint64_t* out_off, const uint64_t* h2v_off,
                               const uint32_t* h2v_mem, uint32_t* out) {
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  for (uint64_t i = warp; i < n; i += nw) {
    const uint64_t d = out_off[i], len = out_off[i + 1] - d;
    const uint64_t s = h2v_off[ids[i]];
    for (uint64_t k = lane; k < len; k += 32) out[d + k] = h2v_mem[s + k];
  }
}

struct CtxLock {
  std::lock_guard<std::mutex> g;
  explicit CtxLock(hm_ctx* c) : g(c->mu) { cudaSetDevice(c->device); }
};

}  // namespace

extern "C" int hm_graph_build(hm_ctx* ctx, const uint64_t* offsets, const uint32_t* members, uint32_t n_edges,
                              uint32_t n_nodes, const int64_t* timestamps, hm_graph** out) {
  if (!ctx || !out || (n_edges && !offsets) || (n_edges && offsets[n_edges] && !members))
    return hm::set_error(HM_ERR_INVALID, "hm_graph_build: NULL argument");
  *out = nullptr;
  if (n_edges && offsets[0] != 0) return hm::set_error(HM_ERR_INVALID, "hm_graph_build: offsets[0] must be 0");
  CtxLock lock(ctx);
  auto* g = new hm_graph();
  g->ctx = ctx;
  g->n_nodes = n_nodes;
  static const uint64_t zero_off = 0;
  const uint64_t* off = n_edges ? offsets : &zero_off;
  int s = hm::build_h2v(g, off, members, n_edges);
  // a temporal graph only needs its member lists; the time-ordered index is
  // built by the first temporal count
  if (s >= 0 && !timestamps) s = hm::build_v2h(g);
  if (s >= 0 && !timestamps) s = hm::build_h2h_rows(g);
  if (s >= 0 && timestamps) {
    s = g->ts.alloc(ctx, n_edges);
    if (s >= 0 && n_edges) {
      cudaError_t e = cudaMemcpyAsync(g->ts.p, timestamps, sizeof(int64_t) * n_edges, cudaMemcpyHostToDevice, ctx->stream);
      if (e != cudaSuccess) s = hm::set_error(HM_ERR_CUDA, "timestamps upload: %s", cudaGetErrorString(e));
    }
    g->temporal = true;
  }
  if (s >= 0) {
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) s = hm::set_error(HM_ERR_CUDA, "hm_graph_build: %s", cudaGetErrorString(e));
  }
  if (s < 0) {
    delete g;
    return s;
  }
  *out = g;
  return HM_OK;
}

extern "C" int hm_graph_destroy(hm_graph* g) {
  if (!g) return HM_OK;
  hm_ctx* ctx = g->ctx;
  {
    CtxLock lock(ctx);
    cudaStreamSynchronize(ctx->stream);
    delete g;
    hm::trim_pool(ctx);
  }
  return HM_OK;
}

extern "C" int hm_graph_info(const hm_graph* g, hm_graph_info_t* info) {
  if (!g || !info) return hm::set_error(HM_ERR_INVALID, "hm_graph_info: NULL argument");
  std::memset(info, 0, sizeof(*info));
  info->n_slots = g->n_slots;
  info->n_live = g->n_live;
  info->n_nodes = g->n_nodes;
  info->n_members = g->h2v_nnz;
  info->n_adjacent = g->h2h_nnz;
  info->n_oriented = g->plus_valid ? g->plus_nnz : 0;
  info->device_bytes = g->ctx->used.load();
  info->temporal = g->temporal ? 1 : 0;
  return HM_OK;
}

extern "C" int hm_graph_timings(const hm_graph* g, hm_timings_t* t) {
  if (!g || !t) return hm::set_error(HM_ERR_INVALID, "hm_graph_timings: NULL argument");
  t->open_ms = g->times.open_ms;
  t->closed_ms = g->times.closed_ms;
  t->count_ms = g->times.total_ms;
  t->update_ms = g->times.update_ms;
  t->temporal_ms = g->times.temporal_ms;
  t->closed_triangles = g->times.closed_triangles;
  return HM_OK;
}

static int static_ok(const hm_graph* g) {
  return g->temporal ? hm::set_error(HM_ERR_STATE, "static count: the graph is temporal; use hm_count_temporal") : HM_OK;
}

extern "C" int hm_count_static30(hm_graph* g, uint64_t out30[HM_N_STATIC_CLASSES]) {
  if (!g || !out30) return hm::set_error(HM_ERR_INVALID, "hm_count_static30: NULL argument");
  HM_TRY(static_ok(g));
  CtxLock lock(g->ctx);
  return hm::count_static30(g, 0, 1, out30);
}

extern "C" int hm_count_static30_shard(hm_graph* g, uint32_t shard, uint32_t n_shards,
                                       uint64_t out30[HM_N_STATIC_CLASSES]) {
  if (!g || !out30) return hm::set_error(HM_ERR_INVALID, "hm_count_static30_shard: NULL argument");
  HM_TRY(static_ok(g));
  CtxLock lock(g->ctx);
  return hm::count_static30(g, shard, n_shards, out30);
}

extern "C" int hm_count_static30_async(hm_graph* g, uint64_t* d_out30, void* stream) {
  if (!g || !d_out30) return hm::set_error(HM_ERR_INVALID, "hm_count_static30_async: NULL argument");
  HM_TRY(static_ok(g));
  CtxLock lock(g->ctx);
  return hm::count_static30_async(g, d_out30, static_cast<cudaStream_t>(stream));
}

extern "C" int hm_graph_set_schedule(hm_graph* g, const hm_schedule* s) {
  if (!g || !s) return hm::set_error(HM_ERR_INVALID, "hm_graph_set_schedule: NULL argument");
  CtxLock lock(g->ctx);
  return hm::set_schedule(g, hm::ClosedSchedule{s->warp_row, s->small_row},
                          hm::TouchSchedule{s->touch_warp_row, s->touch_mid_row});
}

extern "C" int hm_graph_get_schedule(const hm_graph* g, hm_schedule* s) {
  if (!g || !s) return hm::set_error(HM_ERR_INVALID, "hm_graph_get_schedule: NULL argument");
  s->warp_row = g->sched.warp_row;
  s->small_row = g->sched.small_row;
  s->touch_warp_row = g->tsched.warp_row;
  s->touch_mid_row = g->tsched.mid_row;
  return HM_OK;
}

extern "C" int hm_graph_autotune(hm_graph* g, uint32_t sample_stride, hm_tune_report* report) {
  if (!g) return hm::set_error(HM_ERR_INVALID, "hm_graph_autotune: NULL graph");
  HM_TRY(static_ok(g));
  CtxLock lock(g->ctx);
  const auto t0 = std::chrono::steady_clock::now();
  hm_tune_report R{};
  HM_TRY(hm::autotune_closed(g, sample_stride, R));
  HM_TRY(hm::autotune_touch(g, R));
  R.tune_ms = (float)std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (report) *report = R;
  return HM_OK;
}

extern "C" int hm_count_static(hm_graph* g, uint64_t out26[HM_N_STATIC_MOTIFS]) {
  if (!g || !out26) return hm::set_error(HM_ERR_INVALID, "hm_count_static: NULL argument");
  HM_TRY(static_ok(g));
  uint64_t c30[30];
  CtxLock lock(g->ctx);
  HM_TRY(hm::count_static30(g, 0, 1, c30));
  int m = 0;
  for (int k = 0; k < 30; ++k)
    if (hm::static_class_reported(k)) out26[m++] = c30[k];
  return HM_OK;
}

extern "C" int hm_graph_query(hm_graph* g, const uint32_t* ids, uint32_t n, uint64_t* offsets_out,
                              uint32_t* members_out, size_t members_cap) {
  if (!g || (n && (!ids || !offsets_out))) return hm::set_error(HM_ERR_INVALID, "hm_graph_query: NULL argument");
  CtxLock lock(g->ctx);
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  offsets_out[0] = 0;
  if (!n) return HM_OK;
  hm::DArr<uint32_t> d_ids, sizes, d_out;
  hm::DArr<uint64_t> d_off;
  hm::DArr<int> bad;
  HM_TRY(d_ids.alloc(ctx, n));
  HM_TRY(sizes.alloc(ctx, n));
  HM_TRY(d_off.alloc(ctx, (size_t)n + 1));
  HM_TRY(bad.alloc(ctx, 1));
  HM_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
  HM_CUDA(cudaMemcpyAsync(d_ids.p, ids, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st));
  k_query_sizes<<<hm::grid_for(n, kBlock), kBlock, 0, st>>>(d_ids.p, n, g->n_slots, g->live_bits.p, g->h2v_len.p,
                                                           sizes.p, bad.p);
  HM_LAUNCH_CHECK();
  HM_TRY(hm::exclusive_scan(ctx, sizes.p, d_off.p, n));
  int hbad = 0;
  HM_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaMemcpyAsync(offsets_out, d_off.p, sizeof(uint64_t) * ((size_t)n + 1), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  if (hbad) return hm::set_error(HM_ERR_NOT_LIVE, "hm_graph_query: an id is not a live hyperedge");
  const uint64_t total = offsets_out[n];
  if (total > members_cap)
    return hm::set_error(HM_ERR_CAPACITY, "hm_graph_query: %llu members > capacity %zu", (unsigned long long)total,
                         members_cap);
  if (!total) return HM_OK;
  if (!members_out) return hm::set_error(HM_ERR_INVALID, "hm_graph_query: members_out is NULL");
  HM_TRY(d_out.alloc(ctx, total));
  k_query_gather<<<hm::grid_for((uint64_t)n * 32, kBlock), kBlock, 0, st>>>(d_ids.p, n, d_off.p, g->h2v_off.p,
                                                                           g->h2v_mem.p, d_out.p);
  HM_LAUNCH_CHECK();
  HM_CUDA(cudaMemcpyAsync(members_out, d_out.p, sizeof(uint32_t) * total, cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  return HM_OK;
}

extern "C" int hm_classify_static(int pattern) { return hm::static_class_of_pattern(pattern & 127); }

extern "C" int hm_classify_temporal(int pattern) {
  for (int m = 0; m < HM_N_TEMPORAL_MOTIFS; ++m)
    if (hm::kTemporalMotifPattern[m] == (pattern & 127)) return m;
  return -1;
}

extern "C" int hm_graph_apply_batch(hm_graph* g, const uint32_t* del_ids, uint32_t n_del,
                                    const uint64_t* ins_offsets, const uint32_t* ins_members, uint32_t n_ins,
                                    uint32_t* assigned_ids_out, int64_t* delta30_out) {
  if (!g || (n_del && !del_ids) || (n_ins && (!ins_offsets || (ins_offsets[n_ins] && !ins_members))))
    return hm::set_error(HM_ERR_INVALID, "hm_graph_apply_batch: NULL argument");
  CtxLock lock(g->ctx);
  return hm::apply_batch(g, del_ids, n_del, ins_offsets, ins_members, n_ins, assigned_ids_out, delta30_out);
}

extern "C" int hm_graph_fill(hm_graph* g, const uint32_t* ids, uint32_t n, const uint32_t* values,
                             const uint64_t* prefix, int64_t* delta30_out) {
  if (!g || (n && (!ids || !prefix || (prefix[n - 1] && !values))))
    return hm::set_error(HM_ERR_INVALID, "hm_graph_fill: NULL argument");
  CtxLock lock(g->ctx);
  return hm::modify_members(g, ids, n, values, prefix, false, delta30_out);
}

extern "C" int hm_graph_unfill(hm_graph* g, const uint32_t* ids, uint32_t n, const uint32_t* values,
                               const uint64_t* prefix, int64_t* delta30_out) {
  if (!g || (n && (!ids || !prefix || (prefix[n - 1] && !values))))
    return hm::set_error(HM_ERR_INVALID, "hm_graph_unfill: NULL argument");
  CtxLock lock(g->ctx);
  return hm::modify_members(g, ids, n, values, prefix, true, delta30_out);
}

namespace {
struct Delta30 {
  int64_t v[HM_N_STATIC_CLASSES];
};
__global__ void k_store_delta30(Delta30 d, int64_t* out) {
  if (threadIdx.x < HM_N_STATIC_CLASSES) out[threadIdx.x] = d.v[threadIdx.x];
}
}  // namespace

extern "C" int hm_graph_apply_batch_async(hm_graph* g, const uint32_t* del_ids, uint32_t n_del,
                                          const uint64_t* ins_offsets, const uint32_t* ins_members, uint32_t n_ins,
                                          uint32_t* assigned_ids_out, int64_t* d_delta30, void* stream) {
  if (!g || (n_del && !del_ids) || (n_ins && (!ins_offsets || (ins_offsets[n_ins] && !ins_members))))
    return hm::set_error(HM_ERR_INVALID, "hm_graph_apply_batch_async: NULL argument");
  CtxLock lock(g->ctx);
  const cudaStream_t user = static_cast<cudaStream_t>(stream);
  hm::StreamOrder order(g->ctx->stream, user);
  HM_TRY(order.begin("hm_graph_apply_batch_async"));
  Delta30 d{};
  HM_TRY(hm::apply_batch(g, del_ids, n_del, ins_offsets, ins_members, n_ins, assigned_ids_out,
                         d_delta30 ? d.v : nullptr));
  if (d_delta30) {
    k_store_delta30<<<1, 32, 0, g->ctx->stream>>>(d, d_delta30);
    HM_LAUNCH_CHECK();
  }
  return order.end("hm_graph_apply_batch_async");
}

extern "C" int hm_count_touching30(hm_graph* g, const uint32_t* ids, uint32_t n, uint64_t out30[HM_N_STATIC_CLASSES]) {
  if (!g || !out30 || (n && !ids)) return hm::set_error(HM_ERR_INVALID, "hm_count_touching30: NULL argument");
  HM_TRY(static_ok(g));
  std::vector<uint32_t> u(ids, ids + n);
  std::sort(u.begin(), u.end());
  u.erase(std::unique(u.begin(), u.end()), u.end());
  CtxLock lock(g->ctx);
  hm_ctx* ctx = g->ctx;
  hm::DArr<uint32_t> d;
  hm::DArr<int> bad;
  HM_TRY(d.alloc(ctx, u.size()));
  HM_TRY(bad.alloc(ctx, 1));
  HM_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), ctx->stream));
  if (!u.empty()) {
    HM_CUDA(cudaMemcpyAsync(d.p, u.data(), sizeof(uint32_t) * u.size(), cudaMemcpyHostToDevice, ctx->stream));
    k_query_sizes<<<hm::grid_for(u.size(), kBlock), kBlock, 0, ctx->stream>>>(d.p, (uint32_t)u.size(), g->n_slots,
                                                                              g->live_bits.p, g->h2v_len.p, nullptr,
                                                                              bad.p);
    HM_LAUNCH_CHECK();
  }
  int hbad = 0;
  HM_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  HM_CUDA(cudaStreamSynchronize(ctx->stream));
  if (hbad) return hm::set_error(HM_ERR_NOT_LIVE, "hm_count_touching30: an id is not a live hyperedge");
  return hm::count_touching(g, d.p, (uint32_t)u.size(), out30);
}

extern "C" int hm_graph_live_ids(const hm_graph* g, uint32_t* out, uint32_t cap, uint32_t* n_out) {
  if (!g || !n_out) return hm::set_error(HM_ERR_INVALID, "hm_graph_live_ids: NULL argument");
  std::lock_guard<std::mutex> lk(g->ctx->mu);
  cudaSetDevice(g->ctx->device);
  const uint32_t words = (g->n_slots + 31) / 32;
  std::vector<uint32_t> bits(words);
  if (words)
    HM_CUDA(cudaMemcpyAsync(bits.data(), g->live_bits.p, sizeof(uint32_t) * words, cudaMemcpyDeviceToHost,
                            g->ctx->stream));
  HM_CUDA(cudaStreamSynchronize(g->ctx->stream));
  uint32_t n = 0;
  for (uint32_t id = 0; id < g->n_slots; ++id)
    if ((bits[id >> 5] >> (id & 31)) & 1u) {
      if (out && n < cap) out[n] = id;
      ++n;
    }
  *n_out = n;
  if (out && n > cap) return hm::set_error(HM_ERR_CAPACITY, "hm_graph_live_ids: %u live ids > capacity %u", n, cap);
  return HM_OK;
}

namespace hm {
int count_temporal96(hm_graph* g, int64_t delta, uint64_t out96[96]);
}

extern "C" int hm_count_temporal(hm_graph* g, int64_t delta, uint64_t out96[HM_N_TEMPORAL_MOTIFS]) {
  if (!g || !out96) return hm::set_error(HM_ERR_INVALID, "hm_count_temporal: NULL argument");
  CtxLock lock(g->ctx);
  return hm::count_temporal96(g, delta, out96);
}

extern "C" int hm_count_temporal_async(hm_graph* g, int64_t delta, uint64_t* d_out96, void* stream) {
  if (!g || !d_out96) return hm::set_error(HM_ERR_INVALID, "hm_count_temporal_async: NULL argument");
  CtxLock lock(g->ctx);
  hm::StreamOrder order(g->ctx->stream, static_cast<cudaStream_t>(stream));
  HM_TRY(order.begin("hm_count_temporal_async"));
  HM_TRY(hm::count_temporal96_async(g, delta, d_out96));
  return order.end("hm_count_temporal_async");
}

extern "C" int hm_graph_temporal_traffic(const hm_graph* g, hm_temporal_traffic_t* t) {
  if (!g || !t) return hm::set_error(HM_ERR_INVALID, "hm_graph_temporal_traffic: NULL argument");
  const hm::PhaseTimes& x = g->times;
  t->events = x.t_events;
  t->delta = x.t_delta;
  t->window_neighbours = x.t_nbrs;
  t->closed_pairs = x.t_closed_pairs;
  t->open_pairs = x.t_open_pairs;
  t->b_temp = 8 * x.t_nbrs + 8 * (x.t_nbrs + 2 * x.t_closed_pairs + x.t_open_pairs);
  return HM_OK;
}

extern "C" int hm_debug_static_groups(hm_graph* g, int on) {
  if (!g) return hm::set_error(HM_ERR_INVALID, "hm_debug_static_groups: NULL graph");
  CtxLock lock(g->ctx);
  g->use_groups = on != 0;
  if (!g->use_groups) hm::release_plus_groups(g);
  return HM_OK;
}

extern "C" int hm_debug_touch_orientation(hm_graph* g, int by_id) {
  if (!g) return hm::set_error(HM_ERR_INVALID, "hm_debug_touch_orientation: NULL graph");
  g->touch_by_id = by_id != 0;
  return HM_OK;
}

extern "C" int hm_count_vertex_triads(hm_graph* g, uint64_t out3[3]) {
  if (!g || !out3) return hm::set_error(HM_ERR_INVALID, "hm_count_vertex_triads: NULL argument");
  HM_TRY(static_ok(g));
  CtxLock lock(g->ctx);
  return hm::count_vertex_triads(g, out3);
}
