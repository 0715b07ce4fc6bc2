// Engine internals shared by the CUDA translation units: the context, device
// arrays with budget accounting, the graph store, and error helpers.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <functional>
#include <cstdint>
#include <mutex>
#include <vector>

#include "hm_internal.h"

#define HM_CUDA(call)                                                                                  \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if (e_ != cudaSuccess)                                                                             \
      return ::hm::set_error(HM_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
  } while (0)

#define HM_TRY(expr)          \
  do {                        \
    int s_ = (expr);          \
    if (s_ < 0) return s_;    \
  } while (0)

#define HM_LAUNCH_CHECK() HM_CUDA(cudaGetLastError())

struct hm_ctx {
  int device = 0;
  size_t budget = 0;  // bytes; 0 = all free memory at creation
  std::atomic<size_t> used{0};
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;  // every device array of the context, stream-ordered on `stream`
  int n_sms = 148;
  std::mutex mu;  // serialises calls that share this context
};

namespace hm {

int dev_alloc(hm_ctx* ctx, void** p, size_t bytes);
void dev_free(hm_ctx* ctx, void* p, size_t bytes);
void trim_pool(hm_ctx* ctx);  // returns the pool's cached free blocks to the device

// Owning device array; the context's budget is charged for its bytes.
template <class T>
struct DArr {
  hm_ctx* ctx = nullptr;
  T* p = nullptr;
  size_t n = 0;
  DArr() = default;
  DArr(const DArr&) = delete;
  DArr& operator=(const DArr&) = delete;
  DArr(DArr&& o) noexcept { *this = static_cast<DArr&&>(o); }
  DArr& operator=(DArr&& o) noexcept {
    if (this != &o) {
      release();
      ctx = o.ctx; p = o.p; n = o.n;
      o.p = nullptr; o.n = 0;
    }
    return *this;
  }
  ~DArr() { release(); }
  int alloc(hm_ctx* c, size_t count) {
    release();
    ctx = c;
    if (count == 0) count = 1;
    void* q = nullptr;
    HM_TRY(dev_alloc(c, &q, count * sizeof(T)));
    p = static_cast<T*>(q);
    n = count;
    return HM_OK;
  }
  void release() {
    if (p) dev_free(ctx, p, n * sizeof(T));
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return n * sizeof(T); }
};

int charge(hm_ctx* ctx, size_t bytes);  // budget only, no allocation
void uncharge(hm_ctx* ctx, size_t bytes);
bool vmm_available();  // the driver's virtual memory management calls were found

// Device memory that grows without its contents moving: virtual address
// space is reserved ahead and physical chunks are mapped at its end as it
// grows (CUDA virtual memory management). When the reservation is full a
// larger one is reserved and the chunks already held are mapped into it, so
// growth never copies data and never holds two copies at once. Without VMM
// support on the device it falls back to allocate-copy-free. Each grow and
// release synchronises the device (chunks are unmapped only when no kernel
// can use them). Budget-charged like DArr.
struct GrowSpace {
  hm_ctx* ctx = nullptr;
  char* base = nullptr;
  size_t mapped = 0;    // bytes usable from base
  size_t reserved = 0;  // bytes of virtual address space at base
  bool vmm = false;
  std::vector<unsigned long long> handles;
  std::vector<size_t> sizes;
  int grow(hm_ctx* c, size_t bytes);  // mapped >= bytes afterwards, contents kept
  void shrink(size_t bytes);          // gives back whole chunks past bytes (VMM only)
  void release();
  GrowSpace() = default;
  GrowSpace(const GrowSpace&) = delete;
  GrowSpace& operator=(const GrowSpace&) = delete;
  ~GrowSpace() { release(); }
};

template <class T>
struct GrowArr {
  GrowSpace s;
  T* p = nullptr;
  size_t n = 0;  // entries usable
  int alloc(hm_ctx* c, size_t count) {  // fresh, contents undefined
    release();
    return grow(c, count);
  }
  int grow(hm_ctx* c, size_t count) {  // keeps the first n entries
    if (count == 0) count = 1;
    if (count <= n) return 0;
    HM_TRY(s.grow(c, count * sizeof(T)));
    p = reinterpret_cast<T*>(s.base);
    n = s.mapped / sizeof(T);
    return 0;
  }
  void shrink(size_t count) {  // keeps at least the first count entries
    s.shrink(count * sizeof(T));
    n = s.mapped / sizeof(T);
  }
  void release() {
    s.release();
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return s.mapped; }
};

// Per-phase device times of the last count call (CUDA events on the
// context stream), reported through hm_graph_timings().
struct PhaseTimes {
  float open_ms = 0, closed_ms = 0, total_ms = 0, update_ms = 0, temporal_ms = 0;
  uint64_t closed_triangles = 0;
  // last temporal count: events, and the window-projection sizes it walked
  uint64_t t_events = 0, t_nbrs = 0, t_closed_pairs = 0, t_open_pairs = 0;
  int64_t t_delta = 0;
};

// Which launch shape of the closed phase takes a centre, by the length d of
// its oriented row: d <= warp_row one warp each (warp_row <= 128, the warp
// kernel's 256-slot tables), d <= small_row blocks with 4096-slot tables,
// longer rows blocks with 8192-slot tables. Counts never depend on it.
struct ClosedSchedule {
  uint32_t warp_row = 128;
  uint32_t small_row = 2048;
};

// The same for the touched-triple count, by the length of a marked
// hyperedge's row: <= warp_row one warp each (<= 128), <= mid_row blocks with
// 4096-slot tables (<= 2048), longer rows 16384-slot or global tables.
struct TouchSchedule {
  uint32_t warp_row = 128;
  uint32_t mid_row = 2048;
};

// Launch sequences of the static count captured as CUDA graphs (open phase,
// closed phase), replayed while the arguments they were captured with hold.
struct CountCapture {
  static constexpr unsigned kKey = 27;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  uint64_t key[kKey] = {};
  bool valid = false;
  void reset() {
    for (auto& e : exec)
      if (e) {
        cudaGraphExecDestroy(e);
        e = nullptr;
      }
    valid = false;
  }
};

}  // namespace hm

// The device-resident hypergraph. Three segment tables share one layout:
// key k owns entries [off[k], off[k] + len[k]) of its arena.
//   H2V  hyperedge slot -> sorted member node ids (u32)
//   V2H  node          -> sorted hyperedge slots (u32)
//   H2H  hyperedge slot -> sorted adjacent slots (u32), overlap size (u8),
//                          and the shared positions of the row owner's
//                          member list as a bit mask (u64, positions < 64)
// plus the oriented copy of H2H used by the triangle phase (neighbours of
// higher (degree, id) rank only), and per-slot sizes and liveness.
struct hm_graph {
  hm_ctx* ctx = nullptr;
  uint32_t n_slots = 0;  // ids 0..n_slots-1 (live or free)
  uint32_t n_nodes = 0;
  uint32_t n_live = 0;
  uint32_t cap_slots = 0;

  hm::DArr<uint8_t> esize;      // per slot, 0 for free slots
  hm::DArr<uint32_t> live_bits; // one bit per slot

  hm::DArr<uint64_t> h2v_off;
  hm::DArr<uint32_t> h2v_len;
  hm::DArr<uint32_t> h2v_mem;
  uint64_t h2v_tail = 0;
  uint64_t h2v_nnz = 0;  // live members (h2v_tail also counts dead space)

  hm::DArr<uint64_t> v2h_off;
  hm::DArr<uint32_t> v2h_len;
  hm::DArr<uint32_t> v2h_edge;
  uint64_t v2h_tail = 0;

  hm::DArr<uint64_t> h2h_off;
  hm::DArr<uint32_t> h2h_len;
  // the arena grows in place (a regrow compacts the rows, then maps more)
  hm::GrowArr<uint32_t> h2h_nbr;
  hm::GrowArr<uint8_t> h2h_ovl;
  hm::GrowArr<uint64_t> h2h_mask;
  uint64_t h2h_tail = 0;
  uint64_t h2h_nnz = 0;  // live entries
  uint64_t h2h_cap = 0;  // arena entries allocated

  // oriented adjacency (rebuilt lazily after updates)
  bool plus_valid = false;
  // touched-triple counts walk id-ordered row suffixes instead of N+ (no
  // oriented copy to rebuild after each batch; used by pooled stores)
  bool touch_by_id = false;
  hm::DArr<uint64_t> plus_off;
  hm::DArr<uint32_t> plus_len;
  hm::DArr<uint32_t> plus_nbr;
  hm::DArr<uint16_t> plus_os;  // (neighbour size << 8) | overlap
  uint64_t plus_nnz = 0;
  // the masks of the oriented rows longer than kLongRow, which the count
  // kernels search instead of tabling: per slot its start in long_mask
  hm::DArr<uint64_t> long_off;
  hm::DArr<uint64_t> long_mask;
  // The oriented rows once more, grouped for the static count's walk: in
  // each row, first the neighbours that share several members with the row
  // owner (or one at a position past 63 of its member list), then one group
  // per position p < 64 holding the neighbours whose only shared member is
  // the owner's p-th. Per row a group table of min(size, 64) + 2 entries
  // {start relative to the row, neighbours of size 1, of size 2, 0}, the
  // last one's start the row length. grp_opos follows the id-sorted oriented
  // entries: for (a, b) sharing exactly one member, that member's position
  // in b (0xff when they share several, or when it is past 63 in either).
  bool grp_valid = false;
  bool use_groups = true;  // hm_debug_static_groups: off walks every entry (same counts)
  hm::DArr<uint32_t> grp_nbr;
  hm::DArr<uint16_t> grp_os;
  hm::DArr<uint64_t> grp_base;   // per slot: its group table's first entry
  hm::DArr<uint4> grp_tab;
  hm::DArr<uint8_t> grp_opos;

  // static-count state that only changes with the graph
  bool work_valid = false;
  hm::DArr<uint32_t> work;  // centres owning oriented wedges, heaviest first
  uint32_t n_work = 0;
  uint32_t n_work_big = 0;  // the first n_work_big centres have rows longer than the small-table limit
  uint32_t n_work_mid = 0;  // centres [n_work_big, n_work_mid) have rows longer than the warp-kernel limit
  hm::ClosedSchedule sched; // the split of the work list into launch shapes
  hm::TouchSchedule tsched; // the split of marked rows in touched-triple counts
  hm::DArr<unsigned long long> counters;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  bool ev_ready = false;
  hm::CountCapture capture;

  // temporal (optional): timestamps per slot and the time-ordered index
  hm::DArr<int64_t> ts;
  bool temporal = false;
  bool t_ready = false;
  hm::DArr<uint32_t> t_order;   // position -> event (events by time, then index)
  hm::DArr<int64_t> t_time;     // position -> time
  hm::DArr<uint32_t> t_static;  // position -> static id (smallest event with the same node-set)
  hm::DArr<uint32_t> t_prev;    // position -> previous position of the same static id
  hm::DArr<uint64_t> t_ooff;    // static id -> its occurrence positions
  hm::DArr<uint32_t> t_olen;
  hm::DArr<uint32_t> t_opos;
  hm::DArr<uint64_t> t_voff;    // node -> positions of the events containing it
  hm::DArr<uint32_t> t_vlen;
  hm::DArr<uint32_t> t_vpos;

  hm::PhaseTimes times;

  ~hm_graph() {
    capture.reset();
    if (ev_ready)
      for (auto& e : ev) cudaEventDestroy(e);
  }
};

namespace hm {

// Store construction pieces (hm_store.cu).
int build_h2v(hm_graph* g, const uint64_t* h_off, const uint32_t* h_mem, uint32_t n_edges);
int build_v2h(hm_graph* g);
int build_h2h_rows(hm_graph* g);
int h2h_rows_for(hm_graph* g, const uint32_t* d_rows, uint32_t n_rows,
                 const std::function<int(uint64_t, uint64_t*)>& reserve, uint64_t* written);
int build_plus(hm_graph* g);
int build_plus_groups(hm_graph* g);
void release_plus_groups(hm_graph* g);
void release_plus(hm_graph* g);
// Oriented rows of a subset of slots (indexed by slot; only listed slots valid).
struct PlusRows {
  DArr<uint64_t> off;
  DArr<uint32_t> len;
  DArr<uint32_t> nbr;
  DArr<uint16_t> os;
  DArr<uint64_t> loff;   // masks of the rows longer than kLongRow, as hm_graph::long_off
  DArr<uint64_t> lmask;
  uint64_t nnz = 0;
};
// Oriented rows longer than this are searched, not tabled, by the count
// kernels (the largest shared-memory table holds 4096 entries).
constexpr uint32_t kLongRow = 4096;
int build_plus_rows(hm_graph* g, const uint32_t* d_rows, uint32_t n, PlusRows* P);
template <class T>
int exclusive_scan(hm_ctx* ctx, const T* in, uint64_t* out, uint64_t n);

// Temporal count (hm_temporal.cu): the 96 counts into device memory, queued
// on the context stream (all 2^64 - 1 if an event's window overflows the table).
int count_temporal96_async(hm_graph* g, int64_t delta, uint64_t* d_out96);

// Static count (hm_static.cu).
int prepare_static(hm_graph* g);
int launch_static(hm_graph* g, uint32_t shard, uint32_t n_shards, uint8_t* edge_flags);
int finish_static(hm_graph* g, uint64_t out30[30]);
int count_static30(hm_graph* g, uint32_t shard, uint32_t n_shards, uint64_t out30[30]);
int count_static30_async(hm_graph* g, uint64_t* d_out30, cudaStream_t user);
int count_vertex_triads(hm_graph* g, uint64_t out3[3]);
int set_schedule(hm_graph* g, const ClosedSchedule& s, const TouchSchedule& t);
// The autotuner's two parts: static count (hm_static.cu), touched-triple
// count (hm_delta.cu); each fills its half of the report.
int autotune_closed(hm_graph* g, uint32_t stride, hm_tune_report& report);
int autotune_touch(hm_graph* g, hm_tune_report& report);

// Touched-triple counts (hm_delta.cu). With gos set, the triples of each
// touched hyperedge's graph gos[slot] go to output row rog[gos[slot]]
// (n_rows rows of 30); the graphs of one call must not share hyperedges'
// neighbourhoods (pooled graphs are node-disjoint).
struct TouchRows {
  const uint32_t* gos = nullptr;
  const uint32_t* rog = nullptr;
  uint32_t n_rows = 1;
};
int count_touching_rows(hm_graph* g, const uint32_t* d_ids, uint32_t n, const TouchRows& rows, uint64_t* out);
int count_touching(hm_graph* g, const uint32_t* d_ids, uint32_t n, uint64_t out30[30]);
// Full counts of the graphs whose every live slot is listed (hm_static.cu).
int count_static_rows(hm_graph* g, const uint32_t* d_rows, uint32_t n, const TouchRows& rows, uint64_t* out);

// Batch updates (hm_update.cu).
struct BatchHooks {
  std::function<int(const uint32_t* d_dels, uint32_t n_del)> before;  // old graph, deleted slots
  std::function<int(const uint32_t* d_ins, uint32_t n_ins)> after;    // new graph, assigned slots
};
// forced_ids (host, n_ins entries, or null): the ids the insertions take
// instead of smallest-free-first; each must be free once the deletions ran.
int apply_batch_hooks(hm_graph* g, const uint32_t* h_dels, uint32_t n_del, const uint64_t* h_ins_off,
                      const uint32_t* h_ins_mem, uint32_t n_ins, uint32_t* assigned_out, const BatchHooks& hooks,
                      const uint32_t* forced_ids = nullptr);
int apply_batch(hm_graph* g, const uint32_t* h_dels, uint32_t n_del, const uint64_t* h_ins_off,
                const uint32_t* h_ins_mem, uint32_t n_ins, uint32_t* assigned_out, int64_t* delta30,
                const uint32_t* forced_ids = nullptr);
// Members added to (remove = false) or removed from live hyperedges, ids kept.
int modify_members(hm_graph* g, const uint32_t* h_ids, uint32_t n, const uint32_t* values, const uint64_t* prefix,
                   bool remove, int64_t* delta30);
int presize_h2h(hm_graph* g, uint32_t factor);
int trim_h2h(hm_graph* g);  // gives back the H2H arena's free tail

// Orders the context stream's work after a caller's stream and the caller's
// later work after it (two events); a null caller stream is CUDA's legacy
// default stream. Refuses streams under CUDA-graph capture: the calls that use
// it allocate from the context's pool and may wait on the context stream.
struct StreamOrder {
  cudaStream_t ctx_stream, user;
  cudaEvent_t e[2] = {nullptr, nullptr};
  StreamOrder(cudaStream_t c, cudaStream_t u) : ctx_stream(c), user(u) {}
  ~StreamOrder() {
    for (auto x : e)
      if (x) cudaEventDestroy(x);  // released once the recorded work completes
  }
  int begin(const char* where) {
    for (cudaStream_t s : {user, ctx_stream}) {
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      const cudaError_t r = cudaStreamIsCapturing(s, &cs);
      if (r != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return set_error(HM_ERR_STATE, "%s: the stream is being captured into a CUDA graph; call it outside the "
                         "capture", where);
      }
    }
    if (user == ctx_stream) return HM_OK;
    HM_CUDA(cudaEventCreateWithFlags(&e[0], cudaEventDisableTiming));
    HM_CUDA(cudaEventCreateWithFlags(&e[1], cudaEventDisableTiming));
    HM_CUDA(cudaEventRecord(e[0], user));
    HM_CUDA(cudaStreamWaitEvent(ctx_stream, e[0], 0));
    return HM_OK;
  }
  int end(const char* where) {
    (void)where;
    if (user == ctx_stream) return HM_OK;
    HM_CUDA(cudaEventRecord(e[1], ctx_stream));
    HM_CUDA(cudaStreamWaitEvent(user, e[1], 0));
    return HM_OK;
  }
};

#ifdef __CUDACC__
// The orientation of the oriented rows: b is "above" a when (deg b, b) >
// (deg a, a), deg the H2H degree; every triangle is found once, from its
// lowest-ranked corner, and hub rows stay short.
__device__ __forceinline__ bool rank_above(uint32_t a, uint32_t da, uint32_t b, uint32_t db) {
  return db > da || (db == da && b > a);
}

// The shared-position mask of owner's H2H entry for neighbour key (present
// by construction): a binary search of the owner's id-sorted row. The
// oriented rows keep no mask of their own.
__device__ __forceinline__ uint64_t row_mask(const uint64_t* off, const uint32_t* len, const uint32_t* nbr,
                                             const uint64_t* mask, uint32_t owner, uint32_t key) {
  const uint64_t s = off[owner];
  uint32_t lo = 0, hi = len[owner];
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(nbr + s + mid) < key) lo = mid + 1;
    else hi = mid;
  }
  return __ldg(mask + s + lo);
}
#endif

inline unsigned grid_for(uint64_t items, unsigned per_block, unsigned max_blocks = 148u * 32u) {
  uint64_t b = (items + per_block - 1) / per_block;
  if (b == 0) b = 1;
  return (unsigned)(b < max_blocks ? b : max_blocks);
}

}  // namespace hm
