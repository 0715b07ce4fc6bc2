// Request loop over many resident graphs (hm_serve_* in hmotif.h).
//
// Batched mode keeps every graph in one pooled store: graph k's nodes are
// shifted by a node base so that graphs never share a node, hence never a
// triple, and a per-slot graph tag (gos) routes each touched triple's counts
// to the output row of its graph's request. One round then serves one
// request of every admitted graph with a single sequence of launches:
//   1. touched-triple count of all deleted hyperedges on the old store;
//   2. one store update (deletions, insertions, H2H patches);
//   3. touched-triple count of all inserted hyperedges on the new store, and
//      the static count (open pairs, closed triangles over oriented rows
//      built for these graphs only) of every queried graph.
// Update request r gets after[r] - before[r]; count request q gets the static
// count of its graph. With count_from_deltas the server keeps each counted
// graph's counts current with the deltas of its updates and answers later
// count requests from them (both forms). Each graph keeps its
// own ids on the host (smallest free first, like hm_graph_apply_batch) mapped
// to pool slots, so results match a graph served alone.
#include <algorithm>
#include <array>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <queue>
#include <thread>
#include <unordered_map>
#include <vector>

#include "hm_device.h"

namespace {

constexpr uint32_t kNone = 0xffffffffu;
constexpr unsigned kBlock = 256;
// H2H arena headroom at start, in multiples of the live entries. The pooled
// store compacts one arena shared by every graph, so it gets more room
// between compactions; per-graph stores keep what the first batch would
// give them (measured on the served workload: 3x made the pool 12 % faster
// and the per-graph stores slower).
constexpr uint32_t kPoolHeadroom = 3;
constexpr uint32_t kStoreHeadroom = 2;

__global__ void k_set_gos(const uint32_t* slots, const uint32_t* graph, uint32_t n, uint32_t* gos) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    gos[slots[i]] = graph[i];
}

struct Request {
  uint64_t ticket = 0;
  uint32_t graph = 0;
  int kind = HM_REQ_UPDATE;
  std::vector<uint32_t> dels;
  std::vector<uint64_t> ins_off;
  std::vector<uint32_t> ins_mem;
  std::vector<uint32_t> assigned;
  hm_serve_result res{};
  bool done = false;
  uint64_t edits() const { return dels.size() + (ins_off.empty() ? 0 : ins_off.size() - 1); }
  uint32_t n_ins() const { return ins_off.empty() ? 0u : (uint32_t)(ins_off.size() - 1); }
};
using ReqPtr = std::shared_ptr<Request>;

// Host side of one graph's id space in the pooled store.
struct GraphIds {
  uint32_t n_nodes = 0;
  uint32_t node_base = 0;
  std::vector<uint32_t> slot_of_id;  // kNone for free ids
  std::priority_queue<uint32_t, std::vector<uint32_t>, std::greater<uint32_t>> free_ids;
  uint32_t n_live = 0;
};

struct Staged {
  std::vector<uint64_t> off;
  std::vector<uint32_t> mem;
  uint32_t n_nodes = 0;
};

double now_ms(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

struct hm_server {
  hm_ctx* ctx = nullptr;
  hm_serve_config cfg{};
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  std::vector<Staged> staged;
  bool started = false;
  int broken = 0;  // a failed round left the pooled store unusable: its status

  // batched mode
  hm_graph* pool = nullptr;
  hm::DArr<uint32_t> gos;  // per pool slot: its graph
  std::vector<GraphIds> ids;
  // per-request mode
  std::vector<hm_graph*> graphs;
  std::vector<int> graph_broken;  // per graph: status of a failed update that may have left it half updated
  // count_from_deltas: per graph, its current 30-class counts once known
  std::vector<uint8_t> counts_known;
  std::vector<std::array<uint64_t, 30>> counts;

  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<ReqPtr> pending;
  std::unordered_map<uint64_t, ReqPtr> tickets;
  uint64_t next_ticket = 1;
  uint64_t in_flight = 0;
  bool stop = false;
  std::thread loop;
  hm_serve_stats_t stats{};

  size_t budget() const { return cfg.mem_budget_bytes ? cfg.mem_budget_bytes : ctx->budget; }
};

namespace hm {
namespace {

// Device bytes one round may need on top of the store: counting scratch per
// slot, the V2H rebuild, patch buffers per touched H2H entry, and an arena
// regrow when the H2H arena is nearly full. Deliberately generous.
size_t round_estimate(const hm_graph* g, uint64_t edits, uint64_t extra_marked) {
  const double L = g->n_live ? (double)g->h2h_nnz / g->n_live : 0.0;
  const double touched = (double)edits * (L + 1.0);
  size_t est = (64ull << 20) + 48ull * g->n_slots + 32ull * g->h2v_nnz;
  est += (size_t)(320.0 * touched) + 32ull * extra_marked;
  const double entries = (double)g->h2h_nnz + 2.0 * touched;
  if (entries > 0.9 * (double)g->h2h_cap) est += (size_t)(26.0 * entries);
  return est;
}

// Host checks of an update request, in the order hm_graph_apply_batch makes
// them; node and id ranges are the graph's own.
int validate_update(const Request& r, uint32_t n_nodes, const std::function<bool(uint32_t)>& live) {
  {
    std::vector<uint32_t> t(r.dels);
    std::sort(t.begin(), t.end());
    if (std::adjacent_find(t.begin(), t.end()) != t.end())
      return set_error(HM_ERR_INVALID, "serve: a hyperedge id is deleted twice");
  }
  const uint32_t n_ins = r.n_ins();
  if (n_ins) {
    if (r.ins_off[0] != 0) return set_error(HM_ERR_INVALID, "serve: insert offsets must start at 0");
    for (uint32_t e = 0; e < n_ins; ++e)
      if (r.ins_off[e + 1] < r.ins_off[e]) return set_error(HM_ERR_INVALID, "serve: insert offsets decrease");
    if (r.ins_off[n_ins] > r.ins_mem.size()) return set_error(HM_ERR_INVALID, "serve: insert offsets past the members");
  }
  for (uint32_t d : r.dels)
    if (!live(d)) return set_error(HM_ERR_NOT_LIVE, "serve: a deleted id is not a live hyperedge");
  for (uint32_t e = 0; e < n_ins; ++e) {
    const uint64_t a = r.ins_off[e], b = r.ins_off[e + 1];
    for (uint64_t k = a; k < b; ++k)
      if (r.ins_mem[k] >= n_nodes) return set_error(HM_ERR_INVALID, "serve: a member id is >= n_nodes (%u)", n_nodes);
    if (b - a > HM_MAX_EDGE_SIZE) {
      std::vector<uint32_t> t(r.ins_mem.begin() + a, r.ins_mem.begin() + b);
      std::sort(t.begin(), t.end());
      if (std::unique(t.begin(), t.end()) - t.begin() > HM_MAX_EDGE_SIZE)
        return set_error(HM_ERR_LIMIT, "serve: a hyperedge has more than %d distinct members", HM_MAX_EDGE_SIZE);
    }
  }
  return HM_OK;
}

int grow_gos(hm_server* s, uint32_t need) {
  if (s->gos.n >= need) return HM_OK;
  hm::DArr<uint32_t> n;
  HM_TRY(n.alloc(s->ctx, std::max<size_t>(need, s->gos.n + s->gos.n / 2)));
  if (s->gos.n)
    HM_CUDA(cudaMemcpyAsync(n.p, s->gos.p, sizeof(uint32_t) * s->gos.n, cudaMemcpyDeviceToDevice, s->ctx->stream));
  s->gos = std::move(n);
  return HM_OK;
}

int build_stores(hm_server* s) {
  hm_ctx* ctx = s->ctx;
  s->counts_known.assign(s->staged.size(), 0);
  s->counts.assign(s->staged.size(), std::array<uint64_t, 30>{});
  if (s->cfg.mode == HM_SERVE_PER_REQUEST) {
    for (auto& st : s->staged) {
      auto* g = new hm_graph();
      g->ctx = ctx;
      g->n_nodes = st.n_nodes;
      const uint32_t n = (uint32_t)(st.off.size() - 1);
      int rc = build_h2v(g, st.off.data(), st.mem.data(), n);
      if (rc >= 0) rc = build_v2h(g);
      if (rc >= 0) rc = build_h2h_rows(g);
      if (rc >= 0) rc = presize_h2h(g, kStoreHeadroom);
      if (rc < 0) {
        delete g;
        return rc;
      }
      s->graphs.push_back(g);
      s->graph_broken.push_back(0);
    }
  } else {
    std::vector<uint64_t> off(1, 0);
    std::vector<uint32_t> mem, gos_h;
    uint64_t node_base = 0;
    for (uint32_t k = 0; k < s->staged.size(); ++k) {
      auto& st = s->staged[k];
      GraphIds gi;
      gi.n_nodes = st.n_nodes;
      gi.node_base = (uint32_t)node_base;
      const uint32_t n = (uint32_t)(st.off.size() - 1);
      for (uint32_t e = 0; e < n; ++e) {
        gi.slot_of_id.push_back((uint32_t)(off.size() - 1));
        for (uint64_t i = st.off[e]; i < st.off[e + 1]; ++i) mem.push_back(st.mem[i] + gi.node_base);
        off.push_back(mem.size());
        gos_h.push_back(k);
      }
      gi.n_live = n;
      s->ids.push_back(std::move(gi));
      node_base += st.n_nodes;
      if (node_base >= (1ull << 32)) return set_error(HM_ERR_LIMIT, "serve: the graphs hold more than 2^32 nodes");
    }
    auto* g = new hm_graph();
    g->ctx = ctx;
    g->n_nodes = (uint32_t)node_base;
    g->touch_by_id = true;
    const uint32_t n = (uint32_t)(off.size() - 1);
    int rc = build_h2v(g, off.data(), mem.data(), n);
    if (rc >= 0) rc = build_v2h(g);
    if (rc >= 0) rc = build_h2h_rows(g);
    if (rc >= 0) rc = presize_h2h(g, kPoolHeadroom);
    if (rc < 0) {
      delete g;
      return rc;
    }
    s->pool = g;
    HM_TRY(grow_gos(s, std::max<uint32_t>(n, 1)));
    if (n) HM_CUDA(cudaMemcpyAsync(s->gos.p, gos_h.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, ctx->stream));
  }
  HM_CUDA(cudaStreamSynchronize(ctx->stream));
  s->staged.clear();
  s->staged.shrink_to_fit();
  return HM_OK;
}

void finish(hm_server* s, Request& r, int status) {
  r.res.status = status;
  if (status < 0) {
    r.assigned.clear();
    r.res.n_assigned = 0;
    std::memset(r.res.delta30, 0, sizeof(r.res.delta30));
    std::memset(r.res.counts30, 0, sizeof(r.res.counts30));
  }
  r.res.done_ms = now_ms(s->t0);
}

// A count request that needs a full count (no counts kept for its graph).
bool counts_in_full(const hm_server* s, const Request& r) {
  return r.kind == HM_REQ_COUNT && !(s->cfg.count_from_deltas && s->counts_known[r.graph]);
}

// The exact delta of an update of graph k, added to its known counts
// (modulo 2^64, as the counts are uint64).
void add_delta(hm_server* s, uint32_t k, const int64_t delta30[30]) {
  if (!s->cfg.count_from_deltas || !s->counts_known[k]) return;
  for (int c = 0; c < 30; ++c) s->counts[k][c] += (uint64_t)delta30[c];
}

// One request on its own store (the plain per-call form). An update that
// fails for another reason than its own arguments (which are checked before
// the store changes) may have left the graph half updated: the graph then
// answers every later request with that status.
void serve_one(hm_server* s, Request& r) {
  hm_graph* g = s->graphs[r.graph];
  int& broken = s->graph_broken[r.graph];
  if (broken) {
    finish(s, r, broken);
    return;
  }
  int rc;
  if (r.kind == HM_REQ_COUNT) {
    if (s->cfg.count_from_deltas && s->counts_known[r.graph]) {
      std::memcpy(r.res.counts30, s->counts[r.graph].data(), sizeof(r.res.counts30));
      rc = HM_OK;
    } else {
      rc = count_static30(g, 0, 1, r.res.counts30);
      if (rc >= 0 && s->cfg.count_from_deltas) {
        std::memcpy(s->counts[r.graph].data(), r.res.counts30, sizeof(r.res.counts30));
        s->counts_known[r.graph] = 1;
      }
    }
  } else {
    const uint32_t n_ins = r.n_ins();
    r.assigned.resize(n_ins);
    static const uint64_t zero = 0;
    rc = apply_batch(g, r.dels.data(), (uint32_t)r.dels.size(), n_ins ? r.ins_off.data() : &zero, r.ins_mem.data(),
                     n_ins, r.assigned.data(), r.res.delta30);
    r.res.n_assigned = n_ins;
    if (rc < 0 && rc != HM_ERR_INVALID && rc != HM_ERR_NOT_LIVE && rc != HM_ERR_LIMIT) broken = rc;
    if (rc >= 0) add_delta(s, r.graph, r.res.delta30);
  }
  finish(s, r, rc < 0 ? rc : HM_OK);
}

// One round of the batched form over the pooled store.
void serve_round(hm_server* s, std::vector<ReqPtr>& batch) {
  hm_ctx* ctx = s->ctx;
  cudaStream_t st = ctx->stream;
  hm_graph* g = s->pool;
  if (s->broken) {
    for (auto& r : batch) finish(s, *r, s->broken);
    return;
  }
  // host validation and translation; failing requests leave the round
  std::vector<Request*> rows;
  std::vector<uint32_t> rog(s->ids.size(), 0);
  std::vector<uint32_t> dels, ins_graph, qslots;
  std::vector<uint64_t> ins_off(1, 0);
  std::vector<uint32_t> ins_mem;
  for (auto& rp : batch) {
    Request& r = *rp;
    GraphIds& gi = s->ids[r.graph];
    if (r.kind == HM_REQ_UPDATE) {
      auto live = [&](uint32_t id) { return id < gi.slot_of_id.size() && gi.slot_of_id[id] != kNone; };
      const int rc = validate_update(r, gi.n_nodes, live);
      if (rc < 0) {
        finish(s, r, rc);
        continue;
      }
      for (uint32_t d : r.dels) dels.push_back(gi.slot_of_id[d]);
      for (uint32_t e = 0; e < r.n_ins(); ++e) {
        for (uint64_t k = r.ins_off[e]; k < r.ins_off[e + 1]; ++k) ins_mem.push_back(r.ins_mem[k] + gi.node_base);
        ins_off.push_back(ins_mem.size());
        ins_graph.push_back(r.graph);
      }
    } else {
      if (s->cfg.count_from_deltas && s->counts_known[r.graph]) {
        // the graph's earlier requests were served in earlier rounds
        std::memcpy(r.res.counts30, s->counts[r.graph].data(), sizeof(r.res.counts30));
        finish(s, r, HM_OK);
        continue;
      }
      for (uint32_t slot : gi.slot_of_id)
        if (slot != kNone) qslots.push_back(slot);
    }
    rog[r.graph] = (uint32_t)rows.size();
    rows.push_back(&r);
  }
  if (rows.empty()) return;
  const bool trace = std::getenv("HM_TRACE") != nullptr;
  const auto t_prep = std::chrono::steady_clock::now();
  const uint32_t R = (uint32_t)rows.size();
  const uint32_t n_del = (uint32_t)dels.size(), n_ins = (uint32_t)ins_graph.size();
  std::vector<uint64_t> before((size_t)R * 30, 0), after((size_t)R * 30, 0), full((size_t)R * 30, 0);
  std::vector<uint32_t> assigned(n_ins);
  int rc = HM_OK;
  do {
    hm::DArr<uint32_t> d_rog, d_ins_graph, d_q;
    if ((rc = d_rog.alloc(ctx, rog.size())) < 0) break;
    if (cudaMemcpyAsync(d_rog.p, rog.data(), sizeof(uint32_t) * rog.size(), cudaMemcpyHostToDevice, st) != cudaSuccess) {
      rc = set_error(HM_ERR_CUDA, "serve: upload of the row map failed");
      break;
    }
    // on the new store: touched triples of the insertions (update rows) and
    // full counts of the queried graphs (count rows)
    auto count_after = [&](const uint32_t* d_ins, uint32_t n) -> int {
      HM_TRY(grow_gos(s, g->n_slots));
      if (n) {
        HM_TRY(d_ins_graph.alloc(ctx, n));
        HM_CUDA(cudaMemcpyAsync(d_ins_graph.p, ins_graph.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st));
        k_set_gos<<<grid_for(n, kBlock), kBlock, 0, st>>>(d_ins, d_ins_graph.p, n, s->gos.p);
        HM_LAUNCH_CHECK();
        HM_TRY(count_touching_rows(g, d_ins, n, TouchRows{s->gos.p, d_rog.p, R}, after.data()));
      }
      if (!qslots.empty()) {
        HM_TRY(d_q.alloc(ctx, qslots.size()));
        HM_CUDA(cudaMemcpyAsync(d_q.p, qslots.data(), sizeof(uint32_t) * qslots.size(), cudaMemcpyHostToDevice, st));
        HM_TRY(count_static_rows(g, d_q.p, (uint32_t)qslots.size(), TouchRows{s->gos.p, d_rog.p, R}, full.data()));
      }
      return HM_OK;
    };
    if (n_del == 0 && n_ins == 0) {  // queries only: no store update
      rc = count_after(nullptr, 0);
      break;
    }
    BatchHooks hooks;
    hooks.before = [&](const uint32_t* d, uint32_t n) -> int {
      return n ? count_touching_rows(g, d, n, TouchRows{s->gos.p, d_rog.p, R}, before.data()) : (int)HM_OK;
    };
    hooks.after = count_after;
    rc = apply_batch_hooks(g, dels.data(), n_del, ins_off.data(), ins_mem.data(), n_ins, assigned.data(), hooks);
    if (rc < 0) s->broken = rc;  // the store may be half updated
  } while (false);
  if (rc < 0) {
    for (Request* r : rows) finish(s, *r, rc);
    return;
  }
  if (trace)
    std::fprintf(stderr, "[hm_trace serve_round] requests=%u deletions=%u insertions=%u queried_slots=%zu device=%.1fms\n",
                 R, n_del, n_ins, qslots.size(),
                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_prep).count());
  // results and host id bookkeeping, request by request
  uint32_t ins_pos = 0;
  for (uint32_t row = 0; row < R; ++row) {
    Request& r = *rows[row];
    const uint64_t* a = after.data() + (size_t)row * 30;
    const uint64_t* b = before.data() + (size_t)row * 30;
    if (r.kind == HM_REQ_COUNT) {
      std::memcpy(r.res.counts30, full.data() + (size_t)row * 30, sizeof(r.res.counts30));
      if (s->cfg.count_from_deltas) {
        std::memcpy(s->counts[r.graph].data(), r.res.counts30, sizeof(r.res.counts30));
        s->counts_known[r.graph] = 1;
      }
    } else {
      for (int k = 0; k < 30; ++k) r.res.delta30[k] = (int64_t)(a[k] - b[k]);
      add_delta(s, r.graph, r.res.delta30);
      GraphIds& gi = s->ids[r.graph];
      for (uint32_t d : r.dels) {
        gi.slot_of_id[d] = kNone;
        gi.free_ids.push(d);
      }
      gi.n_live -= (uint32_t)r.dels.size();
      const uint32_t ni = r.n_ins();
      r.assigned.resize(ni);
      for (uint32_t e = 0; e < ni; ++e) {
        uint32_t id;
        if (!gi.free_ids.empty()) {
          id = gi.free_ids.top();
          gi.free_ids.pop();
        } else {
          id = (uint32_t)gi.slot_of_id.size();
          gi.slot_of_id.push_back(kNone);
        }
        gi.slot_of_id[id] = assigned[ins_pos + e];
        r.assigned[e] = id;
      }
      ins_pos += ni;
      gi.n_live += ni;
      r.res.n_assigned = ni;
    }
    finish(s, r, HM_OK);
  }
}

// Picks the next round: in arrival order, the oldest waiting request of each
// graph, while the limits and the memory budget allow. A graph whose oldest
// request is held back contributes nothing this round (its order is kept).
std::vector<ReqPtr> select_round(hm_server* s) {
  std::vector<ReqPtr> out;
  if (s->cfg.mode == HM_SERVE_PER_REQUEST) {
    ReqPtr r = s->pending.front();
    s->pending.pop_front();
    out.push_back(r);
    return out;
  }
  std::vector<uint8_t> seen(s->ids.size(), 0);
  uint64_t edits = 0, marked = 0;
  const size_t used = s->ctx->used.load(), budget = s->budget();
  for (auto it = s->pending.begin(); it != s->pending.end();) {
    Request& r = **it;
    if (r.graph >= seen.size() || seen[r.graph]) {
      ++it;
      continue;
    }
    seen[r.graph] = 1;
    const uint64_t e = r.edits();
    const uint64_t m = counts_in_full(s, r) ? s->ids[r.graph].n_live : 0;
    bool take = true;
    if (s->cfg.max_batch_requests && out.size() >= s->cfg.max_batch_requests) take = false;
    if (take && s->cfg.max_batch_edits && !out.empty() && edits + e > s->cfg.max_batch_edits) take = false;
    if (take && !out.empty() && used + round_estimate(s->pool, edits + e, marked + m) > budget) {
      take = false;
      ++s->stats.deferred_budget;
    }
    if (!take) {
      ++it;
      continue;
    }
    edits += e;
    marked += m;
    out.push_back(*it);
    it = s->pending.erase(it);
  }
  return out;
}

void loop_main(hm_server* s) {
  cudaSetDevice(s->ctx->device);
  for (;;) {
    std::vector<ReqPtr> batch;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] { return s->stop || !s->pending.empty(); });
      if (s->pending.empty()) break;  // stop requested and nothing left
      batch = select_round(s);
      s->in_flight = batch.size();
    }
    const double t_start = now_ms(s->t0);
    for (auto& r : batch) {
      r->res.start_ms = t_start;
      r->res.round_requests = (uint32_t)batch.size();
    }
    {
      std::lock_guard<std::mutex> ctx_lock(s->ctx->mu);
      if (s->cfg.mode == HM_SERVE_PER_REQUEST) {
        for (auto& r : batch) {
          // a request that cannot fit the budget alone fails before any device work
          const hm_graph* g = s->graphs[r->graph];
          const size_t est = round_estimate(g, r->edits(), counts_in_full(s, *r) ? g->n_live : 0);
          if (s->ctx->used.load() + est > s->budget())
            finish(s, *r, set_error(HM_ERR_NOMEM, "serve: the request does not fit the memory budget"));
          else
            serve_one(s, *r);
        }
      } else {
        bool fits = true;
        if (batch.size() == 1) {  // a request admitted alone must still fit
          Request& r = *batch[0];
          const uint64_t m = counts_in_full(s, r) ? s->ids[r.graph].n_live : 0;
          if (s->ctx->used.load() + round_estimate(s->pool, r.edits(), m) > s->budget()) {
            finish(s, r, set_error(HM_ERR_NOMEM, "serve: the request does not fit the memory budget"));
            fits = false;
          }
        }
        if (fits) serve_round(s, batch);
      }
    }
    const double t_end = now_ms(s->t0);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      ++s->stats.rounds;
      s->stats.busy_ms += t_end - t_start;
      for (auto& r : batch) {
        r->done = true;
        if (r->res.status < 0) ++s->stats.requests_failed;
        else {
          ++s->stats.requests_done;
          s->stats.edits_done += r->edits();
        }
      }
      s->in_flight = 0;
    }
    s->cv_done.notify_all();
  }
}

int submit(hm_server* s, ReqPtr r, uint64_t* ticket_out) {
  std::lock_guard<std::mutex> lk(s->mu);
  if (!s->started) return set_error(HM_ERR_STATE, "serve: hm_serve_start has not been called");
  if (s->stop) return set_error(HM_ERR_STATE, "serve: the server is stopping");
  const size_t n_graphs = s->cfg.mode == HM_SERVE_PER_REQUEST ? s->graphs.size() : s->ids.size();
  if (r->graph >= n_graphs) return set_error(HM_ERR_INVALID, "serve: graph %u of %zu", r->graph, n_graphs);
  r->ticket = s->next_ticket++;
  r->res.ticket = r->ticket;
  r->res.graph = r->graph;
  r->res.kind = r->kind;
  r->res.submit_ms = now_ms(s->t0);
  s->tickets[r->ticket] = r;
  s->pending.push_back(r);
  if (ticket_out) *ticket_out = r->ticket;
  s->cv_work.notify_one();
  return HM_OK;
}

}  // namespace
}  // namespace hm

extern "C" int hm_serve_create(hm_ctx* ctx, const hm_serve_config* cfg, hm_server** out) {
  if (!ctx || !out) return hm::set_error(HM_ERR_INVALID, "hm_serve_create: NULL argument");
  *out = nullptr;
  auto* s = new hm_server();
  s->ctx = ctx;
  if (cfg) s->cfg = *cfg;
  if (s->cfg.mode != HM_SERVE_BATCHED && s->cfg.mode != HM_SERVE_PER_REQUEST) {
    delete s;
    return hm::set_error(HM_ERR_INVALID, "hm_serve_create: unknown mode %d", (int)cfg->mode);
  }
  if (s->cfg.count_from_deltas != 0 && s->cfg.count_from_deltas != 1) {
    delete s;
    return hm::set_error(HM_ERR_INVALID, "hm_serve_create: count_from_deltas must be 0 or 1");
  }
  *out = s;
  return HM_OK;
}

extern "C" int hm_serve_add_graph(hm_server* s, const uint64_t* offsets, const uint32_t* members, uint32_t n_edges,
                                  uint32_t n_nodes, uint32_t* graph_out) {
  if (!s || (n_edges && !offsets) || (n_edges && offsets[n_edges] && !members))
    return hm::set_error(HM_ERR_INVALID, "hm_serve_add_graph: NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->started) return hm::set_error(HM_ERR_STATE, "hm_serve_add_graph: the server has started");
  if (n_edges && offsets[0] != 0) return hm::set_error(HM_ERR_INVALID, "hm_serve_add_graph: offsets[0] must be 0");
  Staged st;
  st.n_nodes = n_nodes;
  st.off.assign(offsets ? offsets : nullptr, offsets ? offsets + n_edges + 1 : nullptr);
  if (st.off.empty()) st.off.push_back(0);
  for (uint32_t e = 0; e < n_edges; ++e)
    if (st.off[e + 1] < st.off[e]) return hm::set_error(HM_ERR_INVALID, "hm_serve_add_graph: offsets decrease");
  st.mem.assign(members, members + st.off.back());
  for (uint32_t v : st.mem)
    if (v >= n_nodes) return hm::set_error(HM_ERR_INVALID, "hm_serve_add_graph: a member id is >= n_nodes (%u)", n_nodes);
  if (graph_out) *graph_out = (uint32_t)s->staged.size();
  s->staged.push_back(std::move(st));
  return HM_OK;
}

extern "C" int hm_serve_start(hm_server* s) {
  if (!s) return hm::set_error(HM_ERR_INVALID, "hm_serve_start: NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->started) return hm::set_error(HM_ERR_STATE, "hm_serve_start: already started");
  {
    std::lock_guard<std::mutex> ctx_lock(s->ctx->mu);
    cudaSetDevice(s->ctx->device);
    HM_TRY(hm::build_stores(s));
  }
  s->started = true;
  s->loop = std::thread(hm::loop_main, s);
  return HM_OK;
}

extern "C" int hm_serve_submit_update(hm_server* s, uint32_t graph, const uint32_t* del_ids, uint32_t n_del,
                                      const uint64_t* ins_offsets, const uint32_t* ins_members, uint32_t n_ins,
                                      uint64_t* ticket_out) {
  if (!s || (n_del && !del_ids) || (n_ins && !ins_offsets) || (n_ins && ins_offsets[n_ins] && !ins_members))
    return hm::set_error(HM_ERR_INVALID, "hm_serve_submit_update: NULL argument");
  auto r = std::make_shared<Request>();
  r->graph = graph;
  r->kind = HM_REQ_UPDATE;
  r->dels.assign(del_ids, del_ids + n_del);
  if (n_ins) {
    r->ins_off.assign(ins_offsets, ins_offsets + n_ins + 1);
    r->ins_mem.assign(ins_members, ins_members + ins_offsets[n_ins]);
  }
  return hm::submit(s, r, ticket_out);
}

extern "C" int hm_serve_submit_count(hm_server* s, uint32_t graph, uint64_t* ticket_out) {
  if (!s) return hm::set_error(HM_ERR_INVALID, "hm_serve_submit_count: NULL server");
  auto r = std::make_shared<Request>();
  r->graph = graph;
  r->kind = HM_REQ_COUNT;
  return hm::submit(s, r, ticket_out);
}

extern "C" int hm_serve_wait(hm_server* s, uint64_t ticket, hm_serve_result* out, uint32_t* assigned, uint32_t cap) {
  if (!s || !out) return hm::set_error(HM_ERR_INVALID, "hm_serve_wait: NULL argument");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return hm::set_error(HM_ERR_INVALID, "hm_serve_wait: unknown ticket %llu", (unsigned long long)ticket);
  ReqPtr r = it->second;
  s->cv_done.wait(lk, [&] { return r->done; });
  *out = r->res;
  if (assigned && r->res.n_assigned) {
    if (cap < r->res.n_assigned)
      return hm::set_error(HM_ERR_CAPACITY, "hm_serve_wait: %u ids > capacity %u", r->res.n_assigned, cap);
    std::memcpy(assigned, r->assigned.data(), sizeof(uint32_t) * r->res.n_assigned);
  }
  s->tickets.erase(it);
  return HM_OK;
}

extern "C" int hm_serve_drain(hm_server* s) {
  if (!s) return hm::set_error(HM_ERR_INVALID, "hm_serve_drain: NULL server");
  std::unique_lock<std::mutex> lk(s->mu);
  s->cv_done.wait(lk, [&] { return s->pending.empty() && s->in_flight == 0; });
  return HM_OK;
}

extern "C" int hm_serve_stats(hm_server* s, hm_serve_stats_t* out) {
  if (!s || !out) return hm::set_error(HM_ERR_INVALID, "hm_serve_stats: NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  out->waiting = s->pending.size();
  out->device_bytes = s->ctx->used.load();
  return HM_OK;
}

extern "C" int hm_serve_live_ids(hm_server* s, uint32_t graph, uint32_t* out, uint32_t cap, uint32_t* n_out) {
  if (!s || !n_out) return hm::set_error(HM_ERR_INVALID, "hm_serve_live_ids: NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  if (!s->started) return hm::set_error(HM_ERR_STATE, "hm_serve_live_ids: the server has not started");
  if (!s->pending.empty() || s->in_flight) return hm::set_error(HM_ERR_STATE, "hm_serve_live_ids: requests are in flight");
  std::vector<uint32_t> ids;
  if (s->cfg.mode == HM_SERVE_PER_REQUEST) {
    if (graph >= s->graphs.size()) return hm::set_error(HM_ERR_INVALID, "hm_serve_live_ids: graph %u", graph);
    hm_graph* g = s->graphs[graph];
    ids.resize(g->n_live);
    uint32_t n = 0;
    HM_TRY(hm_graph_live_ids(g, ids.data(), (uint32_t)ids.size(), &n));
    ids.resize(n);
  } else {
    if (graph >= s->ids.size()) return hm::set_error(HM_ERR_INVALID, "hm_serve_live_ids: graph %u", graph);
    const auto& so = s->ids[graph].slot_of_id;
    for (uint32_t i = 0; i < so.size(); ++i)
      if (so[i] != kNone) ids.push_back(i);
  }
  *n_out = (uint32_t)ids.size();
  if (ids.size() > cap) return hm::set_error(HM_ERR_CAPACITY, "hm_serve_live_ids: %zu ids > capacity %u", ids.size(), cap);
  if (!ids.empty()) std::memcpy(out, ids.data(), sizeof(uint32_t) * ids.size());
  return HM_OK;
}

extern "C" int hm_serve_destroy(hm_server* s) {
  if (!s) return HM_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->loop.joinable()) s->loop.join();
  std::lock_guard<std::mutex> ctx_lock(s->ctx->mu);
  cudaSetDevice(s->ctx->device);
  cudaStreamSynchronize(s->ctx->stream);
  for (hm_graph* g : s->graphs) delete g;
  delete s->pool;
  s->gos.release();
  hm::trim_pool(s->ctx);
  delete s;
  return HM_OK;
}
