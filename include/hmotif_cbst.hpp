// hmotif_cbst.hpp - header-only C++ shim with the reference's host interface,
// implemented on the C ABI of hmotif.h.
//
// It keeps the shapes a caller of the reference store and counters uses:
//   * CBSTOperations-like store (dynamicHyperGraph/include/structure.hpp:45-64):
//     construct / insert / erase / findAndPrint, 1-based keys, flat int
//     payloads addressed by start offsets or inclusive prefix sizes;
//   * computeMotifCounts (dynamicHyperGraph/include/motif.hpp:10-13), which
//     here also returns the counts (30 bins, the reference's order) instead of
//     only printing them;
//   * computeMotifCountsDelta (dynamicHyperGraph/include/motif_update.hpp:
//     13-19) as one call that applies the batch and returns the exact change;
//   * the temporal ring of three layers (TemporalCBSTOperations /
//     TemporalHypergraphIndex, temporalDynamicHMotif/include/
//     temporal_structure.hpp:22-80, temporal_adjacency.hpp:9-19) and
//     computeTemporalMotifCountsStrictInc / ...Delta /
//     applyTemporalDeltasFromFile (include/temporal_count.hpp:10-30).
// One HypergraphStore holds H2V, V2H and H2H together; the reference needs
// three CBSTOperations for that. Errors throw hm::Error (the reference calls
// exit(-1)).
#pragma once

#include <climits>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "hmotif.h"

namespace hm {

struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& where)
      : std::runtime_error(where + ": " + std::string(hm_last_error()) + " (" + hm_status_string(s) + ")"), status(s) {}
};

inline void check(int s, const char* where) {
  if (s < 0) throw Error(s, where);
}

class Context {
 public:
  explicit Context(int device = 0, size_t budget_bytes = 0) { check(hm_ctx_create(device, budget_bytes, &c_), "hm_ctx_create"); }
  ~Context() { hm_ctx_destroy(c_); }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  hm_ctx* get() const { return c_; }

 private:
  hm_ctx* c_ = nullptr;
};

// Store of one hypergraph. Keys are the reference's 1-based hyperedge ids
// (engine id + 1); node ids are the values of the H2V payload.
class HypergraphStore {
 public:
  HypergraphStore(Context& ctx, const char* dataset_name) : ctx_(ctx), name_(dataset_name ? dataset_name : "") {}
  ~HypergraphStore() { hm_graph_destroy(g_); }
  HypergraphStore(const HypergraphStore&) = delete;
  HypergraphStore& operator=(const HypergraphStore&) = delete;

  // constructCBST's input (structure/operations.cu:31-80) for H2V: record i
  // (key i + 1) starts at startOffsets[i] in flatPayload and ends at a 0 pad
  // or INT_MIN sentinel, or at the next record's start.
  void construct(const int* startOffsets, int numRecords, const int* flatPayload, int flatPayloadSize,
                 uint32_t n_nodes) {
    std::vector<uint64_t> off(1, 0);
    std::vector<uint32_t> mem;
    for (int i = 0; i < numRecords; ++i) {
      const int end = (i + 1 < numRecords) ? startOffsets[i + 1] : flatPayloadSize;
      for (int k = startOffsets[i]; k < end; ++k) {
        const int v = flatPayload[k];
        if (v == 0 || v == INT_MIN) break;
        mem.push_back((uint32_t)v);
      }
      off.push_back(mem.size());
    }
    construct_csr(off, mem, n_nodes);
  }

  // The same from a CSR of 0-based member lists.
  void construct_csr(const std::vector<uint64_t>& offsets, const std::vector<uint32_t>& members, uint32_t n_nodes) {
    hm_graph_destroy(g_);
    g_ = nullptr;
    check(hm_graph_build(ctx_.get(), offsets.data(), members.data(), (uint32_t)(offsets.size() - 1), n_nodes,
                         nullptr, &g_),
          "hm_graph_build");
  }

  // insertCBST (structure/operations.cu:177-356): new records with payloads
  // given by inclusive prefix sizes. The engine assigns ids (smallest free
  // first, then new ones, as insertIntoDeletedKth and the reference's batch
  // builder do); the assigned 1-based keys are returned.
  std::vector<int> insert(const std::vector<int>& payload, const std::vector<int>& prefixSizes,
                          std::vector<int64_t>* delta30 = nullptr) {
    return update({}, payload, prefixSizes, delta30);
  }

  // CBSTOperations::insert(insertKeys, insertPayload, insertPrefixSizes)
  // (structure.hpp:54), i.e. fillCBST (structure/operations.cu:82-127,
  // 417-419): the values are appended to the existing records insertKeys
  // (1-based), insertPrefixSizes[i] the inclusive end of key i's values.
  // Records keep their keys; values a record already holds are ignored (its
  // members are a set). Optionally the exact 30-bin delta.
  void insert(const std::vector<int>& insertKeys, const std::vector<int>& insertPayload,
              const std::vector<int>& insertPrefixSizes, std::vector<int64_t>* delta30 = nullptr) {
    edit_members(insertKeys, insertPayload, insertPrefixSizes, delta30, false);
  }

  // unfillCBST (structure/operations.cu:439-453): the values are removed from
  // the records keysToUnfill.
  void unfill(const std::vector<int>& keysToUnfill, const std::vector<int>& valuesToRemove,
              const std::vector<int>& removePrefixSizes, std::vector<int64_t>* delta30 = nullptr) {
    edit_members(keysToUnfill, valuesToRemove, removePrefixSizes, delta30, true);
  }

  // deleteCBST (structure/operations.cu:129-175) on 1-based keys.
  void erase(const std::vector<int>& keys, std::vector<int64_t>* delta30 = nullptr) { update(keys, {}, {}, delta30); }

  // One batch: erase then insert, optionally with the exact 30-bin delta
  // (computeMotifCountsDelta, src/HMotifCountUpdate.cu:228-301).
  std::vector<int> update(const std::vector<int>& eraseKeys, const std::vector<int>& payload,
                          const std::vector<int>& prefixSizes, std::vector<int64_t>* delta30) {
    std::vector<uint32_t> dels;
    for (int k : eraseKeys) dels.push_back((uint32_t)(k - 1));
    std::vector<uint64_t> off(1, 0);
    std::vector<uint32_t> mem;
    int prev = 0;
    for (int end : prefixSizes) {
      for (int k = prev; k < end; ++k) mem.push_back((uint32_t)payload[k]);
      off.push_back(mem.size());
      prev = end;
    }
    std::vector<uint32_t> ids(prefixSizes.size());
    std::vector<int64_t> d(HM_N_STATIC_CLASSES);
    check(hm_graph_apply_batch(g_, dels.data(), (uint32_t)dels.size(), off.data(), mem.data(),
                               (uint32_t)prefixSizes.size(), ids.data(), delta30 ? d.data() : nullptr),
          "hm_graph_apply_batch");
    if (delta30) *delta30 = d;
    std::vector<int> keys;
    for (uint32_t i : ids) keys.push_back((int)i + 1);
    return keys;
  }

  // findAndPrint (structure/operations.cu:425-433): prints each record's
  // members, and returns them.
  std::vector<std::vector<uint32_t>> findAndPrint(const std::vector<int>& keys) const {
    std::vector<uint32_t> ids;
    for (int k : keys) ids.push_back((uint32_t)(k - 1));
    std::vector<uint64_t> off(ids.size() + 1);
    std::vector<uint32_t> mem(256 * (ids.size() + 1));
    check(hm_graph_query(g_, ids.data(), (uint32_t)ids.size(), off.data(), mem.data(), mem.size()), "hm_graph_query");
    std::vector<std::vector<uint32_t>> out;
    for (size_t i = 0; i < ids.size(); ++i) {
      out.emplace_back(mem.begin() + off[i], mem.begin() + off[i + 1]);
      std::printf("[%s] key %d:", name_.c_str(), keys[i]);
      for (uint32_t v : out.back()) std::printf(" %u", v);
      std::printf("\n");
    }
    return out;
  }

  // Launch schedules of the two counts (no reference counterpart): tune
  // once after construct, or apply a schedule tuned on a graph of the same
  // shape. Counts do not depend on them.
  hm_tune_report autotune(uint32_t sample_stride = 0) {
    hm_tune_report r{};
    check(hm_graph_autotune(g_, sample_stride, &r), "hm_graph_autotune");
    return r;
  }
  hm_schedule schedule() const {
    hm_schedule s{};
    check(hm_graph_get_schedule(g_, &s), "hm_graph_get_schedule");
    return s;
  }
  void set_schedule(const hm_schedule& s) { check(hm_graph_set_schedule(g_, &s), "hm_graph_set_schedule"); }

  hm_graph* context() const { return g_; }

 private:
  void edit_members(const std::vector<int>& keys, const std::vector<int>& values, const std::vector<int>& prefix,
                    std::vector<int64_t>* delta30, bool remove) {
    if (keys.size() != prefix.size()) throw std::invalid_argument("insert/unfill: one prefix size per key");
    std::vector<uint32_t> ids, vals;
    for (int k : keys) ids.push_back((uint32_t)(k - 1));
    for (int v : values) vals.push_back((uint32_t)v);
    if (vals.empty()) vals.push_back(0);
    std::vector<uint64_t> ends(prefix.begin(), prefix.end());
    if (ends.empty()) ends.push_back(0);
    std::vector<int64_t> d(HM_N_STATIC_CLASSES);
    const int s = remove ? hm_graph_unfill(g_, ids.data(), (uint32_t)keys.size(), vals.data(), ends.data(), d.data())
                         : hm_graph_fill(g_, ids.data(), (uint32_t)keys.size(), vals.data(), ends.data(), d.data());
    check(s, remove ? "hm_graph_unfill" : "hm_graph_fill");
    if (delta30) *delta30 = d;
  }

  Context& ctx_;
  std::string name_;
  hm_graph* g_ = nullptr;
};

// computeMotifCounts: 30 bins in the reference's order, printed like the
// reference prints them, and returned.
inline std::vector<uint64_t> computeMotifCounts(const HypergraphStore& store, bool print = true) {
  std::vector<uint64_t> c(HM_N_STATIC_CLASSES);
  check(hm_count_static30(store.context(), c.data()), "hm_count_static30");
  if (print) {
    std::printf("Motif counts (30 bins): ");
    for (int i = 0; i < HM_N_STATIC_CLASSES; ++i)
      std::printf("%llu%c", (unsigned long long)c[i], i + 1 < HM_N_STATIC_CLASSES ? ' ' : '\n');
  }
  return c;
}

// Logical layers of the temporal ring (temporal_structure.hpp:20).
enum class TemporalLayer { Older = HM_LAYER_OLDER, Middle = HM_LAYER_MIDDLE, Newest = HM_LAYER_NEWEST };

// The reference's three-layer ring on one hm_window: the H2V side of each
// layer (V2H follows by itself). Keys are the layer's 1-based hyperedge ids;
// vertex v is node v - 1, as in the delta files. The reference's
// per-layer insert / erase of whole records has no counterpart here: a
// layer is rebuilt with construct.
class TemporalWindow {
 public:
  // max_vertex: the largest vertex id any layer will hold.
  TemporalWindow(Context& ctx, uint32_t max_vertex) {
    check(hm_window_create(ctx.get(), max_vertex, &w_), "hm_window_create");
  }
  ~TemporalWindow() { hm_window_destroy(w_); }
  TemporalWindow(const TemporalWindow&) = delete;
  TemporalWindow& operator=(const TemporalWindow&) = delete;

  // construct(layer, ...) (temporal_structure.hpp:34-39): record i has key
  // cbstKeys[i] (1-based) and starts at cbstStartOffsets[i]; it ends at a
  // 0 pad, a negative value or the next record's start. Keys left out are
  // empty hyperedges. Replaces what the layer held.
  void construct(TemporalLayer layer, const int* cbstKeys, const int* cbstStartOffsets, int numRecords,
                 const int* flatPayload, int flatPayloadSize) {
    std::vector<std::vector<uint32_t>> rows;
    for (int i = 0; i < numRecords; ++i) {
      const int key = cbstKeys ? cbstKeys[i] : i + 1;
      if (key < 1) throw std::invalid_argument("TemporalWindow::construct: keys are 1-based");
      if ((int)rows.size() < key) rows.resize(key);
      const int end = (i + 1 < numRecords) ? cbstStartOffsets[i + 1] : flatPayloadSize;
      for (int k = cbstStartOffsets[i]; k < end; ++k) {
        const int v = flatPayload[k];
        if (v <= 0) break;
        rows[key - 1].push_back((uint32_t)(v - 1));
      }
    }
    std::vector<uint64_t> off(1, 0);
    std::vector<uint32_t> mem;
    for (const auto& r : rows) {
      mem.insert(mem.end(), r.begin(), r.end());
      off.push_back(mem.size());
    }
    check(hm_window_set_layer(w_, (int)layer, off.data(), mem.data(), (uint32_t)rows.size()), "hm_window_set_layer");
  }

  // fill / unfill (fillCBST / unfillCBST): vertices added to or removed from
  // existing hyperedges; prefix[i] is the inclusive end of keys[i]'s values.
  void fill(TemporalLayer layer, const std::vector<int>& keys, const std::vector<int>& payload,
            const std::vector<int>& prefix) {
    edit(layer, keys, payload, prefix, false);
  }
  void unfill(TemporalLayer layer, const std::vector<int>& keys, const std::vector<int>& valuesToRemove,
              const std::vector<int>& removePrefix) {
    edit(layer, keys, valuesToRemove, removePrefix, true);
  }

  // rotate (Middle becomes Older, Newest Middle, Older Newest) and resets.
  void rotate() { check(hm_window_rotate(w_), "hm_window_rotate"); }
  void resetLayer(TemporalLayer layer) { check(hm_window_reset_layer(w_, (int)layer), "hm_window_reset_layer"); }
  void resetNewest() { resetLayer(TemporalLayer::Newest); }

  uint32_t size(TemporalLayer layer) const {
    uint32_t n = 0;
    check(hm_window_layer_size(w_, (int)layer, &n), "hm_window_layer_size");
    return n;
  }
  hm_window* get() const { return w_; }

 private:
  void edit(TemporalLayer layer, const std::vector<int>& keys, const std::vector<int>& values,
            const std::vector<int>& prefix, bool remove) {
    if (keys.size() != prefix.size()) throw std::invalid_argument("TemporalWindow: one prefix end per key");
    std::vector<uint32_t> ids, vals;
    for (int k : keys) ids.push_back((uint32_t)(k - 1));
    for (int v : values) vals.push_back((uint32_t)(v - 1));
    std::vector<uint64_t> ends(prefix.begin(), prefix.end());
    const int s = remove ? hm_window_unfill(w_, (int)layer, ids.data(), (uint32_t)ids.size(), vals.data(), ends.data())
                         : hm_window_fill(w_, (int)layer, ids.data(), (uint32_t)ids.size(), vals.data(), ends.data());
    check(s, remove ? "hm_window_unfill" : "hm_window_fill");
  }

  hm_window* w_ = nullptr;
};

// computeTemporalMotifCountsStrictInc (temporal_count.hpp:10-16): the 30
// classes of the closed triples (i Older, j Middle, k Newest, i < j < k),
// without the reference's cap of 1024 candidates per middle hyperedge.
inline void computeTemporalMotifCountsStrictInc(const TemporalWindow& w, std::vector<int64_t>& outCounts30) {
  std::vector<uint64_t> c(HM_N_STATIC_CLASSES);
  check(hm_window_count30(w.get(), c.data()), "hm_window_count30");
  outCounts30.assign(c.begin(), c.end());
}

// computeTemporalMotifCountsStrictIncDelta: counts(newWindow) - counts(oldWindow).
inline void computeTemporalMotifCountsStrictIncDelta(const TemporalWindow& oldWindow, const TemporalWindow& newWindow,
                                                     std::vector<int64_t>& outDeltaCounts30) {
  std::vector<int64_t> a, b;
  computeTemporalMotifCountsStrictInc(oldWindow, a);
  computeTemporalMotifCountsStrictInc(newWindow, b);
  outDeltaCounts30.assign(HM_N_STATIC_CLASSES, 0);
  for (int i = 0; i < HM_N_STATIC_CLASSES; ++i) outDeltaCounts30[i] = b[i] - a[i];
}

// applyTemporalDeltasFromFile: "A|R <hyperedge> <vertices>" lines on the
// Newest layer; false (and nothing changed) on a bad file.
inline bool applyTemporalDeltasFromFile(const std::string& path, TemporalWindow& w) {
  return hm_window_apply_deltas_file(w.get(), path.c_str()) == HM_OK;
}

// MoCHy's 26 motifs (MoCHy-master/main_exact.cpp:133-137), 1-based "motif i".
inline std::vector<uint64_t> computeMoCHy26(const HypergraphStore& store) {
  std::vector<uint64_t> c(HM_N_STATIC_MOTIFS);
  check(hm_count_static(store.context(), c.data()), "hm_count_static");
  return c;
}

}  // namespace hm
