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
//     13-19) as one call that applies the batch and returns the exact change.
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

// MoCHy's 26 motifs (MoCHy-master/main_exact.cpp:133-137), 1-based "motif i".
inline std::vector<uint64_t> computeMoCHy26(const HypergraphStore& store) {
  std::vector<uint64_t> c(HM_N_STATIC_MOTIFS);
  check(hm_count_static(store.context(), c.data()), "hm_count_static");
  return c;
}

}  // namespace hm
