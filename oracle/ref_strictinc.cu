// TEST INFRASTRUCTURE ONLY: runs the reference's own strictly increasing
// temporal counter (temporalDynamicHMotif/src/temporal_count.cu:91-217,
// computeTemporalMotifCountsStrictInc) on three layers read from a file, and
// prints its 30 bins. build_ref.sh compiles this harness with nvcc together
// with the reference's store and counter sources where they lie; nothing of
// the reference is copied here.
//
// The layers go through the reference's own path: flatten2DVector
// (utils/flatten.cpp:11-31) for the H2V and V2H payloads, a
// TemporalHypergraphIndex (include/temporal_adjacency.hpp:9-19) whose six
// stores are built by constructCBST (structure/operations.cu:31-80), and the
// count call itself.
//
// Input: the largest vertex id V, then for Older, Middle, Newest: a count m
// and m lines "k v1 .. vk" (vertices 1..V, sorted, distinct). Record i of a
// layer has key i + 1; vertex v's V2H record has key v.
//
// Inputs must stay inside the reference's own limits: every hyperedge size
// not a multiple of 4 (flatten2DVector writes no end marker after a full
// group of 4, and the counter then reads on into the next record), and at
// most 1024 candidates per middle hyperedge (TEMPORAL_CAND_LIMIT).
#include <algorithm>
#include <cstdio>
#include <fstream>
#include <numeric>
#include <vector>

#include "structure.hpp"
#include "temporal_adjacency.hpp"
#include "temporal_count.hpp"
#include "utils.hpp"

int main(int argc, char** argv) {
  if (argc != 2) {
    std::fprintf(stderr, "usage: %s LAYERS_FILE\n", argv[0]);
    return 2;
  }
  std::ifstream in(argv[1]);
  int max_v = 0;
  if (!(in >> max_v) || max_v < 1) return 2;
  std::vector<std::vector<int>> h2v[3];
  for (auto& layer : h2v) {
    int m = 0;
    if (!(in >> m) || m < 1) return 2;
    layer.resize(m);
    for (auto& row : layer) {
      int k = 0;
      in >> k;
      row.resize(k);
      for (auto& v : row) in >> v;
    }
  }
  // V2H of each layer, and a capacity above every flat payload (the stores
  // zero what lies past the payload, which ends the last record's scan)
  std::vector<std::vector<int>> v2h[3];
  size_t cap = 0;
  for (int l = 0; l < 3; ++l) {
    v2h[l].assign(max_v, {});
    for (size_t e = 0; e < h2v[l].size(); ++e)
      for (int v : h2v[l][e]) v2h[l][v - 1].push_back((int)e + 1);
    cap = std::max(cap, flatten2DVector(h2v[l]).first.size());
    cap = std::max(cap, flatten2DVector(v2h[l]).first.size());
  }
  TemporalHypergraphIndex thg((int)cap + 64);
  const TemporalLayer layers[3] = {TemporalLayer::Older, TemporalLayer::Middle, TemporalLayer::Newest};
  std::vector<int> keep[12];  // host payloads, alive until the count is done
  for (int l = 0; l < 3; ++l) {
    auto hf = flatten2DVector(h2v[l]);
    keep[4 * l] = hf.first;
    keep[4 * l + 1] = hf.second;
    std::vector<int> hkeys(h2v[l].size());
    std::iota(hkeys.begin(), hkeys.end(), 1);
    thg.h2v.construct(layers[l], hkeys.data(), keep[4 * l + 1].data(), (int)hkeys.size(), keep[4 * l].data(),
                      (int)keep[4 * l].size());
    auto vf = flatten2DVector(v2h[l]);
    keep[4 * l + 2] = vf.first;
    keep[4 * l + 3] = vf.second;
    std::vector<int> vkeys(max_v);
    std::iota(vkeys.begin(), vkeys.end(), 1);
    thg.v2h.construct(layers[l], vkeys.data(), keep[4 * l + 3].data(), max_v, keep[4 * l + 2].data(),
                      (int)keep[4 * l + 2].size());
  }
  std::vector<int> counts;
  computeTemporalMotifCountsStrictInc(thg, counts);
  std::printf("strictinc30:");
  for (int c : counts) std::printf(" %d", c);
  std::printf("\n");
  return 0;
}
