// Seeded synthetic hypergraph generators (host code).
//
// These produce the workloads the engine is measured and checked on: static
// hypergraphs (sorted unique uint32 members, duplicate hyperedges redrawn),
// temporal hypergraphs with strictly increasing bursty int64 timestamps, and
// update batches. Everything is driven by our own xoshiro256** stream and our
// own inverse-CDF samplers, so a (seed, parameters) pair names the same graph
// on every machine and libc++/libstdc++ version.
//
// The laws restate the workload descriptions attached to the reference's
// benchmarks: hyperedge sizes from a truncated discrete power law, members
// drawn without replacement by node popularity P(rank r) ~ (r + q)^-s
// (Zipf-Mandelbrot; q = 0 is plain Zipf). The reference's own generator
// (dynamicHyperGraph/src/graphGeneration.cpp:10-29) draws uniform sizes and
// uniform members with rand(); it is not used because it is unseeded
// (srand(time(0))) and has no skew.
#include "hm_internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <unordered_map>
#include <vector>

namespace hm {

struct Rng {
  uint64_t s[4];
  static uint64_t splitmix(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  explicit Rng(uint64_t seed) {
    uint64_t x = seed;
    for (auto& w : s) w = splitmix(x);
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  // uniform in [0, 1)
  double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }
  // uniform integer in [0, n)
  uint64_t below(uint64_t n) { return (uint64_t)(uniform() * (double)n) % n; }
  // exponential with the given mean (inverse CDF)
  double exponential(double mean) { return -mean * std::log1p(-uniform()); }
};

// Discrete sampler over ranks 0..n-1 with weight w(r): cumulative table plus
// binary search (inverse CDF). Used for both sizes and node popularity.
struct CdfSampler {
  std::vector<double> cdf;
  template <class W>
  void build(uint32_t n, W w) {
    cdf.resize(n);
    double acc = 0.0;
    for (uint32_t r = 0; r < n; ++r) {
      acc += w(r);
      cdf[r] = acc;
    }
    for (auto& c : cdf) c /= acc;
    cdf[n - 1] = 1.0;
  }
  uint32_t draw(Rng& g) const {
    double u = g.uniform();
    return (uint32_t)(std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
  }
};

static uint64_t hash_members(const uint32_t* m, uint32_t k) {
  uint64_t h = 1469598103934665603ull ^ k;
  for (uint32_t i = 0; i < k; ++i) {
    h ^= m[i];
    h *= 1099511628211ull;
    h ^= h >> 29;
  }
  return h;
}

struct EdgeSampler {
  CdfSampler sizes, pop;
  std::vector<uint32_t> perm;  // popularity rank -> node id
  uint32_t k_min = 2, k_max = 2;

  void init(const hm_gen_params& p, Rng& g) {
    k_min = p.k_min;
    k_max = p.k_max;
    const double a = p.size_exp, s = p.pop_exp, q = p.pop_offset;
    sizes.build(k_max - k_min + 1, [&](uint32_t r) { return std::pow((double)(r + k_min), -a); });
    pop.build(p.n_nodes, [&](uint32_t r) { return std::pow((double)(r + 1) + q, -s); });
    perm.resize(p.n_nodes);
    for (uint32_t i = 0; i < p.n_nodes; ++i) perm[i] = i;
    if (p.permute_nodes) {
      for (uint32_t i = p.n_nodes - 1; i > 0; --i) {
        uint32_t j = (uint32_t)g.below((uint64_t)i + 1);
        std::swap(perm[i], perm[j]);
      }
    }
  }
  // Draw one hyperedge into out (sorted, unique); returns its size.
  uint32_t draw(Rng& g, uint32_t* out) const {
    uint32_t k = k_min + sizes.draw(g);
    if (k > perm.size()) k = (uint32_t)perm.size();
    uint32_t have = 0;
    while (have < k) {
      uint32_t v = perm[pop.draw(g)];
      bool dup = false;
      for (uint32_t i = 0; i < have; ++i)
        if (out[i] == v) { dup = true; break; }
      if (!dup) out[have++] = v;
    }
    std::sort(out, out + k);
    return k;
  }
};

// Exact-duplicate detector over sorted member lists.
struct DedupeSet {
  std::unordered_multimap<uint64_t, uint32_t> map;  // hash -> edge index
  const std::vector<uint64_t>* offs = nullptr;
  const std::vector<uint32_t>* mem = nullptr;
  bool contains(const uint32_t* m, uint32_t k, uint64_t h) const {
    auto range = map.equal_range(h);
    for (auto it = range.first; it != range.second; ++it) {
      uint32_t e = it->second;
      uint64_t b = (*offs)[e], len = (*offs)[e + 1] - b;
      if (len == k && std::memcmp(mem->data() + b, m, k * sizeof(uint32_t)) == 0) return true;
    }
    return false;
  }
};

}  // namespace hm

using hm::Rng;


static int check_params(const hm_gen_params* p) {
  if (!p || p->n_nodes == 0 || p->k_min < 1 || p->k_max < p->k_min || p->k_max > HM_MAX_EDGE_SIZE ||
      p->k_min > p->n_nodes)
    return HM_ERR_INVALID;
  return HM_OK;
}

extern "C" int hm_gen_static(const hm_gen_params* p, hm_hostgraph** out) {
  if (!out || check_params(p) != HM_OK) return hm::set_error(HM_ERR_INVALID, "hm_gen_static: bad parameters");
  try {
    Rng g(p->seed);
    hm::EdgeSampler es;
    es.init(*p, g);
    auto* hg = new hm_hostgraph();
    hg->n_nodes = p->n_nodes;
    hg->offsets.reserve((size_t)p->n_edges + 1);
    hg->offsets.push_back(0);
    hm::DedupeSet dd;
    dd.offs = &hg->offsets;
    dd.mem = &hg->members;
    if (p->dedupe) dd.map.reserve(p->n_edges);
    uint32_t buf[HM_MAX_EDGE_SIZE];
    while (hg->offsets.size() <= p->n_edges) {
      uint32_t k = es.draw(g, buf);
      if (p->dedupe) {
        uint64_t h = hm::hash_members(buf, k);
        if (dd.contains(buf, k, h)) {
          if (++hg->redraws > 64ull * p->n_edges + 1000000ull) {
            delete hg;
            return hm::set_error(HM_ERR_INVALID, "hm_gen_static: cannot draw enough distinct hyperedges");
          }
          continue;
        }
        dd.map.emplace(h, (uint32_t)(hg->offsets.size() - 1));
      }
      hg->members.insert(hg->members.end(), buf, buf + k);
      hg->offsets.push_back(hg->members.size());
    }
    *out = hg;
    return HM_OK;
  } catch (const std::bad_alloc&) {
    return hm::set_error(HM_ERR_NOMEM, "hm_gen_static: host allocation failed");
  }
}

extern "C" int hm_gen_temporal(const hm_gen_params* p, const hm_burst_params* b, hm_hostgraph** out) {
  if (!out || !b || check_params(p) != HM_OK || b->events_per_burst == 0 || !(b->burst_rate > 0) ||
      !(b->gap_mean > 0))
    return hm::set_error(HM_ERR_INVALID, "hm_gen_temporal: bad parameters");
  try {
    // Timestamps come from their own stream so that node-sets and times are
    // independent draws.
    Rng g(p->seed);
    Rng gt(p->seed ^ 0x7E3A11C0FFEEull);
    hm::EdgeSampler es;
    es.init(*p, g);
    auto* hg = new hm_hostgraph();
    hg->n_nodes = p->n_nodes;
    const uint32_t n = p->n_edges;
    // Bursts start as a Poisson process of the given rate; each burst holds
    // events_per_burst events separated by exponential gaps.
    std::vector<double> t;
    t.reserve(n);
    double burst_start = 0.0;
    while (t.size() < n) {
      burst_start += gt.exponential(1.0 / b->burst_rate);
      double x = burst_start;
      for (uint32_t i = 0; i < b->events_per_burst && t.size() < n; ++i) {
        if (i) x += gt.exponential(b->gap_mean);
        t.push_back(x);
      }
    }
    std::sort(t.begin(), t.end());
    // Rescale onto [0, span] when a span is requested, round, then force the
    // sequence strictly increasing (t_i <- max(t_i, t_{i-1} + 1)).
    const double scale = (b->span > 0 && t.back() > 0) ? (double)b->span / t.back() : 1.0;
    hg->times.resize(n);
    int64_t prev = INT64_MIN;
    for (uint32_t i = 0; i < n; ++i) {
      int64_t v = (int64_t)std::llround(t[i] * scale);
      if (prev != INT64_MIN && v <= prev) v = prev + 1;
      hg->times[i] = v;
      prev = v;
    }
    hg->offsets.reserve((size_t)n + 1);
    hg->offsets.push_back(0);
    uint32_t buf[HM_MAX_EDGE_SIZE];
    for (uint32_t i = 0; i < n; ++i) {
      uint32_t k = es.draw(g, buf);
      hg->members.insert(hg->members.end(), buf, buf + k);
      hg->offsets.push_back(hg->members.size());
    }
    *out = hg;
    return HM_OK;
  } catch (const std::bad_alloc&) {
    return hm::set_error(HM_ERR_NOMEM, "hm_gen_temporal: host allocation failed");
  }
}

extern "C" int hm_gen_batch(const hm_gen_params* p, uint64_t batch_seed, const uint32_t* live_ids, uint32_t n_live,
                            uint32_t n_edits, double insert_fraction, uint32_t* del_ids_out, uint32_t* n_del_out,
                            hm_hostgraph** ins_out) {
  if (!n_del_out || !ins_out || check_params(p) != HM_OK || (n_live && !live_ids) || !(insert_fraction >= 0) ||
      insert_fraction > 1)
    return hm::set_error(HM_ERR_INVALID, "hm_gen_batch: bad parameters");
  try {
    // The popularity tables come from p->seed (same node permutation as the
    // base graph); the batch's own draws come from batch_seed.
    Rng g0(p->seed);
    hm::EdgeSampler es;
    es.init(*p, g0);
    Rng g(batch_seed);
    uint32_t n_ins = (uint32_t)std::llround((double)n_edits * insert_fraction);
    uint32_t n_del = n_edits - n_ins;
    if (n_del > n_live) n_del = n_live;
    // Deletions: uniform over live hyperedges without replacement (partial
    // Fisher-Yates over a copy of the live list).
    if (n_del) {
      if (!del_ids_out) return hm::set_error(HM_ERR_INVALID, "hm_gen_batch: del_ids_out is NULL");
      std::vector<uint32_t> pool(live_ids, live_ids + n_live);
      for (uint32_t i = 0; i < n_del; ++i) {
        uint32_t j = i + (uint32_t)g.below((uint64_t)(n_live - i));
        std::swap(pool[i], pool[j]);
      }
      std::copy(pool.begin(), pool.begin() + n_del, del_ids_out);
      std::sort(del_ids_out, del_ids_out + n_del);
    }
    *n_del_out = n_del;
    auto* hg = new hm_hostgraph();
    hg->n_nodes = p->n_nodes;
    hg->offsets.reserve((size_t)n_ins + 1);
    hg->offsets.push_back(0);
    uint32_t buf[HM_MAX_EDGE_SIZE];
    for (uint32_t i = 0; i < n_ins; ++i) {
      uint32_t k = es.draw(g, buf);
      hg->members.insert(hg->members.end(), buf, buf + k);
      hg->offsets.push_back(hg->members.size());
    }
    *ins_out = hg;
    return HM_OK;
  } catch (const std::bad_alloc&) {
    return hm::set_error(HM_ERR_NOMEM, "hm_gen_batch: host allocation failed");
  }
}

extern "C" int hm_hostgraph_view(const hm_hostgraph* hg, hm_hostgraph_info* info) {
  if (!hg || !info) return hm::set_error(HM_ERR_INVALID, "hm_hostgraph_view: NULL argument");
  info->n_edges = (uint32_t)(hg->offsets.size() - 1);
  info->n_nodes = hg->n_nodes;
  info->n_members = hg->members.size();
  info->offsets = hg->offsets.data();
  info->members = hg->members.data();
  info->timestamps = hg->times.empty() ? nullptr : hg->times.data();
  info->redraws = hg->redraws;
  return HM_OK;
}

extern "C" void hm_hostgraph_free(hm_hostgraph* hg) { delete hg; }
