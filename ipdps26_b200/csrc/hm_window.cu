// Three-layer temporal window (Older, Middle, Newest) and its strictly
// increasing 30-class count.
//
// Reference: TemporalCBSTOperations, a 3-slot ring buffer of CBST stores
// (temporalDynamicHMotif/include/temporal_structure.hpp:22-80,
// src/temporal_structure.cpp), and computeTemporalMotifCountsStrictInc /
// temporalStrictIncAdjKernel (src/temporal_count.cu:91-217): closed triples
// (i of Older, j of Middle, k of Newest) with layer-local ids i < j < k and all
// three pairwise overlaps non-empty, counted by static class. The reference
// drops candidates beyond 1024 per middle hyperedge; this count has no cap.
//
// Layers are host lists (one id space per layer, ids from 0); a count builds
// one device store of the three layers (older slots first, then middle, then
// newest), reused until a layer changes. Kernel: one block per middle j. Its
// H2H row is sorted by slot, so the older neighbours i < j are a prefix and
// the newest neighbours k > j a suffix; the suffix goes into a shared table
// (each key with its position in row(j), whose overlap and shared-position
// mask a hit then reads), warps take i, and lanes walk the newest suffix of
// row(i) probing the table. g = |i & j & k| is popc(mask_ji & mask_jk) for
// |j| <= 64, else a three-way merge.
#include <algorithm>
#include <cstdio>
#include <fstream>
#include <iterator>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "hm_classes.h"
#include "hm_device.h"

namespace {

constexpr unsigned kBlock = 256;
constexpr unsigned kWarps = kBlock / 32;
constexpr unsigned kSlots = 16384;  // shared table (dynamic): newest neighbours of j, load <= 1/2
constexpr size_t kSmem = kSlots * (sizeof(uint32_t) + sizeof(uint16_t));
constexpr uint32_t kEmpty = 0xffffffffu;

struct Layer {
  std::vector<std::vector<uint32_t>> edges;  // member lists, id = position
};

// First index of row[0, n) with value > key (upper) or >= key, one warp.
template <bool upper>
__device__ __forceinline__ uint32_t wbound(const uint32_t* row, uint32_t n, uint32_t key) {
  const unsigned lane = threadIdx.x & 31u;
  uint32_t lo = 0, hi = n;
  while (hi - lo > 32) {
    const uint32_t step = (hi - lo + 31) / 32;
    const uint32_t p = lo + (lane + 1) * step - 1;
    bool before = false;
    if (p < hi) before = upper ? row[p] <= key : row[p] < key;
    lo += (uint32_t)__popc(__ballot_sync(0xffffffffu, before)) * step;
    hi = min(hi, lo + step);
  }
  bool before = false;
  if (lo + lane < hi) before = upper ? row[lo + lane] <= key : row[lo + lane] < key;
  return lo + (uint32_t)__popc(__ballot_sync(0xffffffffu, before));
}

__device__ uint32_t overlap3(const uint64_t* hoff, const uint32_t* hmem, const uint8_t* esize, uint32_t a, uint32_t b,
                             uint32_t c) {
  const uint32_t* x = hmem + hoff[a];
  const uint32_t* y = hmem + hoff[b];
  const uint32_t* z = hmem + hoff[c];
  const uint32_t nx = esize[a], ny = esize[b], nz = esize[c];
  uint32_t i = 0, j = 0, k = 0, g = 0;
  while (i < nx && j < ny && k < nz) {
    const uint32_t u = x[i], v = y[j], t = z[k];
    const uint32_t m = max(u, max(v, t));
    if (u == m && v == m && t == m) {
      ++g; ++i; ++j; ++k;
    } else {
      i += (u < m);
      j += (v < m);
      k += (t < m);
    }
  }
  return g;
}

struct WinArgs {
  const uint64_t* off;
  const uint32_t* len;
  const uint32_t* nbr;
  const uint8_t* ovl;
  const uint64_t* mask;
  const uint64_t* hoff;
  const uint32_t* hmem;
  const uint8_t* esize;
  uint32_t n0, n1, n2;  // layer sizes; slots: older [0, n0), middle [n0, n0 + n1), newest after
  unsigned int* queue;
  unsigned long long* out;  // 30 classes
  int* overflow;            // a middle row whose newest part exceeds the table
};

__global__ void __launch_bounds__(kBlock) k_strict_inc(WinArgs A) {
  extern __shared__ uint32_t win_smem[];
  uint32_t* keys = win_smem;                                     // kSlots
  uint16_t* sidx = reinterpret_cast<uint16_t*>(keys + kSlots);  // kSlots
  __shared__ unsigned long long cnt[30];
  __shared__ uint32_t s_item;
  const unsigned lane = threadIdx.x & 31u, w = threadIdx.x / 32;
  for (unsigned k = threadIdx.x; k < 30; k += blockDim.x) cnt[k] = 0;
  const uint32_t base2 = A.n0 + A.n1;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(A.queue, 1u);
    __syncthreads();
    const uint32_t j = s_item;
    if (j >= A.n1) break;
    const uint32_t sj = A.n0 + j;
    const uint64_t jo = A.off[sj];
    const uint32_t jl = A.len[sj];
    if (jl < 2) continue;
    const uint32_t* row = A.nbr + jo;
    // older i < j: slots [0, min(n0, j)); newest k > j: slots > base2 + j
    uint32_t i_end = 0, k_begin = 0;
    if (w == 0) {
      i_end = wbound<false>(row, jl, min(A.n0, j));
      k_begin = wbound<true>(row, jl, base2 + j);
    }
    __shared__ uint32_t s_i_end, s_k_begin;
    if (threadIdx.x == 0) {
      s_i_end = i_end;
      s_k_begin = k_begin;
    }
    __syncthreads();
    i_end = s_i_end;
    k_begin = s_k_begin;
    const uint32_t nk = jl - k_begin;
    if (i_end == 0 || nk == 0) continue;
    if (nk > kSlots / 2) {  // more than 8192 newest neighbours: reported, never skipped silently
      if (threadIdx.x == 0) atomicExch(A.overflow, 1);
      continue;
    }
    uint32_t slots = 64;
    while (slots < 2 * nk) slots <<= 1;
    for (uint32_t t = threadIdx.x; t < slots; t += blockDim.x) keys[t] = kEmpty;
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < nk; t += blockDim.x) {
      const uint32_t key = row[k_begin + t];
      uint32_t h = (key * 2654435761u) & (slots - 1);
      while (atomicCAS(&keys[h], kEmpty, key) != kEmpty) h = (h + 1) & (slots - 1);
      sidx[h] = (uint16_t)t;  // position in the newest part (< kSlots / 2)
    }
    __syncthreads();
    const uint32_t sjz = A.esize[sj];
    const bool masks = sjz <= 64;
    for (uint32_t ii = w; ii < i_end; ii += kWarps) {
      const uint32_t si = row[ii];
      const uint32_t cij = A.ovl[jo + ii];
      const uint64_t mji = A.mask[jo + ii];
      const uint32_t siz = A.esize[si];
      const uint64_t io = A.off[si];
      const uint32_t il = A.len[si];
      const uint32_t kb = wbound<true>(A.nbr + io, il, base2 + j);
      for (uint32_t t = kb + lane; t < il; t += 32) {
        const uint32_t sk = A.nbr[io + t];
        uint32_t h = (sk * 2654435761u) & (slots - 1);
        int at = -1;
        for (;;) {
          const uint32_t q = keys[h];
          if (q == sk) {
            at = (int)(k_begin + sidx[h]);
            break;
          }
          if (q == kEmpty) break;
          h = (h + 1) & (slots - 1);
        }
        if (at < 0) continue;
        const uint32_t cik = A.ovl[io + t];
        const uint32_t cjk = A.ovl[jo + at];
        const uint32_t g = masks ? (uint32_t)__popcll(mji & A.mask[jo + at]) : overlap3(A.hoff, A.hmem, A.esize, si, sj, sk);
        const int c = hm::static_class((int)siz, (int)sjz, (int)A.esize[sk], (int)cij, (int)cjk, (int)cik, (int)g);
        if (c >= 0) atomicAdd(&cnt[c], 1ull);
      }
    }
  }
  __syncthreads();
  for (unsigned k = threadIdx.x; k < 30; k += blockDim.x)
    if (cnt[k]) atomicAdd(&A.out[k], cnt[k]);
}

}  // namespace

struct hm_window {
  hm_ctx* ctx = nullptr;
  uint32_t n_nodes = 0;
  Layer slots[3];        // physical slots of the ring
  int oldest = 0;        // physical slot of the Older layer
  hm_graph* dev = nullptr;  // the three layers on the device, or null when stale

  Layer& layer(int l) { return slots[(oldest + l) % 3]; }
  void stale() {
    delete dev;
    dev = nullptr;
  }
};

namespace {

int check_layer(int layer) {
  return (layer < HM_LAYER_OLDER || layer > HM_LAYER_NEWEST)
             ? hm::set_error(HM_ERR_INVALID, "window: layer %d is not Older (0), Middle (1) or Newest (2)", layer)
             : (int)HM_OK;
}

int check_members(const hm_window* w, const uint32_t* mem, uint64_t n) {
  for (uint64_t i = 0; i < n; ++i)
    if (mem[i] >= w->n_nodes) return hm::set_error(HM_ERR_INVALID, "window: node %u >= n_nodes %u", mem[i], w->n_nodes);
  return HM_OK;
}

void normalise(std::vector<uint32_t>& r) {
  std::sort(r.begin(), r.end());
  r.erase(std::unique(r.begin(), r.end()), r.end());
}

int build_device(hm_window* w) {
  if (w->dev) return HM_OK;
  std::vector<uint64_t> off(1, 0);
  std::vector<uint32_t> mem;
  for (int l = 0; l < 3; ++l)
    for (const auto& e : w->layer(l).edges) {
      mem.insert(mem.end(), e.begin(), e.end());
      off.push_back(mem.size());
    }
  auto* g = new hm_graph();
  g->ctx = w->ctx;
  g->n_nodes = w->n_nodes;
  int rc = hm::build_h2v(g, off.data(), mem.data(), (uint32_t)(off.size() - 1));
  if (rc >= 0) rc = hm::build_v2h(g);
  if (rc >= 0) rc = hm::build_h2h_rows(g);
  if (rc < 0) {
    delete g;
    return rc;
  }
  w->dev = g;
  return HM_OK;
}

}  // namespace

extern "C" int hm_window_create(hm_ctx* ctx, uint32_t n_nodes, hm_window** out) {
  if (!ctx || !out) return hm::set_error(HM_ERR_INVALID, "hm_window_create: NULL argument");
  auto* w = new hm_window();
  w->ctx = ctx;
  w->n_nodes = n_nodes;
  *out = w;
  return HM_OK;
}

extern "C" int hm_window_destroy(hm_window* w) {
  if (!w) return HM_OK;
  {
    std::lock_guard<std::mutex> lk(w->ctx->mu);
    cudaSetDevice(w->ctx->device);
    cudaStreamSynchronize(w->ctx->stream);
    w->stale();
  }
  delete w;
  return HM_OK;
}

extern "C" int hm_window_set_layer(hm_window* w, int layer, const uint64_t* offsets, const uint32_t* members,
                                   uint32_t n_edges) {
  if (!w || (n_edges && !offsets) || (n_edges && offsets[n_edges] && !members))
    return hm::set_error(HM_ERR_INVALID, "hm_window_set_layer: NULL argument");
  HM_TRY(check_layer(layer));
  if (n_edges && offsets[0] != 0) return hm::set_error(HM_ERR_INVALID, "hm_window_set_layer: offsets[0] must be 0");
  for (uint32_t e = 0; e < n_edges; ++e)
    if (offsets[e + 1] < offsets[e]) return hm::set_error(HM_ERR_INVALID, "hm_window_set_layer: offsets decrease");
  if (n_edges) HM_TRY(check_members(w, members, offsets[n_edges]));
  Layer L;
  for (uint32_t e = 0; e < n_edges; ++e) {
    L.edges.emplace_back(members + offsets[e], members + offsets[e + 1]);
    normalise(L.edges.back());
    if (L.edges.back().size() > HM_MAX_EDGE_SIZE)
      return hm::set_error(HM_ERR_LIMIT, "hm_window_set_layer: a hyperedge has more than %d members", HM_MAX_EDGE_SIZE);
  }
  w->layer(layer) = std::move(L);
  w->stale();
  return HM_OK;
}

extern "C" int hm_window_rotate(hm_window* w) {
  if (!w) return hm::set_error(HM_ERR_INVALID, "hm_window_rotate: NULL window");
  w->oldest = (w->oldest + 1) % 3;  // Middle becomes Older, Newest Middle, Older Newest
  w->stale();
  return HM_OK;
}

extern "C" int hm_window_reset_layer(hm_window* w, int layer) {
  if (!w) return hm::set_error(HM_ERR_INVALID, "hm_window_reset_layer: NULL window");
  HM_TRY(check_layer(layer));
  w->layer(layer).edges.clear();
  w->stale();
  return HM_OK;
}

// fill (op 0) adds vertices to existing hyperedges, unfill (op 1) removes
// them (fillCBST / unfillCBST on one layer). prefix[i] is the inclusive
// end of key i's values, as the reference's prefix sizes.
static int fill_or_unfill(hm_window* w, int layer, const uint32_t* ids, uint32_t n, const uint32_t* values,
                          const uint64_t* prefix, bool remove) {
  if (!w || (n && (!ids || !prefix)) || (n && prefix[n - 1] && !values))
    return hm::set_error(HM_ERR_INVALID, "window fill: NULL argument");
  HM_TRY(check_layer(layer));
  Layer& L = w->layer(layer);
  for (uint32_t i = 0; i < n; ++i) {
    if (ids[i] >= L.edges.size()) return hm::set_error(HM_ERR_NOT_LIVE, "window fill: hyperedge %u of %zu", ids[i], L.edges.size());
    if (i && prefix[i] < prefix[i - 1]) return hm::set_error(HM_ERR_INVALID, "window fill: prefix sizes decrease");
  }
  if (n) HM_TRY(check_members(w, values, prefix[n - 1]));
  std::vector<std::vector<uint32_t>> next;  // validated copies first: a failure changes nothing
  for (uint32_t i = 0; i < n; ++i) {
    std::vector<uint32_t> r = L.edges[ids[i]];
    const uint64_t a = i ? prefix[i - 1] : 0, b = prefix[i];
    if (remove) {
      std::vector<uint32_t> del(values + a, values + b);
      normalise(del);
      std::vector<uint32_t> keep;
      std::set_difference(r.begin(), r.end(), del.begin(), del.end(), std::back_inserter(keep));
      r = std::move(keep);
    } else {
      r.insert(r.end(), values + a, values + b);
      normalise(r);
      if (r.size() > HM_MAX_EDGE_SIZE)
        return hm::set_error(HM_ERR_LIMIT, "window fill: a hyperedge would exceed %d members", HM_MAX_EDGE_SIZE);
    }
    next.push_back(std::move(r));
  }
  for (uint32_t i = 0; i < n; ++i) L.edges[ids[i]] = next[i];  // a repeated id: its last entry wins
  w->stale();
  return HM_OK;
}

extern "C" int hm_window_fill(hm_window* w, int layer, const uint32_t* ids, uint32_t n, const uint32_t* values,
                              const uint64_t* prefix) {
  return fill_or_unfill(w, layer, ids, n, values, prefix, false);
}

extern "C" int hm_window_unfill(hm_window* w, int layer, const uint32_t* ids, uint32_t n, const uint32_t* values,
                                const uint64_t* prefix) {
  return fill_or_unfill(w, layer, ids, n, values, prefix, true);
}

extern "C" int hm_window_apply_deltas_file(hm_window* w, const char* path) {
  if (!w || !path) return hm::set_error(HM_ERR_INVALID, "hm_window_apply_deltas_file: NULL argument");
  std::ifstream in(path);
  if (!in) return hm::set_error(HM_ERR_INVALID, "cannot open %s", path);
  // "A <hyperedge> v..." adds, "R <hyperedge> v..." removes vertices of a
  // Newest-layer hyperedge; ids and vertices are 1-based as in the
  // reference's delta files (src/temporal_count.cu:239-275). Removals first.
  std::map<uint32_t, std::vector<uint32_t>> add, rem;
  std::string line;
  uint64_t no = 0;
  while (std::getline(in, line)) {
    ++no;
    if (line.empty()) continue;
    std::istringstream iss(line);
    char op = 0;
    long long h = 0;
    if (!(iss >> op >> h) || (op != 'A' && op != 'R') || h <= 0)
      return hm::set_error(HM_ERR_INVALID, "%s:%llu: expected 'A|R <hyperedge> <vertices>'", path,
                           (unsigned long long)no);
    long long v;
    auto& dst = (op == 'A' ? add : rem)[(uint32_t)(h - 1)];
    while (iss >> v) {
      if (v <= 0 || v > (long long)w->n_nodes)
        return hm::set_error(HM_ERR_INVALID, "%s:%llu: vertex %lld outside [1, %u]", path, (unsigned long long)no, v,
                             w->n_nodes);
      dst.push_back((uint32_t)(v - 1));
    }
  }
  for (int pass = 0; pass < 2; ++pass) {
    const auto& m = pass == 0 ? rem : add;
    std::vector<uint32_t> ids, vals;
    std::vector<uint64_t> pre;
    for (const auto& kv : m) {
      ids.push_back(kv.first);
      vals.insert(vals.end(), kv.second.begin(), kv.second.end());
      pre.push_back(vals.size());
    }
    if (!ids.empty())
      HM_TRY(fill_or_unfill(w, HM_LAYER_NEWEST, ids.data(), (uint32_t)ids.size(), vals.data(), pre.data(), pass == 0));
  }
  return HM_OK;
}

extern "C" int hm_window_layer_size(const hm_window* w, int layer, uint32_t* n_edges) {
  if (!w || !n_edges) return hm::set_error(HM_ERR_INVALID, "hm_window_layer_size: NULL argument");
  HM_TRY(check_layer(layer));
  *n_edges = (uint32_t)const_cast<hm_window*>(w)->layer(layer).edges.size();
  return HM_OK;
}

extern "C" int hm_window_count30(hm_window* w, uint64_t out30[HM_N_STATIC_CLASSES]) {
  if (!w || !out30) return hm::set_error(HM_ERR_INVALID, "hm_window_count30: NULL argument");
  std::lock_guard<std::mutex> lk(w->ctx->mu);
  cudaSetDevice(w->ctx->device);
  for (int k = 0; k < 30; ++k) out30[k] = 0;
  const uint32_t n0 = (uint32_t)w->layer(0).edges.size(), n1 = (uint32_t)w->layer(1).edges.size(),
                 n2 = (uint32_t)w->layer(2).edges.size();
  if (!n0 || !n1 || !n2) return HM_OK;
  HM_TRY(build_device(w));
  hm_graph* g = w->dev;
  hm_ctx* ctx = w->ctx;
  cudaStream_t st = ctx->stream;
  hm::DArr<unsigned long long> cnt;
  HM_TRY(cnt.alloc(ctx, 32));
  HM_CUDA(cudaMemsetAsync(cnt.p, 0, 32 * sizeof(unsigned long long), st));
  WinArgs A{g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p, g->h2h_ovl.p, g->h2h_mask.p, g->h2v_off.p, g->h2v_mem.p,
            g->esize.p, n0, n1, n2, reinterpret_cast<unsigned int*>(cnt.p + 30), cnt.p,
            reinterpret_cast<int*>(cnt.p + 31)};
  static bool attr = false;
  if (!attr) {
    HM_CUDA(cudaFuncSetAttribute(k_strict_inc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
    attr = true;
  }
  k_strict_inc<<<std::min<unsigned>((unsigned)ctx->n_sms * 2, n1), kBlock, kSmem, st>>>(A);
  HM_LAUNCH_CHECK();
  unsigned long long h[32];
  HM_CUDA(cudaMemcpyAsync(h, cnt.p, sizeof(h), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  if (h[31]) return hm::set_error(HM_ERR_LIMIT, "hm_window_count30: a middle hyperedge has more than %u newest neighbours", kSlots / 2);
  for (int k = 0; k < 30; ++k) out30[k] = h[k];
  return HM_OK;
}
