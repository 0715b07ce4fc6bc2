// Triple counts touching a set of hyperedges, without allocating device memory.
//
// Some callers cannot call cudaMalloc while they run: a serving thread that
// must not block on the allocator or fail mid-request for want of memory, or
// code that has been given a fixed memory reservation and may not take more.
// For them this file offers hm_count_touching30_noalloc, a variant of
// hm_count_touching30 that works on device buffers the caller already owns
// (the ids to mark and the 30 output counts) and keeps all of its scratch in
// one file-scope device array of fixed size, set aside when the library is
// loaded. The graph itself is built beforehand with the ordinary
// (allocating) calls.
//
// Limits and sharing: graphs of at most kNaMaxSlots hyperedge slots whose
// rows are at most kNaRowMax long in the hash table (longer rows use a slower
// binary search), at most kNaMaxIds distinct ids per call. Every call uses the
// same scratch array; each call clears what must start at zero, but two calls
// that overlap on the GPU (different streams, different threads) race on it,
// so callers must serialise them.
#include <mutex>

#include "hm_classes.h"
#include "hm_device.h"
#include "hm_pairs.cuh"

namespace {

constexpr uint32_t kNaMaxSlots = 1u << 21;  // hyperedge slots of the graph
constexpr uint32_t kNaMaxIds = 1u << 20;    // distinct ids per call
constexpr unsigned kNaBlock = 256;
constexpr unsigned kNaWarps = kNaBlock / 32;
constexpr unsigned kNaSlotsHash = 8192;
constexpr unsigned kNaRowMax = kNaSlotsHash / 2;
constexpr uint32_t kNaEmpty = 0xffffffffu;

// Scratch layout (bytes): counters | mark[kNaMaxSlots] | flag[kNaMaxSlots] | ids[kNaMaxIds]
constexpr size_t kNaCounters = 64;  // u64: [0,30) closed, [30,36) open removals, [36,42) open pairs,
                                    // 42 queue, 43 distinct ids, 44 rejected ids
constexpr size_t kNaMarkOff = kNaCounters * sizeof(unsigned long long);
constexpr size_t kNaFlagOff = kNaMarkOff + kNaMaxSlots;
constexpr size_t kNaIdsOff = kNaFlagOff + kNaMaxSlots;
constexpr size_t kNaBytes = kNaIdsOff + (size_t)kNaMaxIds * sizeof(uint32_t);  // 8 MiB + 512 B

static __device__ __align__(256) unsigned char g_na_scratch[kNaBytes];

struct NaPtrs {
  unsigned long long* cnt;
  uint8_t* mark;
  uint8_t* flag;
  uint32_t* ids;
};

__device__ __forceinline__ unsigned na_lane() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint64_t na_gwarp() { return ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ uint64_t na_nwarps() { return ((uint64_t)gridDim.x * blockDim.x) >> 5; }
__device__ __forceinline__ uint64_t na_tid() { return (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint64_t na_stride() { return (uint64_t)gridDim.x * blockDim.x; }

__global__ void k_na_clear(NaPtrs S, uint32_t n_slots) {
  for (uint64_t i = na_tid(); i < n_slots; i += na_stride()) {
    S.mark[i] = 0;
    S.flag[i] = 0;
  }
  for (uint64_t i = na_tid(); i < kNaCounters; i += na_stride()) S.cnt[i] = 0;
}

// Distinct live ids into the scratch list; the others are counted as rejected.
__global__ void k_na_mark(NaPtrs S, const uint32_t* ids, uint32_t n, uint32_t n_slots, const uint32_t* live) {
  for (uint64_t i = na_tid(); i < n; i += na_stride()) {
    const uint32_t id = ids[i];
    if (id >= n_slots || !((live[id >> 5] >> (id & 31)) & 1u)) {
      atomicAdd(&S.cnt[44], 1ull);
      continue;
    }
    // byte-wide test-and-set through the containing word
    unsigned int* word = reinterpret_cast<unsigned int*>(S.mark + (id & ~3u));
    const unsigned int bit = 1u << ((id & 3u) * 8);
    if (!(atomicOr(word, bit) & bit)) {
      const unsigned long long slot = atomicAdd(&S.cnt[43], 1ull);
      S.ids[slot] = id;
    }
  }
}

__global__ void k_na_flag(NaPtrs S, const uint64_t* off, const uint32_t* len, const uint32_t* nbr) {
  const uint32_t n = (uint32_t)S.cnt[43];
  for (uint64_t i = na_gwarp(); i < n; i += na_nwarps()) {
    const uint32_t m = S.ids[i];
    if (na_lane() == 0) S.flag[m] = 1;
    const uint64_t s = off[m];
    for (uint32_t k = na_lane(); k < len[m]; k += 32) S.flag[nbr[s + k]] = 1;
  }
}

__global__ void __launch_bounds__(kNaBlock) k_na_open(NaPtrs S, uint32_t n_slots, const uint64_t* off,
                                                     const uint32_t* len, const uint32_t* nbr, const uint8_t* ovl,
                                                     const uint8_t* esize) {
  __shared__ uint32_t hist[kNaWarps][4][256];
  const unsigned w = threadIdx.x / 32, lane = na_lane();
  uint64_t acc[6] = {0, 0, 0, 0, 0, 0};
  for (uint64_t a = na_gwarp(); a < n_slots; a += na_nwarps()) {
    if (!S.flag[a]) continue;
    const uint32_t l = len[a];
    if (l < 2) continue;
    const uint32_t s = esize[a];
    const bool ma = S.mark[a];
    for (uint32_t k = lane; k <= s; k += 32)
      for (int t = 0; t < 4; ++t) hist[w][t][k] = 0;
    __syncwarp();
    const uint64_t base = off[a];
    for (uint32_t k = lane; k < l; k += 32) {
      const uint32_t b = nbr[base + k];
      const uint32_t c = ovl[base + k];
      const uint32_t y = c < esize[b];
      atomicAdd(&hist[w][y][c], 1u);
      if (!ma && !S.mark[b]) atomicAdd(&hist[w][2 + y][c], 1u);
    }
    __syncwarp();
    if (lane == 0) {
      for (int t = 0; t < 4; ++t)
        for (uint32_t k = 1; k <= s; ++k) hist[w][t][k] += hist[w][t][k - 1];
      hm::open_pair_counts(hist[w][0], hist[w][1], s, acc, false);
      if (!ma) hm::open_pair_counts(hist[w][2], hist[w][3], s, acc, true);
    }
    __syncwarp();
  }
  if (lane == 0)
    for (int k = 0; k < 6; ++k)
      if (acc[k]) atomicAdd(&S.cnt[36 + k], (unsigned long long)acc[k]);
}

struct NaGraph {
  const uint64_t* off;
  const uint32_t* len;
  const uint32_t* nbr;
  const uint8_t* ovl;
  const uint64_t* mask;
  const uint64_t* hoff;
  const uint32_t* hmem;
  const uint8_t* esize;
};

__device__ uint32_t na_triple(const NaGraph& G, uint32_t a, uint32_t b, uint32_t c) {
  const uint32_t* x = G.hmem + G.hoff[a];
  const uint32_t* y = G.hmem + G.hoff[b];
  const uint32_t* z = G.hmem + G.hoff[c];
  const uint32_t nx = G.esize[a], ny = G.esize[b], nz = G.esize[c];
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

// One block per marked m: row(m) in a shared-memory hash, warps over b in
// row(m), lanes over the neighbours c > b of b; a triangle is counted at its
// smallest marked id.
__global__ void __launch_bounds__(kNaBlock, 2) k_na_closed(NaPtrs S, NaGraph G) {
  extern __shared__ unsigned long long na_smem[];
  unsigned long long* smask = na_smem;
  uint32_t* keys = reinterpret_cast<uint32_t*>(smask + kNaSlotsHash);
  uint8_t* sovl = reinterpret_cast<uint8_t*>(keys + kNaSlotsHash);
  __shared__ unsigned long long wc_all[kNaWarps][36];
  __shared__ uint32_t s_item;
  const unsigned w = threadIdx.x / 32, lane = na_lane();
  unsigned long long* wc = wc_all[w];
  for (unsigned k = lane; k < 36; k += 32) wc[k] = 0;
  const uint32_t n = (uint32_t)S.cnt[43];
  for (;;) {
    if (threadIdx.x == 0) s_item = (uint32_t)atomicAdd(&S.cnt[42], 1ull);
    __syncthreads();
    const uint32_t item = s_item;
    if (item >= n) break;
    const uint32_t m = S.ids[item];
    const uint64_t mo = G.off[m];
    const uint32_t md = G.len[m];
    const uint32_t sm = G.esize[m];
    const bool in_smem = md <= kNaRowMax;
    uint32_t shift = 32, hmask = 0;
    if (in_smem) {
      uint32_t slots = 64;
      while (slots < 4 * md && slots < kNaSlotsHash) slots <<= 1;
      shift = 32 - (31 - __clz(slots));
      hmask = slots - 1;
      for (uint32_t i = threadIdx.x; i < slots; i += blockDim.x) keys[i] = kNaEmpty;
      __syncthreads();
      for (uint32_t i = threadIdx.x; i < md; i += blockDim.x) {
        const uint32_t key = G.nbr[mo + i];
        uint32_t h = (key * 2654435761u) >> shift;
        while (atomicCAS(&keys[h], kNaEmpty, key) != kNaEmpty) h = (h + 1) & hmask;
        smask[h] = G.mask[mo + i];
        sovl[h] = G.ovl[mo + i];
      }
    }
    __syncthreads();
    for (uint32_t bi = w; bi < md; bi += kNaWarps) {
      const uint32_t b = G.nbr[mo + bi];
      if (S.mark[b] && b < m) continue;  // counted at b
      const uint32_t cmb = G.ovl[mo + bi];
      const uint64_t mmb = G.mask[mo + bi];
      const uint32_t sb = G.esize[b];
      const uint64_t bo = G.off[b];
      const uint32_t bl = G.len[b];
      uint32_t lo = 0, hi = bl;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (G.nbr[bo + mid] <= b) lo = mid + 1;
        else hi = mid;
      }
      for (uint32_t j = lo + lane; j < bl; j += 32) {
        const uint32_t c = G.nbr[bo + j];
        uint32_t cmc = 0;
        uint64_t mmc = 0;
        if (in_smem) {
          uint32_t h = (c * 2654435761u) >> shift;
          uint32_t k = keys[h];
          while (k != c && k != kNaEmpty) {
            h = (h + 1) & hmask;
            k = keys[h];
          }
          if (k == c) {
            cmc = sovl[h];
            mmc = smask[h];
          }
        } else {
          uint32_t l2 = 0, h2 = md;
          while (l2 < h2) {
            const uint32_t mid = (l2 + h2) >> 1;
            if (G.nbr[mo + mid] < c) l2 = mid + 1;
            else h2 = mid;
          }
          if (l2 < md && G.nbr[mo + l2] == c) {
            cmc = G.ovl[mo + l2];
            mmc = G.mask[mo + l2];
          }
        }
        if (!cmc) continue;
        if (S.mark[c] && c < m) continue;  // counted at c
        const uint32_t cbc = G.ovl[bo + j];
        const uint32_t sc = G.esize[c];
        const uint32_t g = sm <= 64 ? (uint32_t)__popcll(mmb & mmc) : na_triple(G, m, b, c);
        const int k = hm::static_class((int)sm, (int)sb, (int)sc, (int)cmb, (int)cbc, (int)cmc, (int)g);
        if (k < 0) continue;  // cannot happen for a closed triangle; keeps the index in range
        atomicAdd(&wc[k], 1ull);
        atomicAdd(&wc[30 + (cmb + cmc < sm) + 2 * ((cmb < sb) + (cmc < sc))], 1ull);
        atomicAdd(&wc[30 + (cmb + cbc < sb) + 2 * ((cmb < sm) + (cbc < sc))], 1ull);
        atomicAdd(&wc[30 + (cmc + cbc < sc) + 2 * ((cmc < sm) + (cbc < sb))], 1ull);
      }
    }
    __syncthreads();
  }
  __syncwarp();
  for (unsigned k = lane; k < 36; k += 32)
    if (wc[k]) atomicAdd(&S.cnt[k], wc[k]);
}

__global__ void k_na_finish(NaPtrs S, uint64_t* out30) {
  const unsigned k = threadIdx.x;
  if (k < 30) {
    uint64_t v = S.cnt[k];
    if (k >= 20 && k < 26) v += S.cnt[36 + (k - 20)] - S.cnt[30 + (k - 20)];
    out30[k] = v;
  }
}

// Device address of the scratch array, looked up once per device.
std::mutex g_na_mu;
void* g_na_addr[64] = {nullptr};

int na_setup(int device, NaPtrs* S) {
  if (device < 0 || device >= 64) return hm::set_error(HM_ERR_INVALID, "no-alloc count: device %d", device);
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_na_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_na_scratch);
    if (e != cudaSuccess || !p)
      return hm::set_error(HM_ERR_CUDA, "no-alloc count: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    e = cudaFuncSetAttribute(k_na_closed, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)((sizeof(unsigned long long) + sizeof(uint32_t) + 1) * kNaSlotsHash));
    if (e != cudaSuccess)
      return hm::set_error(HM_ERR_CUDA, "no-alloc count: cudaFuncSetAttribute: %s", cudaGetErrorString(e));
    g_na_addr[device] = p;
  }
  unsigned char* base = static_cast<unsigned char*>(g_na_addr[device]);
  S->cnt = reinterpret_cast<unsigned long long*>(base);
  S->mark = base + kNaMarkOff;
  S->flag = base + kNaFlagOff;
  S->ids = reinterpret_cast<uint32_t*>(base + kNaIdsOff);
  return HM_OK;
}

}  // namespace

extern "C" int hm_count_touching30_noalloc(hm_graph* g, const uint32_t* d_ids, uint32_t n, uint64_t* d_out30,
                                           void* stream) {
  if (!g || !d_out30 || (n && !d_ids)) return hm::set_error(HM_ERR_INVALID, "hm_count_touching30_noalloc: NULL argument");
  if (g->temporal) return hm::set_error(HM_ERR_STATE, "hm_count_touching30_noalloc: the graph is temporal");
  if (g->n_slots > kNaMaxSlots)
    return hm::set_error(HM_ERR_LIMIT, "hm_count_touching30_noalloc: %u hyperedge slots exceed the limit of %u",
                         g->n_slots, kNaMaxSlots);
  if (n > kNaMaxIds)
    return hm::set_error(HM_ERR_LIMIT, "hm_count_touching30_noalloc: %u ids exceed the limit of %u", n, kNaMaxIds);
  std::lock_guard<std::mutex> lk(g->ctx->mu);
  HM_CUDA(cudaSetDevice(g->ctx->device));
  NaPtrs S;
  HM_TRY(na_setup(g->ctx->device, &S));
  // NULL is CUDA's legacy default stream (torch's default stream too), so a
  // caller's earlier work on it (the id upload, clearing d_out30) comes first.
  // Work the engine queued on its own stream (an asynchronous static count)
  // is finished before the kernels start.
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (st != g->ctx->stream) HM_CUDA(cudaStreamSynchronize(g->ctx->stream));
  const uint32_t E = g->n_slots;
  const unsigned sms = (unsigned)g->ctx->n_sms;
  k_na_clear<<<sms * 4, kNaBlock, 0, st>>>(S, E);
  HM_LAUNCH_CHECK();
  if (n) {
    k_na_mark<<<hm::grid_for(n, kNaBlock), kNaBlock, 0, st>>>(S, d_ids, n, E, g->live_bits.p);
    HM_LAUNCH_CHECK();
    k_na_flag<<<sms * 8, kNaBlock, 0, st>>>(S, g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p);
    HM_LAUNCH_CHECK();
    k_na_open<<<sms * 8, kNaBlock, 0, st>>>(S, E, g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p, g->h2h_ovl.p,
                                           g->esize.p);
    HM_LAUNCH_CHECK();
    NaGraph G{g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p, g->h2h_ovl.p, g->h2h_mask.p,
              g->h2v_off.p, g->h2v_mem.p, g->esize.p};
    k_na_closed<<<sms * 2, kNaBlock, (sizeof(unsigned long long) + sizeof(uint32_t) + 1) * kNaSlotsHash, st>>>(S, G);
    HM_LAUNCH_CHECK();
  }
  k_na_finish<<<1, 32, 0, st>>>(S, d_out30);
  HM_LAUNCH_CHECK();
  unsigned long long rejected = 0;
  HM_CUDA(cudaMemcpyAsync(&rejected, S.cnt + 44, sizeof(rejected), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  if (rejected)
    return hm::set_error(HM_ERR_NOT_LIVE, "hm_count_touching30_noalloc: %llu ids are not live hyperedges", rejected);
  return HM_OK;
}
