// Counts of the connected triples that touch a set of marked hyperedges (all
// 30 static classes). The exact incremental recount of a batch is this count
// for the inserted ids on the new graph minus it for the deleted ids on the
// old graph.
//
// Same open/closed split as the static count (hm_static.cu), with its
// bucketized hash, unrolled probes and star fast path:
//   * open phase over the centres that are marked or adjacent to a marked
//     hyperedge: pairs {b, c} of the centre's neighbours that contain a marked
//     hyperedge = all pairs (marked centre) or all pairs minus the pairs of
//     unmarked neighbours (unmarked centre), counted from histograms;
//   * closed phase, one block per marked m: row(m) in a shared-memory hash;
//     each warp takes b in row(m), its lanes walk the oriented row N+(b) and
//     probe. A triangle {m, b, c} is counted at its smallest marked id.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "hm_classes.h"
#include "hm_device.h"
#include "hm_pairs.cuh"
#include "hm_triangles.cuh"

namespace hm {
namespace {

constexpr unsigned kWarp = 32;
constexpr unsigned kBlock = 256;
constexpr unsigned kWarps = kBlock / kWarp;
constexpr unsigned kSlots = 16384;        // shared table of one marked row (the longest rows): 192 KB
constexpr unsigned kBigThreads = 1024;    // its block: 32 warps, one block per SM
constexpr unsigned kRowMax = kSlots / 2;  // longer rows use a global table
constexpr unsigned kMidSlots = 4096;      // rows up to mid_row <= kMidRow: 4096-slot tables, 4 blocks per SM
constexpr unsigned kMidRow = kMidSlots / 2;
constexpr unsigned kWarpRow = 128;        // rows up to warp_row <= kWarpRow: one warp each, 256-slot tables
constexpr unsigned kWarpSlots = 256;
constexpr uint32_t kEmpty = 0xffffffffu;
constexpr unsigned kUnroll = 4;

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint64_t global_warp() { return ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ uint64_t n_warps() { return ((uint64_t)gridDim.x * blockDim.x) >> 5; }
__device__ __forceinline__ uint64_t gtid() { return (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint64_t gstride() { return (uint64_t)gridDim.x * blockDim.x; }

__global__ void k_mark(const uint32_t* ids, uint32_t n, uint8_t* mark) {
  for (uint64_t i = gtid(); i < n; i += gstride()) mark[ids[i]] = 1;
}

// flag = marked or adjacent to a marked hyperedge
__global__ void k_flag_touched(const uint32_t* ids, uint32_t n, const uint64_t* off, const uint32_t* len,
                               const uint32_t* nbr, uint32_t* flag) {
  for (uint64_t i = global_warp(); i < n; i += n_warps()) {
    const uint32_t m = ids[i];
    if (lane_id() == 0) flag[m] = 1;
    const uint64_t s = off[m];
    for (uint32_t k = lane_id(); k < len[m]; k += kWarp) flag[nbr[s + k]] = 1;
  }
}

__global__ void k_list_flagged(const uint32_t* flag, const uint64_t* pos, uint32_t n, uint32_t* out) {
  for (uint64_t i = gtid(); i < n; i += gstride())
    if (flag[i]) out[pos[i]] = (uint32_t)i;
}

// Counter block of one output row: 30 closed classes, 6 open-pair classes
// removed by closed triangles, 6 open-pair counts.
constexpr unsigned kRowStride = 42;

__global__ void __launch_bounds__(kBlock) k_touch_open(const uint32_t* centres, uint32_t n, const uint8_t* mark,
                                                       const uint64_t* off, const uint32_t* len, const uint32_t* nbr,
                                                       const uint8_t* ovl, const uint8_t* esize,
                                                       const uint32_t* gos, const uint32_t* rog,
                                                       unsigned long long* out) {
  __shared__ uint32_t hist[kWarps][4][256];  // all: type 0/1; unmarked: type 0/1
  const unsigned w = threadIdx.x / kWarp, lane = lane_id();
  uint64_t acc[6] = {0, 0, 0, 0, 0, 0};
  for (uint64_t i = global_warp(); i < n; i += n_warps()) {
    const uint32_t a = centres[i];
    const uint32_t l = len[a];
    if (l < 2) continue;
    const uint32_t s = esize[a];
    const bool ma = mark[a];
    for (uint32_t k = lane; k <= s; k += kWarp)
      for (int t = 0; t < 4; ++t) hist[w][t][k] = 0;
    __syncwarp();
    const uint64_t base = off[a];
    uint32_t one[4] = {0, 0, 0, 0};  // overlap-1 neighbours, the common case, counted in registers
    for (uint32_t k = lane; k < l; k += kWarp) {
      const uint32_t b = nbr[base + k];
      const uint32_t c = ovl[base + k];
      const uint32_t y = c < esize[b];
      const bool um = !ma && !mark[b];
      if (c == 1) {
        one[y] += 1;
        if (um) one[2 + y] += 1;
      } else {
        atomicAdd(&hist[w][y][c], 1u);
        if (um) atomicAdd(&hist[w][2 + y][c], 1u);
      }
    }
    for (int t = 0; t < 4; ++t)
      for (int d = 16; d; d >>= 1) one[t] += __shfl_xor_sync(0xffffffffu, one[t], d);
    __syncwarp();
    if (lane == 0) {
      for (int t = 0; t < 4; ++t) hist[w][t][1] += one[t];
      for (int t = 0; t < 4; ++t)
        for (uint32_t k = 1; k <= s; ++k) hist[w][t][k] += hist[w][t][k - 1];
      open_pair_counts(hist[w][0], hist[w][1], s, acc, false);
      if (!ma) open_pair_counts(hist[w][2], hist[w][3], s, acc, true);
      if (gos) {  // per-request rows: each centre's pairs go to its graph's row
        unsigned long long* o = out + (size_t)rog[gos[a]] * kRowStride + 36;
        for (int k = 0; k < 6; ++k)
          if (acc[k]) {
            atomicAdd(&o[k], (unsigned long long)acc[k]);
            acc[k] = 0;
          }
      }
    }
    __syncwarp();
  }
  if (lane == 0)
    for (int k = 0; k < 6; ++k)
      if (acc[k]) atomicAdd(&out[36 + k], (unsigned long long)acc[k]);
}

__device__ uint32_t triple_overlap3(const uint64_t* hoff, const uint32_t* hmem, const uint8_t* esize, uint32_t a,
                                    uint32_t b, uint32_t c) {
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

struct TouchArgs {
  const uint32_t* ids;      // items [0, n_long): slices of rows in global tables
  uint32_t n_long;
  const uint32_t* short_ids;  // items [n_long, n): whole rows, heaviest first
  uint32_t n;
  const uint8_t* mark;
  const uint64_t* off;
  const uint32_t* len;
  const uint32_t* nbr;
  const uint8_t* ovl;
  const uint64_t* mask;
  const uint64_t* hoff;
  const uint32_t* hmem;
  const uint8_t* esize;
  const uint64_t* poff;     // oriented rows: neighbours of higher (degree, id) rank
  const uint32_t* plen;
  const uint32_t* pnbr;
  const uint16_t* pos;      // (neighbour size << 8) | overlap
  const uint64_t* goff;     // per item: offset of its global table (rows longer than kRowMax)
  const uint32_t* gslots;   // per item: slots of that table, 0 for a shared-memory row
  const uint32_t* brange;   // per item: [brange[2i], brange[2i+1]) of row(m) to take b from
  const uint4* gtab;        // global tables: {key, overlap, mask low, mask high}
  const uint32_t* gos;      // per slot: its graph (null: one output row)
  const uint32_t* rog;      // per graph: output row
  bool by_id;               // walk the id-ordered suffix of row(b) instead of N+(b)
  unsigned int* queue;
  unsigned long long* out;  // rows of kRowStride counters
};

// First index of row[0, n) whose value is >= key (or > key with upper),
// found by the whole warp: 32 probes per round.
template <bool upper>
__device__ __forceinline__ uint32_t warp_bound(const uint32_t* row, uint32_t n, uint32_t key) {
  const unsigned lane = threadIdx.x & 31u;
  uint32_t lo = 0, hi = n;
  while (hi - lo > 32) {
    const uint32_t step = (hi - lo + 31) / 32;
    const uint32_t p = lo + (lane + 1) * step - 1;
    bool before = false;
    if (p < hi) {
      const uint32_t v = __ldg(row + p);
      before = upper ? v <= key : v < key;
    }
    const uint32_t k = (uint32_t)__popc(__ballot_sync(0xffffffffu, before));
    lo += k * step;
    hi = min(hi, lo + step);
  }
  bool before = false;
  if (lo + lane < hi) {
    const uint32_t v = __ldg(row + lo + lane);
    before = upper ? v <= key : v < key;
  }
  return lo + (uint32_t)__popc(__ballot_sync(0xffffffffu, before));
}

__device__ __forceinline__ uint32_t size_cat(uint32_t s) { return s >= 3 ? 2u : s - 1u; }

// Adds n triangles {m, b, c} whose three pairs share one node, the same one,
// with size categories cm, cb, cc: closed class = number of members with
// |x| >= 2; open-pair classes at each centre x: [|x| >= 3] + 2 ([|y| >= 2] +
// [|z| >= 2]).
__device__ __forceinline__ void add_star(unsigned long long* wc, uint32_t cm, uint32_t cb, uint32_t cc, uint64_t n) {
  const uint32_t em = cm > 0, eb = cb > 0, ec = cc > 0;
  atomicAdd(&wc[em + eb + ec], (unsigned long long)n);
  atomicAdd(&wc[30 + (cm == 2) + 2 * (eb + ec)], (unsigned long long)n);
  atomicAdd(&wc[30 + (cb == 2) + 2 * (em + ec)], (unsigned long long)n);
  atomicAdd(&wc[30 + (cc == 2) + 2 * (em + eb)], (unsigned long long)n);
}

__device__ __forceinline__ uint32_t hmix(uint32_t key) { return key * 2654435761u; }

// Global-memory tables of the marked rows too long for shared memory: one
// 16-byte entry per key {key, overlap, mask low, mask high}, key all ones
// when empty, so a probe answers with one load.
__global__ void k_build_ghash(const uint32_t* ids, uint32_t n, const uint64_t* goff, const uint32_t* gslots,
                              const uint32_t* brange, const uint64_t* off, const uint32_t* len, const uint32_t* nbr,
                              const uint8_t* ovl, const uint64_t* mask, uint4* tab) {
  for (uint64_t i = global_warp(); i < n; i += n_warps()) {
    const uint32_t slots = gslots[i];
    if (!slots || brange[2 * i] != 0) continue;  // one build per row: its first slice
    const uint32_t m = ids[i];
    uint4* t = tab + goff[i];
    const uint64_t mo = off[m];
    for (uint32_t k = lane_id(); k < len[m]; k += kWarp) {
      const uint32_t key = nbr[mo + k];
      uint32_t h = hmix(key) & (slots - 1);
      while (atomicCAS(&t[h].x, kEmpty, key) != kEmpty) h = (h + 1) & (slots - 1);
      const uint64_t mk = mask[mo + k];
      t[h].y = ovl[mo + k];
      t[h].z = (uint32_t)mk;
      t[h].w = (uint32_t)(mk >> 32);
    }
  }
}

// The table of one marked row: bucketized shared keys (4 per 16-byte bucket)
// with each key's index in the row, or a global table for the longest rows.
// One value per key: m's shared-position mask with it when |m| <= 64 (the
// overlap is its popcount), else the overlap.
struct MarkTable {
  const uint32_t* keys;
  const uint64_t* sval;
  uint32_t shift, bmask;
  uint32_t gslots;  // > 0: global table gt of gslots entries
  const uint4* gt;
};

__device__ __forceinline__ void fill_mark_table(const TouchArgs& A, uint64_t mo, uint32_t md, bool exact,
                                                uint32_t* keys, uint64_t* sval, uint32_t shift, uint32_t bmask,
                                                unsigned first, unsigned stride) {
  for (uint32_t i = first; i < md; i += stride) {
    const uint32_t key = A.nbr[mo + i];
    uint32_t bk = hmix(key) >> shift, h = 0;
    for (bool done = false; !done; bk = (bk + 1) & bmask)
      for (uint32_t t = 0; t < 4; ++t)
        if (atomicCAS(&keys[4 * bk + t], kEmpty, key) == kEmpty) {
          h = 4 * bk + t;
          done = true;
          break;
        }
    sval[h] = exact ? A.mask[mo + i] : (uint64_t)A.ovl[mo + i];
  }
}

// One whole warp: the bi-th neighbour b of the marked m. Lanes walk the
// neighbours c of b ranked above it, N+(b) by (degree, id) or the part of b's
// id-sorted row after b, so each pair {b, c} of m's neighbours is met once,
// from its lower-ranked end, with four probes in flight. A triangle {m, b, c}
// is counted at its smallest marked id. g comes from the position masks of m
// (|m| <= 64) or of b (|b| <= 64), else from a merge. Star triangles (all
// overlaps 1, one shared node) are counted per size category in registers.
// Triangles that are not stars go to the warp's queue q (qn records,
// warp-uniform), classified 32 at a time.
__device__ __forceinline__ void touch_pairs_of_b(const TouchArgs& A, uint32_t m, uint64_t mo, uint32_t sm,
                                                 uint32_t cat_m, uint32_t bi, const MarkTable& T,
                                                 unsigned long long* wc, uint64_t* q, uint32_t& qn) {
  const unsigned lane = lane_id();
  const uint32_t b = A.nbr[mo + bi];
  if (A.mark[b] && b < m) return;  // counted at b (warp-uniform)
  const uint32_t cmb = A.ovl[mo + bi];
  const uint32_t sb = A.esize[b];
  uint64_t bo;
  uint32_t bl;
  if (A.by_id) {
    const uint32_t split = warp_bound<true>(A.nbr + A.off[b], A.len[b], b);
    bo = A.off[b] + split;
    bl = A.len[b] - split;
  } else {
    bo = A.poff[b];
    bl = A.plen[b];
  }
  const uint32_t* cnbr = A.by_id ? A.nbr : A.pnbr;
  // masks: relative to m when |m| <= 64, else relative to b when |b| <= 64
  const bool piv_m = sm <= 64, piv_b = !piv_m && sb <= 64;
  uint64_t pmb = piv_m ? A.mask[mo + bi] : 0;
  if (piv_b) {  // b's entry for m, from b's full row
    const uint64_t fo = A.off[b];
    pmb = A.mask[fo + warp_bound<false>(A.nbr + fo, A.len[b], m)];
  }
  const bool star_ok = cmb == 1 && (piv_m || piv_b);
  uint32_t star0 = 0, star1 = 0, star2 = 0;
  // The next round's loads are issued before this round's probes (software
  // pipelining); by id, a neighbour's size is gathered when it is probed.
  uint32_t cv[kUnroll], ov[kUnroll];
#pragma unroll
  for (unsigned u = 0; u < kUnroll; ++u) {
    const uint32_t j = u * kWarp + lane;
    cv[u] = kEmpty;
    ov[u] = 0;
    if (j < bl) {
      cv[u] = __ldg(cnbr + bo + j);
      ov[u] = A.by_id ? __ldg(A.ovl + bo + j) : __ldg(A.pos + bo + j);
    }
  }
  for (uint32_t j0 = 0; j0 < bl; j0 += kWarp * kUnroll) {
    uint32_t cn[kUnroll], on[kUnroll];
#pragma unroll
    for (unsigned u = 0; u < kUnroll; ++u) {
      const uint32_t j = j0 + kWarp * kUnroll + u * kWarp + lane;
      cn[u] = kEmpty;
      on[u] = 0;
      if (j < bl) {
        cn[u] = __ldg(cnbr + bo + j);
        on[u] = A.by_id ? __ldg(A.ovl + bo + j) : __ldg(A.pos + bo + j);
      }
    }
#pragma unroll
    for (unsigned u = 0; u < kUnroll; ++u) {
      const uint32_t c = cv[u];
      if (A.by_id && c != kEmpty) ov[u] |= (uint32_t)__ldg(A.esize + c) << 8;
      bool push = false;
      uint64_t rec = 0;
      do {
      if (c == kEmpty) break;
      uint32_t cmc = 0;  // overlap of c with m (0: not a neighbour of m)
      uint64_t mmc = 0;  // m's shared positions with c
      if (!T.gslots) {
        uint32_t bk = hmix(c) >> T.shift;
        int t;
        for (;;) {
          const uint4 q = reinterpret_cast<const uint4*>(T.keys)[bk];
          t = q.x == c ? 0 : q.y == c ? 1 : q.z == c ? 2 : q.w == c ? 3 : -1;
          if (t >= 0 || q.w == kEmpty) break;
          bk = (bk + 1) & T.bmask;
        }
        if (t >= 0) {
          const uint64_t v = T.sval[4 * bk + t];
          if (piv_m) {  // |m| <= 64: the mask is exact
            mmc = v;
            cmc = (uint32_t)__popcll(v);
          } else {
            cmc = (uint32_t)v;
          }
        }
      } else {
        uint32_t h = hmix(c) & (T.gslots - 1);
        for (;;) {
          const uint4 e = T.gt[h];
          if (e.x == kEmpty) break;
          if (e.x == c) {
            cmc = e.y;
            mmc = ((uint64_t)e.w << 32) | e.z;
            break;
          }
          h = (h + 1) & (T.gslots - 1);
        }
      }
      if (!cmc) break;
      if (A.mark[c] && c < m) break;  // counted at c
      const uint32_t cbc = ov[u] & 0xffu, sc = ov[u] >> 8;
      uint32_t g;
      if (piv_m || piv_b) {
        const uint64_t jc = bo + j0 + u * kWarp + lane;
        const uint64_t pmc = piv_m ? mmc : A.by_id ? A.mask[jc] : row_mask(A.off, A.len, A.nbr, A.mask, b, c);
        if ((cmb | cmc | cbc) == 1 && pmb == pmc) {
          const uint32_t cc = size_cat(sc);
          star0 += cc == 0;
          star1 += cc == 1;
          star2 += cc == 2;
          break;
        }
        g = (uint32_t)__popcll(pmb & pmc);
      } else {
        g = triple_overlap3(A.hoff, A.hmem, A.esize, m, b, c);
      }
      push = true;
      rec = pack_triangle(sb, sc, cmb, cbc, cmc, g);
      } while (false);
      // warp-converged: queue this slice's triangles (64 places)
      const unsigned bal = __ballot_sync(0xffffffffu, push);
      if (push) q[qn + __popc(bal & ((1u << lane) - 1u))] = rec;
      qn += (uint32_t)__popc(bal);
      if (qn >= kWarp) {
        __syncwarp();
        classify_queue(q, kWarp, sm, wc);
        if (lane < qn - kWarp) q[lane] = q[kWarp + lane];
        __syncwarp();
        qn -= kWarp;
      }
    }
#pragma unroll
    for (unsigned u = 0; u < kUnroll; ++u) {
      cv[u] = cn[u];
      ov[u] = on[u];
    }
  }
  if (star_ok) {
    for (int d = 16; d; d >>= 1) {
      star0 += __shfl_xor_sync(0xffffffffu, star0, d);
      star1 += __shfl_xor_sync(0xffffffffu, star1, d);
      star2 += __shfl_xor_sync(0xffffffffu, star2, d);
    }
    if (lane == 0) {
      const uint32_t cat_b = size_cat(sb);
      if (star0) add_star(wc, cat_m, cat_b, 0, star0);
      if (star1) add_star(wc, cat_m, cat_b, 1, star1);
      if (star2) add_star(wc, cat_m, cat_b, 2, star2);
    }
  }
}

constexpr uint32_t kNoRow = 0xffffffffu;

__device__ __forceinline__ void flush_touch(unsigned long long* wc, unsigned long long* out) {
  for (unsigned k = lane_id(); k < 36; k += kWarp)
    if (wc[k]) {
      atomicAdd(&out[k], wc[k]);
      wc[k] = 0;
    }
  __syncwarp();
}

// Output row of marked m (per-request rows of a pooled store).
__device__ __forceinline__ uint32_t row_of(const TouchArgs& A, uint32_t m) {
  return A.gos ? A.rog[A.gos[m]] : 0u;
}

// Shared-memory bytes of a table of `slots` entries: masks, keys, overlaps.
constexpr size_t touch_smem(unsigned slots) { return (sizeof(uint64_t) + sizeof(uint32_t)) * slots; }

// One block per marked m, heaviest rows first: row(m) in a shared table of
// up to kTab slots (load <= 1/2) with one value per key (mask or overlap) or, for
// rows longer than kRowMax, in a global table, split into slices of
// neighbours (items [0, n_long)); warps take b in row(m).
template <unsigned kTab, unsigned kThreads, unsigned kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_touch_closed(TouchArgs A) {
  constexpr unsigned kW = kThreads / kWarp;
  extern __shared__ uint64_t smem64[];
  uint64_t* sval = smem64;                                           // kTab
  uint32_t* keys = reinterpret_cast<uint32_t*>(sval + kTab);         // kTab
  __shared__ unsigned long long wcnt[kW][36];
  __shared__ uint64_t wqueue[kW][2 * kWarp];  // per warp: triangles waiting to be classified
  __shared__ uint32_t s_item;
  const unsigned w = threadIdx.x / kWarp, lane = lane_id();
  unsigned long long* wc = wcnt[w];
  uint64_t* q = wqueue[w];
  uint32_t qn = 0;
  for (unsigned k = lane; k < 36; k += kWarp) wc[k] = 0;
  uint32_t cur_row = kNoRow;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(A.queue, 1u);
    __syncthreads();
    const uint32_t item = s_item;
    if (item >= A.n) break;
    const bool long_row = item < A.n_long;
    const uint32_t m = long_row ? A.ids[item] : A.short_ids[item - A.n_long];
    const uint32_t row = row_of(A, m);
    if (row != cur_row) {
      if (cur_row != kNoRow) flush_touch(wc, A.out + (size_t)cur_row * kRowStride);
      cur_row = row;
    }
    const uint64_t mo = A.off[m];
    const uint32_t md = A.len[m];
    const uint32_t sm = A.esize[m];
    MarkTable T{keys, sval, 32, 0, long_row ? A.gslots[item] : 0u, A.gtab + (long_row ? A.goff[item] : 0ull)};
    if (!T.gslots) {
      uint32_t slots = 64;
      while (slots < 2 * md && slots < kTab) slots <<= 1;
      const uint32_t buckets = slots / 4;
      T.shift = 32 - (31 - __clz(buckets));
      T.bmask = buckets - 1;
      for (uint32_t i = threadIdx.x; i < slots; i += blockDim.x) keys[i] = kEmpty;
      __syncthreads();
      fill_mark_table(A, mo, md, sm <= 64, keys, sval, T.shift, T.bmask, threadIdx.x, blockDim.x);
    }
    __syncthreads();
    const uint32_t cat_m = size_cat(sm);
    const uint32_t b_begin = long_row ? A.brange[2 * item] : 0u;
    const uint32_t b_end = long_row ? A.brange[2 * item + 1] : md;
    for (uint32_t bi = b_begin + w; bi < b_end; bi += kW) {
      touch_pairs_of_b(A, m, mo, sm, cat_m, bi, T, wc, q, qn);
      __syncwarp();
    }
    if (qn) {  // this item's last triangles (classes depend on |m|)
      classify_queue(q, qn, sm, wc);
      qn = 0;
    }
    __syncthreads();
  }
  __syncwarp();
  flush_touch(wc, A.out + (cur_row == kNoRow ? 0 : (size_t)cur_row * kRowStride));
}

// One warp per marked m with a short row (<= kWarpRow): a 256-slot table of
// its own, no block-wide barriers.
__global__ void __launch_bounds__(kBlock, 4) k_touch_warp(TouchArgs A) {
  __shared__ __align__(16) uint32_t keys_all[kWarps][kWarpSlots];
  __shared__ uint64_t val_all[kWarps][kWarpSlots];
  __shared__ unsigned long long wcnt[kWarps][36];
  __shared__ uint64_t wqueue[kWarps][2 * kWarp];
  const unsigned w = threadIdx.x / kWarp, lane = lane_id();
  uint32_t* keys = keys_all[w];
  uint64_t* sval = val_all[w];
  unsigned long long* wc = wcnt[w];
  uint64_t* q = wqueue[w];
  uint32_t qn = 0;
  for (unsigned k = lane; k < 36; k += kWarp) wc[k] = 0;
  __syncwarp();
  uint32_t cur_row = kNoRow;
  for (;;) {
    uint32_t it = 0;
    if (lane == 0) it = atomicAdd(A.queue, 1u);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= A.n) break;
    const uint32_t m = A.short_ids[it];
    const uint32_t row = row_of(A, m);
    if (row != cur_row) {
      if (cur_row != kNoRow) flush_touch(wc, A.out + (size_t)cur_row * kRowStride);
      cur_row = row;
    }
    const uint64_t mo = A.off[m];
    const uint32_t md = A.len[m];  // <= warp_row <= kWarpRow by the split
    const uint32_t sm = A.esize[m];
    uint32_t slots = 64;
    while (slots < 2 * md && slots < kWarpSlots) slots <<= 1;
    const uint32_t buckets = slots / 4;
    MarkTable T{keys, sval, 32u - (31u - (uint32_t)__clz(buckets)), buckets - 1, 0u, A.gtab};
    for (uint32_t i = lane; i < slots; i += kWarp) keys[i] = kEmpty;
    __syncwarp();
    fill_mark_table(A, mo, md, sm <= 64, keys, sval, T.shift, T.bmask, lane, kWarp);
    __syncwarp();
    const uint32_t cat_m = size_cat(sm);
    for (uint32_t bi = 0; bi < md; ++bi) {
      touch_pairs_of_b(A, m, mo, sm, cat_m, bi, T, wc, q, qn);
      __syncwarp();
    }
    if (qn) {
      classify_queue(q, qn, sm, wc);
      qn = 0;
    }
  }
  __syncwarp();
  flush_touch(wc, A.out + (cur_row == kNoRow ? 0 : (size_t)cur_row * kRowStride));
}

// Sort key of a marked row: [long row: global table] [length class, 2 bits:
// 2 = longer than the schedule's mid_row, 1 = longer than its warp_row; the
// long rows are class 2 too, as mid_row <= kMidRow] [output row of its graph
// when gos is set, 29 bits] [row length, 32 bits]. Descending order gives the
// three launches' lists (long and large rows, medium rows, short rows), each
// keeping one graph's rows together and heaviest first, so that the blocks
// running at one time share one graph's rows in L2.
__global__ void k_touch_keys(const uint32_t* ids, uint32_t n, const uint32_t* len, const uint32_t* gos,
                             const uint32_t* rog, TouchSchedule ts, uint64_t* key) {
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    const uint32_t m = ids[i], l = len[m];
    uint64_t k = l;
    if (gos) k |= (uint64_t)min(rog[gos[m]], 0x1fffffffu) << 32;
    k |= (uint64_t)(l > ts.mid_row ? 2u : l > ts.warp_row ? 1u : 0u) << 61;
    if (l > kRowMax) k |= 1ull << 63;
    key[i] = k;
  }
}

// counts[0] long rows, [1] class-2 rows (long ones included), [2] class-1 rows
__global__ void k_count_classes(const uint64_t* key, uint32_t n, unsigned int* counts) {
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    const uint64_t k = key[i];
    if (k >> 63) atomicAdd(&counts[0], 1u);
    const uint32_t cls = (uint32_t)(k >> 61) & 3u;
    if (cls == 2) atomicAdd(&counts[1], 1u);
    if (cls == 1) atomicAdd(&counts[2], 1u);
  }
}



}  // namespace

int count_touching_rows(hm_graph* g, const uint32_t* d_ids, uint32_t n, const TouchRows& rows, uint64_t* out) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  const uint32_t R = rows.gos ? rows.n_rows : 1u;
  for (size_t k = 0; k < (size_t)R * 30; ++k) out[k] = 0;
  if (!n) return HM_OK;
  const uint32_t E = g->n_slots;
  bool by_id = g->touch_by_id;
  const size_t n_cnt = (size_t)R * kRowStride + 5;  // + three queues, + class counts (u32 pairs)
  DArr<uint8_t> mark;
  DArr<uint32_t> flag, centres;
  DArr<uint64_t> pos;
  DArr<unsigned long long> cnt;
  HM_TRY(mark.alloc(ctx, E));
  HM_TRY(flag.alloc(ctx, E));
  HM_TRY(pos.alloc(ctx, (size_t)E + 1));
  HM_TRY(cnt.alloc(ctx, n_cnt));
  unsigned int* queues = reinterpret_cast<unsigned int*>(cnt.p + (size_t)R * kRowStride);  // 3 used
  unsigned int* classes_d = reinterpret_cast<unsigned int*>(cnt.p + (size_t)R * kRowStride + 2);  // 3 used
  HM_CUDA(cudaMemsetAsync(mark.p, 0, E, st));
  HM_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(uint32_t) * E, st));
  HM_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long) * n_cnt, st));
  k_mark<<<grid_for(n, kBlock), kBlock, 0, st>>>(d_ids, n, mark.p);
  HM_LAUNCH_CHECK();
  k_flag_touched<<<grid_for((uint64_t)n * 32, kBlock), kBlock, 0, st>>>(d_ids, n, g->h2h_off.p, g->h2h_len.p,
                                                                       g->h2h_nbr.p, flag.p);
  HM_LAUNCH_CHECK();
  HM_TRY(exclusive_scan(ctx, flag.p, pos.p, E));
  // marked rows, heaviest first (device sort); rows longer than kRowMax come
  // first and get global tables
  DArr<uint64_t> keys, skeys;
  DArr<uint32_t> sids;
  HM_TRY(keys.alloc(ctx, n));
  HM_TRY(skeys.alloc(ctx, n));
  HM_TRY(sids.alloc(ctx, n));
  k_touch_keys<<<grid_for(n, kBlock), kBlock, 0, st>>>(d_ids, n, g->h2h_len.p, rows.gos, rows.rog, g->tsched,
                                                       keys.p);
  HM_LAUNCH_CHECK();
  {
    size_t tb = 0;
    HM_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, keys.p, skeys.p, d_ids, sids.p, (int64_t)n, 0, 64,
                                                      st));
    DArr<uint8_t> tmp;
    HM_TRY(tmp.alloc(ctx, tb));
    HM_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.p, tb, keys.p, skeys.p, d_ids, sids.p, (int64_t)n, 0, 64,
                                                      st));
  }
  k_count_classes<<<grid_for(n, kBlock), kBlock, 0, st>>>(skeys.p, n, classes_d);
  HM_LAUNCH_CHECK();
  uint64_t nc = 0;
  unsigned int hcls[3] = {0, 0, 0};
  HM_CUDA(cudaMemcpyAsync(&nc, pos.p + E, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaMemcpyAsync(hcls, classes_d, sizeof(hcls), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  const uint32_t n_long = hcls[0], n_large = hcls[1], n_mid = hcls[2];
  HM_TRY(centres.alloc(ctx, nc));
  k_list_flagged<<<grid_for(E, kBlock), kBlock, 0, st>>>(flag.p, pos.p, E, centres.p);
  HM_LAUNCH_CHECK();
  const bool trace = std::getenv("HM_TRACE") != nullptr;
  auto t_open0 = std::chrono::steady_clock::now();
  k_touch_open<<<grid_for(nc * 32, kBlock), kBlock, 0, st>>>(centres.p, (uint32_t)nc, mark.p, g->h2h_off.p,
                                                             g->h2h_len.p, g->h2h_nbr.p, g->h2h_ovl.p, g->esize.p,
                                                             rows.gos, rows.rog, cnt.p);
  HM_LAUNCH_CHECK();
  static bool attr = false;
  if (!attr) {
    HM_CUDA(cudaFuncSetAttribute(k_touch_closed<kSlots, kBigThreads, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)touch_smem(kSlots)));
    HM_CUDA(cudaFuncSetAttribute(k_touch_closed<kMidSlots, kBlock, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)touch_smem(kMidSlots)));
    attr = true;
  }
  // long rows: split into slices of kSlice neighbours b, one item each, all
  // slices of a row sharing its global table
  constexpr uint32_t kSlice = 256;
  std::vector<uint32_t> oid, oslots, orange;
  std::vector<uint64_t> ooff;
  uint64_t gtotal = 0;
  if (n_long) {
    std::vector<uint32_t> hid(n_long), hlen(n_long);
    std::vector<uint64_t> hkey(n_long);
    HM_CUDA(cudaMemcpyAsync(hid.data(), sids.p, sizeof(uint32_t) * n_long, cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaMemcpyAsync(hkey.data(), skeys.p, sizeof(uint64_t) * n_long, cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    for (uint32_t i = 0; i < n_long; ++i) hlen[i] = (uint32_t)hkey[i];
    for (uint32_t i = 0; i < n_long; ++i) {
      uint32_t sl = 1;
      while (sl < 2 * hlen[i]) sl <<= 1;
      for (uint32_t b0 = 0; b0 < hlen[i]; b0 += kSlice) {
        oid.push_back(hid[i]);
        oslots.push_back(sl);
        ooff.push_back(gtotal);
        orange.push_back(b0);
        orange.push_back(std::min(hlen[i], b0 + kSlice));
      }
      gtotal += sl;
    }
  }
  const uint32_t n_items_long = (uint32_t)oid.size();
  const uint32_t n_items = n_items_long + (n_large - n_long);  // the large-table launch
  DArr<uint32_t> d_oid, d_oslots, d_orange;
  DArr<uint64_t> d_ooff;
  DArr<uint4> gtab;
  HM_TRY(d_oid.alloc(ctx, n_items_long));
  HM_TRY(d_oslots.alloc(ctx, n_items_long));
  HM_TRY(d_orange.alloc(ctx, 2 * (size_t)n_items_long));
  HM_TRY(d_ooff.alloc(ctx, n_items_long));
  HM_TRY(gtab.alloc(ctx, gtotal ? gtotal : 1));
  if (n_items_long) {
    HM_CUDA(cudaMemcpyAsync(d_oid.p, oid.data(), sizeof(uint32_t) * n_items_long, cudaMemcpyHostToDevice, st));
    HM_CUDA(cudaMemcpyAsync(d_oslots.p, oslots.data(), sizeof(uint32_t) * n_items_long, cudaMemcpyHostToDevice, st));
    HM_CUDA(cudaMemcpyAsync(d_orange.p, orange.data(), sizeof(uint32_t) * 2 * n_items_long, cudaMemcpyHostToDevice,
                            st));
    HM_CUDA(cudaMemcpyAsync(d_ooff.p, ooff.data(), sizeof(uint64_t) * n_items_long, cudaMemcpyHostToDevice, st));
    HM_CUDA(cudaMemsetAsync(gtab.p, 0xff, sizeof(uint4) * gtotal, st));
    k_build_ghash<<<grid_for((uint64_t)n_items_long * 32, kBlock), kBlock, 0, st>>>(
        d_oid.p, n_items_long, d_ooff.p, d_oslots.p, d_orange.p, g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p,
        g->h2h_ovl.p, g->h2h_mask.p, gtab.p);
    HM_LAUNCH_CHECK();
    // the host copies above read pageable vectors: finish them before they go
    HM_CUDA(cudaStreamSynchronize(st));
  }
  if (!by_id && !g->plus_valid) {
    // The oriented copy does not always fit beside a store that batches have
    // grown: then this count walks the id-ordered row suffixes instead (the
    // same triangles, met from their lower id rather than their lower rank).
    const int s = build_plus(g);
    if (s == HM_ERR_NOMEM) {
      release_plus(g);
      by_id = true;
    } else {
      HM_TRY(s);
    }
  }
  TouchArgs A{d_oid.p, n_items_long, sids.p + n_long, n_items, mark.p, g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p,
              g->h2h_ovl.p, g->h2h_mask.p, g->h2v_off.p, g->h2v_mem.p, g->esize.p, g->plus_off.p, g->plus_len.p,
              g->plus_nbr.p, g->plus_os.p, d_ooff.p, d_oslots.p, d_orange.p, gtab.p,
              rows.gos, rows.rog, by_id, queues, cnt.p};
  if (trace) cudaStreamSynchronize(st);
  auto t_cl0 = std::chrono::steady_clock::now();
  const unsigned sms = (unsigned)ctx->n_sms;
  cudaEvent_t tev[4] = {nullptr, nullptr, nullptr, nullptr};
  if (trace)
    for (auto& e : tev) cudaEventCreate(&e);
  if (trace) cudaEventRecord(tev[0], st);
  if (n_items) {  // long rows (global tables, sliced) and rows longer than mid_row
    k_touch_closed<kSlots, kBigThreads, 1><<<std::min<unsigned>(sms, n_items), kBigThreads, touch_smem(kSlots), st>>>(A);
    HM_LAUNCH_CHECK();
  }
  if (trace) cudaEventRecord(tev[1], st);
  if (n_mid) {  // rows of warp_row + 1 .. mid_row
    TouchArgs B = A;
    B.n_long = 0;
    B.short_ids = sids.p + n_large;
    B.n = n_mid;
    B.queue = queues + 1;
    k_touch_closed<kMidSlots, kBlock, 4><<<std::min<unsigned>(sms * 4, n_mid), kBlock, touch_smem(kMidSlots), st>>>(B);
    HM_LAUNCH_CHECK();
  }
  if (trace) cudaEventRecord(tev[2], st);
  const uint32_t n_short = n - n_large - n_mid;
  if (n_short) {  // rows of at most warp_row, one warp each
    TouchArgs C = A;
    C.n_long = 0;
    C.short_ids = sids.p + n_large + n_mid;
    C.n = n_short;
    C.queue = queues + 2;
    k_touch_warp<<<std::min<unsigned>(sms * 4, (n_short + kWarps - 1) / kWarps), kBlock, 0, st>>>(C);
    HM_LAUNCH_CHECK();
  }
  if (trace) {
    cudaEventRecord(tev[3], st);
    cudaStreamSynchronize(st);
    const auto t_end = std::chrono::steady_clock::now();
    float ms[3] = {0, 0, 0};
    for (int k = 0; k < 3; ++k) cudaEventElapsedTime(&ms[k], tev[k], tev[k + 1]);
    for (auto& e : tev) cudaEventDestroy(e);
    std::fprintf(stderr,
                 "[hm_trace touching] marked=%u centres=%llu long=%u large=%u mid=%u short=%u by_id=%d open=%.1fms "
                 "closed=%.1fms (large %.1f mid %.1f short %.1f)\n",
                 n, (unsigned long long)nc, n_long, n_large, n_mid, n - n_large - n_mid, (int)by_id,
                 std::chrono::duration<double, std::milli>(t_cl0 - t_open0).count(),
                 std::chrono::duration<double, std::milli>(t_end - t_cl0).count(), ms[0], ms[1], ms[2]);
  }
  std::vector<unsigned long long> h((size_t)R * kRowStride);
  HM_CUDA(cudaMemcpyAsync(h.data(), cnt.p, sizeof(unsigned long long) * h.size(), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  for (uint32_t r = 0; r < R; ++r) {
    const unsigned long long* x = h.data() + (size_t)r * kRowStride;
    uint64_t* o = out + (size_t)r * 30;
    for (int k = 0; k < 30; ++k) o[k] = x[k];
    for (int k = 0; k < 6; ++k) o[20 + k] += x[36 + k] - x[30 + k];
  }
  return HM_OK;
}

int count_touching(hm_graph* g, const uint32_t* d_ids, uint32_t n, uint64_t out30[30]) {
  return count_touching_rows(g, d_ids, n, TouchRows{}, out30);
}

namespace {
// Candidate touched-triple schedules; the first is the default. The warp
// limit moves rows between one warp and one block per marked hyperedge, the
// mid limit moves rows between 4096-slot blocks (4 per SM) and the
// 16384-slot block (1 per SM).
constexpr TouchSchedule kTouchCandidates[] = {{128, 2048}, {64, 2048}, {32, 2048}, {0, 2048},
                                              {128, 1024}, {64, 1024}, {128, 512}};
constexpr unsigned kTouchCount = sizeof(kTouchCandidates) / sizeof(kTouchCandidates[0]);
constexpr uint32_t kTouchSample = 4096;  // marked hyperedges in the timed count
constexpr double kTouchMargin = 0.98;    // another schedule must beat the default by 2 %
static_assert(kTouchCount <= HM_TUNE_MAX_CANDIDATES, "report holds every candidate");
}  // namespace

// Times the touched-triple count of one set of live hyperedges (every n-th
// live id, about kTouchSample of them, as a batch's uniform deletions mark
// them) under each candidate schedule, by the wall time of the whole count.
int autotune_touch(hm_graph* g, hm_tune_report& R) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  R.touch_n_candidates = kTouchCount;
  for (unsigned c = 0; c < kTouchCount; ++c) {
    R.touch_rows[c][0] = kTouchCandidates[c].warp_row;
    R.touch_rows[c][1] = kTouchCandidates[c].mid_row;
  }
  const uint32_t words = (g->n_slots + 31) / 32;
  std::vector<uint32_t> bits(words);
  if (words)
    HM_CUDA(cudaMemcpyAsync(bits.data(), g->live_bits.p, sizeof(uint32_t) * words, cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  const uint32_t stride = std::max<uint32_t>(1, g->n_live / kTouchSample);
  std::vector<uint32_t> sample;
  uint32_t k = 0;
  for (uint32_t id = 0; id < g->n_slots; ++id)
    if ((bits[id >> 5] >> (id & 31)) & 1u) {
      if (k % stride == 0) sample.push_back(id);
      ++k;
    }
  const uint32_t n = (uint32_t)sample.size();
  R.touch_sampled = n;
  uint32_t best = 0;
  if (n) {
    DArr<uint32_t> d;
    HM_TRY(d.alloc(ctx, n));
    HM_CUDA(cudaMemcpyAsync(d.p, sample.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st));
    HM_CUDA(cudaStreamSynchronize(st));
    const TouchSchedule keep = g->tsched;
    uint64_t out[30];
    for (int rep = -1; rep < (int)kTouchCount; ++rep) {  // rep -1: untimed warm-up of the default
      const unsigned c = rep < 0 ? 0u : (unsigned)rep;
      g->tsched = kTouchCandidates[c];
      const auto t0 = std::chrono::steady_clock::now();
      const int s = count_touching_rows(g, d.p, n, TouchRows{}, out);  // ends with the counts on the host
      if (s < 0) {
        g->tsched = keep;
        return s;
      }
      if (rep >= 0)
        R.touch_ms[c] = (float)std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    g->tsched = keep;
    for (unsigned c = 1; c < kTouchCount; ++c)
      if (R.touch_ms[c] < kTouchMargin * R.touch_ms[0] && R.touch_ms[c] < R.touch_ms[best]) best = c;
  }
  R.touch_best = best;
  return set_schedule(g, g->sched, kTouchCandidates[best]);
}

}  // namespace hm
