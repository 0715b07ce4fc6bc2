// Exact temporal h-motif counting: THyMe's 96 motifs over a delta window.
//
// Reference semantics: THyMe+ (THyMe-main/code/main_thymeP.cpp:155-368).
// Events (a node-set with a timestamp) are processed in time order; the
// window of event a holds the events at most delta older (t + delta >= t_a).
// Identical node-sets collapse into one static hyperedge carrying the times of
// its occurrences (:164-179). For each event a, every connected static triple
// (a, b, c) of the window projection that contains a is an instance; it adds
// the number of occurrence pairs (b before c) to the motif of the order
// (b, c, a) and the pairs (c before b) to the motif of (c, b, a) (:243-334).
// Pairs of a's earlier occurrences with a neighbour give motifs 87-95, and
// two earlier occurrences of a itself motif 96 (:337-367).
//
// Device layout (built once per graph): events sorted by (time, input
// index); per position its static id (the smallest event index with the same
// node-set) and the previous position of that static id; node -> positions
// of the events containing it; static id -> positions of its occurrences.
//
// Kernel: one block per event a (position p), over the window [lo, p):
//   1. neighbours b of a: walk the window occurrences of a's nodes, keep the
//      first occurrence of each static id, and accumulate the overlap C_ab and
//      the positions of a's members it contains (mask) in a shared hash;
//   2. pairs {b, c} of neighbours: closed when b and c overlap (g from the
//      masks), open at a otherwise;
//   3. open at b: c reaches b through a node outside a and c misses a;
//      counted once per (b, c) at their smallest shared node;
//   4. motifs 87-96 from the occurrence lists.
// Equal times. THyMe shuffles its input and then sorts by time, so its order
// among equal times is random and its counts vary between runs. Here events
// with equal times are processed in input order, and the rest follows THyMe
// with its node-sets numbered in input order: of two occurrences, the one
// strictly earlier in time comes first (main_thymeP.cpp:313-323), and a tie
// counts as "c before b", where b is the node-set of the pair met first in
// the input. The total and the per-static-class sums do not depend on any of
// this; with strictly increasing times none of it arises.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "hm_classes.h"
#include "hm_device.h"

namespace hm {
namespace {

constexpr unsigned kWarp = 32;
constexpr unsigned kBlock = 256;
constexpr unsigned kWarps = kBlock / kWarp;
constexpr uint32_t kEmpty = 0xffffffffu;
constexpr uint32_t kNone = 0xffffffffu;

__constant__ int8_t c_temporal[128];

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint64_t global_warp() { return ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ uint64_t n_warps() { return ((uint64_t)gridDim.x * blockDim.x) >> 5; }
__device__ __forceinline__ uint64_t gtid() { return (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint64_t gstride() { return (uint64_t)gridDim.x * blockDim.x; }

__device__ __forceinline__ int tclass(int s1, int s2, int s3, int c12, int c23, int c31, int g) {
  return c_temporal[region_pattern(s1, s2, s3, c12, c23, c31, g)];
}

// ---- index construction --------------------------------------------------------

__global__ void k_row_hash(const uint64_t* off, const uint32_t* len, const uint32_t* mem, uint32_t n, uint64_t* h) {
  for (uint64_t r = gtid(); r < n; r += gstride()) {
    uint64_t x = 0x9E3779B97F4A7C15ull ^ len[r];
    const uint32_t* m = mem + off[r];
    for (uint32_t i = 0; i < len[r]; ++i) {
      x ^= m[i] + 0x9E3779B97F4A7C15ull + (x << 6) + (x >> 2);
      x *= 0xBF58476D1CE4E5B9ull;
    }
    h[r] = x ^ (x >> 31);
  }
}

__device__ __forceinline__ bool same_rows(const uint64_t* off, const uint32_t* len, const uint32_t* mem, uint32_t a,
                                          uint32_t b) {
  if (len[a] != len[b]) return false;
  const uint32_t* x = mem + off[a];
  const uint32_t* y = mem + off[b];
  for (uint32_t i = 0; i < len[a]; ++i)
    if (x[i] != y[i]) return false;
  return true;
}

// Events sorted by (hash, index): the static id of an event is the first
// event of its hash run with the same node-set.
__global__ void k_static_ids(const uint64_t* hs, const uint32_t* ev, uint32_t n, const uint64_t* off,
                             const uint32_t* len, const uint32_t* mem, uint32_t* sid) {
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    uint64_t s = i;
    while (s > 0 && hs[s - 1] == hs[i]) --s;
    uint32_t rep = ev[i];
    for (uint64_t k = s; k < i; ++k)
      if (same_rows(off, len, mem, ev[k], ev[i])) {
        rep = ev[k];
        break;
      }
    sid[ev[i]] = rep;
  }
}

__global__ void k_time_keys(const int64_t* t, uint32_t n, uint64_t* key, uint32_t* idx) {
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    key[i] = (uint64_t)t[i] ^ 0x8000000000000000ull;  // order-preserving for signed times
    idx[i] = (uint32_t)i;
  }
}

__global__ void k_position_fields(const uint32_t* order, uint32_t n, const int64_t* t, const uint32_t* sid,
                                  int64_t* tp, uint32_t* sp, uint32_t* occ_key, uint32_t* occ_val) {
  for (uint64_t p = gtid(); p < n; p += gstride()) {
    const uint32_t e = order[p];
    tp[p] = t[e];
    sp[p] = sid[e];
    occ_key[p] = sid[e];
    occ_val[p] = (uint32_t)p;
  }
}

__global__ void k_prev_same(const uint32_t* key, const uint32_t* pos, uint32_t n, uint32_t* prev) {
  for (uint64_t i = gtid(); i < n; i += gstride())
    prev[pos[i]] = (i > 0 && key[i - 1] == key[i]) ? pos[i - 1] : kNone;
}

__global__ void k_count_keys(const uint32_t* key, uint32_t n, uint32_t* cnt) {
  for (uint64_t i = gtid(); i < n; i += gstride()) atomicAdd(&cnt[key[i]], 1u);
}

// (node, position) pairs in position order.
__global__ void k_node_positions(const uint32_t* order, uint32_t n, const uint64_t* off, const uint32_t* len,
                                 const uint32_t* mem, const uint64_t* pair_off, uint32_t* key, uint32_t* val,
                                 uint32_t* node_cnt) {
  for (uint64_t p = global_warp(); p < n; p += n_warps()) {
    const uint32_t e = order[p];
    const uint64_t s = off[e], d = pair_off[p];
    for (uint32_t i = lane_id(); i < len[e]; i += kWarp) {
      const uint32_t v = mem[s + i];
      key[d + i] = v;
      val[d + i] = (uint32_t)p;
      atomicAdd(&node_cnt[v], 1u);
    }
  }
}

__global__ void k_gather_len(const uint32_t* order, uint32_t n, const uint32_t* len, uint32_t* out) {
  for (uint64_t p = gtid(); p < n; p += gstride()) out[p] = len[order[p]];
}

__global__ void k_window_lo(const int64_t* t, uint32_t n, int64_t delta, uint32_t* lo) {
  for (uint64_t p = gtid(); p < n; p += gstride()) {
    const int64_t tp = t[p];
    // first q with t[q] + delta >= t[p]
    uint32_t l = 0, h = (uint32_t)p;
    while (l < h) {
      const uint32_t mid = (l + h) >> 1;
      if (t[mid] + delta < tp) l = mid + 1;
      else h = mid;
    }
    lo[p] = l;
  }
}

// ---- counting --------------------------------------------------------------------

struct TArgs {
  uint32_t n;            // events
  const uint32_t* order; // position -> event
  const uint32_t* sp;    // position -> static id
  const uint32_t* prev;  // position -> previous position of the same static id
  const uint32_t* lo;    // position -> window start
  const uint64_t* hoff;  // event -> members
  const uint32_t* hlen;
  const uint32_t* hmem;
  const uint64_t* voff;  // node -> positions
  const uint32_t* vlen;
  const uint32_t* vpos;
  const uint64_t* ooff;  // static id -> occurrence positions
  const uint32_t* olen;
  const uint32_t* opos;
  const int64_t* tp;     // position -> time
  unsigned int* queue;
  unsigned long long* out;  // 96
  int* overflow;
  // window-projection sizes behind the algorithmic bytes: [0] neighbours of
  // each event in its window, [1] adjacent pairs among them, [2] pairs
  // (b, c) with c adjacent to a neighbour b but not to the event
  unsigned long long* stats;
  unsigned int* queue2;      // the deferred launch's queue
  unsigned int* n_deferred;  // events set aside by the first launch
  uint32_t* deferred;
};

// [first, last) of the sorted list x[0..n) restricted to values in [lo, hi)
__device__ __forceinline__ void range_in(const uint32_t* x, uint32_t n, uint32_t lo, uint32_t hi, uint32_t& first,
                                         uint32_t& last) {
  uint32_t l = 0, h = n;
  while (l < h) {
    const uint32_t m = (l + h) >> 1;
    if (x[m] < lo) l = m + 1;
    else h = m;
  }
  first = l;
  h = n;
  while (l < h) {
    const uint32_t m = (l + h) >> 1;
    if (x[m] < hi) l = m + 1;
    else h = m;
  }
  last = l;
}

// Occurrence pairs (x in X, y in Y) with x strictly earlier in time than y,
// X and Y positions sorted ascending (so their times are non-decreasing).
// Times, not positions, are compared, as THyMe compares occurrence times
// (THyMe-main/code/main_thymeP.cpp:313-323): two occurrences with equal
// times count as "y before x", while the window itself follows positions.
__device__ __forceinline__ uint64_t ordered_pairs(const int64_t* T, const uint32_t* X, uint32_t nx,
                                                  const uint32_t* Y, uint32_t ny) {
  if (nx == 1 && ny == 1) return T[X[0]] < T[Y[0]];
  uint64_t c = 0;
  uint32_t j = 0;
  for (uint32_t i = 0; i < nx; ++i) {
    const int64_t tx = T[X[i]];
    while (j < ny && T[Y[j]] <= tx) ++j;
    c += ny - j;
  }
  return c;
}

// |X & Y| and the smallest shared value (kNone if none)
__device__ __forceinline__ uint32_t overlap(const uint32_t* X, uint32_t nx, const uint32_t* Y, uint32_t ny,
                                            uint32_t& first) {
  uint32_t i = 0, j = 0, c = 0;
  first = kNone;
  while (i < nx && j < ny) {
    const uint32_t x = X[i], y = Y[j];
    if (x < y) ++i;
    else if (y < x) ++j;
    else {
      if (!c) first = x;
      ++c;
      ++i;
      ++j;
    }
  }
  return c;
}

// Shared memory of one block: per neighbour (kM of them) its mask, first
// window time, id, overlap with a, first window occurrence, occurrence count
// and hash slot; the hash (kS keys, kS neighbour indices).
template <uint32_t kS, uint32_t kM>
constexpr size_t temporal_smem() {
  return (size_t)kM * (2 * sizeof(unsigned long long) + 4 * sizeof(uint32_t) + sizeof(uint16_t)) +
         (size_t)kS * (sizeof(uint32_t) + sizeof(uint16_t));
}

// Block per event; kS hash slots hold up to kM window neighbours. The first
// launch (kFirst) takes every event and sets aside those with more
// neighbours in a deferred list; the second takes that list with a larger
// table, and reports an event that overflows it too.
template <uint32_t kS, uint32_t kM, bool kFirst>
__global__ void __launch_bounds__(kBlock) k_temporal(TArgs A) {
  static_assert(kM <= 65535 && kS <= 65536 && (kS & (kS - 1)) == 0, "table shape");
  constexpr uint32_t kHashShift = 32 - __builtin_ctz(kS);
  extern __shared__ unsigned long long tsm[];
  unsigned long long* nmask = tsm;                                  // kM: a's member positions in b (< 64)
  long long* nt0 = reinterpret_cast<long long*>(nmask + kM);        // kM: time of b's first window occurrence
  uint32_t* nid = reinterpret_cast<uint32_t*>(nt0 + kM);            // kM: static id b
  uint32_t* ncab = nid + kM;                                        // kM: C_ab
  uint32_t* nof = ncab + kM;                                        // kM: first window occurrence (index into opos)
  uint32_t* non = nof + kM;                                         // kM: window occurrences
  uint32_t* keys = non + kM;                                        // kS
  uint16_t* hidx = reinterpret_cast<uint16_t*>(keys + kS);          // kS: neighbour index of a slot
  uint16_t* la = hidx + kS;                                         // kM: slot of a neighbour
  __shared__ unsigned long long wcnt[kWarps][96];
  __shared__ int8_t tab[128];
  __shared__ uint32_t sam[256];
  __shared__ uint32_t s_item, s_nla;
  const unsigned w = threadIdx.x / kWarp, lane = lane_id();
  unsigned long long n_nbrs = 0, n_closed = 0, n_open_b = 0;  // this thread's share of A.stats
  for (unsigned k = threadIdx.x; k < kWarps * 96; k += blockDim.x) (&wcnt[0][0])[k] = 0;
  for (unsigned k = threadIdx.x; k < 128; k += blockDim.x) tab[k] = c_temporal[k];
  // the table is cleared once here; after each event only the slots it used
  // are reset (all of them after an overflow)
  for (unsigned i = threadIdx.x; i < kS; i += blockDim.x) keys[i] = kEmpty;
  auto tcls = [&](int s1, int s2, int s3, int c12, int c23, int c31, int g) {
    return (int)tab[region_pattern(s1, s2, s3, c12, c23, c31, g)];
  };
  unsigned long long* wc = wcnt[w];
  for (;;) {
    if (threadIdx.x == 0) {
      s_item = atomicAdd(kFirst ? A.queue : A.queue2, 1u);
      s_nla = 0;
    }
    __syncthreads();
    const uint32_t item = s_item;
    if (kFirst ? item >= A.n : item >= *A.n_deferred) break;
    const uint32_t p = kFirst ? item : A.deferred[item];
    const uint32_t lo = A.lo[p];
    const uint32_t ea = A.order[p];
    const uint32_t sa = A.sp[p];
    const uint32_t asz = A.hlen[ea];
    const uint32_t* am = A.hmem + A.hoff[ea];
    if (asz <= 256) {
      for (uint32_t i = threadIdx.x; i < asz; i += blockDim.x) sam[i] = am[i];
      am = sam;
    }
    // 1. neighbours of a in the window (first occurrence of each static id)
    for (uint32_t i = w; i < asz; i += kWarps) {
      const uint32_t v = A.hmem[A.hoff[ea] + i];
      const uint32_t* vp = A.vpos + A.voff[v];
      uint32_t f, l;
      range_in(vp, A.vlen[v], lo, p, f, l);
      for (uint32_t k = f + lane; k < l; k += kWarp) {
        const uint32_t q = vp[k];
        const uint32_t x = A.sp[q];
        if (x == sa) continue;
        const uint32_t pr = A.prev[q];
        if (pr != kNone && pr >= lo) continue;  // not the first occurrence of x in the window
        uint32_t h = (x * 2654435761u) >> kHashShift;
        for (uint32_t probe = 0;; ++probe) {
          if (probe == kS) {  // table full: more neighbours than the window limit
            atomicAdd(&s_nla, kS);
            break;
          }
          const uint32_t old = atomicCAS(&keys[h], kEmpty, x);
          if (old == kEmpty) {
            const uint32_t idx = atomicAdd(&s_nla, 1u);
            if (idx < kM) {
              hidx[h] = (uint16_t)idx;
              la[idx] = (uint16_t)h;
              nid[idx] = x;
              ncab[idx] = 0;
              nmask[idx] = 0;
            }
          }
          if (old == kEmpty || old == x) break;
          h = (h + 1) & (kS - 1);
        }
      }
    }
    __syncthreads();
    const uint32_t nla = s_nla;
    if (nla > kM) {
      if (threadIdx.x == 0) {
        if (kFirst) A.deferred[atomicAdd(A.n_deferred, 1u)] = p;
        else atomicExch(A.overflow, 1);
      }
      for (unsigned i = threadIdx.x; i < kS; i += blockDim.x) keys[i] = kEmpty;
      __syncthreads();
      continue;  // block-uniform
    }
    // overlaps and member positions (a second sweep, after initialisation),
    // and each neighbour's window occurrences
    for (uint32_t i = w; i < asz; i += kWarps) {
      const uint32_t v = am[i];
      const uint32_t* vp = A.vpos + A.voff[v];
      uint32_t f, l;
      range_in(vp, A.vlen[v], lo, p, f, l);
      for (uint32_t k = f + lane; k < l; k += kWarp) {
        const uint32_t q = vp[k];
        const uint32_t x = A.sp[q];
        if (x == sa) continue;
        const uint32_t pr = A.prev[q];
        if (pr != kNone && pr >= lo) continue;
        uint32_t h = (x * 2654435761u) >> kHashShift;
        while (keys[h] != x) h = (h + 1) & (kS - 1);  // present: inserted above
        const uint32_t idx = hidx[h];
        atomicAdd(&ncab[idx], 1u);
        if (i < 64) atomicOr(&nmask[idx], 1ull << i);
      }
    }
    for (uint32_t i = threadIdx.x; i < nla; i += blockDim.x) {
      const uint32_t b = nid[i];
      const uint32_t* bo = A.opos + A.ooff[b];
      uint32_t bf, bl;
      range_in(bo, A.olen[b], lo, p, bf, bl);
      nof[i] = (uint32_t)A.ooff[b] + bf;
      non[i] = bl - bf;
      nt0[i] = A.tp[bo[bf]];  // bl > bf: b occurs in the window
    }
    __syncthreads();
    if (threadIdx.x == 0) n_nbrs += nla;
    const uint32_t* ao = A.opos + A.ooff[sa];
    uint32_t af, al;
    range_in(ao, A.olen[sa], lo, p, af, al);  // a's earlier occurrences in the window
    const uint32_t ta_n = al - af;
    // 2. pairs of neighbours
    for (uint32_t i = w; i < nla; i += kWarps) {
      const uint32_t b = nid[i], cab = ncab[i];
      const unsigned long long mb = nmask[i];
      const uint32_t* bm = A.hmem + A.hoff[b];
      const uint32_t bsz = A.hlen[b];
      const uint32_t bn = non[i];
      const uint32_t* bo = A.opos + nof[i];
      const long long tb = nt0[i];
      for (uint32_t j = i + 1 + lane; j < nla; j += kWarp) {
        const uint32_t c = nid[j], cac = ncab[j];
        const uint32_t* cm = A.hmem + A.hoff[c];
        const uint32_t csz = A.hlen[c];
        uint32_t first;
        const uint32_t cbc = overlap(bm, bsz, cm, csz, first);
        uint32_t g = 0;
        n_closed += cbc != 0;
        if (cbc) {
          if (asz <= 64) {
            g = __popcll(mb & nmask[j]);
          } else {
            // |a & b & c| by merging a's members with the b & c shared list
            uint32_t x = 0, y = 0, z = 0;
            while (x < asz && y < bsz && z < csz) {
              const uint32_t u = am[x], vv = bm[y], t = cm[z];
              const uint32_t mx = max(u, max(vv, t));
              if (u == mx && vv == mx && t == mx) { ++g; ++x; ++y; ++z; }
              else { x += u < mx; y += vv < mx; z += t < mx; }
            }
          }
        }
        const uint32_t cn = non[j];
        // Of the two, the node-set that comes first in the input (the smaller
        // static id) plays THyMe's "b": occurrence pairs with it strictly
        // earlier go to its order, all others (ties too) to the other order.
        uint64_t bc;
        if (bn == 1 && cn == 1) {
          const long long tc = nt0[j];
          bc = b < c ? tb < tc : tb <= tc;
        } else {
          const uint32_t* co = A.opos + nof[j];
          bc = b < c ? ordered_pairs(A.tp, bo, bn, co, cn) : (uint64_t)bn * cn - ordered_pairs(A.tp, co, cn, bo, bn);
        }
        const uint64_t cb = (uint64_t)bn * cn - bc;
        const int kbc = tcls((int)bsz, (int)csz, (int)asz, (int)cbc, (int)cac, (int)cab, (int)g);
        const int kcb = tcls((int)csz, (int)bsz, (int)asz, (int)cbc, (int)cab, (int)cac, (int)g);
        if (bc && kbc >= 0) atomicAdd(&wc[kbc], (unsigned long long)bc);
        if (cb && kcb >= 0) atomicAdd(&wc[kcb], (unsigned long long)cb);
      }
      // 4. motifs 87-95 for the pair (a, b)
      if (lane == 0) {
        const uint64_t ab = ordered_pairs(A.tp, ao + af, ta_n, bo, bn);
        const uint64_t ba = (uint64_t)ta_n * bn - ab;
        const uint64_t bb = (uint64_t)bn * (bn ? bn - 1 : 0) / 2;
        const int kab = tcls((int)asz, (int)bsz, (int)asz, (int)cab, (int)cab, (int)asz, (int)cab);
        const int kba = tcls((int)bsz, (int)asz, (int)asz, (int)cab, (int)asz, (int)cab, (int)cab);
        const int kbb = tcls((int)bsz, (int)bsz, (int)asz, (int)bsz, (int)cab, (int)cab, (int)cab);
        if (ab && kab >= 0) atomicAdd(&wc[kab], (unsigned long long)ab);
        if (ba && kba >= 0) atomicAdd(&wc[kba], (unsigned long long)ba);
        if (bb && kbb >= 0) atomicAdd(&wc[kbb], (unsigned long long)bb);
      }
    }
    // 3. open at b: c meets b outside a and misses a
    for (uint32_t i = w; i < nla; i += kWarps) {
      const uint32_t b = nid[i], cab = ncab[i];
      const uint32_t* bm = A.hmem + A.hoff[b];
      const uint32_t bsz = A.hlen[b];
      const uint32_t bn = non[i];
      const uint32_t* bo = A.opos + nof[i];
      for (uint32_t kk = 0; kk < bsz; ++kk) {
        const uint32_t v = bm[kk];
        // skip nodes of a (a's members are sorted)
        uint32_t l2 = 0, h2 = asz;
        while (l2 < h2) {
          const uint32_t m = (l2 + h2) >> 1;
          if (am[m] < v) l2 = m + 1;
          else h2 = m;
        }
        if (l2 < asz && am[l2] == v) continue;
        const uint32_t* vp = A.vpos + A.voff[v];
        uint32_t f, l;
        range_in(vp, A.vlen[v], lo, p, f, l);
        for (uint32_t k = f + lane; k < l; k += kWarp) {
          const uint32_t q = vp[k];
          const uint32_t c = A.sp[q];
          if (c == b || c == sa) continue;
          const uint32_t pr = A.prev[q];
          if (pr != kNone && pr >= lo) continue;
          // c must miss a: not a neighbour of a
          uint32_t h = (c * 2654435761u) >> kHashShift;
          bool nbr_of_a = false;
          for (;;) {
            const uint32_t kh = keys[h];
            if (kh == c) { nbr_of_a = true; break; }
            if (kh == kEmpty) break;
            h = (h + 1) & (kS - 1);
          }
          if (nbr_of_a) continue;
          const uint32_t* cm = A.hmem + A.hoff[c];
          const uint32_t csz = A.hlen[c];
          uint32_t first;
          const uint32_t cbc = overlap(bm, bsz, cm, csz, first);
          if (first != v) continue;  // counted at the smallest shared node
          ++n_open_b;
          const uint32_t* co = A.opos + A.ooff[c];
          uint32_t cf, cl;
          range_in(co, A.olen[c], lo, p, cf, cl);
          const uint32_t nc = cl - cf;
          const uint64_t bc = ordered_pairs(A.tp, bo, bn, co + cf, nc);
          const uint64_t cb = (uint64_t)bn * nc - bc;
          const int kbc = tcls((int)bsz, (int)csz, (int)asz, (int)cbc, 0, (int)cab, 0);
          const int kcb = tcls((int)csz, (int)bsz, (int)asz, (int)cbc, (int)cab, 0, 0);
          if (bc && kbc >= 0) atomicAdd(&wc[kbc], (unsigned long long)bc);
          if (cb && kcb >= 0) atomicAdd(&wc[kcb], (unsigned long long)cb);
        }
      }
    }
    // 4. motif 96: two earlier occurrences of a
    if (threadIdx.x == 0 && ta_n >= 2) atomicAdd(&wc[95], (unsigned long long)ta_n * (ta_n - 1) / 2);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nla; i += blockDim.x) keys[la[i]] = kEmpty;  // reset the used slots
  }
  __syncthreads();
  for (unsigned k = threadIdx.x; k < 96; k += blockDim.x) {
    unsigned long long t = 0;
    for (unsigned ww = 0; ww < kWarps; ++ww) t += wcnt[ww][k];
    if (t) atomicAdd(&A.out[k], t);
  }
  for (int d = 16; d; d >>= 1) {
    n_nbrs += __shfl_xor_sync(0xffffffffu, n_nbrs, d);
    n_closed += __shfl_xor_sync(0xffffffffu, n_closed, d);
    n_open_b += __shfl_xor_sync(0xffffffffu, n_open_b, d);
  }
  if (lane == 0) {
    if (n_nbrs) atomicAdd(&A.stats[0], n_nbrs);
    if (n_closed) atomicAdd(&A.stats[1], n_closed);
    if (n_open_b) atomicAdd(&A.stats[2], n_open_b);
  }
}

// Table shapes: the first launch's (4 blocks per SM) and the deferred one's.
constexpr uint32_t kSlotsSmall = 2048, kNbrsSmall = 1024;
constexpr uint32_t kSlotsLarge = 8192, kNbrsLarge = 4096;
constexpr uint32_t kMaxNbrs = kNbrsLarge;  // neighbours of one event inside its window

template <class K, class V>
int sort_pairs(hm_ctx* ctx, const K* kin, K* kout, const V* vin, V* vout, uint64_t n, int end_bit) {
  size_t tb = 0;
  HM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, kout, vin, vout, (int64_t)n, 0, end_bit, ctx->stream));
  DArr<uint8_t> tmp;
  HM_TRY(tmp.alloc(ctx, tb));
  HM_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, kin, kout, vin, vout, (int64_t)n, 0, end_bit, ctx->stream));
  return HM_OK;
}

}  // namespace

// Builds the time-ordered index of a temporal graph (once).
static int build_temporal_index(hm_graph* g) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  const uint32_t n = g->n_slots;
  static bool table_ready = false;
  if (!table_ready) {
    int8_t inv[128];
    for (int i = 0; i < 128; ++i) inv[i] = -1;
    for (int m = 0; m < HM_N_TEMPORAL_MOTIFS; ++m) inv[kTemporalMotifPattern[m]] = (int8_t)m;
    HM_CUDA(cudaMemcpyToSymbol(c_temporal, inv, sizeof(inv)));
    table_ready = true;
  }
  // static ids
  DArr<uint64_t> hs, hs_sorted;
  DArr<uint32_t> ev, ev_sorted, sid;
  HM_TRY(hs.alloc(ctx, n));
  HM_TRY(hs_sorted.alloc(ctx, n));
  HM_TRY(ev.alloc(ctx, n));
  HM_TRY(ev_sorted.alloc(ctx, n));
  HM_TRY(sid.alloc(ctx, n));
  k_row_hash<<<grid_for(n, kBlock), kBlock, 0, st>>>(g->h2v_off.p, g->h2v_len.p, g->h2v_mem.p, n, hs.p);
  HM_LAUNCH_CHECK();
  {
    std::vector<uint32_t> iota(n);
    for (uint32_t i = 0; i < n; ++i) iota[i] = i;
    HM_CUDA(cudaMemcpyAsync(ev.p, iota.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st));
    HM_CUDA(cudaStreamSynchronize(st));
  }
  HM_TRY(sort_pairs(ctx, hs.p, hs_sorted.p, ev.p, ev_sorted.p, n, 64));
  k_static_ids<<<grid_for(n, kBlock), kBlock, 0, st>>>(hs_sorted.p, ev_sorted.p, n, g->h2v_off.p, g->h2v_len.p,
                                                        g->h2v_mem.p, sid.p);
  HM_LAUNCH_CHECK();
  // time order
  DArr<uint64_t> tk, tk_sorted;
  HM_TRY(tk.alloc(ctx, n));
  HM_TRY(tk_sorted.alloc(ctx, n));
  HM_TRY(g->t_order.alloc(ctx, n));
  k_time_keys<<<grid_for(n, kBlock), kBlock, 0, st>>>(g->ts.p, n, tk.p, ev.p);
  HM_LAUNCH_CHECK();
  HM_TRY(sort_pairs(ctx, tk.p, tk_sorted.p, ev.p, g->t_order.p, n, 64));
  HM_TRY(g->t_time.alloc(ctx, n));
  HM_TRY(g->t_static.alloc(ctx, n));
  DArr<uint32_t> okey, oval, okey_s;
  HM_TRY(okey.alloc(ctx, n));
  HM_TRY(oval.alloc(ctx, n));
  HM_TRY(okey_s.alloc(ctx, n));
  HM_TRY(g->t_opos.alloc(ctx, n));
  k_position_fields<<<grid_for(n, kBlock), kBlock, 0, st>>>(g->t_order.p, n, g->ts.p, sid.p, g->t_time.p,
                                                             g->t_static.p, okey.p, oval.p);
  HM_LAUNCH_CHECK();
  int eb = 1;
  while (eb < 32 && (1ull << eb) < n) ++eb;
  HM_TRY(sort_pairs(ctx, okey.p, okey_s.p, oval.p, g->t_opos.p, n, eb));
  HM_TRY(g->t_prev.alloc(ctx, n));
  k_prev_same<<<grid_for(n, kBlock), kBlock, 0, st>>>(okey_s.p, g->t_opos.p, n, g->t_prev.p);
  HM_LAUNCH_CHECK();
  HM_TRY(g->t_olen.alloc(ctx, n));
  HM_CUDA(cudaMemsetAsync(g->t_olen.p, 0, sizeof(uint32_t) * n, st));
  k_count_keys<<<grid_for(n, kBlock), kBlock, 0, st>>>(okey_s.p, n, g->t_olen.p);
  HM_LAUNCH_CHECK();
  HM_TRY(g->t_ooff.alloc(ctx, (size_t)n + 1));
  HM_TRY(exclusive_scan(ctx, g->t_olen.p, g->t_ooff.p, n));
  // node -> positions
  DArr<uint32_t> plen;
  DArr<uint64_t> poff;
  HM_TRY(plen.alloc(ctx, n));
  HM_TRY(poff.alloc(ctx, (size_t)n + 1));
  k_gather_len<<<grid_for(n, kBlock), kBlock, 0, st>>>(g->t_order.p, n, g->h2v_len.p, plen.p);
  HM_LAUNCH_CHECK();
  HM_TRY(exclusive_scan(ctx, plen.p, poff.p, n));
  uint64_t nnz = 0;
  HM_CUDA(cudaMemcpyAsync(&nnz, poff.p + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  const uint32_t V = g->n_nodes;
  DArr<uint32_t> nk, nv, nk_s;
  HM_TRY(nk.alloc(ctx, nnz));
  HM_TRY(nv.alloc(ctx, nnz));
  HM_TRY(nk_s.alloc(ctx, nnz));
  HM_TRY(g->t_vpos.alloc(ctx, nnz));
  HM_TRY(g->t_vlen.alloc(ctx, V));
  HM_CUDA(cudaMemsetAsync(g->t_vlen.p, 0, sizeof(uint32_t) * V, st));
  k_node_positions<<<grid_for((uint64_t)n * 32, kBlock), kBlock, 0, st>>>(g->t_order.p, n, g->h2v_off.p, g->h2v_len.p,
                                                                         g->h2v_mem.p, poff.p, nk.p, nv.p,
                                                                         g->t_vlen.p);
  HM_LAUNCH_CHECK();
  int vb = 1;
  while (vb < 32 && (1ull << vb) < V) ++vb;
  if (nnz) HM_TRY(sort_pairs(ctx, nk.p, nk_s.p, nv.p, g->t_vpos.p, nnz, vb));
  HM_TRY(g->t_voff.alloc(ctx, (size_t)V + 1));
  HM_TRY(exclusive_scan(ctx, g->t_vlen.p, g->t_voff.p, V));
  HM_CUDA(cudaStreamSynchronize(st));
  g->t_ready = true;
  return HM_OK;
}

namespace {
// The 96 counts of one temporal count into the caller's buffer, or all ones
// when an event's window overflowed the neighbour table.
__global__ void k_temporal_finish(const unsigned long long* acc, uint64_t* out96) {
  const unsigned k = threadIdx.x;
  if (k < 96) out96[k] = acc[97] ? ~0ull : acc[k];
}
}  // namespace

// Queues the window starts and the counting kernels on the context stream:
// acc receives the 96 counts, [96] the work queue, [97] the overflow flag,
// [98..100] the window-projection sizes, [101] the deferred launch's queue,
// [102] the number of deferred events; lo holds the window starts and then
// the deferred events. Events e0/e1 bracket the kernels.
static int launch_temporal(hm_graph* g, int64_t delta, DArr<uint32_t>& lo, DArr<unsigned long long>& acc,
                           cudaEvent_t e0, cudaEvent_t e1) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  const uint32_t n = g->n_slots;
  if (!g->t_ready) HM_TRY(build_temporal_index(g));
  HM_TRY(lo.alloc(ctx, 2 * (size_t)n));
  HM_TRY(acc.alloc(ctx, 103));
  HM_CUDA(cudaMemsetAsync(acc.p, 0, sizeof(unsigned long long) * 103, st));
  if (e0) HM_CUDA(cudaEventRecord(e0, st));
  k_window_lo<<<grid_for(n, kBlock), kBlock, 0, st>>>(g->t_time.p, n, delta, lo.p);
  HM_LAUNCH_CHECK();
  TArgs A{n,
          g->t_order.p,
          g->t_static.p,
          g->t_prev.p,
          lo.p,
          g->h2v_off.p,
          g->h2v_len.p,
          g->h2v_mem.p,
          g->t_voff.p,
          g->t_vlen.p,
          g->t_vpos.p,
          g->t_ooff.p,
          g->t_olen.p,
          g->t_opos.p,
          g->t_time.p,
          reinterpret_cast<unsigned int*>(acc.p + 96),
          acc.p,
          reinterpret_cast<int*>(acc.p + 97),
          acc.p + 98,
          reinterpret_cast<unsigned int*>(acc.p + 101),
          reinterpret_cast<unsigned int*>(acc.p + 102),
          lo.p + n};
  constexpr size_t kSmemSmall = temporal_smem<kSlotsSmall, kNbrsSmall>();
  constexpr size_t kSmemLarge = temporal_smem<kSlotsLarge, kNbrsLarge>();
  static bool attr = false;
  if (!attr) {
    HM_CUDA(cudaFuncSetAttribute(k_temporal<kSlotsSmall, kNbrsSmall, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemSmall));
    HM_CUDA(cudaFuncSetAttribute(k_temporal<kSlotsLarge, kNbrsLarge, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemLarge));
    attr = true;
  }
  k_temporal<kSlotsSmall, kNbrsSmall, true>
      <<<std::min<unsigned>((unsigned)ctx->n_sms * 4, n), kBlock, kSmemSmall, st>>>(A);
  HM_LAUNCH_CHECK();
  k_temporal<kSlotsLarge, kNbrsLarge, false><<<(unsigned)ctx->n_sms, kBlock, kSmemLarge, st>>>(A);
  HM_LAUNCH_CHECK();
  if (e1) HM_CUDA(cudaEventRecord(e1, st));
  return HM_OK;
}

static int temporal_args_ok(const hm_graph* g, int64_t delta) {
  if (!g->temporal) return set_error(HM_ERR_STATE, "temporal count: the graph has no timestamps");
  if (delta < 0) return set_error(HM_ERR_INVALID, "temporal count: delta must be >= 0");
  return HM_OK;
}

int count_temporal96(hm_graph* g, int64_t delta, uint64_t out96[96]) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  for (int k = 0; k < 96; ++k) out96[k] = 0;
  HM_TRY(temporal_args_ok(g, delta));
  const uint32_t n = g->n_slots;
  if (!n) return HM_OK;
  DArr<uint32_t> lo;
  DArr<unsigned long long> acc;
  cudaEvent_t e0, e1;
  HM_CUDA(cudaEventCreate(&e0));
  HM_CUDA(cudaEventCreate(&e1));
  const int rc = launch_temporal(g, delta, lo, acc, e0, e1);
  unsigned long long h[103];
  cudaError_t ce = rc < 0 ? cudaSuccess : cudaMemcpyAsync(h, acc.p, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (rc >= 0 && ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  float ms = 0;
  if (rc >= 0 && ce == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc < 0) return rc;
  if (ce != cudaSuccess) return set_error(HM_ERR_CUDA, "temporal count: %s", cudaGetErrorString(ce));
  g->times.temporal_ms = ms;
  g->times.t_events = n;
  g->times.t_delta = delta;
  g->times.t_nbrs = h[98];
  g->times.t_closed_pairs = h[99];
  g->times.t_open_pairs = h[100];
  if (h[97])
    return set_error(HM_ERR_LIMIT, "temporal count: an event has more than %u neighbours inside its window",
                     kMaxNbrs);
  for (int k = 0; k < 96; ++k) out96[k] = h[k];
  return HM_OK;
}

// The same, queued: no host wait once the time-ordered index exists; the
// counts land in d_out96 (all ones on a window overflow). The timings and
// the window-projection sizes of an asynchronous count are not read back.
int count_temporal96_async(hm_graph* g, int64_t delta, uint64_t* d_out96) {
  hm_ctx* ctx = g->ctx;
  HM_TRY(temporal_args_ok(g, delta));
  g->times.temporal_ms = -1.0f;
  g->times.t_events = 0;
  if (!g->n_slots) {
    HM_CUDA(cudaMemsetAsync(d_out96, 0, sizeof(uint64_t) * 96, ctx->stream));
    return HM_OK;
  }
  DArr<uint32_t> lo;
  DArr<unsigned long long> acc;
  HM_TRY(launch_temporal(g, delta, lo, acc, nullptr, nullptr));
  k_temporal_finish<<<1, 96, 0, ctx->stream>>>(acc.p, d_out96);
  HM_LAUNCH_CHECK();
  return HM_OK;  // lo and acc are freed in stream order, after the kernels
}

}  // namespace hm
