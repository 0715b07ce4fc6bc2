// Exact static h-motif counting (the 30 classes behind MoCHy's 26 motifs).
//
// Reference semantics: MoCHy exact (MoCHy-master/main_exact.cpp:91-129)
// classifies every connected triple {a, b, c} of distinct hyperedges: open
// triples (exactly two overlapping pairs) at their centre, closed triples once.
// The reference GPU counter (dynamicHyperGraph/src/HMotifCount.cu:16-125) runs
// one thread per hyperedge over closed triangles only and never sees open
// triples; this file counts both.
//
// Algorithm (all integer, exact):
//   1. Open phase, one warp per centre a. Every unordered neighbour pair
//      {b, c} of a is classified as if it were open: its class depends only on
//      [C_ab + C_ac < |a|], [C_ab < |b|], [C_ac < |c|]. A histogram of the
//      neighbours by (overlap, [overlap < size]) gives the six class counts
//      with prefix sums, without touching pairs one by one.
//   2. Closed phase, one block per centre a (the lowest-ranked corner under
//      (degree, id) order): N+(a) goes into a shared-memory hash table, each
//      warp walks N+(b) for one b in N+(a) and probes it. Every triangle is
//      found exactly once; it adds its closed class and removes the three
//      open-pair classes phase 1 gave it at its three centres.
//   The triple overlap g = |a & b & c| is popc(mask_ab & mask_ac), where each
//   adjacency entry carries the positions of the owner's members it shares;
//   centres with more than 64 members fall back to a merge of the lists.
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
constexpr unsigned kOpenBlock = 256;
constexpr unsigned kOpenWarps = kOpenBlock / kWarp;
constexpr unsigned kClosedBlock = 256;
constexpr unsigned kClosedWarps = kClosedBlock / kWarp;
constexpr unsigned kUnroll = 4;               // probes in flight per lane
constexpr unsigned kNumCounters = 36;        // 30 closed classes + 6 open-pair classes
// Block launch shapes of the closed phase: rows up to the schedule's
// small_row with a 4096-slot bucketized table (4 blocks of 256 threads per
// SM), longer rows with a 16384-slot table (one 1024-thread block per SM).
// kSmallRow is the largest small_row the 4096-slot table holds in shared
// memory (load <= 1/2).
constexpr unsigned kSmallRow = 2048;
// Rows up to the schedule's warp_row go to the warp-per-centre kernel; its
// 256-slot table per warp holds at most kWarpRow entries (load <= 1/2).
constexpr unsigned kWarpRow = 128;
constexpr unsigned kWarpSlots = 256;
constexpr uint32_t kEmpty = 0xffffffffu;

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint64_t global_warp() { return ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ uint64_t n_warps() { return ((uint64_t)gridDim.x * blockDim.x) >> 5; }

__device__ __forceinline__ uint64_t warp_sum(uint64_t v) {
  for (int d = 16; d; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  return v;
}

// ---- phase 1: all neighbour pairs of each centre, classified as open --------

// Counter block of one output row: 30 closed classes, 6 open-pair classes
// removed by closed triangles, 6 open-pair counts (per-request rows of a
// pooled store use one block each).
constexpr unsigned kRowStride = 42;

// centres == nullptr: every slot 0..n-1 is a centre; else the n listed ones.
// With gos set, each centre's pairs go to row rog[gos[a]] of out6's blocks.
__global__ void __launch_bounds__(kOpenBlock) k_open_pairs(const uint64_t* __restrict__ off,
                                                           const uint32_t* __restrict__ len,
                                                           const uint32_t* __restrict__ nbr,
                                                           const uint8_t* __restrict__ ovl,
                                                           const uint8_t* __restrict__ esize,
                                                           const uint32_t* __restrict__ centres, uint32_t n,
                                                           uint32_t shard, uint32_t n_shards,
                                                           const uint32_t* __restrict__ gos,
                                                           const uint32_t* __restrict__ rog,
                                                           unsigned long long* __restrict__ out6) {
  __shared__ uint32_t hist[kOpenWarps][2][256];
  const unsigned w = threadIdx.x / kWarp, lane = lane_id();
  uint64_t acc[6] = {0, 0, 0, 0, 0, 0};  // lane 0's running class counts
  for (uint64_t i = shard + global_warp() * n_shards; i < n; i += n_warps() * n_shards) {
    const uint32_t a = centres ? centres[i] : (uint32_t)i;
    const uint32_t l = len[a];
    if (l < 2) continue;
    const uint32_t s = esize[a];
    for (uint32_t i = lane; i <= s; i += kWarp) {
      hist[w][0][i] = 0;
      hist[w][1][i] = 0;
    }
    __syncwarp();
    const uint64_t base = off[a];
    uint32_t one[2] = {0, 0};  // overlap-1 neighbours, the common case, kept in registers
    for (uint32_t i = lane; i < l; i += kWarp) {
      const uint32_t b = nbr[base + i];
      const uint32_t c = ovl[base + i];
      const uint32_t y = c < esize[b];
      if (c == 1) ++one[y];
      else atomicAdd(&hist[w][y][c], 1u);
    }
    for (int d = 16; d; d >>= 1) {
      one[0] += __shfl_xor_sync(0xffffffffu, one[0], d);
      one[1] += __shfl_xor_sync(0xffffffffu, one[1], d);
    }
    __syncwarp();
    if (lane == 0) {
      uint32_t* h0 = hist[w][0];
      uint32_t* h1 = hist[w][1];
      h0[1] += one[0];
      h1[1] += one[1];
      // in-place prefix sums: H_t[k] = #neighbours of type t with overlap <= k
      for (uint32_t k = 1; k <= s; ++k) {
        h0[k] += h0[k - 1];
        h1[k] += h1[k - 1];
      }
      open_pair_counts(h0, h1, s, acc, false);
      if (gos) {
        unsigned long long* o = out6 + (size_t)rog[gos[a]] * kRowStride;
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
      if (acc[k]) atomicAdd(&out6[k], (unsigned long long)acc[k]);
}

// ---- phase 2: closed triangles ------------------------------------------------

struct ClosedArgs {
  const uint64_t* poff;
  const uint32_t* plen;
  const uint32_t* pnbr;
  const uint16_t* pos;    // (neighbour size << 8) | overlap
  const uint32_t* rnbr;   // H2H neighbour ids (a centre's masks are looked up in its H2H row)
  const uint64_t* hoff;   // H2V
  const uint32_t* hmem;
  const uint8_t* esize;
  const uint32_t* work;  // centres, heaviest first
  uint32_t n_work;
  uint32_t shard, n_shards;  // this call takes work items shard, shard + n_shards, ...
  unsigned int* queue;
  unsigned long long* out;  // kNumCounters (rows of kRowStride with gos)
  uint8_t* edge_flags;      // diagnostics only: marks oriented entries that close a triangle
  const uint32_t* gos;      // per slot: its graph (null: one output row)
  const uint32_t* rog;      // per graph: output row
  // The grouped copy of the oriented rows walked as N+(b) (hm_graph::grp_nbr;
  // null: walk pnbr / pos, no group is skipped) and the (degree, id) rank.
  const uint32_t* wnbr;
  const uint16_t* wos;
  const uint64_t* wbase;
  const uint4* wtab;        // per group: {start in the row, size-1 neighbours, size-2 neighbours, 0}
  const uint8_t* wopos;     // per oriented entry (a, b), id-sorted: position in b of the one member
                            // a and b share, 0xff if they share several or it is past 63
  // H2H offsets, masks (the row owner's members < 64), lengths, overlaps
  const uint64_t* roff;
  const uint64_t* rmask;
  const uint32_t* rlen;
  const uint8_t* rovl;
  // masks of the oriented rows longer than kLongRow (hm_graph::long_off)
  const uint64_t* loff;
  const uint64_t* lmask;
};

constexpr uint32_t kGroupPositions = 64;

// |a & b & c| by a three-way merge of the member lists (centres with more
// than 64 members, whose position masks are incomplete).
__device__ uint32_t triple_overlap(const uint64_t* hoff, const uint32_t* hmem, const uint8_t* esize, uint32_t a,
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

__device__ __forceinline__ uint32_t hash_slot(uint32_t key, uint32_t shift) { return (key * 2654435761u) >> shift; }

// Size category used by the star fast path: 0 for |x| = 1, 1 for |x| = 2, 2
// for |x| >= 3 (the classes of a star triple only depend on these).
__device__ __forceinline__ uint32_t size_cat(uint32_t s) { return s >= 3 ? 2u : s - 1u; }

// Adds n triangles {a, b, c} whose three pairs share exactly one node, the
// same one (g = 1), with size categories ca, cb, cc: closed class = number of
// members with |x| >= 2; open-pair classes at each centre x as phase 1 gave
// them: [|x| >= 3] + 2 ([|y| >= 2] + [|z| >= 2]).
__device__ __forceinline__ void add_star(unsigned long long* wc, uint32_t ca, uint32_t cb, uint32_t cc,
                                         uint64_t n) {
  const uint32_t ea = ca > 0, eb = cb > 0, ec = cc > 0;
  wc[ea + eb + ec] += n;
  wc[30 + (ca == 2) + 2 * (eb + ec)] += n;
  wc[30 + (cb == 2) + 2 * (ea + ec)] += n;
  wc[30 + (cc == 2) + 2 * (ea + eb)] += n;
}

// The table of one centre's oriented row: bucketized keys (4 per 16-byte
// bucket), each key's overlap with the centre and shared-position mask (or
// its row index, for the diagnostic pass). Rows too long for it are searched
// in global memory instead.
// One value per key: the shared-position mask when the centre has at most 64
// members (its overlap is then the mask's popcount), else the overlap; the
// row index in the diagnostic pass.
// With skip set (a centre of at most 64 members, grouped rows to walk), the
// walk of N+(b) for a b sharing a single member u with a may leave out b's
// group of neighbours sharing only u: when no neighbour in N+(a) shares two
// or more members with a including u (bit u of heavy_or clear), every entry
// of that group is a star triangle {a, b, c}, counted per size category from
// the group's counts.
struct CentreTable {
  const uint32_t* keys;
  const uint64_t* sval;
  uint32_t shift, bmask;
  bool in_smem;
  uint64_t heavy_or;  // OR of the shared-position masks of a's heavy neighbours in N+(a)
  bool skip;
};

__device__ __forceinline__ void table_insert(uint32_t* keys, uint64_t* sval, uint32_t shift, uint32_t bmask,
                                             uint32_t key, uint64_t value) {
  uint32_t bk = hash_slot(key, shift), h = 0;
  for (bool done = false; !done; bk = (bk + 1) & bmask)
    for (uint32_t t = 0; t < 4; ++t)
      if (atomicCAS(&keys[4 * bk + t], kEmpty, key) == kEmpty) {
        h = 4 * bk + t;
        done = true;
        break;
      }
  sval[h] = value;
}

// Fills the table with N+(a), threads t = first, first + stride, ...; the
// masks of the entries sharing two or more members with a are ORed into
// *heavy_or (when given). Counts read N+(a) from a's H2H row, the entries
// ranked above a (the oriented rows' own rule), so each entry's overlap and
// mask come with it. Diagnostics (flags) read the oriented row and store each
// entry's index.
__device__ __forceinline__ void fill_table(const ClosedArgs& A, uint32_t a, uint64_t ao, uint32_t ad,
                                           uint32_t* keys, uint64_t* sval, uint32_t shift, uint32_t bmask,
                                           bool flags, bool exact, unsigned first, unsigned stride,
                                           unsigned long long* heavy_or) {
  if (flags) {
    for (uint32_t i = first; i < ad; i += stride) table_insert(keys, sval, shift, bmask, A.pnbr[ao + i], i);
    return;
  }
  const uint64_t ro = A.roff[a];
  const uint32_t rd = A.rlen[a];
  for (uint32_t i = first; i < rd; i += stride) {
    const uint32_t key = __ldg(A.rnbr + ro + i);
    if (!rank_above(a, rd, key, __ldg(A.rlen + key))) continue;
    const uint32_t ov = __ldg(A.rovl + ro + i);
    const uint64_t m = exact ? __ldg(A.rmask + ro + i) : 0;
    table_insert(keys, sval, shift, bmask, key, exact ? m : (uint64_t)ov);
    if (heavy_or && exact && ov >= 2u) atomicOr(heavy_or, (unsigned long long)m);
  }
}

// The value the centre's shared table holds for key, a member of N+(a) (so
// present; the probe is bounded by the table size all the same, and a key
// not found has its mask read from the H2H row).
__device__ __forceinline__ uint64_t table_value(const ClosedArgs& A, const CentreTable& T, uint32_t a, uint32_t key) {
  uint32_t bk = hash_slot(key, T.shift);
  for (uint32_t n = 0; n <= T.bmask; ++n) {
    const uint4 q = reinterpret_cast<const uint4*>(T.keys)[bk];
    const int t = q.x == key ? 0 : q.y == key ? 1 : q.z == key ? 2 : q.w == key ? 3 : -1;
    if (t >= 0) return T.sval[4 * bk + (uint32_t)t];
    bk = (bk + 1) & T.bmask;
  }
  return row_mask(A.roff, A.rlen, A.rnbr, A.rmask, a, key);
}

// Whole warp, converged: the lanes with push set append their record to the
// warp's queue (64 places); every full 32 are classified at once.
__device__ __forceinline__ void queue_push(bool push, uint64_t rec, uint64_t* q, uint32_t& qn, uint32_t sa,
                                           unsigned long long* wc) {
  const unsigned lane = lane_id();
  const unsigned bal = __ballot_sync(0xffffffffu, push);
  if (push) q[qn + __popc(bal & ((1u << lane) - 1u))] = rec;
  qn += (uint32_t)__popc(bal);
  if (qn >= kWarp) {
    __syncwarp();
    classify_queue(q, kWarp, sa, wc);
    if (lane < qn - kWarp) q[lane] = q[kWarp + lane];
    __syncwarp();
    qn -= kWarp;
  }
}

// One whole warp: walks N+(b) for the bi-th entry b of N+(a), probes the
// centre's table, and adds every triangle {a, b, c} it closes to wc. For a
// centre with at most 64 members g = |a & b & c| = popc(mask_ab & mask_ac)
// exactly. Star triangles (all three overlaps 1, the same shared node) are
// only counted per size category in registers; the others are classified and
// their four counter updates aggregated across the lanes that share them.
// kTriads: instead of classes, wc[0] collects sum x * y * z over the
// triangles, x, y, z the pairwise overlaps minus the triple overlap (all > 0;
// star triangles give 0), the reference's type-3 vertex triads.
template <bool kTriads>
// Closed triangles that are not stars go to the warp's queue q (qn records,
// warp-uniform); every 32 of them are classified together, at full width.
__device__ __forceinline__ void closed_pairs_of_b(const ClosedArgs& A, uint32_t a, uint32_t sa, uint64_t ao,
                                                  uint32_t ad, uint32_t bi, const CentreTable& T,
                                                  unsigned long long* wc, uint32_t cat_a, bool exact_masks,
                                                  bool flags, uint64_t* q, uint32_t& qn) {
  const unsigned lane = lane_id();
  const uint32_t b = A.pnbr[ao + bi];
  const uint32_t osb = A.pos[ao + bi];
  const uint32_t cab = osb & 0xffu, sb = osb >> 8;
  // the mask of (a, b): from the centre's table (it holds masks when a has at
  // most 64 members), else from a's H2H row
  const uint64_t mab = !exact_masks              ? 0
                       : (T.in_smem && !flags) ? table_value(A, T, a, b)
                                               : row_mask(A.roff, A.rlen, A.rnbr, A.rmask, a, b);
  const uint64_t bo = A.poff[b];
  const uint32_t bd = A.plen[b];
  // N+(b) is walked in its grouped copy when there is one (any order of a
  // row's entries finds the same triangles); the diagnostic pass walks the
  // id-sorted rows, whose entry indices it records.
  const bool grouped = A.wnbr != nullptr && !flags;
  const uint32_t* wnbr = grouped ? A.wnbr : A.pnbr;
  const uint16_t* wos = grouped ? A.wos : A.pos;
  uint32_t star0 = 0, star1 = 0, star2 = 0;
  unsigned long long triads = 0;
  // The group of b's neighbours whose only shared member with b is u, the
  // only member a and b share, is left out of the walk when no heavy
  // neighbour of a contains u: each c of the group closes a triangle
  // {a, b, c} through u and shares only u with a as well (a heavy one would
  // be in N+(a), ranked above b), so all are stars, counted by the size of c
  // (lane 0 holds the group's counts).
  uint32_t gs = 0, glen = 0;
  if (!kTriads && T.skip && grouped && cab == 1) {
    const uint32_t qu = (uint32_t)(__ffsll((long long)mab) - 1);  // u's position in a (a has <= 64 members)
    const uint32_t pb = A.wopos[ao + bi];                        // u's position in b
    if (!((T.heavy_or >> qu) & 1ull) && pb < kGroupPositions) {
      const uint64_t t = A.wbase[b] + 1 + pb;
      const uint4 g0 = A.wtab[t], g1 = A.wtab[t + 1];
      gs = g0.x;
      glen = g1.x - g0.x;
      if (lane == 0) {
        star0 = g0.y;
        star1 = g0.z;
        star2 = glen - g0.y - g0.z;
      }
    }
  }
  const uint32_t bdw = bd - glen;  // entries walked
  // kUnroll probes per lane per round: their id and overlap/size loads are
  // issued together, and the next round's before this round's probes, so
  // that the walk's global loads overlap the probing (software pipelining).
  uint32_t cv[kUnroll], ov[kUnroll];
#pragma unroll
  for (unsigned u = 0; u < kUnroll; ++u) {
    const uint32_t j = u * kWarp + lane;
    cv[u] = kEmpty;
    ov[u] = 0;
    if (j < bdw) {
      const uint32_t jj = j < gs ? j : j + glen;
      cv[u] = __ldg(wnbr + bo + jj);
      ov[u] = __ldg(wos + bo + jj);
    }
  }
  for (uint32_t j0 = 0; j0 < bdw; j0 += kWarp * kUnroll) {
    uint32_t cn[kUnroll], on[kUnroll];
#pragma unroll
    for (unsigned u = 0; u < kUnroll; ++u) {
      const uint32_t j = j0 + kWarp * kUnroll + u * kWarp + lane;
      cn[u] = kEmpty;
      on[u] = 0;
      if (j < bdw) {
        const uint32_t jj = j < gs ? j : j + glen;
        cn[u] = __ldg(wnbr + bo + jj);
        on[u] = __ldg(wos + bo + jj);
      }
    }
#pragma unroll
    for (unsigned u = 0; u < kUnroll; ++u) {
      const uint32_t c = cv[u];
      bool push = false;
      uint64_t rec = 0;
      do {
      if (c == kEmpty) break;
      uint32_t cac = 0;
      uint64_t mac = 0;
      if (T.in_smem) {
        uint32_t bk = hash_slot(c, T.shift);
        int t;
        for (;;) {
          const uint4 q = reinterpret_cast<const uint4*>(T.keys)[bk];
          t = q.x == c ? 0 : q.y == c ? 1 : q.z == c ? 2 : q.w == c ? 3 : -1;
          if (t >= 0 || q.w == kEmpty) break;
          bk = (bk + 1) & T.bmask;
        }
        if (t >= 0) {
          const uint64_t v = T.sval[4 * bk + (uint32_t)t];
          if (flags) {
            const uint32_t j = j0 + u * kWarp + lane;
            A.edge_flags[ao + v] = 1;
            A.edge_flags[ao + bi] = 1;
            A.edge_flags[bo + j] = 1;
            cac = A.pos[ao + v] & 0xffu;
            mac = row_mask(A.roff, A.rlen, A.rnbr, A.rmask, a, c);
          } else if (exact_masks) {
            mac = v;
            cac = (uint32_t)__popcll(v);
          } else {
            cac = (uint32_t)v;
          }
        }
      } else {
        // rows too long for the table (longer than kLongRow: every kernel
        // tables all rows shorter than that it can be given): a search of
        // N+(a), whose masks are kept beside it
        uint32_t lo = 0, hi = ad;
        const uint32_t* row = A.pnbr + ao;
        while (lo < hi) {
          const uint32_t mid = (lo + hi) >> 1;
          if (row[mid] < c) lo = mid + 1;
          else hi = mid;
        }
        if (lo < ad && row[lo] == c) {
          cac = A.pos[ao + lo] & 0xffu;
          mac = exact_masks ? A.lmask[A.loff[a] + lo] : 0;
          if (flags) {
            const uint32_t j = j0 + u * kWarp + lane;
            A.edge_flags[ao + lo] = 1;
            A.edge_flags[ao + bi] = 1;
            A.edge_flags[bo + j] = 1;
          }
        }
      }
      if (!cac) break;
      const uint32_t cbc = ov[u] & 0xffu, sc = ov[u] >> 8;
      uint32_t g;
      if (exact_masks) {
        if ((cab | cac | cbc) == 1 && mab == mac) {
          if (!kTriads) {
            const uint32_t cc = size_cat(sc);
            star0 += cc == 0;
            star1 += cc == 1;
            star2 += cc == 2;
          }
          break;
        }
        g = __popcll(mab & mac);
      } else {
        g = triple_overlap(A.hoff, A.hmem, A.esize, a, b, c);
      }
      if (kTriads) {
        if (cab > g && cbc > g && cac > g) triads += (unsigned long long)(cab - g) * (cbc - g) * (cac - g);
        break;
      }
      push = true;
      rec = pack_triangle(sb, sc, cab, cbc, cac, g);
      } while (false);
      if (!kTriads) queue_push(push, rec, q, qn, sa, wc);  // warp-converged
    }
#pragma unroll
    for (unsigned u = 0; u < kUnroll; ++u) {
      cv[u] = cn[u];
      ov[u] = on[u];
    }
  }
  if (kTriads) {
    for (int d = 16; d; d >>= 1) triads += __shfl_xor_sync(0xffffffffu, triads, d);
    if (lane == 0 && triads) wc[0] += triads;
    return;
  }
  if (cab == 1 && exact_masks) {
    for (int d = 16; d; d >>= 1) {
      star0 += __shfl_xor_sync(0xffffffffu, star0, d);
      star1 += __shfl_xor_sync(0xffffffffu, star1, d);
      star2 += __shfl_xor_sync(0xffffffffu, star2, d);
    }
    if (lane == 0) {
      const uint32_t cat_b = size_cat(sb);
      if (star0) add_star(wc, cat_a, cat_b, 0, star0);
      if (star1) add_star(wc, cat_a, cat_b, 1, star1);
      if (star2) add_star(wc, cat_a, cat_b, 2, star2);
    }
  }
}

// Adds one warp's counters to output row `row` and clears them.
__device__ __forceinline__ void flush_counts(unsigned long long* wc, unsigned long long* out) {
  for (unsigned k = lane_id(); k < kNumCounters; k += kWarp)
    if (wc[k]) {
      atomicAdd(&out[k], wc[k]);
      wc[k] = 0;
    }
  __syncwarp();
}

constexpr uint32_t kNoRow = 0xffffffffu;

// One block per centre a (the lowest-ranked corner of its triangles): N+(a)
// in a shared-memory table (load <= 1/4 up to kHashSlotsMax / 2 entries,
// else searched in global memory), each warp takes one b in N+(a) at a time.
template <unsigned kHashSlotsMax, unsigned kMinBlocks, bool kTriads = false, unsigned kThreads = kClosedBlock>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_closed(ClosedArgs A) {
  constexpr unsigned kWarpsB = kThreads / kWarp;
  static_assert(kHashSlotsMax % 4 == 0, "whole buckets");
  constexpr unsigned kHashRowMax = kHashSlotsMax / 2;
  // rows not tabled must have their masks kept (longer than kLongRow), or
  // never reach this shape (the schedule sends it rows up to kSmallRow)
  static_assert(kHashRowMax == kLongRow || kHashRowMax >= kSmallRow, "untabled rows without masks");
  extern __shared__ uint64_t smem64[];
  uint64_t* sval = smem64;                                             // kHashSlotsMax
  uint32_t* keys = reinterpret_cast<uint32_t*>(sval + kHashSlotsMax);  // kHashSlotsMax
  __shared__ unsigned long long wcnt[kWarpsB][kNumCounters];
  __shared__ uint64_t wqueue[kWarpsB][2 * kWarp];  // per warp: triangles waiting to be classified
  __shared__ unsigned long long s_heavy;
  __shared__ uint32_t s_item;
  const unsigned w = threadIdx.x / kWarp, lane = lane_id();
  unsigned long long* wc = wcnt[w];
  uint64_t* q = wqueue[w];
  uint32_t qn = 0;
  for (unsigned k = lane; k < kNumCounters; k += kWarp) wc[k] = 0;
  uint32_t cur_row = kNoRow;  // per-request rows: the row wc is collecting for

  for (;;) {
    if (threadIdx.x == 0) {
      s_item = atomicAdd(A.queue, 1u);
      s_heavy = 0;
    }
    __syncthreads();
    const uint64_t item = (uint64_t)s_item * A.n_shards + A.shard;
    if (item >= A.n_work) break;
    const uint32_t a = A.work[item];
    if (A.gos) {
      const uint32_t row = A.rog[A.gos[a]];
      if (row != cur_row) {
        if (cur_row != kNoRow) flush_counts(wc, A.out + (size_t)cur_row * kRowStride);
        cur_row = row;
      }
    }
    const uint64_t ao = A.poff[a];
    const uint32_t ad = A.plen[a];
    const uint32_t sa = A.esize[a];
    const bool flags = A.edge_flags != nullptr;
    CentreTable T{keys, sval, 32, 0, ad <= kHashRowMax, 0, false};
    if (T.in_smem) {
      uint32_t slots = 64;
      while (slots < 4 * ad && slots < kHashSlotsMax) slots <<= 1;
      const uint32_t buckets = slots / 4;
      T.shift = 32 - (31 - __clz(buckets));
      T.bmask = buckets - 1;
      for (uint32_t i = threadIdx.x; i < slots; i += blockDim.x) keys[i] = kEmpty;
      __syncthreads();
      fill_table(A, a, ao, ad, keys, sval, T.shift, T.bmask, flags, sa <= 64, threadIdx.x,
                 blockDim.x, &s_heavy);
    }
    __syncthreads();
    const uint32_t cat_a = size_cat(sa);
    const bool exact_masks = sa <= 64;
    T.heavy_or = s_heavy;
    T.skip = T.in_smem && exact_masks && !flags && A.wnbr;
    for (uint32_t bi = w; bi < ad; bi += kWarpsB) {
      closed_pairs_of_b<kTriads>(A, a, sa, ao, ad, bi, T, wc, cat_a, exact_masks, flags, q, qn);
      __syncwarp();
    }
    if (qn) {  // the centre's last triangles (classes depend on |a|)
      classify_queue(q, qn, sa, wc);
      qn = 0;
    }
    __syncthreads();
  }
  __syncwarp();
  flush_counts(wc, A.out + (cur_row == kNoRow ? 0 : (size_t)cur_row * kRowStride));
}

// One warp per centre, for short oriented rows (<= warp_row <= kWarpRow): each warp
// holds its own table (load <= 1/2) and walks all of N+(a) itself, with no
// block-wide barriers; warps take centres from the queue one at a time.
template <bool kTriads = false>
__global__ void __launch_bounds__(kClosedBlock, 4) k_closed_warp(ClosedArgs A) {
  __shared__ __align__(16) uint32_t keys_all[kClosedWarps][kWarpSlots];
  __shared__ uint64_t val_all[kClosedWarps][kWarpSlots];
  __shared__ unsigned long long wcnt[kClosedWarps][kNumCounters];
  __shared__ uint64_t wqueue[kClosedWarps][2 * kWarp];
  __shared__ unsigned long long heavy_all[kClosedWarps];
  const unsigned w = threadIdx.x / kWarp, lane = lane_id();
  uint32_t* keys = keys_all[w];
  uint64_t* sval = val_all[w];
  unsigned long long* wc = wcnt[w];
  uint64_t* q = wqueue[w];
  uint32_t qn = 0;
  for (unsigned k = lane; k < kNumCounters; k += kWarp) wc[k] = 0;
  __syncwarp();
  uint32_t cur_row = kNoRow;
  const bool flags = A.edge_flags != nullptr;
  for (;;) {
    uint32_t it = 0;
    if (lane == 0) it = atomicAdd(A.queue, 1u);
    it = __shfl_sync(0xffffffffu, it, 0);
    const uint64_t item = (uint64_t)it * A.n_shards + A.shard;
    if (item >= A.n_work) break;
    const uint32_t a = A.work[item];
    if (A.gos) {
      const uint32_t row = A.rog[A.gos[a]];
      if (row != cur_row) {
        if (cur_row != kNoRow) flush_counts(wc, A.out + (size_t)cur_row * kRowStride);
        cur_row = row;
      }
    }
    const uint64_t ao = A.poff[a];
    const uint32_t ad = A.plen[a];  // <= warp_row <= kWarpRow by the work split
    const uint32_t sa = A.esize[a];
    uint32_t slots = 64;
    while (slots < 2 * ad && slots < kWarpSlots) slots <<= 1;
    const uint32_t buckets = slots / 4;
    CentreTable T{keys, sval, 32u - (31u - (uint32_t)__clz(buckets)), buckets - 1, true, 0, false};
    for (uint32_t i = lane; i < slots; i += kWarp) keys[i] = kEmpty;
    if (lane == 0) heavy_all[w] = 0;
    __syncwarp();
    fill_table(A, a, ao, ad, keys, sval, T.shift, T.bmask, flags, sa <= 64, lane, kWarp,
               &heavy_all[w]);
    __syncwarp();
    const uint32_t cat_a = size_cat(sa);
    const bool exact_masks = sa <= 64;
    T.heavy_or = heavy_all[w];
    T.skip = exact_masks && !flags && A.wnbr;
    for (uint32_t bi = 0; bi < ad; ++bi) {
      closed_pairs_of_b<kTriads>(A, a, sa, ao, ad, bi, T, wc, cat_a, exact_masks, flags, q, qn);
      __syncwarp();
    }
    if (qn) {
      classify_queue(q, qn, sa, wc);
      qn = 0;
    }
  }
  __syncwarp();
  flush_counts(wc, A.out + (cur_row == kNoRow ? 0 : (size_t)cur_row * kRowStride));
}

// Work estimate per centre: sum of d+(b) over b in N+(a); centres with fewer
// than two oriented neighbours own no triangle and are dropped (key 0). Key
// layout: bit 63 = row longer than small_row (large-table launch), bit 62 =
// row longer than warp_row (block launch; warp_row <= small_row, so the
// large-table rows carry it too), then the estimate; descending
// order gives the three launches' lists, heaviest first. With gos set
// (per-request rows of a pooled store) bits 40..61 hold the output row of the
// centre's graph above a 40-bit estimate, so that the blocks running at one
// time share one graph's rows in L2.
__global__ void k_closed_work(const uint64_t* poff, const uint32_t* plen, const uint32_t* pnbr, const uint32_t* rows,
                              uint32_t n, const uint32_t* gos, const uint32_t* rog, ClosedSchedule sched,
                              uint64_t* est, uint32_t* ids) {
  for (uint64_t r = global_warp(); r < n; r += n_warps()) {
    const uint32_t a = rows ? rows[r] : (uint32_t)r;
    const uint32_t d = plen[a];
    uint64_t s = 0;
    if (d >= 2)
      for (uint32_t i = lane_id(); i < d; i += kWarp) s += plen[pnbr[poff[a] + i]];
    s = warp_sum(s);
    if (lane_id() == 0) {
      uint64_t key = 0;
      if (d >= 2 && s > 0) {
        const uint64_t e = s + d;
        if (gos)
          key = ((uint64_t)min(rog[gos[a]], (1u << 22) - 1u) << 40) | (e < (1ull << 40) ? e : (1ull << 40) - 1);
        else
          key = e < (1ull << 62) ? e : (1ull << 62) - 1;
        if (d > sched.warp_row) key |= 1ull << 62;
        if (d > sched.small_row) key |= 1ull << 63;
      }
      est[r] = key;
      ids[r] = a;
    }
  }
}

}  // namespace

constexpr size_t closed_smem_bytes(unsigned slots) { return (sizeof(uint64_t) + sizeof(uint32_t)) * slots; }
// Rows longer than small_row: one 1024-thread block per SM with a
// 16384-slot table (rows up to 8192 entries in shared memory).
constexpr unsigned kBigSlots = 16384, kSmallSlots = 4096, kBigThreads = 1024;

// Centres that own at least one oriented wedge, heaviest first.
static int closed_worklist(hm_graph* g) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  const uint32_t E = g->n_slots;
  DArr<uint64_t> est, est_sorted;
  DArr<uint32_t> ids;
  HM_TRY(est.alloc(ctx, E));
  HM_TRY(est_sorted.alloc(ctx, E));
  HM_TRY(ids.alloc(ctx, E));
  HM_TRY(g->work.alloc(ctx, E));
  k_closed_work<<<grid_for((uint64_t)E * 32, 256), 256, 0, st>>>(g->plus_off.p, g->plus_len.p, g->plus_nbr.p,
                                                                nullptr, E, nullptr, nullptr, g->sched, est.p, ids.p);
  HM_LAUNCH_CHECK();
  size_t tb = 0;
  HM_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, est.p, est_sorted.p, ids.p, g->work.p, (int64_t)E,
                                                    0, 64, st));
  DArr<uint8_t> tmp;
  HM_TRY(tmp.alloc(ctx, tb));
  HM_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.p, tb, est.p, est_sorted.p, ids.p, g->work.p, (int64_t)E, 0,
                                                    64, st));
  // the number of non-zero estimates is the first zero of the descending list
  std::vector<uint64_t> h(E);
  HM_CUDA(cudaMemcpyAsync(h.data(), est_sorted.p, sizeof(uint64_t) * E, cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  uint32_t lo = 0, hi = E;
  while (lo < hi) {
    uint32_t mid = (lo + hi) / 2;
    if (h[mid] > 0) lo = mid + 1;
    else hi = mid;
  }
  g->n_work = lo;
  lo = 0;
  hi = g->n_work;
  while (lo < hi) {
    uint32_t mid = (lo + hi) / 2;
    if (h[mid] >> 63) lo = mid + 1;
    else hi = mid;
  }
  g->n_work_big = lo;
  hi = g->n_work;  // rows longer than warp_row carry bit 62 (the big ones too)
  while (lo < hi) {
    uint32_t mid = (lo + hi) / 2;
    if ((h[mid] >> 62) & 1u) lo = mid + 1;
    else hi = mid;
  }
  g->n_work_mid = lo;
  g->work_valid = true;
  return HM_OK;
}

static int prepare_static_attrs() {
  static bool attr_set = false;
  if (!attr_set) {
    HM_CUDA(cudaFuncSetAttribute(k_closed<kBigSlots, 1, false, kBigThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)closed_smem_bytes(kBigSlots)));
    HM_CUDA(cudaFuncSetAttribute(k_closed<kSmallSlots, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)closed_smem_bytes(kSmallSlots)));
    HM_CUDA(cudaFuncSetAttribute(k_closed<kBigSlots, 1, true, kBigThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)closed_smem_bytes(kBigSlots)));
    HM_CUDA(cudaFuncSetAttribute(k_closed<kSmallSlots, 4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)closed_smem_bytes(kSmallSlots)));
    attr_set = true;
  }
  return HM_OK;
}

// The grouped rows and the rank the closed phase's walk uses (left null,
// the walk takes the id-sorted rows and skips nothing).
static void with_masks(const hm_graph* g, ClosedArgs& A) {
  A.rnbr = g->h2h_nbr.p;
  A.roff = g->h2h_off.p;
  A.rmask = g->h2h_mask.p;
  A.rlen = g->h2h_len.p;
  A.rovl = g->h2h_ovl.p;
  A.loff = g->long_off.p;
  A.lmask = g->long_mask.p;
}

static void with_groups(const hm_graph* g, ClosedArgs& A) {
  with_masks(g, A);
  if (!g->use_groups || !g->grp_valid) return;
  A.wnbr = g->grp_nbr.p;
  A.wos = g->grp_os.p;
  A.wbase = g->grp_base.p;
  A.wtab = g->grp_tab.p;
  A.wopos = g->grp_opos.p;
}

// Everything the count kernels need that only changes with the graph.
int prepare_static(hm_graph* g) {
  hm_ctx* ctx = g->ctx;
  if (!g->plus_valid) {
    HM_TRY(build_plus(g));
    g->work_valid = false;
  }
  if (g->use_groups && !g->grp_valid) {
    // the grouped rows are a shortcut: without room for them the count walks
    // the oriented rows in full
    const int s = build_plus_groups(g);
    if (s == HM_ERR_NOMEM) release_plus_groups(g);
    else HM_TRY(s);
  }
  if (!g->work_valid && g->n_slots) HM_TRY(closed_worklist(g));
  if (!g->counters.p) HM_TRY(g->counters.alloc(ctx, 64));
  if (!g->ev_ready) {
    for (auto& e : g->ev) HM_CUDA(cudaEventCreate(&e));
    g->ev_ready = true;
  }
  return prepare_static_attrs();
}

// The closed phase over a work list split at bounds[0..3]: rows longer than
// small_row (16384-slot tables, one 1024-thread block per SM; 8192-slot
// tables at 2 blocks of 256 took 9 % longer per count at config 2), rows longer than warp_row
// (4096-slot tables, 4 blocks per SM), then the short rows, one warp each.
// queues holds three zeroed counters, one per launch.
template <bool kTriads = false>
static int launch_closed(hm_ctx* ctx, ClosedArgs base, const uint32_t bounds[4], unsigned int* queues) {
  cudaStream_t st = ctx->stream;
  for (int part = 0; part < 3; ++part) {
    const uint32_t n = bounds[part + 1] - bounds[part];
    if (n <= base.shard) continue;
    ClosedArgs A = base;
    A.work = base.work + bounds[part];
    A.n_work = n;
    A.queue = queues + part;
    const uint32_t items = (n - base.shard + base.n_shards - 1) / base.n_shards;
    if (part == 0) {
      const unsigned grid = std::min<unsigned>((unsigned)ctx->n_sms, items);
      k_closed<kBigSlots, 1, kTriads, kBigThreads><<<grid, kBigThreads, closed_smem_bytes(kBigSlots), st>>>(A);
    } else if (part == 1) {
      const unsigned grid = std::min<unsigned>((unsigned)ctx->n_sms * 4, items);
      k_closed<kSmallSlots, 4, kTriads><<<grid, kClosedBlock, closed_smem_bytes(kSmallSlots), st>>>(A);
    } else {
      const unsigned grid = std::min<unsigned>((unsigned)ctx->n_sms * 4, (items + kClosedWarps - 1) / kClosedWarps);
      k_closed_warp<kTriads><<<grid, kClosedBlock, 0, st>>>(A);
    }
    HM_LAUNCH_CHECK();
  }
  return HM_OK;
}

// Captures the launches body() makes on stream st as an executable graph.
template <class F>
static int capture_graph(cudaStream_t st, F&& body, cudaGraphExec_t* exec) {
  HM_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  const int s = body();
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(st, &graph);
  if (s < 0 || e != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    if (s < 0) return s;
    return set_error(HM_ERR_CUDA, "stream capture of the static count: %s", cudaGetErrorString(e));
  }
  const cudaError_t ei = cudaGraphInstantiate(exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ei != cudaSuccess) {
    *exec = nullptr;
    return set_error(HM_ERR_CUDA, "graph instantiation of the static count: %s", cudaGetErrorString(ei));
  }
  return HM_OK;
}

// Launches both phases for one shard of the centres; the counters land in
// g->counters ([0,30) closed classes, [30,36) open-pair removals, [36,42)
// open-pair counts, [42..44] work queues). edge_flags is for diagnostics.
// Each phase is captured once as a CUDA graph and replayed while everything
// its launches were captured with (store and work-list arrays, the split,
// the shard) is unchanged; the diagnostic form launches directly.
int launch_static(hm_graph* g, uint32_t shard, uint32_t n_shards, uint8_t* edge_flags) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  const uint32_t E = g->n_slots;
  unsigned long long* dev = g->counters.p;
  const uint32_t bounds[4] = {0, g->n_work_big, g->n_work_mid, g->n_work};
  ClosedArgs args{g->plus_off.p, g->plus_len.p, g->plus_nbr.p, g->plus_os.p, g->h2h_nbr.p,
                  g->h2v_off.p,  g->h2v_mem.p,  g->esize.p,    g->work.p,    0,
                  shard,         n_shards,      nullptr,       dev,          edge_flags,
                  nullptr,       nullptr};
  with_groups(g, args);
  auto open_phase = [&]() -> int {
    HM_CUDA(cudaMemsetAsync(dev, 0, sizeof(unsigned long long) * 48, st));
    if (E) {
      k_open_pairs<<<(unsigned)ctx->n_sms * 8, kOpenBlock, 0, st>>>(g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p,
                                                                   g->h2h_ovl.p, g->esize.p, nullptr, E, shard,
                                                                   n_shards, nullptr, nullptr, dev + 36);
      HM_LAUNCH_CHECK();
    }
    return HM_OK;
  };
  auto closed_phase = [&]() -> int {
    return launch_closed(ctx, args, bounds, reinterpret_cast<unsigned int*>(dev + 42));
  };
  if (edge_flags) {
    HM_CUDA(cudaEventRecord(g->ev[0], st));
    HM_TRY(open_phase());
    HM_CUDA(cudaEventRecord(g->ev[1], st));
    HM_TRY(closed_phase());
    HM_CUDA(cudaEventRecord(g->ev[2], st));
    return HM_OK;
  }
  const uint64_t key[CountCapture::kKey] = {
      (uint64_t)g->h2h_off.p,  (uint64_t)g->h2h_len.p,  (uint64_t)g->h2h_nbr.p,   (uint64_t)g->h2h_ovl.p,
      (uint64_t)g->esize.p,    (uint64_t)g->plus_off.p, (uint64_t)g->plus_len.p,  (uint64_t)g->plus_nbr.p,
      (uint64_t)g->plus_os.p,  (uint64_t)g->h2h_nbr.p, (uint64_t)g->h2v_off.p,  (uint64_t)g->h2v_mem.p,
      (uint64_t)g->work.p,     (uint64_t)dev,            E,                       g->n_work,
      g->n_work_big,           g->n_work_mid,            shard,                   n_shards,
      (uint64_t)args.wnbr,     (uint64_t)args.wos,       (uint64_t)args.wbase,    (uint64_t)args.wtab,
      (uint64_t)args.wopos,    (uint64_t)g->h2h_mask.p,  0};
  CountCapture& C = g->capture;
  bool same = C.valid;
  for (unsigned k = 0; k < CountCapture::kKey && same; ++k) same = C.key[k] == key[k];
  if (!same) {
    C.reset();
    HM_TRY(capture_graph(st, open_phase, &C.exec[0]));
    bool any_closed = false;
    for (int part = 0; part < 3; ++part) any_closed = any_closed || bounds[part + 1] - bounds[part] > shard;
    if (any_closed) HM_TRY(capture_graph(st, closed_phase, &C.exec[1]));
    for (unsigned k = 0; k < CountCapture::kKey; ++k) C.key[k] = key[k];
    C.valid = true;
  }
  HM_CUDA(cudaEventRecord(g->ev[0], st));
  HM_CUDA(cudaGraphLaunch(C.exec[0], st));
  HM_CUDA(cudaEventRecord(g->ev[1], st));
  if (C.exec[1]) HM_CUDA(cudaGraphLaunch(C.exec[1], st));
  HM_CUDA(cudaEventRecord(g->ev[2], st));
  return HM_OK;
}

namespace {
// The 30 classes from the counter block: closed classes, plus the open-pair
// counts minus the removals closed triangles made (as finish_static).
__global__ void k_finish30(const unsigned long long* c, uint64_t* out30) {
  const unsigned k = threadIdx.x;
  if (k < 30) out30[k] = c[k] + (k >= 20 && k < 26 ? c[36 + k - 20] - c[30 + k - 20] : 0ull);
}
}  // namespace

// One count queued after `user` (a null handle is CUDA's legacy default
// stream, as everywhere in the runtime API), its classes written to d_out30,
// no host wait once the graph is prepared. The launches run on the context
// stream, ordered after `user` and before its later work by two events.
int count_static30_async(hm_graph* g, uint64_t* d_out30, cudaStream_t user) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  // The first count of a graph captures its launches as CUDA graphs on the
  // context stream and may wait on it; neither works inside a capture that
  // the event below would pull the context stream into.
  for (cudaStream_t s : {user, st}) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const cudaError_t e = cudaStreamIsCapturing(s, &cs);
    if (e != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
      cudaGetLastError();
      return set_error(HM_ERR_STATE, "async static count: the stream is being captured into a CUDA graph (%s); "
                       "call it outside the capture", e != cudaSuccess ? cudaGetErrorString(e) : "active");
    }
  }
  HM_TRY(prepare_static(g));
  // hm_graph_timings reports synchronous counts only; an asynchronous count
  // is not waited for, so its phase times are marked as not measured.
  g->times.open_ms = g->times.closed_ms = g->times.total_ms = -1.0f;
  const bool other = user != st;
  cudaEvent_t e[2] = {nullptr, nullptr};
  auto release = [&]() {
    for (auto x : e)
      if (x) cudaEventDestroy(x);  // released once the recorded work completes
  };
  if (other) {
    cudaError_t r = cudaEventCreateWithFlags(&e[0], cudaEventDisableTiming);
    if (r == cudaSuccess) r = cudaEventCreateWithFlags(&e[1], cudaEventDisableTiming);
    if (r == cudaSuccess) r = cudaEventRecord(e[0], user);
    if (r == cudaSuccess) r = cudaStreamWaitEvent(st, e[0], 0);
    if (r != cudaSuccess) {
      release();
      return set_error(HM_ERR_CUDA, "async static count: ordering after the caller's stream: %s",
                       cudaGetErrorString(r));
    }
  }
  int rc = launch_static(g, 0, 1, nullptr);
  if (rc >= 0) {
    k_finish30<<<1, 32, 0, st>>>(g->counters.p, d_out30);
    const cudaError_t r = cudaGetLastError();
    if (r != cudaSuccess) rc = set_error(HM_ERR_CUDA, "async static count: %s", cudaGetErrorString(r));
  }
  if (rc >= 0 && other) {
    cudaError_t r = cudaEventRecord(e[1], st);
    if (r == cudaSuccess) r = cudaStreamWaitEvent(user, e[1], 0);
    if (r != cudaSuccess) rc = set_error(HM_ERR_CUDA, "async static count: ordering the caller's stream: %s",
                                         cudaGetErrorString(r));
  }
  release();
  return rc;
}

int finish_static(hm_graph* g, uint64_t out30[30]) {
  unsigned long long h[44];
  cudaStream_t st = g->ctx->stream;
  HM_CUDA(cudaMemcpyAsync(h, g->counters.p, sizeof(h), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  float t_open = 0, t_closed = 0;
  cudaEventElapsedTime(&t_open, g->ev[0], g->ev[1]);
  cudaEventElapsedTime(&t_closed, g->ev[1], g->ev[2]);
  g->times.open_ms = t_open;
  g->times.closed_ms = t_closed;
  g->times.total_ms = t_open + t_closed;
  uint64_t tri = 0;
  for (int k = 0; k < 30; ++k) {
    out30[k] = h[k];
    tri += h[k];
  }
  for (int k = 0; k < 6; ++k) out30[20 + k] += h[36 + k] - h[30 + k];
  g->times.closed_triangles = tri;
  return HM_OK;
}

namespace {
__global__ void k_count_work(const uint64_t* est, uint32_t n, unsigned int* out3) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    if (est[i]) atomicAdd(&out3[0], 1u);
    if (est[i] >> 63) atomicAdd(&out3[1], 1u);
    if ((est[i] >> 62) & 1u) atomicAdd(&out3[2], 1u);
  }
}
}  // namespace

// Full counts of the graphs behind the listed slots (every live slot of each
// counted graph, graphs node-disjoint): the static algorithm over the listed
// centres only, with oriented rows built for them alone and each centre's
// counts routed to row rog[gos[a]] of out (n_rows x 30).
int count_static_rows(hm_graph* g, const uint32_t* d_rows, uint32_t n, const TouchRows& rows, uint64_t* out) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  const uint32_t R = rows.n_rows;
  for (size_t k = 0; k < (size_t)R * 30; ++k) out[k] = 0;
  if (!n) return HM_OK;
  const auto t_begin = std::chrono::steady_clock::now();
  HM_TRY(prepare_static_attrs());
  PlusRows P;
  HM_TRY(build_plus_rows(g, d_rows, n, &P));
  DArr<uint64_t> est, est_sorted;
  DArr<uint32_t> ids, work;
  DArr<unsigned long long> cnt;
  const size_t n_cnt = (size_t)R * kRowStride + 5;  // + three queues, + three work counts
  HM_TRY(est.alloc(ctx, n));
  HM_TRY(est_sorted.alloc(ctx, n));
  HM_TRY(ids.alloc(ctx, n));
  HM_TRY(work.alloc(ctx, n));
  HM_TRY(cnt.alloc(ctx, n_cnt));
  HM_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long) * n_cnt, st));
  unsigned long long* tail = cnt.p + (size_t)R * kRowStride;
  k_closed_work<<<grid_for((uint64_t)n * 32, 256), 256, 0, st>>>(P.off.p, P.len.p, P.nbr.p, d_rows, n, rows.gos,
                                                                rows.rog, g->sched, est.p, ids.p);
  HM_LAUNCH_CHECK();
  {
    size_t tb = 0;
    HM_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, est.p, est_sorted.p, ids.p, work.p, (int64_t)n, 0,
                                                      64, st));
    DArr<uint8_t> tmp;
    HM_TRY(tmp.alloc(ctx, tb));
    HM_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.p, tb, est.p, est_sorted.p, ids.p, work.p, (int64_t)n, 0,
                                                      64, st));
  }
  unsigned int* wc = reinterpret_cast<unsigned int*>(tail + 3);
  k_count_work<<<grid_for(n, 256), 256, 0, st>>>(est_sorted.p, n, wc);
  HM_LAUNCH_CHECK();
  k_open_pairs<<<(unsigned)ctx->n_sms * 8, kOpenBlock, 0, st>>>(g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p,
                                                               g->h2h_ovl.p, g->esize.p, d_rows, n, 0, 1, rows.gos,
                                                               rows.rog, cnt.p + 36);
  HM_LAUNCH_CHECK();
  unsigned int hw[3] = {0, 0, 0};
  HM_CUDA(cudaMemcpyAsync(hw, wc, sizeof(hw), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  const uint32_t n_work = hw[0], n_big = hw[1];
  const uint32_t bounds[4] = {0, n_big, hw[2], n_work};
  ClosedArgs pargs{P.off.p, P.len.p, P.nbr.p, P.os.p, g->h2h_nbr.p, g->h2v_off.p, g->h2v_mem.p,
                   g->esize.p, work.p, 0, 0, 1, nullptr, cnt.p, nullptr, rows.gos, rows.rog};
  with_masks(g, pargs);
  pargs.loff = P.loff.p;
  pargs.lmask = P.lmask.p;
  HM_TRY(launch_closed(ctx, pargs, bounds, reinterpret_cast<unsigned int*>(tail)));
  std::vector<unsigned long long> h((size_t)R * kRowStride);
  HM_CUDA(cudaMemcpyAsync(h.data(), cnt.p, sizeof(unsigned long long) * h.size(), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  if (std::getenv("HM_TRACE"))
    std::fprintf(stderr, "[hm_trace static_rows] rows=%u oriented=%llu work=%u big=%u total=%.1fms\n", n,
                 (unsigned long long)P.nnz, n_work, n_big,
                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_begin).count());
  for (uint32_t r = 0; r < R; ++r) {
    const unsigned long long* x = h.data() + (size_t)r * kRowStride;
    uint64_t* o = out + (size_t)r * 30;
    for (int k = 0; k < 30; ++k) o[k] = x[k];
    for (int k = 0; k < 6; ++k) o[20 + k] += x[36 + k] - x[30 + k];
  }
  return HM_OK;
}

namespace {
// type 1 (sum of C(|a|, 3)) and type 2 (adjacent pairs a < b with overlap
// o >= 2: C(o, 2) (|a| - o) (|b| - o)); one warp per slot.
__global__ void k_triads12(const uint64_t* off, const uint32_t* len, const uint32_t* nbr, const uint8_t* ovl,
                           const uint8_t* esize, uint32_t n, unsigned long long* out2) {
  unsigned long long t1 = 0, t2 = 0;
  for (uint64_t a = global_warp(); a < n; a += n_warps()) {
    const uint64_t sa = esize[a];
    if (lane_id() == 0 && sa >= 3) t1 += sa * (sa - 1) * (sa - 2) / 6;
    const uint64_t o0 = off[a];
    for (uint32_t i = lane_id(); i < len[a]; i += kWarp) {
      const uint32_t b = nbr[o0 + i];
      const uint64_t o = ovl[o0 + i], sb = esize[b];
      if (b > a && o >= 2 && sa > o && sb > o) t2 += o * (o - 1) / 2 * (sa - o) * (sb - o);
    }
  }
  t1 = warp_sum(t1);
  t2 = warp_sum(t2);
  if (lane_id() == 0) {
    if (t1) atomicAdd(&out2[0], t1);
    if (t2) atomicAdd(&out2[1], t2);
  }
}
}  // namespace

// The reference's three vertex-triad counts (temporalDynamicHMotif/src/
// type1.cu:27-47, type2.cu:47-86, type3.cu:61-122): type 1 and 2 from the
// sizes and the adjacency, type 3 from one pass of the closed-triangle
// kernels in their triad mode.
int count_vertex_triads(hm_graph* g, uint64_t out3[3]) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  HM_TRY(prepare_static(g));
  DArr<unsigned long long> cnt;
  HM_TRY(cnt.alloc(ctx, 8));  // [0] type 3, [1..3] queues, [4] type 1, [5] type 2
  HM_CUDA(cudaMemsetAsync(cnt.p, 0, 8 * sizeof(unsigned long long), st));
  if (g->n_slots) {
    k_triads12<<<(unsigned)ctx->n_sms * 8, 256, 0, st>>>(g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p, g->h2h_ovl.p,
                                                         g->esize.p, g->n_slots, cnt.p + 4);
    HM_LAUNCH_CHECK();
  }
  const uint32_t bounds[4] = {0, g->n_work_big, g->n_work_mid, g->n_work};
  ClosedArgs targs{g->plus_off.p, g->plus_len.p, g->plus_nbr.p, g->plus_os.p, g->h2h_nbr.p, g->h2v_off.p,
                   g->h2v_mem.p,    g->esize.p,    g->work.p,      0,             0,               1,
                   nullptr,         cnt.p,         nullptr,        nullptr,       nullptr};
  with_masks(g, targs);
  HM_TRY(launch_closed<true>(ctx, targs, bounds, reinterpret_cast<unsigned int*>(cnt.p + 1)));
  unsigned long long h[8];
  HM_CUDA(cudaMemcpyAsync(h, cnt.p, sizeof(h), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  out3[0] = h[4];
  out3[1] = h[5];
  out3[2] = h[0];
  return HM_OK;
}

int count_static30(hm_graph* g, uint32_t shard, uint32_t n_shards, uint64_t out30[30]) {
  if (n_shards == 0 || shard >= n_shards) return set_error(HM_ERR_INVALID, "static count: shard %u of %u", shard, n_shards);
  HM_TRY(prepare_static(g));
  HM_TRY(launch_static(g, shard, n_shards, nullptr));
  return finish_static(g, out30);
}

// The touched-triple launch shapes hold the same row lengths as the static
// ones: one warp up to 128 entries, 4096-slot tables up to 2048.
int set_schedule(hm_graph* g, const ClosedSchedule& s, const TouchSchedule& t) {
  if (s.warp_row > kWarpRow || s.small_row < s.warp_row || s.small_row > kSmallRow)
    return set_error(HM_ERR_INVALID, "schedule {warp_row %u, small_row %u}: need warp_row <= %u and "
                     "warp_row <= small_row <= %u", s.warp_row, s.small_row, kWarpRow, kSmallRow);
  if (t.warp_row > kWarpRow || t.mid_row < t.warp_row || t.mid_row > kSmallRow)
    return set_error(HM_ERR_INVALID, "schedule {touch_warp_row %u, touch_mid_row %u}: need touch_warp_row <= %u "
                     "and touch_warp_row <= touch_mid_row <= %u", t.warp_row, t.mid_row, kWarpRow, kSmallRow);
  if (s.warp_row != g->sched.warp_row || s.small_row != g->sched.small_row) {
    g->sched = s;
    g->work_valid = false;  // the work list is split by the schedule
  }
  g->tsched = t;
  return HM_OK;
}

namespace {
// Every stride-th centre of a work list, in order.
__global__ void k_stride_sample(const uint32_t* work, uint32_t n_out, uint32_t stride, uint32_t* out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_out;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = work[i * stride];
}

struct EventPair {
  cudaEvent_t e[2] = {nullptr, nullptr};
  ~EventPair() {
    for (auto x : e)
      if (x) cudaEventDestroy(x);
  }
};

// Candidate schedules; the first is the default. The warp kernel's limit
// moves rows between one warp and one block per centre, the small-table
// limit moves rows between 4-per-SM and 2-per-SM blocks.
// Only the warp limit is tuned. Moving rows of 513-2048 entries to the
// large-row shape (then 8192 slots) looked 8 % faster on the strided sample of the 2M-hyperedge
// config-2 graph and was 33 % slower on the whole graph (22.5 s against
// 16.9 s per count): the sample's blocks share little of N+ in L2, the whole
// graph's do.
constexpr ClosedSchedule kTuneCandidates[] = {{128, 2048}, {96, 2048}, {64, 2048}, {32, 2048}, {0, 2048}};
constexpr unsigned kTuneCount = sizeof(kTuneCandidates) / sizeof(kTuneCandidates[0]);
constexpr uint32_t kTuneSampleMax = 65536;  // sampled centres with stride 0
constexpr float kTuneMargin = 0.98f;        // another schedule must beat the default by 2 %
static_assert(kTuneCount <= HM_TUNE_MAX_CANDIDATES, "report holds every candidate");
}  // namespace

// Times the closed phase under every candidate schedule on one strided
// sample of the graph's centres: the sample is fixed, each candidate splits
// it into its own launch shapes (work estimates, sort, split as for a full
// count) and runs the three launches into scratch counters.
int autotune_closed(hm_graph* g, uint32_t stride, hm_tune_report& R) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  HM_TRY(prepare_static(g));
  R.n_candidates = kTuneCount;
  for (unsigned c = 0; c < kTuneCount; ++c) {
    R.rows[c][0] = kTuneCandidates[c].warp_row;
    R.rows[c][1] = kTuneCandidates[c].small_row;
  }
  const uint32_t n_work = g->n_work;
  if (stride == 0) stride = std::max<uint32_t>(1, (uint32_t)(((uint64_t)n_work + kTuneSampleMax - 1) / kTuneSampleMax));
  R.sample_stride = stride;
  const uint32_t n = n_work ? (uint32_t)(((uint64_t)n_work + stride - 1) / stride) : 0;
  R.sampled = n;
  uint32_t best = 0;
  if (n) {
    DArr<uint32_t> sample, ids, work;
    DArr<uint64_t> est, est_sorted;
    DArr<unsigned long long> cnt;
    HM_TRY(sample.alloc(ctx, n));
    HM_TRY(ids.alloc(ctx, n));
    HM_TRY(work.alloc(ctx, n));
    HM_TRY(est.alloc(ctx, n));
    HM_TRY(est_sorted.alloc(ctx, n));
    HM_TRY(cnt.alloc(ctx, 48));
    size_t tb = 0;
    HM_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, est.p, est_sorted.p, ids.p, work.p, (int64_t)n,
                                                      0, 64, st));
    DArr<uint8_t> tmp;
    HM_TRY(tmp.alloc(ctx, tb));
    k_stride_sample<<<grid_for(n, 256), 256, 0, st>>>(g->work.p, n, stride, sample.p);
    HM_LAUNCH_CHECK();
    EventPair ev;
    HM_CUDA(cudaEventCreate(&ev.e[0]));
    HM_CUDA(cudaEventCreate(&ev.e[1]));
    unsigned int* wc = reinterpret_cast<unsigned int*>(cnt.p + 44);  // three work counts
    for (int rep = -1; rep < (int)kTuneCount; ++rep) {  // rep -1: untimed warm-up of the default
      const unsigned c = rep < 0 ? 0u : (unsigned)rep;
      HM_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long) * 48, st));
      k_closed_work<<<grid_for((uint64_t)n * 32, 256), 256, 0, st>>>(g->plus_off.p, g->plus_len.p, g->plus_nbr.p,
                                                                    sample.p, n, nullptr, nullptr,
                                                                    kTuneCandidates[c], est.p, ids.p);
      HM_LAUNCH_CHECK();
      HM_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.p, tb, est.p, est_sorted.p, ids.p, work.p, (int64_t)n,
                                                        0, 64, st));
      k_count_work<<<grid_for(n, 256), 256, 0, st>>>(est_sorted.p, n, wc);
      HM_LAUNCH_CHECK();
      unsigned int hw[3] = {0, 0, 0};
      HM_CUDA(cudaMemcpyAsync(hw, wc, sizeof(hw), cudaMemcpyDeviceToHost, st));
      HM_CUDA(cudaStreamSynchronize(st));
      const uint32_t bounds[4] = {0, hw[1], hw[2], hw[0]};
      ClosedArgs targs{g->plus_off.p, g->plus_len.p, g->plus_nbr.p, g->plus_os.p, g->h2h_nbr.p, g->h2v_off.p,
                       g->h2v_mem.p,    g->esize.p,    work.p,         0,             0,               1,
                       nullptr,         cnt.p,         nullptr,        nullptr,       nullptr};
      with_groups(g, targs);
      HM_CUDA(cudaEventRecord(ev.e[0], st));
      HM_TRY(launch_closed(ctx, targs, bounds, reinterpret_cast<unsigned int*>(cnt.p + 42)));
      HM_CUDA(cudaEventRecord(ev.e[1], st));
      HM_CUDA(cudaEventSynchronize(ev.e[1]));
      float ms = 0;
      HM_CUDA(cudaEventElapsedTime(&ms, ev.e[0], ev.e[1]));
      if (rep >= 0) R.ms[c] = ms;
    }
    for (unsigned c = 1; c < kTuneCount; ++c)
      if (R.ms[c] < kTuneMargin * R.ms[0] && R.ms[c] < R.ms[best]) best = c;
  }
  R.best = best;
  return set_schedule(g, kTuneCandidates[best], g->tsched);
}

}  // namespace hm
