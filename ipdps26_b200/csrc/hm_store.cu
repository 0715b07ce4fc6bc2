// Device-resident hypergraph store: construction of H2V, V2H, H2H (with
// overlap sizes and smallest shared node) and the oriented adjacency.
//
// Reference counterpart: constructCBST / CBSTOperations::construct
// (dynamicHyperGraph/structure/operations.cu:31-80, 412-415) and the host
// adjacency builder hyperedgeAdjacency (dynamicHyperGraph/utils/utils.cpp:
// 399-427). There, keys 1..N sit in a level-order BST whose nodes point into
// a padded int payload and H2H is built on the host with std::set and no
// overlap sizes. Here ids are dense, so a direct id -> (offset, length)
// segment table replaces the tree walk; every table is built on the device
// by sort / scan / compact kernels.
#include <cub/cub.cuh>
#include <thrust/iterator/transform_iterator.h>

#include <algorithm>
#include <functional>
#include <vector>

#include "hm_device.h"

namespace hm {

namespace {

constexpr unsigned kWarp = 32;
constexpr unsigned kBlock = 256;

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned lanemask_lt() { return (1u << lane_id()) - 1u; }
__device__ __forceinline__ uint64_t global_warp() { return ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ uint64_t n_warps() { return ((uint64_t)gridDim.x * blockDim.x) >> 5; }

// ---- H2V normalisation ----------------------------------------------------

__global__ void k_seg_bounds(const uint64_t* off, uint32_t n, int* beg, int* end) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x) {
    beg[r] = (int)off[r];
    end[r] = (int)off[r + 1];
  }
}

// Distinct count of each sorted row; flags node ids >= n_nodes.
__global__ void k_row_distinct(const uint64_t* off, const uint32_t* mem, uint32_t n, uint32_t n_nodes,
                               uint32_t* cnt, int* bad) {
  for (uint64_t r = global_warp(); r < n; r += n_warps()) {
    const uint64_t s = off[r], e = off[r + 1];
    uint32_t c = 0;
    for (uint64_t i0 = s; i0 < e; i0 += kWarp) {
      const uint64_t i = i0 + lane_id();
      bool first = false;
      if (i < e) {
        const uint32_t v = mem[i];
        if (v >= n_nodes) atomicExch(bad, 1);
        first = (i == s) || (mem[i - 1] != v);
      }
      c += __popc(__ballot_sync(0xffffffffu, first));
    }
    if (lane_id() == 0) cnt[r] = c;
  }
}

__global__ void k_row_distinct_write(const uint64_t* off, const uint32_t* mem, uint32_t n, const uint64_t* out_off,
                                     uint32_t* out) {
  for (uint64_t r = global_warp(); r < n; r += n_warps()) {
    const uint64_t s = off[r], e = off[r + 1];
    uint64_t w = out_off[r];
    for (uint64_t i0 = s; i0 < e; i0 += kWarp) {
      const uint64_t i = i0 + lane_id();
      bool first = false;
      uint32_t v = 0;
      if (i < e) {
        v = mem[i];
        first = (i == s) || (mem[i - 1] != v);
      }
      const unsigned m = __ballot_sync(0xffffffffu, first);
      if (first) out[w + __popc(m & lanemask_lt())] = v;
      w += __popc(m);
    }
  }
}

__global__ void k_u32_to_u8_checked(const uint32_t* in, uint32_t n, uint8_t* out, uint32_t limit, int* bad) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t v = in[i];
    if (v > limit) atomicExch(bad, 1);
    out[i] = (uint8_t)(v > 255 ? 255 : v);
  }
}

__global__ void k_fill_live_bits(uint32_t* bits, uint32_t n_words, uint32_t n_live) {
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < n_words; w += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t lo = w * 32;
    uint32_t v = 0;
    if (lo + 32 <= n_live) v = 0xffffffffu;
    else if (lo < n_live) v = (1u << (n_live - lo)) - 1u;
    bits[w] = v;
  }
}

// ---- V2H ---------------------------------------------------------------------

// (node, slot) pairs in slot order, so a stable sort by node keeps slots
// ascending within each node.
__global__ void k_member_pairs(const uint64_t* off, const uint32_t* len, const uint32_t* mem, uint32_t n,
                               const uint64_t* pair_off, uint32_t* keys, uint32_t* vals, uint32_t* node_cnt) {
  for (uint64_t r = global_warp(); r < n; r += n_warps()) {
    const uint64_t s = off[r], d = pair_off[r];
    const uint32_t l = len[r];
    for (uint32_t i = lane_id(); i < l; i += kWarp) {
      const uint32_t v = mem[s + i];
      keys[d + i] = v;
      vals[d + i] = (uint32_t)r;
      atomicAdd(&node_cnt[v], 1u);
    }
  }
}

// ---- H2H ---------------------------------------------------------------------

// Rows are addressed through an optional list: list position i is slot
// rows[i] (slot i when rows is null).
__device__ __forceinline__ uint32_t row_at(const uint32_t* rows, uint64_t i) { return rows ? rows[i] : (uint32_t)i; }

__global__ void k_wedge_count(const uint64_t* off, const uint32_t* len, const uint32_t* mem, const uint32_t* vlen,
                              const uint32_t* rows, uint32_t n, uint64_t* wedges) {
  for (uint64_t i = global_warp(); i < n; i += n_warps()) {
    const uint32_t r = row_at(rows, i);
    const uint64_t s = off[r];
    const uint32_t l = len[r];
    uint64_t w = 0;
    for (uint32_t k = lane_id(); k < l; k += kWarp) w += vlen[mem[s + k]] - 1u;
    for (int d = 16; d; d >>= 1) w += __shfl_xor_sync(0xffffffffu, w, d);
    if (lane_id() == 0) wedges[i] = w;
  }
}

// Every (b, position of the shared node in r) for b != r sharing a node with
// r, written as key (b << 8) | pos into r's range of the chunk buffer.
__global__ void k_expand(const uint64_t* h_off, const uint32_t* h_len, const uint32_t* h_mem, const uint64_t* v_off,
                         const uint32_t* v_len, const uint32_t* v_edge, const uint64_t* wedge_off,
                         const uint32_t* rows, uint64_t chunk_base, uint32_t r0, uint32_t r1, uint32_t* keys) {
  for (uint64_t i = r0 + global_warp(); i < r1; i += n_warps()) {
    const uint32_t r = row_at(rows, i);
    uint64_t pos = wedge_off[i] - chunk_base;
    const uint64_t s = h_off[r];
    const uint32_t l = h_len[r];
    for (uint32_t p = 0; p < l; ++p) {
      const uint32_t v = h_mem[s + p];
      const uint64_t lo = v_off[v];
      const uint32_t n = v_len[v];
      for (uint32_t j0 = 0; j0 < n; j0 += kWarp) {
        const uint32_t j = j0 + lane_id();
        uint32_t b = 0;
        bool keep = false;
        if (j < n) {
          b = v_edge[lo + j];
          keep = (b != r);
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) keys[pos + __popc(m & lanemask_lt())] = (b << 8) | p;
        pos += __popc(m);
      }
    }
  }
}

__global__ void k_chunk_bounds(const uint64_t* wedge_off, uint64_t chunk_base, uint32_t r0, uint32_t r1, int* beg,
                               int* end) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < r1 - r0; i += (uint64_t)gridDim.x * blockDim.x) {
    beg[i] = (int)(wedge_off[r0 + i] - chunk_base);
    end[i] = (int)(wedge_off[r0 + i + 1] - chunk_base);
  }
}

// Number of distinct neighbours per row of a sorted chunk.
__global__ void k_chunk_distinct(const int* beg, const int* end, const uint32_t* keys, uint32_t nrows, uint32_t* cnt) {
  for (uint64_t r = global_warp(); r < nrows; r += n_warps()) {
    const int s = beg[r], e = end[r];
    uint32_t c = 0;
    for (int i0 = s; i0 < e; i0 += kWarp) {
      const int i = i0 + (int)lane_id();
      bool first = false;
      if (i < e) first = (i == s) || ((keys[i] >> 8) != (keys[i - 1] >> 8));
      c += __popc(__ballot_sync(0xffffffffu, first));
    }
    if (lane_id() == 0) cnt[r] = c;
  }
}

// Run starts (row-relative) of each row, at the row's local output offset.
__global__ void k_chunk_starts(const int* beg, const int* end, const uint32_t* keys, uint32_t nrows,
                               const uint64_t* local_off, uint32_t* starts) {
  for (uint64_t r = global_warp(); r < nrows; r += n_warps()) {
    const int s = beg[r], e = end[r];
    uint64_t w = local_off[r];
    for (int i0 = s; i0 < e; i0 += kWarp) {
      const int i = i0 + (int)lane_id();
      bool first = false;
      if (i < e) first = (i == s) || ((keys[i] >> 8) != (keys[i - 1] >> 8));
      const unsigned m = __ballot_sync(0xffffffffu, first);
      if (first) starts[w + __popc(m & lanemask_lt())] = (uint32_t)(i - s);
      w += __popc(m);
    }
  }
}

__global__ void k_chunk_emit(const int* beg, const int* end, const uint32_t* keys, const uint32_t* rows, uint32_t r0,
                             uint32_t nrows, const uint64_t* local_off, const uint32_t* cnt, const uint32_t* starts,
                             uint64_t out_base, uint64_t* row_off,
                             uint32_t* row_len, uint32_t* nbr, uint8_t* ovl, uint64_t* pmask) {
  for (uint64_t r = global_warp(); r < nrows; r += n_warps()) {
    const int s = beg[r], e = end[r];
    const uint64_t lo = local_off[r];
    const uint32_t c = cnt[r];
    const uint64_t dst = out_base + lo;
    if (lane_id() == 0) {
      const uint32_t slot = row_at(rows, r0 + r);
      row_off[slot] = dst;
      row_len[slot] = c;
    }
    for (uint32_t k = lane_id(); k < c; k += kWarp) {
      const uint32_t st = starts[lo + k];
      const uint32_t en = (k + 1 < c) ? starts[lo + k + 1] : (uint32_t)(e - s);
      const uint32_t key = keys[s + st];
      nbr[dst + k] = key >> 8;
      ovl[dst + k] = (uint8_t)(en - st);
      uint64_t m = 0;
      for (uint32_t q = st; q < en; ++q) {
        const uint32_t pos = keys[s + q] & 255u;
        if (pos < 64) m |= 1ull << pos;
      }
      pmask[dst + k] = m;
    }
  }
}

// ---- oriented adjacency --------------------------------------------------------

__device__ __forceinline__ bool above(uint32_t a, uint32_t da, uint32_t b, uint32_t db) {
  return rank_above(a, da, b, db);
}

// rows == nullptr: rows 0..n-1; else the listed rows. cnt[i] is the i-th
// row's count.
__global__ void k_plus_count(const uint64_t* off, const uint32_t* len, const uint32_t* nbr, const uint32_t* rows,
                             uint32_t n, uint32_t* cnt) {
  for (uint64_t i = global_warp(); i < n; i += n_warps()) {
    const uint32_t a = rows ? rows[i] : (uint32_t)i;
    const uint64_t s = off[a];
    const uint32_t l = len[a];
    uint32_t c = 0;
    for (uint32_t i0 = 0; i0 < l; i0 += kWarp) {
      const uint32_t i = i0 + lane_id();
      bool up = false;
      if (i < l) {
        const uint32_t b = nbr[s + i];
        up = above(a, l, b, len[b]);
      }
      c += __popc(__ballot_sync(0xffffffffu, up));
    }
    if (lane_id() == 0) cnt[i] = c;
  }
}

__global__ void k_plus_write(const uint64_t* off, const uint32_t* len, const uint32_t* nbr, const uint8_t* ovl,
                             const uint64_t* mask, const uint8_t* esize, const uint32_t* rows, uint32_t n,
                             const uint64_t* poff, const uint32_t* plen, const uint64_t* loff, uint32_t* pnbr,
                             uint16_t* pos, uint64_t* lmask) {
  for (uint64_t r = global_warp(); r < n; r += n_warps()) {
    const uint32_t a = rows ? rows[r] : (uint32_t)r;
    const uint64_t s = off[a];
    const uint32_t l = len[a];
    const uint64_t w0 = poff[a];
    const bool long_row = plen[a] > kLongRow;
    uint64_t w = w0;
    for (uint32_t i0 = 0; i0 < l; i0 += kWarp) {
      const uint32_t i = i0 + lane_id();
      bool up = false;
      uint32_t b = 0;
      if (i < l) {
        b = nbr[s + i];
        up = above(a, l, b, len[b]);
      }
      const unsigned m = __ballot_sync(0xffffffffu, up);
      if (up) {
        const uint64_t d = w + __popc(m & lanemask_lt());
        pnbr[d] = b;
        pos[d] = (uint16_t)(((uint32_t)esize[b] << 8) | ovl[s + i]);
        if (long_row) lmask[loff[a] + (d - w0)] = mask[s + i];
      }
      w += __popc(m);
    }
  }
}

// Groups per oriented row of owner b: group 0 the neighbours sharing several
// members with b, or one at a position >= 64 of b's list (their position mask
// is then empty); group 1 + p those whose only shared member is b's p-th.
constexpr uint32_t kGroupPositions = 64;
__device__ __forceinline__ uint32_t n_groups(uint32_t size) { return 1u + min(size, kGroupPositions); }
__device__ __forceinline__ uint32_t group_of(uint16_t os, uint64_t mask) {
  return ((os & 0xffu) == 1u && mask) ? 1u + (uint32_t)(__ffsll((long long)mask) - 1) : 0u;
}

__global__ void k_group_sizes(const uint8_t* esize, uint32_t n, uint32_t* tsize) {
  for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < n; b += (uint64_t)gridDim.x * blockDim.x)
    tsize[b] = n_groups(esize[b]) + 1;
}

// One warp per row: group histogram (and the size-1 / size-2 neighbours of
// each group) in shared memory, its prefix sums as the group table, then a
// scatter of the row's entries into the grouped copy.
constexpr unsigned kGroupWarps = kBlock / kWarp;
__global__ void __launch_bounds__(kBlock) k_group_rows(const uint64_t* poff, const uint32_t* plen,
                                                       const uint32_t* pnbr, const uint16_t* pos,
                                                       const uint64_t* roff, const uint32_t* rlen,
                                                       const uint32_t* rnbr, const uint64_t* rmask,
                                                       const uint8_t* esize, uint32_t n,
                                                       const uint64_t* gbase, uint4* gtab, uint32_t* gnbr,
                                                       uint16_t* gos) {
  __shared__ uint32_t cnt[kGroupWarps][kGroupPositions + 1];
  __shared__ uint32_t one[kGroupWarps][kGroupPositions + 1];
  __shared__ uint32_t two[kGroupWarps][kGroupPositions + 1];
  const unsigned w = threadIdx.x / kWarp, lane = lane_id();
  for (uint64_t b = global_warp(); b < n; b += n_warps()) {
    const uint32_t G = n_groups(esize[b]);
    for (uint32_t k = lane; k < G; k += kWarp) cnt[w][k] = one[w][k] = two[w][k] = 0;
    __syncwarp();
    const uint64_t s = poff[b];
    const uint32_t l = plen[b];
    for (uint32_t i = lane; i < l; i += kWarp) {
      const uint16_t o = pos[s + i];
      const uint32_t grp = group_of(o, row_mask(roff, rlen, rnbr, rmask, (uint32_t)b, pnbr[s + i]));  // < G: a position bit p < min(size, 64)
      atomicAdd(&cnt[w][grp], 1u);
      const uint32_t sc = o >> 8;
      if (sc == 1) atomicAdd(&one[w][grp], 1u);
      if (sc == 2) atomicAdd(&two[w][grp], 1u);
    }
    __syncwarp();
    const uint64_t t = gbase[b];
    if (lane == 0) {
      uint32_t run = 0;
      for (uint32_t k = 0; k < G; ++k) {
        const uint32_t c = cnt[w][k];
        gtab[t + k] = make_uint4(run, one[w][k], two[w][k], 0u);
        cnt[w][k] = run;  // becomes the group's write cursor
        run += c;
      }
      gtab[t + G] = make_uint4(run, 0u, 0u, 0u);
    }
    __syncwarp();
    for (uint32_t i = lane; i < l; i += kWarp) {
      const uint16_t o = pos[s + i];
      const uint32_t d =
          atomicAdd(&cnt[w][group_of(o, row_mask(roff, rlen, rnbr, rmask, (uint32_t)b, pnbr[s + i]))], 1u);
      gnbr[s + d] = pnbr[s + i];
      gos[s + d] = o;
    }
    __syncwarp();
  }
}

// One warp per row a: for each oriented entry (a, b) whose two hyperedges
// share exactly one member u, at a position p < 64 of a, u's position in b
// (a binary search of b's sorted members), 0xff for every other entry and
// for a position of 64 or more in b.
__global__ void k_shared_positions(const uint64_t* poff, const uint32_t* plen, const uint32_t* pnbr,
                                   const uint16_t* pos, const uint64_t* roff, const uint32_t* rlen,
                                   const uint32_t* rnbr, const uint64_t* rmask, const uint64_t* hoff,
                                   const uint32_t* hmem,
                                   const uint8_t* esize, uint32_t n, uint8_t* opos) {
  for (uint64_t a = global_warp(); a < n; a += n_warps()) {
    const uint64_t s = poff[a];
    const uint32_t* am = hmem + hoff[a];
    for (uint32_t i = lane_id(); i < plen[a]; i += kWarp) {
      const uint64_t m = row_mask(roff, rlen, rnbr, rmask, (uint32_t)a, pnbr[s + i]);
      uint8_t p = 0xff;
      if ((pos[s + i] & 0xffu) == 1u && m) {
        const uint32_t u = am[__ffsll((long long)m) - 1];
        const uint32_t b = pnbr[s + i];
        const uint32_t* bm = hmem + hoff[b];
        uint32_t lo = 0, hi = esize[b];
        while (lo < hi) {
          const uint32_t mid = (lo + hi) >> 1;
          if (bm[mid] < u) lo = mid + 1;
          else hi = mid;
        }
        if (lo < kGroupPositions) p = (uint8_t)lo;
      }
      opos[s + i] = p;
    }
  }
}

}  // namespace

// The grouped copy of the oriented rows (see hm_graph::grp_nbr).
int build_plus_groups(hm_graph* g) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  const uint32_t E = g->n_slots;
  DArr<uint32_t> tsize;
  HM_TRY(tsize.alloc(ctx, E));
  HM_TRY(g->grp_base.alloc(ctx, (size_t)E + 1));
  if (E) {
    k_group_sizes<<<grid_for(E, kBlock), kBlock, 0, st>>>(g->esize.p, E, tsize.p);
    HM_LAUNCH_CHECK();
  }
  HM_TRY(exclusive_scan(ctx, tsize.p, g->grp_base.p, E));
  uint64_t tab = 0;
  HM_CUDA(cudaMemcpyAsync(&tab, g->grp_base.p + E, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  HM_TRY(g->grp_tab.alloc(ctx, tab));
  HM_TRY(g->grp_opos.alloc(ctx, g->plus_nnz));
  HM_TRY(g->grp_nbr.alloc(ctx, g->plus_nnz));
  HM_TRY(g->grp_os.alloc(ctx, g->plus_nnz));
  if (E) {
    k_group_rows<<<grid_for((uint64_t)E * kWarp, kBlock), kBlock, 0, st>>>(
        g->plus_off.p, g->plus_len.p, g->plus_nbr.p, g->plus_os.p, g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p,
        g->h2h_mask.p, g->esize.p, E, g->grp_base.p, g->grp_tab.p, g->grp_nbr.p, g->grp_os.p);
    HM_LAUNCH_CHECK();
    k_shared_positions<<<grid_for((uint64_t)E * kWarp, kBlock), kBlock, 0, st>>>(
        g->plus_off.p, g->plus_len.p, g->plus_nbr.p, g->plus_os.p, g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p,
        g->h2h_mask.p, g->h2v_off.p, g->h2v_mem.p, g->esize.p, E, g->grp_opos.p);
    HM_LAUNCH_CHECK();
  }
  g->grp_valid = true;
  return HM_OK;
}

// Frees the oriented copy (and the grouped one built from it).
void release_plus(hm_graph* g) {
  g->long_off.release();
  g->long_mask.release();
  g->plus_nbr.release();
  g->plus_os.release();
  g->plus_valid = false;
  release_plus_groups(g);
}

void release_plus_groups(hm_graph* g) {
  g->grp_nbr.release();
  g->grp_os.release();
  g->grp_base.release();
  g->grp_tab.release();
  g->grp_opos.release();
  g->grp_valid = false;
}

struct WidenU64 {
  __host__ __device__ uint64_t operator()(uint32_t x) const { return x; }
};

// out[0..n]: exclusive prefix sums of in[0..n) with the total at out[n]; the
// sum is accumulated in 64 bits whatever the input width.
template <class T>
int exclusive_scan(hm_ctx* ctx, const T* in, uint64_t* out, uint64_t n) {
  HM_CUDA(cudaMemsetAsync(out, 0, sizeof(uint64_t), ctx->stream));
  if (!n) return HM_OK;
  size_t tb = 0;
  if constexpr (sizeof(T) == 4) {
    auto it = thrust::make_transform_iterator(in, WidenU64());
    HM_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, it, out + 1, (int64_t)n, ctx->stream));
    DArr<uint8_t> tmp;
    HM_TRY(tmp.alloc(ctx, tb));
    HM_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, tb, it, out + 1, (int64_t)n, ctx->stream));
  } else {
    HM_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, in, out + 1, (int64_t)n, ctx->stream));
    DArr<uint8_t> tmp;
    HM_TRY(tmp.alloc(ctx, tb));
    HM_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, tb, in, out + 1, (int64_t)n, ctx->stream));
  }
  return HM_OK;
}

template int exclusive_scan<uint32_t>(hm_ctx*, const uint32_t*, uint64_t*, uint64_t);
template int exclusive_scan<uint64_t>(hm_ctx*, const uint64_t*, uint64_t*, uint64_t);

// Upload hyperedges, sort and deduplicate each member list on the device.
int build_h2v(hm_graph* g, const uint64_t* h_off, const uint32_t* h_mem, uint32_t n_edges) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  const uint64_t nnz = h_off[n_edges];
  if (nnz >= (1ull << 31)) return set_error(HM_ERR_LIMIT, "hm_graph_build: %llu members exceed 2^31", (unsigned long long)nnz);
  for (uint32_t e = 0; e < n_edges; ++e)
    if (h_off[e + 1] < h_off[e]) return set_error(HM_ERR_INVALID, "hm_graph_build: offsets decrease at %u", e);
  DArr<uint64_t> raw_off;
  DArr<uint32_t> raw, sorted;
  DArr<int> beg, end;
  HM_TRY(raw_off.alloc(ctx, (size_t)n_edges + 1));
  HM_TRY(raw.alloc(ctx, nnz));
  HM_TRY(sorted.alloc(ctx, nnz));
  HM_TRY(beg.alloc(ctx, n_edges));
  HM_TRY(end.alloc(ctx, n_edges));
  HM_CUDA(cudaMemcpyAsync(raw_off.p, h_off, sizeof(uint64_t) * ((size_t)n_edges + 1), cudaMemcpyHostToDevice, st));
  if (nnz) HM_CUDA(cudaMemcpyAsync(raw.p, h_mem, sizeof(uint32_t) * nnz, cudaMemcpyHostToDevice, st));
  if (n_edges) {
    k_seg_bounds<<<grid_for(n_edges, kBlock), kBlock, 0, st>>>(raw_off.p, n_edges, beg.p, end.p);
    HM_LAUNCH_CHECK();
  }
  if (nnz) {
    size_t tb = 0;
    HM_CUDA(cub::DeviceSegmentedSort::SortKeys(nullptr, tb, raw.p, sorted.p, (int)nnz, (int)n_edges, beg.p, end.p, st));
    DArr<uint8_t> tmp;
    HM_TRY(tmp.alloc(ctx, tb));
    HM_CUDA(cub::DeviceSegmentedSort::SortKeys(tmp.p, tb, raw.p, sorted.p, (int)nnz, (int)n_edges, beg.p, end.p, st));
  }
  raw.release();
  DArr<uint32_t> cnt;
  DArr<int> bad;
  HM_TRY(cnt.alloc(ctx, n_edges));
  HM_TRY(bad.alloc(ctx, 2));
  HM_CUDA(cudaMemsetAsync(bad.p, 0, 2 * sizeof(int), st));
  if (n_edges) {
    k_row_distinct<<<grid_for((uint64_t)n_edges * 32, kBlock), kBlock, 0, st>>>(raw_off.p, sorted.p, n_edges,
                                                                              g->n_nodes, cnt.p, bad.p);
    HM_LAUNCH_CHECK();
  }
  HM_TRY(g->h2v_off.alloc(ctx, (size_t)n_edges + 1));
  HM_TRY(exclusive_scan(ctx, cnt.p, g->h2v_off.p, n_edges));
  uint64_t total = 0;
  HM_CUDA(cudaMemcpyAsync(&total, g->h2v_off.p + n_edges, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  HM_TRY(g->esize.alloc(ctx, n_edges));
  if (n_edges) {
    k_u32_to_u8_checked<<<grid_for(n_edges, kBlock), kBlock, 0, st>>>(cnt.p, n_edges, g->esize.p, HM_MAX_EDGE_SIZE,
                                                                      bad.p + 1);
    HM_LAUNCH_CHECK();
  }
  int hbad[2] = {0, 0};
  HM_CUDA(cudaMemcpyAsync(hbad, bad.p, sizeof(hbad), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  if (hbad[0]) return set_error(HM_ERR_INVALID, "hm_graph_build: a member id is >= n_nodes (%u)", g->n_nodes);
  if (hbad[1]) return set_error(HM_ERR_LIMIT, "hm_graph_build: a hyperedge has more than %d distinct members", HM_MAX_EDGE_SIZE);
  HM_TRY(g->h2v_mem.alloc(ctx, total));
  if (n_edges) {
    k_row_distinct_write<<<grid_for((uint64_t)n_edges * 32, kBlock), kBlock, 0, st>>>(raw_off.p, sorted.p, n_edges,
                                                                                    g->h2v_off.p, g->h2v_mem.p);
    HM_LAUNCH_CHECK();
  }
  g->h2v_len = static_cast<DArr<uint32_t>&&>(cnt);
  g->h2v_tail = total;
  g->h2v_nnz = total;
  g->cap_slots = n_edges;
  g->n_slots = n_edges;
  g->n_live = n_edges;
  const uint32_t words = (n_edges + 31) / 32;
  HM_TRY(g->live_bits.alloc(ctx, words ? words : 1));
  k_fill_live_bits<<<grid_for(words ? words : 1, kBlock), kBlock, 0, st>>>(g->live_bits.p, words, n_edges);
  HM_LAUNCH_CHECK();
  return HM_OK;
}

// V2H from the live H2V rows (works on a compact or an updated arena: pairs
// are placed by a scan of the row lengths).
int build_v2h(hm_graph* g) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  const uint32_t V = g->n_nodes;
  DArr<uint64_t> pair_off;
  HM_TRY(pair_off.alloc(ctx, (size_t)g->n_slots + 1));
  HM_TRY(exclusive_scan(ctx, g->h2v_len.p, pair_off.p, g->n_slots));
  uint64_t nnz = 0;
  HM_CUDA(cudaMemcpyAsync(&nnz, pair_off.p + g->n_slots, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  DArr<uint32_t> keys, vals, keys_out;
  HM_TRY(keys.alloc(ctx, nnz));
  HM_TRY(vals.alloc(ctx, nnz));
  HM_TRY(keys_out.alloc(ctx, nnz));
  HM_TRY(g->v2h_edge.alloc(ctx, nnz));
  HM_TRY(g->v2h_len.alloc(ctx, V));
  HM_CUDA(cudaMemsetAsync(g->v2h_len.p, 0, sizeof(uint32_t) * V, st));
  if (g->n_slots) {
    k_member_pairs<<<grid_for((uint64_t)g->n_slots * 32, kBlock), kBlock, 0, st>>>(
        g->h2v_off.p, g->h2v_len.p, g->h2v_mem.p, g->n_slots, pair_off.p, keys.p, vals.p, g->v2h_len.p);
    HM_LAUNCH_CHECK();
  }
  if (nnz) {
    int end_bit = 1;
    while (end_bit < 32 && (1ull << end_bit) < V) ++end_bit;
    size_t tb = 0;
    HM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.p, keys_out.p, vals.p, g->v2h_edge.p, (int64_t)nnz, 0,
                                            end_bit, st));
    DArr<uint8_t> tmp;
    HM_TRY(tmp.alloc(ctx, tb));
    HM_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, keys.p, keys_out.p, vals.p, g->v2h_edge.p, (int64_t)nnz, 0,
                                            end_bit, st));
  }
  HM_TRY(g->v2h_off.alloc(ctx, (size_t)V + 1));
  HM_TRY(exclusive_scan(ctx, g->v2h_len.p, g->v2h_off.p, V));
  g->v2h_tail = nnz;
  return HM_OK;
}

// H2H rows of the listed slots (all slots when d_rows is null), in chunks of
// the wedge stream: expand, segmented sort, run-length. reserve(W) is called
// once with an upper bound on the entries and returns the arena position
// where the rows are written; *written receives the entries emitted.
int h2h_rows_for(hm_graph* g, const uint32_t* d_rows, uint32_t n_rows,
                 const std::function<int(uint64_t, uint64_t*)>& reserve, uint64_t* written) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  *written = 0;
  if (g->n_slots >= (1u << 24))
    return set_error(HM_ERR_LIMIT, "H2H: %u hyperedge slots exceed the 2^24 limit of the packed sort key", g->n_slots);
  DArr<uint64_t> wedges, woff;
  HM_TRY(wedges.alloc(ctx, n_rows));
  HM_TRY(woff.alloc(ctx, (size_t)n_rows + 1));
  if (n_rows) {
    k_wedge_count<<<grid_for((uint64_t)n_rows * 32, kBlock), kBlock, 0, st>>>(g->h2v_off.p, g->h2v_len.p, g->h2v_mem.p,
                                                                            g->v2h_len.p, d_rows, n_rows, wedges.p);
    HM_LAUNCH_CHECK();
  }
  HM_TRY(exclusive_scan(ctx, wedges.p, woff.p, n_rows));
  std::vector<uint64_t> hw((size_t)n_rows + 1);
  HM_CUDA(cudaMemcpyAsync(hw.data(), woff.p, sizeof(uint64_t) * ((size_t)n_rows + 1), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  wedges.release();
  const uint64_t W = hw[n_rows];
  uint64_t base = 0;
  HM_TRY(reserve(W, &base));
  if (n_rows == 0) return HM_OK;
  if (W == 0) {
    // every listed row is empty
    DArr<uint32_t> zero;
    HM_TRY(zero.alloc(ctx, n_rows));
    HM_CUDA(cudaMemsetAsync(zero.p, 0, sizeof(uint32_t) * n_rows, st));
    DArr<int> beg, end;
    DArr<uint64_t> loff;
    HM_TRY(beg.alloc(ctx, n_rows));
    HM_TRY(end.alloc(ctx, n_rows));
    HM_TRY(loff.alloc(ctx, (size_t)n_rows + 1));
    HM_CUDA(cudaMemsetAsync(beg.p, 0, sizeof(int) * n_rows, st));
    HM_CUDA(cudaMemsetAsync(end.p, 0, sizeof(int) * n_rows, st));
    HM_CUDA(cudaMemsetAsync(loff.p, 0, sizeof(uint64_t) * ((size_t)n_rows + 1), st));
    k_chunk_emit<<<grid_for((uint64_t)n_rows * 32, kBlock), kBlock, 0, st>>>(
        beg.p, end.p, nullptr, d_rows, 0, n_rows, loff.p, zero.p, nullptr, base, g->h2h_off.p, g->h2h_len.p,
        g->h2h_nbr.p, g->h2h_ovl.p, g->h2h_mask.p);
    HM_LAUNCH_CHECK();
    return HM_OK;
  }
  uint64_t chunk_cap = std::min<uint64_t>(W, 1ull << 28);
  uint64_t max_row = 0;
  for (uint32_t r = 0; r < n_rows; ++r) max_row = std::max(max_row, hw[r + 1] - hw[r]);
  if (max_row >= (1ull << 31)) return set_error(HM_ERR_LIMIT, "H2H: one row has %llu wedges", (unsigned long long)max_row);
  chunk_cap = std::max(chunk_cap, max_row);
  DArr<uint32_t> kin, kout, starts, cnt;
  DArr<int> beg, end;
  DArr<uint64_t> loff;
  HM_TRY(kin.alloc(ctx, chunk_cap));
  HM_TRY(kout.alloc(ctx, chunk_cap));
  HM_TRY(starts.alloc(ctx, chunk_cap));
  HM_TRY(cnt.alloc(ctx, n_rows));
  HM_TRY(beg.alloc(ctx, n_rows));
  HM_TRY(end.alloc(ctx, n_rows));
  HM_TRY(loff.alloc(ctx, (size_t)n_rows + 1));
  DArr<uint8_t> sort_tmp;
  size_t sort_tb = 0;
  uint64_t out = 0;
  uint32_t r0 = 0;
  while (r0 < n_rows) {
    uint32_t r1 = r0;
    while (r1 < n_rows && hw[r1 + 1] - hw[r0] <= chunk_cap) ++r1;
    const uint32_t nrows = r1 - r0;
    const uint64_t cbase = hw[r0];
    const uint64_t nk = hw[r1] - cbase;
    k_expand<<<grid_for((uint64_t)nrows * 32, kBlock), kBlock, 0, st>>>(
        g->h2v_off.p, g->h2v_len.p, g->h2v_mem.p, g->v2h_off.p, g->v2h_len.p, g->v2h_edge.p, woff.p, d_rows, cbase,
        r0, r1, kin.p);
    HM_LAUNCH_CHECK();
    k_chunk_bounds<<<grid_for(nrows, kBlock), kBlock, 0, st>>>(woff.p, cbase, r0, r1, beg.p, end.p);
    HM_LAUNCH_CHECK();
    if (nk) {
      size_t tb = 0;
      HM_CUDA(cub::DeviceSegmentedSort::SortKeys(nullptr, tb, kin.p, kout.p, (int)nk, (int)nrows, beg.p, end.p, st));
      if (tb > sort_tb) {
        HM_TRY(sort_tmp.alloc(ctx, tb));
        sort_tb = tb;
      }
      HM_CUDA(cub::DeviceSegmentedSort::SortKeys(sort_tmp.p, tb, kin.p, kout.p, (int)nk, (int)nrows, beg.p, end.p,
                                                 st));
    }
    k_chunk_distinct<<<grid_for((uint64_t)nrows * 32, kBlock), kBlock, 0, st>>>(beg.p, end.p, kout.p, nrows, cnt.p);
    HM_LAUNCH_CHECK();
    HM_TRY(exclusive_scan(ctx, cnt.p, loff.p, nrows));
    k_chunk_starts<<<grid_for((uint64_t)nrows * 32, kBlock), kBlock, 0, st>>>(beg.p, end.p, kout.p, nrows, loff.p,
                                                                             starts.p);
    HM_LAUNCH_CHECK();
    k_chunk_emit<<<grid_for((uint64_t)nrows * 32, kBlock), kBlock, 0, st>>>(
        beg.p, end.p, kout.p, d_rows, r0, nrows, loff.p, cnt.p, starts.p, base + out, g->h2h_off.p, g->h2h_len.p,
        g->h2h_nbr.p, g->h2h_ovl.p, g->h2h_mask.p);
    HM_LAUNCH_CHECK();
    uint64_t chunk_total = 0;
    HM_CUDA(cudaMemcpyAsync(&chunk_total, loff.p + nrows, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    out += chunk_total;
    r0 = r1;
  }
  *written = out;
  return HM_OK;
}

int build_h2h_rows(hm_graph* g) {
  hm_ctx* ctx = g->ctx;
  const uint32_t E = g->n_slots;
  HM_TRY(g->h2h_off.alloc(ctx, (size_t)E + 1));
  HM_TRY(g->h2h_len.alloc(ctx, E));
  HM_CUDA(cudaMemsetAsync(g->h2h_len.p, 0, sizeof(uint32_t) * (E ? E : 1), ctx->stream));
  auto reserve = [&](uint64_t W, uint64_t* base) -> int {
    // the arena is sized by the wedge count, an upper bound on the entries
    HM_TRY(g->h2h_nbr.alloc(ctx, W));
    HM_TRY(g->h2h_ovl.alloc(ctx, W));
    HM_TRY(g->h2h_mask.alloc(ctx, W));
    g->h2h_cap = W;
    *base = 0;
    return HM_OK;
  };
  uint64_t written = 0;
  HM_TRY(h2h_rows_for(g, nullptr, E, reserve, &written));
  g->h2h_tail = written;
  g->h2h_nnz = written;
  return HM_OK;
}

// The long rows' lengths (0 for the others), per listed row (rows null: slots).
__global__ void k_long_len(const uint32_t* cnt, uint32_t n, uint32_t* llen) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    llen[i] = cnt[i] > kLongRow ? cnt[i] : 0u;
}

__global__ void k_long_scatter(const uint32_t* rows, uint32_t n, const uint64_t* lpos, uint64_t* loff) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    loff[rows[i]] = lpos[i];
}

// The long rows' mask offsets (per slot) and their mask array; returns its size.
static int long_rows(hm_ctx* ctx, const uint32_t* rows, uint32_t n, const uint32_t* cnt, uint32_t n_slots,
                     DArr<uint64_t>* loff, DArr<uint64_t>* lmask) {
  cudaStream_t st = ctx->stream;
  DArr<uint32_t> llen;
  DArr<uint64_t> lpos;
  HM_TRY(llen.alloc(ctx, n));
  HM_TRY(lpos.alloc(ctx, (size_t)n + 1));
  if (n) {
    k_long_len<<<grid_for(n, kBlock), kBlock, 0, st>>>(cnt, n, llen.p);
    HM_LAUNCH_CHECK();
  }
  HM_TRY(exclusive_scan(ctx, llen.p, lpos.p, n));
  uint64_t total = 0;
  HM_CUDA(cudaMemcpyAsync(&total, lpos.p + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  HM_TRY(lmask->alloc(ctx, total));
  if (!rows) {
    *loff = static_cast<DArr<uint64_t>&&>(lpos);
    return HM_OK;
  }
  HM_TRY(loff->alloc(ctx, (size_t)n_slots + 1));
  if (n) {
    k_long_scatter<<<grid_for(n, kBlock), kBlock, 0, st>>>(rows, n, lpos.p, loff->p);
    HM_LAUNCH_CHECK();
  }
  return HM_OK;
}

__global__ void k_plus_scatter(const uint32_t* rows, uint32_t n, const uint64_t* pos, const uint32_t* cnt,
                               uint64_t* poff, uint32_t* plen) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    poff[rows[i]] = pos[i];
    plen[rows[i]] = cnt[i];
  }
}

// Oriented rows of the listed slots only, in a set of their own (entries of
// other slots are not written). Enough for counts whose triangles stay among
// the listed slots, as a pooled graph's do.
int build_plus_rows(hm_graph* g, const uint32_t* d_rows, uint32_t n, PlusRows* P) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  DArr<uint32_t> cnt;
  DArr<uint64_t> pos;
  HM_TRY(cnt.alloc(ctx, n));
  HM_TRY(pos.alloc(ctx, (size_t)n + 1));
  HM_TRY(P->off.alloc(ctx, (size_t)g->n_slots + 1));
  HM_TRY(P->len.alloc(ctx, g->n_slots));
  if (n) {
    k_plus_count<<<grid_for((uint64_t)n * 32, kBlock), kBlock, 0, st>>>(g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p,
                                                                      d_rows, n, cnt.p);
    HM_LAUNCH_CHECK();
  }
  HM_TRY(exclusive_scan(ctx, cnt.p, pos.p, n));
  uint64_t total = 0;
  HM_CUDA(cudaMemcpyAsync(&total, pos.p + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  HM_TRY(P->nbr.alloc(ctx, total));
  HM_TRY(P->os.alloc(ctx, total));
  HM_TRY(long_rows(ctx, d_rows, n, cnt.p, g->n_slots, &P->loff, &P->lmask));
  if (n) {
    k_plus_scatter<<<grid_for(n, kBlock), kBlock, 0, st>>>(d_rows, n, pos.p, cnt.p, P->off.p, P->len.p);
    HM_LAUNCH_CHECK();
    k_plus_write<<<grid_for((uint64_t)n * 32, kBlock), kBlock, 0, st>>>(
        g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p, g->h2h_ovl.p, g->h2h_mask.p, g->esize.p, d_rows, n, P->off.p,
        P->len.p, P->loff.p, P->nbr.p, P->os.p, P->lmask.p);
    HM_LAUNCH_CHECK();
  }
  P->nnz = total;
  return HM_OK;
}

static int build_plus_once(hm_graph* g);

// Under memory pressure the H2H arena's free tail is given back and the
// build tried once more.
int build_plus(hm_graph* g) {
  const int s = build_plus_once(g);
  if (s != HM_ERR_NOMEM) return s;
  release_plus(g);
  HM_TRY(trim_h2h(g));
  return build_plus_once(g);
}

static int build_plus_once(hm_graph* g) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  const uint32_t E = g->n_slots;
  DArr<uint32_t> cnt;
  HM_TRY(cnt.alloc(ctx, E));
  if (E) {
    k_plus_count<<<grid_for((uint64_t)E * 32, kBlock), kBlock, 0, st>>>(g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p,
                                                                      nullptr, E, cnt.p);
    HM_LAUNCH_CHECK();
  }
  HM_TRY(g->plus_off.alloc(ctx, (size_t)E + 1));
  HM_TRY(exclusive_scan(ctx, cnt.p, g->plus_off.p, E));
  uint64_t total = 0;
  HM_CUDA(cudaMemcpyAsync(&total, g->plus_off.p + E, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  HM_TRY(g->plus_nbr.alloc(ctx, total));
  HM_TRY(g->plus_os.alloc(ctx, total));
  HM_TRY(long_rows(ctx, nullptr, E, cnt.p, E, &g->long_off, &g->long_mask));
  if (E) {
    k_plus_write<<<grid_for((uint64_t)E * 32, kBlock), kBlock, 0, st>>>(
        g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p, g->h2h_ovl.p, g->h2h_mask.p, g->esize.p, nullptr, E,
        g->plus_off.p, cnt.p, g->long_off.p, g->plus_nbr.p, g->plus_os.p, g->long_mask.p);
    HM_LAUNCH_CHECK();
  }
  g->plus_len = static_cast<DArr<uint32_t>&&>(cnt);
  g->plus_nnz = total;
  g->plus_valid = true;
  g->grp_valid = false;  // the grouped copy follows the rows it was built from
  return HM_OK;
}

}  // namespace hm
