// Batch updates of the device store and the exact incremental recount.
//
// Reference counterparts: deleteCBST / unfillCBST / insertCBST / fillCBST
// (dynamicHyperGraph/structure/operations.cu:82-356, 439-453) for the store,
// and computeMotifCountsDelta (dynamicHyperGraph/src/HMotifCountUpdate.cu:
// 228-301) for the recount. The reference updates H2V and V2H in place,
// rebuilds the whole updated graph on the host, never updates H2H on the
// device, and recounts closed triangles around "anchors" with a result that
// is only exact in special cases. Here:
//   * deletions clear the slot (lazy delete, like index = -1 in the CBST);
//   * insertions take the smallest free ids first, ascending, then new ids at
//     the end (the k-th free slot rule of insertIntoDeletedKth,
//     kernel/insert_reuse.cu:16-32), through a two-level free index: free
//     counts per 32-slot word, their prefix sums, then a bit select;
//   * H2V rows of inserted hyperedges are appended to the arena tail; V2H is
//     re-sorted from the live rows; H2H rows of inserted hyperedges are built
//     like at construction, and the rows of their neighbours and of the
//     deleted hyperedges' neighbours are rewritten by sort / merge / compact
//     into the arena tail (compacting the arena when it is full);
//   * the recount is exact by construction: delta = count of the triples that
//     touch an inserted hyperedge in the new graph minus count of the triples
//     that touch a deleted hyperedge in the old graph (a triple containing both
//     cannot exist in either graph), each counted on the device with the same
//     open/closed split as the static count, restricted to the touched part.
#include <cub/cub.cuh>

#include <algorithm>
#include <iterator>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "hm_classes.h"
#include "hm_device.h"

namespace hm {
namespace {

constexpr unsigned kWarp = 32;
constexpr unsigned kBlock = 256;
constexpr uint32_t kEmpty = 0xffffffffu;

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned lanemask_lt() { return (1u << lane_id()) - 1u; }
__device__ __forceinline__ uint64_t global_warp() { return ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ uint64_t n_warps() { return ((uint64_t)gridDim.x * blockDim.x) >> 5; }
__device__ __forceinline__ uint64_t gtid() { return (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint64_t gstride() { return (uint64_t)gridDim.x * blockDim.x; }

__device__ __forceinline__ uint64_t warp_sum(uint64_t v) {
  for (int d = 16; d; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  return v;
}

__device__ __forceinline__ bool is_live(const uint32_t* bits, uint32_t id) { return (bits[id >> 5] >> (id & 31)) & 1u; }

// ---- slots ----------------------------------------------------------------------

__global__ void k_check_live(const uint32_t* ids, uint32_t n, uint32_t n_slots, const uint32_t* bits, int* bad) {
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    const uint32_t id = ids[i];
    if (id >= n_slots || !is_live(bits, id)) atomicExch(bad, 1);
  }
}

// Ids that must be free (not live) before they are given to insertions.
__global__ void k_check_free(const uint32_t* ids, uint32_t n, uint32_t n_slots, const uint32_t* bits, int* bad) {
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    const uint32_t id = ids[i];
    if (id < n_slots && is_live(bits, id)) atomicExch(bad, 1);
  }
}

__global__ void k_set_u8(const uint32_t* ids, uint32_t n, uint8_t* flag, uint8_t v) {
  for (uint64_t i = gtid(); i < n; i += gstride()) flag[ids[i]] = v;
}

__global__ void k_delete_slots(const uint32_t* ids, uint32_t n, uint32_t* bits, uint8_t* esize, uint32_t* h2v_len,
                               uint32_t* h2h_len) {
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    const uint32_t id = ids[i];
    atomicAnd(&bits[id >> 5], ~(1u << (id & 31)));
    esize[id] = 0;
    h2v_len[id] = 0;
    h2h_len[id] = 0;
  }
}

__global__ void k_free_counts(const uint32_t* bits, uint32_t n_words, uint32_t n_slots, uint32_t* cnt) {
  for (uint64_t w = gtid(); w < n_words; w += gstride()) {
    uint32_t valid = 0xffffffffu;
    const uint64_t lo = w * 32;
    if (lo + 32 > n_slots) valid = (1u << (n_slots - lo)) - 1u;
    cnt[w] = __popc(~bits[w] & valid);
  }
}

// k-th insertion -> k-th free slot (ascending) while free slots last, then
// n_slots + (k - n_free).
__global__ void k_assign(uint32_t n_ins, uint64_t n_free, const uint64_t* prefix, const uint32_t* bits,
                         uint32_t n_words, uint32_t n_slots, uint32_t* out) {
  for (uint64_t k = gtid(); k < n_ins; k += gstride()) {
    if (k >= n_free) {
      out[k] = n_slots + (uint32_t)(k - n_free);
      continue;
    }
    uint32_t lo = 0, hi = n_words;  // last word with prefix <= k
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (prefix[mid] <= k) lo = mid;
      else hi = mid;
    }
    uint32_t r = (uint32_t)(k - prefix[lo]);
    uint32_t free_bits = ~bits[lo];
    for (uint32_t t = 0; t < r; ++t) free_bits &= free_bits - 1;  // drop the r lowest free bits
    out[k] = lo * 32 + (uint32_t)(__ffs(free_bits) - 1);
  }
}

__global__ void k_insert_slots(const uint32_t* ids, uint32_t n, const uint64_t* new_off, const uint32_t* new_len,
                               uint64_t tail, uint32_t* bits, uint8_t* esize, uint64_t* h2v_off, uint32_t* h2v_len) {
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    const uint32_t id = ids[i];
    atomicOr(&bits[id >> 5], 1u << (id & 31));
    esize[id] = (uint8_t)new_len[i];
    h2v_off[id] = tail + new_off[i];
    h2v_len[id] = new_len[i];
  }
}

__global__ void k_copy_u32(const uint32_t* src, uint64_t n, uint32_t* dst) {
  for (uint64_t i = gtid(); i < n; i += gstride()) dst[i] = src[i];
}

// ---- H2H patches -----------------------------------------------------------------
// A patch is (row b, neighbour id, op): op 0 removes the neighbour, op 1 adds
// it with an overlap and a position mask over b's members, op 2 (a removal
// and an addition of the same reused id) replaces the entry. Sort key:
// (b << 33) | (id << 1) | op.

__global__ void k_patch_removals(const uint32_t* dels, uint32_t n, const uint64_t* off, const uint32_t* len,
                                 const uint32_t* nbr, const uint64_t* out_off, uint64_t* keys, uint32_t* idx) {
  for (uint64_t i = global_warp(); i < n; i += n_warps()) {
    const uint32_t d = dels[i];
    const uint64_t s = off[d], o = out_off[i];
    const uint32_t l = len[d];
    for (uint32_t k = lane_id(); k < l; k += kWarp) {
      keys[o + k] = ((uint64_t)nbr[s + k] << 33) | ((uint64_t)d << 1);
      idx[o + k] = kEmpty;
    }
  }
}

// Additions from the fresh rows of inserted hyperedges to neighbours that
// were not inserted in this batch; the mask is over the neighbour's members.
__global__ void k_patch_additions(const uint32_t* ins, uint32_t n, const uint64_t* off, const uint32_t* len,
                                  const uint32_t* nbr, const uint8_t* ovl, const uint8_t* ins_mark,
                                  const uint64_t* hoff, const uint32_t* hmem, const uint8_t* esize,
                                  const uint64_t* out_off, uint64_t* keys, uint32_t* idx, uint8_t* povl,
                                  uint64_t* pmask) {
  for (uint64_t i = global_warp(); i < n; i += n_warps()) {
    const uint32_t a = ins[i];
    const uint64_t s = off[a];
    const uint32_t l = len[a];
    uint64_t o = out_off[i];
    const uint32_t* ma = hmem + hoff[a];
    const uint32_t sa = esize[a];
    for (uint32_t k0 = 0; k0 < l; k0 += kWarp) {
      const uint32_t k = k0 + lane_id();
      bool keep = false;
      uint32_t b = 0;
      if (k < l) {
        b = nbr[s + k];
        keep = !ins_mark[b];
      }
      const unsigned m = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        const uint64_t dst = o + __popc(m & lanemask_lt());
        // positions of b's members that a contains (a merge of the two lists)
        const uint32_t* mb = hmem + hoff[b];
        const uint32_t sb = esize[b];
        uint64_t mask = 0;
        uint32_t p = 0, q = 0;
        while (p < sb && q < sa) {
          if (mb[p] < ma[q]) ++p;
          else if (mb[p] > ma[q]) ++q;
          else {
            if (p < 64) mask |= 1ull << p;
            ++p;
            ++q;
          }
        }
        keys[dst] = ((uint64_t)b << 33) | ((uint64_t)a << 1) | 1ull;
        idx[dst] = (uint32_t)dst;
        povl[dst] = ovl[s + k];
        pmask[dst] = mask;
      }
      o += __popc(m);
    }
  }
}

// Marks patches to keep: drops patches of rows that are deleted or rebuilt in
// this batch, and folds (remove id, add id) into one replace.
__global__ void k_patch_fold(const uint64_t* keys, uint64_t n, const uint8_t* row_skip, uint32_t n_slots,
                             uint8_t* keep, uint8_t* op_out) {
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    const uint64_t k = keys[i];
    const uint32_t b = (uint32_t)(k >> 33);
    uint8_t op = (uint8_t)(k & 1);
    bool kp = b < n_slots && !row_skip[b];  // filler keys (all ones) fall outside
    if (kp && op == 0 && i + 1 < n && (keys[i + 1] >> 1) == (k >> 1)) kp = false;  // folded into the next
    if (kp && op == 1 && i > 0 && (keys[i - 1] >> 1) == (k >> 1)) op = 2;
    keep[i] = kp;
    op_out[i] = op;
  }
}

__global__ void k_patch_compact_flags(const uint8_t* keep, uint64_t n, uint32_t* f) {
  for (uint64_t i = gtid(); i < n; i += gstride()) f[i] = keep[i];
}

__global__ void k_patch_gather(const uint64_t* keys, const uint32_t* idx, const uint8_t* op, const uint8_t* keep,
                               const uint64_t* pos, uint64_t n, uint32_t* row, uint32_t* id, uint8_t* pop,
                               uint32_t* pidx) {
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    if (!keep[i]) continue;
    const uint64_t d = pos[i];
    row[d] = (uint32_t)(keys[i] >> 33);
    id[d] = (uint32_t)((keys[i] >> 1) & 0xffffffffu);
    pop[d] = op[i];
    pidx[d] = idx[i];
  }
}

// Per compacted patch: is it the first of its row; removal/addition counts
// before it within the row are done by scans on the host side of the kernel
// chain.
__global__ void k_patch_rowstart(const uint32_t* row, uint64_t n, uint32_t* flag) {
  for (uint64_t i = gtid(); i < n; i += gstride()) flag[i] = (i == 0 || row[i] != row[i - 1]);
}

struct RowPatch {
  uint32_t row;
  uint32_t p0, p1;  // patch range
};

__global__ void k_patch_rows(const uint32_t* row, const uint8_t* pop, uint64_t n, const uint64_t* start_pos,
                             const uint32_t* start_flag, RowPatch* rp, uint32_t* new_len, const uint32_t* h2h_len) {
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    if (!start_flag[i]) continue;
    const uint64_t r = start_pos[i];
    uint64_t e = i + 1;
    int32_t delta = 0;
    for (uint64_t k = i; k < n && (k == i || row[k] == row[i]); ++k) {
      delta += pop[k] == 1 ? 1 : (pop[k] == 0 ? -1 : 0);
      e = k + 1;
    }
    rp[r] = RowPatch{row[i], (uint32_t)i, (uint32_t)e};
    new_len[r] = (uint32_t)((int64_t)h2h_len[row[i]] + delta);
  }
}

// Rewrites one patched row (warp per row) at the arena tail: old entries
// minus removals, replaced entries updated, additions merged in id order.
// remx / addx are exclusive prefix counts of removals / additions over the
// compacted patch list.
__global__ void k_patch_apply(const RowPatch* rp, uint32_t n_rows, const uint64_t* dst_off, uint64_t tail,
                              const uint32_t* pid, const uint8_t* pop, const uint32_t* pidx, const uint64_t* remx,
                              const uint64_t* addx, const uint8_t* add_ovl, const uint64_t* add_mask,
                              uint64_t* h2h_off, const uint32_t* h2h_len, uint32_t* nbr, uint8_t* ovl,
                              uint64_t* mask) {
  for (uint64_t r = global_warp(); r < n_rows; r += n_warps()) {
    const RowPatch P = rp[r];
    const uint64_t so = h2h_off[P.row];
    const uint32_t sl = h2h_len[P.row];
    const uint64_t dst = tail + dst_off[r];
    const uint32_t np = P.p1 - P.p0;
    const uint64_t rem0 = remx[P.p0], add0 = addx[P.p0];
    // old entries: output rank = i - (removals with id < x) + (additions with id < x)
    for (uint32_t i = lane_id(); i < sl; i += kWarp) {
      const uint32_t x = nbr[so + i];
      uint32_t lo = 0, hi = np;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (pid[P.p0 + mid] < x) lo = mid + 1;
        else hi = mid;
      }
      const uint64_t rem = remx[P.p0 + lo] - rem0, add = addx[P.p0 + lo] - add0;
      uint8_t o_here = 3;
      if (lo < np && pid[P.p0 + lo] == x) o_here = pop[P.p0 + lo];
      if (o_here == 0) continue;
      const uint64_t d = dst + i - rem + add;
      nbr[d] = x;
      if (o_here == 2) {
        ovl[d] = add_ovl[pidx[P.p0 + lo]];
        mask[d] = add_mask[pidx[P.p0 + lo]];
      } else {
        ovl[d] = ovl[so + i];
        mask[d] = mask[so + i];
      }
    }
    // additions: output rank = (old entries with id < y) - (removals before) + (additions before)
    for (uint32_t k = lane_id(); k < np; k += kWarp) {
      if (pop[P.p0 + k] != 1) continue;
      const uint32_t y = pid[P.p0 + k];
      uint32_t lo = 0, hi = sl;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (nbr[so + mid] < y) lo = mid + 1;
        else hi = mid;
      }
      const uint64_t rem = remx[P.p0 + k] - rem0, add = addx[P.p0 + k] - add0;
      const uint64_t d = dst + lo - rem + add;
      nbr[d] = y;
      ovl[d] = add_ovl[pidx[P.p0 + k]];
      mask[d] = add_mask[pidx[P.p0 + k]];
    }
    __syncwarp();
    if (lane_id() == 0) h2h_off[P.row] = dst;
  }
}

__global__ void k_op_flags(const uint8_t* pop, uint64_t n, uint32_t* remf, uint32_t* addf) {
  for (uint64_t i = gtid(); i < n; i += gstride()) {
    remf[i] = pop[i] == 0;
    addf[i] = pop[i] == 1;
  }
}

__global__ void k_gather_u32(const uint32_t* ids, uint32_t n, const uint32_t* src, uint32_t* dst) {
  for (uint64_t i = gtid(); i < n; i += gstride()) dst[i] = src[ids[i]];
}

__global__ void k_set_lens(const RowPatch* rp, uint32_t n_rows, const uint32_t* new_len, uint32_t* h2h_len) {
  for (uint64_t r = gtid(); r < n_rows; r += gstride()) h2h_len[rp[r].row] = new_len[r];
}

// Arena compaction: every live row copied to its scanned position.
__global__ void k_compact_rows(const uint64_t* off, const uint32_t* len, uint32_t n, const uint64_t* new_off,
                               const uint32_t* nbr, const uint8_t* ovl, const uint64_t* mask, uint32_t* nnbr,
                               uint8_t* novl, uint64_t* nmask) {
  for (uint64_t r = global_warp(); r < n; r += n_warps()) {
    const uint64_t s = off[r], d = new_off[r];
    const uint32_t l = len[r];
    for (uint32_t k = lane_id(); k < l; k += kWarp) {
      nnbr[d + k] = nbr[s + k];
      novl[d + k] = ovl[s + k];
      nmask[d + k] = mask[s + k];
    }
  }
}

__global__ void k_compact_members(const uint64_t* off, const uint32_t* len, uint32_t n, const uint64_t* new_off,
                                  const uint32_t* mem, uint32_t* nmem) {
  for (uint64_t r = global_warp(); r < n; r += n_warps()) {
    const uint64_t s = off[r], d = new_off[r];
    for (uint32_t k = lane_id(); k < len[r]; k += kWarp) nmem[d + k] = mem[s + k];
  }
}

__global__ void k_arena_keys(const uint64_t* off, uint32_t n, uint64_t* key, uint32_t* slot) {
  for (uint64_t r = gtid(); r < n; r += gstride()) {
    key[r] = off[r];
    slot[r] = (uint32_t)r;
  }
}

// phase 0: rows -> staging buffer (positions relative to base);
// phase 1: staging -> final position, and the row offset is updated.
__global__ void k_stage_rows(const uint32_t* slots, uint32_t n, uint64_t* off, const uint32_t* len,
                             const uint64_t* dst, uint64_t base, uint32_t* nbr, uint8_t* ovl, uint64_t* mask,
                             uint32_t* snbr, uint8_t* sovl, uint64_t* smask, int phase) {
  for (uint64_t i = global_warp(); i < n; i += n_warps()) {
    const uint32_t r = slots[i];
    const uint32_t l = len[r];
    const uint64_t t = dst[i] - base;
    if (phase == 0) {
      const uint64_t s = off[r];
      for (uint32_t k = lane_id(); k < l; k += kWarp) {
        snbr[t + k] = nbr[s + k];
        sovl[t + k] = ovl[s + k];
        smask[t + k] = mask[s + k];
      }
    } else {
      const uint64_t d = dst[i];
      for (uint32_t k = lane_id(); k < l; k += kWarp) {
        nbr[d + k] = snbr[t + k];
        ovl[d + k] = sovl[t + k];
        mask[d + k] = smask[t + k];
      }
      if (lane_id() == 0) off[r] = d;
    }
  }
}

__global__ void k_set_off(const uint64_t* new_off, uint32_t n, uint64_t* off) {
  for (uint64_t r = gtid(); r < n; r += gstride()) off[r] = new_off[r];
}

__global__ void k_sum_u32(const uint32_t* x, uint32_t n, unsigned long long* out) {
  uint64_t s = 0;
  for (uint64_t i = gtid(); i < n; i += gstride()) s += x[i];
  s = warp_sum(s);
  if (lane_id() == 0 && s) atomicAdd(out, (unsigned long long)s);
}

template <class T>
int grow(hm_ctx* ctx, DArr<T>& a, size_t need, size_t keep, bool zero_new) {
  if (a.n >= need && a.p) return HM_OK;
  size_t cap = std::max<size_t>(need, a.n + a.n / 4 + 1024);
  DArr<T> b;
  HM_TRY(b.alloc(ctx, cap));
  if (keep) HM_CUDA(cudaMemcpyAsync(b.p, a.p, keep * sizeof(T), cudaMemcpyDeviceToDevice, ctx->stream));
  if (zero_new && cap > keep) HM_CUDA(cudaMemsetAsync(b.p + keep, 0, (cap - keep) * sizeof(T), ctx->stream));
  a = static_cast<DArr<T>&&>(b);
  return HM_OK;
}

}  // namespace

// Slot arrays hold at least need slots (new slots zeroed = free, empty).
static int ensure_slots(hm_graph* g, uint32_t need) {
  hm_ctx* ctx = g->ctx;
  const uint32_t n = g->n_slots;
  HM_TRY(grow(ctx, g->esize, need, n, true));
  HM_TRY(grow(ctx, g->h2v_len, need, n, true));
  HM_TRY(grow(ctx, g->h2h_len, need, n, true));
  HM_TRY(grow(ctx, g->h2v_off, (size_t)need + 1, (size_t)n + 1, true));
  HM_TRY(grow(ctx, g->h2h_off, (size_t)need + 1, (size_t)n + 1, true));
  HM_TRY(grow(ctx, g->live_bits, (need + 31) / 32, (n + 31) / 32, true));
  return HM_OK;
}

// Re-packs the H2H arena so that the live rows are contiguous, leaving room
// for extra more entries.
// Moves the live H2H rows to the front of the arena, in place: rows are
// taken in arena order and moved in rounds through a bounded staging buffer;
// each row only moves towards the front, and every round reads its rows
// before writing them, so no row is overwritten before it is read.
static int compact_h2h_in_place(hm_graph* g) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  const uint32_t E = g->n_slots;
  if (!E) {
    g->h2h_tail = 0;
    return HM_OK;
  }
  // slots in arena order (empty rows sort anywhere; they move nothing)
  DArr<uint64_t> key, key_s;
  DArr<uint32_t> slot, slot_s, len_s;
  HM_TRY(key.alloc(ctx, E));
  HM_TRY(key_s.alloc(ctx, E));
  HM_TRY(slot.alloc(ctx, E));
  HM_TRY(slot_s.alloc(ctx, E));
  HM_TRY(len_s.alloc(ctx, E));
  k_arena_keys<<<grid_for(E, kBlock), kBlock, 0, st>>>(g->h2h_off.p, E, key.p, slot.p);
  HM_LAUNCH_CHECK();
  {
    size_t tb = 0;
    HM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, key.p, key_s.p, slot.p, slot_s.p, (int64_t)E, 0, 64, st));
    DArr<uint8_t> tmp;
    HM_TRY(tmp.alloc(ctx, tb));
    HM_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, key.p, key_s.p, slot.p, slot_s.p, (int64_t)E, 0, 64, st));
  }
  k_gather_u32<<<grid_for(E, kBlock), kBlock, 0, st>>>(slot_s.p, E, g->h2h_len.p, len_s.p);
  HM_LAUNCH_CHECK();
  DArr<uint64_t> noff;
  HM_TRY(noff.alloc(ctx, (size_t)E + 1));
  HM_TRY(exclusive_scan(ctx, len_s.p, noff.p, E));
  std::vector<uint64_t> h((size_t)E + 1);
  HM_CUDA(cudaMemcpyAsync(h.data(), noff.p, sizeof(uint64_t) * ((size_t)E + 1), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  const uint64_t live = h[E];
  uint64_t stage_cap = std::min<uint64_t>(std::max<uint64_t>(live, 1), 1ull << 28);
  uint64_t max_row = 0;
  for (uint32_t r = 0; r < E; ++r) max_row = std::max(max_row, h[r + 1] - h[r]);
  stage_cap = std::max(stage_cap, max_row);
  DArr<uint32_t> snbr;
  DArr<uint8_t> sovl;
  DArr<uint64_t> smask;
  HM_TRY(snbr.alloc(ctx, stage_cap));
  HM_TRY(sovl.alloc(ctx, stage_cap));
  HM_TRY(smask.alloc(ctx, stage_cap));
  uint32_t r0 = 0;
  while (r0 < E) {
    uint32_t r1 = r0;
    while (r1 < E && h[r1 + 1] - h[r0] <= stage_cap) ++r1;
    const uint32_t n = r1 - r0;
    for (int phase = 0; phase < 2; ++phase) {
      k_stage_rows<<<grid_for((uint64_t)n * 32, kBlock), kBlock, 0, st>>>(
          slot_s.p + r0, n, g->h2h_off.p, g->h2h_len.p, noff.p + r0, h[r0], g->h2h_nbr.p, g->h2h_ovl.p,
          g->h2h_mask.p, snbr.p, sovl.p, smask.p, phase);
      HM_LAUNCH_CHECK();
    }
    r0 = r1;
  }
  g->h2h_tail = live;
  return HM_OK;
}

// Grows the arena to cap entries in place (more physical memory mapped after
// the rows; nothing is copied and no second arena is held).
static int grow_h2h(hm_graph* g, uint64_t cap) {
  hm_ctx* ctx = g->ctx;
  cap = std::max<uint64_t>(cap, g->h2h_tail + 1024);
  // all three arrays or none: a partial grow would hold memory the arena
  // cannot use
  auto more = [cap](size_t have, size_t width) { return cap > have ? (cap - have) * width : 0; };
  const size_t bytes = more(g->h2h_nbr.n, 4) + more(g->h2h_ovl.n, 1) + more(g->h2h_mask.n, 8);
  if (ctx->budget && ctx->used.load() + bytes + (8u << 20) > ctx->budget)
    return set_error(HM_ERR_NOMEM, "H2H arena growth to %llu entries exceeds the device budget",
                     (unsigned long long)cap);
  HM_TRY(g->h2h_nbr.grow(ctx, cap));
  HM_TRY(g->h2h_ovl.grow(ctx, cap));
  HM_TRY(g->h2h_mask.grow(ctx, cap));
  g->h2h_cap = std::min(std::min(g->h2h_nbr.n, g->h2h_ovl.n), g->h2h_mask.n);
  return HM_OK;
}

// Called when the arena tail runs out: drops the oriented copy (rebuilt on
// demand), compacts in place, and grows the arena in place when the live
// rows leave too little room (a batch on a hub-heavy graph rewrites most
// rows, in chunks that each need free tail).
static int compact_h2h(hm_graph* g, uint64_t extra) {
  hm_ctx* ctx = g->ctx;
  release_plus(g);
  HM_TRY(compact_h2h_in_place(g));
  const uint64_t live = g->h2h_tail;
  // Keep about half the live size free after a compaction (at most a tenth
  // of the budget), so that a batch needs few of them, but leave the device
  // room for what the store needs besides the arena: the oriented copy of a
  // count (6 bytes for each of about live / 2 entries), a batch's scratch
  // and the stream-ordered pool's slack (a sixteenth of the budget). Under
  // that pressure the arena only grows to the least that serves this
  // request (later batches compact more often).
  uint64_t slack = live / 2;
  if (ctx->budget) slack = std::min<uint64_t>(slack, ctx->budget / 10 / 13);
  if (live + std::max<uint64_t>(extra, slack) <= g->h2h_cap) return HM_OK;
  const uint64_t lean = live + extra + (live + extra) / 32 + 1024;
  uint64_t want = std::max<uint64_t>(live + slack, live + extra + (live + extra) / 8) + 1024;
  if (ctx->budget) {
    const size_t arena = g->h2h_nbr.bytes() + g->h2h_ovl.bytes() + g->h2h_mask.bytes();
    const size_t other = ctx->used.load() - std::min<size_t>(ctx->used.load(), arena);
    const size_t reserve = (size_t)(live / 2) * 6 + ctx->budget / 16;
    const size_t room = ctx->budget > other + reserve ? ctx->budget - other - reserve : 0;
    want = std::min<uint64_t>(want, room / 13);
  }
  const uint64_t keep = std::max(want, lean);
  if (keep + (keep >> 4) < g->h2h_cap) {  // grown before the pressure: give the excess back
    g->h2h_nbr.shrink(keep);
    g->h2h_ovl.shrink(keep);
    g->h2h_mask.shrink(keep);
    g->h2h_cap = std::min(std::min(g->h2h_nbr.n, g->h2h_ovl.n), g->h2h_mask.n);
  }
  if (want <= g->h2h_cap && live + extra <= g->h2h_cap) return HM_OK;
  const int s = grow_h2h(g, keep);
  if (s != HM_ERR_NOMEM || want <= lean) return s;
  if (live + extra <= g->h2h_cap) return HM_OK;
  return grow_h2h(g, lean);
}

// Gives the arena's free tail back to the device (compaction first), keeping
// room for about 1/64 of the live entries; for callers about to allocate
// under memory pressure.
int trim_h2h(hm_graph* g) {
  if (g->h2h_cap - g->h2h_nnz < (g->h2h_nnz >> 5) + (1u << 20)) return HM_OK;
  HM_TRY(compact_h2h_in_place(g));
  const uint64_t keep = g->h2h_tail + (g->h2h_tail >> 6) + 1024;
  g->h2h_nbr.shrink(keep);
  g->h2h_ovl.shrink(keep);
  g->h2h_mask.shrink(keep);
  g->h2h_cap = std::min(std::min(g->h2h_nbr.n, g->h2h_ovl.n), g->h2h_mask.n);
  return HM_OK;
}

// Grows the H2H arena to `factor` times the live entries (the first batch
// would grow it to twice), so that a store about to take a stream of batches
// pays for the growth up front.
int presize_h2h(hm_graph* g, uint32_t factor) {
  const uint64_t want = (uint64_t)factor * g->h2h_nnz + 1024;
  if (g->h2h_cap >= want) return HM_OK;
  HM_TRY(compact_h2h_in_place(g));
  return grow_h2h(g, want);
}

// Room for n more entries at the H2H arena tail; returns the position.
static int reserve_h2h(hm_graph* g, uint64_t n, uint64_t* base) {
  if (g->h2h_tail + n > g->h2h_cap) HM_TRY(compact_h2h(g, n));
  *base = g->h2h_tail;
  g->h2h_tail += n;
  return HM_OK;
}

static int compact_h2v(hm_graph* g, uint64_t extra) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  const uint32_t E = g->n_slots;
  DArr<uint64_t> noff;
  HM_TRY(noff.alloc(ctx, (size_t)E + 1));
  HM_TRY(exclusive_scan(ctx, g->h2v_len.p, noff.p, E));
  uint64_t live = 0;
  HM_CUDA(cudaMemcpyAsync(&live, noff.p + E, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  const uint64_t cap = live + extra + (live + extra) / 4 + 1024;
  DArr<uint32_t> nmem;
  HM_TRY(nmem.alloc(ctx, cap));
  if (E) {
    k_compact_members<<<grid_for((uint64_t)E * 32, kBlock), kBlock, 0, st>>>(g->h2v_off.p, g->h2v_len.p, E, noff.p,
                                                                           g->h2v_mem.p, nmem.p);
    HM_LAUNCH_CHECK();
    k_set_off<<<grid_for(E, kBlock), kBlock, 0, st>>>(noff.p, E, g->h2v_off.p);
    HM_LAUNCH_CHECK();
  }
  g->h2v_mem = static_cast<DArr<uint32_t>&&>(nmem);
  g->h2v_tail = live;
  return HM_OK;
}

// Per-phase wall times of one batch, printed to stderr when HM_TRACE is set
// in the environment (each mark synchronises the stream; diagnostics only).
struct PhaseTrace {
  cudaStream_t st;
  bool on;
  std::chrono::steady_clock::time_point t0;
  std::string out;
  explicit PhaseTrace(cudaStream_t s) : st(s), on(std::getenv("HM_TRACE") != nullptr) {
    if (on) {
      cudaStreamSynchronize(st);
      t0 = std::chrono::steady_clock::now();
    }
  }
  void mark(const char* name) {
    if (!on) return;
    cudaStreamSynchronize(st);
    const auto t = std::chrono::steady_clock::now();
    char buf[96];
    std::snprintf(buf, sizeof(buf), " %s=%.1fms", name, std::chrono::duration<double, std::milli>(t - t0).count());
    out += buf;
    t0 = t;
  }
  ~PhaseTrace() {
    if (on) std::fprintf(stderr, "[hm_trace apply_batch]%s\n", out.c_str());
  }
};

// Deletes and inserts; hooks.before sees the old graph and the deleted slots,
// hooks.after the new graph and the assigned slots (both device arrays). All
// device work; the host only sequences the kernels.
int apply_batch_hooks(hm_graph* g, const uint32_t* h_dels, uint32_t n_del, const uint64_t* h_ins_off,
                      const uint32_t* h_ins_mem, uint32_t n_ins, uint32_t* assigned_out, const BatchHooks& hooks,
                      const uint32_t* forced_ids) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  if (g->temporal) return set_error(HM_ERR_STATE, "apply_batch: temporal graphs are immutable");
  {
    std::vector<uint32_t> tmp(h_dels, h_dels + n_del);
    std::sort(tmp.begin(), tmp.end());
    if (std::adjacent_find(tmp.begin(), tmp.end()) != tmp.end())
      return set_error(HM_ERR_INVALID, "apply_batch: a hyperedge id is deleted twice");
  }
  uint32_t forced_max = 0;
  if (forced_ids && n_ins) {
    std::vector<uint32_t> tmp(forced_ids, forced_ids + n_ins);
    std::sort(tmp.begin(), tmp.end());
    if (std::adjacent_find(tmp.begin(), tmp.end()) != tmp.end())
      return set_error(HM_ERR_INVALID, "apply_batch: an id is given to two insertions");
    forced_max = tmp.back();
    if ((uint64_t)forced_max + 1 >= (1ull << 24))
      return set_error(HM_ERR_LIMIT, "apply_batch: id %u beyond the 2^24 slot limit", forced_max);
  }
  if (n_ins) {
    if (h_ins_off[0] != 0) return set_error(HM_ERR_INVALID, "apply_batch: insert offsets must start at 0");
    for (uint32_t e = 0; e < n_ins; ++e)
      if (h_ins_off[e + 1] < h_ins_off[e]) return set_error(HM_ERR_INVALID, "apply_batch: insert offsets decrease");
  }
  cudaEvent_t e0, e1;
  HM_CUDA(cudaEventCreate(&e0));
  HM_CUDA(cudaEventCreate(&e1));
  HM_CUDA(cudaEventRecord(e0, st));
  DArr<uint32_t> dels;
  DArr<int> bad;
  HM_TRY(dels.alloc(ctx, n_del));
  HM_TRY(bad.alloc(ctx, 1));
  HM_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
  if (n_del) {
    HM_CUDA(cudaMemcpyAsync(dels.p, h_dels, sizeof(uint32_t) * n_del, cudaMemcpyHostToDevice, st));
    k_check_live<<<grid_for(n_del, kBlock), kBlock, 0, st>>>(dels.p, n_del, g->n_slots, g->live_bits.p, bad.p);
    HM_LAUNCH_CHECK();
  }
  int hbad = 0;
  HM_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  if (hbad) return set_error(HM_ERR_NOT_LIVE, "apply_batch: a deleted id is not a live hyperedge");
  // the static count's grouped rows die with this batch; their memory is
  // better spent on the batch's own scratch
  release_plus_groups(g);

  // normalised inserted member lists (sorted, unique) via a scratch graph
  hm_graph ins;
  ins.ctx = ctx;
  ins.n_nodes = g->n_nodes;
  static const uint64_t zero_off = 0;
  HM_TRY(build_h2v(&ins, n_ins ? h_ins_off : &zero_off, h_ins_mem, n_ins));

  PhaseTrace trace(st);
  trace.mark("validate");
  if (hooks.before) HM_TRY(hooks.before(dels.p, n_del));
  trace.mark("count_deleted");
  release_plus(g);  // the old graph's oriented rows: not used again, and the patching needs the room

  // ---- deletions: H2H removal patches from the rows about to vanish ----------
  DArr<uint64_t> rem_off;
  DArr<uint32_t> rem_len;
  HM_TRY(rem_len.alloc(ctx, n_del));
  HM_TRY(rem_off.alloc(ctx, (size_t)n_del + 1));
  if (n_del) {
    k_gather_u32<<<grid_for(n_del, kBlock), kBlock, 0, st>>>(dels.p, n_del, g->h2h_len.p, rem_len.p);
    HM_LAUNCH_CHECK();
  }
  HM_TRY(exclusive_scan(ctx, rem_len.p, rem_off.p, n_del));
  uint64_t n_rem = 0;
  HM_CUDA(cudaMemcpyAsync(&n_rem, rem_off.p + n_del, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  DArr<uint64_t> pkeys;
  DArr<uint32_t> pidx;
  if (n_rem) {
    HM_TRY(pkeys.alloc(ctx, n_rem));
    HM_TRY(pidx.alloc(ctx, n_rem));
    k_patch_removals<<<grid_for((uint64_t)n_del * 32, kBlock), kBlock, 0, st>>>(
        dels.p, n_del, g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p, rem_off.p, pkeys.p, pidx.p);
    HM_LAUNCH_CHECK();
  }
  if (n_del) {
    k_delete_slots<<<grid_for(n_del, kBlock), kBlock, 0, st>>>(dels.p, n_del, g->live_bits.p, g->esize.p,
                                                                g->h2v_len.p, g->h2h_len.p);
    HM_LAUNCH_CHECK();
  }

  // ---- assign ids: smallest free slots first, then new slots (or the ids
  // the caller gives, which must be free once the deletions are done) -----------
  const uint32_t words = (g->n_slots + 31) / 32;
  DArr<uint32_t> fcnt, ids;
  DArr<uint64_t> fpre;
  HM_TRY(ids.alloc(ctx, n_ins));
  uint32_t new_slots = g->n_slots;
  if (forced_ids) {
    if (n_ins) {
      HM_CUDA(cudaMemcpyAsync(ids.p, forced_ids, sizeof(uint32_t) * n_ins, cudaMemcpyHostToDevice, st));
      HM_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
      k_check_free<<<grid_for(n_ins, kBlock), kBlock, 0, st>>>(ids.p, n_ins, g->n_slots, g->live_bits.p, bad.p);
      HM_LAUNCH_CHECK();
      HM_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
      HM_CUDA(cudaStreamSynchronize(st));
      // the deletions already ran: the store is changed, so this is a caller
      // error the entry points rule out before calling (ids they give are the
      // ones they delete)
      if (hbad) return set_error(HM_ERR_INVALID, "apply_batch: an insertion's id is in use");
      new_slots = std::max(new_slots, forced_max + 1);
    }
  } else {
    HM_TRY(fcnt.alloc(ctx, words));
    HM_TRY(fpre.alloc(ctx, (size_t)words + 1));
    if (words) {
      k_free_counts<<<grid_for(words, kBlock), kBlock, 0, st>>>(g->live_bits.p, words, g->n_slots, fcnt.p);
      HM_LAUNCH_CHECK();
    }
    HM_TRY(exclusive_scan(ctx, fcnt.p, fpre.p, words));
    uint64_t n_free = 0;
    HM_CUDA(cudaMemcpyAsync(&n_free, fpre.p + words, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    if (n_ins) {
      k_assign<<<grid_for(n_ins, kBlock), kBlock, 0, st>>>(n_ins, n_free, fpre.p, g->live_bits.p, words, g->n_slots,
                                                            ids.p);
      HM_LAUNCH_CHECK();
    }
    new_slots = g->n_slots + (n_ins > n_free ? (uint32_t)(n_ins - n_free) : 0u);
  }
  if ((uint64_t)new_slots >= (1ull << 24))
    return set_error(HM_ERR_LIMIT, "apply_batch: %u hyperedge slots exceed the 2^24 limit", new_slots);
  HM_TRY(ensure_slots(g, new_slots));
  DArr<uint8_t> povl;
  DArr<uint64_t> pmask;

  // ---- insertions: H2V rows appended ------------------------------------------
  const uint64_t ins_members = ins.h2v_tail;
  if (g->h2v_tail + ins_members > g->h2v_mem.n) HM_TRY(compact_h2v(g, ins_members));
  if (g->h2v_tail + ins_members > g->h2v_mem.n) HM_TRY(grow(ctx, g->h2v_mem, g->h2v_tail + ins_members, g->h2v_tail, false));
  const uint64_t h2v_base = g->h2v_tail;
  if (ins_members) {
    k_copy_u32<<<grid_for(ins_members, kBlock), kBlock, 0, st>>>(ins.h2v_mem.p, ins_members, g->h2v_mem.p + h2v_base);
    HM_LAUNCH_CHECK();
  }
  g->n_slots = new_slots;
  if (n_ins) {
    k_insert_slots<<<grid_for(n_ins, kBlock), kBlock, 0, st>>>(ids.p, n_ins, ins.h2v_off.p, ins.h2v_len.p, h2v_base,
                                                                g->live_bits.p, g->esize.p, g->h2v_off.p,
                                                                g->h2v_len.p);
    HM_LAUNCH_CHECK();
  }
  g->h2v_tail += ins_members;
  g->h2v_nnz = g->h2v_nnz + ins_members;  // deleted members are subtracted below
  g->n_live = g->n_live - n_del + n_ins;

  trace.mark("delete_assign_h2v");
  // ---- V2H from the live rows -----------------------------------------------------
  HM_TRY(build_v2h(g));
  trace.mark("v2h");

  // ---- H2H: fresh rows for the inserted ids -------------------------------------
  DArr<uint8_t> ins_mark, skip;
  HM_TRY(ins_mark.alloc(ctx, new_slots));
  HM_TRY(skip.alloc(ctx, new_slots));
  HM_CUDA(cudaMemsetAsync(ins_mark.p, 0, new_slots, st));
  if (n_ins) {
    k_set_u8<<<grid_for(n_ins, kBlock), kBlock, 0, st>>>(ids.p, n_ins, ins_mark.p, 1);
    HM_LAUNCH_CHECK();
  }
  HM_CUDA(cudaMemcpyAsync(skip.p, ins_mark.p, new_slots, cudaMemcpyDeviceToDevice, st));
  if (n_del) {
    k_set_u8<<<grid_for(n_del, kBlock), kBlock, 0, st>>>(dels.p, n_del, skip.p, 1);
    HM_LAUNCH_CHECK();
    // a deleted id that was reused is rebuilt, not skipped-as-dead: both skip
  }
  uint64_t written = 0;
  if (n_ins) {
    auto reserve = [&](uint64_t W, uint64_t* base) { return reserve_h2h(g, W, base); };
    HM_TRY(h2h_rows_for(g, ids.p, n_ins, reserve, &written));
  }

  trace.mark("h2h_inserted_rows");
  // ---- H2H addition patches ---------------------------------------------------
  DArr<uint32_t> ilen;
  DArr<uint64_t> ioff;
  HM_TRY(ilen.alloc(ctx, n_ins));
  HM_TRY(ioff.alloc(ctx, (size_t)n_ins + 1));
  uint64_t n_add_max = 0;
  if (n_ins) {
    k_gather_u32<<<grid_for(n_ins, kBlock), kBlock, 0, st>>>(ids.p, n_ins, g->h2h_len.p, ilen.p);
    HM_LAUNCH_CHECK();
    if (assigned_out) HM_CUDA(cudaMemcpyAsync(assigned_out, ids.p, sizeof(uint32_t) * n_ins, cudaMemcpyDeviceToHost, st));
  }
  HM_TRY(exclusive_scan(ctx, ilen.p, ioff.p, n_ins));
  HM_CUDA(cudaMemcpyAsync(&n_add_max, ioff.p + n_ins, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  const uint64_t n_patch = n_rem + n_add_max;
  if (n_patch) {
    DArr<uint64_t> keys;
    DArr<uint32_t> idx;
    HM_TRY(keys.alloc(ctx, n_patch));
    HM_TRY(idx.alloc(ctx, n_patch));
    HM_TRY(povl.alloc(ctx, n_patch));
    HM_TRY(pmask.alloc(ctx, n_patch));
    // unused addition slots (neighbours that were inserted too) become
    // removals of an impossible id in a skipped row: mark them skip
    HM_CUDA(cudaMemsetAsync(keys.p + n_rem, 0xff, sizeof(uint64_t) * n_add_max, st));
    if (n_rem) {
      HM_CUDA(cudaMemcpyAsync(keys.p, pkeys.p, sizeof(uint64_t) * n_rem, cudaMemcpyDeviceToDevice, st));
      HM_CUDA(cudaMemcpyAsync(idx.p, pidx.p, sizeof(uint32_t) * n_rem, cudaMemcpyDeviceToDevice, st));
    }
    if (n_ins) {
      k_patch_additions<<<grid_for((uint64_t)n_ins * 32, kBlock), kBlock, 0, st>>>(
          ids.p, n_ins, g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p, g->h2h_ovl.p, ins_mark.p, g->h2v_off.p,
          g->h2v_mem.p, g->esize.p, ioff.p, keys.p + n_rem, idx.p + n_rem, povl.p + n_rem, pmask.p + n_rem);
      HM_LAUNCH_CHECK();
    }
    // additions index their payload by absolute patch position
    DArr<uint64_t> skeys;
    DArr<uint32_t> sidx;
    HM_TRY(skeys.alloc(ctx, n_patch));
    HM_TRY(sidx.alloc(ctx, n_patch));
    {
      // payload index of an addition: shift by n_rem
      size_t tb = 0;
      HM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.p, skeys.p, idx.p, sidx.p, (int64_t)n_patch, 0, 64,
                                              st));
      DArr<uint8_t> tmp;
      HM_TRY(tmp.alloc(ctx, tb));
      HM_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, keys.p, skeys.p, idx.p, sidx.p, (int64_t)n_patch, 0, 64, st));
    }
    trace.mark("patch_sort");
    // rows of deleted or rebuilt ids, and the all-ones filler keys, are skipped
    DArr<uint8_t> keep, op;
    HM_TRY(keep.alloc(ctx, n_patch));
    HM_TRY(op.alloc(ctx, n_patch));
    DArr<uint8_t> skip_ext;
    HM_TRY(skip_ext.alloc(ctx, (size_t)std::max<uint32_t>(new_slots, 1) + 1));
    HM_CUDA(cudaMemcpyAsync(skip_ext.p, skip.p, new_slots, cudaMemcpyDeviceToDevice, st));
    // filler key row = 0x7fffffff (>> 33 of all ones): outside the slot range
    k_patch_fold<<<grid_for(n_patch, kBlock), kBlock, 0, st>>>(skeys.p, n_patch, skip_ext.p, new_slots, keep.p,
                                                                op.p);
    HM_LAUNCH_CHECK();
    (void)0;
    // compaction of kept patches
    DArr<uint32_t> kf;
    DArr<uint64_t> kpos;
    HM_TRY(kf.alloc(ctx, n_patch));
    HM_TRY(kpos.alloc(ctx, n_patch + 1));
    k_patch_compact_flags<<<grid_for(n_patch, kBlock), kBlock, 0, st>>>(keep.p, n_patch, kf.p);
    HM_LAUNCH_CHECK();
    HM_TRY(exclusive_scan(ctx, kf.p, kpos.p, n_patch));
    uint64_t n_kept = 0;
    HM_CUDA(cudaMemcpyAsync(&n_kept, kpos.p + n_patch, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    HM_CUDA(cudaStreamSynchronize(st));
    if (n_kept) {
      DArr<uint32_t> prow, pid, ppidx;
      DArr<uint8_t> pop;
      HM_TRY(prow.alloc(ctx, n_kept));
      HM_TRY(pid.alloc(ctx, n_kept));
      HM_TRY(ppidx.alloc(ctx, n_kept));
      HM_TRY(pop.alloc(ctx, n_kept));
      k_patch_gather<<<grid_for(n_patch, kBlock), kBlock, 0, st>>>(skeys.p, sidx.p, op.p, keep.p, kpos.p, n_patch,
                                                                    prow.p, pid.p, pop.p, ppidx.p);
      HM_LAUNCH_CHECK();
      // the payload index of additions is relative to the addition block
      DArr<uint32_t> sflag;
      DArr<uint64_t> spos;
      HM_TRY(sflag.alloc(ctx, n_kept));
      HM_TRY(spos.alloc(ctx, n_kept + 1));
      k_patch_rowstart<<<grid_for(n_kept, kBlock), kBlock, 0, st>>>(prow.p, n_kept, sflag.p);
      HM_LAUNCH_CHECK();
      HM_TRY(exclusive_scan(ctx, sflag.p, spos.p, n_kept));
      uint64_t n_rows = 0;
      HM_CUDA(cudaMemcpyAsync(&n_rows, spos.p + n_kept, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
      HM_CUDA(cudaStreamSynchronize(st));
      DArr<RowPatch> rp;
      DArr<uint32_t> nlen;
      DArr<uint64_t> noff;
      HM_TRY(rp.alloc(ctx, n_rows));
      HM_TRY(nlen.alloc(ctx, n_rows));
      HM_TRY(noff.alloc(ctx, n_rows + 1));
      k_patch_rows<<<grid_for(n_kept, kBlock), kBlock, 0, st>>>(prow.p, pop.p, n_kept, spos.p, sflag.p, rp.p, nlen.p,
                                                                 g->h2h_len.p);
      HM_LAUNCH_CHECK();
      HM_TRY(exclusive_scan(ctx, nlen.p, noff.p, n_rows));
      uint64_t need = 0;
      HM_CUDA(cudaMemcpyAsync(&need, noff.p + n_rows, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
      HM_CUDA(cudaStreamSynchronize(st));
      DArr<uint32_t> remf, addf;
      DArr<uint64_t> remx, addx;
      HM_TRY(remf.alloc(ctx, n_kept));
      HM_TRY(addf.alloc(ctx, n_kept));
      HM_TRY(remx.alloc(ctx, n_kept + 1));
      HM_TRY(addx.alloc(ctx, n_kept + 1));
      k_op_flags<<<grid_for(n_kept, kBlock), kBlock, 0, st>>>(pop.p, n_kept, remf.p, addf.p);
      HM_LAUNCH_CHECK();
      HM_TRY(exclusive_scan(ctx, remf.p, remx.p, n_kept));
      HM_TRY(exclusive_scan(ctx, addf.p, addx.p, n_kept));
      (void)need;
      trace.mark("patch_rows");
      // Patched rows go to the arena tail in chunks that fit the free space;
      // between chunks the arena is compacted in place, so a batch never
      // needs a second copy of the store.
      std::vector<uint64_t> hno(n_rows + 1);
      HM_CUDA(cudaMemcpyAsync(hno.data(), noff.p, sizeof(uint64_t) * (n_rows + 1), cudaMemcpyDeviceToHost, st));
      HM_CUDA(cudaStreamSynchronize(st));
      uint64_t r0 = 0;
      while (r0 < n_rows) {
        uint64_t free_space = g->h2h_cap - g->h2h_tail;
        if (hno[r0 + 1] - hno[r0] > free_space || (free_space < (hno[n_rows] - hno[r0]) && free_space < g->h2h_cap / 4)) {
          trace.mark("patch_apply");
          HM_TRY(compact_h2h(g, hno[r0 + 1] - hno[r0]));
          trace.mark("compact");
          free_space = g->h2h_cap - g->h2h_tail;
        }
        uint64_t r1 = r0 + 1;
        {
          uint64_t lo = r0 + 1, hi = n_rows;  // largest r1 with hno[r1] - hno[r0] <= free_space
          while (lo < hi) {
            const uint64_t mid = (lo + hi + 1) / 2;
            if (hno[mid] - hno[r0] <= free_space) lo = mid;
            else hi = mid - 1;
          }
          r1 = lo;
        }
        const uint32_t nr = (uint32_t)(r1 - r0);
        const uint64_t base = g->h2h_tail - hno[r0];  // dst = base + noff[r], modulo 2^64
        k_patch_apply<<<grid_for((uint64_t)nr * 32, kBlock), kBlock, 0, st>>>(
            rp.p + r0, nr, noff.p + r0, base, pid.p, pop.p, ppidx.p, remx.p, addx.p, povl.p + n_rem,
            pmask.p + n_rem, g->h2h_off.p, g->h2h_len.p, g->h2h_nbr.p, g->h2h_ovl.p, g->h2h_mask.p);
        HM_LAUNCH_CHECK();
        k_set_lens<<<grid_for(nr, kBlock), kBlock, 0, st>>>(rp.p + r0, nr, nlen.p + r0, g->h2h_len.p);
        HM_LAUNCH_CHECK();
        g->h2h_tail += hno[r1] - hno[r0];
        r0 = r1;
      }
    }
  }

  trace.mark("h2h_patch");
  // ---- bookkeeping ---------------------------------------------------------------
  DArr<unsigned long long> sums;
  HM_TRY(sums.alloc(ctx, 2));
  HM_CUDA(cudaMemsetAsync(sums.p, 0, 2 * sizeof(unsigned long long), st));
  k_sum_u32<<<grid_for(g->n_slots, kBlock), kBlock, 0, st>>>(g->h2h_len.p, g->n_slots, sums.p);
  HM_LAUNCH_CHECK();
  k_sum_u32<<<grid_for(g->n_slots, kBlock), kBlock, 0, st>>>(g->h2v_len.p, g->n_slots, sums.p + 1);
  HM_LAUNCH_CHECK();
  unsigned long long hs[2];
  HM_CUDA(cudaMemcpyAsync(hs, sums.p, sizeof(hs), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  g->h2h_nnz = hs[0];
  g->h2v_nnz = hs[1];
  g->plus_valid = false;
  g->work_valid = false;
  release_plus_groups(g);  // rebuilt by the next static count; frees memory for the batches before it

  trace.mark("bookkeeping");
  if (hooks.after) {
    HM_TRY(hooks.after(ids.p, n_ins));
    trace.mark("count_inserted");
  }
  HM_CUDA(cudaEventRecord(e1, st));
  HM_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  g->times.update_ms = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return HM_OK;
}

// Exact change of the 30 static classes: touched triples of the inserted
// hyperedges in the new graph minus those of the deleted ones in the old.
int apply_batch(hm_graph* g, const uint32_t* h_dels, uint32_t n_del, const uint64_t* h_ins_off,
                const uint32_t* h_ins_mem, uint32_t n_ins, uint32_t* assigned_out, int64_t* delta30,
                const uint32_t* forced_ids) {
  if (!delta30)
    return apply_batch_hooks(g, h_dels, n_del, h_ins_off, h_ins_mem, n_ins, assigned_out, BatchHooks{}, forced_ids);
  uint64_t before[30] = {0}, after[30] = {0};
  BatchHooks hooks;
  hooks.before = [&](const uint32_t* d, uint32_t n) { return n ? count_touching(g, d, n, before) : (int)HM_OK; };
  hooks.after = [&](const uint32_t* d, uint32_t n) { return n ? count_touching(g, d, n, after) : (int)HM_OK; };
  HM_TRY(apply_batch_hooks(g, h_dels, n_del, h_ins_off, h_ins_mem, n_ins, assigned_out, hooks, forced_ids));
  for (int k = 0; k < 30; ++k) delta30[k] = (int64_t)(after[k] - before[k]);
  return HM_OK;
}

// fillCBST / unfillCBST on H2V: the members of live hyperedges ids[0..n)
// gain (or lose) the values [prefix[i-1], prefix[i]); each hyperedge keeps its
// id. Done as one batch that deletes the hyperedges and inserts their new
// member lists at the same ids, so the store, the adjacency and the exact
// delta follow from the batch path.
int modify_members(hm_graph* g, const uint32_t* h_ids, uint32_t n, const uint32_t* values, const uint64_t* prefix,
                   bool remove, int64_t* delta30) {
  hm_ctx* ctx = g->ctx;
  cudaStream_t st = ctx->stream;
  if (g->temporal) return set_error(HM_ERR_STATE, "fill/unfill: temporal graphs are immutable");
  if (!n) {
    if (delta30)
      for (int k = 0; k < 30; ++k) delta30[k] = 0;
    return HM_OK;
  }
  for (uint32_t i = 0; i < n; ++i)
    if (i && prefix[i] < prefix[i - 1]) return set_error(HM_ERR_INVALID, "fill/unfill: prefix sizes decrease");
  {
    std::vector<uint32_t> tmp(h_ids, h_ids + n);
    std::sort(tmp.begin(), tmp.end());
    if (std::adjacent_find(tmp.begin(), tmp.end()) != tmp.end())
      return set_error(HM_ERR_INVALID, "fill/unfill: a hyperedge id is listed twice");
  }
  for (uint32_t i = 0; i < prefix[n - 1]; ++i)
    if (values[i] >= g->n_nodes)
      return set_error(HM_ERR_INVALID, "fill/unfill: node %u out of range (%u nodes)", values[i], g->n_nodes);
  // current member lists (device -> host), the live check included
  DArr<uint32_t> ids;
  DArr<int> bad;
  HM_TRY(ids.alloc(ctx, n));
  HM_TRY(bad.alloc(ctx, 1));
  HM_CUDA(cudaMemcpyAsync(ids.p, h_ids, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st));
  HM_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
  k_check_live<<<grid_for(n, kBlock), kBlock, 0, st>>>(ids.p, n, g->n_slots, g->live_bits.p, bad.p);
  HM_LAUNCH_CHECK();
  int hbad = 0;
  HM_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  if (hbad) return set_error(HM_ERR_NOT_LIVE, "fill/unfill: a hyperedge id is not live");
  std::vector<uint64_t> off(g->n_slots), cur_off(n + 1, 0);
  std::vector<uint32_t> len(g->n_slots);
  HM_CUDA(cudaMemcpyAsync(off.data(), g->h2v_off.p, sizeof(uint64_t) * g->n_slots, cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaMemcpyAsync(len.data(), g->h2v_len.p, sizeof(uint32_t) * g->n_slots, cudaMemcpyDeviceToHost, st));
  HM_CUDA(cudaStreamSynchronize(st));
  std::vector<uint64_t> new_off(n + 1, 0);
  std::vector<uint32_t> new_mem, row;
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t id = h_ids[i];
    row.resize(len[id]);
    if (len[id])
      HM_CUDA(cudaMemcpyAsync(row.data(), g->h2v_mem.p + off[id], sizeof(uint32_t) * len[id], cudaMemcpyDeviceToHost,
                              st));
    HM_CUDA(cudaStreamSynchronize(st));
    std::vector<uint32_t> vals(values + (i ? prefix[i - 1] : 0), values + prefix[i]);
    std::sort(vals.begin(), vals.end());
    vals.erase(std::unique(vals.begin(), vals.end()), vals.end());
    std::vector<uint32_t> next;
    if (remove)
      std::set_difference(row.begin(), row.end(), vals.begin(), vals.end(), std::back_inserter(next));
    else
      std::set_union(row.begin(), row.end(), vals.begin(), vals.end(), std::back_inserter(next));
    if (next.size() > HM_MAX_EDGE_SIZE)
      return set_error(HM_ERR_LIMIT, "fill: hyperedge %u would have %zu members (limit %d)", id, next.size(),
                       HM_MAX_EDGE_SIZE);
    new_mem.insert(new_mem.end(), next.begin(), next.end());
    new_off[i + 1] = new_mem.size();
  }
  if (new_mem.empty()) new_mem.push_back(0);  // a valid pointer for an all-empty batch
  return apply_batch(g, h_ids, n, new_off.data(), new_mem.data(), n, nullptr, delta30, h_ids);
}

}  // namespace hm
