// Deferred classification of closed triangles: lanes that find a triangle
// which is not a star push a packed record to their warp's queue; the warp
// classifies 32 records at a time with every lane busy, instead of running
// the classification on the few lanes that hit. Shared by the static count
// and the touched-triple count.
#pragma once

#include <cstdint>

#include "hm_classes.h"

namespace hm {

// Classifies the first n records of a warp's queue of closed triangles that
// are not stars, one per lane, and adds their counts. A record packs |b|,
// |c|, C_ab, C_bc, C_ac and g (8 bits each); sa is the centre's size.
__device__ __forceinline__ void classify_queue(const uint64_t* q, uint32_t n, uint32_t sa, unsigned long long* wc) {
  const unsigned lane = threadIdx.x & 31u;
  if (lane < n) {
    const uint64_t r = q[lane];
    const uint32_t sb = r & 0xffu, sc = (r >> 8) & 0xffu, cab = (r >> 16) & 0xffu, cbc = (r >> 24) & 0xffu,
                   cac = (r >> 32) & 0xffu, g = (r >> 40) & 0xffu;
    const int k = static_class((int)sa, (int)sb, (int)sc, (int)cab, (int)cbc, (int)cac, (int)g);
    if (k >= 0) {  // always, for a closed triangle; keeps the index in range
      const uint32_t oa = (cab + cac < sa) + 2 * ((cab < sb) + (cac < sc));
      const uint32_t ob = (cab + cbc < sb) + 2 * ((cab < sa) + (cbc < sc));
      const uint32_t oc = (cac + cbc < sc) + 2 * ((cac < sa) + (cbc < sb));
      const uint32_t key = (uint32_t)k | (oa << 5) | (ob << 8) | (oc << 11);
      const unsigned peers = __match_any_sync(__activemask(), key);
      if (lane == (unsigned)(__ffs(peers) - 1)) {
        const unsigned long long cnt = (unsigned long long)__popc(peers);
        atomicAdd(&wc[k], cnt);
        atomicAdd(&wc[30 + oa], cnt);
        atomicAdd(&wc[30 + ob], cnt);
        atomicAdd(&wc[30 + oc], cnt);
      }
    }
  }
  __syncwarp();
}

// Sizes and overlaps are at most 255, so a record fits 48 bits.
__device__ __forceinline__ uint64_t pack_triangle(uint32_t sb, uint32_t sc, uint32_t cab, uint32_t cbc, uint32_t cac,
                                                  uint32_t g) {
  return (uint64_t)sb | ((uint64_t)sc << 8) | ((uint64_t)cab << 16) | ((uint64_t)cbc << 24) |
         ((uint64_t)cac << 32) | ((uint64_t)g << 40);
}

}  // namespace hm
