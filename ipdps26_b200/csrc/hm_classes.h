// Motif classification from the seven Venn regions of a hyperedge triple.
// Host and device. The static rule and the temporal numbering are the
// reference's (MoCHy-master/motif_id.cpp:5-34, THyMe-main/code/motif_id.cpp:
// 25-109); the static table is derived here from the structure of the
// pattern rather than stored.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define HM_HD __host__ __device__ __forceinline__
#else
#define HM_HD inline
#endif

namespace hm {

// Bits: 0..2 exclusive regions of x, y, z; 3 x&y only; 4 y&z only;
// 5 z&x only; 6 x&y&z. Sizes sx.., pairwise overlaps cxy.., triple g.
HM_HD int region_pattern(int sx, int sy, int sz, int cxy, int cyz, int czx, int g) {
  const int ex = sx - (cxy + czx) + g, ey = sy - (cyz + cxy) + g, ez = sz - (czx + cyz) + g;
  return (ex > 0) | ((ey > 0) << 1) | ((ez > 0) << 2) | ((cxy - g > 0) << 3) | ((cyz - g > 0) << 4) |
         ((czx - g > 0) << 5) | ((g > 0) << 6);
}

// Static class 0..29 of a connected pattern (-1 otherwise). With p the number
// of non-empty pairwise-only regions:
//   g, p=0: 1 + #excl; g, p=1: 5 + rank(excl of the pair, excl of the loner);
//   g, p=2: 11 + excl(hub) + 2 #excl(ends); g, p=3: 17 + #excl;
//   no g, p=2: 21 + excl(hub) + 2 #excl(ends); no g, p=3: 27 + #excl;
// minus one. The hub is the hyperedge in both non-empty pair regions.
HM_HD int static_class_of_pattern(int pat) {
  const int ex = pat & 1, ey = (pat >> 1) & 1, ez = (pat >> 2) & 1;
  const int pxy = (pat >> 3) & 1, pyz = (pat >> 4) & 1, pzx = (pat >> 5) & 1, g = (pat >> 6) & 1;
  const int p = pxy + pyz + pzx, nex = ex + ey + ez;
  if (p == 3) return (g ? 16 : 26) + nex;
  if (p == 2) {
    const int hub = (pzx && pxy) ? ex : ((pxy && pyz) ? ey : ez);
    return (g ? 10 : 20) + hub + 2 * (nex - hub);
  }
  if (!g) return -1;
  if (p == 1) {
    const int loner = pxy ? ez : (pyz ? ex : ey);
    const int pair = nex - loner;  // 0..2
    // (pair, loner) -> 0,1,3 for loner 0 and 2,4,5 for loner 1
    return 4 + (loner ? (pair == 0 ? 2 : 3 + pair) : (pair == 2 ? 3 : pair));
  }
  return nex;  // p == 0
}

HM_HD int static_class(int sx, int sy, int sz, int cxy, int cyz, int czx, int g) {
  return static_class_of_pattern(region_pattern(sx, sy, sz, cxy, cyz, czx, g));
}

// Class of an open wedge (y - x - z, y and z disjoint) seen from its centre x:
// pattern (excl x, excl y, excl z, x&y, -, z&x, -) -> 20 + ex + 2 (ey + ez).
// x_ex = [cxy + cxz < |x|], ey = [cxy < |y|], ez = [cxz < |z|].
HM_HD int open_class(int x_ex, int n_end_ex) { return 20 + x_ex + 2 * n_end_ex; }

// MoCHy reports classes other than these four (MoCHy-master/main_exact.cpp:135).
HM_HD bool static_class_reported(int k) { return !(k == 0 || k == 1 || k == 4 || k == 6); }

// THyMe's numbering of the 96 temporal patterns (hyperedges in time order):
// entry m-1 holds the pattern of motif m. It is a bijection with no closed
// form, so it is data (THyMe-main/code/motif_id.cpp:25-42, inverted).
constexpr uint8_t kTemporalMotifPattern[96] = {
    67,  69,  70,  71,  73,  74,  82,  84,  97,  100, 75,  86,  101, 77,  78,  83,  85,  99,  102, 79,
    87,  103, 88,  104, 112, 90,  105, 116, 89,  92,  106, 108, 113, 114, 91,  94,  107, 109, 117, 118,
    93,  110, 115, 95,  111, 119, 120, 121, 122, 124, 123, 125, 126, 127, 24,  40,  48,  26,  41,  52,
    25,  28,  42,  44,  49,  50,  27,  30,  43,  45,  53,  54,  29,  46,  51,  31,  47,  55,  56,  57,
    58,  60,  59,  61,  62,  63,  65,  66,  68,  72,  80,  96,  76,  81,  98,  64};

}  // namespace hm
