// Open-pair class counts of one centre from its neighbour histogram.
//
// h0 / h1 hold, for overlaps 1..s (s = |centre|), the number of neighbours b
// with [C_ab < |b|] = 0 / 1, already turned into prefix sums (h[k] = number
// with overlap <= k). An unordered pair {b, c} seen from the centre a, taken
// as open, has class 20 + [C_ab + C_ac < s] + 2 ([C_ab < |b|] + [C_ac < |c|]);
// the six counts are added (or subtracted) into acc[0..6) at index
// [C_ab + C_ac < s] + 2 (number of ends with an exclusive part).
#pragma once

#include <cstdint>

namespace hm {

__device__ __forceinline__ void open_pair_counts(const uint32_t* h0, const uint32_t* h1, uint32_t s, uint64_t acc[6],
                                                 bool subtract) {
  const uint64_t n0 = h0[s], n1 = h1[s];
  // ordered pairs (b, c), b of type t, c of type u, with C_b + C_c <= s - 1
  uint64_t l00 = 0, l01 = 0, l11 = 0, d0 = 0, d1 = 0;
  for (uint32_t c1 = 1; c1 + 1 < s; ++c1) {
    const uint64_t x0 = h0[c1] - h0[c1 - 1], x1 = h1[c1] - h1[c1 - 1];
    const uint32_t m = s - 1 - c1;
    l00 += x0 * h0[m];
    l01 += x0 * h1[m];
    l11 += x1 * h1[m];
    if (2 * c1 <= s - 1) {
      d0 += x0;
      d1 += x1;
    }
  }
  const uint64_t p00 = (l00 - d0) / 2, p11 = (l11 - d1) / 2, p01 = l01;
  const uint64_t t00 = n0 * (n0 - (n0 > 0)) / 2, t11 = n1 * (n1 - (n1 > 0)) / 2, t01 = n0 * n1;
  const uint64_t v[6] = {t00 - p00, p00, t01 - p01, p01, t11 - p11, p11};
  for (int k = 0; k < 6; ++k) acc[k] = subtract ? acc[k] - v[k] : acc[k] + v[k];
}

}  // namespace hm
