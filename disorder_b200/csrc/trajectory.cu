// Host side of the DISORDER sample orders: the greedy electrostatic order
// of a tile's positions (Acquisition/electrostaticRepulsionDISORDER.m:9-52),
// used by samplingDISORDER.m:104 to spread consecutive segments over a tile.
//
// Position 0 is the tile's centre (sub2ind(N, ceil(N/2))). Each next
// position is the free one whose summed inverse squared distance to the
// positions already placed is least, the distance to a placed point being
// the nearest of its 9 periodic images (shifts by 0 and +-N per axis). The
// scan goes in column-major order and a candidate replaces the best so far
// only when it is lower by more than 1e-9 (electrostaticRepulsionDISORDER.m:
// 44), so ties keep the first position. The nearest image separates per
// axis, min over a, b of (d1 - a)^2 + (d2 - b)^2 = min_a (d1 - a)^2 +
// min_b (d2 - b)^2, exactly in integers, and the sum runs over the placed
// points in placement order in double precision.
#include <cstdint>
#include <cstdlib>
#include <limits>
#include <vector>

#include "internal.h"

extern "C" int disorder_electrostatic_order(int32_t n1, int32_t n2, int32_t* order) {
  if (n1 < 1 || n2 < 1 || !order || (long long)n1 * n2 > (1 << 20)) return DISORDER_BAD_ARG;
  const int P = n1 * n2;
  std::vector<int> p1, p2;
  p1.reserve(P);
  p2.reserve(P);
  std::vector<char> free_(P, 1);
  std::vector<double> rep(P, 0.0);  // summed 1/d^2 of each position to the placed points
  auto place = [&](int idx, int n) {
    order[n] = idx;
    free_[idx] = 0;
    const int a = idx % n1, b = idx / n1;
    p1.push_back(a);
    p2.push_back(b);
    // add the new point's term to every free position (placement order is
    // the summation order, as in the reference's per-candidate sum)
    for (int m = 0; m < P; ++m) {
      if (!free_[m]) continue;
      int d1 = std::abs(m % n1 - a), d2 = std::abs(m / n1 - b);
      if (n1 - d1 < d1) d1 = n1 - d1;
      if (n2 - d2 < d2) d2 = n2 - d2;
      rep[m] += 1.0 / (double)(d1 * d1 + d2 * d2);
    }
  };
  place((n1 + 1) / 2 - 1 + n1 * ((n2 + 1) / 2 - 1), 0);
  for (int n = 1; n < P; ++n) {
    double best = std::numeric_limits<double>::infinity();
    int bi = -1;
    for (int m = 0; m < P; ++m)
      if (free_[m] && rep[m] < best - 1e-9) {
        best = rep[m];
        bi = m;
      }
    place(bi, n);
  }
  return DISORDER_OK;
}
