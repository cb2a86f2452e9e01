// k_order.cuh — tile orders that keep operand panels in L2.
//
// The tiles in flight at a time should share operand panels (a panel is a
// tile's rows x K; at the K of the large trailing updates a panel is several
// MB, and the operands exceed the 126 MB L2 by far).  Rectangular problems
// run in groups of kRowGroup tile rows, column by column within a group, so
// a wave of ~150 tiles reads ~16 row panels and ~9 column panels; lower
// triangles run in bands of kBand tile columns, row by row within a band.
#pragma once

namespace rfp {
namespace order {

constexpr int kRowGroup = 16, kBand = 8;

// lt-th tile of a tiles_m x tiles_n grid in row-group order.
__device__ __forceinline__ void grouped_tile(int tiles_m, int tiles_n, int lt, int& r,
                                             int& c) {
  const int per = kRowGroup * tiles_n;
  const int grp = lt / per, e = lt % per;
  const int rows = min(kRowGroup, tiles_m - grp * kRowGroup);
  r = grp * kRowGroup + e % rows;
  c = e / rows;
}

// lt-th tile of the lower triangle (c <= r) of a t x t tile grid in band
// order: band b covers tile columns [b0, b0 + w); its own w x w triangle
// first, then the rows below it, w tiles per row.
__device__ __forceinline__ void tri_band_tile(int t, int lt, int& r, int& c) {
  int b0 = 0;
  for (;;) {
    const int w = min(kBand, t - b0);
    const int cnt = w * (w + 1) / 2 + (t - b0 - w) * w;
    if (lt < cnt || b0 + w >= t) {
      const int head = w * (w + 1) / 2;
      if (lt < head) {
        int a = (int)((sqrtf(8.0f * (float)lt + 1.0f) - 1.0f) * 0.5f);
        while ((a + 1) * (a + 2) / 2 <= lt) ++a;
        while (a * (a + 1) / 2 > lt) --a;
        r = b0 + a;
        c = b0 + lt - a * (a + 1) / 2;
      } else {
        const int e = lt - head;
        r = b0 + w + e / w;
        c = b0 + e % w;
      }
      return;
    }
    lt -= cnt;
    b0 += w;
  }
}

}  // namespace order
}  // namespace rfp
