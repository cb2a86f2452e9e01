// symv_layout.h — work and partial-sum layout of the single-read symmetric
// matrix-vector kernels (k_symv.cuh), host- and device-callable so that the
// host tests can enumerate it.
//
// The logical lower triangle is cut into 64 x 64 tiles (I >= J); tile row I
// is walked in strips of up to S tiles, strip s covering J in [sS, sS + S);
// CTA b of the launch takes the strip strip_of(b).  Row products leave one
// 64-vector per strip (row_part, T x strips x 64), column products one per
// tile (col_part, tile (I, J) at entry col_base(J) + I - J, 64 elements).
#pragma once
#include <stdint.h>

#include "rfp.h"

namespace rfp {
namespace ksymv {

constexpr int TB = 64;  // tile edge
constexpr int S = 16;   // tiles per strip

struct Parts {
  int tiles;      // T = ceil(n / 64)
  int strips;     // ceil(T / S): row_part stride per tile row
  int64_t n_row;  // T * strips * 64 elements
  int64_t n_col;  // T (T + 1) / 2 * 64 elements
};
RFP_HD Parts parts(int n) {
  Parts p;
  p.tiles = (n + TB - 1) / TB;
  p.strips = (p.tiles + S - 1) / S;
  p.n_row = (int64_t)p.tiles * p.strips * TB;
  p.n_col = (int64_t)p.tiles * (p.tiles + 1) / 2 * TB;
  return p;
}
// Strips over tile rows 0 .. I-1: sum_{i < I} (floor(i / S) + 1); the launch
// has strips_before(T) CTAs.
RFP_HD int64_t strips_before(int64_t I) {
  const int64_t q = I / S, r = I - q * S;
  return I + S * q * (q - 1) / 2 + q * r;
}
// First col_part entry of tile column J: sum_{j < J} (T - j).
RFP_HD int64_t col_base(int64_t J, int64_t T) { return J * T - J * (J - 1) / 2; }
// The strip of CTA b: tile row I (the largest with strips_before(I) <= b)
// and strip s within it.
RFP_HD void strip_of(int64_t b, int tiles, int& I, int& s) {
  int lo = 0, hi = tiles - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (strips_before(mid) <= b) lo = mid;
    else hi = mid - 1;
  }
  I = lo;
  s = (int)(b - strips_before(lo));
}

}  // namespace ksymv
}  // namespace rfp
