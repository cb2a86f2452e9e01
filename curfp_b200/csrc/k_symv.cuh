// k_symv.cuh — y := alpha A x + beta y for a symmetric A held in RFP (any
// variant), one right-hand side (ssfmv / dsfmv).
//
// Bandwidth-bound, and every stored element is read exactly once.  The
// logical lower triangle is cut into 64 x 64 tiles (I >= J).  A tile (I, J)
// feeds both halves of the symmetric product: its rows, A_IJ x_J -> y_I, and
// its columns, A_IJ^T x_I -> y_J.  CTA (I, s) walks the strip of up to S
// tiles J in [sS, sS + S) of tile row I:
//   * the row products of its tiles accumulate in registers and leave as one
//     64-vector per strip (row_part[I][s]);
//   * the column products leave as one 64-vector per tile
//     (col_part[J][I - J]; the diagonal tile contributes its strictly lower
//     part here and its lower part, diagonal included, to the row product).
// symv_reduce then forms y_J = alpha (sum_s row_part[J][s] + sum_I
// col_part[J][I - J]) + beta y_J.  Partials are written once and summed in a
// fixed order (registers, shuffle butterflies whose tree is the same in every
// lane, fixed-order combines through shared memory): the result is bitwise
// repeatable.  The partials take n^2 / 128 + n^2 / (64 S) elements.
//
// Tile reads follow the contiguous dimension of the RFP block that stores the
// tile: "row-fast" tiles (unit stride along i) put lanes on rows l, l + 32
// and warps on 8 columns each, "column-fast" tiles the transpose; a warp
// load is 32 consecutive elements either way.  Diagonal tiles and tiles
// across the n1 boundary take per-element offsets.  The next tile's elements
// are loaded while the current one is reduced.
#pragma once
#include <cstdint>

#include "rfp.h"
#include "symv_layout.h"

namespace rfp {
namespace ksymv {

constexpr int kThreads = 256;

enum : int { kRowFast = 0, kColFast = 1, kSlow = 2 };

// Sum over the 32 lanes of 8 values: returns, in lane L, the total of value
// L >> 2 (reduce-scatter halving the values per step, then two exchanges).
template <typename E>
__device__ __forceinline__ E warp_sum8(E (&v)[8], int lane) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {  // lanes with bit 4 keep values 4..7
    const bool hi = lane & 16;
    const E send = hi ? v[q] : v[q + 4], keep = hi ? v[q + 4] : v[q];
    v[q] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
#pragma unroll
  for (int q = 0; q < 2; ++q) {  // bit 3 keeps values 2, 3 of the four
    const bool hi = lane & 8;
    const E send = hi ? v[q] : v[q + 2], keep = hi ? v[q + 2] : v[q];
    v[q] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  {
    const bool hi = lane & 4;
    const E send = hi ? v[0] : v[1], keep = hi ? v[1] : v[0];
    v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
  E s = v[0];
  s += __shfl_xor_sync(0xffffffffu, s, 2);
  s += __shfl_xor_sync(0xffffffffu, s, 1);
  return s;  // value index (bit4 << 2) | (bit3 << 1) | bit2 = lane >> 2
}

template <typename E>
struct Tile {
  E v[16];   // row-fast / slow: v[8a + b] = (row l + 32a, col 8w + b);
             // column-fast: v[8a + b] = (row 8w + b, col l + 32a)
  int kind;
};

// Tile (I, J) of the logical lower triangle into registers (zero outside
// the matrix; the diagonal tile keeps i >= j).  Inside one RFP block the
// addresses advance by pointer increments from one per-thread base; tiles
// wholly inside the matrix load without bounds predicates.
template <typename E>
__device__ __forceinline__ void load_tile(const Geometry& g, const E* __restrict__ arf, int I,
                                          int J, int lane, int w, Tile<E>& t) {
  const int n = g.n;
  const int64_t i0 = (int64_t)I * TB, j0 = (int64_t)J * TB;
  const int64_t im = min((int64_t)n - 1, i0 + TB - 1), jm = min((int64_t)n - 1, j0 + TB - 1);
  const bool one_block = (i0 < g.n1) == (im < g.n1) && (j0 < g.n1) == (jm < g.n1);
  if (I != J && one_block) {
    int64_t off, rs, cs, ib, jb;
    if (j0 >= g.n1) {
      off = g.b22.off; rs = g.b22.rs; cs = g.b22.cs; ib = g.n1; jb = g.n1;
    } else if (i0 >= g.n1) {
      off = g.b21.off; rs = g.b21.rs; cs = g.b21.cs; ib = g.n1; jb = 0;
    } else {
      off = g.b11.off; rs = g.b11.rs; cs = g.b11.cs; ib = 0; jb = 0;
    }
    const E* base = arf + off + (i0 - ib) * rs + (j0 - jb) * cs;
    const bool full = i0 + TB <= n;  // j0 < i0 here, so the columns are inside too
    const bool rowf = rs == 1 || rs == -1;
    t.kind = rowf ? kRowFast : kColFast;
    // row-fast: (row lane + 32a, col 8w + b); column-fast: (row 8w + b, col lane + 32a)
    const int64_t s_lane = rowf ? rs : cs, s_b = rowf ? cs : rs;
    const E* pw = base + (int64_t)lane * s_lane + (int64_t)(8 * w) * s_b;
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      const E* q = pw + (int64_t)(32 * a) * s_lane;
      if (full) {
#pragma unroll
        for (int b = 0; b < 8; ++b, q += s_b) t.v[8 * a + b] = __ldg(q);
      } else {
#pragma unroll
        for (int b = 0; b < 8; ++b, q += s_b) {
          const int64_t i = i0 + (rowf ? lane + 32 * a : 8 * w + b);
          t.v[8 * a + b] = i < n ? __ldg(q) : E(0);
        }
      }
    }
  } else {
    t.kind = kSlow;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const int64_t i = i0 + lane + 32 * a, j = j0 + 8 * w + b;
        t.v[8 * a + b] = (i < n && j < n && i >= j) ? __ldg(arf + lower_offset(g, i, j)) : E(0);
      }
  }
}

template <typename E>
__device__ __forceinline__ E xval(const E* __restrict__ x, int64_t inc, int64_t i, int n) {
  return i < n ? __ldg(x + i * inc) : E(0);
}

// grid: strips_before(T) CTAs; part: [row_part | col_part] (parts(n)).
template <typename E>
__global__ void __launch_bounds__(kThreads)
    symv_tiles(Geometry g, const E* __restrict__ arf, const E* __restrict__ x, int64_t incx,
               E* __restrict__ part) {
  const int n = g.n;
  const Parts P = parts(n);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int I, s;
  strip_of(blockIdx.x, P.tiles, I, s);
  const int Jb = s * S, Je = min(Jb + S, I + 1);
  const int64_t i0 = (int64_t)I * TB;
  E* row_part = part + ((int64_t)I * P.strips + s) * TB;
  E* col_part = part + P.n_row;  // tile (I, J): + (col_base(J) + I - J) * 64

  // x over the tile row: lanes' rows (row-fast / slow) and the warp's rows
  // (column-fast)
  E xi_l[2], xi_w[8];
#pragma unroll
  for (int a = 0; a < 2; ++a) xi_l[a] = xval(x, incx, i0 + lane + 32 * a, n);
#pragma unroll
  for (int b = 0; b < 8; ++b) xi_w[b] = xval(x, incx, i0 + 8 * w + b, n);

  E racc_l[2] = {E(0), E(0)};  // row products of rows l, l + 32 (this warp's columns)
  E racc_w = E(0);             // row products of row 8w + (lane >> 2) (column-fast tiles)
  // column-fast tiles alternate between two buffers (counted over those
  // tiles only, so a buffer is rewritten only after a barrier that follows
  // its readers)
  __shared__ E cbuf[2][8][TB];
  __shared__ E rbuf[9][TB];
  int ncf = 0;

  Tile<E> cur, nxt;
  load_tile(g, arf, I, Jb, lane, w, cur);
  for (int J = Jb; J < Je; ++J) {
    if (J + 1 < Je) load_tile(g, arf, I, J + 1, lane, w, nxt);
    const int64_t j0 = (int64_t)J * TB;
    E* cp = col_part + (col_base(J, P.tiles) + (I - J)) * TB;
    if (cur.kind != kColFast) {
      // rows: v[8a + b] x_{j0 + 8w + b}; columns: sum over the 64 rows
      E xj[8], cv[8];
      {
        const E* xq = x + (j0 + 8 * w) * incx;
        const bool xin = j0 + TB <= n;
#pragma unroll
        for (int b = 0; b < 8; ++b, xq += incx)
          xj[b] = (xin || j0 + 8 * w + b < n) ? __ldg(xq) : E(0);
      }
      const bool diag = I == J;
#pragma unroll
      for (int a = 0; a < 2; ++a) {
        E r = E(0);
#pragma unroll
        for (int b = 0; b < 8; ++b) r = fma(cur.v[8 * a + b], xj[b], r);
        racc_l[a] += r;
      }
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        E c0 = cur.v[b], c1 = cur.v[8 + b];
        if (diag) {  // strictly lower part only
          if (lane <= 8 * w + b) c0 = E(0);
          if (lane + 32 <= 8 * w + b) c1 = E(0);
        }
        cv[b] = fma(c1, xi_l[1], c0 * xi_l[0]);
      }
      const E tot = warp_sum8(cv, lane);
      if ((lane & 3) == 0) cp[8 * w + (lane >> 2)] = tot;
    } else {
      // rows 8w + b: sum over the 64 columns (lanes); columns l, l + 32: sum
      // over this warp's 8 rows, then over the warps
      E xj0 = xval(x, incx, j0 + lane, n), xj1 = xval(x, incx, j0 + lane + 32, n);
      E rv[8];
#pragma unroll
      for (int b = 0; b < 8; ++b) rv[b] = fma(cur.v[8 + b], xj1, cur.v[b] * xj0);
      racc_w += warp_sum8(rv, lane);
      E c0 = E(0), c1 = E(0);
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        c0 = fma(cur.v[b], xi_w[b], c0);
        c1 = fma(cur.v[8 + b], xi_w[b], c1);
      }
      E (*cb)[TB] = cbuf[ncf++ & 1];
      cb[w][lane] = c0;
      cb[w][lane + 32] = c1;
      __syncthreads();
      if (threadIdx.x < TB) {
        E t = cb[0][threadIdx.x];
#pragma unroll
        for (int q = 1; q < 8; ++q) t += cb[q][threadIdx.x];
        cp[threadIdx.x] = t;
      }
    }
    if (J + 1 < Je) cur = nxt;
  }
  // row product of the strip: the 8 warps' lane sums, then the column-fast sums
  rbuf[w][lane] = racc_l[0];
  rbuf[w][lane + 32] = racc_l[1];
  if ((lane & 3) == 0) rbuf[8][8 * w + (lane >> 2)] = racc_w;
  __syncthreads();
  if (threadIdx.x < TB) {
    E t = rbuf[0][threadIdx.x];
#pragma unroll
    for (int q = 1; q < 9; ++q) t += rbuf[q][threadIdx.x];
    row_part[threadIdx.x] = t;
  }
}

// y_J (64 rows per CTA) from the partials: four groups of 64 threads sum
// quarters of the column list, then thread r adds the strips' row products
// and the four quarters in order.
template <typename E>
__global__ void __launch_bounds__(kThreads)
    symv_reduce(int n, const E* __restrict__ part, E* y, int64_t incy, E alpha, E beta) {
  const Parts P = parts(n);
  const int J = blockIdx.x, r = threadIdx.x % TB, q = threadIdx.x / TB;
  const int64_t cnt = P.tiles - J;  // col_part entries I = J .. T-1
  const int64_t per = (cnt + 3) / 4, b0 = q * per, b1 = min(cnt, b0 + per);
  const E* cp = part + P.n_row + col_base(J, P.tiles) * TB + r;
  E t = E(0);
  for (int64_t e = b0; e < b1; ++e) t += cp[e * TB];
  __shared__ E qs[4][TB];
  qs[q][r] = t;
  __syncthreads();
  if (q == 0) {
    const int64_t i = (int64_t)J * TB + r;
    if (i < n) {
      E sum = E(0);
      const E* rp = part + (int64_t)J * P.strips * TB + r;
      const int ns = J / S + 1;
      for (int s = 0; s < ns; ++s) sum += rp[(int64_t)s * TB];
#pragma unroll
      for (int k = 0; k < 4; ++k) sum += qs[k][r];
      E* yi = y + i * incy;
      *yi = beta == E(0) ? alpha * sum : fma(beta, *yi, alpha * sum);
    }
  }
}

}  // namespace ksymv
}  // namespace rfp
