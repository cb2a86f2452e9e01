// k_pack.cuh — bandwidth-bound RFP conversions and diagonal helpers.
//
// strttf / stfttr copy the stored triangle between a row-major n x n matrix
// and the RFP array (semantics of LAPACK xTRTTF / xTFTTR on the same
// mathematical matrix, reference src/curfp_strttf.cu:46-415 and
// src/curfp_stfttr.cu:24-128).  Instead of one thread per dense element with a
// closed-form 8-case index map (half of those threads idle and, for
// TRANSR=T, scattered RFP writes), the work here is tiled per RFP block: a
// 32 x 32 tile of a block is read with the warp running along the contiguous
// dimension of the source, transposed through shared memory when the two
// sides disagree, and written with the warp running along the contiguous
// dimension of the destination, so both HBM streams coalesce.  Only tiles
// that touch the block's stored region are launched, and indices are 64-bit
// (n(n+1)/2 overflows int32 for n >= 46341).
#pragma once
#include <cstdint>

#include "rfp.h"

namespace rfp {
namespace kpack {

constexpr int TS = 64;     // tile edge
constexpr int TX = 32;     // threads along the contiguous dimension
constexpr int TY = 8;      // thread rows (block = 32 x 8)

struct PackBlock {
  int64_t off, rs, cs;     // RFP view of the block (logical lower element)
  int rows, cols;          // block extent
  int p_base, q_base;      // logical row/col of the block's (0,0)
  int tri;                 // 1: only p >= q is stored
  int tiles_p, tiles_q;    // tile grid
  int tile_begin;          // first linear tile of this block
};

struct PackArgs {
  PackBlock b[3];
  int nblocks;
  int total_tiles;
  // Dense element of logical (P,Q) at P*drs + Q*dcs: row-major A[P][Q] for
  // UPLO=L (drs = lda, dcs = 1), A[Q][P] for UPLO=U (drs = 1, dcs = lda).
  int64_t drs, dcs;
  float diag_scale;        // dense -> RFP: diagonal elements are multiplied by this
};

// The tile list of the three RFP blocks of geometry g (64 x 64 tiles; the
// triangular blocks list only their lower-triangle tiles).  Returns the
// number of tiles; drs / dcs / diag_scale are left to the caller.
inline int pack_blocks(const Geometry& g, PackArgs* a) {
  const BlockGeom* bg[3] = {&g.b11, &g.b21, &g.b22};
  const int rows[3] = {g.n1, g.n2, g.n2}, cols[3] = {g.n1, g.n1, g.n2};
  const int pb[3] = {0, g.n1, g.n1}, qb[3] = {0, 0, g.n1};
  int tiles = 0, cnt = 0;
  for (int b = 0; b < 3; ++b) {
    if (rows[b] <= 0 || cols[b] <= 0) continue;
    PackBlock& B = a->b[cnt++];
    B.off = bg[b]->off; B.rs = bg[b]->rs; B.cs = bg[b]->cs;
    B.rows = rows[b]; B.cols = cols[b];
    B.p_base = pb[b]; B.q_base = qb[b];
    B.tri = (b != 1);
    B.tiles_p = (rows[b] + TS - 1) / TS;
    B.tiles_q = (cols[b] + TS - 1) / TS;
    B.tile_begin = tiles;
    tiles += B.tri ? B.tiles_p * (B.tiles_p + 1) / 2 : B.tiles_p * B.tiles_q;
  }
  a->nblocks = cnt;
  a->total_tiles = tiles;
  return tiles;
}

__device__ __forceinline__ void pack_tile_coords(const PackBlock& B, int lt,
                                                 int& tp, int& tq) {
  if (!B.tri) {
    tp = lt % B.tiles_p;
    tq = lt / B.tiles_p;
    return;
  }
  int r = (int)((sqrt(8.0 * (double)lt + 1.0) - 1.0) * 0.5);
  while ((int64_t)(r + 1) * (r + 2) / 2 <= lt) ++r;
  while ((int64_t)r * (r + 1) / 2 > lt) --r;
  tp = r;
  tq = lt - (int)((int64_t)r * (r + 1) / 2);
}

// One side of a tile copy: element (p, q) of the tile at base[p*sp + q*sq];
// the warp runs along the side's contiguous dimension (qc = 1: q, else p).
// 16 elements per thread, addressed by pointer increments.  dpq = p0 - q0 of
// the tile (the stored-triangle test of a triangular block is p >= q).
template <typename T, bool kLoad, bool kChecked>
__device__ __forceinline__ void tile_pass(T (*tile)[TS + 1], T* base, int64_t sp, int64_t sq,
                                          int qc, int prow, int qcol, int tri, int dpq,
                                          T dscale, bool diag) {
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int64_t sc = qc ? sq : sp, so = qc ? sp : sq;  // contiguous / other stride
  T* ptr = base + (int64_t)tx * sc + (int64_t)ty * so;
#pragma unroll
  for (int r = 0; r < TS / TY; ++r) {
#pragma unroll
    for (int h = 0; h < TS / TX; ++h) {
      const int c = tx + TX * h, o = ty + TY * r;
      const int lp = qc ? o : c, lq = qc ? c : o;
      T* e = ptr + (int64_t)(TX * h) * sc + (int64_t)(TY * r) * so;
      bool ok = true;
      if (kChecked) ok = lp < prow && lq < qcol && (!tri || lp + dpq >= lq);  // p >= q
      if (ok) {
        if (kLoad) {
          tile[lp][lq] = *e;
        } else {
          T v = tile[lp][lq];
          if (kChecked && diag && lp == lq) v *= dscale;
          *e = v;
        }
      }
    }
  }
}

// to_rfp = 1: strttf (dense -> RFP); 0: stfttr (RFP -> dense).  A 64 x 64
// tile of an RFP block is read with the warp along the source's contiguous
// dimension, transposed through shared memory when the two sides disagree,
// and written with the warp along the destination's contiguous dimension,
// so both HBM streams coalesce.  Tiles strictly inside their block (and, in
// the triangles, strictly below the diagonal) take a path without per-element
// bounds tests.
template <typename T>
__global__ void __launch_bounds__(TX * TY) pack_kernel(const PackArgs args,
                                                       const T* __restrict__ src,
                                                       T* __restrict__ dst, int to_rfp) {
  __shared__ T tile[TS][TS + 1];
  int t = blockIdx.x, bi = 0;
  while (bi + 1 < args.nblocks && t >= args.b[bi + 1].tile_begin) ++bi;
  const PackBlock& B = args.b[bi];
  int tp, tq;
  pack_tile_coords(B, t - B.tile_begin, tp, tq);
  const int p0 = tp * TS, q0 = tq * TS;
  const int prow = B.rows - p0, qcol = B.cols - q0;  // extent left in the block
  const int64_t P0 = (int64_t)B.p_base + p0, Q0 = (int64_t)B.q_base + q0;
  T* dense = const_cast<T*>(to_rfp ? src : dst) + P0 * args.drs + Q0 * args.dcs;
  T* rfp = const_cast<T*>(to_rfp ? dst : src) + B.off + (int64_t)p0 * B.rs + (int64_t)q0 * B.cs;
  const int dense_q = (args.dcs == 1 || args.dcs == -1) ? 1 : 0;
  const int rfp_q = (B.cs == 1 || B.cs == -1) ? 1 : 0;
  const bool interior = prow >= TS && qcol >= TS && (!B.tri || q0 + TS <= p0);
  const bool diag = to_rfp && B.tri && tp == tq && args.diag_scale != 1.0f;
  const T ds = (T)args.diag_scale;
  if (interior) {
    if (to_rfp) {
      tile_pass<T, true, false>(tile, dense, args.drs, args.dcs, dense_q, prow, qcol, B.tri, p0 - q0, ds, false);
      __syncthreads();
      tile_pass<T, false, false>(tile, rfp, B.rs, B.cs, rfp_q, prow, qcol, B.tri, p0 - q0, ds, false);
    } else {
      tile_pass<T, true, false>(tile, rfp, B.rs, B.cs, rfp_q, prow, qcol, B.tri, p0 - q0, ds, false);
      __syncthreads();
      tile_pass<T, false, false>(tile, dense, args.drs, args.dcs, dense_q, prow, qcol, B.tri, p0 - q0, ds, false);
    }
  } else {
    if (to_rfp) {
      tile_pass<T, true, true>(tile, dense, args.drs, args.dcs, dense_q, prow, qcol, B.tri, p0 - q0, ds, false);
      __syncthreads();
      tile_pass<T, false, true>(tile, rfp, B.rs, B.cs, rfp_q, prow, qcol, B.tri, p0 - q0, ds, diag);
    } else {
      tile_pass<T, true, true>(tile, rfp, B.rs, B.cs, rfp_q, prow, qcol, B.tri, p0 - q0, ds, false);
      __syncthreads();
      tile_pass<T, false, true>(tile, dense, args.drs, args.dcs, dense_q, prow, qcol, B.tri, p0 - q0, ds, false);
    }
  }
}

// BLAS-2 rank updates over the stored elements (tiles of pack_blocks, warp
// along the block's contiguous dimension, read-modify-write once):
//   two = 0:  a(p,q) += (alpha x_q) x_p                      (ssfr, SSYR form)
//   two = 1:  a(p,q) += x_p (alpha y_q) + y_p (alpha x_q)    (ssfr2, SSYR2 form)
// x and y element i at x[i * incx] (the caller shifts the base for negative
// increments).
template <typename T>
__global__ void __launch_bounds__(TX * TY)
    rank_update(const PackArgs args, T* arf, const T* __restrict__ x, int64_t incx,
                const T* __restrict__ y, int64_t incy, T alpha, int two) {
  __shared__ T xp[TS], xq[TS], yp[TS], yq[TS];
  int t = blockIdx.x, bi = 0;
  while (bi + 1 < args.nblocks && t >= args.b[bi + 1].tile_begin) ++bi;
  const PackBlock& B = args.b[bi];
  int tp, tq;
  pack_tile_coords(B, t - B.tile_begin, tp, tq);
  const int p0 = tp * TS, q0 = tq * TS;
  const int prow = B.rows - p0, qcol = B.cols - q0;
  const int64_t P0 = (int64_t)B.p_base + p0, Q0 = (int64_t)B.q_base + q0;
  const int tx = threadIdx.x, ty = threadIdx.y, lin = ty * TX + tx;
  if (lin < TS) {
    xp[lin] = lin < prow ? x[(P0 + lin) * incx] : T(0);
    xq[lin] = lin < qcol ? alpha * x[(Q0 + lin) * incx] : T(0);
    if (two) {
      yp[lin] = lin < prow ? y[(P0 + lin) * incy] : T(0);
      yq[lin] = lin < qcol ? alpha * y[(Q0 + lin) * incy] : T(0);
    }
  }
  __syncthreads();
  T* base = arf + B.off + (int64_t)p0 * B.rs + (int64_t)q0 * B.cs;
  const bool qc = (B.cs == 1 || B.cs == -1);
  const int64_t sl = qc ? B.cs : B.rs, sw = qc ? B.rs : B.cs;
#pragma unroll
  for (int r = 0; r < TS / TY; ++r) {
#pragma unroll
    for (int h = 0; h < TS / TX; ++h) {
      const int l = tx + TX * h, w = ty + TY * r;
      const int lp = qc ? w : l, lq = qc ? l : w;
      if (lp < prow && lq < qcol && (!B.tri || p0 + lp >= q0 + lq)) {
        T* e = base + (int64_t)l * sl + (int64_t)w * sw;
        *e = two ? fma(yp[lp], xq[lq], fma(xp[lp], yq[lq], *e)) : fma(xp[lp], xq[lq], *e);
      }
    }
  }
}

// idx[i] = RFP offset of diagonal element i (reference
// curfp/__init__.py:194-269 builds the same two arithmetic progressions).
static __global__ void diag_indices(Geometry g, int64_t* idx) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < g.n) idx[i] = diag_offset(g, i);
}

template <typename T>
__global__ void add_diag(Geometry g, T value, T* arf) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < g.n) arf[diag_offset(g, i)] += value;
}

}  // namespace kpack
}  // namespace rfp
