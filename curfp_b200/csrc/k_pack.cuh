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

constexpr int TS = 32;     // tile edge
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

// to_rfp = 1: strttf (dense -> RFP); 0: stfttr (RFP -> dense).
template <typename T>
__global__ void __launch_bounds__(TS * TY) pack_kernel(const PackArgs args,
                                                       const T* __restrict__ src,
                                                       T* __restrict__ dst,
                                                       int to_rfp) {
  __shared__ T tile[TS][TS + 1];
  int t = blockIdx.x, bi = 0;
  while (bi + 1 < args.nblocks && t >= args.b[bi + 1].tile_begin) ++bi;
  const PackBlock& B = args.b[bi];
  int tp, tq;
  pack_tile_coords(B, t - B.tile_begin, tp, tq);
  const int p0 = tp * TS, q0 = tq * TS;
  const int tx = threadIdx.x, ty = threadIdx.y;

  // Contiguous dimension of each side: 0 -> p, 1 -> q.
  const int dense_q = (args.dcs == 1 || args.dcs == -1) ? 1 : 0;
  const int rfp_q = (B.rs == 1 || B.rs == -1) ? 0 : 1;
  const int src_q = to_rfp ? dense_q : rfp_q;
  const int dst_q = to_rfp ? rfp_q : dense_q;

  auto dense_ptr = [&](int p, int q) -> int64_t {
    int64_t P = (int64_t)B.p_base + p, Q = (int64_t)B.q_base + q;
    return P * args.drs + Q * args.dcs;
  };
  auto rfp_ptr = [&](int p, int q) -> int64_t {
    return B.off + (int64_t)p * B.rs + (int64_t)q * B.cs;
  };
  auto inside = [&](int p, int q) -> bool {
    return p < B.rows && q < B.cols && (!B.tri || p >= q);
  };

#pragma unroll
  for (int r = 0; r < TS / TY; ++r) {
    int lp, lq;
    if (src_q) { lq = tx; lp = ty + r * TY; }
    else       { lp = tx; lq = ty + r * TY; }
    int p = p0 + lp, q = q0 + lq;
    if (inside(p, q))
      tile[lp][lq] = src[to_rfp ? dense_ptr(p, q) : rfp_ptr(p, q)];
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < TS / TY; ++r) {
    int lp, lq;
    if (dst_q) { lq = tx; lp = ty + r * TY; }
    else       { lp = tx; lq = ty + r * TY; }
    int p = p0 + lp, q = q0 + lq;
    if (inside(p, q)) {
      T v = tile[lp][lq];
      if (to_rfp && B.p_base + p == B.q_base + q) v *= (T)args.diag_scale;
      dst[to_rfp ? rfp_ptr(p, q) : dense_ptr(p, q)] = v;
    }
  }
}

// idx[i] = RFP offset of diagonal element i (reference
// curfp/__init__.py:194-269 builds the same two arithmetic progressions).
__global__ void diag_indices(Geometry g, int64_t* idx) {
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
