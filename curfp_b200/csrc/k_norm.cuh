// k_norm.cuh — norms of a symmetric matrix held in RFP, and the vector
// kernels of the 1-norm condition estimator.
//
// Norms (reference src/curfp_slansf.cu:1-26 states them on the blocks
// [T1 S^T; S T2]): every stored RFP element is one distinct element (p, q),
// p >= q, of the symmetric matrix, so
//   max |A|     = max over the flat array,
//   ||A||_F^2   = 2 sum_all a^2 - sum_diag a^2   (FP64 sums),
//   ||A||_1     = max_j sum_i |A(i,j)|: element (p, q) adds |a| to column q
//                 and, when p != q, to column p.
// The first two are one grid-stride pass; the column sums walk 64 x 64 tiles
// of the three RFP blocks (the tile list of the packing kernels) with the
// warp along the stored block's contiguous dimension, reduce inside the tile
// and add one exact fixed-point partial per tile row and column to global
// memory, so every result is independent of scheduling (bitwise repeatable).
#pragma once
#include <cstdint>

#include "k_pack.cuh"
#include "rfp.h"

namespace rfp {
namespace knorm {

constexpr int kThreads = 256;

// Device results of one norm / estimator step (read back with one copy).
// Every reduction is deterministic: fixed-order combines inside a CTA,
// per-CTA partials summed in a fixed order, exact integer (fixed-point)
// atomics across CTAs, and order-independent max.
struct Stats {
  double sum;          // sum a^2 (norms) or sum |x| (estimator)
  double diag;         // sum of squared diagonal elements
  unsigned long long key;  // max |a| bits (norms); (|x| bits << 32) | ~index (argmax)
  unsigned long long colmax;  // max column sum (fixed point, see colsum)
  int mismatch;        // estimator: count of sign(x_i) != isgn_i
  int pad;
  float xj;            // estimator: |x[j]| for the caller's previous index j
  float pad2;
};

constexpr int kMaxParts = 148 * 8;  // grid cap of the flat passes (per-CTA partials)

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ unsigned long long warp_max(unsigned long long v) {
  for (int o = 16; o; o >>= 1) {
    const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

// Block-wide sum (fixed order) and max of per-thread values; thread 0
// stores the sum to *part (if given) and max-combines into *gmax.
__device__ __forceinline__ double block_reduce(double s, unsigned long long m, double* part,
                                               unsigned long long* gmax) {
  __shared__ double ss[kThreads / 32];
  __shared__ unsigned long long sm[kThreads / 32];
  s = warp_sum(s);
  m = warp_max(m);
  const int w = threadIdx.x / 32, l = threadIdx.x % 32;
  if (l == 0) { ss[w] = s; sm[w] = m; }
  __syncthreads();
  double t = 0;
  if (threadIdx.x == 0) {
    unsigned long long x = 0;
    for (int i = 0; i < kThreads / 32; ++i) { t += ss[i]; x = sm[i] > x ? sm[i] : x; }
    if (part) *part = t;
    if (gmax) atomicMax(gmax, x);
  }
  return t;
}

__device__ __forceinline__ unsigned abs_bits(float v) {
  return __float_as_uint(v) & 0x7fffffffu;  // NaN keeps the largest patterns
}

// sum a^2 (per-CTA partial into part[blockIdx.x]) and max |a| over the flat
// array (count elements).  Launch with at most kMaxParts CTAs.
__global__ void __launch_bounds__(kThreads) flat_stats(const float* __restrict__ a, int64_t count,
                                                       double* part, Stats* st) {
  double s = 0.0;
  unsigned m = 0;
  const int64_t tid = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  const int64_t lead = (int64_t)(((16 - (reinterpret_cast<uintptr_t>(a) & 15)) & 15) >> 2);
  const int64_t head = lead < count ? lead : count;
  if (tid < head) {
    const float v = a[tid];
    s += (double)v * v;
    m = max(m, abs_bits(v));
  }
  const int64_t nvec = (count - head) >> 2;
  const float4* a4 = reinterpret_cast<const float4*>(a + head);
  for (int64_t e = tid; e < nvec; e += stride) {
    const float4 v = __ldg(a4 + e);
    s += (double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z + (double)v.w * v.w;
    m = max(max(m, abs_bits(v.x)), max(abs_bits(v.y), max(abs_bits(v.z), abs_bits(v.w))));
  }
  for (int64_t e = head + 4 * nvec + tid; e < count; e += stride) {
    const float v = a[e];
    s += (double)v * v;
    m = max(m, abs_bits(v));
  }
  block_reduce(s, (unsigned long long)m, part + blockIdx.x, &st->key);
}

// st->sum := part[0] + ... + part[np - 1] in a fixed order (one CTA).
__global__ void __launch_bounds__(kThreads) sum_parts(const double* __restrict__ part, int np,
                                                      Stats* st) {
  double s = 0.0;
  for (int i = threadIdx.x; i < np; i += kThreads) s += part[i];
  const double t = block_reduce(s, 0ull, nullptr, nullptr);
  if (threadIdx.x == 0) st->sum = t;
}

// sum of squared diagonal elements (one CTA, fixed order).
__global__ void __launch_bounds__(kThreads) diag_sumsq(Geometry g, const float* __restrict__ a,
                                                       Stats* st) {
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < g.n; i += kThreads) {
    const float v = a[diag_offset(g, i)];
    s += (double)v * v;
  }
  const double t = block_reduce(s, 0ull, nullptr, nullptr);
  if (threadIdx.x == 0) st->diag = t;
}

// Fixed-point exponent of the column sums: every column sum is at most
// n max|a| < 2^(e_max), so sums scaled by 2^(62 - e_max) fit in 63 bits.
__device__ __forceinline__ int colsum_shift(const Stats* st, int n) {
  const float amax = __uint_as_float((unsigned)st->key);
  if (!(amax > 0.f) || !(amax <= 3.0e38f)) return 0;  // zero, inf or NaN: handled by the caller
  int e;
  frexp((double)amax * (double)n, &e);  // amax * n < 2^e
  return 62 - e;
}

// Column sums of |A| over the tiles of the RFP blocks (block 32 x 8, one
// 64 x 64 tile per CTA) as 64-bit fixed-point integers (scale 2^shift from
// colsum_shift; the max pass of flat_stats runs first).  Inside a tile every
// partial is combined in a fixed order; across tiles the integer atomics are
// exact, so the result does not depend on scheduling.  col (n words) must
// start at zero.
__global__ void __launch_bounds__(kpack::TX * kpack::TY) colsum(const kpack::PackArgs args,
                                                                const float* __restrict__ arf,
                                                                int n, const Stats* st,
                                                                unsigned long long* col) {
  using namespace kpack;
  __shared__ double lpart[TY][TS];  // lane-indexed partials of each thread row
  __shared__ double wpart[TS];      // warp-indexed partials (one owner each)
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int lin = ty * TX + tx;
  int t = blockIdx.x, bi = 0;
  while (bi + 1 < args.nblocks && t >= args.b[bi + 1].tile_begin) ++bi;
  const PackBlock& B = args.b[bi];
  int tp, tq;
  pack_tile_coords(B, t - B.tile_begin, tp, tq);
  const int p0 = tp * TS, q0 = tq * TS;
  const int prow = B.rows - p0, qcol = B.cols - q0;
  const int64_t P0 = (int64_t)B.p_base + p0, Q0 = (int64_t)B.q_base + q0;
  const float* base = arf + B.off + (int64_t)p0 * B.rs + (int64_t)q0 * B.cs;
  // warp along the contiguous dimension: lane index L, warp index W
  const bool qc = (B.cs == 1 || B.cs == -1);
  const int64_t sl = qc ? B.cs : B.rs, sw = qc ? B.rs : B.cs;
  double accL[TS / TX] = {0.0, 0.0};
#pragma unroll
  for (int r = 0; r < TS / TY; ++r) {
    const int w = ty + TY * r;
    double accW = 0.0;
#pragma unroll
    for (int h = 0; h < TS / TX; ++h) {
      const int l = tx + TX * h;
      const int lp = qc ? w : l, lq = qc ? l : w;
      float v = 0.f;
      if (lp < prow && lq < qcol && (!B.tri || p0 + lp >= q0 + lq))
        v = fabsf(base[(int64_t)l * sl + (int64_t)w * sw]);
      // column q gets every element; row p only the off-diagonal ones
      const float vr = (P0 + lp != Q0 + lq) ? v : 0.f;
      if (qc) { accL[h] += v; accW += vr; }
      else    { accL[h] += vr; accW += v; }
    }
    accW = warp_sum(accW);
    if (tx == 0) wpart[w] = accW;
  }
#pragma unroll
  for (int h = 0; h < TS / TX; ++h) lpart[ty][tx + TX * h] = accL[h];
  __syncthreads();
  const int shift = colsum_shift(st, n);
  if (lin < 2 * TS) {
    const int i = lin % TS;
    const bool lane_side = lin < TS;  // lane-indexed (L) or warp-indexed (W) partial
    double v;
    if (lane_side) {
      v = 0.0;
#pragma unroll
      for (int y = 0; y < TY; ++y) v += lpart[y][i];
    } else {
      v = wpart[i];
    }
    // lane index is q when the warp runs along q, else p
    const bool is_col = lane_side == qc;
    const int lim = is_col ? qcol : prow;
    const int64_t g = (is_col ? Q0 : P0) + i;
    if (i < lim && v != 0.0)
      atomicAdd(col + g, (unsigned long long)llrint(ldexp(v, shift)));
  }
}

// Largest column sum (fixed point) into st->colmax.
__global__ void __launch_bounds__(kThreads) max_of(const unsigned long long* __restrict__ v,
                                                   int n, Stats* st) {
  unsigned long long m = 0;
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * kThreads)
    m = v[i] > m ? v[i] : m;
  block_reduce(0.0, m, nullptr, &st->colmax);
}

// ---------------------------------------------------------------------------
// Estimator vectors (one right-hand side, length n)
// ---------------------------------------------------------------------------

__global__ void fill(float* x, int n, float v) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = v;
}

// x := sign(x), isgn := sign(x) (sign(0) = +1)
__global__ void sign_save(float* x, float* isgn, int n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const float s = x[i] >= 0.f ? 1.f : -1.f;
    x[i] = s;
    isgn[i] = s;
  }
}

// x := e_j (0-based j)
__global__ void unit(float* x, int n, int j) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = i == j ? 1.f : 0.f;
}

// x_i := (-1)^i (1 + i / (n - 1))   (x_0 = 1 for n = 1)
__global__ void altsgn(float* x, int n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const float sc = n > 1 ? 1.f + (float)i / (float)(n - 1) : 1.f;
    x[i] = (i & 1) ? -sc : sc;
  }
}

// sum |x| (FP64), first index of max |x|, the number of i with
// sign(x_i) != isgn_i (zeros match; isgn may be null) and |x[j]| for the
// given j.  One CTA, fixed-order sums.
__global__ void __launch_bounds__(kThreads) vstats(const float* __restrict__ x,
                                                   const float* __restrict__ isgn, int n, int j,
                                                   Stats* st) {
  double s = 0.0;
  unsigned long long key = 0;
  int mis = 0;
  for (int64_t i = threadIdx.x; i < n; i += kThreads) {
    const float v = x[i];
    s += fabs((double)v);
    const unsigned long long k = ((unsigned long long)abs_bits(v) << 32) |
                                 (unsigned long long)(0xffffffffu - (unsigned)i);
    key = k > key ? k : key;
    if (isgn) mis += (v != 0.f && (v > 0.f ? 1.f : -1.f) != isgn[i]);
    if (i == j) st->xj = fabsf(v);
  }
  for (int o = 16; o; o >>= 1) mis += __shfl_xor_sync(0xffffffffu, mis, o);
  if ((threadIdx.x & 31) == 0 && mis) atomicAdd(&st->mismatch, mis);
  const double t = block_reduce(s, key, nullptr, &st->key);
  if (threadIdx.x == 0) st->sum = t;
}

}  // namespace knorm
}  // namespace rfp
