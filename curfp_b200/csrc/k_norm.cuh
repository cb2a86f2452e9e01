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
  unsigned long long key;  // norms: bits of max |a| (float or double)
  unsigned long long colmax;  // max column sum (fixed point, see colsum)
  int mismatch;        // estimator: count of sign(x_i) != isgn_i
  int argmax;          // estimator: first index of max |x|
  double xmax;         // estimator: max |x|
  double xj;           // estimator: |x[j]| for the caller's previous index j
};

// Non-negative values order as their bit patterns.
__device__ __forceinline__ unsigned long long abs_key(float v) {
  return __float_as_uint(v) & 0x7fffffffu;  // NaN keeps the largest patterns
}
__device__ __forceinline__ unsigned long long abs_key(double v) {
  return (unsigned long long)__double_as_longlong(v) & 0x7fffffffffffffffull;
}
// The value of a key (host and device): max |a| as double.
__host__ __device__ inline double key_value(unsigned long long key, bool is_double) {
  if (is_double) {
    union { unsigned long long u; double d; } c;
    c.u = key;
    return c.d;
  }
  union { unsigned u; float f; } c;
  c.u = (unsigned)key;
  return (double)c.f;
}

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

// One 16-byte vector of elements.
template <typename T> struct Vec16;
template <> struct Vec16<float> { using type = float4; static constexpr int n = 4; };
template <> struct Vec16<double> { using type = double2; static constexpr int n = 2; };
__device__ __forceinline__ void acc_vec(const float4& v, double& s, unsigned long long& m) {
  s += (double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z + (double)v.w * v.w;
  const unsigned long long a = max(abs_key(v.x), abs_key(v.y)), b = max(abs_key(v.z), abs_key(v.w));
  m = max(m, max(a, b));
}
__device__ __forceinline__ void acc_vec(const double2& v, double& s, unsigned long long& m) {
  s += v.x * v.x + v.y * v.y;
  m = max(m, max(abs_key(v.x), abs_key(v.y)));
}

// sum a^2 (per-CTA partial into part[blockIdx.x]) and max |a| over the flat
// array (count elements).  Launch with at most kMaxParts CTAs.
template <typename T>
__global__ void __launch_bounds__(kThreads) flat_stats(const T* __restrict__ a, int64_t count,
                                                       double* part, Stats* st) {
  using V = typename Vec16<T>::type;
  constexpr int VN = Vec16<T>::n;
  double s = 0.0;
  unsigned long long m = 0;
  const int64_t tid = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  const int64_t lead =
      (int64_t)(((16 - (reinterpret_cast<uintptr_t>(a) & 15)) & 15) / sizeof(T));
  const int64_t head = lead < count ? lead : count;
  if (tid < head) {
    const double v = (double)a[tid];
    s += v * v;
    m = max(m, abs_key(a[tid]));
  }
  const int64_t nvec = (count - head) / VN;
  const V* av = reinterpret_cast<const V*>(a + head);
  for (int64_t e = tid; e < nvec; e += stride) acc_vec(__ldg(av + e), s, m);
  for (int64_t e = head + VN * nvec + tid; e < count; e += stride) {
    const double v = (double)a[e];
    s += v * v;
    m = max(m, abs_key(a[e]));
  }
  block_reduce(s, m, part + blockIdx.x, &st->key);
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
template <typename T>
__global__ void __launch_bounds__(kThreads) diag_sumsq(Geometry g, const T* __restrict__ a,
                                                       Stats* st) {
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < g.n; i += kThreads) {
    const double v = (double)a[diag_offset(g, i)];
    s += v * v;
  }
  const double t = block_reduce(s, 0ull, nullptr, nullptr);
  if (threadIdx.x == 0) st->diag = t;
}

// Fixed-point exponent of the column sums: every column sum is at most
// n max|a| < 2^(e_max), so sums scaled by 2^(62 - e_max) fit in 63 bits.
__host__ __device__ inline int colsum_shift(double amax, int n) {
  if (!(amax > 0.0) || !(amax <= 1.0e300)) return 0;  // zero, inf or NaN: handled by the caller
  int e;
  frexp(amax * (double)n, &e);  // amax * n < 2^e
  return 62 - e;
}

// Column sums of |A| over the tiles of the RFP blocks (block 32 x 8, one
// 64 x 64 tile per CTA) as 64-bit fixed-point integers (scale 2^shift from
// colsum_shift; the max pass of flat_stats runs first).  Inside a tile every
// partial is combined in a fixed order; across tiles the integer atomics are
// exact, so the result does not depend on scheduling.  col (n words) must
// start at zero.
template <typename T>
__global__ void __launch_bounds__(kpack::TX * kpack::TY) colsum(const kpack::PackArgs args,
                                                                const T* __restrict__ arf,
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
  const T* base = arf + B.off + (int64_t)p0 * B.rs + (int64_t)q0 * B.cs;
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
      double v = 0.0;
      if (lp < prow && lq < qcol && (!B.tri || p0 + lp >= q0 + lq))
        v = fabs((double)base[(int64_t)l * sl + (int64_t)w * sw]);
      // column q gets every element; row p only the off-diagonal ones
      const double vr = (P0 + lp != Q0 + lq) ? v : 0.0;
      if (qc) { accL[h] += v; accW += vr; }
      else    { accL[h] += vr; accW += v; }
    }
    accW = warp_sum(accW);
    if (tx == 0) wpart[w] = accW;
  }
#pragma unroll
  for (int h = 0; h < TS / TX; ++h) lpart[ty][tx + TX * h] = accL[h];
  __syncthreads();
  const int shift = colsum_shift(key_value(st->key, sizeof(T) == 8), n);
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

template <typename T>
__global__ void fill(T* x, int n, T v) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = v;
}

// x := sign(x), isgn := sign(x) (sign(0) = +1)
template <typename T>
__global__ void sign_save(T* x, T* isgn, int n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const T s = x[i] >= T(0) ? T(1) : T(-1);
    x[i] = s;
    isgn[i] = s;
  }
}

// x := e_j (0-based j)
template <typename T>
__global__ void unit(T* x, int n, int j) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = i == j ? T(1) : T(0);
}

// x_i := (-1)^i (1 + i / (n - 1))   (x_0 = 1 for n = 1)
template <typename T>
__global__ void altsgn(T* x, int n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const T sc = n > 1 ? T(1) + (T)i / (T)(n - 1) : T(1);
    x[i] = (i & 1) ? -sc : sc;
  }
}

// sum |x| (FP64), the first index of max |x| and that maximum, the number of
// i with sign(x_i) != isgn_i (zeros match; isgn may be null) and |x[j]| for
// the given j.  One CTA, fixed-order reductions.
template <typename T>
__global__ void __launch_bounds__(kThreads) vstats(const T* __restrict__ x,
                                                   const T* __restrict__ isgn, int n, int j,
                                                   Stats* st) {
  __shared__ double sv[kThreads / 32];
  __shared__ int si[kThreads / 32];
  double s = 0.0, best = -1.0;
  int bi = 0, mis = 0;
  for (int64_t i = threadIdx.x; i < n; i += kThreads) {
    const T v = x[i];
    const double a = fabs((double)v);
    s += a;
    if (a > best) { best = a; bi = (int)i; }  // increasing i: ties keep the first
    if (isgn) mis += (v != T(0) && (v > T(0) ? T(1) : T(-1)) != isgn[i]);
    if (i == j) st->xj = a;
  }
  for (int o = 16; o; o >>= 1) {
    const double b2 = __shfl_xor_sync(0xffffffffu, best, o);
    const int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
    if (b2 > best || (b2 == best && i2 < bi)) { best = b2; bi = i2; }
    mis += __shfl_xor_sync(0xffffffffu, mis, o);
  }
  const int w = threadIdx.x / 32;
  if ((threadIdx.x & 31) == 0) { sv[w] = best; si[w] = bi; if (mis) atomicAdd(&st->mismatch, mis); }
  const double t = block_reduce(s, 0ull, nullptr, nullptr);  // synchronises the CTA
  if (threadIdx.x == 0) {
    best = sv[0];
    bi = si[0];
    for (int k = 1; k < kThreads / 32; ++k)
      if (sv[k] > best || (sv[k] == best && si[k] < bi)) { best = sv[k]; bi = si[k]; }
    st->sum = t;
    st->argmax = bi;
    st->xmax = best;
  }
}

}  // namespace knorm
}  // namespace rfp
