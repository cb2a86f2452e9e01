// k_skinny.cuh — C(m x N) := alpha A(m x k) B(k x N) + beta C for few columns
// (N <= 8): the RFP solves' rectangle update with one or a few right-hand
// sides (spftrs with nrhs <= 8, the condition estimator's solves, the GP
// alpha solve).
//
// Bandwidth-bound: A (an RFP rectangle of up to n^2/4 elements) is read once,
// along its contiguous dimension, with many independent loads in flight per
// thread; B (k x N) is small and is re-read from L1/L2.  There is no split
// of k across CTAs, so no partial sums leave the CTA and nothing is
// allocated: each output element is summed in a fixed order (registers, then
// a fixed-order combine through shared memory or warp shuffles), so the
// result is bitwise repeatable.
//
//  * skinny_rows (A's row index is the unit-stride one): a CTA owns 32 rows,
//    lane = row; its 8 warps take interleaved blocks of U columns kk; the 8
//    warp partials of each output are added in warp order.
//  * skinny_cols (A's column index kk is the unit-stride one): a warp owns
//    RW rows, lane = kk within 32-wide steps; the 32 lane partials of each
//    output are combined by a shuffle butterfly (the same tree in every
//    lane, so the lanes agree bit for bit) and lane 0 writes.
#pragma once
#include <climits>
#include <cstdint>

namespace rfp {
namespace kskinny {

constexpr int kThreads = 256;

template <typename T>
struct Args {
  const T* A; int64_t a_rs, a_cs;
  const T* B; int64_t b_rs, b_cs;
  T* C; int64_t c_rs, c_cs;
  int m, n, k;  // n <= N of the instantiation (columns past n are neither read nor written)
  T alpha, beta;
};

template <typename T>
__device__ __forceinline__ void store_out(const Args<T>& a, int i, int c, T s) {
  T* p = a.C + (int64_t)i * a.c_rs + (int64_t)c * a.c_cs;
  *p = a.beta == T(0) ? a.alpha * s : fma(a.beta, *p, a.alpha * s);
}

// Rows per CTA: 32.  Rows past m read row m - 1 (in bounds) and are not
// written.
template <typename T, int N>
__global__ void __launch_bounds__(kThreads) skinny_rows(const Args<T> a, const int* abort_flag) {
  if (abort_flag && *abort_flag != INT_MAX) return;
  constexpr int U = sizeof(T) == 4 ? 32 : 16;  // columns per warp block (loads in flight)
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i = blockIdx.x * 32 + lane;
  const T* Ai = a.A + (int64_t)min(i, a.m - 1) * a.a_rs;
  T acc[N];
#pragma unroll
  for (int c = 0; c < N; ++c) acc[c] = T(0);
  auto step = [&](int kk, T av) {
    const T* bk = a.B + (int64_t)kk * a.b_rs;
#pragma unroll
    for (int c = 0; c < N; ++c)
      if (c < a.n) acc[c] = fma(av, __ldg(bk + (int64_t)c * a.b_cs), acc[c]);
  };
  int k0 = w * U;
  for (; k0 + U <= a.k; k0 += 8 * U) {
    T av[U];
#pragma unroll
    for (int t = 0; t < U; ++t) av[t] = __ldg(Ai + (int64_t)(k0 + t) * a.a_cs);
#pragma unroll
    for (int t = 0; t < U; ++t) step(k0 + t, av[t]);
  }
  if (k0 < a.k)
    for (int t = 0; k0 + t < a.k; ++t) step(k0 + t, __ldg(Ai + (int64_t)(k0 + t) * a.a_cs));
  __shared__ T part[8][N][32];
#pragma unroll
  for (int c = 0; c < N; ++c) part[w][c][lane] = acc[c];
  __syncthreads();
  if (threadIdx.x < 32 * N) {
    const int c = threadIdx.x / 32, l = threadIdx.x % 32, ii = blockIdx.x * 32 + l;
    if (ii < a.m && c < a.n) {
      T s = part[0][c][l];
#pragma unroll
      for (int q = 1; q < 8; ++q) s += part[q][c][l];
      store_out(a, ii, c, s);
    }
  }
}

template <typename T, int N>
__global__ void __launch_bounds__(kThreads) skinny_cols(const Args<T> a, const int* abort_flag) {
  if (abort_flag && *abort_flag != INT_MAX) return;
  constexpr int RW = 4;               // rows per warp (32 per CTA)
  constexpr int U = N <= 2 ? 8 : 4;   // 32-wide steps of kk per iteration
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i0 = (blockIdx.x * 8 + w) * RW;
  const T* Ar[RW];
  bool rok[RW];
#pragma unroll
  for (int r = 0; r < RW; ++r) {  // rows past m read row m - 1 and are not written
    rok[r] = i0 + r < a.m;
    Ar[r] = a.A + (int64_t)min(i0 + r, a.m - 1) * a.a_rs;
  }
  T acc[RW][N];
#pragma unroll
  for (int r = 0; r < RW; ++r)
#pragma unroll
    for (int c = 0; c < N; ++c) acc[r][c] = T(0);
  auto block = [&](int k0, bool guard) {
    T av[U][RW], bv[U][N];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int kk = k0 + 32 * u + lane;
      const bool kok = !guard || kk < a.k;
#pragma unroll
      for (int r = 0; r < RW; ++r) av[u][r] = kok ? __ldg(Ar[r] + (int64_t)kk * a.a_cs) : T(0);
#pragma unroll
      for (int c = 0; c < N; ++c)
        bv[u][c] = (kok && c < a.n) ? __ldg(a.B + (int64_t)kk * a.b_rs + (int64_t)c * a.b_cs)
                                    : T(0);
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int r = 0; r < RW; ++r)
#pragma unroll
        for (int c = 0; c < N; ++c) acc[r][c] = fma(av[u][r], bv[u][c], acc[r][c]);
  };
  int k0 = 0;
  for (; k0 + 32 * U <= a.k; k0 += 32 * U) block(k0, false);
  if (k0 < a.k) block(k0, true);
#pragma unroll
  for (int r = 0; r < RW; ++r)
#pragma unroll
    for (int c = 0; c < N; ++c) {
      T v = acc[r][c];
#pragma unroll
      for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      acc[r][c] = v;
    }
  if (lane == 0) {
#pragma unroll
    for (int r = 0; r < RW; ++r)
      if (rok[r])
#pragma unroll
        for (int c = 0; c < N; ++c)
          if (c < a.n) store_out(a, i0 + r, c, acc[r][c]);
  }
}

}  // namespace kskinny
}  // namespace rfp
