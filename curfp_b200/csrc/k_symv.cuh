// k_symv.cuh — y := alpha A x + beta y for a symmetric A held in RFP (any
// variant), one right-hand side (ssfmv / dsfmv).
//
// Bandwidth-bound: each CTA owns 64 rows of y and sweeps the 64-wide column
// blocks; the 64 x 64 tile (rows i0.., columns j0..) of the symmetric matrix
// is read through the RFP block that stores it, with the warp along the
// block's contiguous dimension, so the reads coalesce (each stored element is
// read twice over the launch, once per symmetric half).  A tile that lies in
// one RFP block and off the diagonal is addressed by a base pointer and two
// strides; the diagonal tiles (and any tile across the n1 boundary) take
// per-element offsets.  Products are summed in the element type in a fixed
// order (registers, then a fixed-order combine through shared memory): the
// result is bitwise repeatable.
#pragma once
#include <cstdint>

#include "rfp.h"

namespace rfp {
namespace ksymv {

constexpr int TB = 64;
constexpr int kThreads = 256;

// x[j0 .. j0 + 15] (BLAS increment inc, zero past n): four 16-byte loads when
// the run is contiguous and aligned.
__device__ __forceinline__ void load16(const float* x, int j0, int64_t inc, int n,
                                       float (&v)[16]) {
  const float* p = x + (int64_t)j0 * inc;
  if (inc == 1 && j0 + 16 <= n && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float4 w = __ldg(reinterpret_cast<const float4*>(p) + q);
      v[4 * q] = w.x; v[4 * q + 1] = w.y; v[4 * q + 2] = w.z; v[4 * q + 3] = w.w;
    }
  } else {
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = j0 + r < n ? __ldg(p + r * inc) : 0.f;
  }
}
__device__ __forceinline__ void load16(const double* x, int j0, int64_t inc, int n,
                                       double (&v)[16]) {
  const double* p = x + (int64_t)j0 * inc;
  if (inc == 1 && j0 + 16 <= n && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const double2 w = __ldg(reinterpret_cast<const double2*>(p) + q);
      v[2 * q] = w.x; v[2 * q + 1] = w.y;
    }
  } else {
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = j0 + r < n ? __ldg(p + r * inc) : 0.0;
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads)
    symv_rows(Geometry g, const T* __restrict__ arf, const T* __restrict__ x, int64_t incx,
              T* y, int64_t incy, T alpha, T beta) {
  const int n = g.n;
  const int i0 = blockIdx.x * TB;
  const int tid = threadIdx.x, tl = tid % TB, tg = tid / TB;  // tg in 0..3
  T acc_row = T(0);        // warp along i: this thread's row tl
  T acc_rows[16];          // warp along j: rows 16 tg + r
#pragma unroll
  for (int r = 0; r < 16; ++r) acc_rows[r] = T(0);

  for (int j0 = 0; j0 < n; j0 += TB) {
    const bool lower = i0 >= j0;
    const int64_t pb = lower ? i0 : j0, qb = lower ? j0 : i0;
    const int64_t pm = min((int64_t)n - 1, pb + TB - 1), qm = min((int64_t)n - 1, qb + TB - 1);
    const bool one_block = (pb < g.n1) == (pm < g.n1) && (qb < g.n1) == (qm < g.n1);
    if (i0 != j0 && one_block) {
      const BlockGeom& bg = qb < g.n1 ? (pb < g.n1 ? g.b11 : g.b21) : g.b22;
      const int64_t pbase = pb < g.n1 ? 0 : g.n1, qbase = qb < g.n1 ? 0 : g.n1;
      const T* base = arf + bg.off + (pb - pbase) * bg.rs + (qb - qbase) * bg.cs;
      // element (li, lj) of the tile: lower tile (p, q) = (i, j), upper (j, i)
      const int64_t s_li = lower ? bg.rs : bg.cs, s_lj = lower ? bg.cs : bg.rs;
      const bool i_fast = (s_li == 1 || s_li == -1);
      if (i_fast) {  // this thread: row tl, the 16 consecutive columns 16 tg + r
        const bool row_ok = i0 + tl < n;
        const int jb = j0 + 16 * tg;
        T xs[16];
        load16(x, jb, incx, n, xs);
        T s = T(0);
#pragma unroll
        for (int r = 0; r < 16; ++r) {
          if (row_ok && jb + r < n)
            s = fma(base[(int64_t)tl * s_li + (int64_t)(16 * tg + r) * s_lj], xs[r], s);
        }
        acc_row += s;
      } else {  // this thread: column tl, the 16 consecutive rows 16 tg + r
        const bool col_ok = j0 + tl < n;
        const T xv = col_ok ? x[(j0 + tl) * incx] : T(0);
#pragma unroll
        for (int r = 0; r < 16; ++r) {
          const int li = 16 * tg + r;
          if (col_ok && i0 + li < n)
            acc_rows[r] = fma(base[(int64_t)li * s_li + (int64_t)tl * s_lj], xv, acc_rows[r]);
        }
      }
    } else {  // diagonal tile or a tile across the n1 boundary
      const int64_t i = i0 + tl;
      T s = T(0);
#pragma unroll 4
      for (int r = 0; r < 16; ++r) {
        const int64_t j = j0 + 16 * tg + r;
        if (i < n && j < n)
          s = fma(arf[i >= j ? lower_offset(g, i, j) : lower_offset(g, j, i)], x[j * incx], s);
      }
      acc_row += s;
    }
  }

  // Fixed-order combine: row li gets the four acc_row of threads (li, tg) and
  // the 64 acc_rows[li % 16] of the threads with tg == li / 16.
  __shared__ T part_a[4][TB];
  __shared__ T part_b[2 * 4][16];  // [warp][r]: one partial per warp of each row group
  part_a[tg][tl] = acc_row;
  const int warp = tid / 32, lane = tid % 32;
#pragma unroll
  for (int r = 0; r < 16; ++r) {
    T v = acc_rows[r];
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) part_b[warp][r] = v;
  }
  __syncthreads();
  if (tid < TB) {
    const int li = tid, i = i0 + li;
    if (i < n) {
      const int grp = li / 16, r = li % 16;  // threads with tg == grp: warps 2 grp, 2 grp + 1
      T s = part_a[0][li] + part_a[1][li] + part_a[2][li] + part_a[3][li];
      s += part_b[2 * grp][r] + part_b[2 * grp + 1][r];
      T* yi = y + (int64_t)i * incy;
      *yi = beta == T(0) ? alpha * s : fma(beta, *yi, alpha * s);
    }
  }
}

}  // namespace ksymv
}  // namespace rfp
