// k_refine.cuh — kernels of the iterative-refinement solve.
//
// symm_acc64: Y := alpha * A X + beta * Y for a symmetric A held in RFP (any
// variant) and column-major X, Y (n x nrhs).  Products of the FP32 inputs are
// exact in FP64 and are summed in FP64; each output is rounded to FP32 once.
// This is the only FP64 arithmetic of the solver (the residual b - A x).
// One CTA owns a 64-row x 64-column output block and sweeps the 64-wide column
// blocks of A; A elements are addressed through the RFP geometry (the upper
// half of the symmetric matrix is read from the stored lower element).
#pragma once
#include <cstdint>

#include "rfp.h"

namespace rfp {
namespace kref {

constexpr int TB = 64;

// Operands are converted to FP64 once, when staged in shared memory, so the
// inner loop is pure DFMA (16 per 8 shared loads).  The loads of the next
// 64-wide column block are issued before the current block is multiplied
// (software pipelining through registers).  gridDim.z splits the sum over
// the column blocks; with a split the partial sums are added atomically into
// an FP64 accumulator R (n x nrhs, zeroed) and symm_finish rounds once.
// Dynamic shared memory: 2 x 64 x 65 doubles.
constexpr int SYMM_SMEM = 2 * TB * (TB + 1) * 8;

__device__ __forceinline__ void symm_load(const Geometry& g, const float* __restrict__ arf,
                                          const float* __restrict__ X, int64_t ldx, int nrhs,
                                          int i0, int c0, int j0, int tid, float* av,
                                          float* xv, bool& i_fast) {
  const int n = g.n;
  // The warp runs along the RFP block's contiguous direction: element (i,j)
  // of the symmetric matrix is the stored lower element (max, min) = (p, q)
  // at off + p*rs + q*cs.
  const bool lower_tile = i0 >= j0;
  const int64_t p0 = lower_tile ? i0 : j0, q0 = lower_tile ? j0 : i0;
  const BlockGeom& bg = q0 < g.n1 ? (p0 < g.n1 ? g.b11 : g.b21) : g.b22;
  const bool p_cont = (bg.rs == 1 || bg.rs == -1);
  i_fast = lower_tile ? p_cont : !p_cont;
#pragma unroll
  for (int r = 0; r < 16; ++r) {
    const int e = tid + 256 * r;
    const int li = i_fast ? e % TB : e / TB, lj = i_fast ? e / TB : e % TB;
    const int64_t i = i0 + li, j = j0 + lj;
    av[r] = (i < n && j < n) ? arf[i >= j ? lower_offset(g, i, j) : lower_offset(g, j, i)]
                             : 0.f;
    const int64_t xr = j0 + (e % TB), c = c0 + (e / TB);  // X column-major: rows fastest
    xv[r] = (xr < n && c < nrhs) ? X[xr + c * ldx] : 0.f;
  }
}

__global__ void __launch_bounds__(256) symm_acc64(Geometry g, const float* __restrict__ arf,
                                                  const float* __restrict__ X, int64_t ldx,
                                                  float* Y, int64_t ldy, int nrhs,
                                                  float alpha, float beta, double* R) {
  extern __shared__ double dsm[];
  double (*As)[TB + 1] = reinterpret_cast<double (*)[TB + 1]>(dsm);
  double (*Xs)[TB + 1] = reinterpret_cast<double (*)[TB + 1]>(dsm + TB * (TB + 1));
  const int n = g.n;
  const int i0 = blockIdx.x * TB, c0 = blockIdx.y * TB;
  const int tid = threadIdx.x;
  const int tr = tid / 16, tc = tid % 16;
  const int nblk = (n + TB - 1) / TB;
  const int per = (nblk + gridDim.z - 1) / gridDim.z;
  const int jb0 = blockIdx.z * per, jb1 = min(nblk, jb0 + per);
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;

  float av[16], xv[16];
  bool i_fast = true;
  if (jb0 < jb1) symm_load(g, arf, X, ldx, nrhs, i0, c0, jb0 * TB, tid, av, xv, i_fast);
  for (int jb = jb0; jb < jb1; ++jb) {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      const int e = tid + 256 * r;
      const int li = i_fast ? e % TB : e / TB, lj = i_fast ? e / TB : e % TB;
      As[li][lj] = (double)av[r];
      Xs[e % TB][e / TB] = (double)xv[r];
    }
    __syncthreads();
    if (jb + 1 < jb1)
      symm_load(g, arf, X, ldx, nrhs, i0, c0, (jb + 1) * TB, tid, av, xv, i_fast);
    // rows tr + 16 p, columns tc + 16 q: consecutive threads read
    // consecutive doubles of an Xs row (no bank conflicts)
#pragma unroll 8
    for (int k = 0; k < TB; ++k) {
      double a[4], x[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        a[q] = As[tr + 16 * q][k];
        x[q] = Xs[k][tc + 16 * q];
      }
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] = fma(a[p], x[q], acc[p][q]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int64_t i = i0 + tr + 16 * p;
    if (i >= n) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int64_t c = c0 + tc + 16 * q;
      if (c >= nrhs) continue;
      if (R) {
        atomicAdd(R + i + c * (int64_t)n, acc[p][q]);
      } else {
        float* y = Y + i + c * ldy;
        double v = (double)alpha * acc[p][q];
        if (beta != 0.f) v += (double)beta * (double)*y;
        *y = (float)v;
      }
    }
  }
}

// The same product with a wider register tile, for nrhs >= 32: one CTA of
// 128 threads owns a 128-row x 64-column output block, each thread 8 x 8
// FP64 accumulators on rows {2 tr, 2 tr + 1} + 32 q and columns
// {2 tc, 2 tc + 1} + 16 q (q < 4).  Per k the thread reads its 8 A and 8 X
// values as eight 16-byte shared loads, all conflict-free or broadcast
// (consecutive tr / tc read consecutive 16-byte words), for 64 DFMA: half
// the shared-memory bytes per DFMA of the 4 x 4 tile above, which the FP64
// pipe can consume at full rate.  A 128 x 32 block of A (addressed through
// the RFP geometry, the upper half from the stored lower element) and a
// 32 x 64 block of X are loaded into registers one block ahead, converted
// to FP64 once and staged k-major.  gridDim.z splits the sum over the
// 32-wide column blocks as in symm_acc64.
constexpr int WR = 128, WC = 64, WK = 32, WTHREADS = 128;
// k-major rows padded by two doubles: 16-byte aligned, and the staging
// stores of one warp (consecutive k) spread over the banks
constexpr int WRP = WR + 2, WCP = WC + 2;
constexpr int SYMMW_SMEM = WK * (WRP + WCP) * 8;  // 48.5 KB

__global__ void __launch_bounds__(WTHREADS, 2)
    symm_acc64_wide(Geometry g, const float* __restrict__ arf, const float* __restrict__ X,
                    int64_t ldx, float* Y, int64_t ldy, int nrhs, float alpha, float beta,
                    double* R) {
  extern __shared__ double dsw[];
  double* As = dsw;             // [WK][WRP]: element (row, k) at As[k * WRP + row]
  double* Xs = dsw + WK * WRP;  // [WK][WCP]
  const int n = g.n;
  const int i0 = blockIdx.x * WR, c0 = blockIdx.y * WC;
  const int tid = threadIdx.x;
  const int tr = tid / 8, tc = tid % 8;
  const int nkb = (n + WK - 1) / WK;
  const int per = (nkb + gridDim.z - 1) / gridDim.z;
  const int kb0 = blockIdx.z * per, kb1 = min(nkb, kb0 + per);
  double acc[8][8];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b) acc[a][b] = 0.0;

  float av[WR * WK / WTHREADS], xv[WK * WC / WTHREADS];  // 32 + 16
  bool i_fast = true;
  auto load = [&](int k0) {
    // the warp runs along the RFP block's contiguous direction (see symm_load)
    const bool lower_tile = i0 >= k0;
    const int64_t p0 = lower_tile ? i0 : k0, q0 = lower_tile ? k0 : i0;
    const BlockGeom& bg = q0 < g.n1 ? (p0 < g.n1 ? g.b11 : g.b21) : g.b22;
    const bool p_cont = (bg.rs == 1 || bg.rs == -1);
    i_fast = lower_tile ? p_cont : !p_cont;
#pragma unroll
    for (int r = 0; r < WR * WK / WTHREADS; ++r) {
      const int e = tid + WTHREADS * r;
      const int li = i_fast ? e % WR : e / WK, lk = i_fast ? e / WR : e % WK;
      const int64_t i = i0 + li, j = k0 + lk;
      av[r] = (i < n && j < n) ? arf[i >= j ? lower_offset(g, i, j) : lower_offset(g, j, i)]
                               : 0.f;
    }
#pragma unroll
    for (int r = 0; r < WK * WC / WTHREADS; ++r) {
      const int e = tid + WTHREADS * r;
      const int64_t xr = k0 + e % WK, c = c0 + e / WK;  // X column-major: rows fastest
      xv[r] = (xr < n && c < nrhs) ? X[xr + c * ldx] : 0.f;
    }
  };
  if (kb0 < kb1) load(kb0 * WK);
  for (int kb = kb0; kb < kb1; ++kb) {
#pragma unroll
    for (int r = 0; r < WR * WK / WTHREADS; ++r) {
      const int e = tid + WTHREADS * r;
      const int li = i_fast ? e % WR : e / WK, lk = i_fast ? e / WR : e % WK;
      As[lk * WRP + li] = (double)av[r];
    }
#pragma unroll
    for (int r = 0; r < WK * WC / WTHREADS; ++r) {
      const int e = tid + WTHREADS * r;
      Xs[(e % WK) * WCP + e / WK] = (double)xv[r];
    }
    __syncthreads();
    if (kb + 1 < kb1) load((kb + 1) * WK);
#pragma unroll 4
    for (int k = 0; k < WK; ++k) {
      double a[8], x[8];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double2 av2 = *reinterpret_cast<const double2*>(As + k * WRP + 2 * tr + 32 * q);
        const double2 xv2 = *reinterpret_cast<const double2*>(Xs + k * WCP + 2 * tc + 16 * q);
        a[2 * q] = av2.x; a[2 * q + 1] = av2.y;
        x[2 * q] = xv2.x; x[2 * q + 1] = xv2.y;
      }
#pragma unroll
      for (int p = 0; p < 8; ++p)
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[p][q] = fma(a[p], x[q], acc[p][q]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int p = 0; p < 8; ++p) {
    const int64_t i = i0 + 2 * tr + (p & 1) + 32 * (p >> 1);
    if (i >= n) continue;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int64_t c = c0 + 2 * tc + (q & 1) + 16 * (q >> 1);
      if (c >= nrhs) continue;
      if (R) {
        atomicAdd(R + i + c * (int64_t)n, acc[p][q]);
      } else {
        float* y = Y + i + c * ldy;
        double v = (double)alpha * acc[p][q];
        if (beta != 0.f) v += (double)beta * (double)*y;
        *y = (float)v;
      }
    }
  }
}

// Y := alpha * R + beta * Y (R the FP64 accumulator of a split symm_acc64).
__global__ void symm_finish(const double* __restrict__ R, int n, int nrhs, float* Y,
                            int64_t ldy, float alpha, float beta) {
  const int64_t total = (int64_t)n * nrhs;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = e / n, i = e % n;
    float* y = Y + i + c * ldy;
    double v = (double)alpha * R[e];
    if (beta != 0.f) v += (double)beta * (double)*y;
    *y = (float)v;
  }
}

// max |R| over an n x nrhs column-major block into *out (as float bits; the
// values are non-negative so integer max orders them).  *out must start at 0.
__global__ void absmax(const float* __restrict__ R, int64_t ld, int n, int nrhs,
                       unsigned* out) {
  float m = 0.f;
  const int64_t total = (int64_t)n * nrhs;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = e / n, i = e % n;
    const float v = fabsf(R[i + c * ld]);
    m = (v > m || v != v) ? v : m;
  }
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

// X := X + D (column-major n x nrhs blocks).
__global__ void add_inplace(float* X, int64_t ldx, const float* D, int64_t ldd, int n,
                            int nrhs) {
  const int64_t total = (int64_t)n * nrhs;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = e / n, i = e % n;
    X[i + c * ldx] += D[i + c * ldd];
  }
}

// Dst := Src (column-major n x nrhs blocks with their own leading dimensions).
__global__ void copy_block(float* Dst, int64_t ldd, const float* Src, int64_t lds, int n,
                           int nrhs) {
  const int64_t total = (int64_t)n * nrhs;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = e / n, i = e % n;
    Dst[i + c * ldd] = Src[i + c * lds];
  }
}

}  // namespace kref
}  // namespace rfp
