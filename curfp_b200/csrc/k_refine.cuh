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
