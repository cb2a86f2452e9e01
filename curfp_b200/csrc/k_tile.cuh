// k_tile.cuh — single-CTA kernels on small triangular tiles held in shared
// memory: the diagonal Cholesky tile (the only place pivots are checked), the
// inverses of diagonal blocks used by the blocked TRSM, and the in-place
// inverse / L^T L tiles of the blocked spftri.
#pragma once
#include <climits>
#include <cstdint>

#include "engine.h"

namespace rfp {
namespace ktile {

constexpr int T = 64;        // tile size (== kPotrfTile == kTrsmLeaf == kTriTile)
constexpr int LD = T + 1;    // padded shared-memory leading dimension

static_assert(T == kPotrfTile && T == kTrsmLeaf && T == kTriTile,
              "tile kernels assume one tile size");

// Lower-triangular Cholesky of an n x n (n <= 64) tile, right-looking, one
// column per step.  Thread t owns column t % 64 and rows t/64 + 4r.
// On a pivot that is not > 0 (or NaN) the device info word becomes
// min(info, info_base + j + 1), the partially factored tile is written back
// and the kernel returns (LAPACK xPOTF2 semantics).
__global__ void __launch_bounds__(256) potrf_tile(View L, int n, int info_base,
                                                  int* info) {
  if (info && *info != INT_MAX) return;
  __shared__ float s[T][LD];
  const int tid = threadIdx.x;
  for (int e = tid; e < n * n; e += 256) {
    int i = e % n, j = e / n;
    s[i][j] = (i >= j) ? L.p[(int64_t)i * L.rs + (int64_t)j * L.cs] : 0.f;
  }
  __syncthreads();
  const int col = tid % T, row0 = tid / T;
  int fail = 0;
  for (int j = 0; j < n; ++j) {
    const float d = s[j][j];
    if (!(d > 0.f)) {  // also catches NaN
      fail = j + 1;
      break;
    }
    const float ljj = sqrtf(d);
    __syncthreads();  // every thread has read s[j][j]
    if (col == j) {
      for (int i = row0; i < n; i += 4) {
        if (i > j) s[i][j] = s[i][j] / ljj;
        else if (i == j) s[j][j] = ljj;
      }
    }
    __syncthreads();
    if (col > j && col < n) {
      const float lkj = s[col][j];
      for (int i = row0; i < n; i += 4)
        if (i >= col) s[i][col] = fmaf(-s[i][j], lkj, s[i][col]);
    }
    __syncthreads();
  }
  if (fail && tid == 0) atomicMin(info, info_base + fail);
  for (int e = tid; e < n * n; e += 256) {
    int i = e % n, j = e / n;
    if (i >= j) L.p[(int64_t)i * L.rs + (int64_t)j * L.cs] = s[i][j];
  }
}

// Inverse of lower-triangular diagonal blocks.  Block b = blockIdx.x covers
// rows/cols [b*64, min(n, b*64+64)).  Thread c computes column c of the
// inverse by forward substitution (all threads walk the same (i,k) so the
// reads of the tile are broadcasts).  W != nullptr: block b is written to
// W + b*64*64 (column-major, ld 64, zeros above the diagonal and outside the
// block); W == nullptr: the inverse replaces the lower triangle in place.
__global__ void __launch_bounds__(T) trtri_blocks(View L, int n, float* W,
                                                  const int* abort_flag) {
  if (abort_flag && *abort_flag != INT_MAX) return;
  __shared__ float s[T][LD];
  __shared__ float x[T][LD];
  const int b = blockIdx.x, r0 = b * T;
  const int sz = min(T, n - r0);
  const int c = threadIdx.x;
  const View Lb = sub(L, r0, r0);
  for (int i = 0; i < T; ++i) {
    // thread c loads column c of row i: coalesced when cs == +-1
    float v = 0.f;
    if (i < sz && c <= i) v = Lb.p[(int64_t)i * Lb.rs + (int64_t)c * Lb.cs];
    s[i][c] = v;
    x[i][c] = 0.f;
  }
  __syncthreads();
  if (c < sz) {
    x[c][c] = 1.0f / s[c][c];
    for (int i = c + 1; i < sz; ++i) {
      float acc = 0.f;
      for (int k = c; k < i; ++k) acc = fmaf(s[i][k], x[k][c], acc);
      x[i][c] = -acc / s[i][i];
    }
  }
  __syncthreads();
  if (W) {
    float* Wb = W + (int64_t)b * T * T;
    for (int j = 0; j < T; ++j) Wb[(int64_t)j * T + c] = (c < sz && j < sz) ? x[c][j] : 0.f;
  } else {
    for (int i = 0; i < sz; ++i)
      if (c <= i) Lb.p[(int64_t)i * Lb.rs + (int64_t)c * Lb.cs] = x[i][c];
  }
}

// In-place L := L^T L (lower part) for an n x n tile, n <= 64.
// (L^T L)(i,j) = sum_{k >= i} L(k,i) L(k,j) for i >= j.
__global__ void __launch_bounds__(256) lauum_tile(View L, int n) {
  __shared__ float s[T][LD];
  const int tid = threadIdx.x;
  for (int e = tid; e < n * n; e += 256) {
    int i = e % n, j = e / n;
    s[i][j] = (i >= j) ? L.p[(int64_t)i * L.rs + (int64_t)j * L.cs] : 0.f;
  }
  __syncthreads();
  float out[16];
  const int j = tid % T, i0 = tid / T;
#pragma unroll
  for (int r = 0; r < 16; ++r) {
    const int i = i0 + 4 * r;
    float acc = 0.f;
    if (i < n && j < n && i >= j)
      for (int k = i; k < n; ++k) acc = fmaf(s[k][i], s[k][j], acc);
    out[r] = acc;
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < 16; ++r) {
    const int i = i0 + 4 * r;
    if (i < n && j < n && i >= j)
      L.p[(int64_t)i * L.rs + (int64_t)j * L.cs] = out[r];
  }
}

}  // namespace ktile
}  // namespace rfp
