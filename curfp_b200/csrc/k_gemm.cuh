// k_gemm.cuh — FP32 SIMT GEMM over strided views, several independent
// problems per launch (the plain-FP32 contraction engine).
//
// C(m x n) := alpha * (A B + A2 B2) + beta * C on views whose element (i,j)
// is p[i*rs + j*cs]; strides may be negative and either dimension may be the
// contiguous one, so RFP blocks (T1, S, T2 in any of the 8 variants, their
// transposes and their index reversals) are addressed in place, never
// unpacked.  One CTA computes a BM x BN tile with 256 threads, each holding a
// (BM/16) x (BN/16) register tile; A and B tiles of depth 16 are staged in
// shared memory by 4-byte cp.async with zero fill (RFP leading dimensions are
// often odd, so 16-byte vector loads are not generally legal), double
// buffered.  The global-load thread mapping follows the contiguous dimension
// of each operand so every warp-wide load is coalesced.
//
// c_lower problems enumerate only tiles on or below the diagonal and mask the
// diagonal tiles element-wise, which is how SYRK updates of the RFP triangles
// never touch the other triangle that shares their storage.
#pragma once
#include <climits>
#include <cstdint>

#include "engine.h"

namespace rfp {
namespace kgemm {

constexpr int kThreads = 256;
constexpr int kBK = 16;
constexpr int kPad = 4;

struct Prob {
  const float* A; int64_t a_rs, a_cs;
  const float* B; int64_t b_rs, b_cs;
  const float* A2; int64_t a2_rs, a2_cs;
  const float* B2; int64_t b2_rs, b2_cs;
  float* C; int64_t c_rs, c_cs;
  int m, n, k, k2;
  float alpha, beta;
  int c_lower;
  int a_tri, b_tri, a2_tri, b2_tri;  // 0 full, 1 lower, 2 upper (incl. diagonal)
  int tiles_m, tiles_n;
  int tile_begin;
};

struct Batch {
  Prob p[kMaxBatch];
  int count;
  int total_tiles;
  const int* abort_flag;  // if non-null and *abort_flag != INT_MAX: no-op
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async4(void* smem, const float* g, bool pred) {
  unsigned s = smem_u32(smem);
  int sz = pred ? 4 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s),
               "l"(g), "r"(sz));
}
__device__ __forceinline__ void cp_commit() {
  asm volatile("cp.async.commit_group;\n" ::);
}
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Map a linear tile index of a problem to (ti, tj).
__device__ __forceinline__ void tile_coords(const Prob& P, int lt, int& ti,
                                            int& tj) {
  if (!P.c_lower) {
    ti = lt % P.tiles_m;
    tj = lt / P.tiles_m;
    return;
  }
  // Lower triangle of a square tile grid, row-major: lt = ti(ti+1)/2 + tj.
  int r = (int)((sqrt(8.0 * (double)lt + 1.0) - 1.0) * 0.5);
  while ((int64_t)(r + 1) * (r + 2) / 2 <= lt) ++r;
  while ((int64_t)r * (r + 1) / 2 > lt) --r;
  ti = r;
  tj = lt - (int)((int64_t)r * (r + 1) / 2);
}

template <int BM, int BN>
struct Smem {
  float a[2][kBK][BM + kPad];
  float b[2][kBK][BN + kPad];
};

// Stage one BK-deep slice of product (A, B) into shared memory.
template <int BM, int BN>
__device__ __forceinline__ void load_stage(Smem<BM, BN>& sm, int buf,
                                           const float* A, int64_t a_rs,
                                           int64_t a_cs, const float* B,
                                           int64_t b_rs, int64_t b_cs, int m,
                                           int n, int k, int m0, int n0,
                                           int k0, int a_tri, int b_tri) {
  const int tid = threadIdx.x;
  constexpr int LA = BM * kBK / kThreads;
  constexpr int LB = BN * kBK / kThreads;
  const bool a_mcont = (a_rs == 1 || a_rs == -1);
#pragma unroll
  for (int r = 0; r < LA; ++r) {
    int e = tid + kThreads * r;
    int i, kk;
    if (a_mcont) { i = e % BM; kk = e / BM; }
    else         { i = e / kBK; kk = e % kBK; }
    int gi = m0 + i, gk = k0 + kk;
    bool ok = gi < m && gk < k && (a_tri != 1 || gk <= gi) && (a_tri != 2 || gk >= gi);
    const float* src = ok ? A + (int64_t)gi * a_rs + (int64_t)gk * a_cs : A;
    cp_async4(&sm.a[buf][kk][i], src, ok);
  }
  const bool b_ncont = (b_cs == 1 || b_cs == -1);
#pragma unroll
  for (int r = 0; r < LB; ++r) {
    int e = tid + kThreads * r;
    int j, kk;
    if (b_ncont) { j = e % BN; kk = e / BN; }
    else         { j = e / kBK; kk = e % kBK; }
    int gj = n0 + j, gk = k0 + kk;
    bool ok = gj < n && gk < k && (b_tri != 1 || gk >= gj) && (b_tri != 2 || gk <= gj);
    const float* src = ok ? B + (int64_t)gk * b_rs + (int64_t)gj * b_cs : B;
    cp_async4(&sm.b[buf][kk][j], src, ok);
  }
}

template <int BM, int BN>
__global__ void __launch_bounds__(kThreads, 2) sgemm_batch(const Batch batch) {
  if (batch.abort_flag && *batch.abort_flag != INT_MAX) return;
  constexpr int TM = BM / 16, TN = BN / 16;
  constexpr int GM = TM / 4, GN = TN / 4;
  __shared__ __align__(16) Smem<BM, BN> sm;

  // Locate the problem and tile.
  int t = blockIdx.x, pi = 0;
#pragma unroll 1
  while (pi + 1 < batch.count && t >= batch.p[pi + 1].tile_begin) ++pi;
  const Prob& P = batch.p[pi];
  int ti, tj;
  tile_coords(P, t - P.tile_begin, ti, tj);
  const int m0 = ti * BM, n0 = tj * BN;

  const int tid = threadIdx.x;
  const int tr = tid / 16, tc = tid % 16;

  float acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = 0.f;

  const int kt1 = (P.k + kBK - 1) / kBK;
  const int kt2 = (P.k2 + kBK - 1) / kBK;
  const int ktiles = kt1 + kt2;

  auto issue = [&](int kt, int buf) {
    if (kt < kt1)
      load_stage<BM, BN>(sm, buf, P.A, P.a_rs, P.a_cs, P.B, P.b_rs, P.b_cs,
                         P.m, P.n, P.k, m0, n0, kt * kBK, P.a_tri, P.b_tri);
    else
      load_stage<BM, BN>(sm, buf, P.A2, P.a2_rs, P.a2_cs, P.B2, P.b2_rs,
                         P.b2_cs, P.m, P.n, P.k2, m0, n0, (kt - kt1) * kBK, P.a2_tri, P.b2_tri);
  };

  if (ktiles > 0) {
    issue(0, 0);
    cp_commit();
  }
#pragma unroll 1
  for (int kt = 0; kt < ktiles; ++kt) {
    const int buf = kt & 1;
    if (kt + 1 < ktiles) {
      issue(kt + 1, buf ^ 1);
      cp_commit();
      cp_wait<1>();
    } else {
      cp_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kBK; ++kk) {
      float a[TM], b[TN];
#pragma unroll
      for (int g = 0; g < GM; ++g) {
        float4 v = *reinterpret_cast<const float4*>(
            &sm.a[buf][kk][g * (BM / GM) + tr * 4]);
        a[g * 4 + 0] = v.x; a[g * 4 + 1] = v.y;
        a[g * 4 + 2] = v.z; a[g * 4 + 3] = v.w;
      }
#pragma unroll
      for (int g = 0; g < GN; ++g) {
        float4 v = *reinterpret_cast<const float4*>(
            &sm.b[buf][kk][g * (BN / GN) + tc * 4]);
        b[g * 4 + 0] = v.x; b[g * 4 + 1] = v.y;
        b[g * 4 + 2] = v.z; b[g * 4 + 3] = v.w;
      }
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }

  // Epilogue.
  const float alpha = P.alpha, beta = P.beta;
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const int gi = m0 + (i / 4) * (BM / GM) + tr * 4 + (i % 4);
    if (gi >= P.m) continue;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int gj = n0 + (j / 4) * (BN / GN) + tc * 4 + (j % 4);
      if (gj >= P.n) continue;
      if (P.c_lower && gj > gi) continue;
      float* c = P.C + (int64_t)gi * P.c_rs + (int64_t)gj * P.c_cs;
      float v = alpha * acc[i][j];
      if (beta != 0.f) v = fmaf(beta, *c, v);
      *c = v;
    }
  }
}

}  // namespace kgemm
}  // namespace rfp
