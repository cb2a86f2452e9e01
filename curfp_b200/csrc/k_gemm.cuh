// k_gemm.cuh — FP32 SIMT GEMM over strided views, several independent
// problems per launch (the plain-FP32 contraction engine).
//
// C(m x n) := alpha * (A B + A2 B2) + beta * C on views whose element (i,j)
// is p[i*rs + j*cs]; strides may be negative and either dimension may be the
// contiguous one, so RFP blocks (T1, S, T2 in any of the 8 variants, their
// transposes and their index reversals) are addressed in place, never
// unpacked.  One CTA computes a BM x BN tile with 256 threads, each holding a
// (BM/16) x (BN/16) register tile; A and B tiles of depth 8-32 are loaded into
// registers one tile ahead (float4 loads where the operand's unit stride,
// base and other stride allow it -- RFP leading dimensions are often odd --
// scalar loads with zero fill otherwise) and stored to double-buffered,
// swizzled shared memory after the FMAs of the current tile.  The
// global-load thread mapping follows the contiguous dimension of each
// operand so every warp-wide load is coalesced.  Triangular operand masks
// also shrink the k range of a tile to the k-tiles they leave non-zero.
//
// c_lower problems enumerate only tiles on or below the diagonal and mask the
// diagonal tiles element-wise, which is how SYRK updates of the RFP triangles
// never touch the other triangle that shares their storage.
#pragma once
#include <climits>
#include <cstdint>

#include "engine.h"
#include "k_order.cuh"

namespace rfp {
namespace kgemm {

constexpr int kThreads = 256;

template <typename T>
struct Prob {
  const T* A; int64_t a_rs, a_cs;
  const T* B; int64_t b_rs, b_cs;
  const T* A2; int64_t a2_rs, a2_cs;
  const T* B2; int64_t b2_rs, b2_cs;
  T* C; int64_t c_rs, c_cs;
  int m, n, k, k2;
  T alpha, beta;
  int c_lower;
  int a_tri, b_tri, a2_tri, b2_tri;  // 0 full, 1 lower, 2 upper (incl. diagonal)
  int tiles_m, tiles_n;
  int tile_begin;
};

template <typename T>
struct Batch {
  Prob<T> p[kMaxBatch];
  int count;
  int total_tiles;
  const int* abort_flag;  // if non-null and *abort_flag != INT_MAX: no-op
};

// Map a linear tile index of a problem to (ti, tj), in the L2-friendly
// orders of k_order.cuh (c_lower problems: lower tile triangle).
template <typename T>
__device__ __forceinline__ void tile_coords(const Prob<T>& P, int lt, int& ti,
                                            int& tj) {
  if (!P.c_lower) order::grouped_tile(P.tiles_m, P.tiles_n, lt, ti, tj);
  else order::tri_band_tile(P.tiles_m, lt, ti, tj);
}

// Shared-memory operand tiles are k-major, s[kk][r] with r the tile row (m
// for A, n for B).  Groups of 4 consecutive r are permuted within aligned
// groups of 8 by kk: the inner loop still reads aligned float4 runs, and the
// transposing stores of k-contiguous operands hit 32 distinct banks (depth
// 32: 8 threads per row, 4 rows per warp, col4 ^ ((kk>>2)&7); depth 16: 4
// threads per row, 8 rows per warp, col4 ^ 2*((kk>>2)&3); depth 8: 2 threads
// per row, 16 rows per warp, col4 ^ 4*((kk>>2)&1)).
template <int BK>
__device__ __forceinline__ int swz(int r, int kk) {
  const int h = BK == 8 ? (((kk >> 2) & 1) << 2)
                        : (BK == 16 ? (((kk >> 2) & 3) << 1) : ((kk >> 2) & 7));
  return (((r >> 2) ^ h) << 2) | (r & 3);
}

// One operand of one product is seen as rows r (m of A or n of B) by kk:
// element (r, kk) at p[r*sr + kk*sk]; tri in the (r, kk) convention: 1 keeps
// kk <= r, 2 keeps kk >= r, 3 keeps kk > r.  Flags: bit 0 = kk is the unit-stride dimension
// (else r), bit 1 = vector loads of 4-element groups allowed (unit stride +1,
// 16-byte aligned base, other stride a multiple of 4).
template <typename T>
__device__ __forceinline__ int operand_flags(const T* p, int64_t sr, int64_t sk) {
  const bool kcont = (sk == 1 || sk == -1) && !(sr == 1 || sr == -1);
  const int64_t unit = kcont ? sk : sr, other = kcont ? sr : sk;
  const bool vec = unit == 1 && (other & 3) == 0 && ((reinterpret_cast<uintptr_t>(p) & 15) == 0);
  return (kcont ? 1 : 0) | (vec ? 2 : 0);
}

// Register staging of one R x BK tile: NG groups of 4 elements along the
// operand's unit-stride dimension, G per thread.
template <typename T, int R, int BK>
struct Stage {
  static constexpr int NG = R * BK / 4;
  static constexpr int G = (NG + kThreads - 1) / kThreads;
  T v[G][4];
};

// Four consecutive elements as 16-byte accesses (one float4 / two double2).
__device__ __forceinline__ void ld4(const float* p, float (&v)[4]) {
  const float4 x = __ldg(reinterpret_cast<const float4*>(p));
  v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
__device__ __forceinline__ void ld4(const double* p, double (&v)[4]) {
  const double2 x = __ldg(reinterpret_cast<const double2*>(p));
  const double2 y = __ldg(reinterpret_cast<const double2*>(p) + 1);
  v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
}
__device__ __forceinline__ void lds4(const float* p, float* v) {
  const float4 x = *reinterpret_cast<const float4*>(p);
  v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
__device__ __forceinline__ void lds4(const double* p, double* v) {
  const double2 x = reinterpret_cast<const double2*>(p)[0];
  const double2 y = reinterpret_cast<const double2*>(p)[1];
  v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
}
__device__ __forceinline__ void sts4(float* p, const float (&v)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void sts4(double* p, const double (&v)[4]) {
  reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}

template <typename T, int R, int BK>
__device__ __forceinline__ void stage_load(Stage<T, R, BK>& st, const T* p, int64_t sr, int64_t sk,
                                           int rows, int depth, int tri, int flags, int r0,
                                           int k0) {
  const int tid = threadIdx.x;
  const bool kcont = flags & 1;
  constexpr int KG = BK / 4;  // groups per row along k
#pragma unroll
  for (int u = 0; u < Stage<T, R, BK>::G; ++u) {
    const int e = tid + kThreads * u;
    if (Stage<T, R, BK>::NG % kThreads != 0 && e >= Stage<T, R, BK>::NG) break;
    int r, kk;  // first element of the group
    if (kcont) { r = e / KG; kk = (e % KG) << 2; }
    else       { r = (e % (R / 4)) << 2; kk = e / (R / 4); }
    const int gr = r0 + r, gk = k0 + kk;
    const int lim_r = rows - gr, lim_k = depth - gk;
    const bool full = tri == 0 && (kcont ? (lim_r > 0 && lim_k >= 4) : (lim_k > 0 && lim_r >= 4));
    if ((flags & 2) && full) {
      ld4(p + (int64_t)gr * sr + (int64_t)gk * sk, st.v[u]);
    } else {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int rr = gr + (kcont ? 0 : c), kc = gk + (kcont ? c : 0);
        const bool ok = rr < rows && kc < depth && (tri != 1 || kc <= rr) &&
                        (tri != 2 || kc >= rr) && (tri != 3 || kc > rr);
        st.v[u][c] = ok ? __ldg(p + (int64_t)rr * sr + (int64_t)kc * sk) : T(0);
      }
    }
  }
}

template <typename T, int R, int BK>
__device__ __forceinline__ void stage_store(const Stage<T, R, BK>& st, T (*s)[R], bool kcont) {
  const int tid = threadIdx.x;
  constexpr int KG = BK / 4;
#pragma unroll
  for (int u = 0; u < Stage<T, R, BK>::G; ++u) {
    const int e = tid + kThreads * u;
    if (Stage<T, R, BK>::NG % kThreads != 0 && e >= Stage<T, R, BK>::NG) break;
    if (kcont) {
      const int r = e / KG, kk = (e % KG) << 2;
#pragma unroll
      for (int c = 0; c < 4; ++c) s[kk + c][swz<BK>(r, kk + c)] = st.v[u][c];
    } else {
      const int r = (e % (R / 4)) << 2, kk = e / (R / 4);
      sts4(&s[kk][swz<BK>(r, kk)], st.v[u]);
    }
  }
}

// One operand's load groups for tiles whose k-tiles are all whole and in
// bounds (no masks): the same groups as stage_load / stage_store, each with
// a pointer that advances one k-tile per load and a fixed shared-memory
// offset.  The four elements of a group share one swizzle (it depends on
// kk >> 2 only), so a k-contiguous group's transposing stores are R apart.
// Steps are 32-bit (the caller keeps strides below 2^26 elements), which
// keeps the 128 x 128 FP32 tile within 128 registers without spills.
template <typename T, int R, int BK>
struct Lane {
  static constexpr int G = Stage<T, R, BK>::G;
  static_assert(Stage<T, R, BK>::NG % kThreads == 0, "whole groups per thread");
  const T* p[G];
  int off[G];
  int step, unit;
  bool kcont, vec;

  __device__ __forceinline__ Lane(const T* base, int64_t sr, int64_t sk, int flags, int r0,
                                  int k0) {
    constexpr int KG = BK / 4;
    kcont = flags & 1;
    vec = flags & 2;
#pragma unroll
    for (int u = 0; u < G; ++u) {
      const int e = threadIdx.x + kThreads * u;
      int r, kk;
      if (kcont) { r = e / KG; kk = (e % KG) << 2; }
      else       { r = (e % (R / 4)) << 2; kk = e / (R / 4); }
      p[u] = base + (int64_t)(r0 + r) * sr + (int64_t)(k0 + kk) * sk;
      off[u] = kk * R + swz<BK>(r, kk);
    }
    step = BK * (int)sk;
    unit = (int)(kcont ? sk : sr);
  }
  __device__ __forceinline__ void load(Stage<T, R, BK>& st) {
#pragma unroll
    for (int u = 0; u < G; ++u) {
      if (vec) {
        ld4(p[u], st.v[u]);
      } else {
#pragma unroll
        for (int c = 0; c < 4; ++c) st.v[u][c] = __ldg(p[u] + c * unit);
      }
      p[u] += step;
    }
  }
  __device__ __forceinline__ void store(const Stage<T, R, BK>& st, T* s) const {
#pragma unroll
    for (int u = 0; u < G; ++u) {
      if (kcont) {
#pragma unroll
        for (int c = 0; c < 4; ++c) s[off[u] + c * R] = st.v[u][c];
      } else {
        sts4(s + off[u], st.v[u]);
      }
    }
  }
};

// k range [kb, ke) of a product that the triangular masks leave non-zero for
// the tile at (m0, n0), rounded out to BK.
template <int BK>
__device__ __forceinline__ void k_range(int k, int a_tri, int b_tri, int m0, int n0, int BM,
                                        int BN, int& kb, int& ke) {
  kb = 0;
  ke = k;
  if (a_tri == 1) ke = min(ke, m0 + BM);   // kk <= i
  if (a_tri == 2 || a_tri == 3) kb = max(kb, m0);  // kk >= i (kk > i)
  if (b_tri == 1) kb = max(kb, n0);        // kk >= j
  if (b_tri == 2) ke = min(ke, n0 + BN);   // kk <= j
  kb = (kb / BK) * BK;
  if (ke < kb) ke = kb;
}

template <typename T, int BM, int BN>
__global__ void __launch_bounds__(kThreads, (sizeof(T) == 8 && BM >= 128) ? 1 : 2)
    sgemm_batch(const Batch<T> batch) {
  if (batch.abort_flag && *batch.abort_flag != INT_MAX) return;
  constexpr int TM = BM / 16, TN = BN / 16;
  constexpr int GM = TM / 4, GN = TN / 4;
  // depth 16 for the FP32 128 x 128 tile (two CTAs per SM, 128 registers,
  // no spills; it halves the per-k-tile barrier and staging work of depth 8:
  // 6.4 against 6.6 ms for ssfrk n = 16384, k = 1024), 8 for the FP64 one;
  // the FP32 64 x 64 tile takes 32 (its FMAs per k-tile then cover the
  // global-load latency of the next one)
  constexpr int BK = BM >= 128 ? (sizeof(T) == 4 ? 16 : 8) : (sizeof(T) == 4 ? 32 : 16);
  __shared__ __align__(16) T sa[2][BK][BM];
  __shared__ __align__(16) T sb[2][BK][BN];

  // Locate the problem and tile.
  int t = blockIdx.x, pi = 0;
#pragma unroll 1
  while (pi + 1 < batch.count && t >= batch.p[pi + 1].tile_begin) ++pi;
  const Prob<T>& P = batch.p[pi];
  int ti, tj;
  tile_coords(P, t - P.tile_begin, ti, tj);
  const int m0 = ti * BM, n0 = tj * BN;

  const int tid = threadIdx.x;
  const int tr = tid / 16, tc = tid % 16;

  T acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = T(0);

  // B's mask codes map to the (r = j, kk) convention: lower B keeps kk >= j
  // (code 2 there), upper keeps kk <= j (code 1).
  auto bcode = [](int b) { return b == 1 ? 2 : (b == 2 ? 1 : 0); };
  const int fl = operand_flags(P.A, P.a_rs, P.a_cs) | (operand_flags(P.B, P.b_cs, P.b_rs) << 2) |
                 (operand_flags(P.A2, P.a2_rs, P.a2_cs) << 4) |
                 (operand_flags(P.B2, P.b2_cs, P.b2_rs) << 6);
  int kb1, ke1, kb2, ke2;
  k_range<BK>(P.k, P.a_tri, P.b_tri, m0, n0, BM, BN, kb1, ke1);
  k_range<BK>(P.k2, P.a2_tri, P.b2_tri, m0, n0, BM, BN, kb2, ke2);
  const int kt1 = (ke1 - kb1 + BK - 1) / BK;
  const int kt2 = (ke2 - kb2 + BK - 1) / BK;
  const int ktiles = kt1 + kt2;

  Stage<T, BM, BK> ra;
  Stage<T, BN, BK> rb;
  auto load = [&](int kt) {
    if (kt < kt1) {
      const int k0 = kb1 + kt * BK;
      stage_load<T, BM, BK>(ra, P.A, P.a_rs, P.a_cs, P.m, P.k, P.a_tri, fl & 3, m0, k0);
      stage_load<T, BN, BK>(rb, P.B, P.b_cs, P.b_rs, P.n, P.k, bcode(P.b_tri), (fl >> 2) & 3, n0,
                            k0);
    } else {
      const int k0 = kb2 + (kt - kt1) * BK;
      stage_load<T, BM, BK>(ra, P.A2, P.a2_rs, P.a2_cs, P.m, P.k2, P.a2_tri, (fl >> 4) & 3, m0,
                            k0);
      stage_load<T, BN, BK>(rb, P.B2, P.b2_cs, P.b2_rs, P.n, P.k2, bcode(P.b2_tri), (fl >> 6) & 3,
                            n0, k0);
    }
  };
  auto store = [&](int kt, int buf) {
    const int f = kt >= kt1 ? fl >> 4 : fl;
    stage_store<T, BM, BK>(ra, sa[buf], f & 1);
    stage_store<T, BN, BK>(rb, sb[buf], (f >> 2) & 1);
  };

  // The FMAs of one k-tile from shared buffer buf.  Both main loops below
  // run this same sequence, so a tile's result does not depend on the loop.
  auto fmas = [&](int buf) {
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      T a[TM], b[TN];
#pragma unroll
      for (int g = 0; g < GM; ++g)
        lds4(&sa[buf][kk][swz<BK>(g * (BM / GM) + tr * 4, kk)], a + g * 4);
      if constexpr (sizeof(T) == 8) {
        // FP64: column pairs 2 tc + 32 h, so that consecutive lanes read
        // consecutive 16-byte pairs (groups of four doubles would put the
        // lanes 32 bytes apart and conflict)
#pragma unroll
        for (int h = 0; h < TN / 2; ++h) {
          const double2 v =
              *reinterpret_cast<const double2*>(&sb[buf][kk][swz<BK>(tc * 2 + 32 * h, kk)]);
          b[2 * h] = v.x;
          b[2 * h + 1] = v.y;
        }
      } else {
#pragma unroll
        for (int g = 0; g < GN; ++g)
          lds4(&sb[buf][kk][swz<BK>(g * (BN / GN) + tc * 4, kk)], b + g * 4);
      }
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
  };

  // Interior tiles of single-product problems without triangular masks (the
  // bulk of a large update): every k-tile is whole and in bounds, so each
  // thread's load groups advance by a fixed pointer step and land at fixed
  // shared-memory offsets, with no bounds or mask arithmetic per k-tile.
  // The values loaded are the ones the general loop loads.  FP32 only: the
  // FP64 tiles measured slower with it (dsfrk n = 16384, k = 512: 7.57
  // against 7.43 ms; dpftrf n = 16384: 112.5 against 107.4 ms).
  auto small = [](int64_t s) { return s > -(int64_t(1) << 26) && s < (int64_t(1) << 26); };
  const bool whole = sizeof(T) == 4 && kt2 == 0 && P.a_tri == 0 && P.b_tri == 0 && m0 + BM <= P.m &&
                     n0 + BN <= P.n && (ke1 - kb1) % BK == 0 && small(P.a_rs) &&
                     small(P.a_cs) && small(P.b_rs) && small(P.b_cs);
  if (whole) {
    Lane<T, BM, BK> la(P.A, P.a_rs, P.a_cs, fl & 3, m0, kb1);
    Lane<T, BN, BK> lb(P.B, P.b_cs, P.b_rs, (fl >> 2) & 3, n0, kb1);
    if (ktiles > 0) {
      la.load(ra);
      lb.load(rb);
      la.store(ra, &sa[0][0][0]);
      lb.store(rb, &sb[0][0][0]);
      __syncthreads();
    }
#pragma unroll 1
    for (int kt = 0; kt < ktiles; ++kt) {
      const int buf = kt & 1;
      const bool more = kt + 1 < ktiles;
      if (more) {  // global loads in flight during the FMAs
        la.load(ra);
        lb.load(rb);
      }
      fmas(buf);
      if (more) {
        la.store(ra, &sa[buf ^ 1][0][0]);
        lb.store(rb, &sb[buf ^ 1][0][0]);
      }
      __syncthreads();
    }
  } else {
    if (ktiles > 0) {
      load(0);
      store(0, 0);
      __syncthreads();
    }
#pragma unroll 1
    for (int kt = 0; kt < ktiles; ++kt) {
      const int buf = kt & 1;
      const bool more = kt + 1 < ktiles;
      if (more) load(kt + 1);  // global loads in flight during the FMAs
      fmas(buf);
      if (more) store(kt + 1, buf ^ 1);
      __syncthreads();
    }
  }

  // Epilogue.
  const T alpha = P.alpha, beta = P.beta;
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const int gi = m0 + (i / 4) * (BM / GM) + tr * 4 + (i % 4);
    if (gi >= P.m) continue;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int gj = sizeof(T) == 8 ? n0 + tc * 2 + 32 * (j / 2) + (j % 2)
                                    : n0 + (j / 4) * (BN / GN) + tc * 4 + (j % 4);
      if (gj >= P.n) continue;
      if (P.c_lower && gj > gi) continue;
      T* c = P.C + (int64_t)gi * P.c_rs + (int64_t)gj * P.c_cs;
      T v = alpha * acc[i][j];
      if (beta != T(0)) v = fma(beta, *c, v);
      *c = v;
    }
  }
}

}  // namespace kgemm
}  // namespace rfp
