// k_trsv.cuh — wavefront triangular solve for few right-hand sides.
//
// Solves L X = alpha B in place (L n x n lower, non-unit, any strided view;
// B n x m view, m small) in ONE launch.  The rows are cut into 64-row blocks;
// CTA tickets are handed out in (block row, 64-column RHS chunk) order by an
// atomic counter, so a CTA only ever waits on CTAs holding smaller tickets,
// which are already running or done: the scheme needs no co-residency and
// cannot deadlock.  CTA (j, c) accumulates L_ji X_ic for i < j as soon as each
// X_ic is published (flag per block, release/acquire through L2), then forms
// X_jc = inv(L_jj) (alpha B_jc - acc) with the inverse of the diagonal block
// precomputed by trtri_blocks, stores it and publishes its own flag.  Each
// L tile is read once; the sequential chain is one tile product, one inverse
// product and one flag hand-off per block row.
//
// Waits are bounded (~2 s of wall time); on timeout a CTA records an error
// code, publishes a poisoned flag (-1) so that every dependent CTA stops
// immediately instead of waiting in turn, and returns.
#pragma once
#include <climits>
#include <cstdint>

#include "rfp.h"

namespace rfp {
namespace ktrsv {

constexpr int NB = 64;
constexpr uint64_t WAIT_NS = 2000000000ull;
constexpr int SMEM = (NB * (NB + 1) * 2 + NB * (NB + 4)) * 4;  // Ls, Ws, Xs

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// sync layout: sync[0] = ticket counter, sync[1 + b*nchunk + c] = flag of
// block row b, chunk c (0 = not ready, 1 = ready, -1 = poisoned).
// All zero at launch.
__global__ void __launch_bounds__(256) trsm_wave(View L, int n, View B, int m, float alpha,
                                                 const float* __restrict__ W, int* sync,
                                                 int* err, const int* abort_flag) {
  extern __shared__ float dyn_tsv[];
  float (*Ls)[NB + 1] = reinterpret_cast<float (*)[NB + 1]>(dyn_tsv);
  float (*Ws)[NB + 1] = reinterpret_cast<float (*)[NB + 1]>(dyn_tsv + NB * (NB + 1));
  float (*Xs)[NB + 4] = reinterpret_cast<float (*)[NB + 4]>(dyn_tsv + 2 * NB * (NB + 1));
  __shared__ int sh_ticket, sh_state;
  if (abort_flag && *abort_flag != INT_MAX) return;
  const int tid = threadIdx.x;
  const int nchunk = (m + NB - 1) / NB;
  if (tid == 0) sh_ticket = atomicAdd(sync, 1);
  __syncthreads();
  const int t = sh_ticket;
  const int j = t / nchunk, c = t % nchunk;
  const int r0 = j * NB, c0 = c * NB;
  const int rows = min(NB, n - r0), cols = min(NB, m - c0);
  const int tr = tid / 16, tc = tid % 16;  // 4 x 4 register tile
  int* flags = sync + 1;
  const bool l_rowcont = (L.cs == 1 || L.cs == -1);  // consecutive columns adjacent
  const bool x_rowcont = (B.cs == 1 || B.cs == -1) && !(B.rs == 1 || B.rs == -1);
  float acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.f;

  // Loads that do not depend on other CTAs are issued up front / one tile
  // ahead: the inverse W_j, the right-hand side block B_jc, the next L tile.
  const View Bt = sub(B, r0, c0);
  const float* Wj = W + (int64_t)j * NB * NB;
  float br[16], lr[16];
#pragma unroll
  for (int u = 0; u < 16; ++u) {
    const int e = tid + 256 * u;
    Ws[e % NB][e / NB] = __ldg(Wj + e);
  }
#pragma unroll
  for (int u = 0; u < 16; ++u) {
    const int e = tid + 256 * u;
    const int a = x_rowcont ? e / NB : e % NB, b = x_rowcont ? e % NB : e / NB;
    br[u] = (a < rows && b < cols) ? __ldcg(Bt.p + (int64_t)a * Bt.rs + (int64_t)b * Bt.cs) : 0.f;
  }
  auto load_l = [&](int i) {
    const View Lt = sub(L, r0, (int64_t)i * NB);
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int e = tid + 256 * u;
      const int a = l_rowcont ? e / NB : e % NB, b = l_rowcont ? e % NB : e / NB;
      lr[u] = (a < rows) ? __ldg(Lt.p + (int64_t)a * Lt.rs + (int64_t)b * Lt.cs) : 0.f;
    }
  };
  if (j > 0) load_l(0);

  bool poisoned = false;
  for (int i = 0; i < j; ++i) {
    if (tid == 0) {
      int st = ld_acquire(&flags[i * nchunk + c]);
      const uint64_t t0 = gtimer();
      while (st == 0) {
        st = ld_acquire(&flags[i * nchunk + c]);
        if (st == 0 && gtimer() - t0 > WAIT_NS) {
          atomicExch(err, 5);
          st = -1;
        }
      }
      sh_state = st;
    }
    __syncthreads();
    if (sh_state < 0) { poisoned = true; break; }
    const View Xt = sub(B, (int64_t)i * NB, c0);
    float xr[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int e = tid + 256 * u;
      const int a = x_rowcont ? e / NB : e % NB, b = x_rowcont ? e % NB : e / NB;
      xr[u] = (b < cols) ? __ldcg(Xt.p + (int64_t)a * Xt.rs + (int64_t)b * Xt.cs) : 0.f;
    }
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int e = tid + 256 * u;
      const int a = l_rowcont ? e / NB : e % NB, b = l_rowcont ? e % NB : e / NB;
      Ls[a][b] = lr[u];
    }
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int e = tid + 256 * u;
      const int a = x_rowcont ? e / NB : e % NB, b = x_rowcont ? e % NB : e / NB;
      Xs[a][b] = xr[u];
    }
    __syncthreads();
    if (i + 1 < j) load_l(i + 1);
#pragma unroll 8
    for (int k = 0; k < NB; ++k) {
      float a4[4], x4[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        a4[q] = Ls[tr * 4 + q][k];
        x4[q] = Xs[k][tc * 4 + q];
      }
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] = fmaf(a4[p], x4[q], acc[p][q]);
    }
    __syncthreads();
  }
  if (poisoned) {
    if (tid == 0) st_release(&flags[j * nchunk + c], -1);
    return;
  }
  // T = alpha B_jc - acc (into Xs); W_j is already in Ws (column-major source)
#pragma unroll
  for (int u = 0; u < 16; ++u) {
    const int e = tid + 256 * u;
    const int a = x_rowcont ? e / NB : e % NB, b = x_rowcont ? e % NB : e / NB;
    Xs[a][b] = alpha * br[u];
  }
  __syncthreads();
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) Xs[tr * 4 + p][tc * 4 + q] -= acc[p][q];
  __syncthreads();
  float out[4][4];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) out[p][q] = 0.f;
#pragma unroll 8
  for (int k = 0; k < NB; ++k) {
    float w4[4], x4[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      w4[q] = Ws[tr * 4 + q][k];
      x4[q] = Xs[k][tc * 4 + q];
    }
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int q = 0; q < 4; ++q) out[p][q] = fmaf(w4[p], x4[q], out[p][q]);
  }
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int a = tr * 4 + p, b = tc * 4 + q;
      if (a < rows && b < cols) Bt.p[(int64_t)a * Bt.rs + (int64_t)b * Bt.cs] = out[p][q];
    }
  __threadfence();
  __syncthreads();
  if (tid == 0) st_release(&flags[j * nchunk + c], 1);
}

}  // namespace ktrsv
}  // namespace rfp
