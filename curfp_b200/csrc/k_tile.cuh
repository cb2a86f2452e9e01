// k_tile.cuh — single-CTA kernels on small triangular tiles held in shared
// memory: the diagonal Cholesky tile (the only place pivots are checked), the
// inverses of diagonal blocks used by the blocked TRSM, the in-place
// inverse / L^T L tiles of the blocked spftri and the diagonal tiles of the
// Cholesky adjoint.
#pragma once
#include <climits>
#include <cstdint>
#include <type_traits>

#include "engine.h"

namespace rfp {
namespace ktile {

// Copy the lower triangle of an n x n view tile into shared memory s[i][j]
// (zeros above the diagonal).  The warp runs along the view's contiguous
// dimension and each thread keeps 8 loads in flight.  n <= 32 * RW.
template <int LDS, typename E>
__device__ __forceinline__ void load_lower(ViewT<E> L, int n, E* s) {
  const bool rcont = (L.cs == 1 || L.cs == -1);
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32, nw = blockDim.x / 32;
  for (int base = warp; base < n; base += 8 * nw) {
    E v[8][4];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int a = base + u * nw;  // row (rcont) or column (!rcont)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int b = lane + 32 * q;
        const int i = rcont ? a : b, j = rcont ? b : a;
        v[u][q] = (a < n && b < n && i >= j) ? L.p[(int64_t)i * L.rs + (int64_t)j * L.cs] : E(0);
      }
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int a = base + u * nw;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int b = lane + 32 * q;
        const int i = rcont ? a : b, j = rcont ? b : a;
        if (a < n && b < n) s[i * LDS + j] = v[u][q];
      }
    }
  }
}

// Store the lower triangle of s back to the view (same thread mapping).
template <int LDS, typename E>
__device__ __forceinline__ void store_lower(ViewT<E> L, int n, const E* s) {
  const bool rcont = (L.cs == 1 || L.cs == -1);
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32, nw = blockDim.x / 32;
  for (int a = warp; a < n; a += nw) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int b = lane + 32 * q;
      const int i = rcont ? a : b, j = rcont ? b : a;
      if (b < n && i >= j) L.p[(int64_t)i * L.rs + (int64_t)j * L.cs] = s[i * LDS + j];
    }
  }
}

constexpr int T = 64;        // trtri / lauum / TRSM-leaf tile (== kTrsmLeaf == kTriTile)
constexpr int LD = T + 1;    // padded shared-memory leading dimension

static_assert(T == kTrsmLeaf && T == kTriTile, "tile kernels assume one tile size");

// Lower-triangular Cholesky of an n x n tile (n <= NT = 128), one CTA of THR
// threads, the tile's lower triangle in shared memory.  Blocked
// by 32 columns:
//   (1) warp 0 factors the 32 x 32 diagonal block in registers (lane = row;
//       each column is broadcast through shared memory as 16-byte reads;
//       warp-uniform control flow, no block barrier inside);
//   (2) the rows below solve against it (one thread per row, forward
//       substitution with broadcast reads of the factor);
//   (3) all threads apply the rank-32 update to the trailing triangle in
//       4 x 4 register blocks.
// Shared-memory layout, panel-blocked: panel p (columns 32p .. 32p+31) holds
// rows 32p .. NT-1 with a row stride of 33, so consecutive rows of a column
// fall in consecutive banks and only the lower triangle is stored.
// On a pivot that is not > 0 (or NaN) the device info word becomes
// min(info, info_base + column + 1), the partially factored tile is written
// back and the kernel returns (LAPACK xPOTRF semantics).
constexpr int PT = 128;           // potrf tile (FP32 and FP64 executors, CPU planner tests)
constexpr int PLDP = 33;          // row stride inside a panel
template <int NT>
__host__ __device__ constexpr int panel_off(int p) {
  return PLDP * (p * NT - 16 * p * (p - 1));
}
template <int NT>
__device__ __forceinline__ int pidx(int i, int j) {
  const int p = j >> 5;
  return panel_off<NT>(p) + (i - 32 * p) * PLDP + (j & 31);
}
template <typename E, int NT>
constexpr int potrf_smem() { return (panel_off<NT>(NT / 32) + 64) * (int)sizeof(E); }
constexpr int POTRF_SMEM = potrf_smem<float, PT>();
static_assert(PT == kPotrfTile, "potrf tile size");

// 1/sqrt(d): the hardware estimate refined by one Newton-Raphson step for
// y = x^-1/2 (y <- y (3 - d y^2) / 2).
__device__ __forceinline__ float rsqrt_nr(float d) {
  const float r = rsqrtf(d);
  return r * fmaf(-0.5f * d * r, r, 1.5f);
}
__device__ __forceinline__ double rsqrt_nr(double d) {
  const double r = rsqrt(d);
  return r * fma(-0.5 * d * r, r, 1.5);
}

template <typename E, int NT, int THR>
__global__ void __launch_bounds__(THR) potrf_tile(ViewT<E> L, int n, int info_base, int* info) {
  if (info && *info != INT_MAX) return;
  extern __shared__ __align__(16) unsigned char dyn_raw[];
  E* s = reinterpret_cast<E*>(dyn_raw);
  E* rdiag = s + panel_off<NT>(NT / 32);  // 32 reciprocals of the current diagonal block
  E* col = rdiag + 32;                     // the current column of the diagonal block
  // 16-byte vectors of E (the two 32-element buffers are 16-byte aligned)
  using Vec = typename std::conditional<sizeof(E) == 4, float4, double2>::type;
  constexpr int VW = 16 / (int)sizeof(E);
  static_assert((panel_off<NT>(NT / 32) * (int)sizeof(E)) % 16 == 0, "buffer alignment");
  __shared__ int fail_sh;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  constexpr int NW = THR / 32;
  // Load the lower triangle; the warp runs along the view's contiguous
  // dimension with NT / 32 loads in flight per lane.
  {
    const bool rcont = (L.cs == 1 || L.cs == -1);
    for (int a = warp; a < n; a += NW) {
      E v[NT / 32];
#pragma unroll
      for (int q = 0; q < NT / 32; ++q) {
        const int b = lane + 32 * q;
        const int i = rcont ? a : b, j = rcont ? b : a;
        v[q] = (b < n && i >= j) ? L.p[(int64_t)i * L.rs + (int64_t)j * L.cs] : E(0);
      }
#pragma unroll
      for (int q = 0; q < NT / 32; ++q) {
        const int b = lane + 32 * q;
        const int i = rcont ? a : b, j = rcont ? b : a;
        if (b < n && i >= j) s[pidx<NT>(i, j)] = v[q];
      }
    }
  }
  if (tid == 0) fail_sh = 0;
  __syncthreads();
  for (int c0 = 0; c0 < n; c0 += 32) {
    const int w = min(32, n - c0);
    const int pb = panel_off<NT>(c0 >> 5);  // this panel's base; row r at pb + (r - c0) * 33
    // (1) diagonal block in registers
    if (warp == 0) {
      E a[32];
#pragma unroll
      for (int k = 0; k < 32; ++k) a[k] = (lane < w && k < w) ? s[pb + lane * PLDP + k] : E(0);
      int fail = 0;
      // The exit tests are warp-uniform (w is, and the pivot test goes
      // through a vote), so the loop body runs without divergence handling.
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        if (j >= w) break;
        const E d = __shfl_sync(0xffffffffu, a[j], j);
        if (__any_sync(0xffffffffu, !(d > E(0)))) {
          fail = c0 + j + 1;
          break;
        }
        // the column is scaled by multiplication, branch-free across the warp
        const E r = rsqrt_nr(d);
        a[j] = (lane == j) ? d * r : (lane > j ? a[j] * r : a[j]);
        if (lane == j) rdiag[j] = r;
        // the scaled column goes through shared memory once and comes back
        // as 16-byte broadcast reads (instead of one shuffle per row)
        col[lane] = a[j];
        __syncwarp();
        E lk[32];
#pragma unroll
        for (int k4 = (j + 1) / VW; k4 < 32 / VW; ++k4) {
          const Vec v = reinterpret_cast<const Vec*>(col)[k4];
          const E* pv = reinterpret_cast<const E*>(&v);
#pragma unroll
          for (int t = 0; t < VW; ++t) lk[VW * k4 + t] = pv[t];
        }
        __syncwarp();
#pragma unroll
        for (int k = j + 1; k < 32; ++k)
          if (lane >= k) a[k] = fma(-a[j], lk[k], a[k]);
      }
      if (lane < w) {
#pragma unroll
        for (int k = 0; k < 32; ++k)
          if (k <= lane && k < w) s[pb + lane * PLDP + k] = a[k];
      }
      if (lane == 0 && fail) fail_sh = fail;
    }
    __syncthreads();
    if (fail_sh) break;
    const int r1 = c0 + w;
    // (2) rows below: X L_blk^T = A_r
    for (int r = r1 + tid; r < n; r += THR) {
      E x[32];
      E* row = s + pb + (r - c0) * PLDP;
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        if (j < w) {
          E v = row[j];
#pragma unroll
          for (int k = 0; k < j; ++k) v = fma(-x[k], s[pb + j * PLDP + k], v);
          x[j] = v * rdiag[j];
        } else {
          x[j] = E(0);
        }
      }
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (j < w) row[j] = x[j];
    }
    __syncthreads();
    // (3) trailing update of the lower triangle rows/cols >= r1, in 4 x 4
    // register blocks (16 independent accumulators per thread); r1 is a
    // multiple of 32 here, so a block's 4 columns share one panel.
    const int m = n - r1, nb4 = (m + 3) / 4, nblk4 = nb4 * (nb4 + 1) / 2;
    for (int e = tid; e < nblk4; e += THR) {
      int bi = (int)((sqrtf(8.0f * (float)e + 1.0f) - 1.0f) * 0.5f);
      while ((bi + 1) * (bi + 2) / 2 <= e) ++bi;
      while (bi * (bi + 1) / 2 > e) --bi;
      const int bj = e - bi * (bi + 1) / 2;
      const int ri = r1 + 4 * bi, cj = r1 + 4 * bj;
      const int pc = panel_off<NT>(cj >> 5) + (cj & 31);  // + (row - 32*(cj>>5)) * 33
      const int prow0 = 32 * (cj >> 5);
      E acc[4][4];
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q)
          acc[p][q] = (ri + p < n && cj + q <= ri + p) ? s[pc + (ri + p - prow0) * PLDP + q] : E(0);
      const E* ar[4];
      const E* br[4];
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        ar[p] = s + pb + (min(ri + p, n - 1) - c0) * PLDP;
        br[p] = s + pb + (min(cj + p, n - 1) - c0) * PLDP;
      }
#pragma unroll 4
      for (int k = 0; k < w; ++k) {
        E a4[4], b4[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
          a4[p] = ar[p][k];
          b4[p] = br[p][k];
        }
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[p][q] = fma(-a4[p], b4[q], acc[p][q]);
      }
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (ri + p < n && cj + q <= ri + p) s[pc + (ri + p - prow0) * PLDP + q] = acc[p][q];
    }
    __syncthreads();
  }
  if (fail_sh && tid == 0) atomicMin(info, info_base + fail_sh);
  // Store the lower triangle back (same thread mapping as the load).
  {
    const bool rcont = (L.cs == 1 || L.cs == -1);
    for (int a = warp; a < n; a += NW) {
#pragma unroll
      for (int q = 0; q < NT / 32; ++q) {
        const int b = lane + 32 * q;
        const int i = rcont ? a : b, j = rcont ? b : a;
        if (b < n && i >= j) L.p[(int64_t)i * L.rs + (int64_t)j * L.cs] = s[pidx<NT>(i, j)];
      }
    }
  }
}

// Inverse of lower-triangular diagonal blocks.  Block b = blockIdx.x covers
// rows/cols [b*64, min(n, b*64+64)); 256 threads.  The two 32 x 32 diagonal
// quarters are inverted in registers by warps 0 and 1 (lane = row, right-
// looking: row j of the inverse is final once scaled by 1/D_jj, then is
// broadcast to the rows below), and the off-diagonal quarter follows as
// inv([D0 0; B D1]) = [inv(D0) 0; -inv(D1) (B inv(D0))  inv(D1)] by two
// 32 x 32 products over all threads.  W != nullptr: block b writes the record
// W + b*kInvStride = [W_b | M_b], both 64 x 64 column-major (ld 64, zeros
// outside the block): W_b = inv(L_bb) and, for b >= 1, M_b = W_b L_{b,b-1}
// (the block left of the diagonal block), which lets the wavefront solve
// finish a block row with one product after its predecessor is published.
// W == nullptr: the inverse replaces the lower triangle in place.
constexpr int TRTRI_THREADS = 256;
template <typename E>
constexpr int trtri_smem() { return 2 * T * LD * (int)sizeof(E); }

template <typename E>
__global__ void __launch_bounds__(TRTRI_THREADS) trtri_blocks(ViewT<E> L, int n, E* W,
                                                              const int* abort_flag) {
  if (abort_flag && *abort_flag != INT_MAX) return;
  extern __shared__ __align__(16) unsigned char trtri_raw[];
  E (*s)[LD] = reinterpret_cast<E (*)[LD]>(trtri_raw);  // L_bb, later the block left of it
  E (*x)[LD] = s + T;  // the inverse (upper-right quarter: scratch)
  const int b = blockIdx.x, r0 = b * T;
  const int sz = min(T, n - r0);
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const ViewT<E> Lb = sub(L, r0, r0);
  // both buffers start at zero: the quarter products read whole 32 x 32
  // quarters, also rows beyond a partial last block
  for (int e = tid; e < T * LD; e += TRTRI_THREADS) {
    (&x[0][0])[e] = E(0);
    (&s[0][0])[e] = E(0);
  }
  __syncthreads();
  load_lower<LD>(Lb, sz, &s[0][0]);
  __syncthreads();
  if (warp < 2) {
    const int q0 = warp * 32, w = min(32, sz - q0);
    if (w > 0) {
      E a[32], xr[32];
#pragma unroll
      for (int k = 0; k < 32; ++k) {
        a[k] = (lane < w && k <= lane) ? s[q0 + lane][q0 + k] : E(0);
        xr[k] = (k == lane && lane < w) ? E(1) : E(0);
      }
      const E rl = lane < w ? E(1) / s[q0 + lane][q0 + lane] : E(0);
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        if (j < w) {
          const E sc = lane == j ? rl : E(1);
#pragma unroll
          for (int k = 0; k <= j; ++k) {
            xr[k] *= sc;
            const E v = __shfl_sync(0xffffffffu, xr[k], j);
            if (lane > j) xr[k] = fma(-a[j], v, xr[k]);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < 32; ++k) x[q0 + lane][q0 + k] = xr[k];
    }
  }
  __syncthreads();
  if (sz > 32) {
    // T = B inv(D0) into the upper-right quarter (inv(D0) zero above its
    // diagonal, so the sums may run over all k)
    for (int e = tid; e < 1024; e += TRTRI_THREADS) {
      const int i = e >> 5, j = e & 31;
      E a0 = E(0), a1 = E(0);
#pragma unroll
      for (int k = 0; k < 32; k += 2) {
        a0 = fma(s[32 + i][k], x[k][j], a0);
        a1 = fma(s[32 + i][k + 1], x[k + 1][j], a1);
      }
      x[i][32 + j] = a0 + a1;
    }
    __syncthreads();
    // lower-left = -inv(D1) T
    for (int e = tid; e < 1024; e += TRTRI_THREADS) {
      const int i = e >> 5, j = e & 31;
      E a0 = E(0), a1 = E(0);
#pragma unroll
      for (int k = 0; k < 32; k += 2) {
        a0 = fma(x[32 + i][32 + k], x[k][32 + j], a0);
        a1 = fma(x[32 + i][33 + k], x[k + 1][32 + j], a1);
      }
      x[32 + i][j] = -(a0 + a1);
    }
    __syncthreads();
    for (int e = tid; e < 1024; e += TRTRI_THREADS) x[e >> 5][32 + (e & 31)] = E(0);
    __syncthreads();
  }
  if (!W) {
    store_lower<LD>(Lb, sz, &x[0][0]);
    return;
  }
  E* Wb = W + (int64_t)b * kInvStride;
  for (int e = tid; e < T * T; e += TRTRI_THREADS) Wb[e] = x[e & 63][e >> 6];
  if (b == 0) return;
  // M_b = W_b L_{b,b-1}: the 64 x 64 block left of the diagonal block (rows
  // beyond sz are zero), 4 x 4 outputs per thread.
  const ViewT<E> Lp = sub(L, r0, r0 - T);
  for (int e = tid; e < T * T; e += TRTRI_THREADS) {
    const int i = e >> 6, c = e & 63;
    s[i][c] = i < sz ? Lp.p[(int64_t)i * Lp.rs + (int64_t)c * Lp.cs] : E(0);
  }
  __syncthreads();
  const int ri = (tid >> 4) * 4, ci = (tid & 15) * 4;
  E acc[4][4];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[p][q] = E(0);
#pragma unroll 4
  for (int k = 0; k < T; ++k) {
    E x4[4], s4[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      x4[p] = x[ri + p][k];
      s4[p] = s[k][ci + p];
    }
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[p][q] = fma(x4[p], s4[q], acc[p][q]);
  }
  E* Mb = Wb + T * T;
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) Mb[(int64_t)(ci + q) * T + ri + p] = acc[p][q];
}

// In-place L := L^T L (lower part) for an n x n tile, n <= 64.
// (L^T L)(i,j) = sum_{k >= i} L(k,i) L(k,j) for i >= j.
template <typename E>
__global__ void __launch_bounds__(256) lauum_tile(ViewT<E> L, int n) {
  __shared__ E s[T][LD];
  const int tid = threadIdx.x;
  load_lower<LD>(L, n, &s[0][0]);
  __syncthreads();
  E out[16];
  const int j = tid % T, i0 = tid / T;
#pragma unroll
  for (int r = 0; r < 16; ++r) {
    const int i = i0 + 4 * r;
    E acc = E(0);
    if (i < n && j < n && i >= j)
      for (int k = i; k < n; ++k) acc = fma(s[k][i], s[k][j], acc);
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

// Adjoint of the Cholesky factorization of one diagonal tile (n <= T), in
// place on G's lower triangle.  Column j = n-1 .. 0 reverses the forward
// step that produced column j of L (l = L(j,j), v = L(j+1:, j)) once the
// trailing block's cotangent G(j+1:, j+1:) is final:
//   w = (tril(G_t) + tril(G_t)^T) v      (G_t's diagonal counted twice)
//   G(j+1:, j) = (G(j+1:, j) - w) / l
//   G(j, j)    = (G(j, j) - G(j+1:, j)^T v) / (2 l)
// Four threads share a row of w (strided k, shuffle sum); warp 0 forms the
// diagonal dot product.  Two block barriers per column.
constexpr int ADJ_THREADS = 256;
template <typename E>
constexpr int adj_smem() { return 2 * T * LD * (int)sizeof(E); }

template <typename E>
__global__ void __launch_bounds__(ADJ_THREADS) potrf_adj_tile(ViewT<E> L, ViewT<E> G, int n) {
  extern __shared__ __align__(16) unsigned char adj_raw[];
  E* Ls = reinterpret_cast<E*>(adj_raw);
  E* Gs = Ls + T * LD;
  load_lower<LD>(L, n, Ls);
  load_lower<LD>(G, n, Gs);
  __syncthreads();
  const int tid = threadIdx.x, r = tid >> 2, sl = tid & 3;
  for (int j = n - 1; j >= 0; --j) {
    const E l = Ls[j * LD + j];
    const int p = j + 1 + r;
    E w = E(0);
    if (p < n) {
      for (int q = j + 1 + sl; q < n; q += 4) {
        const E g = q < p ? Gs[p * LD + q] : (q > p ? Gs[q * LD + p] : E(2) * Gs[p * LD + p]);
        w += g * Ls[q * LD + j];
      }
    }
    w += __shfl_xor_sync(0xffffffffu, w, 1);
    w += __shfl_xor_sync(0xffffffffu, w, 2);
    // column j is not read above (q, p > j), so it is updated in place
    if (p < n && sl == 0) Gs[p * LD + j] = (Gs[p * LD + j] - w) / l;
    __syncthreads();
    if (tid < 32) {
      E d = E(0);
      for (int i = j + 1 + tid; i < n; i += 32) d += Gs[i * LD + j] * Ls[i * LD + j];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
      if (tid == 0) Gs[j * LD + j] = (Gs[j * LD + j] - d) / (E(2) * l);
    }
    __syncthreads();
  }
  store_lower<LD>(G, n, Gs);
}

}  // namespace ktile
}  // namespace rfp
