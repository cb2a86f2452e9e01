// k_trsv.cuh — wavefront triangular solve.
//
// Solves L X = alpha B in place (L n x n lower, non-unit, any strided view;
// B n x m view) in ONE launch.  The rows are cut into 64-row blocks and the
// right-hand sides into 64-column chunks; CTA tickets are handed out in
// (block row, chunk) order by an atomic counter, so a CTA only ever waits on
// CTAs holding smaller tickets, which are already running or done: the scheme
// needs no co-residency and cannot deadlock.
//
// CTA (j, c) accumulates acc = sum_{i < j-1} L_ji X_ic as each X_ic is
// published (flag per block, release/acquire through L2), with the L and X
// tiles double-buffered in shared memory (the next pair is in flight while
// the current one is multiplied: L by cp.async, X through registers with
// L2-only loads, requested as soon as its flag is seen).  Then, still before
// its predecessor is done, it forms Y = W_j (alpha B_jc - acc) with
// W_j = inv(L_jj).  The one product left after X_{j-1,c} is published is
// X_jc = Y - M_j X_{j-1,c} with M_j = W_j L_{j,j-1} (both from trtri_blocks),
// so the sequential chain per block row is a flag hand-off, one tile load and
// one 64^3 product.
//
// Waits are bounded (~2 s of wall time); on timeout a CTA records an error
// code, publishes a poisoned flag (-1) so that every dependent CTA stops
// immediately instead of waiting in turn, and returns.
#pragma once
#include <climits>
#include <cstdint>

#include "engine.h"
#include "rfp.h"

namespace rfp {
namespace ktrsv {

constexpr int NB = 64;
// L / W / M tiles are held k-major (element (a, b) at s[b * LDL + a]) so that
// the products read four consecutive rows of a column with one 16-byte load.
constexpr int LDL = NB + 4;
constexpr uint64_t WAIT_NS = 2000000000ull;

// Right-hand-side chunk of one CTA: NC columns, each thread a TR x TC
// register tile of the 64 x NC block; EPT elements of an X tile per thread;
// X / T tiles with row stride LDX.  NC = 64 for many right-hand sides, NC = 8
// for few (a single vector keeps the chain's per-block product small).
template <int NC> struct Chunk;
template <> struct Chunk<64> {
  static constexpr int TR = 4, TC = 4, EPT = 16, LDX = NB + 4;  // 16-byte reads along a row
};
template <> struct Chunk<8> {
  static constexpr int TR = 2, TC = 1, EPT = 2, LDX = 8;
};
constexpr int LDX = Chunk<64>::LDX;

// Ls[2], Ws (L tiles; W_j; M_j reuses Ls[0]) and Xs[2], Ts (X tiles; B_jc / T);
// 8-column chunks add the partial sums of their k-split products.
constexpr int LDP = NB + 1;  // row stride of the partial sums
template <int NC> constexpr int kparts() { return NC == 8 ? 4 * 8 * LDP : 0; }
template <typename T, int NC = 64>
constexpr int smem_bytes() {
  return (3 * NB * LDL + 3 * NB * Chunk<NC>::LDX + kparts<NC>()) * (int)sizeof(T);
}
constexpr int SMEM = smem_bytes<float>();
// The dynamic shared-memory limit set on every instantiation: its own need,
// or at least 116 KB so that a launch may ask for one CTA per SM.
template <typename T, int NC = 64>
constexpr int smem_limit() {
  return smem_bytes<T, NC>() > 116 * 1024 ? smem_bytes<T, NC>() : 116 * 1024;
}

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
// One element by cp.async (4 or 8 bytes), zero-filled when !pred.
__device__ __forceinline__ void cp1(float* smem, const float* g, bool pred) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(g),
               "r"(pred ? 4 : 0));
}
__device__ __forceinline__ void cp1(double* smem, const double* g, bool pred) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(g),
               "r"(pred ? 8 : 0));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Read-only tile (rows x cols of a strided view; L) -> element (a, b) at
// s[b * LD + a] by cp.async, zero fill outside; the thread mapping follows
// the view's contiguous dimension.  (cp.async of 4 bytes caches in L1, which is not
// coherent with other CTAs' stores: only data that no CTA of this launch
// writes goes this way.)
template <int LD, typename T>
__device__ __forceinline__ void load_tile(T* s, ViewT<T> v, int rows, int cols) {
  const bool rowcont = (v.cs == 1 || v.cs == -1) && !(v.rs == 1 || v.rs == -1);
#pragma unroll 4
  for (int u = 0; u < 16; ++u) {
    const int e = threadIdx.x + 256 * u;
    const int a = rowcont ? e / NB : e % NB, b = rowcont ? e % NB : e / NB;
    const bool ok = a < rows && b < cols;
    cp1(s + b * LD + a, ok ? v.p + (int64_t)a * v.rs + (int64_t)b * v.cs : v.p, ok);
  }
}
// Tile of B / X (64 x NC, written by CTAs of this launch): L2-only loads
// into registers (ld.global.cg), stored to shared memory by store_regs.
template <int NC, typename T>
__device__ __forceinline__ void load_regs(T (&r)[Chunk<NC>::EPT], ViewT<T> v, int rows,
                                          int cols) {
  const bool rowcont = (v.cs == 1 || v.cs == -1) && !(v.rs == 1 || v.rs == -1);
#pragma unroll
  for (int u = 0; u < Chunk<NC>::EPT; ++u) {
    const int e = threadIdx.x + 256 * u;
    const int a = rowcont ? e / NC : e % NB, b = rowcont ? e % NC : e / NB;
    r[u] = (a < rows && b < cols) ? __ldcg(v.p + (int64_t)a * v.rs + (int64_t)b * v.cs) : T(0);
  }
}
template <int NC, typename T>
__device__ __forceinline__ void store_regs(T* s, const T (&r)[Chunk<NC>::EPT], ViewT<T> v) {
  const bool rowcont = (v.cs == 1 || v.cs == -1) && !(v.rs == 1 || v.rs == -1);
#pragma unroll
  for (int u = 0; u < Chunk<NC>::EPT; ++u) {
    const int e = threadIdx.x + 256 * u;
    const int a = rowcont ? e / NC : e % NB, b = rowcont ? e % NC : e / NB;
    s[a * Chunk<NC>::LDX + b] = r[u];
  }
}
// 64 x 64 column-major workspace tile -> element (a, b) at s[b * LDL + a].
template <typename T>
__device__ __forceinline__ void load_ws(T* s, const T* w) {
#pragma unroll 4
  for (int u = 0; u < 16; ++u) {
    const int e = threadIdx.x + 256 * u;
    cp1(s + (e / NB) * LDL + e % NB, w + e, true);
  }
}
// Four consecutive shared-memory elements (16-byte reads).
__device__ __forceinline__ void lds4(const float* p, float (&v)[4]) {
  const float4 x = *reinterpret_cast<const float4*>(p);
  v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
__device__ __forceinline__ void lds4(const double* p, double (&v)[4]) {
  const double2 x = reinterpret_cast<const double2*>(p)[0];
  const double2 y = reinterpret_cast<const double2*>(p)[1];
  v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
}
// acc (+)= sign * A(64 x 64, k-major, stride LDL) * X(64 x NC, row stride LDX)
// on the thread's TR x TC register tile (rows tr*TR.., columns tc*TC..).
// 64 columns: per k one 16-byte read of A's column and one of X's row feed 16
// FMAs.  8 columns: the k range is split over four groups of 64 threads
// (thread = row), whose partial sums meet in P (4 x 8 rows of LDP) in group
// order;
// the call contains two block barriers, so every thread of the CTA makes it.
template <bool kSub, int NC, typename T>
__device__ __forceinline__ void tile_mma(T (&acc)[Chunk<NC>::TR][Chunk<NC>::TC], const T* A,
                                         const T* X, int tr, int tc, T* P) {
  constexpr int TR = Chunk<NC>::TR, TC = Chunk<NC>::TC, LX = Chunk<NC>::LDX;
  if constexpr (NC == 64) {
#pragma unroll 8
    for (int k = 0; k < NB; ++k) {
      T a[4], x[4];
      lds4(A + k * LDL + tr * 4, a);
      lds4(X + k * LX + tc * 4, x);
#pragma unroll
      for (int p = 0; p < TR; ++p)
#pragma unroll
        for (int q = 0; q < TC; ++q)
          acc[p][q] = kSub ? fma(-a[p], x[q], acc[p][q]) : fma(a[p], x[q], acc[p][q]);
    }
  } else {
    static_assert(NC == 8 && TC == 1, "8-column chunk layout");
    const int r = threadIdx.x % NB, g = threadIdx.x / NB;
    T part[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) part[q] = T(0);
#pragma unroll 4
    for (int kk = 0; kk < NB / 4; ++kk) {
      const int k = g * (NB / 4) + kk;
      const T a = A[k * LDL + r];
      T x[8];
      lds4(X + k * LX, *reinterpret_cast<T(*)[4]>(x));
      lds4(X + k * LX + 4, *reinterpret_cast<T(*)[4]>(x + 4));
#pragma unroll
      for (int q = 0; q < 8; ++q) part[q] = fma(a, x[q], part[q]);
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) P[(g * 8 + q) * LDP + r] = part[q];
    __syncthreads();
#pragma unroll
    for (int p = 0; p < TR; ++p) {
      const int row = tr * TR + p;
      const T v = ((P[tc * LDP + row] + P[(8 + tc) * LDP + row]) + P[(16 + tc) * LDP + row]) +
                  P[(24 + tc) * LDP + row];
      acc[p][0] = kSub ? acc[p][0] - v : acc[p][0] + v;
    }
    __syncthreads();
  }
}

// Bounded wait by thread 0 for a flag to become non-zero; returns the flag
// (-1 on timeout or poison).
__device__ __forceinline__ int wait_flag(const int* f, int* err) {
  int st = ld_acquire(f);
  const uint64_t t0 = gtimer();
  while (st == 0) {
    st = ld_acquire(f);
    if (st == 0 && gtimer() - t0 > WAIT_NS) {
      atomicExch(err, 5);
      st = -1;
    }
  }
  return st;
}

// sync layout: sync[0] = ticket counter, sync[1 + b*nchunk + c] = flag of
// block row b, chunk c (0 = not ready, 1 = ready, -1 = poisoned).
// All zero at launch.  W: kInvStride elements per block row ([W_j | M_j]).
// FP32: up to two CTAs per SM (104 KB of shared memory each; launches of at
// most two chunks ask for one CTA per SM); FP64: one (204 KiB).
template <typename T, int NC = 64>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1)
    trsm_wave(ViewT<T> L, int n, ViewT<T> B, int m, T alpha, const T* __restrict__ W,
              int* sync, int* err, const int* abort_flag) {
  constexpr int TR = Chunk<NC>::TR, TC = Chunk<NC>::TC, EPT = Chunk<NC>::EPT;
  constexpr int LX = Chunk<NC>::LDX;
  extern __shared__ __align__(16) unsigned char dyn_tsv_raw[];
  T* Ls0 = reinterpret_cast<T*>(dyn_tsv_raw);
  T* Ls1 = Ls0 + NB * LDL;
  T* Ws = Ls1 + NB * LDL;
  T* Xs0 = Ws + NB * LDL;
  T* Xs1 = Xs0 + NB * LX;
  T* Ts = Xs1 + NB * LX;
  T* Ps = Ts + NB * LX;  // k-split partial sums (8-column chunks)
  __shared__ int sh_ticket, sh_state, sh_ready[2], sh_last;
  if (abort_flag && *abort_flag != INT_MAX) return;
  const int tid = threadIdx.x;
  const int nchunk = (m + NC - 1) / NC;
  if (tid == 0) sh_ticket = atomicAdd(sync, 1);
  __syncthreads();
  const int t = sh_ticket;
  const int j = t / nchunk, c = t % nchunk;
  const int r0 = j * NB, c0 = c * NC;
  const int rows = min(NB, n - r0), cols = min(NC, m - c0);
  const int tr = tid / (NC / TC), tc = tid % (NC / TC);  // TR x TC register tile
  int* flags = sync + 1;
  const ViewT<T> Bt = sub(B, r0, c0);
  const T* Wj = W + (int64_t)j * kInvStride;
  auto xview = [&](int i) { return sub(B, (int64_t)i * NB, c0); };
  auto lview = [&](int i) { return sub(L, r0, (int64_t)i * NB); };

  T acc[TR][TC];
#pragma unroll
  for (int a = 0; a < TR; ++a)
#pragma unroll
    for (int b = 0; b < TC; ++b) acc[a][b] = T(0);

  // Loads that depend on no other CTA: W_j, B_jc, the first L tile.
  T xr[EPT];
  load_ws(Ws, Wj);
  load_regs<NC>(xr, Bt, rows, cols);
  store_regs<NC>(Ts, xr, Bt);
  const int iend = j - 1;  // products in the loop: i < iend
  bool poisoned = false;
  if (iend > 0) {
    load_tile<LDL>(Ls0, lview(0), rows, NB);
    if (tid == 0) sh_state = wait_flag(&flags[c], err);
    __syncthreads();
    if (sh_state < 0) {
      poisoned = true;
    } else {
      load_regs<NC>(xr, xview(0), NB, cols);
      store_regs<NC>(Xs0, xr, xview(0));
    }
  }
  cp_commit();

  for (int i = 0; i < iend && !poisoned; ++i) {
    T* Lb = (i & 1) ? Ls1 : Ls0;
    T* Xb = (i & 1) ? Xs1 : Xs0;
    T* Ln = (i & 1) ? Ls0 : Ls1;
    T* Xn = (i & 1) ? Xs0 : Xs1;
    const bool more = i + 1 < iend;
    if (tid == 0) sh_ready[i & 1] = more ? ld_acquire(&flags[(i + 1) * nchunk + c]) : 0;
    cp_wait_all();
    __syncthreads();  // tile i landed; every thread is done with the other buffers
    const bool ready = more && sh_ready[i & 1] > 0;
    if (more) load_tile<LDL>(Ln, lview(i + 1), rows, NB);
    cp_commit();
    if (ready) load_regs<NC>(xr, xview(i + 1), NB, cols);
    tile_mma<false, NC>(acc, Lb, Xb, tr, tc, Ps);
    if (more) {
      if (!ready) {
        if (tid == 0) sh_state = wait_flag(&flags[(i + 1) * nchunk + c], err);
        __syncthreads();
        if (sh_state < 0) {
          poisoned = true;
          break;
        }
        load_regs<NC>(xr, xview(i + 1), NB, cols);
      }
      store_regs<NC>(Xn, xr, xview(i + 1));
    }
  }
  if (poisoned) {
    cp_wait_all();
    __syncthreads();
    if (tid == 0) st_release(&flags[j * nchunk + c], -1);
    return;
  }

  // T = alpha B_jc - acc, then Y = W_j T (into acc).  M_j goes to Ls0 and,
  // if already published, X_{j-1} to registers while Y is formed.
  if (tid == 0) sh_last = j > 0 ? ld_acquire(&flags[(j - 1) * nchunk + c]) : 0;
  cp_wait_all();
  __syncthreads();
  const bool ready = j > 0 && sh_last > 0;
  if (j > 0) load_ws(Ls0, Wj + NB * NB);
  cp_commit();
  if (ready) load_regs<NC>(xr, xview(j - 1), NB, cols);
#pragma unroll
  for (int p = 0; p < TR; ++p)
#pragma unroll
    for (int q = 0; q < TC; ++q) {
      T* tp = Ts + (tr * TR + p) * LX + tc * TC + q;
      *tp = fma(alpha, *tp, -acc[p][q]);
      acc[p][q] = T(0);
    }
  __syncthreads();
  tile_mma<false, NC>(acc, Ws, Ts, tr, tc, Ps);
  if (j > 0) {
    if (!ready) {
      if (tid == 0) sh_state = wait_flag(&flags[(j - 1) * nchunk + c], err);
      __syncthreads();
      if (sh_state < 0) {
        cp_wait_all();
        __syncthreads();
        if (tid == 0) st_release(&flags[j * nchunk + c], -1);
        return;
      }
      load_regs<NC>(xr, xview(j - 1), NB, cols);
    }
    store_regs<NC>(Xs0, xr, xview(j - 1));
    cp_wait_all();
    __syncthreads();
    tile_mma<true, NC>(acc, Ls0, Xs0, tr, tc, Ps);  // X_j = Y - M_j X_{j-1}
  }
  // X_jc -> B through shared memory (Xs1 is free here), so that the global
  // stores run along B's contiguous dimension like the loads of load_regs.
#pragma unroll
  for (int p = 0; p < TR; ++p)
#pragma unroll
    for (int q = 0; q < TC; ++q) Xs1[(tr * TR + p) * LX + tc * TC + q] = acc[p][q];
  __syncthreads();
  {
    const bool rowcont = (Bt.cs == 1 || Bt.cs == -1) && !(Bt.rs == 1 || Bt.rs == -1);
#pragma unroll
    for (int u = 0; u < EPT; ++u) {
      const int e = tid + 256 * u;
      const int a = rowcont ? e / NC : e % NB, b = rowcont ? e % NC : e / NB;
      if (a < rows && b < cols) Bt.p[(int64_t)a * Bt.rs + (int64_t)b * Bt.cs] = Xs1[a * LX + b];
    }
  }
  // The block's stores are ordered before thread 0's release by the
  // barrier; a release store is cumulative (a release fence plus the flag
  // store), so it publishes them at GPU scope without a separate
  // sequentially consistent fence.
  __syncthreads();
  if (tid == 0) st_release(&flags[j * nchunk + c], 1);
}

}  // namespace ktrsv
}  // namespace rfp
