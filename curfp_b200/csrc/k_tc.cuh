// k_tc.cuh — split-BF16 tensor-core contraction for sm_100a (tcgen05 + TMA).
//
// Operand representation.  Every row i of an FP32 operand is scaled by a
// power of two s_i >= max_k |x_ik| and written as three integer digits,
//     x_ik = s_i * 2^-7 * (d0 + d1 * 2^-8 + d2 * 2^-16),  |d_t| <= 128,
// each digit exact in BF16 (8 significant bits); the truncation is at most
// 2^-24 s_i.  The staged BF16 planes are  h = d0, m = d1, l' = 2^-8 d2 and
// m' = 2^-8 d1 (power-of-two scalings of small integers: exact).  The six
// products whose weight is >= 2^-16 go to two FP32 accumulators in tensor
// memory:
//     L0  = h*h
//     L12 = h*m + m*h + h*l' + l'*h + m*m'   (= level 1 + 2^-8 level 2)
// Digit products are integers <= 2^14, so over a chunk of 1024 of the K
// dimension L0 is an integer of magnitude <= 2^24 and its tensor-core
// accumulation is EXACT; L12 carries 2^-8 of the result's weight, so the bits
// its round-toward-zero accumulation drops weigh at most ~2^-23 of the result
// over a chunk (typically far less).  After each chunk the epilogue warps fold
// the two sums into an FP32 register accumulator with round-to-nearest,
//     acc += L0 + L12 * 2^-8,
// and at the end C := alpha * s_i s_j 2^-14 * acc + beta * C: FP32-level
// accuracy from BF16 tensor cores.  (Summing floating BF16 splits directly in
// one accumulator loses several bits: tcgen05 accumulation rounds toward zero
// at every step, which is why L0 is kept apart and exact.)
//
// Kernel shape: persistent, one CTA of 256 threads per SM walking a static
// list of 128 x 128 output tiles (triangular tasks list only the tiles of
// their triangle) in the L2-friendly orders of k_order.cuh.
//   warp 0   : TMA producer — per K-block of 32, seven boxes (A h/m/l' and
//              B h/m/l'/m', 128 x 32 BF16 each, SWIZZLE_64B) into a 4-stage
//              shared-memory ring that runs across tiles;
//   warp 1   : MMA issuer — one elected thread issues, per 16-deep K step,
//              five tcgen05.mma.cta_group::1.kind::f16 (one M=128 N=256 over
//              the adjacent B planes h|m, four M=128 N=128); tcgen05.commit
//              frees the stage and signals the end of each 1024-deep chunk;
//   warp 2   : allocates / frees the tensor memory: two accumulator buffers
//              of 256 columns (L0 | L12), chunk g using buffer g & 1, so the
//              MMAs of one chunk overlap the epilogue of the previous one;
//   warps 4-7: epilogue — per chunk, tcgen05.ld of the two sums of their TMEM
//              lane quarter into registers, then release of the buffer; per
//              tile, C is written through an arbitrary strided FP32 view (RFP
//              block, any variant) with lower/upper masking.
// Operands come from dense K-major staging buffers written by digits_kernel,
// so every TMA box is 16-byte aligned whatever the RFP variant's leading
// dimension or block offset.
//
// Every mbarrier wait is bounded (polls and ~2 s of wall time); on timeout the
// kernel records an error code in *err_flag, the roles leave their loops,
// tensor memory is freed and the CTA returns (the host then reports
// CURFP_STATUS_EXECUTION_FAILED).
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>

#include <climits>
#include <cstdint>

#include "k_order.cuh"
#include "rfp.h"

namespace rfp {
namespace ktc {

constexpr int BM = 128, BN = 128, BK = 32, STAGES = 4;
constexpr int PLANES = 4;    // staged digit planes: h, m, l' = 2^-8 d2, m' = 2^-8 d1
constexpr int PLANES_A = 3;  // planes read for the A side: h, m, l'
constexpr int CHUNK_KB = 32;                                    // 32 x 32 = 1024 deep
constexpr int A_BYTES = BM * BK * 2;                            // 8 KB
constexpr int B_BYTES = BN * BK * 2;                            // 8 KB
constexpr int STAGE_BYTES = PLANES_A * A_BYTES + PLANES * B_BYTES;  // 56 KB
constexpr int THREADS = 256;
constexpr int ACC_COLS = 2 * BN;                                // one buffer: L0 | L12
constexpr int TMEM_COLS = 512;                                  // two buffers
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
constexpr int MAX_TASKS = 4;
constexpr uint32_t WAIT_LIMIT = 1u << 24;          // polls per wait
constexpr uint64_t WAIT_NS = 2000000000ull;        // and at most ~2 s of wall time

// Instruction descriptor, kind::f16: D = F32 (bits 4-5 = 1), A = B = BF16
// (bits 7-9 = 1, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at bits
// 17-22, M >> 4 at bits 24-28.
constexpr uint32_t idesc_for(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(BM >> 4) << 24);
}
constexpr uint32_t IDESC = idesc_for(BN);        // M=128, N=128
constexpr uint32_t IDESC2 = idesc_for(2 * BN);   // M=128, N=256 (two B planes)

struct Task {
  int a_row0, b_row0, m, n;
  float* C;
  int64_t c_rs, c_cs;
  float alpha, beta;
  int c_mask;  // 0 full, 1: write i >= j only, 2: write i <= j only
  int tri;     // 1: square task whose tile list is its mask's triangle only
  int tiles_m, tiles_n, tile_begin;
};

struct Batch {
  Task t[MAX_TASKS];
  int count;
  int total_tiles;
  int kblocks;
  const float* a_scale;   // per staged row of A: s_i (power of two)
  const float* b_scale;   // per staged row of B
  const int* abort_flag;  // non-null and != INT_MAX: no-op
  int* err_flag;          // set non-zero on a wait timeout
};

__device__ __forceinline__ uint32_t su32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(su32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait; returns false on timeout or when another role aborted.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity,
                                          volatile int* abort_sh, int* err_flag,
                                          int code) {
  const uint64_t t0 = globaltimer();
  for (uint32_t it = 0; it < WAIT_LIMIT; ++it) {
    if (mbar_try(b, parity)) return true;
    if (*abort_sh) return false;
    if ((it & 1023u) == 1023u && globaltimer() - t0 > WAIT_NS) break;
  }
  *abort_sh = 1;
  if (err_flag) atomicExch(err_flag, code);
  return false;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0,
                                            int c1, int c2, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(su32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(su32(bar))
      : "memory");
}

// Shared-memory matrix descriptor, K-major, SWIZZLE_64B: rows of 64 bytes,
// 8-row swizzle atoms 512 bytes apart (SBO), version 1 (bits 46-47),
// layout type 4 (bits 61-63).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) |
         ((uint64_t)(512 >> 4) << 32) | ((uint64_t)1 << 46) | ((uint64_t)4 << 61);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t ad, uint64_t bd,
                                         uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
      "l"(ad), "l"(bd), "r"(idesc), "r"(accum));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          su32(bar))
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 16 consecutive 32-bit columns of this warp's TMEM lane quarter; the load is
// asynchronous until tmem_wait().
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}


// Tile g of the batch's tile list -> task index, m0, n0.
__device__ __forceinline__ int tile_of(const Batch& batch, int g, int& m0, int& n0) {
  int ti = 0;
  while (ti + 1 < batch.count && g >= batch.t[ti + 1].tile_begin) ++ti;
  const Task& T = batch.t[ti];
  const int lt = g - T.tile_begin;
  int r, c;
  if (T.tri) {
    order::tri_band_tile(T.tiles_m, lt, r, c);  // c <= r
    if (T.c_mask == 2) { const int x = r; r = c; c = x; }
  } else {
    order::grouped_tile(T.tiles_m, T.tiles_n, lt, r, c);
  }
  m0 = r * BM;
  n0 = c * BN;
  return ti;
}

__global__ void __launch_bounds__(THREADS, 1)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA,
                   const __grid_constant__ CUtensorMap tmB, const Batch batch) {
  if (batch.abort_flag && *batch.abort_flag != INT_MAX) return;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* acc_full = empty + STAGES;   // [2]: MMA -> epilogue, per chunk
  uint64_t* acc_empty = acc_full + 2;    // [2]: epilogue -> MMA, per chunk
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 2);
  volatile int* abort_sh = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 128);
    }
    *abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     su32(tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int KB = batch.kblocks;
  const int NCHUNK = (KB + CHUNK_KB - 1) / CHUNK_KB;
  const int G = gridDim.x;

  if (warp == 0) {
    if (lane == 0) {
      // ---------------- TMA producer ----------------
      uint32_t it = 0;  // ring position over all tiles of this CTA
      bool ok = true;
      for (int g = blockIdx.x; g < batch.total_tiles && ok; g += G) {
        int m0, n0;
        const Task& T = batch.t[tile_of(batch, g, m0, n0)];
        for (int kb = 0; kb < KB; ++kb, ++it) {
          const int s = it % STAGES;
          const uint32_t ph = (it / STAGES) & 1;
          if (it >= STAGES && !mbar_wait(&empty[s], ph ^ 1, abort_sh, batch.err_flag, 1)) {
            ok = false;
            break;
          }
          uint8_t* st = smem + s * STAGE_BYTES;
          mbar_expect_tx(&full[s], STAGE_BYTES);
          const int k0 = kb * BK;
#pragma unroll
          for (int p = 0; p < PLANES_A; ++p)
            tma_load_3d(st + p * A_BYTES, &tmA, k0, T.a_row0 + m0, p, &full[s]);
#pragma unroll
          for (int p = 0; p < PLANES; ++p)
            tma_load_3d(st + PLANES_A * A_BYTES + p * B_BYTES, &tmB, k0, T.b_row0 + n0, p,
                        &full[s]);
        }
      }
      // Drain: no copy may still be landing when the CTA exits.
      for (uint32_t j = it > (uint32_t)STAGES ? it - STAGES : 0u; j < it; ++j)
        mbar_wait(&full[j % STAGES], (j / STAGES) & 1, abort_sh, nullptr, 0);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ---------------- MMA issuer ----------------
      uint32_t it = 0, gc = 0;  // ring position, chunk counter
      bool ok = true;
      for (int g = blockIdx.x; g < batch.total_tiles && ok; g += G) {
        int kb = 0;
        for (int c = 0; c < NCHUNK && ok; ++c, ++gc) {
          const uint32_t b = gc & 1, use = gc >> 1;
          if (use > 0) {
            if (!mbar_wait(&acc_empty[b], (use - 1) & 1, abort_sh, batch.err_flag, 4)) {
              ok = false;
              break;
            }
            tc_fence_after();
          }
          const uint32_t tb = tmem + b * ACC_COLS;  // L0 at tb, L12 at tb + BN
          uint32_t started = 0;  // 0 until the chunk's first K-step is issued
          const int kb_end = (kb + CHUNK_KB < KB) ? kb + CHUNK_KB : KB;
          for (; kb < kb_end; ++kb, ++it) {
            const int s = it % STAGES;
            const uint32_t ph = (it / STAGES) & 1;
            if (!mbar_wait(&full[s], ph, abort_sh, batch.err_flag, 2)) { ok = false; break; }
            tc_fence_after();
            const uint32_t a0 = su32(smem + s * STAGE_BYTES);
            const uint32_t b0 = a0 + PLANES_A * A_BYTES;
            // Planes: A h, m, l' at a0 + {0,1,2} * A_BYTES; B h, m, l', m' at
            // b0 + {0,1,2,3} * B_BYTES.  B h|m is one 256-row operand, so the
            // first MMA writes L0 and starts L12 in one N = 256 instruction:
            //   A_h  x [B_h|B_m] -> L0, L12
            //   A_h  x  B_l'     -> L12
            //   A_m  x  B_h      -> L12
            //   A_m  x  B_m'     -> L12
            //   A_l' x  B_h      -> L12
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk) {
              const uint32_t ak = a0 + kk * 32, bk = b0 + kk * 32;
              mma_bf16(tb, sdesc(ak), sdesc(bk), IDESC2, started);
              mma_bf16(tb + BN, sdesc(ak), sdesc(bk + 2 * B_BYTES), IDESC, 1u);
              mma_bf16(tb + BN, sdesc(ak + A_BYTES), sdesc(bk), IDESC, 1u);
              mma_bf16(tb + BN, sdesc(ak + A_BYTES), sdesc(bk + 3 * B_BYTES), IDESC, 1u);
              mma_bf16(tb + BN, sdesc(ak + 2 * A_BYTES), sdesc(bk), IDESC, 1u);
              started = 1u;
            }
            mma_commit(&empty[s]);
          }
          mma_commit(&acc_full[b]);
        }
      }
    }
  } else if (warp >= 4) {
    // ---------------- epilogue ----------------
    const int q = warp - 4;
    const uint32_t lane_off = (uint32_t)(q * 32) << 16;
    uint32_t gc = 0;
    bool ok = true;
    for (int g = blockIdx.x; g < batch.total_tiles && ok; g += G) {
      int m0, n0;
      const Task& T = batch.t[tile_of(batch, g, m0, n0)];
      float acc[BN];
#pragma unroll
      for (int j = 0; j < BN; ++j) acc[j] = 0.f;
      for (int c = 0; c < NCHUNK; ++c, ++gc) {
        const uint32_t b = gc & 1, use = gc >> 1;
        const bool w = mbar_wait(&acc_full[b], use & 1, abort_sh, batch.err_flag, 3);
        ok = __all_sync(0xffffffffu, w && !*abort_sh);
        if (!ok) break;
        tc_fence_after();
        const uint32_t tq = tmem + b * ACC_COLS + lane_off;
#pragma unroll
        for (int c0 = 0; c0 < BN; c0 += 16) {
          uint32_t l0[16], l12[16];
          tmem_ld16(tq + (uint32_t)c0, l0);
          tmem_ld16(tq + (uint32_t)(BN + c0), l12);
          tmem_wait();
#pragma unroll
          for (int j = 0; j < 16; ++j)
            acc[c0 + j] += __uint_as_float(l0[j]) + __uint_as_float(l12[j]) * 0x1p-8f;
        }
        tc_fence_before();
        mbar_arrive(&acc_empty[b]);
      }
      if (!ok) break;
      // The write-back runs while the MMA warp fills the other accumulator
      // buffer, and under that load every global round trip is slow: the
      // task's fields are read once into registers (a store through C could
      // otherwise force them to be re-read), the 128 column scales come in
      // with one coalesced load (lane l holds columns l + 32 i) and are
      // broadcast by shuffle, and the write mask is a per-row column range.
      const int r = q * 32 + lane;
      const int gi = m0 + r;
      const int64_t ccs = T.c_cs;
      const float beta = T.beta;
      const int tn = T.n, tm = T.m, cmask = T.c_mask;
      float bsr[BN / 32];
#pragma unroll
      for (int i = 0; i < BN / 32; ++i) {
        const int j = lane + 32 * i;
        bsr[i] = (n0 + j < tn) ? batch.b_scale[T.b_row0 + n0 + j] : 0.f;
      }
      int jlo = 0, jhi = tn - n0 < BN ? tn - n0 : BN;  // columns n0 + [jlo, jhi)
      if (cmask == 1 && gi - n0 + 1 < jhi) jhi = gi - n0 + 1;
      if (cmask == 2 && gi - n0 > jlo) jlo = gi - n0;
      if (gi >= tm) jhi = 0;
      // alpha s_i 2^-14 s_j is alpha times a power of two: out rounds once.
      const float sa = (gi < tm ? batch.a_scale[T.a_row0 + gi] : 0.f) * 0x1p-14f * T.alpha;
      float* const crow = T.C + (int64_t)(gi < tm ? gi : 0) * T.c_rs + (int64_t)n0 * ccs;
      const bool rd = beta != 0.f;
#pragma unroll
      for (int j0 = 0; j0 < BN; j0 += 16) {
        float cv[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int jj = j0 + j;
          cv[j] = (rd && jj >= jlo && jj < jhi) ? crow[jj * ccs] : 0.f;
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int jj = j0 + j;
          const float bs = __shfl_sync(0xffffffffu, bsr[jj >> 5], jj & 31);
          float out = acc[jj] * (sa * bs);
          if (rd) out = fmaf(beta, cv[j], out);
          if (jj >= jlo && jj < jhi) crow[jj * ccs] = out;
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS));
  }
}

// Triangular operand mask of the staging kernels: element (r, c) of the
// staged operand (c counted from column koff of the full operand) is kept
// when mask == 0, when mask == 1 and c + koff <= r (lower, diagonal
// included), or when mask == 2 and c + koff >= r (upper, diagonal
// included); masked elements are staged as zeros and never read.
__device__ __forceinline__ bool keep_elem(int mask, int r, int c, int koff) {
  return mask == 0 || (mask == 1 ? c + koff <= r : c + koff >= r);
}

// Row maxima of |X| for an FP32 view X (rows x k).  Block (blockIdx.x,
// blockIdx.y) covers rows 32 blockIdx.x .. +31 and the columns
// [blockIdx.y * kseg, +kseg) (kseg a multiple of 128); every thread keeps 16
// loads in flight, the warp running along X's contiguous dimension (a warp
// takes four rows in turn when k is contiguous).  With
// one column segment (atomic == 0) the block stores the row maxima (0 for
// rows >= rows, the padding); with several, each block combines its partial
// maxima by atomicMax on the bit patterns (non-negative floats order like
// their bits) into an array zeroed beforehand.  NaN elements are skipped
// here as by fmaxf; they reach the digits and the products unchanged.
__global__ void __launch_bounds__(256, 4) rowmax_kernel(View X, int rows, int k, int kseg,
                                                     unsigned* maxbits, int mask, int koff,
                                                     int atomic) {
  __shared__ float red[8][33];
  const int r0 = blockIdx.x * 32;
  const int cb = blockIdx.y * kseg, ce = min(k, cb + kseg);
  const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;
  const bool kcont = (X.cs == 1 || X.cs == -1);
  float m = 0.f;  // the maximum of row r0 + threadIdx.x, in threads < 32
  if (kcont) {
    // warp ty: rows r0 + ty + 8 j (j < 4) in turn, lanes along k, 16
    // columns in flight
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
      const int r = r0 + ty + 8 * j;
      float mj = 0.f;
      if (r < rows) {
        const float* row = X.p + (int64_t)r * X.rs;
        for (int c = cb + tx; c < ce; c += 512) {
          float v[16];
#pragma unroll
          for (int u = 0; u < 16; ++u) {
            const int cc = c + 32 * u;
            v[u] = (cc < ce && keep_elem(mask, r, cc, koff)) ? fabsf(row[(int64_t)cc * X.cs]) : 0.f;
          }
#pragma unroll
          for (int u = 0; u < 16; ++u) mj = fmaxf(mj, v[u]);
        }
      }
      for (int o = 16; o; o >>= 1) mj = fmaxf(mj, __shfl_xor_sync(0xffffffffu, mj, o));
      if (tx == 0) red[0][ty + 8 * j] = mj;
    }
    __syncthreads();
    if (threadIdx.x < 32) m = red[0][threadIdx.x];
  } else {
    // thread (tx, ty): row r0 + tx, columns ty + 8 u (u < 16) of each 128
    const int r = r0 + tx;
    const float* row = X.p + (int64_t)(r < rows ? r : 0) * X.rs;
    float mt = 0.f;
    for (int c = cb + ty; c < ce; c += 128) {
      float v[16];
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        const int cc = c + 8 * u;
        v[u] = (r < rows && cc < ce && keep_elem(mask, r, cc, koff))
                   ? fabsf(row[(int64_t)cc * X.cs])
                   : 0.f;
      }
#pragma unroll
      for (int u = 0; u < 16; ++u) mt = fmaxf(mt, v[u]);
    }
    red[ty][tx] = mt;
    __syncthreads();
    if (threadIdx.x < 32) {
      m = red[0][threadIdx.x];
      for (int y = 1; y < 8; ++y) m = fmaxf(m, red[y][threadIdx.x]);
    }
  }
  if (threadIdx.x < 32) {
    const int r = r0 + threadIdx.x;
    const unsigned bits = __float_as_uint(m);
    if (atomic) {
      if (r < rows && bits) atomicMax(maxbits + r, bits);
    } else {
      maxbits[r] = r < rows ? bits : 0u;
    }
  }
}

// Row scale from the row maximum m: the smallest power of two 2^e with
// 2^e > m/2 and 2^e >= m (frexpf: m = f 2^e, f in [0.5, 1)); 1 for m = 0.
__device__ __forceinline__ float row_scale(unsigned maxbits) {
  const float m = __uint_as_float(maxbits);
  if (!(m > 0.f)) return 1.0f;
  int e;
  frexpf(m, &e);
  return ldexpf(1.0f, e);
}

// Digits of X (see the header), with the row scales s_i = row_scale(max_i)
// (block column 0 also stores them in scale[] for the contraction's
// epilogue): nplanes (3 or 4) BF16 planes h = d0, m = d1,
// l' = 2^-8 d2 and m' = 2^-8 d1, row-major with K contiguous, out[p][i][j],
// plane stride rows_pad * k_pad; zero padding.  A block stages a 32 x 64 tile
// through shared memory (the warp reads along X's contiguous dimension) and
// writes BF16 pairs (128 bytes per warp store).  Grid (k_pad/64, rows_pad/32),
// block (32, 8); k_pad is a multiple of 64.
__global__ void __launch_bounds__(256) digits_kernel(View X, int rows, int k,
                                                     const unsigned* __restrict__ maxbits,
                                                     float* scale, __nv_bfloat16* out,
                                                     int rows_pad, int k_pad, int nplanes,
                                                     int mask, int koff) {
  __shared__ float t[32][65];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 64;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const bool kcont = (X.cs == 1 || X.cs == -1);
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    int lr, lc;
    if (kcont) { lc = tx + 32 * (r & 1); lr = ty + 8 * (r >> 1); }
    else       { lr = tx; lc = ty + 8 * r; }
    const int gr = r0 + lr, gc = c0 + lc;
    t[lr][lc] = (gr < rows && gc < k && keep_elem(mask, gr, gc, koff))
                    ? X.p[(int64_t)gr * X.rs + (int64_t)gc * X.cs]
                    : 0.f;
  }
  __syncthreads();
  const int64_t plane = (int64_t)rows_pad * k_pad;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int lr = ty + 8 * r;
    const float sc = row_scale(maxbits[r0 + lr]);
    if (blockIdx.x == 0 && tx == 0) scale[r0 + lr] = sc;  // for the contraction's epilogue
    const float inv = 1.0f / sc;                          // power of two: exact
    float d[4][2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const float y0 = t[lr][2 * tx + h] * inv * 128.0f;  // |y0| <= 128, exact
      const float d0 = rintf(y0);
      const float y1 = (y0 - d0) * 256.0f;                // exact, |y1| <= 128
      const float d1 = rintf(y1);
      const float y2 = (y1 - d1) * 256.0f;                // exact
      d[0][h] = d0;
      d[1][h] = d1;
      d[2][h] = rintf(y2) * 0x1p-8f;                      // exact scalings
      d[3][h] = d1 * 0x1p-8f;
    }
    const int64_t o = (int64_t)(r0 + lr) * k_pad + c0 + 2 * tx;
#pragma unroll
    for (int p = 0; p < 4; ++p)  // integers <= 128 times powers of two: exact in BF16
      if (p < nplanes)
        *reinterpret_cast<__nv_bfloat162*>(out + o + p * plane) =
            __floats2bfloat162_rn(d[p][0], d[p][1]);
  }
}

}  // namespace ktc
}  // namespace rfp
