// tc_engine.cu — host side of the split-BF16 tensor-core contraction:
// operand staging (FP32 -> BF16 digit planes), TMA descriptors, the tile list
// and the persistent launch of ktc::tc_gemm_kernel on the handle's stream.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "context.h"
#include "k_tc.cuh"

namespace rfp {

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

inline int64_t round_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

constexpr size_t kStageBudget = (size_t)4 << 30;  // staged bytes per operand
constexpr int64_t kStageSlab = 1024;              // k granularity of a split

struct Staged {
  __nv_bfloat16* p;   // digit planes
  float* scale;       // per-row power-of-two scales
  int rows_pad;
  int k_pad;
  int planes;
};

int sm_count(const curfpContext* ctx) {
  static int sms = 0;
  if (!sms && (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device) !=
                   cudaSuccess ||
               sms <= 0))
    sms = 148;
  return sms;
}

// Stage X (rows x k) as row scales + `planes` BF16 digit planes in a context
// staging buffer: row maxima (split along k into enough blocks for about
// eight per SM; the partial maxima meet by atomicMax in a zeroed array), then
// the digits, whose first block column also stores the scales.
int stage(curfpContext* ctx, void** buf, size_t* cur, View X, int rows, int k, int planes,
          int mask, int koff, Staged* out) {
  out->rows_pad = (int)(round_up(rows, ktc::BN) + ktc::BN);
  out->k_pad = (int)round_up(k, 64);
  out->planes = planes;
  const size_t plane_bytes =
      (size_t)planes * out->rows_pad * out->k_pad * sizeof(__nv_bfloat16);
  const size_t off = (size_t)round_up((int64_t)plane_bytes, 256);
  void* p = grow_buffer(ctx, buf, cur,
                        off + (size_t)out->rows_pad * (sizeof(float) + sizeof(unsigned)));
  if (!p) return 2;
  out->p = static_cast<__nv_bfloat16*>(p);
  out->scale = reinterpret_cast<float*>(static_cast<char*>(p) + off);
  unsigned* maxbits = reinterpret_cast<unsigned*>(out->scale + out->rows_pad);
  ProfScope ps(ctx->prof, ctx->stream, K_TC_STAGE, 0,
               (double)rows * k * 8.0 + (double)out->rows_pad * out->k_pad * 2.0 * planes);
  const int groups = out->rows_pad / 32;
  const int kchunks = k > 0 ? (k + 127) / 128 : 1;
  int nsplit = (8 * sm_count(ctx) + groups - 1) / groups;
  if (nsplit > kchunks) nsplit = kchunks;
  const int kseg = 128 * ((kchunks + nsplit - 1) / nsplit);
  const int ksplit = k > 0 ? (k + kseg - 1) / kseg : 1;
  if (ksplit > 1 &&
      cudaMemsetAsync(maxbits, 0, (size_t)out->rows_pad * sizeof(unsigned), ctx->stream) !=
          cudaSuccess)
    return 4;
  ktc::rowmax_kernel<<<dim3(groups, ksplit), 256, 0, ctx->stream>>>(
      X, rows, k, kseg, maxbits, mask, koff, ksplit > 1 ? 1 : 0);
  dim3 grid(out->k_pad / 64, out->rows_pad / 32);
  ktc::digits_kernel<<<grid, dim3(32, 8), 0, ctx->stream>>>(X, rows, k, maxbits, out->scale,
                                                            out->p, out->rows_pad, out->k_pad,
                                                            planes, mask, koff);
  ctx->launches += 2;
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

int make_map(const Staged& s, int box_rows, CUtensorMap* map) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return 4;
  cuuint64_t dims[3] = {(cuuint64_t)s.k_pad, (cuuint64_t)s.rows_pad, (cuuint64_t)s.planes};
  cuuint64_t strides[2] = {(cuuint64_t)s.k_pad * 2, (cuuint64_t)s.k_pad * 2 * s.rows_pad};
  cuuint32_t box[3] = {(cuuint32_t)ktc::BK, (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, s.p, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : 4;
}

}  // namespace

bool tc_worthwhile(int m, int n, int k) {
  return m >= 128 && n >= 128 && k >= 128 && (double)m * n * k >= 2.7e8;
}

bool tc_single_slab(int rows, int k) {
  const size_t per_k = (size_t)(round_up(rows, ktc::BN) + ktc::BN) * ktc::PLANES *
                       sizeof(__nv_bfloat16);
  return (size_t)k * per_k <= kStageBudget;
}

namespace {

int tc_slab(curfpContext* ctx, const int* abort_flag, View A, int arows, int amask, View B,
            int brows, int bmask, int k, int koff, const SharedTask* tasks, int count) {
  // The A side reads planes h, m, l'; the B side also m'.  A shared operand
  // is staged once with all four.
  Staged sa, sb;
  int rc = stage(ctx, &ctx->stage, &ctx->stage_bytes, A, arows, k,
                 B.p ? ktc::PLANES_A : ktc::PLANES, amask, koff, &sa);
  if (rc) return rc;
  if (B.p) {
    if ((rc = stage(ctx, &ctx->stage2, &ctx->stage2_bytes, B, brows, k, ktc::PLANES, bmask,
                    koff, &sb)))
      return rc;
  } else {
    sb = sa;
  }
  CUtensorMap mA, mB;
  if ((rc = make_map(sa, ktc::BM, &mA)) || (rc = make_map(sb, ktc::BN, &mB))) return rc;

  ktc::Batch b{};
  int tiles = 0, cnt = 0;
  double flops = 0;
  for (int i = 0; i < count; ++i) {
    const SharedTask& s = tasks[i];
    flops += 2.0 * s.m * s.n * (double)k * (s.c_lower ? 0.5 : 1.0);
    if (s.m <= 0 || s.n <= 0) continue;
    ktc::Task& t = b.t[cnt++];
    t.a_row0 = s.a_row0; t.b_row0 = s.b_row0; t.m = s.m; t.n = s.n;
    t.C = s.C.p; t.c_rs = s.C.rs; t.c_cs = s.C.cs;
    t.alpha = s.alpha; t.beta = s.beta;
    t.c_mask = s.c_lower;  // 0 full, 1 lower, 2 upper
    t.tiles_m = (s.m + ktc::BM - 1) / ktc::BM;
    t.tiles_n = (s.n + ktc::BN - 1) / ktc::BN;
    // a masked square task lists only the tiles of its triangle
    t.tri = (t.c_mask != 0 && s.m == s.n) ? 1 : 0;
    t.tile_begin = tiles;
    tiles += t.tri ? t.tiles_m * (t.tiles_m + 1) / 2 : t.tiles_m * t.tiles_n;
  }
  if (cnt == 0) return 0;
  b.count = cnt;
  b.total_tiles = tiles;
  b.kblocks = sa.k_pad / ktc::BK;
  b.a_scale = sa.scale;
  b.b_scale = sb.scale;
  b.abort_flag = abort_flag;
  b.err_flag = ctx->d_info + 1;
  static bool attr_set = false;
  if (!attr_set) {
    if (cudaFuncSetAttribute(ktc::tc_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             ktc::SMEM_BYTES) != cudaSuccess)
      return 4;
    attr_set = true;
  }
  const int sms = sm_count(ctx);
  const int grid = tiles < sms ? tiles : sms;  // persistent: one CTA per SM
  ProfScope ps(ctx->prof, ctx->stream, K_TC_GEMM, flops, 0);
  {
    int sm = 0, sn = 0;
    for (int i = 0; i < cnt; ++i) { sm += b.t[i].m; sn += b.t[i].n; }
    ps.shape(sm, sn, k, tiles);
  }
  ktc::tc_gemm_kernel<<<grid, ktc::THREADS, ktc::SMEM_BYTES, ctx->stream>>>(mA, mB, b);
  ++ctx->launches;
  ++ctx->wait_launches;
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

}  // namespace

// Contractions whose staged digit planes would exceed kStageBudget bytes per
// operand are split along k into slabs; C accumulates across the slabs
// (beta = 1 after the first).  Bounds the staging memory of the large
// trailing updates (n = 131072: a 65536 x 65536 operand would take 34 GB of
// planes) at the cost of one extra read-modify-write of C per slab.
int tc_contract(curfpContext* ctx, const int* abort_flag, View A, int arows, View B,
                int brows, int k, const SharedTask* tasks, int count) {
  return tc_contract_masked(ctx, abort_flag, A, arows, 0, B, brows, 0, k, tasks, count);
}

int tc_contract_masked(curfpContext* ctx, const int* abort_flag, View A, int arows, int amask,
                       View B, int brows, int bmask, int k, const SharedTask* tasks,
                       int count) {
  if (count <= 0 || k <= 0) return 0;
  if (!B.p && amask) return 3;  // a shared operand is staged once, unmasked
  if (count > ktc::MAX_TASKS) return 3;
  const int rows = B.p && brows > arows ? brows : arows;
  const size_t per_k = (size_t)(round_up(rows, ktc::BN) + ktc::BN) * ktc::PLANES *
                       sizeof(__nv_bfloat16);
  int64_t kc = (int64_t)(kStageBudget / per_k) / kStageSlab * kStageSlab;
  if (kc < kStageSlab) kc = kStageSlab;
  if (kc >= k)
    return tc_slab(ctx, abort_flag, A, arows, amask, B, brows, bmask, k, 0, tasks, count);
  const int64_t nslab = (k + kc - 1) / kc;  // balanced slabs
  kc = round_up((k + nslab - 1) / nslab, kStageSlab);
  SharedTask t[ktc::MAX_TASKS];
  for (int i = 0; i < count; ++i) t[i] = tasks[i];
  for (int64_t k0 = 0; k0 < k; k0 += kc) {
    const int kk = (int)(k - k0 < kc ? k - k0 : kc);
    const View As = sub(A, 0, k0);
    const View Bs = B.p ? sub(B, 0, k0) : B;
    int rc = tc_slab(ctx, abort_flag, As, arows, amask, Bs, brows, bmask, kk, (int)k0, t, count);
    if (rc) return rc;
    for (int i = 0; i < count; ++i) t[i].beta = 1.0f;
  }
  return 0;
}

}  // namespace rfp
