// exec_cuda.cu — CUDA executor: turns planner primitives into sm_100a kernel
// launches on the handle's stream.
#include <climits>
#include <cstdint>
#include <type_traits>

#include "context.h"
#include "k_gemm.cuh"
#include "gemm_route.h"
#include "k_skinny.cuh"
#include "k_tile.cuh"
#include "k_trsv.cuh"

namespace rfp {

void* grow_buffer(curfpContext* ctx, void** buf, size_t* cur, size_t bytes) {
  if (*buf && *cur >= bytes) return *buf;
  if (*buf) {
    cudaFreeAsync(*buf, ctx->stream);
    *buf = nullptr;
  }
  // grow geometrically so that a recursion of increasing sizes reallocates
  // O(log) times
  size_t want = bytes < 256 ? 256 : bytes;
  if (*cur && want < *cur + *cur / 2) want = *cur + *cur / 2;
  void* p = nullptr;
  if (cudaMallocFromPoolAsync(&p, want, ctx->pool, ctx->stream) != cudaSuccess) {
    cudaGetLastError();
    want = bytes;  // retry without the growth margin
    if (cudaMallocFromPoolAsync(&p, want, ctx->pool, ctx->stream) != cudaSuccess) {
      cudaGetLastError();
      *cur = 0;
      return nullptr;
    }
  }
  *buf = p;
  *cur = want;
  return p;
}

template <typename T>
T* CudaExecT<T>::workspace(size_t count) {
  return static_cast<T*>(grow_buffer(ctx_, &ctx_->ws, &ctx_->ws_bytes, count * sizeof(T)));
}

namespace {

template <typename T, int BM, int BN>
int launch_gemm(const GemmProbT<T>* p, int count, const int* abort_flag,
                curfpContext* ctx) {
  cudaStream_t st = ctx->stream;
  double flops = 0;
  kgemm::Batch<T> b{};
  int tiles = 0, cnt = 0;
  for (int i = 0; i < count; ++i) {
    const GemmProbT<T>& g = p[i];
    if (g.m <= 0 || g.n <= 0) continue;
    kgemm::Prob<T>& q = b.p[cnt];
    q.A = g.A.p; q.a_rs = g.A.rs; q.a_cs = g.A.cs;
    q.B = g.B.p; q.b_rs = g.B.rs; q.b_cs = g.B.cs;
    q.A2 = g.A2.p; q.a2_rs = g.A2.rs; q.a2_cs = g.A2.cs;
    q.B2 = g.B2.p; q.b2_rs = g.B2.rs; q.b2_cs = g.B2.cs;
    q.C = g.C.p; q.c_rs = g.C.rs; q.c_cs = g.C.cs;
    q.m = g.m; q.n = g.n; q.k = g.k; q.k2 = g.k2;
    q.alpha = g.alpha; q.beta = g.beta;
    q.c_lower = g.c_lower;
    q.a_tri = g.a_tri; q.b_tri = g.b_tri; q.a2_tri = g.a2_tri; q.b2_tri = g.b2_tri;
    q.tiles_m = (g.m + BM - 1) / BM;
    q.tiles_n = (g.n + BN - 1) / BN;
    if (g.inplace && q.tiles_m != 1) return 3;  // planner contract
    if (g.c_lower && (q.tiles_m != q.tiles_n || BM != BN || g.m != g.n))
      return 3;
    q.tile_begin = tiles;
    tiles += g.c_lower ? q.tiles_m * (q.tiles_m + 1) / 2 : q.tiles_m * q.tiles_n;
    flops += 2.0 * g.m * g.n * (double)(g.k + g.k2) * (g.c_lower ? 0.5 : 1.0);
    ++cnt;
  }
  if (cnt == 0) return 0;
  b.count = cnt;
  b.total_tiles = tiles;
  b.abort_flag = abort_flag;
  ProfScope ps(ctx->prof, st, K_SGEMM, flops, 0);
  ps.shape(b.p[0].m, b.p[0].n, b.p[0].k + b.p[0].k2, tiles);
  kgemm::sgemm_batch<T, BM, BN><<<tiles, kgemm::kThreads, 0, st>>>(b);
  ++ctx->launches;
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

// The few-column kernels (k_skinny.cuh) for the products gemm_route.h
// routes to them; -1 when it does not.
template <typename T>
int launch_skinny(const GemmProbT<T>& g0, const int* abort_flag, curfpContext* ctx) {
  GemmProbT<T> g;
  const SkinnyRoute r = skinny_route(g0, &g);
  if (!r.use) return -1;
  const kskinny::Args<T> a{g.A.p, g.A.rs, g.A.cs, g.B.p, g.B.rs, g.B.cs, g.C.p, g.C.rs, g.C.cs,
                           g.m, g.n, g.k, g.alpha, g.beta};
  ProfScope ps(ctx->prof, ctx->stream, K_SGEMM, 2.0 * g.m * g.n * (double)g.k,
               (double)sizeof(T) * g.m * (double)g.k);
  const int grid = (g.m + 31) / 32;
  cudaStream_t st = ctx->stream;
  auto go = [&](auto ncols) {
    constexpr int N = decltype(ncols)::value;
    if (r.rows) kskinny::skinny_rows<T, N><<<grid, kskinny::kThreads, 0, st>>>(a, abort_flag);
    else kskinny::skinny_cols<T, N><<<grid, kskinny::kThreads, 0, st>>>(a, abort_flag);
  };
  switch (r.inst) {
    case 1: go(std::integral_constant<int, 1>{}); break;
    case 2: go(std::integral_constant<int, 2>{}); break;
    case 4: go(std::integral_constant<int, 4>{}); break;
    default: go(std::integral_constant<int, 8>{}); break;
  }
  ++ctx->launches;
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

}  // namespace

// Output written through a column-contiguous view keeps the tensor-core
// epilogue's warp-wide stores coalesced: C = A B^T is computed as
// C^T = B A^T when C's contiguous dimension is its column index.
// Returns whether it swapped the operands.
static bool orient(View& A, int& arows, View& B, int& brows, SharedTask& t) {
  const bool col_contig = (t.C.cs == 1 || t.C.cs == -1) && !(t.C.rs == 1 || t.C.rs == -1);
  if (!col_contig) return false;
  View tv = A; A = B; B = tv;
  int tr_ = arows; arows = brows; brows = tr_;
  int x = t.a_row0; t.a_row0 = t.b_row0; t.b_row0 = x;
  x = t.m; t.m = t.n; t.n = x;
  t.C = tr(t.C);
  t.c_lower = t.c_lower ? 2 : 0;  // 2 = upper mask after transposition
  return true;
}

template <>
int CudaExecT<double>::gemm_shared(ViewT<double> X, int rows, int k,
                                   const SharedTaskT<double>* t, int count, int math) {
  return ExecT<double>::gemm_shared(X, rows, k, t, count, math);  // SIMT FP64 only
}

template <>
int CudaExecT<float>::gemm_shared(View X, int rows, int k, const SharedTask* t, int count,
                                  int math) {
  bool tc = math != 0 && count <= kMaxBatch;
  for (int i = 0; tc && i < count; ++i)
    tc = tc_worthwhile(t[i].m, t[i].n, k);
  if (!tc) return Exec::gemm_shared(X, rows, k, t, count, math);
  SharedTask tt[kMaxBatch];
  for (int i = 0; i < count; ++i) {
    tt[i] = t[i];
    View A = X, B{nullptr, 0, 0};
    int ar = rows, br = rows;
    orient(A, ar, B, br, tt[i]);  // shared operand: swapping keeps B == A
  }
  return tc_contract(ctx_, abort_, X, rows, View{nullptr, 0, 0}, rows, k, tt, count);
}

template <>
int CudaExecT<double>::gemm_pair(ViewT<double> X, ViewT<double> Y, int rows, int k,
                                 const SharedTaskT<double>* t, int count, int math) {
  return ExecT<double>::gemm_pair(X, Y, rows, k, t, count, math);  // SIMT FP64 only
}

// Rank-2k blocks on the tensor cores: two split-BF16 contractions over all
// blocks.  Launch 0 contracts (X, Y), launch 1 (Y, X).  A task whose C is
// column-contiguous is written transposed (orient()): C^T = Y[b] X[a]^T +
// X[b] Y[a]^T takes its two products from the launches in the other order,
// which sums to the same result.  beta applies in launch 0 only.
template <>
int CudaExecT<float>::gemm_pair(View X, View Y, int rows, int k, const SharedTask* t, int count,
                                int math) {
  bool tc = math != 0 && count <= kMaxBatch;
  for (int i = 0; tc && i < count; ++i)
    tc = tc_worthwhile(t[i].m, t[i].n, k);
  if (!tc) return Exec::gemm_pair(X, Y, rows, k, t, count, math);
  SharedTask tt[kMaxBatch];
  for (int pass = 0; pass < 2; ++pass) {
    View P = pass ? Y : X, Q = pass ? X : Y;
    for (int i = 0; i < count; ++i) {
      tt[i] = t[i];
      if (pass) tt[i].beta = 1.0f;
      View a = P, b = Q;
      int r0 = rows, r1 = rows;
      orient(a, r0, b, r1, tt[i]);  // only the task's rows and C are used here
    }
    const int rc = tc_contract(ctx_, abort_, P, rows, Q, rows, k, tt, count);
    if (rc) return rc;
  }
  return 0;
}

template <>
int CudaExecT<double>::gemm(const GemmProbT<double>* p, int count) {
  if (count <= 0) return 0;
  if (count > kMaxBatch) return 3;
  if (count == 1) {
    const int rc = launch_skinny<double>(p[0], abort_, ctx_);
    if (rc >= 0) return rc;
  }
  // 128 x 128 tiles (64 accumulators per thread, one CTA per SM) when they
  // fill the machine, else 64 x 64
  int64_t t128 = 0;
  bool inplace = false;
  for (int i = 0; i < count; ++i) {
    const int64_t tm = (p[i].m + 127) / 128, tn = (p[i].n + 127) / 128;
    t128 += p[i].c_lower ? tm * (tm + 1) / 2 : tm * tn;
    inplace = inplace || p[i].inplace;
  }
  if (t128 >= 148 && !inplace) return launch_gemm<double, 128, 128>(p, count, abort_, ctx_);
  return launch_gemm<double, 64, 64>(p, count, abort_, ctx_);
}

template <>
int CudaExecT<float>::gemm(const GemmProb* p, int count) {
  if (count <= 0) return 0;
  if (count > kMaxBatch) return 3;
  if (count == 1) {
    const int rc = launch_skinny<float>(p[0], abort_, ctx_);
    if (rc >= 0) return rc;
  }
  // One problem, one or two products, on the tensor cores: the A operands
  // may be triangular (lower / upper, staged with zeros), the B operands
  // full; the second product accumulates with beta = 1.
  // An in-place problem (C aliases B) qualifies when its operands are staged
  // whole before the product runs (one slab, one product).
  if (count == 1 && p[0].math && p[0].b_tri == 0 && p[0].b2_tri == 0 &&
      p[0].a_tri <= 2 && p[0].a2_tri <= 2 && tc_worthwhile(p[0].m, p[0].n, p[0].k) &&
      (p[0].k2 == 0 || tc_worthwhile(p[0].m, p[0].n, p[0].k2)) &&
      (!p[0].inplace ||
       (p[0].k2 == 0 && tc_single_slab(p[0].m > p[0].n ? p[0].m : p[0].n, p[0].k)))) {
    const GemmProb& g = p[0];
    for (int prod = 0; prod < (g.k2 ? 2 : 1); ++prod) {
      View A = prod ? g.A2 : g.A, Bt = tr(prod ? g.B2 : g.B);  // A: m x k, Bt: n x k
      int ar = g.m, br = g.n;
      int amask = prod ? g.a2_tri : g.a_tri, bmask = 0;
      SharedTask t{0, 0, g.m, g.n, g.C, g.alpha, prod ? 1.0f : g.beta, g.c_lower};
      if (orient(A, ar, Bt, br, t)) {  // operands swapped: the mask moves with A
        bmask = amask;
        amask = 0;
      }
      const int rc = (amask || bmask)
                         ? tc_contract_masked(ctx_, abort_, A, ar, amask, Bt, br, bmask,
                                              prod ? g.k2 : g.k, &t, 1)
                         : tc_contract(ctx_, abort_, A, ar, Bt, br, prod ? g.k2 : g.k, &t, 1);
      if (rc) return rc;
    }
    return 0;
  }
  // Tile choice: 128 x 128 when it fills the machine, else 64 x 64.
  int64_t t128 = 0;
  int maxm = 0;
  for (int i = 0; i < count; ++i) {
    int64_t tm = (p[i].m + 127) / 128, tn = (p[i].n + 127) / 128;
    t128 += p[i].c_lower ? tm * (tm + 1) / 2 : tm * tn;
    if (p[i].inplace && p[i].m > maxm) maxm = p[i].m;
  }
  if (t128 >= 2 * 148 && maxm == 0)
    return launch_gemm<float, 128, 128>(p, count, abort_, ctx_);
  return launch_gemm<float, 64, 64>(p, count, abort_, ctx_);
}

namespace {
// Opt a kernel into more than 48 KB of dynamic shared memory (once per
// instantiation).
template <typename K>
bool smem_attr(K kernel, int bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) ==
         cudaSuccess;
}
}  // namespace

template <typename T>
int CudaExecT<T>::potrf_adj_tile(ViewT<T> L, ViewT<T> G, int n) {
  if (n <= 0) return 0;
  if (n > ktile::T) return 3;
  ProfScope ps(ctx_->prof, ctx_->stream, K_POTRF, 2.0 * n * (double)n * n / 3.0, 0);
  constexpr int smem = ktile::adj_smem<T>();
  static const bool attr = smem_attr(ktile::potrf_adj_tile<T>, smem);
  if (!attr) return 4;
  ktile::potrf_adj_tile<T><<<1, ktile::ADJ_THREADS, smem, ctx_->stream>>>(L, G, n);
  ++ctx_->launches;
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

namespace {
template <typename T, int NT, int THR>
int launch_potrf(curfpContext* ctx, ViewT<T> L, int n, int info_base) {
  constexpr int smem = ktile::potrf_smem<T, NT>();
  static const bool attr = smem_attr(ktile::potrf_tile<T, NT, THR>, smem);
  if (!attr) return 4;
  ktile::potrf_tile<T, NT, THR><<<1, THR, smem, ctx->stream>>>(L, n, info_base, ctx->d_info);
  ++ctx->launches;
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}
}  // namespace

template <typename T>
int CudaExecT<T>::potrf_tile(ViewT<T> L, int n, int info_base) {
  if (n <= 0) return 0;
  if (n > potrf_tile_rows()) return 3;
  ProfScope ps(ctx_->prof, ctx_->stream, K_POTRF, (double)n * n * n / 3.0, 0);
  return launch_potrf<T, ktile::PT, 256>(ctx_, L, n, info_base);
}

template <typename T>
int CudaExecT<T>::trtri_blocks(ViewT<T> L, int n, int nb, T* W) {
  if (n <= 0) return 0;
  if (nb != ktile::T) return 3;
  int nblk = (n + nb - 1) / nb;
  ProfScope ps(ctx_->prof, ctx_->stream, K_TRTRI, (double)n * nb * nb / 3.0, 0);
  constexpr int smem = ktile::trtri_smem<T>();
  static const bool attr = smem_attr(ktile::trtri_blocks<T>, smem);
  if (!attr) return 4;
  ktile::trtri_blocks<T>
      <<<nblk, ktile::TRTRI_THREADS, smem, ctx_->stream>>>(L, n, W, abort_);
  ++ctx_->launches;
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

template <typename T>
int CudaExecT<T>::trtri_tile(ViewT<T> L, int n) {
  if (n <= 0) return 0;
  if (n > ktile::T) return 3;
  ProfScope ps(ctx_->prof, ctx_->stream, K_TRTRI, (double)n * n * n / 3.0, 0);
  constexpr int smem = ktile::trtri_smem<T>();
  static const bool attr = smem_attr(ktile::trtri_blocks<T>, smem);
  if (!attr) return 4;
  ktile::trtri_blocks<T>
      <<<1, ktile::TRTRI_THREADS, smem, ctx_->stream>>>(L, n, nullptr, abort_);
  ++ctx_->launches;
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

template <typename T>
int CudaExecT<T>::lauum_tile(ViewT<T> L, int n) {
  if (n <= 0) return 0;
  if (n > ktile::T) return 3;
  ProfScope ps(ctx_->prof, ctx_->stream, K_LAUUM, (double)n * n * n / 3.0, 0);
  ktile::lauum_tile<T><<<1, 256, 0, ctx_->stream>>>(L, n);
  ++ctx_->launches;
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

namespace {
// The wavefront solve with NC right-hand-side columns per CTA.
template <typename T, int NC>
int launch_wave(curfpContext* ctx, const int* abort_flag, ViewT<T> L, int n, ViewT<T> B, int m,
                T alpha, const T* W) {
  const int nblk = (n + ktrsv::NB - 1) / ktrsv::NB, nchunk = (m + NC - 1) / NC;
  const size_t words = 1 + (size_t)nblk * nchunk;
  int* sync = static_cast<int*>(grow_buffer(ctx, &ctx->tsv, &ctx->tsv_bytes, words * 4));
  if (!sync) return 2;
  if (cudaMemsetAsync(sync, 0, words * 4, ctx->stream) != cudaSuccess) return 4;
  // With at most two chunks the chain of block rows sets the time: the
  // shared-memory request is padded to one CTA per SM, so the chain's product
  // does not share its SM with another CTA's accumulation.
  constexpr int smem = ktrsv::smem_bytes<T, NC>();
  constexpr int smem_one = ktrsv::smem_limit<T, NC>();
  static const bool attr = smem_attr(ktrsv::trsm_wave<T, NC>, smem_one);
  if (!attr) return 4;
  const int smem_launch = nchunk <= 2 ? smem_one : smem;
  ProfScope ps(ctx->prof, ctx->stream, K_TRSV, (double)n * n * m,
               (double)n * n * sizeof(T) / 2.0);
  ps.shape(n, m, n, nblk * nchunk);
  ktrsv::trsm_wave<T, NC><<<nblk * nchunk, 256, smem_launch, ctx->stream>>>(
      L, n, B, m, alpha, W, sync, ctx->d_info + 1, abort_flag);
  ++ctx->launches;
  ++ctx->wait_launches;
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}
}  // namespace

// Up to 8 right-hand sides: 8-column chunks (the per-block products of the
// chain shrink with the chunk); otherwise 64-column chunks.
template <typename T>
int CudaExecT<T>::trsm_wave(ViewT<T> L, int n, ViewT<T> B, int m, T alpha, const T* W) {
  if (n <= 0 || m <= 0) return 0;
  if (m <= 8) return launch_wave<T, 8>(ctx_, abort_, L, n, B, m, alpha, W);
  return launch_wave<T, 64>(ctx_, abort_, L, n, B, m, alpha, W);
}

template class CudaExecT<float>;
template class CudaExecT<double>;

// Bounded-wait self-test: a wavefront solve of three 64-row block rows in
// which the CTA of block row 0 is never launched (the ticket counter starts
// at 1), so block rows 1 and 2 wait on a flag that nothing sets.  Their
// waits give up after ~2 s, set error code 5 in the handle's error word and
// return; the caller reads the word.  All buffers are zeroed first.
int wave_wait_selftest(curfpContext* ctx) {
  constexpr int n = 3 * ktrsv::NB, m = 1, nblk = 3;
  const size_t fl = (size_t)n * n + n * m + (size_t)nblk * kInvStride;
  const size_t bytes = fl * sizeof(float) + (1 + nblk) * sizeof(int);
  char* buf = static_cast<char*>(grow_buffer(ctx, &ctx->ws, &ctx->ws_bytes, bytes));
  if (!buf) return 2;
  if (cudaMemsetAsync(buf, 0, bytes, ctx->stream) != cudaSuccess) return 4;
  float* Lp = reinterpret_cast<float*>(buf);
  float* Bp = Lp + (size_t)n * n;
  float* Wp = Bp + n * m;
  int* sync = reinterpret_cast<int*>(Wp + (size_t)nblk * kInvStride);
  static const int one = 1;
  if (cudaMemcpyAsync(sync, &one, sizeof(int), cudaMemcpyHostToDevice, ctx->stream) !=
      cudaSuccess)
    return 4;
  constexpr int smem = ktrsv::smem_bytes<float, 8>();
  static const bool attr = smem_attr(ktrsv::trsm_wave<float, 8>, ktrsv::smem_limit<float, 8>());
  if (!attr) return 4;
  ktrsv::trsm_wave<float, 8><<<nblk - 1, 256, smem, ctx->stream>>>(
      View{Lp, n, 1}, n, View{Bp, 1, n}, m, 1.0f, Wp, sync, ctx->d_info + 1, nullptr);
  ++ctx->launches;
  ++ctx->wait_launches;
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

int launch_trsm_wave_fixed(curfpContext* ctx, const int* abort_flag, View L, int n, View B,
                           int m, float alpha, const float* W, int* sync, size_t sync_words) {
  if (n <= 0 || m <= 0) return 0;
  const int nblk = (n + ktrsv::NB - 1) / ktrsv::NB, nchunk = (m + ktrsv::NB - 1) / ktrsv::NB;
  const size_t words = 1 + (size_t)nblk * nchunk;
  if (words > sync_words) return 3;
  if (cudaMemsetAsync(sync, 0, words * 4, ctx->stream) != cudaSuccess) return 4;
  if (cudaFuncSetAttribute(ktrsv::trsm_wave<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           ktrsv::smem_limit<float>()) != cudaSuccess)
    return 4;
  ProfScope ps(ctx->prof, ctx->stream, K_TRSV, (double)n * n * m, (double)n * n * 2.0);
  ktrsv::trsm_wave<float><<<nblk * nchunk, 256, ktrsv::SMEM, ctx->stream>>>(
      L, n, B, m, alpha, W, sync, ctx->d_info + 1, abort_flag);
  ++ctx->launches;
  ++ctx->wait_launches;
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

}  // namespace rfp
