// capi.cu — the extern "C" boundary (include/curfp.h).
//
// Argument checks, quick returns and status codes follow the reference entry
// points (cited per function); the work itself is planned by plan.cpp and
// executed by the native kernels.  No cuBLAS / cuSOLVER is linked.
#include <climits>
#include <cstdint>
#include <new>

#include "../../include/curfp.h"
#include "context.h"
#include "k_pack.cuh"

using rfp::CudaExec;
using rfp::Geometry;

namespace {

inline int ok_launch() { return cudaGetLastError() == cudaSuccess; }

inline curfpStatus_t status_of(int rc) {
  switch (rc) {
    case 0: return CURFP_STATUS_SUCCESS;
    case 2: return CURFP_STATUS_ALLOC_FAILED;
    case 3: return CURFP_STATUS_INVALID_VALUE;
    default: return CURFP_STATUS_EXECUTION_FAILED;
  }
}

inline int n1_of(int n, int lower) {
  return (n & 1) ? (lower ? n - n / 2 : n / 2) : n / 2;
}

__global__ void set_int(int* p, int v) { *p = v; }

// Flags a zero on the diagonal of the factor (the condition on which the
// reference's SPOTRI reports failure, src/curfp_spftri.cu:318,326).
__global__ void diag_zero_check(Geometry g, const float* arf, int* flag) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < g.n && arf[rfp::diag_offset(g, i)] == 0.0f) atomicMin(flag, (int)i + 1);
}

curfpStatus_t pack(curfpHandle_t h, int transr, int lower, int n,
                   const float* src, float* dst, int64_t lda, int to_rfp) {
  Geometry g = rfp::geometry(n, transr, lower);
  rfp::kpack::PackArgs a{};
  const rfp::BlockGeom* bg[3] = {&g.b11, &g.b21, &g.b22};
  const int rows[3] = {g.n1, g.n2, g.n2}, cols[3] = {g.n1, g.n1, g.n2};
  const int pb[3] = {0, g.n1, g.n1}, qb[3] = {0, 0, g.n1};
  int tiles = 0, cnt = 0;
  for (int b = 0; b < 3; ++b) {
    if (rows[b] <= 0 || cols[b] <= 0) continue;
    rfp::kpack::PackBlock& B = a.b[cnt++];
    B.off = bg[b]->off; B.rs = bg[b]->rs; B.cs = bg[b]->cs;
    B.rows = rows[b]; B.cols = cols[b];
    B.p_base = pb[b]; B.q_base = qb[b];
    B.tri = (b != 1);
    B.tiles_p = (rows[b] + rfp::kpack::TS - 1) / rfp::kpack::TS;
    B.tiles_q = (cols[b] + rfp::kpack::TS - 1) / rfp::kpack::TS;
    B.tile_begin = tiles;
    tiles += B.tri ? B.tiles_p * (B.tiles_p + 1) / 2 : B.tiles_p * B.tiles_q;
  }
  a.nblocks = cnt;
  a.total_tiles = tiles;
  a.upper = !lower;
  a.lda = lda;
  if (tiles == 0) return CURFP_STATUS_SUCCESS;
  rfp::kpack::pack_kernel<float>
      <<<tiles, dim3(rfp::kpack::TS, rfp::kpack::TY), 0, h->stream>>>(a, src, dst,
                                                                     to_rfp);
  return ok_launch() ? CURFP_STATUS_SUCCESS : CURFP_STATUS_EXECUTION_FAILED;
}

}  // namespace

extern "C" {

// src/curfp_handle.cpp:4-26
curfpStatus_t curfpCreate(curfpHandle_t* handle) {
  if (!handle) return CURFP_STATUS_INVALID_VALUE;
  curfpContext* ctx = new (std::nothrow) curfpContext();
  if (!ctx) return CURFP_STATUS_ALLOC_FAILED;
  if (cudaGetDevice(&ctx->device) != cudaSuccess ||
      cudaMalloc(&ctx->d_info, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    delete ctx;
    return CURFP_STATUS_NOT_INITIALIZED;
  }
  *handle = ctx;
  return CURFP_STATUS_SUCCESS;
}

// src/curfp_handle.cpp:28-35
curfpStatus_t curfpDestroy(curfpHandle_t handle) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  cudaStreamSynchronize(handle->stream);
  if (handle->ws) cudaFree(handle->ws);
  if (handle->stage) cudaFree(handle->stage);
  if (handle->d_info) cudaFree(handle->d_info);
  delete handle;
  return CURFP_STATUS_SUCCESS;
}

// src/curfp_handle.cpp:37-43
curfpStatus_t curfpSetStream(curfpHandle_t handle, cudaStream_t stream) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  handle->stream = stream;
  return CURFP_STATUS_SUCCESS;
}

// src/curfp_handle.cpp:45-51
curfpStatus_t curfpGetStream(curfpHandle_t handle, cudaStream_t* stream) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (!stream) return CURFP_STATUS_INVALID_VALUE;
  *stream = handle->stream;
  return CURFP_STATUS_SUCCESS;
}

// Checks and quick returns: src/curfp_ssfrk.cpp:147-161.  The leading
// dimension bound is the one the reference's cuBLAS calls enforce
// (lda >= rows of the A sub-blocks for trans=N, >= k for trans=T).
curfpStatus_t curfpSsfrk(curfpHandle_t handle, curfpOperation_t transr,
                         curfpFillMode_t uplo, curfpOperation_t trans, int n,
                         int k, const float* alpha, const float* A, int lda,
                         const float* beta, float* C) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0 || k < 0 || lda < 1) return CURFP_STATUS_INVALID_VALUE;
  if (!alpha || !beta) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  if ((*alpha == 0.0f || k == 0) && *beta == 1.0f) return CURFP_STATUS_SUCCESS;
  if (*alpha == 0.0f && *beta == 0.0f) {
    size_t nt = (size_t)n * (n + 1) / 2;
    return cudaMemsetAsync(C, 0, nt * sizeof(float), handle->stream) == cudaSuccess
               ? CURFP_STATUS_SUCCESS
               : CURFP_STATUS_EXECUTION_FAILED;
  }
  const int lower = uplo == CURFP_FILL_MODE_LOWER;
  const int n1 = n1_of(n, lower), nmax = n1 > n - n1 ? n1 : n - n1;
  if (lda < (trans == CURFP_OP_N ? nmax : (k > 1 ? k : 1)))
    return CURFP_STATUS_INVALID_VALUE;
  CudaExec ex(handle);
  return status_of(rfp::plan::ssfrk(ex, transr == CURFP_OP_T, lower,
                                    trans == CURFP_OP_T, n, k, *alpha, A, lda,
                                    *beta, C));
}

// src/curfp_ssfr2k.cpp:121-232
curfpStatus_t curfpSsfr2k(curfpHandle_t handle, curfpOperation_t transr,
                          curfpFillMode_t uplo, curfpOperation_t trans, int n,
                          int k, const float* alpha, const float* A, int lda,
                          const float* B, int ldb, const float* beta,
                          float* C) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0 || k < 0 || lda < 1 || ldb < 1) return CURFP_STATUS_INVALID_VALUE;
  if (!alpha || !beta) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  if ((*alpha == 0.0f || k == 0) && *beta == 1.0f) return CURFP_STATUS_SUCCESS;
  if (*alpha == 0.0f && *beta == 0.0f) {
    size_t nt = (size_t)n * (n + 1) / 2;
    return cudaMemsetAsync(C, 0, nt * sizeof(float), handle->stream) == cudaSuccess
               ? CURFP_STATUS_SUCCESS
               : CURFP_STATUS_EXECUTION_FAILED;
  }
  const int lower = uplo == CURFP_FILL_MODE_LOWER;
  const int n1 = n1_of(n, lower), nmax = n1 > n - n1 ? n1 : n - n1;
  const int need = trans == CURFP_OP_N ? nmax : (k > 1 ? k : 1);
  if (lda < need || ldb < need) return CURFP_STATUS_INVALID_VALUE;
  CudaExec ex(handle);
  return status_of(rfp::plan::ssfr2k(ex, transr == CURFP_OP_T, lower,
                                     trans == CURFP_OP_T, n, k, *alpha, A, lda,
                                     B, ldb, *beta, C));
}

// src/curfp_spftrf.cpp:182-292.  One stream, no host synchronisation until
// the single info read-back at the end (the reference syncs after each of its
// two SPOTRF calls).  A failed pivot makes every later kernel return early.
curfpStatus_t curfpSpftrf(curfpHandle_t handle, curfpOperation_t transr,
                          curfpFillMode_t uplo, int n, float* A, int* info) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0) return CURFP_STATUS_INVALID_VALUE;
  if (!info) return CURFP_STATUS_INVALID_VALUE;
  *info = 0;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  set_int<<<1, 1, 0, handle->stream>>>(handle->d_info, INT_MAX);
  if (!ok_launch()) return CURFP_STATUS_EXECUTION_FAILED;
  CudaExec ex(handle, handle->d_info);
  int rc = rfp::plan::spftrf(ex, transr == CURFP_OP_T,
                             uplo == CURFP_FILL_MODE_LOWER, n, A);
  if (rc) return status_of(rc);
  int h = 0;
  if (cudaMemcpyAsync(&h, handle->d_info, sizeof(int), cudaMemcpyDeviceToHost,
                      handle->stream) != cudaSuccess ||
      cudaStreamSynchronize(handle->stream) != cudaSuccess)
    return CURFP_STATUS_EXECUTION_FAILED;
  *info = (h == INT_MAX) ? 0 : h;
  return CURFP_STATUS_SUCCESS;
}

// src/curfp_spftrs.cpp:215-302
curfpStatus_t curfpSpftrs(curfpHandle_t handle, curfpOperation_t transr,
                          curfpFillMode_t uplo, int n, int nrhs, const float* A,
                          float* B, int ldb) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0 || nrhs < 0 || ldb < 1) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0 || nrhs == 0) return CURFP_STATUS_SUCCESS;
  const int lower = uplo == CURFP_FILL_MODE_LOWER;
  const int n1 = n1_of(n, lower), nmax = n1 > n - n1 ? n1 : n - n1;
  if (ldb < nmax) return CURFP_STATUS_INVALID_VALUE;
  CudaExec ex(handle);
  return status_of(rfp::plan::spftrs(ex, transr == CURFP_OP_T, lower, n, nrhs,
                                     A, B, ldb));
}

// src/curfp_spftri.cu:159-388.  A zero on the factor's diagonal is reported
// as EXECUTION_FAILED before anything is overwritten.
curfpStatus_t curfpSpftri(curfpHandle_t handle, curfpOperation_t transr,
                          curfpFillMode_t uplo, int n, float* arf) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  const int tr = transr == CURFP_OP_T, lower = uplo == CURFP_FILL_MODE_LOWER;
  Geometry g = rfp::geometry(n, tr, lower);
  set_int<<<1, 1, 0, handle->stream>>>(handle->d_info, INT_MAX);
  diag_zero_check<<<(n + 255) / 256, 256, 0, handle->stream>>>(g, arf,
                                                              handle->d_info);
  if (!ok_launch()) return CURFP_STATUS_EXECUTION_FAILED;
  int h = 0;
  if (cudaMemcpyAsync(&h, handle->d_info, sizeof(int), cudaMemcpyDeviceToHost,
                      handle->stream) != cudaSuccess ||
      cudaStreamSynchronize(handle->stream) != cudaSuccess)
    return CURFP_STATUS_EXECUTION_FAILED;
  if (h != INT_MAX) return CURFP_STATUS_EXECUTION_FAILED;
  CudaExec ex(handle);
  return status_of(rfp::plan::spftri(ex, tr, lower, n, arf));
}

// src/curfp_strttf.cu:420-462 (n == 1 handled by the same kernel).
curfpStatus_t curfpSstrttf(curfpHandle_t handle, curfpOperation_t transr,
                           curfpFillMode_t uplo, int n, const float* A, int lda,
                           float* arf) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0 || lda < n) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  return pack(handle, transr == CURFP_OP_T, uplo == CURFP_FILL_MODE_LOWER, n,
              A, arf, lda, 1);
}

// src/curfp_stfttr.cu:134-175
curfpStatus_t curfpSstfttr(curfpHandle_t handle, curfpOperation_t transr,
                           curfpFillMode_t uplo, int n, const float* arf,
                           float* A, int lda) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0 || lda < n) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  return pack(handle, transr == CURFP_OP_T, uplo == CURFP_FILL_MODE_LOWER, n,
              arf, A, lda, 0);
}

// curfp/__init__.py:194-269
curfpStatus_t curfpRfpDiagIndices(curfpHandle_t handle, curfpOperation_t transr,
                                  curfpFillMode_t uplo, int n, int64_t* idx) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  Geometry g = rfp::geometry(n, transr == CURFP_OP_T, uplo == CURFP_FILL_MODE_LOWER);
  rfp::kpack::diag_indices<<<(n + 255) / 256, 256, 0, handle->stream>>>(g, idx);
  return ok_launch() ? CURFP_STATUS_SUCCESS : CURFP_STATUS_EXECUTION_FAILED;
}

// curfp/__init__.py:272-296
curfpStatus_t curfpSaddToDiagonal(curfpHandle_t handle, curfpOperation_t transr,
                                  curfpFillMode_t uplo, int n, float value,
                                  float* arf) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  Geometry g = rfp::geometry(n, transr == CURFP_OP_T, uplo == CURFP_FILL_MODE_LOWER);
  rfp::kpack::add_diag<float><<<(n + 255) / 256, 256, 0, handle->stream>>>(g, value, arf);
  return ok_launch() ? CURFP_STATUS_SUCCESS : CURFP_STATUS_EXECUTION_FAILED;
}

curfpStatus_t curfpDaddToDiagonal(curfpHandle_t handle, curfpOperation_t transr,
                                  curfpFillMode_t uplo, int n, double value,
                                  double* arf) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  Geometry g = rfp::geometry(n, transr == CURFP_OP_T, uplo == CURFP_FILL_MODE_LOWER);
  rfp::kpack::add_diag<double><<<(n + 255) / 256, 256, 0, handle->stream>>>(g, value, arf);
  return ok_launch() ? CURFP_STATUS_SUCCESS : CURFP_STATUS_EXECUTION_FAILED;
}

}  // extern "C"
