// capi.cu — the extern "C" boundary (include/curfp.h).
//
// Argument checks, quick returns and status codes follow the reference entry
// points (cited per function); the work itself is planned by plan.cpp and
// executed by the native kernels.  No cuBLAS / cuSOLVER is linked.
#include <climits>
#include <cstdint>
#include <cmath>
#include <cstring>
#include <new>

#include "../../include/curfp.h"
#include "context.h"
#include "k_pack.cuh"
#include "k_refine.cuh"
#include "k_symv.cuh"
#include "status.cuh"

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

// Contraction arithmetic of a drop-in routine: the handle's math mode for
// FP32 (curfpSetMathMode), SIMT FP64 for the D twins.
template <typename T>
inline int drop_math(curfpHandle_t h) {
  return sizeof(T) == sizeof(float) ? h->math : 0;
}

inline int n1_of(int n, int lower) {
  return (n & 1) ? (lower ? n - n / 2 : n / 2) : n / 2;
}

inline int reset_info(curfpHandle_t h) { return rfp::status::reset(h); }
inline int read_info(curfpHandle_t h, int* info, int* err) {
  return rfp::status::read(h, info, err);
}

// Launch the FP64-accumulated symmetric multiply; when the row blocks alone
// do not fill the GPU the column-block sum is split over gridDim.z with an
// FP64 accumulator in workspace (atomic adds, rounded once by symm_finish).
int symm_launch(curfpHandle_t h, const Geometry& g, const float* A, const float* X,
                int64_t ldx, float* Y, int64_t ldy, int nrhs, float alpha, float beta);

inline bool symm_attr() {
  static bool done = false;
  if (!done) {
    if (cudaFuncSetAttribute(rfp::kref::symm_acc64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             rfp::kref::SYMM_SMEM) != cudaSuccess)
      return false;
    done = true;
  }
  return true;
}

// Flags a zero on the diagonal of the factor (the condition on which the
// reference's SPOTRI reports failure, src/curfp_spftri.cu:318,326).
template <typename T>
__global__ void diag_zero_check(Geometry g, const T* arf, int* flag) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < g.n && arf[rfp::diag_offset(g, i)] == T(0)) atomicMin(flag, (int)i + 1);
}

// Copy between the logical lower triangle of a dense n x n view (element
// (P,Q) at src/dst[P*drs + Q*dcs]) and an RFP array; dense -> RFP multiplies
// the diagonal by diag_scale.
template <typename T>
curfpStatus_t pack_strided(curfpHandle_t h, int transr, int lower, int n, const T* src,
                           T* dst, int64_t drs, int64_t dcs, int to_rfp,
                           float diag_scale) {
  Geometry g = rfp::geometry(n, transr, lower);
  rfp::kpack::PackArgs a{};
  const int tiles = rfp::kpack::pack_blocks(g, &a);
  a.drs = drs;
  a.dcs = dcs;
  a.diag_scale = diag_scale;
  if (tiles == 0) return CURFP_STATUS_SUCCESS;
  rfp::ProfScope ps(h->prof, h->stream, rfp::K_PACK, 0, (double)sizeof(T) * n * ((double)n + 1));
  rfp::kpack::pack_kernel<T>
      <<<tiles, dim3(rfp::kpack::TX, rfp::kpack::TY), 0, h->stream>>>(a, src, dst,
                                                                     to_rfp);
  ++h->launches;
  return ok_launch() ? CURFP_STATUS_SUCCESS : CURFP_STATUS_EXECUTION_FAILED;
}

// strttf / stfttr on a row-major n x n matrix with leading dimension lda.
template <typename T>
curfpStatus_t pack(curfpHandle_t h, int transr, int lower, int n, const T* src,
                   T* dst, int64_t lda, int to_rfp) {
  return pack_strided(h, transr, lower, n, src, dst, lower ? lda : 1, lower ? 1 : lda,
                      to_rfp, 1.0f);
}

int symm_launch(curfpHandle_t h, const Geometry& g, const float* A, const float* X,
                int64_t ldx, float* Y, int64_t ldy, int nrhs, float alpha, float beta) {
  if (!symm_attr()) return 4;
  const int n = g.n;
  const int bx = (n + rfp::kref::TB - 1) / rfp::kref::TB, by = (nrhs + rfp::kref::TB - 1) / rfp::kref::TB;
  int split = 1;
  while ((int64_t)bx * by * split < 4 * 148 && split < 16 && bx / (split * 2) >= 4) split *= 2;
  double* R = nullptr;
  if (split > 1) {
    R = static_cast<double*>(rfp::grow_buffer(h, &h->ws3, &h->ws3_bytes,
                                              (size_t)n * nrhs * sizeof(double)));
    if (!R) return 2;
    if (cudaMemsetAsync(R, 0, (size_t)n * nrhs * sizeof(double), h->stream) != cudaSuccess)
      return 4;
  }
  {
    rfp::ProfScope ps(h->prof, h->stream, rfp::K_SYMM64, 2.0 * n * (double)n * nrhs,
                      4.0 * n * (double)n);
    rfp::kref::symm_acc64<<<dim3(bx, by, split), 256, rfp::kref::SYMM_SMEM, h->stream>>>(
        g, A, X, ldx, Y, ldy, nrhs, alpha, beta, R);
    ++h->launches;
    if (R) {
      rfp::kref::symm_finish<<<148 * 4, 256, 0, h->stream>>>(R, n, nrhs, Y, ldy, alpha, beta);
      ++h->launches;
    }
  }
  return ok_launch() ? 0 : 4;
}

}  // namespace

// Entry points: C linkage from their declarations in include/curfp.h (the
// shared implementations below are C++ templates over the element type).

// src/curfp_handle.cpp:4-26
curfpStatus_t curfpCreate(curfpHandle_t* handle) {
  if (!handle) return CURFP_STATUS_INVALID_VALUE;
  curfpContext* ctx = new (std::nothrow) curfpContext();
  if (!ctx) return CURFP_STATUS_ALLOC_FAILED;
  if (cudaGetDevice(&ctx->device) != cudaSuccess ||
      cudaMalloc(&ctx->d_info, 2 * sizeof(int)) != cudaSuccess ||
      cudaMemset(ctx->d_info, 0, 2 * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    if (ctx->d_info) cudaFree(ctx->d_info);
    delete ctx;
    return CURFP_STATUS_NOT_INITIALIZED;
  }
  // Workspaces come from a pool of the handle's own, which keeps memory
  // released by a growing workspace (re-mapping on every growth is slow);
  // the device's default pool is not touched.
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = ctx->device;
  if (cudaMemPoolCreate(&ctx->pool, &props) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(ctx->d_info);
    delete ctx;
    return CURFP_STATUS_NOT_INITIALIZED;
  }
  uint64_t keep = UINT64_MAX;
  cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  cudaGetLastError();
  *handle = ctx;
  return CURFP_STATUS_SUCCESS;
}

// src/curfp_handle.cpp:28-35
curfpStatus_t curfpDestroy(curfpHandle_t handle) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  cudaStreamSynchronize(handle->stream);
  if (handle->ws) cudaFree(handle->ws);
  if (handle->stage) cudaFree(handle->stage);
  if (handle->stage2) cudaFree(handle->stage2);
  if (handle->ws2) cudaFree(handle->ws2);
  if (handle->ws3) cudaFree(handle->ws3);
  if (handle->tsv) cudaFree(handle->tsv);
  if (handle->wsg) cudaFree(handle->wsg);
  if (handle->d_info) cudaFree(handle->d_info);
  if (handle->copy_stream) {
    cudaStreamSynchronize(handle->copy_stream);
    cudaStreamDestroy(handle->copy_stream);
  }
  if (handle->ev_start) cudaEventDestroy(handle->ev_start);
  if (handle->ev_rest) cudaEventDestroy(handle->ev_rest);
  if (handle->pool) cudaMemPoolDestroy(handle->pool);
  cudaGetLastError();
  delete handle;
  return CURFP_STATUS_SUCCESS;
}

// Not in the reference (its workspace is allocated and freed per call,
// src/curfp_spftrf.cpp:231-232); here workspaces are handle-owned and grow.
curfpStatus_t curfpReleaseWorkspace(curfpHandle_t handle) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (cudaStreamSynchronize(handle->stream) != cudaSuccess) {
    cudaGetLastError();
    return CURFP_STATUS_EXECUTION_FAILED;
  }
  void** bufs[] = {&handle->ws, &handle->stage, &handle->stage2, &handle->ws2,
                   &handle->ws3, &handle->tsv, &handle->wsg};
  size_t* sizes[] = {&handle->ws_bytes, &handle->stage_bytes, &handle->stage2_bytes,
                     &handle->ws2_bytes, &handle->ws3_bytes, &handle->tsv_bytes,
                     &handle->wsg_bytes};
  bool ok = true;
  for (int i = 0; i < 7; ++i) {
    if (*bufs[i]) ok &= cudaFree(*bufs[i]) == cudaSuccess;
    *bufs[i] = nullptr;
    *sizes[i] = 0;
  }
  ok &= cudaMemPoolTrimTo(handle->pool, 0) == cudaSuccess;
  cudaGetLastError();
  return ok ? CURFP_STATUS_SUCCESS : CURFP_STATUS_EXECUTION_FAILED;
}

curfpStatus_t curfpDiagWaitTimeout(curfpHandle_t handle, int* err_code) {
  if (!handle || !err_code) return CURFP_STATUS_INVALID_VALUE;
  if (!reset_info(handle)) return CURFP_STATUS_EXECUTION_FAILED;
  // The error word is read and cleared by the same check that every routine
  // with bounded waits runs before it returns (status.cuh), so the code
  // reported here is the one a real solve would surface, and later calls on
  // this handle do not inherit it.
  rfp::status::WaitCheck wc(handle);
  const int rc = wc.finish(rfp::wave_wait_selftest(handle));
  *err_code = wc.err;
  return status_of(rc);
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
template <typename T>
static curfpStatus_t ssfrk_impl(curfpHandle_t handle, curfpOperation_t transr,
                                curfpFillMode_t uplo, curfpOperation_t trans, int n,
                                int k, const T* alpha, const T* A, int lda,
                                const T* beta, T* C, int math) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0 || k < 0 || lda < 1) return CURFP_STATUS_INVALID_VALUE;
  if (!alpha || !beta) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  if ((*alpha == T(0) || k == 0) && *beta == T(1)) return CURFP_STATUS_SUCCESS;
  if (*alpha == T(0) && *beta == T(0)) {
    size_t nt = (size_t)n * (n + 1) / 2;
    return cudaMemsetAsync(C, 0, nt * sizeof(T), handle->stream) == cudaSuccess
               ? CURFP_STATUS_SUCCESS
               : CURFP_STATUS_EXECUTION_FAILED;
  }
  const int lower = uplo == CURFP_FILL_MODE_LOWER;
  const int n1 = n1_of(n, lower), nmax = n1 > n - n1 ? n1 : n - n1;
  if (lda < (trans == CURFP_OP_N ? nmax : (k > 1 ? k : 1)))
    return CURFP_STATUS_INVALID_VALUE;
  rfp::CudaExecT<T> ex(handle);
  rfp::status::WaitCheck wc(handle);
  return status_of(wc.finish(rfp::plan::ssfrk(ex, transr == CURFP_OP_T, lower,
                                              trans == CURFP_OP_T, n, k, *alpha, A, lda,
                                              *beta, C, math)));
}

curfpStatus_t curfpSsfrk(curfpHandle_t handle, curfpOperation_t transr,
                         curfpFillMode_t uplo, curfpOperation_t trans, int n,
                         int k, const float* alpha, const float* A, int lda,
                         const float* beta, float* C) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  return ssfrk_impl(handle, transr, uplo, trans, n, k, alpha, A, lda, beta, C,
                    drop_math<float>(handle));
}

curfpStatus_t curfpSsfrkEx(curfpHandle_t handle, curfpOperation_t transr,
                           curfpFillMode_t uplo, curfpOperation_t trans, int n, int k,
                           const float* alpha, const float* A, int lda, const float* beta,
                           float* C, curfpMath_t math) {
  if (math != CURFP_MATH_FP32 && math != CURFP_MATH_SPLIT_BF16)
    return CURFP_STATUS_INVALID_VALUE;
  return ssfrk_impl(handle, transr, uplo, trans, n, k, alpha, A, lda, beta, C, (int)math);
}

// src/curfp_ssfr2k.cpp:121-232
template <typename T>
static curfpStatus_t sfr2k_impl(curfpHandle_t handle, curfpOperation_t transr,
                                curfpFillMode_t uplo, curfpOperation_t trans, int n, int k,
                                const T* alpha, const T* A, int lda, const T* B, int ldb,
                                const T* beta, T* C) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0 || k < 0 || lda < 1 || ldb < 1) return CURFP_STATUS_INVALID_VALUE;
  if (!alpha || !beta) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  if ((*alpha == T(0) || k == 0) && *beta == T(1)) return CURFP_STATUS_SUCCESS;
  if (*alpha == T(0) && *beta == T(0)) {
    size_t nt = (size_t)n * (n + 1) / 2;
    return cudaMemsetAsync(C, 0, nt * sizeof(T), handle->stream) == cudaSuccess
               ? CURFP_STATUS_SUCCESS
               : CURFP_STATUS_EXECUTION_FAILED;
  }
  const int lower = uplo == CURFP_FILL_MODE_LOWER;
  const int n1 = n1_of(n, lower), nmax = n1 > n - n1 ? n1 : n - n1;
  const int need = trans == CURFP_OP_N ? nmax : (k > 1 ? k : 1);
  if (lda < need || ldb < need) return CURFP_STATUS_INVALID_VALUE;
  rfp::CudaExecT<T> ex(handle);
  rfp::status::WaitCheck wc(handle);
  return status_of(wc.finish(rfp::plan::ssfr2k(ex, transr == CURFP_OP_T, lower,
                                               trans == CURFP_OP_T, n, k, *alpha, A, lda,
                                               B, ldb, *beta, C, drop_math<T>(handle))));
}

curfpStatus_t curfpSsfr2k(curfpHandle_t handle, curfpOperation_t transr,
                          curfpFillMode_t uplo, curfpOperation_t trans, int n,
                          int k, const float* alpha, const float* A, int lda,
                          const float* B, int ldb, const float* beta,
                          float* C) {
  return sfr2k_impl(handle, transr, uplo, trans, n, k, alpha, A, lda, B, ldb, beta, C);
}

// src/curfp_spftrf.cpp:182-292.  One stream, no host synchronisation until
// the single info read-back at the end (the reference syncs after each of its
// two SPOTRF calls).  A failed pivot makes every later kernel return early.
template <typename T>
static curfpStatus_t spftrf_impl(curfpHandle_t handle, curfpOperation_t transr,
                                 curfpFillMode_t uplo, int n, T* A, int* info,
                                 int math) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0) return CURFP_STATUS_INVALID_VALUE;
  if (!info) return CURFP_STATUS_INVALID_VALUE;
  *info = 0;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  if (!reset_info(handle)) return CURFP_STATUS_EXECUTION_FAILED;
  rfp::CudaExecT<T> ex(handle, handle->d_info);
  int rc = rfp::plan::spftrf(ex, transr == CURFP_OP_T,
                             uplo == CURFP_FILL_MODE_LOWER, n, A, math);
  if (rc) return status_of(rc);
  int h = 0, err = 0;
  if (!read_info(handle, &h, &err)) return CURFP_STATUS_EXECUTION_FAILED;
  if (err) return CURFP_STATUS_EXECUTION_FAILED;
  *info = (h == INT_MAX) ? 0 : h;
  return CURFP_STATUS_SUCCESS;
}

curfpStatus_t curfpSpftrf(curfpHandle_t handle, curfpOperation_t transr,
                          curfpFillMode_t uplo, int n, float* A, int* info) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  return spftrf_impl(handle, transr, uplo, n, A, info, drop_math<float>(handle));
}

curfpStatus_t curfpSpftrfEx(curfpHandle_t handle, curfpOperation_t transr,
                            curfpFillMode_t uplo, int n, float* A, int* info,
                            curfpMath_t math) {
  if (math != CURFP_MATH_FP32 && math != CURFP_MATH_SPLIT_BF16)
    return CURFP_STATUS_INVALID_VALUE;
  return spftrf_impl(handle, transr, uplo, n, A, info, (int)math);
}

// Not in the reference: the factorization of an RFP matrix held in host
// memory.  The span of the array that the first diagonal block touches is
// copied first, on the handle's stream; the rest is copied on an internal
// stream (after everything already enqueued on the handle's stream) and the
// factorization waits for it only after the first diagonal block, so that
// for layouts where that block occupies its own part of the array (TRANSR =
// T) the rest of the transfer overlaps its factorization.  With arf_orig the
// host array is copied there and, region by region, on to arf (one
// host-to-device transfer for both).
curfpStatus_t curfpSpftrfFromHost(curfpHandle_t handle, curfpOperation_t transr,
                                  curfpFillMode_t uplo, int n, const float* arf_host,
                                  float* arf, float* arf_orig, int* info, curfpMath_t math) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0 || !info || (n > 0 && (!arf_host || !arf)) || (arf_orig && arf_orig == arf))
    return CURFP_STATUS_INVALID_VALUE;
  if (math != CURFP_MATH_FP32 && math != CURFP_MATH_SPLIT_BF16)
    return CURFP_STATUS_INVALID_VALUE;
  *info = 0;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  if (!handle->copy_stream &&
      cudaStreamCreateWithFlags(&handle->copy_stream, cudaStreamNonBlocking) != cudaSuccess)
    return CURFP_STATUS_EXECUTION_FAILED;
  if (!handle->ev_start &&
      cudaEventCreateWithFlags(&handle->ev_start, cudaEventDisableTiming) != cudaSuccess)
    return CURFP_STATUS_EXECUTION_FAILED;
  if (!handle->ev_rest &&
      cudaEventCreateWithFlags(&handle->ev_rest, cudaEventDisableTiming) != cudaSuccess)
    return CURFP_STATUS_EXECUTION_FAILED;
  const Geometry g = rfp::geometry(n, transr == CURFP_OP_T, uplo == CURFP_FILL_MODE_LOWER);
  const int64_t total = (int64_t)n * (n + 1) / 2;
  // Offsets the first diagonal block touches: [lo, hi) (its strides are
  // positive in every variant, so (0, 0) and (n1 - 1, n1 - 1) bound it).
  int64_t lo = 0, hi = total;
  if (g.n1 > 0) {
    lo = g.b11.off;
    hi = g.b11.off + (int64_t)(g.n1 - 1) * (g.b11.rs + g.b11.cs) + 1;
  }
  float* first = arf_orig ? arf_orig : arf;
  auto copy = [&](int64_t a, int64_t b, cudaStream_t st) {
    if (b <= a) return true;
    const size_t bytes = (size_t)(b - a) * sizeof(float);
    if (cudaMemcpyAsync(first + a, arf_host + a, bytes, cudaMemcpyHostToDevice, st) !=
        cudaSuccess)
      return false;
    return !arf_orig ||
           cudaMemcpyAsync(arf + a, arf_orig + a, bytes, cudaMemcpyDeviceToDevice, st) ==
               cudaSuccess;
  };
  cudaStream_t cs = handle->copy_stream;
  if (cudaEventRecord(handle->ev_start, handle->stream) != cudaSuccess ||
      cudaStreamWaitEvent(cs, handle->ev_start, 0) != cudaSuccess || !copy(lo, hi, handle->stream) ||
      !copy(0, lo, cs) || !copy(hi, total, cs) ||
      cudaEventRecord(handle->ev_rest, cs) != cudaSuccess) {
    cudaGetLastError();
    return CURFP_STATUS_EXECUTION_FAILED;
  }
  if (!reset_info(handle)) return CURFP_STATUS_EXECUTION_FAILED;
  rfp::CudaExecT<float> ex(handle, handle->d_info);
  ex.rest_ready = handle->ev_rest;
  const int rc = rfp::plan::spftrf(ex, transr == CURFP_OP_T,
                                   uplo == CURFP_FILL_MODE_LOWER, n, arf, (int)math);
  // Whatever the plan enqueued, nothing later on the handle's stream may run
  // ahead of the copy.
  if (cudaStreamWaitEvent(handle->stream, handle->ev_rest, 0) != cudaSuccess) {
    cudaGetLastError();
    return CURFP_STATUS_EXECUTION_FAILED;
  }
  if (rc) return status_of(rc);
  int h = 0, err = 0;
  if (!read_info(handle, &h, &err)) return CURFP_STATUS_EXECUTION_FAILED;
  if (err) return CURFP_STATUS_EXECUTION_FAILED;
  *info = (h == INT_MAX) ? 0 : h;
  return CURFP_STATUS_SUCCESS;
}

// src/curfp_spftrs.cpp:215-302
template <typename T>
static curfpStatus_t pftrs_impl(curfpHandle_t handle, curfpOperation_t transr,
                                curfpFillMode_t uplo, int n, int nrhs, const T* A, T* B,
                                int ldb) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0 || nrhs < 0 || ldb < 1) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0 || nrhs == 0) return CURFP_STATUS_SUCCESS;
  const int lower = uplo == CURFP_FILL_MODE_LOWER;
  const int n1 = n1_of(n, lower), nmax = n1 > n - n1 ? n1 : n - n1;
  if (ldb < nmax) return CURFP_STATUS_INVALID_VALUE;
  rfp::CudaExecT<T> ex(handle);
  rfp::status::WaitCheck wc(handle);
  return status_of(wc.finish(rfp::plan::spftrs(ex, transr == CURFP_OP_T, lower, n, nrhs,
                                               A, B, ldb, drop_math<T>(handle))));
}

curfpStatus_t curfpSpftrs(curfpHandle_t handle, curfpOperation_t transr,
                          curfpFillMode_t uplo, int n, int nrhs, const float* A,
                          float* B, int ldb) {
  return pftrs_impl(handle, transr, uplo, n, nrhs, A, B, ldb);
}

// src/curfp_spftri.cu:159-388.  A zero on the factor's diagonal is reported
// as EXECUTION_FAILED before anything is overwritten.
template <typename T>
static curfpStatus_t pftri_impl(curfpHandle_t handle, curfpOperation_t transr,
                                curfpFillMode_t uplo, int n, T* arf) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  const int tr = transr == CURFP_OP_T, lower = uplo == CURFP_FILL_MODE_LOWER;
  Geometry g = rfp::geometry(n, tr, lower);
  if (!reset_info(handle)) return CURFP_STATUS_EXECUTION_FAILED;
  diag_zero_check<T><<<(n + 255) / 256, 256, 0, handle->stream>>>(g, arf, handle->d_info);
  ++handle->launches;
  if (!ok_launch()) return CURFP_STATUS_EXECUTION_FAILED;
  int h = 0, err = 0;
  if (!read_info(handle, &h, &err)) return CURFP_STATUS_EXECUTION_FAILED;
  if (h != INT_MAX) return CURFP_STATUS_EXECUTION_FAILED;
  rfp::CudaExecT<T> ex(handle);
  rfp::status::WaitCheck wc(handle);
  return status_of(wc.finish(rfp::plan::spftri(ex, tr, lower, n, arf, drop_math<T>(handle))));
}

curfpStatus_t curfpSpftri(curfpHandle_t handle, curfpOperation_t transr,
                          curfpFillMode_t uplo, int n, float* arf) {
  return pftri_impl(handle, transr, uplo, n, arf);
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
  ++handle->launches;
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
  ++handle->launches;
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
  ++handle->launches;
  return ok_launch() ? CURFP_STATUS_SUCCESS : CURFP_STATUS_EXECUTION_FAILED;
}

// Y := alpha*A*X + beta*Y, A symmetric in RFP, products summed in FP64.
curfpStatus_t curfpSsfmmAcc64(curfpHandle_t handle, curfpOperation_t transr,
                              curfpFillMode_t uplo, int n, int nrhs, const float* alpha,
                              const float* A, const float* X, int ldx, const float* beta,
                              float* Y, int ldy) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0 || nrhs < 0 || !alpha || !beta) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0 || nrhs == 0) return CURFP_STATUS_SUCCESS;
  if (ldx < n || ldy < n) return CURFP_STATUS_INVALID_VALUE;
  Geometry g = rfp::geometry(n, transr == CURFP_OP_T, uplo == CURFP_FILL_MODE_LOWER);
  return status_of(symm_launch(handle, g, A, X, ldx, Y, ldy, nrhs, *alpha, *beta));
}

// src/curfp_ssfmm.cpp:108-306.  side = LEFT: C := alpha A B + beta C (A of
// order m); side = RIGHT: C := alpha B A + beta C (A of order n), computed as
// C^T = alpha A B^T + beta C^T on transposed views.  B and C are column-major
// m x n; the leading dimensions must cover m (the bound the reference's cuBLAS
// calls enforce).  alpha = 0 reads neither A nor B; beta = 0 does not read C.
template <typename T>
static curfpStatus_t sfmm_impl(curfpHandle_t handle, curfpOperation_t transr,
                               curfpFillMode_t uplo, curfpSideMode_t side, int m, int n,
                               const T* alpha, const T* arf, const T* B, int ldb, const T* beta,
                               T* C, int ldc) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (m < 0 || n < 0 || ldb < 1 || ldc < 1) return CURFP_STATUS_INVALID_VALUE;
  if (!alpha || !beta) return CURFP_STATUS_INVALID_VALUE;
  if (m == 0 || n == 0) return CURFP_STATUS_SUCCESS;
  if (side != CURFP_SIDE_LEFT && side != CURFP_SIDE_RIGHT) return CURFP_STATUS_INVALID_VALUE;
  if (ldb < m || ldc < m) return CURFP_STATUS_INVALID_VALUE;
  const bool left = side == CURFP_SIDE_LEFT;
  rfp::ViewT<T> Bv{const_cast<T*>(B), 1, ldb}, Cv{C, 1, ldc};
  if (!left) {
    Bv = rfp::tr(Bv);
    Cv = rfp::tr(Cv);
  }
  rfp::CudaExecT<T> ex(handle);
  return status_of(rfp::plan::rfp_symm(ex, transr == CURFP_OP_T, uplo == CURFP_FILL_MODE_LOWER,
                                       left ? m : n, arf, Bv, Cv, left ? n : m, *alpha,
                                       *beta));
}

curfpStatus_t curfpSsfmm(curfpHandle_t handle, curfpOperation_t transr, curfpFillMode_t uplo,
                         curfpSideMode_t side, int m, int n, const float* alpha,
                         const float* arf, const float* B, int ldb, const float* beta,
                         float* C, int ldc) {
  return sfmm_impl(handle, transr, uplo, side, m, n, alpha, arf, B, ldb, beta, C, ldc);
}

// src/curfp_ssfmv.cpp:134-255: y := alpha A x + beta y.  Increments follow
// BLAS (a negative increment walks the vector backwards); zero is rejected.
template <typename T>
static curfpStatus_t sfmv_impl(curfpHandle_t handle, curfpOperation_t transr,
                               curfpFillMode_t uplo, int n, const T* alpha, const T* arf,
                               const T* x, int incx, const T* beta, T* y, int incy) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  if (!alpha || !beta || incx == 0 || incy == 0) return CURFP_STATUS_INVALID_VALUE;
  const int64_t ox = incx < 0 ? -(int64_t)(n - 1) * incx : 0;
  const int64_t oy = incy < 0 ? -(int64_t)(n - 1) * incy : 0;
  const int tr = transr == CURFP_OP_T, lower = uplo == CURFP_FILL_MODE_LOWER;
  if (*alpha == T(0)) {  // y := beta y, neither A nor x read
    rfp::ViewT<T> X{const_cast<T*>(x) + ox, incx, 1}, Y{y + oy, incy, 1};
    rfp::CudaExecT<T> ex(handle);
    return status_of(rfp::plan::rfp_symm(ex, tr, lower, n, arf, X, Y, 1, *alpha, *beta));
  }
  const Geometry g = rfp::geometry(n, tr, lower);
  const rfp::ksymv::Parts P = rfp::ksymv::parts(n);
  T* part = static_cast<T*>(rfp::grow_buffer(handle, &handle->ws, &handle->ws_bytes,
                                             (size_t)(P.n_row + P.n_col) * sizeof(T)));
  if (!part) return CURFP_STATUS_ALLOC_FAILED;
  const double nt = (double)n * (n + 1) / 2;
  rfp::ProfScope ps(handle->prof, handle->stream, rfp::K_SGEMM, 4.0 * nt, sizeof(T) * nt);
  rfp::ksymv::symv_tiles<T>
      <<<(unsigned)rfp::ksymv::strips_before(P.tiles), rfp::ksymv::kThreads, 0, handle->stream>>>(
          g, arf, x + ox, incx, part);
  rfp::ksymv::symv_reduce<T><<<P.tiles, rfp::ksymv::kThreads, 0, handle->stream>>>(
      n, part, y + oy, incy, *alpha, *beta);
  handle->launches += 2;
  return ok_launch() ? CURFP_STATUS_SUCCESS : CURFP_STATUS_EXECUTION_FAILED;
}

curfpStatus_t curfpSsfmv(curfpHandle_t handle, curfpOperation_t transr, curfpFillMode_t uplo,
                         int n, const float* alpha, const float* arf, const float* x,
                         int incx, const float* beta, float* y, int incy) {
  return sfmv_impl(handle, transr, uplo, n, alpha, arf, x, incx, beta, y, incy);
}

namespace {
// Shared body of the rank-1 / rank-2 updates (y == nullptr: rank 1).
template <typename T>
curfpStatus_t rank_update(curfpHandle_t h, curfpOperation_t transr, curfpFillMode_t uplo, int n,
                          const T* alpha, const T* x, int incx, const T* y, int incy, T* arf) {
  if (!h) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0 || !alpha) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0 || *alpha == T(0)) return CURFP_STATUS_SUCCESS;
  if (incx == 0 || (y && incy == 0) || !x || !arf) return CURFP_STATUS_INVALID_VALUE;
  Geometry g = rfp::geometry(n, transr == CURFP_OP_T, uplo == CURFP_FILL_MODE_LOWER);
  rfp::kpack::PackArgs a{};
  const int tiles = rfp::kpack::pack_blocks(g, &a);
  const T* xb = x + (incx < 0 ? -(int64_t)(n - 1) * incx : 0);
  const T* yb = y ? y + (incy < 0 ? -(int64_t)(n - 1) * incy : 0) : nullptr;
  const double nt = (double)n * (n + 1) / 2;
  rfp::ProfScope ps(h->prof, h->stream, rfp::K_PACK, (y ? 4.0 : 2.0) * nt,
                    2.0 * sizeof(T) * nt);
  rfp::kpack::rank_update<T><<<tiles, dim3(rfp::kpack::TX, rfp::kpack::TY), 0, h->stream>>>(
      a, arf, xb, incx, yb, incy, *alpha, y ? 1 : 0);
  ++h->launches;
  return ok_launch() ? CURFP_STATUS_SUCCESS : CURFP_STATUS_EXECUTION_FAILED;
}
}  // namespace

// src/curfp_ssfr.cpp:99-173: C := alpha x x^T + C (alpha == 0: no-op).
curfpStatus_t curfpSsfr(curfpHandle_t handle, curfpOperation_t transr, curfpFillMode_t uplo,
                        int n, const float* alpha, const float* x, int incx, float* arf) {
  return rank_update<float>(handle, transr, uplo, n, alpha, x, incx, nullptr, 0, arf);
}

// src/curfp_ssfr2.cpp:94-190: C := alpha (x y^T + y x^T) + C (alpha == 0: no-op).
curfpStatus_t curfpSsfr2(curfpHandle_t handle, curfpOperation_t transr, curfpFillMode_t uplo,
                         int n, const float* alpha, const float* x, int incx, const float* y,
                         int incy, float* arf) {
  if (!y && handle && n > 0 && alpha && *alpha != 0.0f) return CURFP_STATUS_INVALID_VALUE;
  return rank_update<float>(handle, transr, uplo, n, alpha, x, incx, y ? y : x, incy, arf);
}

// ---------------------------------------------------------------------------
// D-prefix (FP64) twins: the same planner and kernels instantiated for
// double (SIMT DFMA contractions; reference src/curfp_d*.cpp / .cu).
// ---------------------------------------------------------------------------

curfpStatus_t curfpDsfrk(curfpHandle_t handle, curfpOperation_t transr, curfpFillMode_t uplo,
                         curfpOperation_t trans, int n, int k, const double* alpha,
                         const double* A, int lda, const double* beta, double* C) {
  return ssfrk_impl(handle, transr, uplo, trans, n, k, alpha, A, lda, beta, C, 0);
}

curfpStatus_t curfpDsfr2k(curfpHandle_t handle, curfpOperation_t transr, curfpFillMode_t uplo,
                          curfpOperation_t trans, int n, int k, const double* alpha,
                          const double* A, int lda, const double* B, int ldb,
                          const double* beta, double* C) {
  return sfr2k_impl(handle, transr, uplo, trans, n, k, alpha, A, lda, B, ldb, beta, C);
}

curfpStatus_t curfpDpftrf(curfpHandle_t handle, curfpOperation_t transr, curfpFillMode_t uplo,
                          int n, double* A, int* info) {
  return spftrf_impl(handle, transr, uplo, n, A, info, 0);
}

curfpStatus_t curfpDpftrs(curfpHandle_t handle, curfpOperation_t transr, curfpFillMode_t uplo,
                          int n, int nrhs, const double* A, double* B, int ldb) {
  return pftrs_impl(handle, transr, uplo, n, nrhs, A, B, ldb);
}

curfpStatus_t curfpDpftri(curfpHandle_t handle, curfpOperation_t transr, curfpFillMode_t uplo,
                          int n, double* arf) {
  return pftri_impl(handle, transr, uplo, n, arf);
}

curfpStatus_t curfpDstrttf(curfpHandle_t handle, curfpOperation_t transr, curfpFillMode_t uplo,
                           int n, const double* A, int lda, double* arf) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0 || lda < n) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  return pack(handle, transr == CURFP_OP_T, uplo == CURFP_FILL_MODE_LOWER, n, A, arf, lda, 1);
}

curfpStatus_t curfpDstfttr(curfpHandle_t handle, curfpOperation_t transr, curfpFillMode_t uplo,
                           int n, const double* arf, double* A, int lda) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0 || lda < n) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  return pack(handle, transr == CURFP_OP_T, uplo == CURFP_FILL_MODE_LOWER, n, arf, A, lda, 0);
}

curfpStatus_t curfpDsfmm(curfpHandle_t handle, curfpOperation_t transr, curfpFillMode_t uplo,
                         curfpSideMode_t side, int m, int n, const double* alpha,
                         const double* arf, const double* B, int ldb, const double* beta,
                         double* C, int ldc) {
  return sfmm_impl(handle, transr, uplo, side, m, n, alpha, arf, B, ldb, beta, C, ldc);
}

curfpStatus_t curfpDsfmv(curfpHandle_t handle, curfpOperation_t transr, curfpFillMode_t uplo,
                         int n, const double* alpha, const double* arf, const double* x,
                         int incx, const double* beta, double* y, int incy) {
  return sfmv_impl(handle, transr, uplo, n, alpha, arf, x, incx, beta, y, incy);
}

curfpStatus_t curfpDsfr(curfpHandle_t handle, curfpOperation_t transr, curfpFillMode_t uplo,
                        int n, const double* alpha, const double* x, int incx, double* arf) {
  return rank_update<double>(handle, transr, uplo, n, alpha, x, incx, nullptr, 0, arf);
}

curfpStatus_t curfpDsfr2(curfpHandle_t handle, curfpOperation_t transr, curfpFillMode_t uplo,
                         int n, const double* alpha, const double* x, int incx, const double* y,
                         int incy, double* arf) {
  if (!y && handle && n > 0 && alpha && *alpha != 0.0) return CURFP_STATUS_INVALID_VALUE;
  return rank_update<double>(handle, transr, uplo, n, alpha, x, incx, y ? y : x, incy, arf);
}

// ---------------------------------------------------------------------------
// Adjoints (differentiation form)
// ---------------------------------------------------------------------------

// Abar := alpha (tril(Cbar) + tril(Cbar)^T) op(A): the cotangent of A for
// C = alpha op(A) op(A)^T + beta C when Cbar is the cotangent of C's stored
// elements (an off-diagonal stored element is two entries of the symmetric
// matrix, hence the doubled diagonal of the symmetric factor).
curfpStatus_t curfpSsfrkBackward(curfpHandle_t handle, curfpOperation_t transr,
                                 curfpFillMode_t uplo, curfpOperation_t trans, int n, int k,
                                 const float* alpha, const float* A, int lda,
                                 const float* Cbar, float* Abar, int ldabar) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0 || k < 0 || lda < 1 || ldabar < 1 || !alpha) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0 || k == 0) return CURFP_STATUS_SUCCESS;
  const int tt = trans == CURFP_OP_T;
  if (lda < (tt ? k : n) || ldabar < (tt ? k : n)) return CURFP_STATUS_INVALID_VALUE;
  rfp::View X = tt ? rfp::View{const_cast<float*>(A), lda, 1}
                   : rfp::View{const_cast<float*>(A), 1, lda};
  rfp::View Y = tt ? rfp::View{Abar, ldabar, 1} : rfp::View{Abar, 1, ldabar};
  CudaExec ex(handle);
  return status_of(rfp::plan::rfp_symm_dbl(ex, transr == CURFP_OP_T,
                                           uplo == CURFP_FILL_MODE_LOWER, n, Cbar, X, Y, k,
                                           *alpha, 0.0f));
}

// Cotangent of the stored elements of A from that of its Cholesky factor,
// computed in place in Abar by the blocked RFP adjoint
// (rfp::plan::spftrf_adjoint): only L and the cotangent are held, plus the
// solves' diagonal-block inverses (n/64 records of 32 KB).  Abar may alias
// Lbar; it must not alias L, which is read throughout.
static curfpStatus_t spftrf_backward_body(curfpHandle_t handle, curfpOperation_t transr,
                                          curfpFillMode_t uplo, int n, const float* L,
                                          const float* Lbar, float* Abar, curfpMath_t math) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0) return CURFP_STATUS_INVALID_VALUE;
  if (math != CURFP_MATH_FP32 && math != CURFP_MATH_SPLIT_BF16) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  if (!L || !Lbar || !Abar || Abar == L) return CURFP_STATUS_INVALID_VALUE;
  const int tr = transr == CURFP_OP_T, lower = uplo == CURFP_FILL_MODE_LOWER;
  if (Abar != Lbar &&
      cudaMemcpyAsync(Abar, Lbar, (size_t)n * (n + 1) / 2 * sizeof(float),
                      cudaMemcpyDeviceToDevice, handle->stream) != cudaSuccess)
    return CURFP_STATUS_EXECUTION_FAILED;
  CudaExec ex(handle);
  return status_of(rfp::plan::spftrf_adjoint(ex, tr, lower, n, L, Abar, (int)math));
}

// X = A^-1 B with A = L L^T:  Bbar := A^-1 Xbar and
// Lbar := -tril(Bbar (L^T X)^T + X (L^T Bbar)^T) on the factor's stored elements.
static curfpStatus_t spftrs_backward_body(curfpHandle_t handle, curfpOperation_t transr,
                                          curfpFillMode_t uplo, int n, int nrhs, const float* L,
                                          const float* X, int ldx, const float* Xbar, int ldxbar,
                                          float* Bbar, int ldbbar, float* Lbar) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0 || nrhs < 0) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0) return CURFP_STATUS_SUCCESS;
  if (ldx < n || ldxbar < n || ldbbar < n) return CURFP_STATUS_INVALID_VALUE;
  const int tr = transr == CURFP_OP_T, lower = uplo == CURFP_FILL_MODE_LOWER;
  if (nrhs == 0) {
    if (!Lbar) return CURFP_STATUS_SUCCESS;
    return cudaMemsetAsync(Lbar, 0, (size_t)n * (n + 1) / 2 * sizeof(float),
                           handle->stream) == cudaSuccess
               ? CURFP_STATUS_SUCCESS
               : CURFP_STATUS_EXECUTION_FAILED;
  }
  cudaStream_t st = handle->stream;
  const int cb = (int)(((int64_t)n * nrhs + 255) / 256 < 4096 ? ((int64_t)n * nrhs + 255) / 256
                                                               : 4096);
  if (Bbar != Xbar) {
    rfp::kref::copy_block<<<cb, 256, 0, st>>>(Bbar, ldbbar, Xbar, ldxbar, n, nrhs);
    ++handle->launches;
    if (!ok_launch()) return CURFP_STATUS_EXECUTION_FAILED;
  }
  CudaExec ex(handle);
  int rc = rfp::plan::spftrs(ex, tr, lower, n, nrhs, L, Bbar, ldbbar);
  if (rc || !Lbar) return status_of(rc);
  // W = [L^T X | L^T Bbar]  (n x 2 nrhs, column-major)
  float* W = static_cast<float*>(rfp::grow_buffer(handle, &handle->wsg, &handle->wsg_bytes,
                                                  (size_t)2 * n * nrhs * sizeof(float)));
  if (!W) return CURFP_STATUS_ALLOC_FAILED;
  float* W2 = W + (size_t)n * nrhs;
  rfp::kref::copy_block<<<cb, 256, 0, st>>>(W, n, X, ldx, n, nrhs);
  rfp::kref::copy_block<<<cb, 256, 0, st>>>(W2, n, Bbar, ldbbar, n, nrhs);
  handle->launches += 2;
  if (!ok_launch()) return CURFP_STATUS_EXECUTION_FAILED;
  rfp::View Wv{W, 1, n};
  if ((rc = rfp::plan::rfp_trmm_t(ex, tr, lower, n, L, Wv, 2 * nrhs))) return status_of(rc);
  rfp::View Bb{Bbar, 1, ldbbar}, Xv{const_cast<float*>(X), 1, ldx};
  return status_of(rfp::plan::rfp_gemm_lower2(ex, tr, lower, n, Lbar, Bb, rfp::tr(Wv), Xv,
                                              rfp::tr(rfp::View{W2, 1, n}), nrhs, -1.0f,
                                              0.0f));
}

// Mixed-precision refinement around spftrs (see include/curfp.h).
static curfpStatus_t refine_body(curfpHandle_t handle, curfpOperation_t transr,
                                 curfpFillMode_t uplo, int n, int nrhs, const float* Aorig,
                                 const float* factor, float* B, int ldb, int max_iter,
                                 int* iters) {
  if (iters) *iters = 0;
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0 || nrhs < 0 || ldb < 1 || max_iter < 0) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0 || nrhs == 0) return CURFP_STATUS_SUCCESS;
  if (ldb < n) return CURFP_STATUS_INVALID_VALUE;
  const int tr = transr == CURFP_OP_T, lower = uplo == CURFP_FILL_MODE_LOWER;
  cudaStream_t st = handle->stream;
  const size_t blk = (size_t)n * nrhs;
  // scratch: saved right-hand side, residual, one word for the norm
  float* scratch = static_cast<float*>(rfp::grow_buffer(
      handle, &handle->ws2, &handle->ws2_bytes, (2 * blk + 64) * sizeof(float)));
  if (!scratch) return CURFP_STATUS_ALLOC_FAILED;
  float* B0 = scratch;
  float* R = scratch + blk;
  unsigned* nrm = reinterpret_cast<unsigned*>(scratch + 2 * blk);
  const int grid = 148 * 8;
  rfp::kref::copy_block<<<grid, 256, 0, st>>>(B0, n, B, ldb, n, nrhs);
  ++handle->launches;
  CudaExec ex(handle);
  // The solves take split-BF16 tensor-core updates where large enough: the
  // corrections need only FP32-level accuracy, the FP64 residual carries the
  // refinement.
  const int kMath = CURFP_MATH_SPLIT_BF16;
  int rc = rfp::plan::spftrs(ex, tr, lower, n, nrhs, factor, B, ldb, kMath);
  if (rc) return status_of(rc);
  Geometry g = rfp::geometry(n, tr, lower);
  float prev = INFINITY;
  auto absmax_of = [&](const float* M, int64_t ld, float* out) -> bool {
    if (cudaMemsetAsync(nrm, 0, sizeof(unsigned), st) != cudaSuccess) return false;
    rfp::kref::absmax<<<grid, 256, 0, st>>>(M, ld, n, nrhs, nrm);
    ++handle->launches;
    unsigned bits = 0;
    if (!ok_launch() ||
        cudaMemcpyAsync(&bits, nrm, sizeof(unsigned), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return false;
    memcpy(out, &bits, sizeof(float));
    return true;
  };
  for (int it = 0; it < max_iter; ++it) {
    // R := B0 - A X in FP64
    rfp::kref::copy_block<<<grid, 256, 0, st>>>(R, n, B0, n, n, nrhs);
    if ((rc = symm_launch(handle, g, Aorig, B, ldb, R, n, nrhs, -1.0f, 1.0f)))
      return status_of(rc);
    ++handle->launches;
    float r;
    if (!absmax_of(R, n, &r)) return CURFP_STATUS_EXECUTION_FAILED;
    if (!(r < 0.5f * prev) || r == 0.0f) break;  // converged or stalled
    prev = r;
    if ((rc = rfp::plan::spftrs(ex, tr, lower, n, nrhs, factor, R, n, kMath)))
      return status_of(rc);
    rfp::kref::add_inplace<<<grid, 256, 0, st>>>(B, ldb, R, n, n, nrhs);
    ++handle->launches;
    if (!ok_launch()) return CURFP_STATUS_EXECUTION_FAILED;
    if (iters) *iters = it + 1;
    // A correction below 4 ulp of the solution: another residual would not
    // change the FP32 result.
    float d, x;
    if (it + 1 < max_iter) {
      if (!absmax_of(R, n, &d) || !absmax_of(B, ldb, &x)) return CURFP_STATUS_EXECUTION_FAILED;
      if (d <= 0x1p-22f * x) break;
    }
  }
  return CURFP_STATUS_SUCCESS;
}

// The three entry points above, each under a check of the kernel error word
// (status.cuh): a wait that ran out surfaces as EXECUTION_FAILED.
curfpStatus_t curfpSpftrfBackward(curfpHandle_t handle, curfpOperation_t transr,
                                  curfpFillMode_t uplo, int n, const float* L,
                                  const float* Lbar, float* Abar, curfpMath_t math) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  return rfp::status::checked(handle, [&] {
    return spftrf_backward_body(handle, transr, uplo, n, L, Lbar, Abar, math);
  });
}

curfpStatus_t curfpSpftrsBackward(curfpHandle_t handle, curfpOperation_t transr,
                                  curfpFillMode_t uplo, int n, int nrhs, const float* L,
                                  const float* X, int ldx, const float* Xbar, int ldxbar,
                                  float* Bbar, int ldbbar, float* Lbar) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  return rfp::status::checked(handle, [&] {
    return spftrs_backward_body(handle, transr, uplo, n, nrhs, L, X, ldx, Xbar, ldxbar, Bbar,
                                ldbbar, Lbar);
  });
}

curfpStatus_t curfpSpftrsRefine(curfpHandle_t handle, curfpOperation_t transr,
                                curfpFillMode_t uplo, int n, int nrhs, const float* Aorig,
                                const float* factor, float* B, int ldb, int max_iter,
                                int* iters) {
  if (iters) *iters = 0;
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  return rfp::status::checked(handle, [&] {
    return refine_body(handle, transr, uplo, n, nrhs, Aorig, factor, B, ldb, max_iter, iters);
  });
}

// Math mode of the drop-in FP32 routines (curfpSsfrk, curfpSsfr2k,
// curfpSpftrf, curfpSpftrs, curfpSpftri); include/curfp.h.
curfpStatus_t curfpSetMathMode(curfpHandle_t handle, curfpMath_t math) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (math != CURFP_MATH_FP32 && math != CURFP_MATH_SPLIT_BF16) return CURFP_STATUS_INVALID_VALUE;
  handle->math = (int)math;
  return CURFP_STATUS_SUCCESS;
}

curfpStatus_t curfpGetMathMode(curfpHandle_t handle, curfpMath_t* math) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (!math) return CURFP_STATUS_INVALID_VALUE;
  *math = (curfpMath_t)handle->math;
  return CURFP_STATUS_SUCCESS;
}

// Per-kernel-class event timing (profile.h).
curfpStatus_t curfpProfileEnable(curfpHandle_t handle, int enable) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  cudaStreamSynchronize(handle->stream);
  handle->prof.reset();
  handle->prof.on = enable != 0;
  return CURFP_STATUS_SUCCESS;
}

curfpStatus_t curfpProfileRead(curfpHandle_t handle, int kclass, double* ms, double* flops,
                               double* bytes, long long* launches) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (kclass < 0 || kclass >= rfp::K_NCLASS || !ms || !flops || !bytes || !launches)
    return CURFP_STATUS_INVALID_VALUE;
  if (cudaStreamSynchronize(handle->stream) != cudaSuccess) return CURFP_STATUS_EXECUTION_FAILED;
  double t = 0, f = 0, b = 0;
  long long c = 0;
  for (const auto& r : handle->prof.recs) {
    if (r.cls != kclass) continue;
    float e = 0.f;
    if (cudaEventElapsedTime(&e, r.e0, r.e1) != cudaSuccess) return CURFP_STATUS_EXECUTION_FAILED;
    t += e; f += r.flops; b += r.bytes; ++c;
  }
  *ms = t; *flops = f; *bytes = b; *launches = c;
  return CURFP_STATUS_SUCCESS;
}

// Every record since curfpProfileEnable, 8 doubles each: class, device ms,
// flops, bytes, and the contraction shape (m, n, k, output tiles; zeros when
// not given).  Writes at most max_records; *count receives the number held.
curfpStatus_t curfpProfileRecords(curfpHandle_t handle, long long max_records,
                                  long long* count, double* out) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (!count || (max_records > 0 && !out)) return CURFP_STATUS_INVALID_VALUE;
  if (cudaStreamSynchronize(handle->stream) != cudaSuccess) return CURFP_STATUS_EXECUTION_FAILED;
  const auto& recs = handle->prof.recs;
  *count = (long long)recs.size();
  for (long long i = 0; i < max_records && i < (long long)recs.size(); ++i) {
    const auto& r = recs[(size_t)i];
    float e = 0.f;
    if (cudaEventElapsedTime(&e, r.e0, r.e1) != cudaSuccess) return CURFP_STATUS_EXECUTION_FAILED;
    double* o = out + 8 * i;
    o[0] = r.cls; o[1] = e; o[2] = r.flops; o[3] = r.bytes;
    o[4] = r.m; o[5] = r.n; o[6] = r.k; o[7] = r.tiles;
  }
  return CURFP_STATUS_SUCCESS;
}

// Number of kernels this handle has launched (diagnostic counter).
curfpStatus_t curfpGetKernelLaunchCount(curfpHandle_t handle, long long* count) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (!count) return CURFP_STATUS_INVALID_VALUE;
  *count = handle->launches;
  return CURFP_STATUS_SUCCESS;
}

