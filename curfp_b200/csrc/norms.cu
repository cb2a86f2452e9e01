// norms.cu — curfpSlansf (norms of an RFP symmetric matrix) and curfpSpfcon
// (reciprocal 1-norm condition estimate from the RFP Cholesky factor).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "../../include/curfp.h"
#include "context.h"
#include "status.cuh"
#include "engine.h"
#include "k_norm.cuh"

namespace {

using rfp::knorm::Stats;

inline int blocks_for(int64_t work, int cap) {
  const int64_t b = (work + rfp::knorm::kThreads - 1) / rfp::knorm::kThreads;
  return (int)(b < 1 ? 1 : (b < cap ? b : cap));
}

constexpr int kGridCap = 148 * 8;

// Scratch: Stats first, then `extra` bytes (256-byte aligned).
inline Stats* scratch(curfpHandle_t h, size_t extra, void** tail) {
  const size_t head = 256;
  void* p = rfp::grow_buffer(h, &h->ws2, &h->ws2_bytes, head + extra);
  if (!p) return nullptr;
  if (tail) *tail = static_cast<char*>(p) + head;
  return static_cast<Stats*>(p);
}

// Synchronise and copy the Stats record back.
inline bool read_stats(curfpHandle_t h, const Stats* d, Stats* out) {
  if (cudaMemcpyAsync(out, d, sizeof(Stats), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess)
    return false;
  return cudaStreamSynchronize(h->stream) == cudaSuccess;
}

}  // namespace

// Reference src/curfp_slansf.cu:280-435 (and src/curfp_dlansf.cu): argument
// checks, n = 0 -> 0, an unknown norm -> INVALID_VALUE.  MAX is the largest
// |element| of the flat array, FRO = sqrt(2 sum a^2 - sum diag^2), ONE the
// largest column sum.
template <typename T>
static curfpStatus_t lansf_impl(curfpHandle_t handle, curfpNormType_t norm,
                                curfpOperation_t transr, curfpFillMode_t uplo, int n,
                                const T* arf, T* result) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (!result) return CURFP_STATUS_INVALID_VALUE;
  if (n < 0) return CURFP_STATUS_INVALID_VALUE;
  *result = T(0);
  if (n == 0) return CURFP_STATUS_SUCCESS;
  if (norm != CURFP_NORM_MAX && norm != CURFP_NORM_ONE && norm != CURFP_NORM_FRO)
    return CURFP_STATUS_INVALID_VALUE;
  if (!arf) return CURFP_STATUS_INVALID_VALUE;
  const int tr = transr == CURFP_OP_T, lower = uplo == CURFP_FILL_MODE_LOWER;
  const rfp::Geometry g = rfp::geometry(n, tr, lower);
  const int64_t nt = (int64_t)n * (n + 1) / 2;
  using namespace rfp::knorm;
  // scratch: per-CTA partials (kMaxParts doubles), then the column sums
  void* tail = nullptr;
  const size_t parts = (size_t)kMaxParts * sizeof(double);
  Stats* st = scratch(handle, parts + (norm == CURFP_NORM_ONE ? (size_t)n * 8 : 0), &tail);
  if (!st) return CURFP_STATUS_ALLOC_FAILED;
  double* part = static_cast<double*>(tail);
  cudaStream_t s = handle->stream;
  if (cudaMemsetAsync(st, 0, sizeof(Stats), s) != cudaSuccess)
    return CURFP_STATUS_EXECUTION_FAILED;
  const int fb = blocks_for((nt + 3) / 4, kMaxParts);
  {
    rfp::ProfScope ps(handle->prof, s, rfp::K_NORM, 0, (double)sizeof(T) * nt);
    flat_stats<T><<<fb, kThreads, 0, s>>>(arf, nt, part, st);  // max |a| (all norms), sum a^2
    ++handle->launches;
  }
  if (norm == CURFP_NORM_FRO) {
    sum_parts<<<1, kThreads, 0, s>>>(part, fb, st);
    diag_sumsq<T><<<1, kThreads, 0, s>>>(g, arf, st);
    handle->launches += 2;
  } else if (norm == CURFP_NORM_ONE) {
    auto* col = reinterpret_cast<unsigned long long*>(static_cast<char*>(tail) + parts);
    if (cudaMemsetAsync(col, 0, (size_t)n * 8, s) != cudaSuccess)
      return CURFP_STATUS_EXECUTION_FAILED;
    rfp::kpack::PackArgs a{};
    const int tiles = rfp::kpack::pack_blocks(g, &a);
    rfp::ProfScope ps(handle->prof, s, rfp::K_NORM, 0, (double)sizeof(T) * nt + 16.0 * n);
    colsum<T><<<tiles, dim3(rfp::kpack::TX, rfp::kpack::TY), 0, s>>>(a, arf, n, st, col);
    max_of<<<blocks_for(n, kGridCap), kThreads, 0, s>>>(col, n, st);
    handle->launches += 2;
  }
  if (cudaGetLastError() != cudaSuccess) return CURFP_STATUS_EXECUTION_FAILED;
  Stats hs;
  if (!read_stats(handle, st, &hs)) return CURFP_STATUS_EXECUTION_FAILED;
  const double amax = key_value(hs.key, sizeof(T) == 8);
  if (norm == CURFP_NORM_MAX) {
    *result = (T)amax;
  } else if (norm == CURFP_NORM_FRO) {
    const double f2 = 2.0 * hs.sum - hs.diag;
    *result = f2 > 0.0 ? (T)std::sqrt(f2) : T(0);
    if (!(amax <= 1.0e300)) *result = (T)amax;  // inf or NaN element
  } else if (!(amax > 0.0) || !(amax <= 1.0e300)) {
    *result = (T)amax;  // zero matrix (0), inf or NaN element
  } else {
    *result = (T)std::ldexp((double)hs.colmax, -colsum_shift(amax, n));
  }
  return CURFP_STATUS_SUCCESS;
}

// Reference src/curfp_spfcon.cu:88-271 (and src/curfp_dpfcon.cu): LAPACK
// SLACN2's reverse-communication loop written as a state machine, with A^-T =
// A^-1 for the SPD matrix so every step applies the same solve.  As there: at
// most ITMAX = 5 iterations, no cycling test (SLACN2's "est <= estold" exit),
// the convergence test of the e_j loop compares |x| at the previous and the
// new argmax, and the final alternating-sign vector may raise the estimate.
// The repeated-sign test counts sign changes directly (zeros count as
// matching, as in the reference's dot-product form of the test).  Each step
// launches one fused statistics kernel and reads back one record.
template <typename T>
static curfpStatus_t pfcon_impl(curfpHandle_t handle, curfpOperation_t transr,
                                curfpFillMode_t uplo, int n, const T* arf, T anorm, T* rcond) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (!rcond) return CURFP_STATUS_INVALID_VALUE;
  *rcond = T(0);
  if (n == 0 || anorm == T(0)) return CURFP_STATUS_SUCCESS;
  if (n < 0) return CURFP_STATUS_INVALID_VALUE;
  if (!arf) return CURFP_STATUS_INVALID_VALUE;
  const int tr = transr == CURFP_OP_T, lower = uplo == CURFP_FILL_MODE_LOWER;
  void* tail = nullptr;
  const size_t vec = ((size_t)n * sizeof(T) + 255) & ~(size_t)255;
  Stats* st = scratch(handle, 2 * vec, &tail);
  if (!st) return CURFP_STATUS_ALLOC_FAILED;
  T* x = static_cast<T*>(tail);
  T* isgn = reinterpret_cast<T*>(static_cast<char*>(tail) + vec);
  cudaStream_t s = handle->stream;
  using namespace rfp::knorm;
  const int vb = (int)((n + 255) / 256);
  Stats hs;
  auto solve = [&]() -> curfpStatus_t {
    rfp::CudaExecT<T> ex(handle);
    rfp::status::WaitCheck wc(handle);
    const int rc = wc.finish(rfp::plan::spftrs(ex, tr, lower, n, 1, arf, x, n));
    return rc == 0 ? CURFP_STATUS_SUCCESS
                   : (rc == 2 ? CURFP_STATUS_ALLOC_FAILED : CURFP_STATUS_EXECUTION_FAILED);
  };
  auto stats = [&](const T* sg, int j) -> bool {
    if (cudaMemsetAsync(st, 0, sizeof(Stats), s) != cudaSuccess) return false;
    rfp::ProfScope ps(handle->prof, s, rfp::K_NORM, 0, 2.0 * sizeof(T) * n);
    vstats<T><<<1, kThreads, 0, s>>>(x, sg, n, j, st);
    ++handle->launches;
    return cudaGetLastError() == cudaSuccess && read_stats(handle, st, &hs);
  };
  auto launched = [&]() {
    ++handle->launches;
    return cudaGetLastError() == cudaSuccess;
  };
  const int kItMax = 5;
  T est = T(0);
  int j = 0, iter = 0, jump = 0;
  for (;;) {
    curfpStatus_t rc;
    switch (jump) {
      case 0:  // x = 1/n
        fill<T><<<vb, 256, 0, s>>>(x, n, T(1) / (T)n);
        if (!launched()) return CURFP_STATUS_EXECUTION_FAILED;
        jump = 1;
        break;
      case 1:  // x = A^-1 (1/n)
        if (!stats(nullptr, 0)) return CURFP_STATUS_EXECUTION_FAILED;
        est = (T)hs.sum;
        if (n == 1) goto done;
        sign_save<T><<<vb, 256, 0, s>>>(x, isgn, n);
        if (!launched()) return CURFP_STATUS_EXECUTION_FAILED;
        jump = 2;
        break;
      case 2:  // x = A^-1 sign(x)
        if (!stats(nullptr, 0)) return CURFP_STATUS_EXECUTION_FAILED;
        j = hs.argmax;
        iter = 2;
        unit<T><<<vb, 256, 0, s>>>(x, n, j);
        if (!launched()) return CURFP_STATUS_EXECUTION_FAILED;
        jump = 3;
        break;
      case 3:  // x = A^-1 e_j
        if (!stats(isgn, 0)) return CURFP_STATUS_EXECUTION_FAILED;
        est = (T)hs.sum;
        if (hs.mismatch == 0) {  // repeated sign vector: converged
          altsgn<T><<<vb, 256, 0, s>>>(x, n);
          jump = 5;
        } else {
          sign_save<T><<<vb, 256, 0, s>>>(x, isgn, n);
          jump = 4;
        }
        if (!launched()) return CURFP_STATUS_EXECUTION_FAILED;
        break;
      case 4: {  // x = A^-1 sign(x)
        if (!stats(nullptr, j)) return CURFP_STATUS_EXECUTION_FAILED;
        if (hs.xj != hs.xmax && iter < kItMax) {
          j = hs.argmax;
          ++iter;
          unit<T><<<vb, 256, 0, s>>>(x, n, j);
          jump = 3;
        } else {
          altsgn<T><<<vb, 256, 0, s>>>(x, n);
          jump = 5;
        }
        if (!launched()) return CURFP_STATUS_EXECUTION_FAILED;
        break;
      }
      default: {  // 5: x = A^-1 altsgn
        if (!stats(nullptr, 0)) return CURFP_STATUS_EXECUTION_FAILED;
        const T temp = T(2) * (T)hs.sum / (T(3) * (T)n);
        if (temp > est) est = temp;
        goto done;
      }
    }
    if ((rc = solve()) != CURFP_STATUS_SUCCESS) return rc;
  }
done:
  if (est > T(0)) *rcond = (T(1) / est) / anorm;
  return CURFP_STATUS_SUCCESS;
}

curfpStatus_t curfpSlansf(curfpHandle_t handle, curfpNormType_t norm, curfpOperation_t transr,
                          curfpFillMode_t uplo, int n, const float* arf, float* result) {
  return lansf_impl(handle, norm, transr, uplo, n, arf, result);
}

curfpStatus_t curfpDlansf(curfpHandle_t handle, curfpNormType_t norm, curfpOperation_t transr,
                          curfpFillMode_t uplo, int n, const double* arf, double* result) {
  return lansf_impl(handle, norm, transr, uplo, n, arf, result);
}

curfpStatus_t curfpSpfcon(curfpHandle_t handle, curfpOperation_t transr, curfpFillMode_t uplo,
                          int n, const float* arf, float anorm, float* rcond) {
  return pfcon_impl(handle, transr, uplo, n, arf, anorm, rcond);
}

curfpStatus_t curfpDpfcon(curfpHandle_t handle, curfpOperation_t transr, curfpFillMode_t uplo,
                          int n, const double* arf, double anorm, double* rcond) {
  return pfcon_impl(handle, transr, uplo, n, arf, anorm, rcond);
}
