// norms.cu — curfpSlansf (norms of an RFP symmetric matrix) and curfpSpfcon
// (reciprocal 1-norm condition estimate from the RFP Cholesky factor).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "../../include/curfp.h"
#include "context.h"
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

extern "C" {

// Reference src/curfp_slansf.cu:280-435: argument checks, n = 0 -> 0, an
// unknown norm -> INVALID_VALUE.  MAX is the largest |element| of the flat
// array, FRO = sqrt(2 sum a^2 - sum diag^2), ONE the largest column sum.
curfpStatus_t curfpSlansf(curfpHandle_t handle, curfpNormType_t norm, curfpOperation_t transr,
                          curfpFillMode_t uplo, int n, const float* arf, float* result) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (!result) return CURFP_STATUS_INVALID_VALUE;
  if (n < 0) return CURFP_STATUS_INVALID_VALUE;
  *result = 0.0f;
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
    rfp::ProfScope ps(handle->prof, s, rfp::K_NORM, 0, 4.0 * (double)nt);
    flat_stats<<<fb, kThreads, 0, s>>>(arf, nt, part, st);  // max |a| (all norms), sum a^2
    ++handle->launches;
  }
  if (norm == CURFP_NORM_FRO) {
    sum_parts<<<1, kThreads, 0, s>>>(part, fb, st);
    diag_sumsq<<<1, kThreads, 0, s>>>(g, arf, st);
    handle->launches += 2;
  } else if (norm == CURFP_NORM_ONE) {
    auto* col = reinterpret_cast<unsigned long long*>(static_cast<char*>(tail) + parts);
    if (cudaMemsetAsync(col, 0, (size_t)n * 8, s) != cudaSuccess)
      return CURFP_STATUS_EXECUTION_FAILED;
    rfp::kpack::PackArgs a{};
    const int tiles = rfp::kpack::pack_blocks(g, &a);
    rfp::ProfScope ps(handle->prof, s, rfp::K_NORM, 0, 4.0 * (double)nt + 16.0 * n);
    colsum<<<tiles, dim3(rfp::kpack::TX, rfp::kpack::TY), 0, s>>>(a, arf, n, st, col);
    max_of<<<blocks_for(n, kGridCap), kThreads, 0, s>>>(col, n, st);
    handle->launches += 2;
  }
  if (cudaGetLastError() != cudaSuccess) return CURFP_STATUS_EXECUTION_FAILED;
  Stats hs;
  if (!read_stats(handle, st, &hs)) return CURFP_STATUS_EXECUTION_FAILED;
  const unsigned mb = (unsigned)hs.key;
  float amax;
  std::memcpy(&amax, &mb, sizeof amax);
  if (norm == CURFP_NORM_MAX) {
    *result = amax;
  } else if (norm == CURFP_NORM_FRO) {
    const double f2 = 2.0 * hs.sum - hs.diag;
    *result = f2 > 0.0 ? (float)std::sqrt(f2) : 0.0f;
    if (!(amax <= 3.0e38f)) *result = amax;  // inf or NaN element
  } else if (!(amax > 0.0f) || !(amax <= 3.0e38f)) {
    *result = amax;  // zero matrix (0), inf or NaN element
  } else {
    // the fixed-point scale of colsum_shift
    int e;
    std::frexp((double)amax * (double)n, &e);
    *result = (float)std::ldexp((double)hs.colmax, -(62 - e));
  }
  return CURFP_STATUS_SUCCESS;
}

// Reference src/curfp_spfcon.cu:88-271: LAPACK SLACN2's reverse-communication
// loop written as a state machine, with A^-T = A^-1 for the SPD matrix so
// every step applies the same solve.  As there: at most ITMAX = 5
// iterations, no cycling test (SLACN2's "est <= estold" exit), the
// convergence test of the e_j loop compares |x| at the previous and the new
// argmax, and the final alternating-sign vector may raise the estimate.  The
// repeated-sign test counts sign changes directly (zeros count as matching,
// as in the reference's dot-product form of the test).  Each step launches
// one fused statistics kernel and reads back one record.
curfpStatus_t curfpSpfcon(curfpHandle_t handle, curfpOperation_t transr, curfpFillMode_t uplo,
                          int n, const float* arf, float anorm, float* rcond) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (!rcond) return CURFP_STATUS_INVALID_VALUE;
  *rcond = 0.0f;
  if (n == 0 || anorm == 0.0f) return CURFP_STATUS_SUCCESS;
  if (n < 0) return CURFP_STATUS_INVALID_VALUE;
  if (!arf) return CURFP_STATUS_INVALID_VALUE;
  const int tr = transr == CURFP_OP_T, lower = uplo == CURFP_FILL_MODE_LOWER;
  void* tail = nullptr;
  const size_t vec = ((size_t)n * sizeof(float) + 255) & ~(size_t)255;
  Stats* st = scratch(handle, 2 * vec, &tail);
  if (!st) return CURFP_STATUS_ALLOC_FAILED;
  float* x = static_cast<float*>(tail);
  float* isgn = reinterpret_cast<float*>(static_cast<char*>(tail) + vec);
  cudaStream_t s = handle->stream;
  using namespace rfp::knorm;
  const int vb = (int)((n + 255) / 256);
  Stats hs;
  auto solve = [&]() -> curfpStatus_t {
    rfp::CudaExec ex(handle);
    const int rc = rfp::plan::spftrs(ex, tr, lower, n, 1, arf, x, n);
    return rc == 0 ? CURFP_STATUS_SUCCESS
                   : (rc == 2 ? CURFP_STATUS_ALLOC_FAILED : CURFP_STATUS_EXECUTION_FAILED);
  };
  auto stats = [&](const float* sg, int j) -> bool {
    if (cudaMemsetAsync(st, 0, sizeof(Stats), s) != cudaSuccess) return false;
    rfp::ProfScope ps(handle->prof, s, rfp::K_NORM, 0, 8.0 * n);
    vstats<<<1, kThreads, 0, s>>>(x, sg, n, j, st);
    ++handle->launches;
    return cudaGetLastError() == cudaSuccess && read_stats(handle, st, &hs);
  };
  auto launched = [&]() {
    ++handle->launches;
    return cudaGetLastError() == cudaSuccess;
  };
  const int kItMax = 5;
  float est = 0.0f;
  int j = 0, iter = 0, jump = 0;
  for (;;) {
    curfpStatus_t rc;
    switch (jump) {
      case 0:  // x = 1/n
        fill<<<vb, 256, 0, s>>>(x, n, 1.0f / (float)n);
        if (!launched()) return CURFP_STATUS_EXECUTION_FAILED;
        jump = 1;
        break;
      case 1:  // x = A^-1 (1/n)
        if (!stats(nullptr, 0)) return CURFP_STATUS_EXECUTION_FAILED;
        est = (float)hs.sum;
        if (n == 1) goto done;
        sign_save<<<vb, 256, 0, s>>>(x, isgn, n);
        if (!launched()) return CURFP_STATUS_EXECUTION_FAILED;
        jump = 2;
        break;
      case 2:  // x = A^-1 sign(x)
        if (!stats(nullptr, 0)) return CURFP_STATUS_EXECUTION_FAILED;
        j = (int)(0xffffffffu - (unsigned)(hs.key & 0xffffffffu));
        iter = 2;
        unit<<<vb, 256, 0, s>>>(x, n, j);
        if (!launched()) return CURFP_STATUS_EXECUTION_FAILED;
        jump = 3;
        break;
      case 3:  // x = A^-1 e_j
        if (!stats(isgn, 0)) return CURFP_STATUS_EXECUTION_FAILED;
        est = (float)hs.sum;
        if (hs.mismatch == 0) {  // repeated sign vector: converged
          altsgn<<<vb, 256, 0, s>>>(x, n);
          jump = 5;
        } else {
          sign_save<<<vb, 256, 0, s>>>(x, isgn, n);
          jump = 4;
        }
        if (!launched()) return CURFP_STATUS_EXECUTION_FAILED;
        break;
      case 4: {  // x = A^-1 sign(x)
        if (!stats(nullptr, j)) return CURFP_STATUS_EXECUTION_FAILED;
        const int jn = (int)(0xffffffffu - (unsigned)(hs.key & 0xffffffffu));
        unsigned top = (unsigned)(hs.key >> 32);
        float xnew;
        std::memcpy(&xnew, &top, sizeof xnew);
        if (hs.xj != xnew && iter < kItMax) {
          j = jn;
          ++iter;
          unit<<<vb, 256, 0, s>>>(x, n, j);
          jump = 3;
        } else {
          altsgn<<<vb, 256, 0, s>>>(x, n);
          jump = 5;
        }
        if (!launched()) return CURFP_STATUS_EXECUTION_FAILED;
        break;
      }
      default: {  // 5: x = A^-1 altsgn
        if (!stats(nullptr, 0)) return CURFP_STATUS_EXECUTION_FAILED;
        const float temp = 2.0f * (float)hs.sum / (3.0f * (float)n);
        if (temp > est) est = temp;
        goto done;
      }
    }
    if ((rc = solve()) != CURFP_STATUS_SUCCESS) return rc;
  }
done:
  if (est > 0.0f) *rcond = (1.0f / est) / anorm;
  return CURFP_STATUS_SUCCESS;
}

}  // extern "C"
