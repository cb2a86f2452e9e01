// nll.cu — fused gradient of the Gaussian-process negative log marginal
// likelihood  f = 1/2 y^T C^-1 y + sum_i log L_ii,  C = s X X^T + sigma2 I
// = L L^T, from the factor alone (nothing of the forward pass but L, X and
// alpha = C^-1 y is kept):
//   Cbar = 1/2 (C^-1 - alpha alpha^T)
//   Xbar = 2 s Cbar X = s (C^-1 X - alpha (alpha^T X))
//   sbar = <Cbar, X X^T> = 1/2 (|L^-1 X|_F^2 - |X^T alpha|^2)
//   sigma2bar = tr Cbar = 1/2 (|L^-1|_F^2 - |alpha|^2)
// C^-1 X comes from two RFP triangular solves with d right-hand sides,
// tr C^-1 = |L^-1|_F^2 from the RFP triangular inverse; every inner product
// is accumulated in FP64.
#include <cuda_runtime.h>

#include <climits>

#include "../../include/curfp.h"
#include "context.h"
#include "status.cuh"
#include "engine.h"
#include "k_nll.cuh"

namespace {

inline curfpStatus_t nll_status(int rc) {
  switch (rc) {
    case 0: return CURFP_STATUS_SUCCESS;
    case 2: return CURFP_STATUS_ALLOC_FAILED;
    case 3: return CURFP_STATUS_INVALID_VALUE;
    default: return CURFP_STATUS_EXECUTION_FAILED;
  }
}

inline int grid_for(int64_t work) {
  int64_t b = (work + rfp::knll::kThreads - 1) / rfp::knll::kThreads;
  return (int)(b < 4 * 148 ? (b > 0 ? b : 1) : 4 * 148);
}

}  // namespace

static curfpStatus_t nll_body(curfpHandle_t handle, curfpOperation_t transr,
                              curfpFillMode_t uplo, int n, int d, float s, const float* L,
                              const float* X, int ldx, const float* alpha, const float* g,
                              float* Xbar, int ldxbar, double* sums, curfpMath_t math) {
  if (n < 0 || d < 0 || ldx < (d > 1 ? d : 1) || ldxbar < (d > 1 ? d : 1))
    return CURFP_STATUS_INVALID_VALUE;
  if (math != CURFP_MATH_FP32 && math != CURFP_MATH_SPLIT_BF16) return CURFP_STATUS_INVALID_VALUE;
  if (!L || !alpha || !g || !sums || (d > 0 && (!X || !Xbar))) return CURFP_STATUS_INVALID_VALUE;
  cudaStream_t st = handle->stream;
  if (n == 0) return cudaMemsetAsync(sums, 0, 2 * sizeof(double), st) == cudaSuccess
                         ? CURFP_STATUS_SUCCESS
                         : CURFP_STATUS_EXECUTION_FAILED;
  const int tr = transr == CURFP_OP_T, lower = uplo == CURFP_FILL_MODE_LOWER;
  const int64_t nd = (int64_t)n * d, nt = (int64_t)n * (n + 1) / 2;
  // scratch: W (n x d row-major) | inverse factor (RFP) | acc[3] u[d] (FP64)
  const size_t fl = (size_t)(nd + nt + 1) & ~(size_t)1;
  const size_t bytes = fl * sizeof(float) + (3 + (size_t)d) * sizeof(double);
  float* W = static_cast<float*>(rfp::grow_buffer(handle, &handle->wsg, &handle->wsg_bytes, bytes));
  if (!W) return CURFP_STATUS_ALLOC_FAILED;
  float* Linv = W + nd;
  double* acc = reinterpret_cast<double*>(W + fl);
  double* u = acc + 3;
  if (cudaMemsetAsync(acc, 0, (3 + (size_t)d) * sizeof(double), st) != cudaSuccess)
    return CURFP_STATUS_EXECUTION_FAILED;
  rfp::CudaExec ex(handle);
  int rc;
  using namespace rfp::knll;
  if (d > 0) {
    if (cudaMemcpy2DAsync(W, (size_t)d * sizeof(float), X, (size_t)ldx * sizeof(float),
                          (size_t)d * sizeof(float), n, cudaMemcpyDeviceToDevice, st) !=
        cudaSuccess)
      return CURFP_STATUS_EXECUTION_FAILED;
    rfp::View Wv{W, d, 1};
    if ((rc = rfp::plan::rfp_trsm(ex, tr, lower, n, L, 0, Wv, d, 1.0f, (int)math)))
      return nll_status(rc);
    sumsq64<<<grid_for(nd), kThreads, 0, st>>>(W, nd, acc + 0);
    if ((rc = rfp::plan::rfp_trsm(ex, tr, lower, n, L, 1, Wv, d, 1.0f, (int)math)))
      return nll_status(rc);
    const int chunks = (int)(n / 64 < 4 * 148 ? (n / 64 > 0 ? n / 64 : 1) : 4 * 148);
    gemv_t64<<<dim3((d + kThreads - 1) / kThreads, chunks), kThreads, 0, st>>>(X, ldx, n, d,
                                                                              alpha, u);
    xbar<<<grid_for(nd), kThreads, 0, st>>>(Xbar, ldxbar, W, alpha, u, s, g, n, d);
    handle->launches += 3;
  }
  sumsq64<<<grid_for(n), kThreads, 0, st>>>(alpha, n, acc + 2);
  if (cudaMemcpyAsync(Linv, L, (size_t)nt * sizeof(float), cudaMemcpyDeviceToDevice, st) !=
      cudaSuccess)
    return CURFP_STATUS_EXECUTION_FAILED;
  if ((rc = rfp::plan::rfp_trtri(ex, tr, lower, n, Linv, (int)math))) return nll_status(rc);
  sumsq64<<<grid_for(nt), kThreads, 0, st>>>(Linv, nt, acc + 1);
  scalars<<<1, kThreads, 0, st>>>(acc, u, d, g, sums);
  handle->launches += 3;
  return cudaGetLastError() == cudaSuccess ? CURFP_STATUS_SUCCESS
                                           : CURFP_STATUS_EXECUTION_FAILED;
}

// The body above under a check of the kernel error word (status.cuh).
curfpStatus_t curfpSgpnllBackward(curfpHandle_t handle, curfpOperation_t transr,
                                  curfpFillMode_t uplo, int n, int d, float s, const float* L,
                                  const float* X, int ldx, const float* alpha, const float* g,
                                  float* Xbar, int ldxbar, double* sums, curfpMath_t math) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  return rfp::status::checked(handle, [&] {
    return nll_body(handle, transr, uplo, n, d, s, L, X, ldx, alpha, g, Xbar, ldxbar, sums,
                    math);
  });
}
