// k_nll.cuh — reductions and the gradient epilogue of the Gaussian-process
// negative log marginal likelihood (FP64 accumulation throughout: the
// gradient is dominated by alpha (alpha^T X), whose inner products cancel
// heavily, so they are summed in FP64 and rounded once).
#pragma once
#include <cstdint>

namespace rfp {
namespace knll {

constexpr int kThreads = 256;

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double part[kThreads / 32];
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < kThreads / 32 ? part[threadIdx.x] : 0.0;
    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  }
  return t;
}

// *out += sum x[i]^2 over a contiguous array (grid-stride, one atomic per CTA).
__global__ void __launch_bounds__(kThreads) sumsq64(const float* __restrict__ x, int64_t count,
                                                    double* out) {
  double acc = 0.0;
  for (int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x; e < count;
       e += (int64_t)gridDim.x * kThreads) {
    const double v = x[e];
    acc = fma(v, v, acc);
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) atomicAdd(out, acc);
}

// u[k] += sum_j a[j] X[j*ldx + k] for a row-major n x d X: threads run along k
// (coalesced), blockIdx.y takes a chunk of rows; one FP64 atomic per column
// per CTA.
__global__ void __launch_bounds__(kThreads) gemv_t64(const float* __restrict__ X, int64_t ldx,
                                                     int n, int d, const float* __restrict__ a,
                                                     double* u) {
  const int k = blockIdx.x * kThreads + threadIdx.x;
  const int per = (n + gridDim.y - 1) / gridDim.y;
  const int j0 = blockIdx.y * per, j1 = min(n, j0 + per);
  if (k >= d) return;
  double acc = 0.0;
  for (int j = j0; j < j1; ++j) acc = fma((double)a[j], (double)X[(int64_t)j * ldx + k], acc);
  atomicAdd(u + k, acc);
}

// Xbar[j*ldb + k] = s * g * (V[j*d + k] - a[j] u[k]), evaluated in FP64.
__global__ void __launch_bounds__(kThreads) xbar(float* __restrict__ Xbar, int64_t ldb,
                                                 const float* __restrict__ V,
                                                 const float* __restrict__ a,
                                                 const double* __restrict__ u, float s,
                                                 const float* __restrict__ g, int n, int d) {
  const double sg = (double)s * (double)*g;
  const int64_t total = (int64_t)n * d;
  for (int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * kThreads) {
    const int64_t j = e / d, k = e % d;
    Xbar[j * ldb + k] = (float)(sg * ((double)V[e] - (double)a[j] * u[k]));
  }
}

// out[0] = g/2 (acc[0] - |u|^2)  (d/ds),  out[1] = g/2 (acc[1] - acc[2])
// (d/dsigma2), with acc = {|L^-1 X|_F^2, |L^-1|_F^2, |alpha|^2}.
__global__ void __launch_bounds__(kThreads) scalars(const double* __restrict__ acc,
                                                    const double* __restrict__ u, int d,
                                                    const float* __restrict__ g, double* out) {
  double t = 0.0;
  for (int k = threadIdx.x; k < d; k += kThreads) t = fma(u[k], u[k], t);
  t = block_sum(t);
  if (threadIdx.x == 0) {
    const double h = 0.5 * (double)*g;
    out[0] = h * (acc[0] - t);
    out[1] = h * (acc[1] - acc[2]);
  }
}

}  // namespace knll
}  // namespace rfp
