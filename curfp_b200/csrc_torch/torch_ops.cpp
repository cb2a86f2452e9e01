// torch_ops.cpp — the torch extension over the C ABI (include/curfp.h).
//
// Registers the RFP routines and their adjoints as torch operators
// (torch.ops.curfp_b200.*).  Each operator checks its tensors (CUDA,
// float32 / float64 where stated, contiguous), switches to the tensors'
// device, binds that device's library handle to torch's current CUDA stream
// and calls the entry point; a non-success status raises
// RuntimeError("curfp error: status=N") as the reference's extension does
// (curfp/_ext.cpp:21-25).  Tensors stay tensors here: no raw pointers cross
// into Python.  The differentiation form (curfp_b200.autograd) calls these.
#include <ATen/cuda/CUDAContext.h>
#include <c10/cuda/CUDAGuard.h>
#include <torch/library.h>

#include <mutex>

#include "curfp.h"

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
curfpHandle_t g_handles[kMaxDevices] = {};

// The device's handle (created on first use with that device current),
// bound to torch's current stream on that device.
curfpHandle_t handle_for(const at::Tensor& t) {
  const int dev = t.get_device();
  TORCH_CHECK(dev >= 0 && dev < kMaxDevices, "curfp: unsupported device index ", dev);
  curfpHandle_t h;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_handles[dev]) {
      const curfpStatus_t st = curfpCreate(&g_handles[dev]);
      TORCH_CHECK(st == CURFP_STATUS_SUCCESS, "curfp error: status=", (int)st);
    }
    h = g_handles[dev];
  }
  const curfpStatus_t st = curfpSetStream(h, at::cuda::getCurrentCUDAStream(dev).stream());
  TORCH_CHECK(st == CURFP_STATUS_SUCCESS, "curfp error: status=", (int)st);
  return h;
}

void check_status(curfpStatus_t st) {
  TORCH_CHECK(st == CURFP_STATUS_SUCCESS, "curfp error: status=", (int)st);
}

void check_f32(const at::Tensor& t, const char* name) {
  TORCH_CHECK(t.is_cuda(), name, " must be a CUDA tensor");
  TORCH_CHECK(t.scalar_type() == at::kFloat, name, " must be float32");
  TORCH_CHECK(t.is_contiguous(), name, " must be contiguous");
}

inline curfpOperation_t op(int64_t v) { return v ? CURFP_OP_T : CURFP_OP_N; }
inline curfpFillMode_t fill(int64_t v) { return v ? CURFP_FILL_MODE_UPPER : CURFP_FILL_MODE_LOWER; }
inline curfpMath_t math(int64_t v) { return v ? CURFP_MATH_SPLIT_BF16 : CURFP_MATH_FP32; }

// C := alpha op(A) op(A)^T + beta C (curfpSsfrkEx).
void ssfrk(const at::Tensor& A, const at::Tensor& C, double alpha, double beta, int64_t transr,
           int64_t uplo, int64_t trans, int64_t n, int64_t k, int64_t lda, int64_t m) {
  check_f32(A, "A");
  check_f32(C, "C");
  c10::cuda::CUDAGuard g(C.device());
  const float a = (float)alpha, b = (float)beta;
  check_status(curfpSsfrkEx(handle_for(C), op(transr), fill(uplo), op(trans), (int)n, (int)k, &a,
                            A.data_ptr<float>(), (int)lda, &b, C.data_ptr<float>(), math(m)));
}

// C := C + value I (curfpSaddToDiagonal).
void add_to_diagonal(const at::Tensor& C, double value, int64_t transr, int64_t uplo, int64_t n) {
  check_f32(C, "C");
  c10::cuda::CUDAGuard g(C.device());
  check_status(curfpSaddToDiagonal(handle_for(C), op(transr), fill(uplo), (int)n, (float)value,
                                   C.data_ptr<float>()));
}

// In-place Cholesky (curfpSpftrfEx); returns info.
int64_t spftrf(const at::Tensor& C, int64_t transr, int64_t uplo, int64_t n, int64_t m) {
  check_f32(C, "C");
  c10::cuda::CUDAGuard g(C.device());
  int info = 0;
  check_status(curfpSpftrfEx(handle_for(C), op(transr), fill(uplo), (int)n, C.data_ptr<float>(),
                             &info, math(m)));
  return info;
}

// B (column-major n x nrhs, ld ldb) := A^-1 B with the factor L (curfpSpftrs).
void spftrs(const at::Tensor& L, const at::Tensor& B, int64_t transr, int64_t uplo, int64_t n,
            int64_t nrhs, int64_t ldb) {
  check_f32(L, "L");
  check_f32(B, "B");
  c10::cuda::CUDAGuard g(B.device());
  check_status(curfpSpftrs(handle_for(B), op(transr), fill(uplo), (int)n, (int)nrhs,
                           L.data_ptr<float>(), B.data_ptr<float>(), (int)ldb));
}

// Solve with FP64-residual refinement (curfpSpftrsRefine); returns the
// number of corrections applied.
int64_t spftrs_refine(const at::Tensor& A, const at::Tensor& F, const at::Tensor& B, int64_t transr,
                      int64_t uplo, int64_t n, int64_t nrhs, int64_t ldb, int64_t max_iter) {
  check_f32(A, "A");
  check_f32(F, "F");
  check_f32(B, "B");
  c10::cuda::CUDAGuard g(B.device());
  int iters = 0;
  check_status(curfpSpftrsRefine(handle_for(B), op(transr), fill(uplo), (int)n, (int)nrhs,
                                 A.data_ptr<float>(), F.data_ptr<float>(), B.data_ptr<float>(),
                                 (int)ldb, (int)max_iter, &iters));
  return iters;
}

// Abar := alpha (tril(Cbar) + tril(Cbar)^T) op(A) (curfpSsfrkBackward).
void ssfrk_backward(const at::Tensor& A, const at::Tensor& Cbar, const at::Tensor& Abar, double alpha,
                    int64_t transr, int64_t uplo, int64_t trans, int64_t n, int64_t k,
                    int64_t lda) {
  check_f32(A, "A");
  check_f32(Cbar, "Cbar");
  check_f32(Abar, "Abar");
  c10::cuda::CUDAGuard g(Abar.device());
  const float a = (float)alpha;
  check_status(curfpSsfrkBackward(handle_for(Abar), op(transr), fill(uplo), op(trans), (int)n,
                                  (int)k, &a, A.data_ptr<float>(), (int)lda,
                                  Cbar.data_ptr<float>(), Abar.data_ptr<float>(), (int)lda));
}

// Cotangent of A's stored elements from that of its factor
// (curfpSpftrfBackward, in RFP layout; Abar may be Lbar itself).
void spftrf_backward(const at::Tensor& L, const at::Tensor& Lbar, const at::Tensor& Abar,
                     int64_t transr, int64_t uplo, int64_t n, int64_t m) {
  check_f32(L, "L");
  check_f32(Lbar, "Lbar");
  check_f32(Abar, "Abar");
  c10::cuda::CUDAGuard g(Abar.device());
  check_status(curfpSpftrfBackward(handle_for(Abar), op(transr), fill(uplo), (int)n,
                                   L.data_ptr<float>(), Lbar.data_ptr<float>(),
                                   Abar.data_ptr<float>(), math(m)));
}

// Solve adjoint (curfpSpftrsBackward): Bbar holds Xbar on entry (column-major
// n x nrhs) and A^-1 Xbar on exit; Lbar (RFP) receives the factor's cotangent
// unless it is empty.
void spftrs_backward(const at::Tensor& L, const at::Tensor& X, const at::Tensor& Bbar, const at::Tensor& Lbar,
                     int64_t transr, int64_t uplo, int64_t n, int64_t nrhs) {
  check_f32(L, "L");
  check_f32(X, "X");
  check_f32(Bbar, "Bbar");
  const bool want_l = Lbar.numel() > 0;
  if (want_l) check_f32(Lbar, "Lbar");
  c10::cuda::CUDAGuard g(Bbar.device());
  float* bb = Bbar.data_ptr<float>();
  check_status(curfpSpftrsBackward(handle_for(Bbar), op(transr), fill(uplo), (int)n, (int)nrhs,
                                   L.data_ptr<float>(), X.data_ptr<float>(), (int)n, bb, (int)n,
                                   bb, (int)n, want_l ? Lbar.data_ptr<float>() : nullptr));
}

// Fused GP NLL gradient (curfpSgpnllBackward); sums (float64, 2) receives
// (sbar, sigma2bar).
void gpnll_backward(const at::Tensor& L, const at::Tensor& X, const at::Tensor& alpha,
                    const at::Tensor& gscale, const at::Tensor& Xbar, const at::Tensor& sums, double s,
                    int64_t transr, int64_t uplo, int64_t n, int64_t d, int64_t m) {
  check_f32(L, "L");
  check_f32(X, "X");
  check_f32(alpha, "alpha");
  check_f32(gscale, "g");
  check_f32(Xbar, "Xbar");
  TORCH_CHECK(sums.is_cuda() && sums.scalar_type() == at::kDouble && sums.numel() >= 2,
              "sums must be a float64 CUDA tensor of 2 elements");
  c10::cuda::CUDAGuard g(Xbar.device());
  const int ld = d > 1 ? (int)d : 1;
  check_status(curfpSgpnllBackward(handle_for(Xbar), op(transr), fill(uplo), (int)n, (int)d,
                                   (float)s, L.data_ptr<float>(), X.data_ptr<float>(), ld,
                                   alpha.data_ptr<float>(), gscale.data_ptr<float>(),
                                   Xbar.data_ptr<float>(), ld, sums.data_ptr<double>(), math(m)));
}

}  // namespace

TORCH_LIBRARY(curfp_b200, m) {
  m.def("ssfrk(Tensor A, Tensor(a!) C, float alpha, float beta, int transr, int uplo, "
        "int trans, int n, int k, int lda, int math) -> ()");
  m.def("add_to_diagonal(Tensor(a!) C, float value, int transr, int uplo, int n) -> ()");
  m.def("spftrf(Tensor(a!) C, int transr, int uplo, int n, int math) -> int");
  m.def("spftrs(Tensor L, Tensor(a!) B, int transr, int uplo, int n, int nrhs, int ldb) -> ()");
  m.def("spftrs_refine(Tensor A, Tensor F, Tensor(a!) B, int transr, int uplo, int n, "
        "int nrhs, int ldb, int max_iter) -> int");
  m.def("ssfrk_backward(Tensor A, Tensor Cbar, Tensor(a!) Abar, float alpha, int transr, "
        "int uplo, int trans, int n, int k, int lda) -> ()");
  m.def("spftrf_backward(Tensor L, Tensor Lbar, Tensor(a!) Abar, int transr, int uplo, int n, "
        "int math) -> ()");
  m.def("spftrs_backward(Tensor L, Tensor X, Tensor(a!) Bbar, Tensor(b!) Lbar, int transr, "
        "int uplo, int n, int nrhs) -> ()");
  m.def("gpnll_backward(Tensor L, Tensor X, Tensor alpha, Tensor g, Tensor(a!) Xbar, "
        "Tensor(b!) sums, float s, int transr, int uplo, int n, int d, int math) -> ()");
}

TORCH_LIBRARY_IMPL(curfp_b200, CUDA, m) {
  m.impl("ssfrk", &ssfrk);
  m.impl("add_to_diagonal", &add_to_diagonal);
  m.impl("spftrf", &spftrf);
  m.impl("spftrs", &spftrs);
  m.impl("spftrs_refine", &spftrs_refine);
  m.impl("ssfrk_backward", &ssfrk_backward);
  m.impl("spftrf_backward", &spftrf_backward);
  m.impl("spftrs_backward", &spftrs_backward);
  m.impl("gpnll_backward", &gpnll_backward);
}
