// context.h — the library handle (struct curfpContext) and the CUDA executor.
//
// The reference context wraps a cuBLAS and a cuSOLVER handle
// (src/curfp_internal.h:11-14); this one holds what the native kernels need:
// the stream, the device, one device-side info word (pivot failures, also used
// as the abort flag that makes later kernels of a failed factorization return
// immediately), a grow-only stream-ordered workspace and the staging buffers
// of the split-BF16 path.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "engine.h"

struct curfpContext {
  cudaStream_t stream = nullptr;
  int device = 0;
  int* d_info = nullptr;   // INT_MAX = no failure
  void* ws = nullptr;      // TRSM diagonal-block inverses and other scratch
  size_t ws_bytes = 0;
  void* stage = nullptr;   // split-BF16 operand staging
  size_t stage_bytes = 0;
};

namespace rfp {

class CudaExec : public Exec {
 public:
  explicit CudaExec(curfpContext* ctx, const int* abort_flag = nullptr)
      : ctx_(ctx), abort_(abort_flag) {}
  int gemm(const GemmProb* p, int count) override;
  int potrf_tile(View L, int n, int info_base) override;
  int trtri_blocks(View L, int n, int nb, float* W) override;
  int trtri_tile(View L, int n) override;
  int lauum_tile(View L, int n) override;
  float* workspace(size_t nfloats) override;
  int inplace_rows() const override { return 64; }

 private:
  curfpContext* ctx_;
  const int* abort_;
};

// Grow a stream-ordered buffer to at least `bytes`; returns nullptr on failure.
void* grow_buffer(curfpContext* ctx, void** buf, size_t* cur, size_t bytes);

}  // namespace rfp
