// context.h — the library handle (struct curfpContext) and the CUDA executor.
//
// The reference context wraps a cuBLAS and a cuSOLVER handle
// (src/curfp_internal.h:11-14); this one holds what the native kernels need:
// the stream, the device, one device-side info word (pivot failures, also used
// as the abort flag that makes later kernels of a failed factorization return
// immediately), a kernel error word, grow-only stream-ordered workspaces and
// the staging buffers of the split-BF16 path.  Workspaces come from the
// handle's own memory pool (created with the handle, kept across calls), so
// the device's default pool and its settings are left to the caller.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "engine.h"
#include "profile.h"

struct curfpContext {
  cudaStream_t stream = nullptr;
  int device = 0;
  cudaMemPool_t pool = nullptr;  // the handle's workspace pool
  int math = 1;            // contraction arithmetic of the drop-in routines (curfpSetMathMode)
  long long wait_launches = 0;  // kernels with bounded waits launched (status.cuh)
  int* d_info = nullptr;   // [0]: INT_MAX = no pivot failure; [1]: kernel error code
  void* ws = nullptr;      // TRSM diagonal-block inverses and other scratch
  size_t ws_bytes = 0;
  void* stage = nullptr;   // split-BF16 operand staging (first operand)
  size_t stage_bytes = 0;
  void* stage2 = nullptr;  // split-BF16 operand staging (second operand)
  size_t stage2_bytes = 0;
  void* ws2 = nullptr;     // refinement scratch (saved RHS, residual)
  size_t ws2_bytes = 0;
  void* ws3 = nullptr;     // FP64 accumulator of split symmetric multiplies
  size_t ws3_bytes = 0;
  long long launches = 0;  // kernels launched through this handle
  rfp::Profiler prof;      // optional per-class event timing
  void* tsv = nullptr;     // wavefront solve flags / tickets
  size_t tsv_bytes = 0;
  void* wsg = nullptr;     // adjoint scratch (solve adjoint n x 2nrhs, NLL gradient)
  size_t wsg_bytes = 0;
  cudaStream_t copy_stream = nullptr;  // host-input factorization: the overlapped copy
  cudaEvent_t ev_start = nullptr, ev_rest = nullptr;
};

namespace rfp {

// The CUDA executor for FP32 (SIMT and split-BF16 tensor-core contractions)
// and FP64 (SIMT DFMA) element types.
template <typename T>
class CudaExecT : public ExecT<T> {
 public:
  explicit CudaExecT(curfpContext* ctx, const int* abort_flag = nullptr)
      : ctx_(ctx), abort_(abort_flag) {}
  int gemm(const GemmProbT<T>* p, int count) override;
  int potrf_tile(ViewT<T> L, int n, int info_base) override;
  // 128-row tiles.  (A 256-row FP32 tile, one CTA of 512 threads, measured
  // 157 us per tile against 2 x 57 us for two 128-row tiles: it moves the
  // 128^3 trailing update of the level above from a multi-CTA SYRK into one
  // CTA.)
  int potrf_tile_rows() const override { return kPotrfTile; }
  int trtri_blocks(ViewT<T> L, int n, int nb, T* W) override;
  int trtri_tile(ViewT<T> L, int n) override;
  int lauum_tile(ViewT<T> L, int n) override;
  T* workspace(size_t count) override;
  int inplace_rows() const override { return 64; }
  int gemm_shared(ViewT<T> X, int rows, int k, const SharedTaskT<T>* t, int count,
                  int math) override;
  int gemm_pair(ViewT<T> X, ViewT<T> Y, int rows, int k, const SharedTaskT<T>* t, int count,
                int math) override;
  int trsm_wave(ViewT<T> L, int n, ViewT<T> B, int m, T alpha, const T* W) override;
  int potrf_adj_tile(ViewT<T> L, ViewT<T> G, int n) override;
  // When set, work after the first diagonal block waits for this event.
  int after_first_block() override {
    if (!rest_ready) return 0;
    return cudaStreamWaitEvent(ctx_->stream, rest_ready, 0) == cudaSuccess ? 0 : 4;
  }
  cudaEvent_t rest_ready = nullptr;

 protected:
  curfpContext* ctx_;
  const int* abort_;
};
using CudaExec = CudaExecT<float>;
using CudaExecD = CudaExecT<double>;

// Grow a stream-ordered buffer to at least `bytes`; returns nullptr on failure.
void* grow_buffer(curfpContext* ctx, void** buf, size_t* cur, size_t bytes);

// Split-BF16 tensor-core contraction (tc_engine.cu).  C_t := alpha_t *
// A[a_row0:+m, :] B[b_row0:+n, :]^T + beta_t C_t with A (arows x k) and B
// (brows x k) FP32 views; B.p == nullptr means B is A.
int tc_contract(curfpContext* ctx, const int* abort_flag, View A, int arows, View B,
                int brows, int k, const SharedTask* tasks, int count);
// The same with triangular operand masks (0 full, 1 keep column <= row,
// 2 keep column >= row, columns counted over the whole k range): masked
// elements are staged as zeros and never read.  B.p must be set.
int tc_contract_masked(curfpContext* ctx, const int* abort_flag, View A, int arows, int amask,
                       View B, int brows, int bmask, int k, const SharedTask* tasks,
                       int count);
// The wavefront solve with a caller-provided flag buffer of sync_words words
// (cleared here on the stream); no allocation.
int launch_trsm_wave_fixed(curfpContext* ctx, const int* abort_flag, View L, int n, View B,
                           int m, float alpha, const float* W, int* sync, size_t sync_words);
// Bounded-wait self-test of the wavefront solve (exec_cuda.cu): launches a
// solve whose first block row never runs; its dependents time out (~2 s) and
// set error code 5 in ctx->d_info[1].
int wave_wait_selftest(curfpContext* ctx);
// Whether a contraction of this size goes to the tensor-core path.
bool tc_worthwhile(int m, int n, int k);
// Whether a contraction with operands of at most `rows` rows stages its
// whole k range at once (no k slabs): every operand is then read before the
// product writes C, so C may alias an operand.
bool tc_single_slab(int rows, int k);

}  // namespace rfp
