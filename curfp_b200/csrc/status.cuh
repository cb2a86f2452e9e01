// status.cuh — the handle's two device status words and how entry points
// report them.
//
// d_info[0] holds the first failing pivot of a factorization (INT_MAX: none);
// d_info[1] is the kernel error word: a kernel whose bounded wait (a
// wavefront flag, an mbarrier of the tensor-core pipeline) ran out sets it to
// a nonzero code and returns.  Entry points that launched such a kernel read
// the word back before they return, turn a nonzero code into
// CURFP_STATUS_EXECUTION_FAILED and clear it, so that no later call inherits
// it.  Entry points that launched none stay asynchronous.
#pragma once
#include <cuda_runtime.h>

#include <climits>

#include "../../include/curfp.h"
#include "context.h"

namespace rfp {
namespace status {

namespace {
__global__ void set_words(int* p, int v0, int v1) {
  p[0] = v0;
  p[1] = v1;
}
__global__ void clear_word(int* p) { p[0] = 0; }
}  // namespace

// Reset both words (no pivot failure, no kernel error) on the stream.
inline bool reset(curfpContext* h) {
  set_words<<<1, 1, 0, h->stream>>>(h->d_info, INT_MAX, 0);
  ++h->launches;
  return cudaGetLastError() == cudaSuccess;
}

// Synchronise the stream and read both words.
inline bool read(curfpContext* h, int* info, int* err) {
  int w[2] = {0, 0};
  if (cudaMemcpyAsync(w, h->d_info, 2 * sizeof(int), cudaMemcpyDeviceToHost, h->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  *info = w[0];
  *err = w[1];
  return true;
}

// Brackets an entry point.  When a kernel with bounded waits ran since
// construction, finish(rc) synchronises, reads the error word and clears a
// nonzero word; it returns rc when that is nonzero (the planner's own
// failure), else 5 (execution failed) for a nonzero word, else 0.
struct WaitCheck {
  curfpContext* h;
  long long w0;
  int err = 0;  // the error word as read by finish()
  explicit WaitCheck(curfpContext* ctx) : h(ctx), w0(ctx->wait_launches) {}
  int finish(int rc) {
    if (h->wait_launches == w0) return rc;
    int info = 0;
    if (!read(h, &info, &err)) return rc ? rc : 4;
    if (err == 0) return rc;
    clear_word<<<1, 1, 0, h->stream>>>(h->d_info + 1);
    ++h->launches;
    return rc ? rc : 5;
  }
};

// Runs an entry point's body (a callable returning curfpStatus_t) under a
// WaitCheck.
template <class F>
inline curfpStatus_t checked(curfpContext* h, F&& body) {
  WaitCheck wc(h);
  const curfpStatus_t st = body();
  const int rc = wc.finish(st == CURFP_STATUS_SUCCESS ? 0 : 1);
  if (st != CURFP_STATUS_SUCCESS) return st;
  return rc == 0 ? CURFP_STATUS_SUCCESS : CURFP_STATUS_EXECUTION_FAILED;
}

}  // namespace status
}  // namespace rfp
