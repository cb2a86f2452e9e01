// noalloc.cu — curfpSpftrsNoAlloc: the RFP solve without any device
// allocation on the call path.
//
// Some callers cannot let a library allocate device memory while they run:
// processes whose GPU memory is entirely owned by another allocator (a
// framework's caching allocator that reserved the device), and latency-
// critical loops where a cudaMalloc -- which may synchronise the device or
// fail under memory pressure -- is not acceptable.  curfpSpftrs allocates its
// scratch (the inverted 64 x 64 diagonal blocks used by the blocked solve and
// the wavefront solve's ticket/flag words) from a stream-ordered pool; this
// variant takes that scratch from one file-scope device array instead.
//
// Scratch: g_solve_scratch holds kInvFloats floats of diagonal-block inverses
// followed by kSyncWords 32-bit words of solve flags (4 MiB + 4 KiB), which
// every GPU that loads the library keeps until the process exits.  Limits:
// n <= 16384 (so each half is <= 8192 rows) and nrhs <= 512.  Every call
// shares the array and leaves its contents behind; the flag words are
// cleared at the start of each solve.  Calls that overlap on the GPU (on
// different streams, or from different handles) race on the array.
//
// The device address of the array is fetched once per device with
// cudaGetSymbolAddress on the first call with a handle of that device (the
// handle's device is made current for the lookup); make that first call
// before any stream capture.  Each call synchronises the handle's stream
// once, to read the kernel error word: a wavefront wait that ran out is
// reported as CURFP_STATUS_EXECUTION_FAILED.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/curfp.h"
#include "context.h"
#include "status.cuh"

namespace {

constexpr int kNoAllocMaxN = 16384;
constexpr int kNoAllocMaxRhs = 512;
constexpr size_t kHalfMax = kNoAllocMaxN / 2;
constexpr size_t kInvFloats = (kHalfMax / rfp::kTrsmLeaf) * rfp::kInvStride;  // [W | M] records of one half
constexpr size_t kWaveRows = 64;  // row / column block of the wavefront solve
constexpr size_t kSyncWords = 1 + (kHalfMax / kWaveRows) * (kNoAllocMaxRhs / kWaveRows);

static __device__ __align__(256) float g_solve_scratch[kInvFloats + kSyncWords + 64];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
float* g_addr[kMaxDevices] = {};

// Device address of g_solve_scratch on device `dev` (the handle's device,
// whatever device is current in the calling thread); nullptr on error.  The
// lookup runs with `dev` current and restores the caller's device.
float* scratch_address(int dev) {
  if (dev < 0 || dev >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    if (prev != dev && cudaSetDevice(dev) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_solve_scratch);
    if (prev != dev) cudaSetDevice(prev);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    g_addr[dev] = static_cast<float*>(p);
  }
  return g_addr[dev];
}

// The CUDA executor with its two allocating primitives redirected to the
// static array.
class NoAllocExec : public rfp::CudaExec {
 public:
  NoAllocExec(curfpContext* ctx, float* scratch) : rfp::CudaExec(ctx), scratch_(scratch) {}

  float* workspace(size_t nfloats) override {
    return nfloats <= kInvFloats ? scratch_ : nullptr;
  }

  int trsm_wave(rfp::View L, int n, rfp::View B, int m, float alpha,
                const float* W) override {
    int* sync = reinterpret_cast<int*>(scratch_ + kInvFloats);
    return rfp::launch_trsm_wave_fixed(ctx_, abort_, L, n, B, m, alpha, W, sync, kSyncWords);
  }

 private:
  float* scratch_;
};

}  // namespace

extern "C" curfpStatus_t curfpSpftrsNoAlloc(curfpHandle_t handle, curfpOperation_t transr,
                                            curfpFillMode_t uplo, int n, int nrhs,
                                            const float* A, float* B, int ldb) {
  if (!handle) return CURFP_STATUS_NOT_INITIALIZED;
  if (n < 0 || nrhs < 0 || ldb < 1) return CURFP_STATUS_INVALID_VALUE;
  if (n == 0 || nrhs == 0) return CURFP_STATUS_SUCCESS;
  if (n > kNoAllocMaxN || nrhs > kNoAllocMaxRhs) return CURFP_STATUS_INVALID_VALUE;
  const int lower = uplo == CURFP_FILL_MODE_LOWER;
  const int n1 = (n & 1) ? (lower ? n - n / 2 : n / 2) : n / 2;
  const int nmax = n1 > n - n1 ? n1 : n - n1;
  if (ldb < nmax) return CURFP_STATUS_INVALID_VALUE;
  float* scratch = scratch_address(handle->device);
  if (!scratch) return CURFP_STATUS_EXECUTION_FAILED;
  NoAllocExec ex(handle, scratch);
  // A wavefront wait that runs out leaves B partly solved and sets the
  // handle's kernel error word; the word is read back (one stream
  // synchronisation, no allocation) and reported as EXECUTION_FAILED.
  rfp::status::WaitCheck wc(handle);
  const int rc = wc.finish(rfp::plan::spftrs(ex, transr == CURFP_OP_T, lower, n, nrhs, A, B, ldb));
  switch (rc) {
    case 0: return CURFP_STATUS_SUCCESS;
    case 3: return CURFP_STATUS_INVALID_VALUE;
    case 2: return CURFP_STATUS_ALLOC_FAILED;
    default: return CURFP_STATUS_EXECUTION_FAILED;
  }
}
