// profile.h — optional per-kernel-class timing with CUDA events.
//
// When enabled on a handle (curfpProfileEnable), every kernel launch of the
// library is bracketed by two events on the handle's stream and attributed
// to a kernel class together with its algorithmic work (flops and/or bytes).
// curfpProfileRead synchronises the stream and returns, per class, the summed
// device time, work and launch count.  Disabled (the default), the cost is
// one branch per launch.
#pragma once
#include <cuda_runtime.h>

#include <vector>

namespace rfp {

enum KClass : int {
  K_SGEMM = 0,    // SIMT FP32 GEMM / SYRK / TRMM / TRSM-leaf multiply
  K_TC_GEMM = 1,  // split-BF16 tcgen05 contraction
  K_TC_STAGE = 2, // row scales + digit planes of the tensor-core operands
  K_POTRF = 3,    // diagonal Cholesky tiles
  K_TRTRI = 4,    // triangular inverses
  K_LAUUM = 5,    // L^T L tiles
  K_PACK = 6,     // strttf / stfttr
  K_DIAG = 7,     // diagonal index / shift / small helpers
  K_SYMM64 = 8,   // FP64-accumulated RFP symmetric multiply (residuals)
  K_TRSV = 9,     // wavefront triangular solves
  K_NORM = 10,    // RFP norms and condition-estimator vector kernels
  K_NCLASS = 11
};

struct ProfRec {
  int cls;
  double flops, bytes;
  cudaEvent_t e0, e1;
  int m = 0, n = 0, k = 0, tiles = 0;  // shape of a contraction launch (0: not given)
};

struct Profiler {
  bool on = false;
  std::vector<ProfRec> recs;
  std::vector<cudaEvent_t> pool;
  size_t used = 0;

  cudaEvent_t ev() {
    if (used == pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      pool.push_back(e);
    }
    return pool[used++];
  }
  void reset() {
    recs.clear();
    used = 0;
  }
  ~Profiler() {
    for (auto e : pool) cudaEventDestroy(e);
  }
};

// RAII bracket around one launch.
struct ProfScope {
  Profiler* p;
  cudaStream_t s;
  int idx;
  ProfScope(Profiler& prof, cudaStream_t st, int cls, double flops, double bytes)
      : p(&prof), s(st), idx(-1) {
    if (!prof.on) return;
    ProfRec r{cls, flops, bytes, prof.ev(), prof.ev()};
    cudaEventRecord(r.e0, st);
    idx = (int)prof.recs.size();
    prof.recs.push_back(r);
  }
  ~ProfScope() {
    if (idx >= 0) cudaEventRecord(p->recs[idx].e1, s);
  }
  // Shape of the bracketed contraction: output rows and columns summed over
  // its tasks, depth, and output tiles.
  void shape(int m, int n, int k, int tiles) {
    if (idx < 0) return;
    ProfRec& r = p->recs[idx];
    r.m = m; r.n = n; r.k = k; r.tiles = tiles;
  }
};

}  // namespace rfp
