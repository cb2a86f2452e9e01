// exec_bounds.cpp — TEST-ONLY dry-run executor: runs the library's planner
// (curfp_b200/csrc/plan.cpp) without arithmetic and checks that every element
// range a primitive would read or write lies inside one caller buffer (the
// RFP array, the right-hand sides, the operand matrix) or a workspace the
// planner asked for.  The sizes it is meant for (n up to 131072, RFP arrays
// of 8.6e9 elements) are far beyond what a computing CPU executor can run, so
// buffers are virtual: address ranges in a fake address space, never
// dereferenced.
//
// For an affine view element (i, j) -> p + i*rs + j*cs, the extreme
// addresses over a convex index region are taken at its vertices, so a
// rectangle is checked at its four corners and a masked triangle (the
// kernels read only elements with j <= i, or j >= i) at the corners of the
// triangle clipped to the rectangle.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "engine.h"

using namespace rfp;

namespace {

struct Range {
  uintptr_t lo, hi;  // [lo, hi) in bytes
  const char* name;
};

class BoundsExec : public Exec {
 public:
  std::vector<Range> bufs;
  long checks = 0, violations = 0, calls = 0;
  char first[256] = {0};
  uintptr_t next = (uintptr_t)1 << 44;  // fake address space, 4 KiB gaps between buffers

  float* add(const char* name, size_t nfloats) {
    uintptr_t b = next;
    bufs.push_back({b, b + nfloats * sizeof(float), name});
    next = (b + nfloats * sizeof(float) + 8192) & ~(uintptr_t)4095;
    return reinterpret_cast<float*>(b);
  }

  // tri: 0 full, 1 keep j <= i, 2 keep j >= i, 3 keep j > i (checked as its
  // superset 2) (row i, column j of the view)
  void check(const char* what, View v, int64_t rows, int64_t cols, int tri) {
    ++checks;
    if (tri == 3) tri = 2;
    if (rows <= 0 || cols <= 0) return;
    int64_t vi[4], vj[4];
    int nv = 0;
    const int64_t r1 = rows - 1, c1 = cols - 1;
    if (tri == 0) {
      vi[0] = 0; vj[0] = 0; vi[1] = r1; vj[1] = 0; vi[2] = 0; vj[2] = c1; vi[3] = r1; vj[3] = c1;
      nv = 4;
    } else if (tri == 1) {  // {0 <= j <= i < rows, j < cols}
      const int64_t d = std::min(r1, c1);
      vi[0] = 0; vj[0] = 0; vi[1] = r1; vj[1] = 0; vi[2] = r1; vj[2] = d; vi[3] = d; vj[3] = d;
      nv = 4;
    } else {  // {0 <= i <= j < cols, i < rows}
      const int64_t d = std::min(r1, c1);
      vi[0] = 0; vj[0] = 0; vi[1] = 0; vj[1] = c1; vi[2] = d; vj[2] = c1; vi[3] = d; vj[3] = d;
      nv = 4;
    }
    const uintptr_t base = reinterpret_cast<uintptr_t>(v.p);
    intptr_t lo = INTPTR_MAX, hi = INTPTR_MIN;
    for (int t = 0; t < nv; ++t) {
      const intptr_t a = (intptr_t)base + (intptr_t)((vi[t] * v.rs + vj[t] * v.cs) * 4);
      lo = std::min(lo, a);
      hi = std::max(hi, a + 4);
    }
    for (const Range& r : bufs)
      if ((uintptr_t)lo >= r.lo && (uintptr_t)hi <= r.hi) return;
    if (violations++ == 0)
      snprintf(first, sizeof first,
               "%s: %lld x %lld tri %d, rs %lld cs %lld, bytes [%#llx, %#llx) outside every buffer",
               what, (long long)rows, (long long)cols, tri, (long long)v.rs, (long long)v.cs,
               (unsigned long long)lo, (unsigned long long)hi);
  }

  int gemm(const GemmProb* p, int count) override {
    if (count > kMaxBatch) return 3;
    ++calls;
    for (int t = 0; t < count; ++t) {
      const GemmProb& g = p[t];
      if (g.m <= 0 || g.n <= 0) continue;
      if (g.inplace && g.m > inplace_rows()) return 3;
      if (g.c_lower && g.m != g.n) return 3;
      check("gemm A", g.A, g.m, g.k, g.a_tri);
      check("gemm B", g.B, g.k, g.n, g.b_tri);
      if (g.k2 > 0) {
        check("gemm A2", g.A2, g.m, g.k2, g.a2_tri);
        check("gemm B2", g.B2, g.k2, g.n, g.b2_tri);
      }
      check("gemm C", g.C, g.m, g.n, g.c_lower ? 1 : 0);
    }
    return 0;
  }
  int gemm_shared(View X, int rows, int k, const SharedTask* t, int count, int math) override {
    (void)math;
    if (count > kMaxBatch) return 3;
    ++calls;
    check("shared X", X, rows, k, 0);
    for (int i = 0; i < count; ++i) {
      if (t[i].m <= 0 || t[i].n <= 0) continue;
      if (t[i].a_row0 + t[i].m > rows || t[i].b_row0 + t[i].n > rows) return 3;
      if (t[i].c_lower && t[i].m != t[i].n) return 3;
      check("shared C", t[i].C, t[i].m, t[i].n, t[i].c_lower ? 1 : 0);
    }
    return 0;
  }
  int potrf_tile(View L, int n, int info_base) override {
    (void)info_base;
    ++calls;
    if (n > kPotrfTile) return 3;
    check("potrf_tile", L, n, n, 1);
    return 0;
  }
  int trtri_blocks(View L, int n, int nb, float* W) override {
    ++calls;
    check("trtri_blocks L", L, n, n, 1);
    const int nblk = (n + nb - 1) / nb;
    check("trtri_blocks W", View{W, 1, kInvStride}, kInvStride, nblk, 0);
    return 0;
  }
  int trtri_tile(View L, int n) override {
    ++calls;
    if (n > kTriTile) return 3;
    check("trtri_tile", L, n, n, 1);
    return 0;
  }
  int lauum_tile(View L, int n) override {
    ++calls;
    if (n > kTriTile) return 3;
    check("lauum_tile", L, n, n, 1);
    return 0;
  }
  float* workspace(size_t nfloats) override { return add("workspace", nfloats); }
  int inplace_rows() const override { return 64; }
  // The CUDA executor's wavefront solve: L lower (n x n), B (n x m), W one
  // record per 64-row block.
  int trsm_wave(View L, int n, View B, int m, float alpha, const float* W) override {
    (void)alpha;
    ++calls;
    check("trsm_wave L", L, n, n, 1);
    check("trsm_wave B", B, n, m, 0);
    const int nblk = (n + kTrsmLeaf - 1) / kTrsmLeaf;
    check("trsm_wave W", View{const_cast<float*>(W), 1, kInvStride}, kInvStride, nblk, 0);
    return 0;
  }
  int potrf_adj_tile(View L, View G, int n) override {
    ++calls;
    if (n > kAdjTile) return 3;
    check("potrf_adj_tile L", L, n, n, 1);
    check("potrf_adj_tile G", G, n, n, 1);
    return 0;
  }
};

}  // namespace

extern "C" {

// Dry run of one RFP routine at order n (transr 0/1 = N/T, lower 1/0 = L/U):
//   op 0 ssfrk (trans = T, A row-major n x k, lda = k)   op 1 spftrf
//   op 2 spftrs (k right-hand sides, ldb = n)            op 3 spftri
//   op 4 L X = B and op 5 L^T X = B on the RFP factor (B n x k row-major)
//   op 6 in-place RFP triangular inverse
//   op 7 Cholesky adjoint (a second RFP array holds the cotangent)
//   op 8 ssfr2k (trans = T, A and B row-major n x k)
// Returns the planner's status; out[0..2] = calls, range checks, violations.
// msg (256 bytes) receives the first violation.
int hs_bounds(int op, int transr, int lower, int n, int k, int math, int64_t* out, char* msg) {
  BoundsExec ex;
  const size_t nt = (size_t)n * (n + 1) / 2;
  float* C = ex.add("rfp", nt);
  int rc = -100;
  switch (op) {
    case 0: {
      float* A = ex.add("A", (size_t)n * k);
      rc = plan::ssfrk(ex, transr, lower, 1, n, k, 1.0f, A, k, 0.0f, C, math);
      break;
    }
    case 1: rc = plan::spftrf(ex, transr, lower, n, C, math); break;
    case 2: {
      float* B = ex.add("B", (size_t)n * k);
      rc = plan::spftrs(ex, transr, lower, n, k, C, B, n);
      break;
    }
    case 3: rc = plan::spftri(ex, transr, lower, n, C); break;
    case 4:
    case 5: {
      float* B = ex.add("B", (size_t)n * k);
      rc = plan::rfp_trsm(ex, transr, lower, n, C, op - 4, View{B, k, 1}, k, 1.0f, math);
      break;
    }
    case 6: rc = plan::rfp_trtri(ex, transr, lower, n, C, math); break;
    case 7: {
      float* G = ex.add("cotangent", nt);
      rc = plan::spftrf_adjoint(ex, transr, lower, n, C, G, math);
      break;
    }
    case 8: {
      float* A = ex.add("A", (size_t)n * k);
      float* B = ex.add("B", (size_t)n * k);
      rc = plan::ssfr2k(ex, transr, lower, 1, n, k, 1.0f, A, k, B, k, 0.0f, C, math);
      break;
    }
    default: break;
  }
  out[0] = ex.calls;
  out[1] = ex.checks;
  out[2] = ex.violations;
  memcpy(msg, ex.first, sizeof ex.first);
  return rc;
}

// Self-check of the checker: spftrs of k right-hand sides with a B buffer
// registered one column short must report violations.
int hs_bounds_short_b(int n, int k, int64_t* out, char* msg) {
  BoundsExec ex;
  float* C = ex.add("rfp", (size_t)n * (n + 1) / 2);
  float* B = ex.add("B", (size_t)n * (k - 1));
  int rc = plan::spftrs(ex, 1, 0, n, k, C, B, n);
  out[0] = ex.calls;
  out[1] = ex.checks;
  out[2] = ex.violations;
  memcpy(msg, ex.first, sizeof ex.first);
  return rc;
}

}  // extern "C"
