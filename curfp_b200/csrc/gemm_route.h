// gemm_route.h — which contractions the few-column kernels (k_skinny.cuh)
// take; host code, shared by the CUDA executor and the host tests.
#pragma once
#include "engine.h"

namespace rfp {

constexpr int kSkinnyMaxCols = 8;

struct SkinnyRoute {
  bool use;        // the few-column kernels take the product
  bool transpose;  // computed as C^T = B^T A^T (m <= 8 < n)
  bool rows;       // A's row index is its unit-stride one (skinny_rows), else its column index
  int inst;        // column count of the instantiation: 1, 2, 4 or 8
};

// A single full product (no second product, no triangular masks, no
// in-place output) with at most 8 columns -- or at most 8 rows, through the
// transpose -- at least 2^20 elements of A, and A unit-stride along one of
// its dimensions.  *out is the product as the kernels compute it.
template <typename T>
inline SkinnyRoute skinny_route(const GemmProbT<T>& g0, GemmProbT<T>* out) {
  SkinnyRoute r{false, false, false, 0};
  GemmProbT<T> g = g0;
  if (g.k2 || g.a_tri || g.b_tri || g.c_lower || g.inplace) return r;
  if (g.n > kSkinnyMaxCols && g.m <= kSkinnyMaxCols) {
    const ViewT<T> A = tr(g.B), B = tr(g.A);
    g.A = A;
    g.B = B;
    g.C = tr(g.C);
    const int t = g.m;
    g.m = g.n;
    g.n = t;
    r.transpose = true;
  }
  if (g.n > kSkinnyMaxCols || g.m <= 0 || g.n <= 0 || g.k <= 0) return r;
  if ((int64_t)g.m * g.k < ((int64_t)1 << 20)) return r;
  r.rows = g.A.rs == 1 || g.A.rs == -1;
  if (!r.rows && !(g.A.cs == 1 || g.A.cs == -1)) return r;
  r.use = true;
  r.inst = g.n == 1 ? 1 : (g.n == 2 ? 2 : (g.n <= 4 ? 4 : 8));
  *out = g;
  return r;
}

}  // namespace rfp
