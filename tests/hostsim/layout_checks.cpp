// layout_checks.cpp — TEST-ONLY host entry points for the index arithmetic
// of the single-read symmetric matrix-vector kernel (symv_layout.h) and the
// routing of few-column products (gemm_route.h), run without a GPU.
#include <cstdint>
#include <vector>

#include "engine.h"
#include "gemm_route.h"
#include "symv_layout.h"

using namespace rfp;

extern "C" {

// Enumerates the CTAs of the ssfmv launch at order n the way the kernel maps
// them.  out: [0] CTAs, [1] lower tiles visited, [2] visits to a tile
// already visited or outside the lower triangle, [3] row_part entries past
// n_row, [4] col_part entries past n_col, [5] col_part entries written by two
// tiles, [6] strips with an empty tile range.
int hs_symv_layout(int n, int64_t* out) {
  const ksymv::Parts P = ksymv::parts(n);
  const int T = P.tiles;
  const int64_t ctas = ksymv::strips_before(T);
  std::vector<int> seen((size_t)T * T, 0);
  std::vector<int> col((size_t)(P.n_col / ksymv::TB), 0);
  int64_t visited = 0, dup = 0, row_over = 0, col_over = 0, col_dup = 0, empty = 0;
  for (int64_t b = 0; b < ctas; ++b) {
    int I, s;
    ksymv::strip_of(b, T, I, s);
    const int Jb = s * ksymv::S, Je = Jb + ksymv::S < I + 1 ? Jb + ksymv::S : I + 1;
    if (Jb >= Je) ++empty;
    if (((int64_t)I * P.strips + s + 1) * ksymv::TB > P.n_row) ++row_over;
    for (int J = Jb; J < Je; ++J) {
      if (J > I || J < 0 || seen[(size_t)I * T + J]++) ++dup;
      ++visited;
      const int64_t e = ksymv::col_base(J, T) + (I - J);
      if ((e + 1) * ksymv::TB > P.n_col) {
        ++col_over;
      } else if (col[(size_t)e]++) {
        ++col_dup;
      }
    }
  }
  out[0] = ctas;
  out[1] = visited;
  out[2] = dup;
  out[3] = row_over;
  out[4] = col_over;
  out[5] = col_dup;
  out[6] = empty;
  return 0;
}

// skinny_route of a product C (m x n) = A (m x k, strides a_rs, a_cs) B
// (k x n, column-major) with the given flags.  out: use, transpose, rows,
// instantiation, and the routed m, n, k.
int hs_skinny_route(int m, int n, int k, int k2, int a_tri, int b_tri, int c_lower, int inplace,
                    int64_t a_rs, int64_t a_cs, int* out) {
  static float buf[1];
  GemmProb g{};
  g.A = View{buf, a_rs, a_cs};
  g.B = View{buf, 1, k};
  g.C = View{buf, 1, m};
  g.A2 = g.A;
  g.B2 = g.B;
  g.m = m;
  g.n = n;
  g.k = k;
  g.k2 = k2;
  g.alpha = -1.0f;
  g.beta = 1.0f;
  g.a_tri = a_tri;
  g.b_tri = b_tri;
  g.c_lower = c_lower;
  g.inplace = inplace;
  GemmProb r{};
  const SkinnyRoute s = skinny_route(g, &r);
  out[0] = s.use;
  out[1] = s.transpose;
  out[2] = s.rows;
  out[3] = s.inst;
  out[4] = s.use ? r.m : 0;
  out[5] = s.use ? r.n : 0;
  out[6] = s.use ? r.k : 0;
  return 0;
}

}  // extern "C"
