// rfp.h — strided matrix views and the RFP geometry of all 8 storage variants.
//
// Every RFP variant (n odd/even x TRANSR N/T x UPLO L/U) stores the n x n
// symmetric matrix as three blocks inside one array of n(n+1)/2 elements.
// Here each block is described as a *view of the logical lower triangle*:
//
//     logical L(p,q), p >= q   lives at   arf[off + p*rs + q*cs]
//
// with (off, rs, cs) constant inside a block:
//     V11: rows/cols [0, n1)            (lower triangle of the leading block)
//     V21: rows [n1, n), cols [0, n1)   (full rectangle)
//     V22: rows/cols [n1, n)            (lower triangle of the trailing block)
// For UPLO=U the stored element a(q,p) (q <= p) equals the logical lower
// element (p,q) by symmetry, and the Cholesky factor U(q,p) = L(p,q), so one
// lower-triangular algorithm on these views serves all 8 variants.
//
// The offsets and strides restate, per case, the sub-block pointers and
// leading dimensions of the reference tables (src/curfp_spftrf.cpp:62-180,
// src/curfp_ssfrk.cpp:52-133, src/curfp_spftrs.cpp:60-213,
// src/curfp_spftri.cu:71-136) and of rfp_diag_indices
// (curfp/__init__.py:194-269), rewritten from cuBLAS (fill, op, ld) triples
// into (off, rs, cs) of the logical lower factor.  The n1/n2 split follows
// src/curfp_spftrf.cpp:208-215 (odd n: lower -> n1 = ceil(n/2), upper ->
// n1 = floor(n/2); even n: n1 = n2 = n/2).
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define RFP_HD __host__ __device__ __forceinline__
#else
#define RFP_HD inline
#endif

namespace rfp {

// Element (i,j) of a view is p[i*rs + j*cs].  Strides may be negative
// (reversed views turn upper-triangular problems into lower ones).
template <typename T>
struct ViewT {
  T* p;
  int64_t rs;
  int64_t cs;
};
using View = ViewT<float>;

template <typename T>
RFP_HD ViewT<T> sub(ViewT<T> v, int64_t i, int64_t j) {
  return ViewT<T>{v.p + i * v.rs + j * v.cs, v.rs, v.cs};
}
// Transpose: element (i,j) of the result is element (j,i) of v.
template <typename T>
RFP_HD ViewT<T> tr(ViewT<T> v) { return ViewT<T>{v.p, v.cs, v.rs}; }
// Reverse both indices of an m x n view: (i,j) -> (m-1-i, n-1-j).
template <typename T>
RFP_HD ViewT<T> rev(ViewT<T> v, int64_t m, int64_t n) {
  return ViewT<T>{v.p + (m - 1) * v.rs + (n - 1) * v.cs, -v.rs, -v.cs};
}
// Reverse the row index of an m-row view.
template <typename T>
RFP_HD ViewT<T> rev_rows(ViewT<T> v, int64_t m) {
  return ViewT<T>{v.p + (m - 1) * v.rs, -v.rs, v.cs};
}

struct BlockGeom {
  int64_t off, rs, cs;
};

struct Geometry {
  int n, n1, n2;
  BlockGeom b11, b21, b22;
};

// transr: 0 = N, 1 = T.  lower: 1 = UPLO L, 0 = UPLO U.
RFP_HD Geometry geometry(int n, int transr, int lower) {
  Geometry g;
  g.n = n;
  const int64_t N = n;
  if (n & 1) {
    if (lower) { g.n2 = n / 2; g.n1 = n - g.n2; }
    else       { g.n1 = n / 2; g.n2 = n - g.n1; }
    const int64_t n1 = g.n1, n2 = g.n2;
    if (transr == 0) {
      if (lower) {  // case 1: ld = n
        g.b11 = {0, 1, N};  g.b21 = {n1, 1, N};  g.b22 = {N, N, 1};
      } else {      // case 2: ld = n
        g.b11 = {n2, 1, N}; g.b21 = {0, N, 1};   g.b22 = {n1, N, 1};
      }
    } else {
      if (lower) {  // case 3: ld = n1
        g.b11 = {0, n1, 1}; g.b21 = {n1 * n1, n1, 1}; g.b22 = {1, 1, n1};
      } else {      // case 4: ld = n2
        g.b11 = {n2 * n2, n2, 1}; g.b21 = {0, 1, n2}; g.b22 = {n1 * n2, 1, n2};
      }
    }
  } else {
    g.n1 = g.n2 = n / 2;
    const int64_t k = n / 2;
    if (transr == 0) {
      if (lower) {  // case 5: ld = n+1
        g.b11 = {1, 1, N + 1};     g.b21 = {k + 1, 1, N + 1}; g.b22 = {0, N + 1, 1};
      } else {      // case 6: ld = n+1
        g.b11 = {k + 1, 1, N + 1}; g.b21 = {0, N + 1, 1};     g.b22 = {k, N + 1, 1};
      }
    } else {
      if (lower) {  // case 7: ld = k
        g.b11 = {k, k, 1};           g.b21 = {k * (k + 1), k, 1}; g.b22 = {0, 1, k};
      } else {      // case 8: ld = k
        g.b11 = {k * (k + 1), k, 1}; g.b21 = {0, 1, k};           g.b22 = {k * k, 1, k};
      }
    }
  }
  return g;
}

// Flat RFP offset of logical lower element (p,q), p >= q.
RFP_HD int64_t lower_offset(const Geometry& g, int64_t p, int64_t q) {
  if (q < g.n1) {
    if (p < g.n1) return g.b11.off + p * g.b11.rs + q * g.b11.cs;
    return g.b21.off + (p - g.n1) * g.b21.rs + q * g.b21.cs;
  }
  return g.b22.off + (p - g.n1) * g.b22.rs + (q - g.n1) * g.b22.cs;
}

RFP_HD int64_t diag_offset(const Geometry& g, int64_t i) {
  if (i < g.n1) return g.b11.off + i * (g.b11.rs + g.b11.cs);
  return g.b22.off + (i - g.n1) * (g.b22.rs + g.b22.cs);
}

template <typename T>
RFP_HD ViewT<T> block_view(T* arf, const BlockGeom& b) {
  return ViewT<T>{arf + b.off, b.rs, b.cs};
}

}  // namespace rfp
