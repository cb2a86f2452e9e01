// plan.cpp — recursive blocked algorithms over strided views.
//
// All routines reduce to one canonical form (left side, lower triangular, no
// transpose) by view transposition and index reversal; see rfp.h.  The
// RFP-level routines split the logical matrix at n1 exactly as the reference
// does (T1 / S / T2: src/curfp_spftrf.cpp:254-282, src/curfp_spftrs.cpp:257-299,
// src/curfp_ssfrk.cpp:193-209), and every dense sub-problem is then solved
// recursively on the views.
#include "engine.h"

namespace rfp {
namespace plan {

namespace {

// Split n into n1 + n2 with n1 a multiple of `blk`, n1 ~ n/2.
inline int split(int n, int blk) {
  int half = (n + 1) / 2;
  int n1 = ((half + blk - 1) / blk) * blk;
  if (n1 >= n) n1 = n - blk;  // only reached for n <= 2*blk
  if (n1 <= 0) n1 = n / 2;
  return n1;
}

template <typename T>
inline GemmProbT<T> gemm_prob(ViewT<T> A, ViewT<T> B, ViewT<T> C, int m, int n, int k,
                              Scalar<T> alpha, Scalar<T> beta, int math) {
  GemmProbT<T> p{};
  p.A = A; p.B = B; p.C = C;
  p.A2 = A; p.B2 = B;
  p.m = m; p.n = n; p.k = k; p.k2 = 0;
  p.alpha = alpha; p.beta = beta;
  p.c_lower = 0; p.inplace = 0;
  p.a_tri = p.b_tri = p.a2_tri = p.b2_tri = 0;
  p.math = math;
  return p;
}

template <typename T>
int trsm_rec(ExecT<T>& ex, ViewT<T> L, int n, ViewT<T> B, int m, Scalar<T> alpha,
             const T* W, int blk0, int math) {
  if (n <= 0 || m <= 0) return 0;
  const T* Wb = W + (int64_t)blk0 * kInvStride;
  if (n <= kTrsmLeaf) {
    ViewT<T> Wv{const_cast<T*>(Wb), 1, kTrsmLeaf};
    GemmProbT<T> p = gemm_prob(Wv, B, B, n, m, n, alpha, 0.0f, 0);
    p.inplace = 1;
    return ex.gemm(&p, 1);
  }
  // Few right-hand sides: the whole block goes to the wavefront solve (its
  // chain is short relative to the work).  Many right-hand sides: small
  // leaves, so that most of the work is in the (tensor-core) GEMM updates.
  if (n <= (m <= kTrsvMaxRhs * 4 ? kWaveLeaf : (math ? kWaveLeafWideTc : kWaveLeafWide))) {
    int rc = ex.trsm_wave(L, n, B, m, alpha, Wb);
    if (rc != kNotSupported) return rc;
  }
  int n1 = split(n, kTrsmLeaf), n2 = n - n1;
  int rc = trsm_rec(ex, L, n1, B, m, alpha, W, blk0, math);
  if (rc) return rc;
  GemmProbT<T> p = gemm_prob(sub(L, n1, 0), B, sub(B, n1, 0), n2, m, n1, -1.0f,
                         alpha, math);
  if ((rc = ex.gemm(&p, 1))) return rc;
  return trsm_rec(ex, sub(L, n1, n1), n2, sub(B, n1, 0), m, 1.0f, W,
                  blk0 + n1 / kTrsmLeaf, math);
}

}  // namespace

template <typename T>
int trsm_lln(ExecT<T>& ex, ViewT<T> L, int n, ViewT<T> B, int m, Scalar<T> alpha, int math) {
  if (n <= 0 || m <= 0) return 0;
  int nblk = (n + kTrsmLeaf - 1) / kTrsmLeaf;
  T* W = ex.workspace((size_t)nblk * kInvStride);
  if (!W) return 2;
  int rc = ex.trtri_blocks(L, n, kTrsmLeaf, W);
  if (rc) return rc;
  // One wavefront launch for few right-hand sides; with tensor-core updates
  // available the recursive solve wins above kTrsvMaxRhsTc of them.
  if (m <= (math ? kTrsvMaxRhsTc : kTrsvMaxRhs)) {
    rc = ex.trsm_wave(L, n, B, m, alpha, W);
    if (rc != kNotSupported) return rc;
  }
  return trsm_rec(ex, L, n, B, m, alpha, W, 0, math);
}

template <typename T>
int trsm(ExecT<T>& ex, int left, int lower, int trans, ViewT<T> Tm, ViewT<T> B, int rows,
         int cols, Scalar<T> alpha, int math) {
  if (!left) {  // X op(T) = B  <=>  op(T)^T X^T = B^T
    B = tr(B);
    int t = rows; rows = cols; cols = t;
    trans = !trans;
  }
  ViewT<T> E = trans ? tr(Tm) : Tm;
  int e_lower = lower ^ trans;
  if (e_lower) return trsm_lln(ex, E, rows, B, cols, alpha, math);
  return trsm_lln(ex, rev(E, rows, rows), rows, rev_rows(B, rows), cols,
                  alpha, math);
}

template <typename T>
int trmm_lln(ExecT<T>& ex, ViewT<T> L, int n, ViewT<T> B, int m, Scalar<T> alpha, int math) {
  if (n <= 0 || m <= 0) return 0;
  int leaf = kTrmmLeaf < ex.inplace_rows() ? kTrmmLeaf : ex.inplace_rows();
  if (n <= leaf) {
    GemmProbT<T> p = gemm_prob(L, B, B, n, m, n, alpha, 0.0f, 0);
    p.a_tri = 1;
    p.inplace = 1;
    return ex.gemm(&p, 1);
  }
  int n1 = split(n, leaf), n2 = n - n1;
  int rc = trmm_lln(ex, sub(L, n1, n1), n2, sub(B, n1, 0), m, alpha, math);
  if (rc) return rc;
  GemmProbT<T> p = gemm_prob(sub(L, n1, 0), B, sub(B, n1, 0), n2, m, n1, alpha,
                         1.0f, math);
  if ((rc = ex.gemm(&p, 1))) return rc;
  return trmm_lln(ex, L, n1, B, m, alpha, math);
}

template <typename T>
int trmm(ExecT<T>& ex, int left, int lower, int trans, ViewT<T> Tm, ViewT<T> B, int rows,
         int cols, Scalar<T> alpha, int math) {
  if (!left) {  // B op(T)  <=>  (op(T)^T B^T)^T
    B = tr(B);
    int t = rows; rows = cols; cols = t;
    trans = !trans;
  }
  ViewT<T> E = trans ? tr(Tm) : Tm;
  int e_lower = lower ^ trans;
  if (e_lower) return trmm_lln(ex, E, rows, B, cols, alpha, math);
  return trmm_lln(ex, rev(E, rows, rows), rows, rev_rows(B, rows), cols,
                  alpha, math);
}

template <typename T>
int potrf_lower(ExecT<T>& ex, ViewT<T> A, int n, int info_base, int math) {
  if (n <= 0) return 0;
  const int tile = ex.potrf_tile_rows();
  if (n <= tile) return ex.potrf_tile(A, n, info_base);
  int n1 = split(n, tile), n2 = n - n1;
  int rc = potrf_lower(ex, A, n1, info_base, math);
  if (rc) return rc;
  ViewT<T> A21 = sub(A, n1, 0);
  // A21 := A21 L11^{-T}   <=>   L11 A21^T = A21^T
  if ((rc = trsm_lln(ex, A, n1, tr(A21), n2, 1.0f, math))) return rc;
  // A22 := A22 - A21 A21^T (lower)
  SharedTaskT<T> t{0, 0, n2, n2, sub(A, n1, n1), -1.0f, 1.0f, 1};
  if ((rc = ex.gemm_shared(A21, n2, n1, &t, 1, math))) return rc;
  return potrf_lower(ex, sub(A, n1, n1), n2, info_base + n1, math);
}

template <typename T>
int trtri_lower(ExecT<T>& ex, ViewT<T> L, int n, int math) {
  if (n <= 0) return 0;
  if (n <= kTriTile) return ex.trtri_tile(L, n);
  int n1 = split(n, kTriTile), n2 = n - n1;
  int rc = trtri_lower(ex, L, n1, math);
  if (rc) return rc;
  if ((rc = trtri_lower(ex, sub(L, n1, n1), n2, math))) return rc;
  ViewT<T> L21 = sub(L, n1, 0);
  // L21 := -inv(L22) L21 inv(L11)
  if ((rc = trmm(ex, 0, 1, 0, L, L21, n2, n1, 1.0f, math))) return rc;
  return trmm(ex, 1, 1, 0, sub(L, n1, n1), L21, n2, n1, -1.0f, math);
}

template <typename T>
int lauum_lower(ExecT<T>& ex, ViewT<T> L, int n, int math) {
  if (n <= 0) return 0;
  if (n <= kTriTile) return ex.lauum_tile(L, n);
  int n1 = split(n, kTriTile), n2 = n - n1;
  ViewT<T> L21 = sub(L, n1, 0);
  int rc = lauum_lower(ex, L, n1, math);
  if (rc) return rc;
  // L11 += L21^T L21 (lower): a SYRK whose one operand is L21^T (n1 x n2)
  SharedTaskT<T> t{0, 0, n1, n1, L, 1.0f, 1.0f, 1};
  if ((rc = ex.gemm_shared(tr(L21), n1, n2, &t, 1, math))) return rc;
  if ((rc = trmm(ex, 1, 1, 1, sub(L, n1, n1), L21, n2, n1, 1.0f, math)))
    return rc;
  return lauum_lower(ex, sub(L, n1, n1), n2, math);
}

// ---------------------------------------------------------------------------
// RFP routines
// ---------------------------------------------------------------------------

template <typename T>
int ssfrk(ExecT<T>& ex, int transr, int lower, int trans, int n, int k,
          Scalar<T> alpha, const T* A, int lda, Scalar<T> beta, T* C,
          int math) {
  Geometry g = geometry(n, transr, lower);
  // op(A) is n x k.  trans = N: A is n x k column-major; trans = T: A is
  // k x n column-major and op(A) = A^T.
  ViewT<T> opA = trans ? ViewT<T>{const_cast<T*>(A), lda, 1}
                   : ViewT<T>{const_cast<T*>(A), 1, lda};
  if (alpha == 0.0f) k = 0;  // C := beta*C; A is not read
  ViewT<T> C11 = block_view(C, g.b11), C21 = block_view(C, g.b21),
       C22 = block_view(C, g.b22);
  SharedTaskT<T> t[3];
  int cnt = 0;
  if (g.n1 > 0) t[cnt++] = SharedTaskT<T>{0, 0, g.n1, g.n1, C11, alpha, beta, 1};
  if (g.n1 > 0 && g.n2 > 0)
    t[cnt++] = SharedTaskT<T>{g.n1, 0, g.n2, g.n1, C21, alpha, beta, 0};
  if (g.n2 > 0) t[cnt++] = SharedTaskT<T>{g.n1, g.n1, g.n2, g.n2, C22, alpha, beta, 1};
  return ex.gemm_shared(opA, n, k, t, cnt, math);
}

template <typename T>
int ssfr2k(ExecT<T>& ex, int transr, int lower, int trans, int n, int k,
           Scalar<T> alpha, const T* A, int lda, const T* B, int ldb,
           Scalar<T> beta, T* C, int math) {
  Geometry g = geometry(n, transr, lower);
  ViewT<T> opA = trans ? ViewT<T>{const_cast<T*>(A), lda, 1}
                   : ViewT<T>{const_cast<T*>(A), 1, lda};
  ViewT<T> opB = trans ? ViewT<T>{const_cast<T*>(B), ldb, 1}
                   : ViewT<T>{const_cast<T*>(B), 1, ldb};
  if (alpha == 0.0f) k = 0;
  // The blocks of the reference's 2 SSYR2K + 2 SGEMM (src/curfp_ssfr2k.cpp:
  // 193-229): T1 (lower), S, T2 (lower), each alpha (A_i B_j^T + B_i A_j^T).
  ViewT<T> C11 = block_view(C, g.b11), C21 = block_view(C, g.b21),
       C22 = block_view(C, g.b22);
  SharedTaskT<T> t[3];
  int cnt = 0;
  if (g.n1 > 0) t[cnt++] = SharedTaskT<T>{0, 0, g.n1, g.n1, C11, alpha, beta, 1};
  if (g.n1 > 0 && g.n2 > 0)
    t[cnt++] = SharedTaskT<T>{g.n1, 0, g.n2, g.n1, C21, alpha, beta, 0};
  if (g.n2 > 0) t[cnt++] = SharedTaskT<T>{g.n1, g.n1, g.n2, g.n2, C22, alpha, beta, 1};
  return ex.gemm_pair(opA, opB, n, k, t, cnt, math);
}

template <typename T>
int spftrf(ExecT<T>& ex, int transr, int lower, int n, T* A, int math) {
  Geometry g = geometry(n, transr, lower);
  ViewT<T> V11 = block_view(A, g.b11), V21 = block_view(A, g.b21),
       V22 = block_view(A, g.b22);
  int rc = potrf_lower(ex, V11, g.n1, 0, math);
  if (rc) return rc;
  if ((rc = ex.after_first_block())) return rc;
  if (g.n2 == 0) return 0;
  if (g.n1 > 0) {
    if ((rc = trsm_lln(ex, V11, g.n1, tr(V21), g.n2, 1.0f, math))) return rc;
    SharedTaskT<T> t{0, 0, g.n2, g.n2, V22, -1.0f, 1.0f, 1};
    if ((rc = ex.gemm_shared(V21, g.n2, g.n1, &t, 1, math))) return rc;
  }
  return potrf_lower(ex, V22, g.n2, g.n1, math);
}

template <typename T>
int spftrs(ExecT<T>& ex, int transr, int lower, int n, int nrhs, const T* A,
           T* B, int ldb, int math) {
  Geometry g = geometry(n, transr, lower);
  T* Af = const_cast<T*>(A);
  ViewT<T> V11 = block_view(Af, g.b11), V21 = block_view(Af, g.b21),
       V22 = block_view(Af, g.b22);
  ViewT<T> B1{B, 1, ldb};
  ViewT<T> B2 = sub(B1, g.n1, 0);
  int rc;
  // Forward: L Y = B.
  if ((rc = trsm_lln(ex, V11, g.n1, B1, nrhs, 1.0f, math))) return rc;
  if (g.n1 > 0 && g.n2 > 0) {
    GemmProbT<T> p = gemm_prob(V21, B1, B2, g.n2, nrhs, g.n1, -1.0f, 1.0f, math);
    if ((rc = ex.gemm(&p, 1))) return rc;
  }
  if ((rc = trsm_lln(ex, V22, g.n2, B2, nrhs, 1.0f, math))) return rc;
  // Backward: L^T X = Y.
  if ((rc = trsm(ex, 1, 1, 1, V22, B2, g.n2, nrhs, 1.0f, math))) return rc;
  if (g.n1 > 0 && g.n2 > 0) {
    GemmProbT<T> p = gemm_prob(tr(V21), B2, B1, g.n1, nrhs, g.n2, -1.0f, 1.0f, math);
    if ((rc = ex.gemm(&p, 1))) return rc;
  }
  return trsm(ex, 1, 1, 1, V11, B1, g.n1, nrhs, 1.0f, math);
}

template <typename T>
int rfp_trtri(ExecT<T>& ex, int transr, int lower, int n, T* A, int math) {
  Geometry g = geometry(n, transr, lower);
  ViewT<T> V11 = block_view(A, g.b11), V21 = block_view(A, g.b21),
       V22 = block_view(A, g.b22);
  int rc;
  // inv(L) = [M11 0; -M22 L21 M11  M22]
  if ((rc = trtri_lower(ex, V11, g.n1, math))) return rc;
  if ((rc = trtri_lower(ex, V22, g.n2, math))) return rc;
  if (g.n1 > 0 && g.n2 > 0) {
    if ((rc = trmm(ex, 0, 1, 0, V11, V21, g.n2, g.n1, 1.0f, math))) return rc;
    if ((rc = trmm(ex, 1, 1, 0, V22, V21, g.n2, g.n1, -1.0f, math))) return rc;
  }
  return 0;
}

template <typename T>
int spftri(ExecT<T>& ex, int transr, int lower, int n, T* A, int math) {
  Geometry g = geometry(n, transr, lower);
  ViewT<T> V11 = block_view(A, g.b11), V21 = block_view(A, g.b21),
       V22 = block_view(A, g.b22);
  int rc;
  if ((rc = rfp_trtri(ex, transr, lower, n, A, math))) return rc;
  // inv(A) = M^T M:  (11) = M11^T M11 + M21^T M21, (21) = M22^T M21,
  //                  (22) = M22^T M22
  if ((rc = lauum_lower(ex, V11, g.n1, math))) return rc;
  if (g.n1 > 0 && g.n2 > 0) {
    SharedTaskT<T> t{0, 0, g.n1, g.n1, V11, 1.0f, 1.0f, 1};
    if ((rc = ex.gemm_shared(tr(V21), g.n1, g.n2, &t, 1, math))) return rc;
    if ((rc = trmm(ex, 1, 1, 1, V22, V21, g.n2, g.n1, 1.0f, math))) return rc;
  }
  return lauum_lower(ex, V22, g.n2, math);
}

// ---------------------------------------------------------------------------
// Adjoint building blocks
// ---------------------------------------------------------------------------

namespace {
template <typename T>
struct Blocks {
  Geometry g;
  ViewT<T> V11, V21, V22;
};
template <typename T>
inline Blocks<T> blocks(int transr, int lower, int n, const T* A) {
  Blocks<T> b;
  b.g = geometry(n, transr, lower);
  T* p = const_cast<T*>(A);
  b.V11 = block_view(p, b.g.b11);
  b.V21 = block_view(p, b.g.b21);
  b.V22 = block_view(p, b.g.b22);
  return b;
}
}  // namespace

template <typename T>
int rfp_trsm(ExecT<T>& ex, int transr, int lower, int n, const T* L, int trans, ViewT<T> B,
             int m, Scalar<T> alpha, int math) {
  Blocks<T> b = blocks(transr, lower, n, L);
  const int n1 = b.g.n1, n2 = b.g.n2;
  ViewT<T> B1 = B, B2 = sub(B, n1, 0);
  int rc;
  if (!trans) {
    if ((rc = trsm_lln(ex, b.V11, n1, B1, m, alpha, math))) return rc;
    if (n1 > 0 && n2 > 0) {
      GemmProbT<T> p = gemm_prob(b.V21, B1, B2, n2, m, n1, -1.0f, alpha, math);
      if ((rc = ex.gemm(&p, 1))) return rc;
    }
    return trsm_lln(ex, b.V22, n2, B2, m, n1 > 0 ? 1.0f : alpha, math);
  }
  if ((rc = trsm(ex, 1, 1, 1, b.V22, B2, n2, m, alpha, math))) return rc;
  if (n1 > 0 && n2 > 0) {
    GemmProbT<T> p = gemm_prob(tr(b.V21), B2, B1, n1, m, n2, -1.0f, alpha, math);
    if ((rc = ex.gemm(&p, 1))) return rc;
  }
  return trsm(ex, 1, 1, 1, b.V11, B1, n1, m, n2 > 0 ? 1.0f : alpha, math);
}

template <typename T>
int rfp_trmm_t(ExecT<T>& ex, int transr, int lower, int n, const T* L, ViewT<T> B, int m) {
  Blocks<T> b = blocks(transr, lower, n, L);
  const int n1 = b.g.n1, n2 = b.g.n2;
  ViewT<T> B1 = B, B2 = sub(B, n1, 0);
  int rc;
  // (L^T B)_1 = L11^T B1 + L21^T B2 ; (L^T B)_2 = L22^T B2
  if ((rc = trmm(ex, 1, 1, 1, b.V11, B1, n1, m, 1.0f))) return rc;
  if (n1 > 0 && n2 > 0) {
    GemmProbT<T> p = gemm_prob(tr(b.V21), B2, B1, n1, m, n2, 1.0f, 1.0f, 0);
    if ((rc = ex.gemm(&p, 1))) return rc;
  }
  return trmm(ex, 1, 1, 1, b.V22, B2, n2, m, 1.0f);
}

template <typename T>
int rfp_gemm_lower2(ExecT<T>& ex, int transr, int lower, int n, T* C, ViewT<T> A1, ViewT<T> B1,
                    ViewT<T> A2, ViewT<T> B2, int k, Scalar<T> alpha, Scalar<T> beta) {
  Blocks<T> c = blocks(transr, lower, n, C);
  const int n1 = c.g.n1, n2 = c.g.n2;
  ViewT<T> Cb[3] = {c.V11, c.V21, c.V22};
  const int r0[3] = {0, n1, n1}, c0[3] = {0, 0, n1};
  const int dm[3] = {n1, n2, n2}, dn[3] = {n1, n1, n2};
  GemmProbT<T> p[3];
  int cnt = 0;
  for (int b = 0; b < 3; ++b) {
    if (dm[b] <= 0 || dn[b] <= 0) continue;
    GemmProbT<T> q = gemm_prob(sub(A1, r0[b], 0), sub(B1, 0, c0[b]), Cb[b], dm[b], dn[b], k,
                           alpha, beta, 0);
    q.A2 = sub(A2, r0[b], 0);
    q.B2 = sub(B2, 0, c0[b]);
    q.k2 = k;
    q.c_lower = (b != 1);
    p[cnt++] = q;
  }
  return ex.gemm(p, cnt);
}

namespace {
// One panel step of the blocked Cholesky adjoint.  With the trailing block's
// adjoint G22 final (stored lower triangle of the cotangent of
// S = A22 - L21 L21^T):
//   G21 -= (tril(G22) + tril(G22)^T) L21     (S's diagonal counted twice)
//   G21 := G21 L11^{-1}                       (cotangent of A21 = L21 L11^T)
//   G11 -= tril(G21^T L21)                    (L11's share through L21)
template <typename T>
int adj_panel(ExecT<T>& ex, ViewT<T> L11, ViewT<T> L21, ViewT<T> G11, ViewT<T> G21,
              ViewT<T> G22, int n1, int n2, int math) {
  GemmProbT<T> p = gemm_prob(G22, L21, G21, n2, n1, n2, -1.0f, 1.0f, math);
  p.a_tri = 1;          // lower(G22), diagonal included
  p.A2 = tr(G22);
  p.B2 = L21;
  p.k2 = n2;
  p.a2_tri = 2;         // lower(G22)^T, diagonal included again
  int rc;
  if ((rc = ex.gemm(&p, 1))) return rc;
  if ((rc = trsm(ex, 0, 1, 0, L11, G21, n2, n1, 1.0f, math))) return rc;
  GemmProbT<T> q = gemm_prob(tr(G21), L21, G11, n1, n1, n2, -1.0f, 1.0f, math);
  q.c_lower = 1;
  return ex.gemm(&q, 1);
}
}  // namespace

template <typename T>
int potrf_adj_lower(ExecT<T>& ex, ViewT<T> L, ViewT<T> G, int n, int math) {
  if (n <= 0) return 0;
  if (n <= kAdjTile) return ex.potrf_adj_tile(L, G, n);
  const int n1 = split(n, kAdjTile), n2 = n - n1;
  int rc;
  if ((rc = potrf_adj_lower(ex, sub(L, n1, n1), sub(G, n1, n1), n2, math))) return rc;
  if ((rc = adj_panel(ex, L, sub(L, n1, 0), G, sub(G, n1, 0), sub(G, n1, n1), n1, n2, math)))
    return rc;
  return potrf_adj_lower(ex, L, G, n1, math);
}

// The RFP factor's three logical blocks follow the forward decomposition
// (src/curfp_spftrf.cpp:254-282: POTRF T1, TRSM S, SYRK T2, POTRF T2), so the
// adjoint runs the same panel step once on the blocks, between the two
// diagonal-block adjoints taken in reverse order.
template <typename T>
int spftrf_adjoint(ExecT<T>& ex, int transr, int lower, int n, const T* L, T* G, int math) {
  Blocks<T> b = blocks(transr, lower, n, L), c = blocks(transr, lower, n, (const T*)G);
  const int n1 = b.g.n1, n2 = b.g.n2;
  int rc;
  if ((rc = potrf_adj_lower(ex, b.V22, c.V22, n2, math))) return rc;
  if (n1 > 0 && n2 > 0 &&
      (rc = adj_panel(ex, b.V11, b.V21, c.V11, c.V21, c.V22, n1, n2, math)))
    return rc;
  return potrf_adj_lower(ex, b.V11, c.V11, n1, math);
}

namespace {
// Y := alpha (G_L + G_L^T - s D) X + beta Y with D the diagonal of G_L:
// s = 0 counts the diagonal twice, s = 1 once (the symmetric matrix itself;
// the transposed triangles then exclude their diagonal).  The blocks follow
// the reference's SSYMM + 2 SGEMM split (src/curfp_ssfmm.cpp:150-306):
//   Y1 = a (G11 sym) X1 + a G21^T X2 + b Y1,  Y2 = a G21 X1 + a (G22 sym) X2 + b Y2
template <typename T>
int symm_blocks(ExecT<T>& ex, int transr, int lower, int n, const T* G, ViewT<T> X, ViewT<T> Y,
                int m, Scalar<T> alpha, Scalar<T> beta, int once) {
  Blocks<T> g = blocks(transr, lower, n, G);
  const int n1 = g.g.n1, n2 = g.g.n2;
  const int up = once ? 3 : 2;  // mask of the transposed triangles
  ViewT<T> X1 = X, X2 = sub(X, n1, 0), Y1 = Y, Y2 = sub(Y, n1, 0);
  const bool zero = alpha == 0.0f;  // C := beta C, A and X not read
  GemmProbT<T> p[2];
  int cnt = 0;
  if (n1 > 0) {
    GemmProbT<T> q = gemm_prob(g.V11, X1, Y1, n1, m, zero ? 0 : n1, alpha, beta, 0);
    q.a_tri = 1;
    q.A2 = tr(g.V11);
    q.B2 = X1;
    q.k2 = zero ? 0 : n1;
    q.a2_tri = up;
    p[cnt++] = q;
  }
  if (n2 > 0) {
    GemmProbT<T> q = gemm_prob(g.V21, X1, Y2, n2, m, (zero || n1 == 0) ? 0 : n1, alpha, beta, 0);
    q.A2 = g.V22;
    q.B2 = X2;
    q.k2 = zero ? 0 : n2;
    q.a2_tri = 1;
    p[cnt++] = q;
  }
  int rc;
  if ((rc = ex.gemm(p, cnt))) return rc;
  if (zero) return 0;
  cnt = 0;
  if (n1 > 0 && n2 > 0) {
    GemmProbT<T> q = gemm_prob(tr(g.V21), X2, Y1, n1, m, n2, alpha, 1.0f, 0);
    p[cnt++] = q;
  }
  if (n2 > 0) {
    GemmProbT<T> q = gemm_prob(tr(g.V22), X2, Y2, n2, m, n2, alpha, 1.0f, 0);
    q.a_tri = up;
    p[cnt++] = q;
  }
  return ex.gemm(p, cnt);
}
}  // namespace

template <typename T>
int rfp_symm(ExecT<T>& ex, int transr, int lower, int n, const T* A, ViewT<T> X, ViewT<T> Y, int m,
             Scalar<T> alpha, Scalar<T> beta) {
  return symm_blocks(ex, transr, lower, n, A, X, Y, m, alpha, beta, 1);
}

template <typename T>
int rfp_symm_dbl(ExecT<T>& ex, int transr, int lower, int n, const T* G, ViewT<T> X, ViewT<T> Y,
                 int m, Scalar<T> alpha, Scalar<T> beta) {
  return symm_blocks(ex, transr, lower, n, G, X, Y, m, alpha, beta, 0);
}

// The planner is instantiated for the FP32 routines and their FP64 twins.
#define RFP_PLAN_INSTANTIATE(T)                                                              \
  template int trsm_lln<T>(ExecT<T>&, ViewT<T>, int, ViewT<T>, int, Scalar<T>, int);          \
  template int trsm<T>(ExecT<T>&, int, int, int, ViewT<T>, ViewT<T>, int, int, Scalar<T>,     \
                       int);                                                                 \
  template int trmm_lln<T>(ExecT<T>&, ViewT<T>, int, ViewT<T>, int, Scalar<T>, int);          \
  template int trmm<T>(ExecT<T>&, int, int, int, ViewT<T>, ViewT<T>, int, int, Scalar<T>,     \
                       int);                                                                 \
  template int potrf_lower<T>(ExecT<T>&, ViewT<T>, int, int, int);                            \
  template int trtri_lower<T>(ExecT<T>&, ViewT<T>, int, int);                                 \
  template int lauum_lower<T>(ExecT<T>&, ViewT<T>, int, int);                                 \
  template int ssfrk<T>(ExecT<T>&, int, int, int, int, int, Scalar<T>, const T*, int,         \
                        Scalar<T>, T*, int);                                                 \
  template int ssfr2k<T>(ExecT<T>&, int, int, int, int, int, Scalar<T>, const T*, int,        \
                         const T*, int, Scalar<T>, T*, int);                                 \
  template int spftrf<T>(ExecT<T>&, int, int, int, T*, int);                                  \
  template int spftrs<T>(ExecT<T>&, int, int, int, int, const T*, T*, int, int);              \
  template int spftri<T>(ExecT<T>&, int, int, int, T*, int);                                  \
  template int rfp_trtri<T>(ExecT<T>&, int, int, int, T*, int);                               \
  template int rfp_trsm<T>(ExecT<T>&, int, int, int, const T*, int, ViewT<T>, int, Scalar<T>, \
                           int);                                                             \
  template int rfp_trmm_t<T>(ExecT<T>&, int, int, int, const T*, ViewT<T>, int);              \
  template int rfp_gemm_lower2<T>(ExecT<T>&, int, int, int, T*, ViewT<T>, ViewT<T>, ViewT<T>, \
                                  ViewT<T>, int, Scalar<T>, Scalar<T>);                      \
  template int potrf_adj_lower<T>(ExecT<T>&, ViewT<T>, ViewT<T>, int, int);                 \
  template int spftrf_adjoint<T>(ExecT<T>&, int, int, int, const T*, T*, int);                \
  template int rfp_symm<T>(ExecT<T>&, int, int, int, const T*, ViewT<T>, ViewT<T>, int,       \
                           Scalar<T>, Scalar<T>);                                            \
  template int rfp_symm_dbl<T>(ExecT<T>&, int, int, int, const T*, ViewT<T>, ViewT<T>, int,   \
                               Scalar<T>, Scalar<T>);

RFP_PLAN_INSTANTIATE(float)
RFP_PLAN_INSTANTIATE(double)

}  // namespace plan
}  // namespace rfp
