/*
 * rfp_oracle.c — CPU oracle for the RFP rank-k / Cholesky / solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the library's
 * results are compared against; it is never linked into libcurfp_b200.so and
 * nothing on the product path calls it.
 *
 * It restates, in plain C and FP64, the reference's own algorithm: the same
 * per-variant parameter tables (which sub-block, fill mode, offset, leading
 * dimension and operation each BLAS/LAPACK call gets) and the same call
 * sequences as the reference sources cited per function, executed by a naive
 * column-major mini-BLAS with cuBLAS/LAPACK semantics (o_syrk, o_gemm, ...).
 * It deliberately does NOT use the library's view geometry, so the two are
 * independent; both are pinned to LAPACK (scipy) golden vectors in tests/.
 *
 * All arrays are double; callers convert from/to float.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef int64_t idx;

enum { LO = 0, UP = 1 };          /* fill */
enum { OPN = 0, OPT = 1 };        /* op   */
enum { SL = 0, SR = 1 };          /* side */

#define AT(M, ld, i, j) (M)[(idx)(i) + (idx)(j) * (idx)(ld)]

/* ------------------------------------------------------------------------
 * Mini-BLAS (column-major, cuBLAS argument conventions, non-unit diagonal).
 * Only the `fill` triangle of a triangular/symmetric operand is ever read.
 * ---------------------------------------------------------------------- */

static double opget(const double *A, int lda, int op, int i, int j) {
  return op == OPN ? AT(A, lda, i, j) : AT(A, lda, j, i);
}

/* C := alpha op(A) op(A)^T + beta C  on the fill triangle of C (n x n). */
static void o_syrk(int fill, int op, int n, int k, double alpha,
                   const double *A, int lda, double beta, double *C, int ldc) {
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      if (fill == LO ? i < j : i > j) continue;
      double s = 0.0;
      for (int l = 0; l < k; ++l) s += opget(A, lda, op, i, l) * opget(A, lda, op, j, l);
      double c = beta == 0.0 ? 0.0 : beta * AT(C, ldc, i, j);
      AT(C, ldc, i, j) = alpha * s + c;
    }
}

/* C := alpha (op(A) op(B)^T + op(B) op(A)^T) + beta C on fill triangle. */
static void o_syr2k(int fill, int op, int n, int k, double alpha,
                    const double *A, int lda, const double *B, int ldb,
                    double beta, double *C, int ldc) {
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      if (fill == LO ? i < j : i > j) continue;
      double s = 0.0;
      for (int l = 0; l < k; ++l)
        s += opget(A, lda, op, i, l) * opget(B, ldb, op, j, l) +
             opget(B, ldb, op, i, l) * opget(A, lda, op, j, l);
      double c = beta == 0.0 ? 0.0 : beta * AT(C, ldc, i, j);
      AT(C, ldc, i, j) = alpha * s + c;
    }
}

/* C := alpha op(A) op(B) + beta C,  C m x n. */
static void o_gemm(int opa, int opb, int m, int n, int k, double alpha,
                   const double *A, int lda, const double *B, int ldb,
                   double beta, double *C, int ldc) {
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) {
      double s = 0.0;
      for (int l = 0; l < k; ++l) s += opget(A, lda, opa, i, l) * opget(B, ldb, opb, l, j);
      double c = beta == 0.0 ? 0.0 : beta * AT(C, ldc, i, j);
      AT(C, ldc, i, j) = alpha * s + c;
    }
}

/* Dense d x d copy of op(T) with zeros outside the (effective) triangle. */
static double *tri_dense(int fill, int op, int d, const double *T, int ldt,
                         int *eff_lower) {
  double *E = (double *)calloc((size_t)d * d + 1, sizeof(double));
  for (int j = 0; j < d; ++j)
    for (int i = 0; i < d; ++i) {
      int in = fill == LO ? i >= j : i <= j;
      if (in) {
        if (op == OPN) E[i + (idx)j * d] = AT(T, ldt, i, j);
        else E[j + (idx)i * d] = AT(T, ldt, i, j);
      }
    }
  *eff_lower = (fill == LO) != (op == OPT);
  return E;
}

/* side L: op(T) X = alpha B (B m x n); side R: X op(T) = alpha B. */
static void o_trsm(int side, int fill, int op, int m, int n, double alpha,
                   const double *T, int ldt, double *B, int ldb) {
  int d = side == SL ? m : n, low;
  double *E = tri_dense(fill, op, d, T, ldt, &low);
  if (side == SL) {
    for (int c = 0; c < n; ++c) {
      if (low) {
        for (int i = 0; i < m; ++i) {
          double s = alpha * AT(B, ldb, i, c);
          for (int l = 0; l < i; ++l) s -= E[i + (idx)l * d] * AT(B, ldb, l, c);
          AT(B, ldb, i, c) = s / E[i + (idx)i * d];
        }
      } else {
        for (int i = m - 1; i >= 0; --i) {
          double s = alpha * AT(B, ldb, i, c);
          for (int l = i + 1; l < m; ++l) s -= E[i + (idx)l * d] * AT(B, ldb, l, c);
          AT(B, ldb, i, c) = s / E[i + (idx)i * d];
        }
      }
    }
  } else {
    /* X E = alpha B  <=>  E^T X^T = alpha B^T: row r of X. */
    for (int r = 0; r < m; ++r) {
      if (low) { /* E lower -> E^T upper: solve last column first */
        for (int j = n - 1; j >= 0; --j) {
          double s = alpha * AT(B, ldb, r, j);
          for (int l = j + 1; l < n; ++l) s -= AT(B, ldb, r, l) * E[l + (idx)j * d];
          AT(B, ldb, r, j) = s / E[j + (idx)j * d];
        }
      } else {
        for (int j = 0; j < n; ++j) {
          double s = alpha * AT(B, ldb, r, j);
          for (int l = 0; l < j; ++l) s -= AT(B, ldb, r, l) * E[l + (idx)j * d];
          AT(B, ldb, r, j) = s / E[j + (idx)j * d];
        }
      }
    }
  }
  free(E);
}

/* LAPACK xPOTRF semantics on the fill triangle; returns info. */
static int o_potrf(int fill, int n, double *A, int lda) {
  for (int j = 0; j < n; ++j) {
    double d = fill == LO ? AT(A, lda, j, j) : AT(A, lda, j, j);
    for (int l = 0; l < j; ++l) {
      double v = fill == LO ? AT(A, lda, j, l) : AT(A, lda, l, j);
      d -= v * v;
    }
    if (!(d > 0.0)) { AT(A, lda, j, j) = d; return j + 1; }
    d = sqrt(d);
    AT(A, lda, j, j) = d;
    for (int i = j + 1; i < n; ++i) {
      double s;
      if (fill == LO) {
        s = AT(A, lda, i, j);
        for (int l = 0; l < j; ++l) s -= AT(A, lda, i, l) * AT(A, lda, j, l);
        AT(A, lda, i, j) = s / d;
      } else {
        s = AT(A, lda, j, i);
        for (int l = 0; l < j; ++l) s -= AT(A, lda, l, i) * AT(A, lda, l, j);
        AT(A, lda, j, i) = s / d;
      }
    }
  }
  return 0;
}

/* LAPACK xPOTRI semantics: inverse of A from its factor (fill triangle). */
static int o_potri(int fill, int n, double *A, int lda) {
  for (int i = 0; i < n; ++i)
    if (AT(A, lda, i, i) == 0.0) return i + 1;
  /* L = factor as lower (L = U^T for fill U) */
  double *L = (double *)calloc((size_t)n * n + 1, sizeof(double));
  double *M = (double *)calloc((size_t)n * n + 1, sizeof(double));
  for (int j = 0; j < n; ++j)
    for (int i = j; i < n; ++i)
      L[i + (idx)j * n] = fill == LO ? AT(A, lda, i, j) : AT(A, lda, j, i);
  /* M = inv(L) */
  for (int c = 0; c < n; ++c)
    for (int i = c; i < n; ++i) {
      double s = (i == c) ? 1.0 : 0.0;
      for (int l = c; l < i; ++l) s -= L[i + (idx)l * n] * M[l + (idx)c * n];
      M[i + (idx)c * n] = s / L[i + (idx)i * n];
    }
  /* inv(A) = M^T M */
  for (int j = 0; j < n; ++j)
    for (int i = j; i < n; ++i) {
      double s = 0.0;
      for (int l = i; l < n; ++l) s += M[l + (idx)i * n] * M[l + (idx)j * n];
      if (fill == LO) AT(A, lda, i, j) = s; else AT(A, lda, j, i) = s;
    }
  free(L);
  free(M);
  return 0;
}

/* side L: C := alpha S B + beta C (S m x m symmetric); side R: alpha B S. */
static void o_symm(int side, int fill, int m, int n, double alpha,
                   const double *S, int lds, const double *B, int ldb,
                   double beta, double *C, int ldc) {
  int d = side == SL ? m : n;
  double *F = (double *)calloc((size_t)d * d + 1, sizeof(double));
  for (int j = 0; j < d; ++j)
    for (int i = 0; i < d; ++i) {
      int in = fill == LO ? i >= j : i <= j;
      if (in) { F[i + (idx)j * d] = AT(S, lds, i, j); F[j + (idx)i * d] = AT(S, lds, i, j); }
    }
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) {
      double s = 0.0;
      if (side == SL) for (int l = 0; l < m; ++l) s += F[i + (idx)l * d] * AT(B, ldb, l, j);
      else for (int l = 0; l < n; ++l) s += AT(B, ldb, i, l) * F[l + (idx)j * d];
      double c = beta == 0.0 ? 0.0 : beta * AT(C, ldc, i, j);
      AT(C, ldc, i, j) = alpha * s + c;
    }
  free(F);
}

static void split_n(int n, int lower, int *n1, int *n2, int *nk) {
  if (n % 2) {
    if (lower) { *n2 = n / 2; *n1 = n - *n2; }
    else { *n1 = n / 2; *n2 = n - *n1; }
    *nk = 0;
  } else {
    *nk = n / 2; *n1 = *nk; *n2 = *nk;
  }
}

/* ------------------------------------------------------------------------
 * ssfrk — table of reference src/curfp_ssfrk.cpp:52-133, calls :193-209.
 * ---------------------------------------------------------------------- */
typedef struct {
  int fill1, dim1; idx off1;
  int fill2, dim2; idx off2;
  int gm, gn; idx offg; int a1_first;
  idx a2; int ldc;
} frk_t;

static frk_t frk_table(int n, int normal, int lower) {
  int n1, n2, nk;
  split_n(n, lower, &n1, &n2, &nk);
  frk_t p;
  if (n % 2) {
    if (normal) {
      if (lower) { p = (frk_t){LO, n1, 0, UP, n2, n, n2, n1, n1, 0, n1, n}; }
      else       { p = (frk_t){LO, n1, n2, UP, n2, n1, n1, n2, 0, 1, n2 - 1, n}; }
    } else {
      if (lower) { p = (frk_t){UP, n1, 0, LO, n2, 1, n1, n2, (idx)n1 * n1, 1, n1, n1}; }
      else       { p = (frk_t){UP, n1, (idx)n2 * n2, LO, n2, (idx)n1 * n2, n2, n1, 0, 0, n1, n2}; }
    }
  } else {
    if (normal) {
      if (lower) { p = (frk_t){LO, nk, 1, UP, nk, 0, nk, nk, nk + 1, 0, nk, n + 1}; }
      else       { p = (frk_t){LO, nk, nk + 1, UP, nk, nk, nk, nk, 0, 1, nk, n + 1}; }
    } else {
      if (lower) { p = (frk_t){UP, nk, nk, LO, nk, 0, nk, nk, (idx)(nk + 1) * nk, 1, nk, nk}; }
      else       { p = (frk_t){UP, nk, (idx)nk * (nk + 1), LO, nk, (idx)nk * nk, nk, nk, 0, 0, nk, nk}; }
    }
  }
  return p;
}

void orc_ssfrk(int transr, int uplo, int trans, int n, int k, double alpha,
               const double *A, int lda, double beta, double *C) {
  if (n == 0) return;
  if ((alpha == 0.0 || k == 0) && beta == 1.0) return;
  if (alpha == 0.0 && beta == 0.0) { memset(C, 0, sizeof(double) * (size_t)n * (n + 1) / 2); return; }
  frk_t p = frk_table(n, transr == 0, uplo == 0);
  int op = trans == 0 ? OPN : OPT, opt = trans == 0 ? OPT : OPN;
  const double *A1 = A, *A2 = trans == 0 ? A + p.a2 : A + p.a2 * (idx)lda;
  if (alpha == 0.0) k = 0;
  o_syrk(p.fill1, op, p.dim1, k, alpha, A1, lda, beta, C + p.off1, p.ldc);
  o_syrk(p.fill2, op, p.dim2, k, alpha, A2, lda, beta, C + p.off2, p.ldc);
  const double *G1 = p.a1_first ? A1 : A2, *G2 = p.a1_first ? A2 : A1;
  o_gemm(op, opt, p.gm, p.gn, k, alpha, G1, lda, G2, lda, beta, C + p.offg, p.ldc);
}

/* ssfr2k — reference src/curfp_ssfr2k.cpp:121-232 (same table as ssfrk). */
void orc_ssfr2k(int transr, int uplo, int trans, int n, int k, double alpha,
                const double *A, int lda, const double *B, int ldb, double beta,
                double *C) {
  if (n == 0) return;
  if ((alpha == 0.0 || k == 0) && beta == 1.0) return;
  if (alpha == 0.0 && beta == 0.0) { memset(C, 0, sizeof(double) * (size_t)n * (n + 1) / 2); return; }
  frk_t p = frk_table(n, transr == 0, uplo == 0);
  int op = trans == 0 ? OPN : OPT, opt = trans == 0 ? OPT : OPN;
  const double *A1 = A, *A2 = trans == 0 ? A + p.a2 : A + p.a2 * (idx)lda;
  const double *B1 = B, *B2 = trans == 0 ? B + p.a2 : B + p.a2 * (idx)ldb;
  if (alpha == 0.0) k = 0;
  o_syr2k(p.fill1, op, p.dim1, k, alpha, A1, lda, B1, ldb, beta, C + p.off1, p.ldc);
  o_syr2k(p.fill2, op, p.dim2, k, alpha, A2, lda, B2, ldb, beta, C + p.off2, p.ldc);
  const double *Ag1 = p.a1_first ? A1 : A2, *Ag2 = p.a1_first ? A2 : A1;
  const double *Bg1 = p.a1_first ? B1 : B2, *Bg2 = p.a1_first ? B2 : B1;
  o_gemm(op, opt, p.gm, p.gn, k, alpha, Ag1, lda, Bg2, ldb, beta, C + p.offg, p.ldc);
  o_gemm(op, opt, p.gm, p.gn, k, alpha, Bg1, ldb, Ag2, lda, 1.0, C + p.offg, p.ldc);
}

/* strttf / stfttr: which mathematical element every RFP slot holds, read
 * off the ssfrk table (block 1 = C(0:n1,0:n1), block 2 = C(n1:,n1:), gemm
 * block = C12 (a1_first) or C21), restating reference
 * src/curfp_strttf.cu:46-415 / src/curfp_stfttr.cu:24-128.  A is row-major. */
static void rfp_map(int transr, int uplo, int n, void (*fn)(idx, int, int, void *),
                    void *ctx) {
  if (n == 0) return;
  frk_t p = frk_table(n, transr == 0, uplo == 0);
  int n1 = p.dim1;
  for (int j = 0; j < p.dim1; ++j)
    for (int i = 0; i < p.dim1; ++i)
      if (p.fill1 == LO ? i >= j : i <= j) fn(p.off1 + i + (idx)j * p.ldc, i, j, ctx);
  for (int j = 0; j < p.dim2; ++j)
    for (int i = 0; i < p.dim2; ++i)
      if (p.fill2 == LO ? i >= j : i <= j) fn(p.off2 + i + (idx)j * p.ldc, n1 + i, n1 + j, ctx);
  for (int j = 0; j < p.gn; ++j)
    for (int i = 0; i < p.gm; ++i) {
      idx a = p.offg + i + (idx)j * p.ldc;
      if (p.a1_first) fn(a, i, n1 + j, ctx); else fn(a, n1 + i, j, ctx);
    }
}

typedef struct { const double *A; double *arf; idx lda; int upper; int to_rfp; } cp_t;

static void cp_fn(idx a, int r, int c, void *vc) {
  cp_t *t = (cp_t *)vc;
  int hi = r > c ? r : c, lo = r > c ? c : r;
  idx d = t->upper ? (idx)lo * t->lda + hi : (idx)hi * t->lda + lo;
  if (t->to_rfp) t->arf[a] = t->A[d];
  else ((double *)t->A)[d] = t->arf[a];
}

void orc_strttf(int transr, int uplo, int n, const double *A, int lda, double *arf) {
  cp_t t = {A, arf, lda, uplo == 1, 1};
  rfp_map(transr, uplo, n, cp_fn, &t);
}

void orc_stfttr(int transr, int uplo, int n, const double *arf, double *A, int lda) {
  cp_t t = {A, (double *)arf, lda, uplo == 1, 0};
  rfp_map(transr, uplo, n, cp_fn, &t);
}

/* Diagonal offsets: restates curfp/__init__.py:194-269. */
void orc_diag_indices(int transr, int uplo, int n, int64_t *out) {
  int lower = uplo == 0, n1, n2, nk;
  split_n(n, lower, &n1, &n2, &nk);
  idx c = 0;
  if (n % 2) {
    if (transr == 0) {
      idx b1 = lower ? 0 : n2, b2 = lower ? n : n1;
      for (int i = 0; i < n1; ++i) out[c++] = b1 + (idx)i * (n + 1);
      for (int i = 0; i < n2; ++i) out[c++] = b2 + (idx)i * (n + 1);
    } else if (lower) {
      for (int i = 0; i < n1; ++i) out[c++] = (idx)i * (n1 + 1);
      for (int i = 0; i < n2; ++i) out[c++] = 1 + (idx)i * (n1 + 1);
    } else {
      for (int i = 0; i < n1; ++i) out[c++] = (idx)n2 * n2 + (idx)i * (n2 + 1);
      for (int i = 0; i < n2; ++i) out[c++] = (idx)n1 * n2 + (idx)i * (n2 + 1);
    }
  } else {
    if (transr == 0) {
      idx b1 = lower ? 1 : nk + 1, b2 = lower ? 0 : nk;
      for (int i = 0; i < nk; ++i) out[c++] = b1 + (idx)i * (n + 2);
      for (int i = 0; i < nk; ++i) out[c++] = b2 + (idx)i * (n + 2);
    } else {
      idx b1 = lower ? nk : (idx)nk * (nk + 1), b2 = lower ? 0 : (idx)nk * nk;
      for (int i = 0; i < nk; ++i) out[c++] = b1 + (idx)i * (nk + 1);
      for (int i = 0; i < nk; ++i) out[c++] = b2 + (idx)i * (nk + 1);
    }
  }
}

/* ------------------------------------------------------------------------
 * spftrf — table of reference src/curfp_spftrf.cpp:62-180, sequence
 * :254-282 (POTRF T1 -> TRSM S -> SYRK T2 -= S S^T -> POTRF T2).
 * ---------------------------------------------------------------------- */
typedef struct {
  int fill11, dim11; idx off11; int lda11;
  int tside, tfill, top; idx ta, tb; int tm, tn, tlda, tldb;
  int sfill, sop, sn, sk; idx sa; int slda; idx sc; int sldc;
  int fill22, dim22; idx off22; int lda22; int info_off;
} ftrf_t;

static ftrf_t ftrf_table(int n, int normal, int lower) {
  int n1, n2, nk;
  split_n(n, lower, &n1, &n2, &nk);
  ftrf_t p;
  idx N = n;
  if (n % 2) {
    if (normal) {
      if (lower) p = (ftrf_t){LO, n1, 0, n, SR, LO, OPT, 0, n1, n2, n1, n, n,
                              UP, OPN, n2, n1, n1, n, N, n, UP, n2, N, n, n1};
      else       p = (ftrf_t){LO, n1, n2, n, SL, LO, OPN, n2, 0, n1, n2, n, n,
                              UP, OPT, n2, n1, 0, n, n1, n, UP, n2, n1, n, n1};
    } else {
      if (lower) p = (ftrf_t){UP, n1, 0, n1, SL, UP, OPT, 0, (idx)n1 * n1, n1, n2, n1, n1,
                              LO, OPT, n2, n1, (idx)n1 * n1, n1, 1, n1, LO, n2, 1, n1, n1};
      else       p = (ftrf_t){UP, n1, (idx)n2 * n2, n2, SR, UP, OPN, (idx)n2 * n2, 0, n2, n1, n2, n2,
                              LO, OPN, n2, n1, 0, n2, (idx)n1 * n2, n2, LO, n2, (idx)n1 * n2, n2, n1};
    }
  } else {
    if (normal) {
      if (lower) p = (ftrf_t){LO, nk, 1, n + 1, SR, LO, OPT, 1, nk + 1, nk, nk, n + 1, n + 1,
                              UP, OPN, nk, nk, nk + 1, n + 1, 0, n + 1, UP, nk, 0, n + 1, nk};
      else       p = (ftrf_t){LO, nk, nk + 1, n + 1, SL, LO, OPN, nk + 1, 0, nk, nk, n + 1, n + 1,
                              UP, OPT, nk, nk, 0, n + 1, nk, n + 1, UP, nk, nk, n + 1, nk};
    } else {
      if (lower) p = (ftrf_t){UP, nk, nk, nk, SL, UP, OPT, nk, (idx)nk * (nk + 1), nk, nk, nk, nk,
                              LO, OPT, nk, nk, (idx)nk * (nk + 1), nk, 0, nk, LO, nk, 0, nk, nk};
      else       p = (ftrf_t){UP, nk, (idx)nk * (nk + 1), nk, SR, UP, OPN, (idx)nk * (nk + 1), 0, nk, nk, nk, nk,
                              LO, OPN, nk, nk, 0, nk, (idx)nk * nk, nk, LO, nk, (idx)nk * nk, nk, nk};
    }
  }
  return p;
}

int orc_spftrf(int transr, int uplo, int n, double *A) {
  if (n == 0) return 0;
  ftrf_t p = ftrf_table(n, transr == 0, uplo == 0);
  int info = o_potrf(p.fill11, p.dim11, A + p.off11, p.lda11);
  if (info) return info;
  o_trsm(p.tside, p.tfill, p.top, p.tm, p.tn, 1.0, A + p.ta, p.tlda, A + p.tb, p.tldb);
  o_syrk(p.sfill, p.sop, p.sn, p.sk, -1.0, A + p.sa, p.slda, 1.0, A + p.sc, p.sldc);
  info = o_potrf(p.fill22, p.dim22, A + p.off22, p.lda22);
  return info ? info + p.info_off : 0;
}

/* ------------------------------------------------------------------------
 * spftrs — reference src/curfp_spftrs.cpp:60-213 table, :257-299 sequence.
 * The six calls are expressed with the spftrf table: the first-block
 * triangle (T1), the off-diagonal block and the second-block triangle (T2),
 * with the ops the reference table assigns per case.
 * ---------------------------------------------------------------------- */
void orc_spftrs(int transr, int uplo, int n, int nrhs, const double *A,
                double *B, int ldb) {
  if (n == 0 || nrhs == 0) return;
  int lower = uplo == 0, normal = transr == 0, n1, n2, nk;
  split_n(n, lower, &n1, &n2, &nk);
  ftrf_t p = ftrf_table(n, normal, lower);
  /* Per case the reference table (src/curfp_spftrs.cpp:66-212) assigns:
   * forward op on T1 = N when T1 is LOWER-stored, T when UPPER-stored
   * (backward: the other); on T2 = T when UPPER-stored, N when LOWER; the
   * off-diagonal GEMM uses the spftrf TRSM's B block with op N when that
   * TRSM is right-sided and T when left-sided.  The lines below compute
   * exactly those entries from the spftrf table. */
  int t1op = p.fill11 == LO ? OPN : OPT, t6op = t1op == OPN ? OPT : OPN;
  int t3op = p.fill22 == UP ? OPT : OPN, t4op = t3op == OPN ? OPT : OPN;
  /* Off-diagonal: g2 maps block-1 unknowns into block-2 equations. */
  int g2op, g2ld = p.tldb;
  idx g2a = p.tb;
  /* S stores L21 (n2 x n1) when the reference's TRSM is right-sided,
   * U12 = L21^T (n1 x n2) when left-sided (src/curfp_spftrs.cpp:66-212). */
  g2op = p.tside == SR ? OPN : OPT;
  int g5op = g2op == OPN ? OPT : OPN;
  double *B1 = B, *B2 = B + n1;
  o_trsm(SL, p.fill11, t1op, n1, nrhs, 1.0, A + p.off11, p.lda11, B1, ldb);
  o_gemm(g2op, OPN, n2, nrhs, n1, -1.0, A + g2a, g2ld, B1, ldb, 1.0, B2, ldb);
  o_trsm(SL, p.fill22, t3op, n2, nrhs, 1.0, A + p.off22, p.lda22, B2, ldb);
  o_trsm(SL, p.fill22, t4op, n2, nrhs, 1.0, A + p.off22, p.lda22, B2, ldb);
  o_gemm(g5op, OPN, n1, nrhs, n2, -1.0, A + g2a, g2ld, B2, ldb, 1.0, B1, ldb);
  o_trsm(SL, p.fill11, t6op, n1, nrhs, 1.0, A + p.off11, p.lda11, B1, ldb);
}

/* ------------------------------------------------------------------------
 * spftri — reference src/curfp_spftri.cu:159-388 (steps 1-7: G = S-solve,
 * H = T2-solve of G, POTRI(T2), POTRI(T1), T1 += H^T H (or H H^T),
 * S = -P22 G (or -G P22)).  Returns 0, or -1 where the reference returns
 * CURFP_STATUS_EXECUTION_FAILED.
 * ---------------------------------------------------------------------- */
int orc_spftri(int transr, int uplo, int n, double *A) {
  if (n == 0) return 0;
  if (n == 1) { A[0] = 1.0 / (A[0] * A[0]); return 0; }
  ftrf_t p = ftrf_table(n, transr == 0, uplo == 0);
  int m = p.tm, nb = p.tn;
  double *G = (double *)calloc((size_t)m * nb + 1, sizeof(double));
  double *H = (double *)calloc((size_t)m * nb + 1, sizeof(double));
  for (int j = 0; j < nb; ++j)
    for (int i = 0; i < m; ++i) G[i + (idx)j * m] = AT(A + p.tb, p.tldb, i, j);
  int op_opp = p.top == OPT ? OPN : OPT;
  o_trsm(p.tside, p.tfill, op_opp, m, nb, 1.0, A + p.ta, p.tlda, G, m);
  memcpy(H, G, sizeof(double) * (size_t)m * nb);
  int f22u = p.fill22 == UP, sl = p.tside == SL;
  int op_h = (f22u ^ sl) ? OPT : OPN, h_side = sl ? SR : SL;
  o_trsm(h_side, p.fill22, op_h, m, nb, 1.0, A + p.off22, p.lda22, H, m);
  int rc = 0;
  if (o_potri(p.fill22, p.dim22, A + p.off22, p.lda22)) { rc = -1; goto done; }
  if (o_potri(p.fill11, p.dim11, A + p.off11, p.lda11)) { rc = -1; goto done; }
  if (p.tside == SR) o_syrk(p.fill11, OPT, nb, m, 1.0, H, m, 1.0, A + p.off11, p.lda11);
  else o_syrk(p.fill11, OPN, m, nb, 1.0, H, m, 1.0, A + p.off11, p.lda11);
  if (p.tside == SR)
    o_symm(SL, p.fill22, m, nb, -1.0, A + p.off22, p.lda22, G, m, 0.0, A + p.tb, p.tldb);
  else
    o_symm(SR, p.fill22, m, nb, -1.0, A + p.off22, p.lda22, G, m, 0.0, A + p.tb, p.tldb);
done:
  free(G);
  free(H);
  return rc;
}
