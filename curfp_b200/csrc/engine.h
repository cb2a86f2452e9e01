// engine.h — the primitive operations every RFP routine is planned onto, and
// the recursive dense-triangular algorithms (potrf / trsm / trmm / trtri /
// lauum) written against them.
//
// The planner (plan.cpp) only manipulates views and calls an Exec.  The
// product library binds it to the CUDA executor (exec_cuda.cu), which launches
// the sm_100a kernels on the handle's stream.  The host-logic tests bind the
// same planner source to a CPU executor so that view arithmetic, recursion
// splits and masks are checked without a GPU.
#pragma once
#include <stddef.h>
#include <stdint.h>

#include "rfp.h"

namespace rfp {

// C(m x n) := alpha * (A(m x k) B(k x n) + A2(m x k2) B2(k2 x n)) + beta * C
// beta == 0 means C is not read.  k2 == 0 disables the second product.
template <typename T>
struct GemmProbT {
  ViewT<T> A, B, A2, B2, C;
  int m, n, k, k2;
  T alpha, beta;
  int c_lower;  // write only C(i,j) with i >= j (tiles above the diagonal skipped)
  // Triangular operands: 0 = full, 1 = lower (incl. diagonal), 2 = upper
  // (incl. diagonal), 3 = strictly upper (A operands only); elements outside
  // are treated as 0 and never read.  For A (m x k): lower keeps kk <= i,
  // upper kk >= i, strictly upper kk > i.  For B (k x n): lower keeps
  // kk >= j, upper kk <= j.  a_tri/b_tri apply to product 1, a2_tri/b2_tri
  // to product 2.
  int a_tri, b_tri, a2_tri, b2_tri;
  int inplace;  // C aliases B: the executor must read all of B's column block
                // before writing it (the planner guarantees m <= inplace_rows())
  int math;     // 0 = FP32 FMA, 1 = split-BF16 tensor cores (engine may ignore
                // for small problems and for FP64)
};
using GemmProb = GemmProbT<float>;

constexpr int kMaxBatch = 4;

// One output block of a contraction whose two operands are row ranges of the
// same matrix X (rows x k): C := alpha * X[a_row0:+m, :] X[b_row0:+n, :]^T
// + beta * C.  SYRK updates of the RFP blocks and the three blocks of ssfrk
// are of this form, so the operand is staged (split) once for all of them.
template <typename T>
struct SharedTaskT {
  int a_row0, b_row0, m, n;
  ViewT<T> C;
  T alpha, beta;
  int c_lower;  // 1: write only i >= j; 2 (executor-internal): only i <= j
};
using SharedTask = SharedTaskT<float>;

// Non-deduced scalar parameter: the element type comes from the executor.
template <typename T>
struct Id {
  using type = T;
};
template <typename T>
using Scalar = typename Id<T>::type;

// Block sizes of the recursive algorithms.
constexpr int kPotrfTile = 128;  // diagonal Cholesky tiles (executors may take larger ones)
constexpr int kTrsmLeaf = 64;    // TRSM diagonal blocks (inverted, then multiplied)
// Workspace record per 64-row TRSM block: [W_b | M_b], 64 x 64 each
// (W_b = inv(L_bb); M_b = W_b L_{b,b-1}, written by executors whose
// wavefront solve uses it).
constexpr int kInvStride = 2 * kTrsmLeaf * kTrsmLeaf;
constexpr int kTriTile = 64;     // trtri / lauum tiles
constexpr int kAdjTile = 64;     // Cholesky-adjoint diagonal tiles
constexpr int kTrmmLeaf = 64;    // TRMM leaves (masked in-place multiply)
constexpr int kTrsvMaxRhs = 512; // wavefront solve for at most this many RHS
constexpr int kTrsvMaxRhsTc = 64;  // ... when the updates may use the tensor cores
constexpr int kWaveLeaf = 512;   // recursive TRSM hands blocks <= this to the wavefront solve
constexpr int kWaveLeafWide = 512;  // ... when there are more than 4 * kTrsvMaxRhs RHS
constexpr int kWaveLeafWideTc = 512;  // ... and the updates may use the tensor cores
constexpr int kNotSupported = -1;

template <typename T>
class ExecT {
 public:
  virtual ~ExecT() {}
  // Independent problems, executed as one launch where possible.
  virtual int gemm(const GemmProbT<T>* p, int count) = 0;
  // In-place Cholesky of the lower triangle of L (n <= potrf_tile_rows()).
  // On the first non-positive (or NaN) pivot at local column j the device
  // info word becomes min(info, info_base + j + 1) and the tile stops.
  virtual int potrf_tile(ViewT<T> L, int n, int info_base) = 0;
  // Largest diagonal tile potrf_tile takes (a multiple of kPotrfTile); the
  // recursive Cholesky splits down to it.
  virtual int potrf_tile_rows() const { return kPotrfTile; }
  // Called by the RFP factorization once the first diagonal block's work is
  // enqueued and before any work that reads the other blocks: an executor
  // may order that work after data it is still bringing in.
  virtual int after_first_block() { return 0; }
  // Inverses of the diagonal nb x nb blocks of lower L (n x n): block b is
  // written to W + b*nb*nb, column-major with ld nb, zeros above the diagonal.
  // (W: nblk records of kInvStride floats, see kInvStride)
  virtual int trtri_blocks(ViewT<T> L, int n, int nb, T* W) = 0;
  // In-place inverse of lower L (n <= kTriTile).
  virtual int trtri_tile(ViewT<T> L, int n) = 0;
  // In-place L := L^T L (lower triangle; n <= kTriTile).
  virtual int lauum_tile(ViewT<T> L, int n) = 0;
  // Scratch of at least count elements, valid until the next workspace() call.
  virtual T* workspace(size_t count) = 0;
  // Largest m of an in-place GEMM.
  virtual int inplace_rows() const = 0;
  // One-launch triangular solve L X = alpha B for few right-hand sides, with
  // W holding the inverted 64 x 64 diagonal blocks (trtri_blocks).  Returns
  // kNotSupported when the executor has no such path (the planner then uses
  // the recursive blocked solve).
  virtual int trsm_wave(ViewT<T> L, int n, ViewT<T> B, int m, T alpha, const T* W) {
    (void)L; (void)n; (void)B; (void)m; (void)alpha; (void)W;
    return kNotSupported;
  }
  // Adjoint of the Cholesky factorization of one diagonal tile
  // (n <= kAdjTile): L is the factor (lower triangle read), G holds the
  // cotangent of L's stored lower elements on entry and that of the factored
  // matrix's stored lower elements on exit (lower triangle, in place).
  virtual int potrf_adj_tile(ViewT<T> L, ViewT<T> G, int n) = 0;
  // Contractions sharing one operand matrix.  The default lowers them to
  // gemm(); the CUDA executor stages X once for the tensor-core path.
  virtual int gemm_shared(ViewT<T> X, int rows, int k, const SharedTaskT<T>* t, int count,
                          int math) {
    (void)rows;
    GemmProbT<T> p[kMaxBatch];
    if (count > kMaxBatch) return 3;
    for (int i = 0; i < count; ++i) {
      GemmProbT<T>& g = p[i];
      g.A = sub(X, t[i].a_row0, 0);
      g.B = tr(sub(X, t[i].b_row0, 0));
      g.A2 = g.A; g.B2 = g.B;
      g.C = t[i].C;
      g.m = t[i].m; g.n = t[i].n; g.k = k; g.k2 = 0;
      g.alpha = t[i].alpha; g.beta = t[i].beta;
      g.c_lower = t[i].c_lower; g.inplace = 0;
      g.a_tri = g.b_tri = g.a2_tri = g.b2_tri = 0;
      g.math = math;
    }
    return gemm(p, count);
  }
  // Symmetric rank-2k blocks over two operand matrices X, Y (rows x k):
  // C_t := alpha_t (X[a_row0:+m, :] Y[b_row0:+n, :]^T + Y[a_row0:+m, :]
  // X[b_row0:+n, :]^T) + beta_t C_t.  The default lowers them to two-product
  // gemm() problems; the CUDA executor runs large ones as two tensor-core
  // contractions.
  virtual int gemm_pair(ViewT<T> X, ViewT<T> Y, int rows, int k, const SharedTaskT<T>* t,
                        int count, int math) {
    (void)rows;
    GemmProbT<T> p[kMaxBatch];
    if (count > kMaxBatch) return 3;
    for (int i = 0; i < count; ++i) {
      GemmProbT<T>& g = p[i];
      g.A = sub(X, t[i].a_row0, 0);
      g.B = tr(sub(Y, t[i].b_row0, 0));
      g.A2 = sub(Y, t[i].a_row0, 0);
      g.B2 = tr(sub(X, t[i].b_row0, 0));
      g.C = t[i].C;
      g.m = t[i].m; g.n = t[i].n; g.k = k; g.k2 = k;
      g.alpha = t[i].alpha; g.beta = t[i].beta;
      g.c_lower = t[i].c_lower; g.inplace = 0;
      g.a_tri = g.b_tri = g.a2_tri = g.b2_tri = 0;
      g.math = math;
    }
    return gemm(p, count);
  }
};
using Exec = ExecT<float>;

namespace plan {

// L X = alpha B (L n x n lower, non-unit; B n x m), X overwrites B.
template <typename T>
int trsm_lln(ExecT<T>& ex, ViewT<T> L, int n, ViewT<T> B, int m, Scalar<T> alpha, int math = 0);
// op(T) X = alpha B (left) or X op(T) = alpha B (right); B is rows x cols.
template <typename T>
int trsm(ExecT<T>& ex, int left, int lower, int trans, ViewT<T> Tm, ViewT<T> B, int rows,
         int cols, Scalar<T> alpha, int math = 0);
// B := alpha L B (L lower n x n, B n x m).
template <typename T>
int trmm_lln(ExecT<T>& ex, ViewT<T> L, int n, ViewT<T> B, int m, Scalar<T> alpha, int math = 0);
// B := alpha op(T) B (left) or alpha B op(T) (right).
template <typename T>
int trmm(ExecT<T>& ex, int left, int lower, int trans, ViewT<T> Tm, ViewT<T> B, int rows,
         int cols, Scalar<T> alpha, int math = 0);
// In-place lower Cholesky; info_base is added to local failure columns.
template <typename T>
int potrf_lower(ExecT<T>& ex, ViewT<T> A, int n, int info_base, int math = 0);
// In-place inverse of a lower triangular matrix.
template <typename T>
int trtri_lower(ExecT<T>& ex, ViewT<T> L, int n, int math = 0);
// In-place L := L^T L (lower part).
template <typename T>
int lauum_lower(ExecT<T>& ex, ViewT<T> L, int n, int math = 0);

// RFP routines (logical level, all 8 variants through rfp::geometry).
// transr: 0 = N, 1 = T; lower: 1 = L, 0 = U; trans: 0 = N, 1 = T.
template <typename T>
int ssfrk(ExecT<T>& ex, int transr, int lower, int trans, int n, int k,
          Scalar<T> alpha, const T* A, int lda, Scalar<T> beta, T* C,
          int math = 0);
template <typename T>
int ssfr2k(ExecT<T>& ex, int transr, int lower, int trans, int n, int k,
           Scalar<T> alpha, const T* A, int lda, const T* B, int ldb,
           Scalar<T> beta, T* C, int math = 0);
template <typename T>
int spftrf(ExecT<T>& ex, int transr, int lower, int n, T* A, int math = 0);
template <typename T>
int spftrs(ExecT<T>& ex, int transr, int lower, int n, int nrhs, const T* A,
           T* B, int ldb, int math = 0);
template <typename T>
int spftri(ExecT<T>& ex, int transr, int lower, int n, T* A, int math = 0);
// In place: the RFP factor L := L^-1 (the first half of spftri).
template <typename T>
int rfp_trtri(ExecT<T>& ex, int transr, int lower, int n, T* A, int math = 0);

// Building blocks of the adjoints, on the logical lower factor L held in an
// RFP array (all 8 variants):
// L X = alpha B (trans = 0) or L^T X = alpha B (trans = 1), B dense n x m.
template <typename T>
int rfp_trsm(ExecT<T>& ex, int transr, int lower, int n, const T* L, int trans, ViewT<T> B,
             int m, Scalar<T> alpha, int math = 0);
// B := L^T B (B dense n x m).
template <typename T>
int rfp_trmm_t(ExecT<T>& ex, int transr, int lower, int n, const T* L, ViewT<T> B, int m);
// Lower triangle of the logical matrix C (RFP): C := alpha (A1 B1 + A2 B2)
// + beta C with A1, A2 n x k and B1, B2 k x n dense views.
template <typename T>
int rfp_gemm_lower2(ExecT<T>& ex, int transr, int lower, int n, T* C, ViewT<T> A1, ViewT<T> B1,
                    ViewT<T> A2, ViewT<T> B2, int k, Scalar<T> alpha, Scalar<T> beta);
// Adjoint of the Cholesky factorization, in place on the lower triangle
// (recursive blocked algorithm; no scratch beyond the solves' diagonal-block
// inverses).  L is the factor; G holds the cotangent of L's stored lower
// elements on entry and, on exit, the cotangent of the factored matrix's
// stored lower elements (an off-diagonal stored element stands for two
// entries of the symmetric matrix).
template <typename T>
int potrf_adj_lower(ExecT<T>& ex, ViewT<T> L, ViewT<T> G, int n, int math = 0);
// The same for RFP arrays of the same variant: L the factor, G the cotangent
// (overwritten in place).
template <typename T>
int spftrf_adjoint(ExecT<T>& ex, int transr, int lower, int n, const T* L, T* G, int math = 0);
// Y := alpha A X + beta Y for the symmetric matrix A held in the RFP array
// (any variant); X, Y dense n x m views.  alpha == 0 reads neither A nor X.
template <typename T>
int rfp_symm(ExecT<T>& ex, int transr, int lower, int n, const T* A, ViewT<T> X, ViewT<T> Y, int m,
             Scalar<T> alpha, Scalar<T> beta);
// Y := alpha (G_L + G_L^T) X + beta Y where G_L is the stored lower triangle
// (diagonal included, so the diagonal counts twice) of the RFP array G; X, Y
// dense n x m views.
template <typename T>
int rfp_symm_dbl(ExecT<T>& ex, int transr, int lower, int n, const T* G, ViewT<T> X, ViewT<T> Y,
                 int m, Scalar<T> alpha, Scalar<T> beta);

}  // namespace plan
}  // namespace rfp
