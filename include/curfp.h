/*
 * curfp.h — C ABI of the B200-native RFP (Rectangular Full Packed) library.
 *
 * Drop-in for the reference header include/curfp.h of andersx/curfp on the
 * rank-k update + Cholesky + solve path.  Enum names, enum values, status
 * codes, the opaque handle and every routine signature below are the ones the
 * reference declares (cited per declaration), so code compiled against the
 * reference header links against libcurfp_b200.so unchanged for these routines.
 *
 * Differences from the reference header:
 *   - it includes <cuda_runtime.h> only (no cuBLAS / cuSOLVER headers): the
 *     library has no cuBLAS/cuSOLVER dependency;
 *   - routines outside the Cholesky path (slansf, spfcon, ssfmv, ssfmm, ssfr,
 *     ssfr2 and the D-prefix twins) are not declared;
 *   - a block of extension entry points at the end (add_to_diagonal and the
 *     diagonal index map as device kernels, the split-BF16 precision form, and
 *     the adjoint kernels of the differentiation form).  They have no C-level
 *     counterpart in the reference; each comment names the reference Python
 *     function it replaces where there is one.
 *
 * Conventions (same as the reference): all matrices are device pointers;
 * alpha/beta/info are HOST pointers; dense operands are column-major with a
 * leading dimension (cuBLAS convention) except strttf/stfttr, whose full
 * matrix is row-major; every routine enqueues on the handle's stream.
 */
#ifndef CURFP_H
#define CURFP_H

#include <stdint.h>
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes — reference include/curfp.h:14-20. */
typedef enum {
    CURFP_STATUS_SUCCESS          = 0,
    CURFP_STATUS_NOT_INITIALIZED  = 1,
    CURFP_STATUS_ALLOC_FAILED     = 2,
    CURFP_STATUS_INVALID_VALUE    = 3,
    CURFP_STATUS_EXECUTION_FAILED = 4
} curfpStatus_t;

/* Operation (TRANSR / TRANS) — reference include/curfp.h:25-28. */
typedef enum {
    CURFP_OP_N = 0,
    CURFP_OP_T = 1
} curfpOperation_t;

/* Fill mode — reference include/curfp.h:33-36. */
typedef enum {
    CURFP_FILL_MODE_LOWER = 0,
    CURFP_FILL_MODE_UPPER = 1
} curfpFillMode_t;

/* Side of curfpSsfmm — reference include/curfp.h:41-44. */
typedef enum {
    CURFP_SIDE_LEFT  = 0,  /* C = alpha * A * B + beta * C */
    CURFP_SIDE_RIGHT = 1   /* C = alpha * B * A + beta * C */
} curfpSideMode_t;

/* Norm type of curfpSlansf — reference include/curfp.h:47-53. */
typedef enum {
    CURFP_NORM_MAX = 0,  /* max |A(i,j)|                              */
    CURFP_NORM_ONE = 1,  /* max column sum of |A| (= infinity norm)   */
    CURFP_NORM_FRO = 2   /* Frobenius norm                            */
} curfpNormType_t;

/* Opaque handle — reference include/curfp.h:58.  The context holds the
 * stream, the device, a device-side info word, a kernel error word, the math
 * mode of the drop-in routines and grow-only workspaces taken from a memory
 * pool of the handle's own (the device's default pool is not touched). */
typedef struct curfpContext *curfpHandle_t;

/* Handle management — reference include/curfp.h:63-66
 * (src/curfp_handle.cpp:4-51). */
curfpStatus_t curfpCreate(curfpHandle_t *handle);
curfpStatus_t curfpDestroy(curfpHandle_t handle);
curfpStatus_t curfpSetStream(curfpHandle_t handle, cudaStream_t stream);
curfpStatus_t curfpGetStream(curfpHandle_t handle, cudaStream_t *stream);

/* Arithmetic of the contractions (SYRK / GEMM / TRSM and TRMM updates)
 * inside the FP32 routines; set per handle with curfpSetMathMode, or per call
 * through the *Ex entry points below.
 *   CURFP_MATH_SPLIT_BF16 (the handle's default): contractions with
 *     m, n, k >= 128 and m*n*k >= 2.7e8 run on the tcgen05 tensor cores; every
 *     FP32 operand row is scaled by a power of two and split into three
 *     integer BF16 digits, and the six digit products of weight >= 2^-16 are
 *     accumulated exactly per 1024-deep chunk and summed in FP32.  Measured
 *     against FP64 it is more accurate than FP32 FMA (about 2e-7 against
 *     3e-6 relative on a rank-1024 update).  Diagonal blocks, triangular
 *     leaves and smaller updates use FP32 FMA.
 *   CURFP_MATH_FP32: every contraction in FP32 FMA on the SIMT cores (the
 *     arithmetic of the reference's cuBLAS calls in their default math mode).
 * The D-prefix routines always use FP64 FMA. */
typedef enum {
    CURFP_MATH_FP32       = 0,
    CURFP_MATH_SPLIT_BF16 = 1
} curfpMath_t;

/* Math mode of curfpSsfrk, curfpSsfr2k, curfpSpftrf, curfpSpftrs and
 * curfpSpftri on this handle (no counterpart in the reference, whose math
 * is the one of its cuBLAS handle). */
curfpStatus_t curfpSetMathMode(curfpHandle_t handle, curfpMath_t math);
curfpStatus_t curfpGetMathMode(curfpHandle_t handle, curfpMath_t *math);

/* Kernels that wait on other blocks (the wavefront solve, the tensor-core
 * pipeline) give up after about 2 s and set the handle's kernel error word;
 * a routine that launched such a kernel reads the word before it returns
 * (one stream synchronisation) and reports CURFP_STATUS_EXECUTION_FAILED if
 * it was set.  Routines that launched none return without synchronising. */

/* C := alpha*op(A)*op(A)^T + beta*C, C n x n symmetric in RFP.
 * trans = N: A is n x k; trans = T: A is k x n (column-major, lda).
 * Replaces reference include/curfp.h:79-91 (src/curfp_ssfrk.cpp:135-212). */
curfpStatus_t curfpSsfrk(curfpHandle_t handle, curfpOperation_t transr,
                         curfpFillMode_t uplo, curfpOperation_t trans,
                         int n, int k, const float *alpha, const float *A,
                         int lda, const float *beta, float *C);

/* In-place RFP Cholesky: A = L*L^T (lower) or U^T*U (upper).  *info (host)
 * = 0 on success, i > 0 when the leading minor of order i is not positive
 * definite.  Replaces include/curfp.h:105-112 (src/curfp_spftrf.cpp:182-292). */
curfpStatus_t curfpSpftrf(curfpHandle_t handle, curfpOperation_t transr,
                          curfpFillMode_t uplo, int n, float *A, int *info);

/* Solve A*X = B with the RFP factor from curfpSpftrf; B is n x nrhs
 * column-major (ldb), overwritten by X.
 * Replaces include/curfp.h:123-132 (src/curfp_spftrs.cpp:215-302). */
curfpStatus_t curfpSpftrs(curfpHandle_t handle, curfpOperation_t transr,
                          curfpFillMode_t uplo, int n, int nrhs,
                          const float *A, float *B, int ldb);

/* Full row-major n x n (lda >= n) triangle -> RFP.
 * Replaces include/curfp.h:141-149 (src/curfp_strttf.cu:420-462). */
curfpStatus_t curfpSstrttf(curfpHandle_t handle, curfpOperation_t transr,
                           curfpFillMode_t uplo, int n, const float *A,
                           int lda, float *arf);

/* In-place inverse from the RFP Cholesky factor.
 * Replaces include/curfp.h:180-186 (src/curfp_spftri.cu:159-388). */
curfpStatus_t curfpSpftri(curfpHandle_t handle, curfpOperation_t transr,
                          curfpFillMode_t uplo, int n, float *arf);

/* RFP -> triangle of a full row-major n x n (lda >= n); the other triangle is
 * not written.  Replaces include/curfp.h:197-205 (src/curfp_stfttr.cu:134-175). */
curfpStatus_t curfpSstfttr(curfpHandle_t handle, curfpOperation_t transr,
                           curfpFillMode_t uplo, int n, const float *arf,
                           float *A, int lda);

/* C := alpha*(op(A)op(B)^T + op(B)op(A)^T) + beta*C in RFP.
 * Replaces include/curfp.h:305-319 (src/curfp_ssfr2k.cpp:121-232). */
curfpStatus_t curfpSsfr2k(curfpHandle_t handle, curfpOperation_t transr,
                          curfpFillMode_t uplo, curfpOperation_t trans,
                          int n, int k, const float *alpha, const float *A,
                          int lda, const float *B, int ldb, const float *beta,
                          float *C);

/* ===========================================================================
 * Extension entry points (no C-level counterpart in the reference).
 * ===========================================================================*/

/* Diagonal of an RFP matrix: idx[i] = flat RFP offset of element (i,i), as
 * int64 in device memory (n entries).  Replaces the Python function
 * rfp_diag_indices, reference curfp/__init__.py:194-269 (same values). */
curfpStatus_t curfpRfpDiagIndices(curfpHandle_t handle,
                                  curfpOperation_t transr,
                                  curfpFillMode_t uplo, int n, int64_t *idx);

/* arf[(i,i)] += value for i < n: M := M + value*I in RFP, one kernel.
 * Replaces the Python add_to_diagonal, reference curfp/__init__.py:272-296. */
curfpStatus_t curfpSaddToDiagonal(curfpHandle_t handle,
                                  curfpOperation_t transr,
                                  curfpFillMode_t uplo, int n, float value,
                                  float *arf);
curfpStatus_t curfpDaddToDiagonal(curfpHandle_t handle,
                                  curfpOperation_t transr,
                                  curfpFillMode_t uplo, int n, double value,
                                  double *arf);

/* curfpSsfrk with the contraction arithmetic given per call (curfpMath_t). */
curfpStatus_t curfpSsfrkEx(curfpHandle_t handle, curfpOperation_t transr,
                           curfpFillMode_t uplo, curfpOperation_t trans,
                           int n, int k, const float *alpha, const float *A,
                           int lda, const float *beta, float *C,
                           curfpMath_t math);

/* curfpSpftrf with the contraction arithmetic given per call (curfpMath_t). */
curfpStatus_t curfpSpftrfEx(curfpHandle_t handle, curfpOperation_t transr,
                            curfpFillMode_t uplo, int n, float *A, int *info,
                            curfpMath_t math);

/* Factor an RFP matrix held in HOST memory: arf_host (n(n+1)/2 floats, page-
 * locked for the copy to overlap) is copied to the device array arf, which is
 * then factored in place as by curfpSpftrfEx.  If arf_orig is not NULL (it
 * must not be arf), the unfactored matrix is also left there, as the
 * refined solve (curfpSpftrsRefine) needs it; the host array crosses the
 * bus once.  The part of the array the first diagonal block touches is
 * copied first; the rest is copied on an internal stream and waited for only
 * after that block is factored, so for TRANSR = T (where that block occupies
 * its own half of the array) the transfer overlaps the factorization.
 * Synchronises the handle's stream once to read info.  Not in the reference. */
curfpStatus_t curfpSpftrfFromHost(curfpHandle_t handle, curfpOperation_t transr,
                                  curfpFillMode_t uplo, int n, const float *arf_host,
                                  float *arf, float *arf_orig, int *info,
                                  curfpMath_t math);

/* Solve A*X = B with iterative refinement: X0 = spftrs(factor, B), then
 * repeatedly R = B - A*X with the products of the ORIGINAL matrix Aorig (RFP,
 * same transr/uplo) summed in FP64, D = spftrs(factor, R), X += D, for at most
 * max_iter corrections, stopping when max|R| no longer halves or when a
 * correction is below 4 ulp of max|X|.  The solves use split-BF16 tensor-core
 * updates where they are large enough (the FP64 residual carries the
 * accuracy).  B (n x nrhs, column-major, ldb >= n) is overwritten with X;
 * *iters (host, may be NULL) receives the number of corrections applied.
 * Synchronises the stream for each stopping test. */
curfpStatus_t curfpSpftrsRefine(curfpHandle_t handle, curfpOperation_t transr,
                                curfpFillMode_t uplo, int n, int nrhs,
                                const float *Aorig, const float *factor,
                                float *B, int ldb, int max_iter, int *iters);

/* Y := alpha*A*X + beta*Y, A symmetric in RFP (n x n), X and Y n x nrhs
 * column-major; products summed in FP64, each result rounded once. */
curfpStatus_t curfpSsfmmAcc64(curfpHandle_t handle, curfpOperation_t transr,
                              curfpFillMode_t uplo, int n, int nrhs,
                              const float *alpha, const float *A,
                              const float *X, int ldx, const float *beta,
                              float *Y, int ldy);

/* curfpSpftrs without any device allocation on the call path; no
 * counterpart in the reference.  For callers that cannot let the library
 * allocate device memory while they run (their GPU memory is owned by
 * another allocator, or a cudaMalloc's possible synchronisation or failure
 * is not acceptable in their loop).  The solve's scratch (inverted diagonal
 * blocks and wavefront flags) lives in one static device array of
 * 4 MiB + 4 KiB that each GPU loading the library keeps until exit.
 * Limits: n <= 16384, nrhs <= 512 (larger sizes return
 * CURFP_STATUS_INVALID_VALUE).  The array's device address is fetched on the
 * first call per device (make that call before any stream capture).  All
 * calls share the array: calls that overlap on the GPU race. */
curfpStatus_t curfpSpftrsNoAlloc(curfpHandle_t handle, curfpOperation_t transr,
                                 curfpFillMode_t uplo, int n, int nrhs,
                                 const float *A, float *B, int ldb);

/* ---- Differentiation form: adjoints (no counterpart in the reference) ----
 * Cotangents of RFP arrays are RFP arrays of the same variant holding the
 * derivative with respect to each STORED element (an off-diagonal stored
 * element stands for two entries of the symmetric matrix). */

/* Adjoint of curfpSsfrk with respect to A:
 *   Abar := alpha * (tril(Cbar) + tril(Cbar)^T) * op(A),
 * stored like A (n x k column-major for trans = N, k x n for trans = T). */
curfpStatus_t curfpSsfrkBackward(curfpHandle_t handle, curfpOperation_t transr,
                                 curfpFillMode_t uplo, curfpOperation_t trans,
                                 int n, int k, const float *alpha,
                                 const float *A, int lda, const float *Cbar,
                                 float *Abar, int ldabar);

/* Adjoint of curfpSpftrf: L is the factor (as curfpSpftrf leaves it), Lbar
 * the cotangent of its stored elements; Abar receives the cotangent of the
 * stored elements of A.  Computed in RFP layout by a recursive blocked
 * algorithm, in place in Abar (which may alias Lbar, not L): no n x n
 * scratch, only the solves' diagonal-block inverses.  math selects the
 * arithmetic of its triangular solves (CURFP_MATH_SPLIT_BF16: split-BF16
 * tensor-core updates where large). */
curfpStatus_t curfpSpftrfBackward(curfpHandle_t handle, curfpOperation_t transr,
                                  curfpFillMode_t uplo, int n, const float *L,
                                  const float *Lbar, float *Abar,
                                  curfpMath_t math);

/* Adjoint of curfpSpftrs (X = A^-1 B, A = L L^T; X, Xbar, Bbar column-major
 * n x nrhs): Bbar := A^-1 Xbar (Bbar may alias Xbar) and Lbar (RFP, written;
 * NULL skips it) := -tril(Bbar (L^T X)^T + X (L^T Bbar)^T). */
curfpStatus_t curfpSpftrsBackward(curfpHandle_t handle, curfpOperation_t transr,
                                  curfpFillMode_t uplo, int n, int nrhs,
                                  const float *L, const float *X, int ldx,
                                  const float *Xbar, int ldxbar, float *Bbar,
                                  int ldbbar, float *Lbar);

/* Fused gradient of the Gaussian-process negative log marginal likelihood
 *   f = 1/2 y^T C^-1 y + sum_i log L_ii,  C = s X X^T + sigma2 I = L L^T,
 * from the factor L (RFP), X (n x d row-major, ldx >= d) and
 * alpha = C^-1 y (device, n), scaled by the device scalar *g (the incoming
 * gradient of f):
 *   Xbar    := g s (C^-1 X - alpha (X^T alpha)^T)   (n x d row-major, ldxbar)
 *   sums[0] := g/2 (|L^-1 X|_F^2 - |X^T alpha|^2)   (df/ds)
 *   sums[1] := g/2 (|L^-1|_F^2 - |alpha|^2)          (df/dsigma2)
 * sums is device memory (2 doubles).  Inner products are accumulated in
 * FP64.  Uses n*d + n(n+1)/2 floats of handle-owned scratch. */
curfpStatus_t curfpSgpnllBackward(curfpHandle_t handle, curfpOperation_t transr,
                                  curfpFillMode_t uplo, int n, int d, float s,
                                  const float *L, const float *X, int ldx,
                                  const float *alpha, const float *g,
                                  float *Xbar, int ldxbar, double *sums,
                                  curfpMath_t math);

/* Symmetric matrix (RFP) times dense: side = LEFT C := alpha*A*B + beta*C
 * with A m x m; side = RIGHT C := alpha*B*A + beta*C with A n x n.  B, C
 * column-major m x n (ldb, ldc >= m); alpha, beta host pointers.  FP32
 * products on the SIMT GEMM kernels.  Replaces reference include/curfp.h:
 * 334-348 (src/curfp_ssfmm.cpp:108-306). */
curfpStatus_t curfpSsfmm(curfpHandle_t handle, curfpOperation_t transr,
                         curfpFillMode_t uplo, curfpSideMode_t side, int m, int n,
                         const float *alpha, const float *arf, const float *B,
                         int ldb, const float *beta, float *C, int ldc);

/* y := alpha*A*x + beta*y, A symmetric in RFP (n x n), x and y device vectors
 * with BLAS increments (non-zero).  Replaces reference include/curfp.h:
 * 160-172 (src/curfp_ssfmv.cpp:134-255). */
curfpStatus_t curfpSsfmv(curfpHandle_t handle, curfpOperation_t transr,
                         curfpFillMode_t uplo, int n, const float *alpha,
                         const float *arf, const float *x, int incx,
                         const float *beta, float *y, int incy);

/* Rank-1 update C := alpha*x*x^T + C of the RFP matrix (alpha host pointer,
 * x device vector with BLAS increment; alpha = 0 is a no-op).  Replaces
 * reference include/curfp.h:261-270 (src/curfp_ssfr.cpp:99-173). */
curfpStatus_t curfpSsfr(curfpHandle_t handle, curfpOperation_t transr,
                        curfpFillMode_t uplo, int n, const float *alpha,
                        const float *x, int incx, float *arf);

/* Rank-2 update C := alpha*(x*y^T + y*x^T) + C.  Replaces reference
 * include/curfp.h:281-292 (src/curfp_ssfr2.cpp:94-190). */
curfpStatus_t curfpSsfr2(curfpHandle_t handle, curfpOperation_t transr,
                         curfpFillMode_t uplo, int n, const float *alpha,
                         const float *x, int incx, const float *y, int incy,
                         float *arf);

/* *result := the requested norm of the symmetric matrix held in arf (RFP,
 * not a factor).  Waits for the handle's stream (host result).  n = 0 gives
 * 0.  Replaces reference include/curfp.h:219-227 (src/curfp_slansf.cu:
 * 280-435); sums of squares and column sums are accumulated in FP64 and
 * there is no limit of 2^31 elements on MAX / FRO. */
curfpStatus_t curfpSlansf(curfpHandle_t handle, curfpNormType_t norm,
                          curfpOperation_t transr, curfpFillMode_t uplo, int n,
                          const float *arf, float *result);

/* *rcond := 1 / (||A^-1||_1 * anorm) from the RFP Cholesky factor, with
 * ||A^-1||_1 estimated by the Hager-Higham iteration (LAPACK SLACN2, at most
 * 5 iterations, each applying A^-1 by curfpSpftrs to one vector).  *rcond =
 * 0 when n = 0 or anorm = 0.  Replaces reference include/curfp.h:242-250
 * (src/curfp_spfcon.cu:88-271). */
curfpStatus_t curfpSpfcon(curfpHandle_t handle, curfpOperation_t transr,
                          curfpFillMode_t uplo, int n, const float *arf,
                          float anorm, float *rcond);

/* ---------------------------------------------------------------------------
 * D-prefix (FP64) twins — reference include/curfp.h:357-545.  Same planner
 * and kernels as the S routines, instantiated for double (SIMT DFMA
 * contractions), same argument checks and status codes.
 * ---------------------------------------------------------------------------*/
curfpStatus_t curfpDsfrk(curfpHandle_t handle, curfpOperation_t transr,
                         curfpFillMode_t uplo, curfpOperation_t trans, int n,
                         int k, const double *alpha, const double *A, int lda,
                         const double *beta, double *C);
curfpStatus_t curfpDsfr2k(curfpHandle_t handle, curfpOperation_t transr,
                          curfpFillMode_t uplo, curfpOperation_t trans, int n,
                          int k, const double *alpha, const double *A, int lda,
                          const double *B, int ldb, const double *beta,
                          double *C);
curfpStatus_t curfpDpftrf(curfpHandle_t handle, curfpOperation_t transr,
                          curfpFillMode_t uplo, int n, double *A, int *info);
curfpStatus_t curfpDpftrs(curfpHandle_t handle, curfpOperation_t transr,
                          curfpFillMode_t uplo, int n, int nrhs, const double *A,
                          double *B, int ldb);
curfpStatus_t curfpDpftri(curfpHandle_t handle, curfpOperation_t transr,
                          curfpFillMode_t uplo, int n, double *arf);
curfpStatus_t curfpDstrttf(curfpHandle_t handle, curfpOperation_t transr,
                           curfpFillMode_t uplo, int n, const double *A, int lda,
                           double *arf);
curfpStatus_t curfpDstfttr(curfpHandle_t handle, curfpOperation_t transr,
                           curfpFillMode_t uplo, int n, const double *arf,
                           double *A, int lda);
curfpStatus_t curfpDsfmm(curfpHandle_t handle, curfpOperation_t transr,
                         curfpFillMode_t uplo, curfpSideMode_t side, int m, int n,
                         const double *alpha, const double *arf, const double *B,
                         int ldb, const double *beta, double *C, int ldc);
curfpStatus_t curfpDsfmv(curfpHandle_t handle, curfpOperation_t transr,
                         curfpFillMode_t uplo, int n, const double *alpha,
                         const double *arf, const double *x, int incx,
                         const double *beta, double *y, int incy);
curfpStatus_t curfpDsfr(curfpHandle_t handle, curfpOperation_t transr,
                        curfpFillMode_t uplo, int n, const double *alpha,
                        const double *x, int incx, double *arf);
curfpStatus_t curfpDsfr2(curfpHandle_t handle, curfpOperation_t transr,
                         curfpFillMode_t uplo, int n, const double *alpha,
                         const double *x, int incx, const double *y, int incy,
                         double *arf);
curfpStatus_t curfpDlansf(curfpHandle_t handle, curfpNormType_t norm,
                          curfpOperation_t transr, curfpFillMode_t uplo, int n,
                          const double *arf, double *result);
curfpStatus_t curfpDpfcon(curfpHandle_t handle, curfpOperation_t transr,
                          curfpFillMode_t uplo, int n, const double *arf,
                          double anorm, double *rcond);

/* Release the handle's workspaces (staging planes of the split-BF16 path,
 * refinement and adjoint scratch): waits for the handle's stream, frees every
 * buffer and returns the device pool's unused memory to the driver.  The
 * buffers grow again on demand; the next call of a routine re-allocates what
 * it needs.  At n = 131072 the split-BF16 Cholesky stages up to ~52 GB. */
curfpStatus_t curfpReleaseWorkspace(curfpHandle_t handle);

/* Number of kernels launched through this handle since its creation. */
curfpStatus_t curfpGetKernelLaunchCount(curfpHandle_t handle, long long *count);

/* Self-test of the kernels' failure detection (no counterpart in the
 * reference): launches a small wavefront solve whose first block row never
 * runs, so the CTAs of the next rows wait on a flag that nothing sets.  Their
 * waits are bounded: after ~2 s they record error code 5 in the handle's
 * error word and return, and the call reports CURFP_STATUS_EXECUTION_FAILED
 * with *err_code = 5.  The context stays usable.  Takes ~2 s. */
curfpStatus_t curfpDiagWaitTimeout(curfpHandle_t handle, int *err_code);

/* Optional kernel timing: when enabled, every kernel this handle launches is
 * bracketed by CUDA events on its stream and attributed to a kernel class
 * (0 SIMT GEMM, 1 tensor-core contraction, 2 tensor-core operand staging,
 * 3 Cholesky tiles, 4 triangular inverses, 5 L^T L tiles, 6 strttf/stfttr,
 * 7 diagonal helpers, 8 FP64-accumulated symmetric multiply, 9 wavefront
 * triangular solves, 10 norms and condition-estimator vectors).  Enabling (or disabling) clears the records;
 * curfpProfileRead synchronises the stream and returns the summed device
 * milliseconds, algorithmic flops and bytes, and the launch count of one
 * class. */
curfpStatus_t curfpProfileEnable(curfpHandle_t handle, int enable);
curfpStatus_t curfpProfileRead(curfpHandle_t handle, int kclass, double *ms,
                               double *flops, double *bytes,
                               long long *launches);
/* Every record since curfpProfileEnable, 8 doubles each: class, device
 * milliseconds, flops, bytes, and for contractions and solves the shape
 * (m, n, k, output tiles; zeros otherwise).  At most max_records are
 * written; *count receives the number held.  Synchronises the stream. */
curfpStatus_t curfpProfileRecords(curfpHandle_t handle, long long max_records,
                                  long long *count, double *out);

#ifdef __cplusplus
}
#endif

#endif /* CURFP_H */
