/*
 * rblas_b200.h -- C ABI of the B200 (sm_100a) GEMM engine that stands behind
 * rblas's Level-3 API (blasrodri/rblas).
 *
 * Every entry point is extern "C" with plain pointers and sizes. Enum values
 * mirror rblas's Rust enums (src/types.rs). Errors mirror rblas's BlasError
 * (src/error.rs:15-39) and are returned, never raised: a binding that wants
 * rblas's panicking `gemm` unwraps the status itself.
 *
 * Two pointer conventions:
 *   - host entry points (rb_sgemm, ...) take host buffers plus their slice
 *     lengths, exactly the arguments of rblas's slice-based functions; they
 *     copy to the GPU, compute, copy back, and return when C is written.
 *   - device entry points (*_dev) take device pointers and a CUDA stream
 *     (as void*), enqueue, and return without synchronising.
 *
 * Sizes are size_t (Rust usize). Leading dimensions are in elements.
 */
#ifndef RBLAS_B200_H
#define RBLAS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* src/types.rs:9-14 */
typedef enum { RB_ROW_MAJOR = 0, RB_COL_MAJOR = 1 } rb_layout;
/* src/types.rs:30-37 (ConjTrans == Trans for real types, src/types.rs:42-44) */
typedef enum { RB_NO_TRANS = 0, RB_TRANS = 1, RB_CONJ_TRANS = 2 } rb_transpose;
/* src/types.rs:49-54 */
typedef enum { RB_UPPER = 0, RB_LOWER = 1 } rb_uplo;
/* src/types.rs:58-63 */
typedef enum { RB_LEFT = 0, RB_RIGHT = 1 } rb_side;
/* src/types.rs:67-72 */
typedef enum { RB_NON_UNIT = 0, RB_UNIT = 1 } rb_diag;

/* Arithmetic form of a call. PLAIN is the drop-in (true FP32 / FP64
 * products). BF16X3 (f32 only): split each operand into bf16 hi+lo and sum
 * hi*hi + hi*lo + lo*hi on the tensor cores with FP32 accumulation. BF16X6
 * (f32 only): three bf16 planes hi/mid/lo and the six products of weight
 * <= 2. OZAKI (f64 only): INT8 slice emulation with per-row/column
 * power-of-two scaling and exact INT32 slice products; the slice count is
 * rb_set_ozaki_slices(). */
typedef enum {
    RB_PREC_PLAIN = 0,
    RB_PREC_BF16X3 = 1,
    RB_PREC_OZAKI = 2,
    RB_PREC_BF16X6 = 3
} rb_precision;

typedef enum {
    RB_OK = 0,
    RB_ERR_INVALID_LEADING_DIM = 1, /* BlasError::InvalidLeadingDim, src/error.rs:17-24 */
    RB_ERR_BUFFER_TOO_SMALL = 2,    /* BlasError::BufferTooSmall,   src/error.rs:26-33 */
    RB_ERR_ZERO_STRIDE = 3,         /* BlasError::ZeroStride,       src/error.rs:35-38 */
    RB_ERR_INVALID_ARG = 4,         /* enum value out of range, null pointer with nonzero size */
    RB_ERR_UNSUPPORTED = 5,         /* precision form not available for this dtype/op */
    RB_ERR_CUDA = 6,                /* a CUDA runtime/driver call failed (see cuda_error) */
    RB_ERR_ALLOC = 7,               /* device or pinned allocation failed */
    RB_ERR_TIMEOUT = 8,             /* a bounded device-side wait gave up */
    RB_ERR_DEVICE = 9,              /* a kernel reported an error word */
    RB_ERR_BUSY = 10,               /* admission refused (serving budget) */
    RB_ERR_CANCELLED = 11,          /* request cancelled before it ran */
    RB_ERR_SCRATCH_LIMIT = 12       /* problem needs more than the fixed no-allocation scratch */
} rb_status;

/* Mirrors BlasError's fields: which operand ('a', 'b', 'c', 'x', 'y'),
 * the value supplied and the minimum (InvalidLeadingDim) or required length
 * (BufferTooSmall). cuda_error carries the cudaError_t / CUresult for
 * RB_ERR_CUDA. */
typedef struct {
    int32_t code;
    char which;
    uint64_t got;
    uint64_t min_or_need;
    int32_t cuda_error;
} rb_error;

/* src/complex.rs:17-24: #[repr(C)] Complex<T> { re, im } -- interleaved. */
typedef struct { float re, im; } rb_complex32;
typedef struct { double re, im; } rb_complex64;

/* Human-readable text of a status, in the wording of BlasError's Display
 * (src/error.rs:41-57) for the validation errors. */
const char* rb_status_string(int32_t status);

/* ---------------------------------------------------------------------------
 * Real GEMM: C := alpha * op(A) * op(B) + beta * C
 * ------------------------------------------------------------------------- */

/* Drop-in for level3::try_gemm (src/level3.rs:68-103) over host slices:
 * validates a, b, c in that order with check_matrix's rules
 * (src/level3.rs:107-140), then computes with the plain form
 * (level3::gemm, src/level3.rs:32-62, true FP32 products). */
rb_status rb_sgemm(rb_layout layout, rb_transpose transa, rb_transpose transb, size_t m, size_t n,
                   size_t k, float alpha, const float* a, size_t lda, size_t a_len, const float* b,
                   size_t ldb, size_t b_len, float beta, float* c, size_t ldc, size_t c_len,
                   rb_error* err);
/* Same for f64 (plain form: FP64 products). */
rb_status rb_dgemm(rb_layout layout, rb_transpose transa, rb_transpose transb, size_t m, size_t n,
                   size_t k, double alpha, const double* a, size_t lda, size_t a_len,
                   const double* b, size_t ldb, size_t b_len, double beta, double* c, size_t ldc,
                   size_t c_len, rb_error* err);

/* Host-slice GEMM with a chosen arithmetic form (level3::try_gemm semantics). */
rb_status rb_sgemm_prec(rb_layout layout, rb_transpose transa, rb_transpose transb, size_t m,
                        size_t n, size_t k, float alpha, const float* a, size_t lda, size_t a_len,
                        const float* b, size_t ldb, size_t b_len, float beta, float* c,
                        size_t ldc, size_t c_len, rb_precision prec, rb_error* err);
rb_status rb_dgemm_prec(rb_layout layout, rb_transpose transa, rb_transpose transb, size_t m,
                        size_t n, size_t k, double alpha, const double* a, size_t lda,
                        size_t a_len, const double* b, size_t ldb, size_t b_len, double beta,
                        double* c, size_t ldc, size_t c_len, rb_precision prec, rb_error* err);

/* Device-pointer GEMM (same math as level3::gemm, src/level3.rs:32-62),
 * enqueued on `stream` (a cudaStream_t; NULL = legacy default stream).
 * Leading dimensions are validated (InvalidLeadingDim); buffer lengths are
 * the caller's responsibility. Returns when the work is enqueued.
 * The BF16 forms take stream-ordered scratch for the operands' bf16 planes;
 * for a column-major product (after RowMajor's swap) with A NoTrans,
 * 16-byte aligned, lda a multiple of 4 and n <= 256, A is split inside the
 * GEMM and only B's planes take scratch (same results bit for bit). */
rb_status rb_sgemm_dev(rb_layout layout, rb_transpose transa, rb_transpose transb, size_t m,
                       size_t n, size_t k, float alpha, const float* a, size_t lda,
                       const float* b, size_t ldb, float beta, float* c, size_t ldc,
                       rb_precision prec, void* stream, rb_error* err);
rb_status rb_dgemm_dev(rb_layout layout, rb_transpose transa, rb_transpose transb, size_t m,
                       size_t n, size_t k, double alpha, const double* a, size_t lda,
                       const double* b, size_t ldb, double beta, double* c, size_t ldc,
                       rb_precision prec, void* stream, rb_error* err);

/* ---------------------------------------------------------------------------
 * Complex GEMM (col-major, interleaved {re, im}): C := alpha*op(A)*op(B) + beta*C
 * op = NoTrans / Trans / ConjTrans per operand.
 * ------------------------------------------------------------------------- */

/* Drop-in for complex3::gemm (src/complex3.rs:27-74; C32 = rb_complex32,
 * C64 = rb_complex64). rblas splits into planes and runs four real GEMMs
 * (4M); here the four products share one real GEMM over block operands
 * (same 8mnk flops) and a complex alpha/beta epilogue with rblas's complex
 * multiply. prec: PLAIN, or BF16X3/BF16X6 (C32), OZAKI (C64). The slice
 * lengths are validated like check_matrix (col-major). */
rb_status rb_cgemm(rb_transpose transa, rb_transpose transb, size_t m, size_t n, size_t k,
                   rb_complex32 alpha, const rb_complex32* a, size_t lda, size_t a_len,
                   const rb_complex32* b, size_t ldb, size_t b_len, rb_complex32 beta,
                   rb_complex32* c, size_t ldc, size_t c_len, rb_precision prec, rb_error* err);
rb_status rb_zgemm(rb_transpose transa, rb_transpose transb, size_t m, size_t n, size_t k,
                   rb_complex64 alpha, const rb_complex64* a, size_t lda, size_t a_len,
                   const rb_complex64* b, size_t ldb, size_t b_len, rb_complex64 beta,
                   rb_complex64* c, size_t ldc, size_t c_len, rb_precision prec, rb_error* err);
/* Device-pointer twins (enqueue on `stream`, no synchronisation). */
rb_status rb_cgemm_dev(rb_transpose transa, rb_transpose transb, size_t m, size_t n, size_t k,
                       rb_complex32 alpha, const rb_complex32* a, size_t lda, const rb_complex32* b,
                       size_t ldb, rb_complex32 beta, rb_complex32* c, size_t ldc,
                       rb_precision prec, void* stream, rb_error* err);
rb_status rb_zgemm_dev(rb_transpose transa, rb_transpose transb, size_t m, size_t n, size_t k,
                       rb_complex64 alpha, const rb_complex64* a, size_t lda, const rb_complex64* b,
                       size_t ldb, rb_complex64 beta, rb_complex64* c, size_t ldc,
                       rb_precision prec, void* stream, rb_error* err);

/* ---------------------------------------------------------------------------
 * syrk / symm / hemm / trsm (col-major), routed through the GEMM kernels
 * ------------------------------------------------------------------------- */

/* level3::syrk (src/level3.rs:236-294): C := alpha*op(A)*op(A)^T + beta*C on
 * the uplo triangle of the n x n C only; op(A) is n x k. */
rb_status rb_ssyrk(rb_uplo uplo, rb_transpose trans, size_t n, size_t k, float alpha,
                   const float* a, size_t lda, size_t a_len, float beta, float* c, size_t ldc,
                   size_t c_len, rb_error* err);
rb_status rb_dsyrk(rb_uplo uplo, rb_transpose trans, size_t n, size_t k, double alpha,
                   const double* a, size_t lda, size_t a_len, double beta, double* c, size_t ldc,
                   size_t c_len, rb_error* err);

/* level3::symm (src/level3.rs:301-354): A symmetric, uplo triangle stored;
 * C := alpha*A*B + beta*C (Left) or alpha*B*A + beta*C (Right). */
rb_status rb_ssymm(rb_side side, rb_uplo uplo, size_t m, size_t n, float alpha, const float* a,
                   size_t lda, size_t a_len, const float* b, size_t ldb, size_t b_len, float beta,
                   float* c, size_t ldc, size_t c_len, rb_error* err);
rb_status rb_dsymm(rb_side side, rb_uplo uplo, size_t m, size_t n, double alpha, const double* a,
                   size_t lda, size_t a_len, const double* b, size_t ldb, size_t b_len, double beta,
                   double* c, size_t ldc, size_t c_len, rb_error* err);
/* complex3::symm (src/complex3.rs:130-145): complex symmetric A = A^T. */
rb_status rb_csymm(rb_side side, rb_uplo uplo, size_t m, size_t n, rb_complex32 alpha,
                   const rb_complex32* a, size_t lda, size_t a_len, const rb_complex32* b,
                   size_t ldb, size_t b_len, rb_complex32 beta, rb_complex32* c, size_t ldc,
                   size_t c_len, rb_error* err);
rb_status rb_zsymm(rb_side side, rb_uplo uplo, size_t m, size_t n, rb_complex64 alpha,
                   const rb_complex64* a, size_t lda, size_t a_len, const rb_complex64* b,
                   size_t ldb, size_t b_len, rb_complex64 beta, rb_complex64* c, size_t ldc,
                   size_t c_len, rb_error* err);
/* complex3::hemm (src/complex3.rs:151-166): Hermitian A = A^H (mirrored half
 * conjugated, diagonal imaginary part taken as zero). */
rb_status rb_chemm(rb_side side, rb_uplo uplo, size_t m, size_t n, rb_complex32 alpha,
                   const rb_complex32* a, size_t lda, size_t a_len, const rb_complex32* b,
                   size_t ldb, size_t b_len, rb_complex32 beta, rb_complex32* c, size_t ldc,
                   size_t c_len, rb_error* err);
rb_status rb_zhemm(rb_side side, rb_uplo uplo, size_t m, size_t n, rb_complex64 alpha,
                   const rb_complex64* a, size_t lda, size_t a_len, const rb_complex64* b,
                   size_t ldb, size_t b_len, rb_complex64 beta, rb_complex64* c, size_t ldc,
                   size_t c_len, rb_error* err);

/* level3::trsm (src/level3.rs:390-437) and complex3::trsm
 * (src/complex3.rs:252-340): op(A)*X = alpha*B (Left) or X*op(A) = alpha*B
 * (Right), B overwritten by X. Blocked: diagonal blocks by substitution,
 * off-diagonal updates as GEMMs. */
rb_status rb_strsm(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m,
                   size_t n, float alpha, const float* a, size_t lda, size_t a_len, float* b,
                   size_t ldb, size_t b_len, rb_error* err);
rb_status rb_dtrsm(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m,
                   size_t n, double alpha, const double* a, size_t lda, size_t a_len, double* b,
                   size_t ldb, size_t b_len, rb_error* err);
rb_status rb_ctrsm(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m,
                   size_t n, rb_complex32 alpha, const rb_complex32* a, size_t lda, size_t a_len,
                   rb_complex32* b, size_t ldb, size_t b_len, rb_error* err);
rb_status rb_ztrsm(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m,
                   size_t n, rb_complex64 alpha, const rb_complex64* a, size_t lda, size_t a_len,
                   rb_complex64* b, size_t ldb, size_t b_len, rb_error* err);
/* Device-pointer f64 trsm (enqueue on `stream`). */
rb_status rb_dtrsm_dev(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m,
                       size_t n, double alpha, const double* a, size_t lda, double* b, size_t ldb,
                       void* stream, rb_error* err);

/* ---------------------------------------------------------------------------
 * Level 1: vector-vector routines (level1::axpy / dot / scal / nrm2 / asum /
 * copy / swap, src/level1.rs:17-163; complex1::axpy / dotu / dotc / scal /
 * nrm2, src/complex1.rs:8-112). Vectors are strided (incx, incy in
 * elements). The argument rules follow rblas in its order: n == 0, real axpy
 * with alpha == 0 and real scal with alpha == 1 return at once (reductions
 * give 0); a zero stride is RB_ERR_ZERO_STRIDE where rblas asserts a positive
 * one (axpy, dot, scal, nrm2; src/level1.rs:31,53,78,100, src/complex1.rs:
 * 19,75,90) and is accepted where rblas's loop accepts it (asum, copy, dotu,
 * dotc; copy with incy == 0 leaves x's last element in y[0]); swap with a
 * zero stride and n > 1 is RB_ERR_ZERO_STRIDE (rblas would rotate elements
 * one at a time). Host-slice forms then check each vector reaches its last
 * strided element (RB_ERR_BUFFER_TOO_SMALL, which 'x' / 'y'), where rblas's
 * indexing panics. axpy, scal, copy and swap compute every element exactly
 * as rblas does; dot, dotu, dotc, asum and nrm2 sum in a fixed parallel
 * order (the same result on every call) and agree with rblas's sequential
 * sum within rounding; nrm2 keeps the scaled sum of squares, so it neither
 * overflows nor underflows where rblas does not.
 * ------------------------------------------------------------------------- */

/* y := alpha*x + y. Replaces level1::axpy (src/level1.rs:17-41),
 * complex1::axpy (src/complex1.rs:8-27). */
rb_status rb_saxpy(size_t n, float alpha, const float* x, size_t incx, size_t x_len, float* y, size_t incy,
                   size_t y_len, rb_error* err);
rb_status rb_daxpy(size_t n, double alpha, const double* x, size_t incx, size_t x_len, double* y, size_t incy,
                   size_t y_len, rb_error* err);
rb_status rb_caxpy(size_t n, rb_complex32 alpha, const rb_complex32* x, size_t incx, size_t x_len,
                   rb_complex32* y, size_t incy, size_t y_len, rb_error* err);
rb_status rb_zaxpy(size_t n, rb_complex64 alpha, const rb_complex64* x, size_t incx, size_t x_len,
                   rb_complex64* y, size_t incy, size_t y_len, rb_error* err);
/* x := alpha*x. Replaces level1::scal (src/level1.rs:70-86), complex1::scal
 * (src/complex1.rs:71-81). */
rb_status rb_sscal(size_t n, float alpha, float* x, size_t incx, size_t x_len, rb_error* err);
rb_status rb_dscal(size_t n, double alpha, double* x, size_t incx, size_t x_len, rb_error* err);
rb_status rb_cscal(size_t n, rb_complex32 alpha, rb_complex32* x, size_t incx, size_t x_len, rb_error* err);
rb_status rb_zscal(size_t n, rb_complex64 alpha, rb_complex64* x, size_t incx, size_t x_len, rb_error* err);
/* y := x; x <-> y. Replace level1::copy / swap (src/level1.rs:139-163). */
rb_status rb_scopy(size_t n, const float* x, size_t incx, size_t x_len, float* y, size_t incy, size_t y_len,
                   rb_error* err);
rb_status rb_dcopy(size_t n, const double* x, size_t incx, size_t x_len, double* y, size_t incy, size_t y_len,
                   rb_error* err);
rb_status rb_sswap(size_t n, float* x, size_t incx, size_t x_len, float* y, size_t incy, size_t y_len,
                   rb_error* err);
rb_status rb_dswap(size_t n, double* x, size_t incx, size_t x_len, double* y, size_t incy, size_t y_len,
                   rb_error* err);
/* *result := x^T y. Replaces level1::dot (src/level1.rs:45-66). */
rb_status rb_sdot(size_t n, const float* x, size_t incx, size_t x_len, const float* y, size_t incy, size_t y_len,
                  float* result, rb_error* err);
rb_status rb_ddot(size_t n, const double* x, size_t incx, size_t x_len, const double* y, size_t incy,
                  size_t y_len, double* result, rb_error* err);
/* *result := sum x_i y_i (dotu) or sum conj(x_i) y_i (dotc). Replace
 * complex1::dotu / dotc (src/complex1.rs:31-67). */
rb_status rb_cdotu(size_t n, const rb_complex32* x, size_t incx, size_t x_len, const rb_complex32* y, size_t incy,
                   size_t y_len, rb_complex32* result, rb_error* err);
rb_status rb_zdotu(size_t n, const rb_complex64* x, size_t incx, size_t x_len, const rb_complex64* y, size_t incy,
                   size_t y_len, rb_complex64* result, rb_error* err);
rb_status rb_cdotc(size_t n, const rb_complex32* x, size_t incx, size_t x_len, const rb_complex32* y, size_t incy,
                   size_t y_len, rb_complex32* result, rb_error* err);
rb_status rb_zdotc(size_t n, const rb_complex64* x, size_t incx, size_t x_len, const rb_complex64* y, size_t incy,
                   size_t y_len, rb_complex64* result, rb_error* err);
/* *result := sum |x_i|. Replaces level1::asum (src/level1.rs:127-135). */
rb_status rb_sasum(size_t n, const float* x, size_t incx, size_t x_len, float* result, rb_error* err);
rb_status rb_dasum(size_t n, const double* x, size_t incx, size_t x_len, double* result, rb_error* err);
/* *result := ||x||_2 by the scaled sum of squares. Replaces level1::nrm2
 * (src/level1.rs:96-123), complex1::nrm2 (src/complex1.rs:86-112). */
rb_status rb_snrm2(size_t n, const float* x, size_t incx, size_t x_len, float* result, rb_error* err);
rb_status rb_dnrm2(size_t n, const double* x, size_t incx, size_t x_len, double* result, rb_error* err);
rb_status rb_scnrm2(size_t n, const rb_complex32* x, size_t incx, size_t x_len, float* result, rb_error* err);
rb_status rb_dznrm2(size_t n, const rb_complex64* x, size_t incx, size_t x_len, double* result, rb_error* err);
/* Device-pointer twins, enqueued on `stream` (strides checked; lengths are
 * the caller's). Reductions write their result to device memory. */
rb_status rb_saxpy_dev(size_t n, float alpha, const float* x, size_t incx, float* y, size_t incy, void* stream,
                       rb_error* err);
rb_status rb_daxpy_dev(size_t n, double alpha, const double* x, size_t incx, double* y, size_t incy, void* stream,
                       rb_error* err);
rb_status rb_caxpy_dev(size_t n, rb_complex32 alpha, const rb_complex32* x, size_t incx, rb_complex32* y,
                       size_t incy, void* stream, rb_error* err);
rb_status rb_zaxpy_dev(size_t n, rb_complex64 alpha, const rb_complex64* x, size_t incx, rb_complex64* y,
                       size_t incy, void* stream, rb_error* err);
rb_status rb_sscal_dev(size_t n, float alpha, float* x, size_t incx, void* stream, rb_error* err);
rb_status rb_dscal_dev(size_t n, double alpha, double* x, size_t incx, void* stream, rb_error* err);
rb_status rb_cscal_dev(size_t n, rb_complex32 alpha, rb_complex32* x, size_t incx, void* stream, rb_error* err);
rb_status rb_zscal_dev(size_t n, rb_complex64 alpha, rb_complex64* x, size_t incx, void* stream, rb_error* err);
rb_status rb_scopy_dev(size_t n, const float* x, size_t incx, float* y, size_t incy, void* stream, rb_error* err);
rb_status rb_dcopy_dev(size_t n, const double* x, size_t incx, double* y, size_t incy, void* stream,
                       rb_error* err);
rb_status rb_sswap_dev(size_t n, float* x, size_t incx, float* y, size_t incy, void* stream, rb_error* err);
rb_status rb_dswap_dev(size_t n, double* x, size_t incx, double* y, size_t incy, void* stream, rb_error* err);
rb_status rb_sdot_dev(size_t n, const float* x, size_t incx, const float* y, size_t incy, float* result,
                      void* stream, rb_error* err);
rb_status rb_ddot_dev(size_t n, const double* x, size_t incx, const double* y, size_t incy, double* result,
                      void* stream, rb_error* err);
rb_status rb_cdotu_dev(size_t n, const rb_complex32* x, size_t incx, const rb_complex32* y, size_t incy,
                       rb_complex32* result, void* stream, rb_error* err);
rb_status rb_zdotu_dev(size_t n, const rb_complex64* x, size_t incx, const rb_complex64* y, size_t incy,
                       rb_complex64* result, void* stream, rb_error* err);
rb_status rb_cdotc_dev(size_t n, const rb_complex32* x, size_t incx, const rb_complex32* y, size_t incy,
                       rb_complex32* result, void* stream, rb_error* err);
rb_status rb_zdotc_dev(size_t n, const rb_complex64* x, size_t incx, const rb_complex64* y, size_t incy,
                       rb_complex64* result, void* stream, rb_error* err);
rb_status rb_sasum_dev(size_t n, const float* x, size_t incx, float* result, void* stream, rb_error* err);
rb_status rb_dasum_dev(size_t n, const double* x, size_t incx, double* result, void* stream, rb_error* err);
rb_status rb_snrm2_dev(size_t n, const float* x, size_t incx, float* result, void* stream, rb_error* err);
rb_status rb_dnrm2_dev(size_t n, const double* x, size_t incx, double* result, void* stream, rb_error* err);
rb_status rb_scnrm2_dev(size_t n, const rb_complex32* x, size_t incx, float* result, void* stream, rb_error* err);
rb_status rb_dznrm2_dev(size_t n, const rb_complex64* x, size_t incx, double* result, void* stream,
                        rb_error* err);

/* ---------------------------------------------------------------------------
 * Level 2: gemv and rank-1 updates (level2::gemv / ger, src/level2.rs:11-88;
 * complex2::gemv / geru / gerc, src/complex2.rs:11-145). x and y are strided
 * (incx, incy in elements; incx may be 0). Host-slice forms check A like
 * check_matrix and each vector against its slice length ('x', 'y'), then
 * return RB_ERR_ZERO_STRIDE for incy == 0 with more than one output (rblas
 * would update one element serially; there is no parallel form). The beta
 * pass follows rblas: real beta == 1 leaves y, beta == 0 writes 0 without
 * reading y; complex always runs it (src/complex2.rs:31-40). alpha == 0
 * stops after the beta pass (gemv) or writes nothing (rank-1 updates).
 * ------------------------------------------------------------------------- */

/* y := alpha*op(A)*x + beta*y; A is m x n in `layout`; op(A) is A for
 * RB_NO_TRANS (x has n elements, y m), A^T for RB_TRANS (x m, y n), A^H for
 * RB_CONJ_TRANS (complex). Replaces level2::gemv (src/level2.rs:11-62) and
 * complex2::gemv (src/complex2.rs:11-77). */
rb_status rb_sgemv(rb_layout layout, rb_transpose trans, size_t m, size_t n, float alpha, const float* a,
                   size_t lda, size_t a_len, const float* x, size_t incx, size_t x_len, float beta, float* y,
                   size_t incy, size_t y_len, rb_error* err);
rb_status rb_dgemv(rb_layout layout, rb_transpose trans, size_t m, size_t n, double alpha, const double* a,
                   size_t lda, size_t a_len, const double* x, size_t incx, size_t x_len, double beta, double* y,
                   size_t incy, size_t y_len, rb_error* err);
rb_status rb_cgemv(rb_layout layout, rb_transpose trans, size_t m, size_t n, rb_complex32 alpha,
                   const rb_complex32* a, size_t lda, size_t a_len, const rb_complex32* x, size_t incx,
                   size_t x_len, rb_complex32 beta, rb_complex32* y, size_t incy, size_t y_len, rb_error* err);
rb_status rb_zgemv(rb_layout layout, rb_transpose trans, size_t m, size_t n, rb_complex64 alpha,
                   const rb_complex64* a, size_t lda, size_t a_len, const rb_complex64* x, size_t incx,
                   size_t x_len, rb_complex64 beta, rb_complex64* y, size_t incy, size_t y_len, rb_error* err);
/* A := alpha*x*y^T + A (A m x n in `layout`, x m elements, y n).
 * Replaces level2::ger (src/level2.rs:65-88); each element is computed as
 * rblas does (fma(alpha*x_i, y_j, a_ij)). */
rb_status rb_sger(rb_layout layout, size_t m, size_t n, float alpha, const float* x, size_t incx, size_t x_len,
                  const float* y, size_t incy, size_t y_len, float* a, size_t lda, size_t a_len, rb_error* err);
rb_status rb_dger(rb_layout layout, size_t m, size_t n, double alpha, const double* x, size_t incx, size_t x_len,
                  const double* y, size_t incy, size_t y_len, double* a, size_t lda, size_t a_len, rb_error* err);
/* A := alpha*x*y^T + A (geru) or alpha*x*y^H + A (gerc): complex2::geru /
 * gerc (src/complex2.rs:80-145), each element as rblas computes it. */
rb_status rb_cgeru(rb_layout layout, size_t m, size_t n, rb_complex32 alpha, const rb_complex32* x, size_t incx,
                   size_t x_len, const rb_complex32* y, size_t incy, size_t y_len, rb_complex32* a, size_t lda,
                   size_t a_len, rb_error* err);
rb_status rb_zgeru(rb_layout layout, size_t m, size_t n, rb_complex64 alpha, const rb_complex64* x, size_t incx,
                   size_t x_len, const rb_complex64* y, size_t incy, size_t y_len, rb_complex64* a, size_t lda,
                   size_t a_len, rb_error* err);
rb_status rb_cgerc(rb_layout layout, size_t m, size_t n, rb_complex32 alpha, const rb_complex32* x, size_t incx,
                   size_t x_len, const rb_complex32* y, size_t incy, size_t y_len, rb_complex32* a, size_t lda,
                   size_t a_len, rb_error* err);
rb_status rb_zgerc(rb_layout layout, size_t m, size_t n, rb_complex64 alpha, const rb_complex64* x, size_t incx,
                   size_t x_len, const rb_complex64* y, size_t incy, size_t y_len, rb_complex64* a, size_t lda,
                   size_t a_len, rb_error* err);
/* Device-pointer twins of the above, enqueued on `stream` (lda checked;
 * buffer lengths are the caller's responsibility). */
rb_status rb_sgemv_dev(rb_layout layout, rb_transpose trans, size_t m, size_t n, float alpha, const float* a,
                       size_t lda, const float* x, size_t incx, float beta, float* y, size_t incy, void* stream,
                       rb_error* err);
rb_status rb_dgemv_dev(rb_layout layout, rb_transpose trans, size_t m, size_t n, double alpha, const double* a,
                       size_t lda, const double* x, size_t incx, double beta, double* y, size_t incy, void* stream,
                       rb_error* err);
rb_status rb_cgemv_dev(rb_layout layout, rb_transpose trans, size_t m, size_t n, rb_complex32 alpha,
                       const rb_complex32* a, size_t lda, const rb_complex32* x, size_t incx, rb_complex32 beta,
                       rb_complex32* y, size_t incy, void* stream, rb_error* err);
rb_status rb_zgemv_dev(rb_layout layout, rb_transpose trans, size_t m, size_t n, rb_complex64 alpha,
                       const rb_complex64* a, size_t lda, const rb_complex64* x, size_t incx, rb_complex64 beta,
                       rb_complex64* y, size_t incy, void* stream, rb_error* err);
rb_status rb_sger_dev(rb_layout layout, size_t m, size_t n, float alpha, const float* x, size_t incx,
                      const float* y, size_t incy, float* a, size_t lda, void* stream, rb_error* err);
rb_status rb_dger_dev(rb_layout layout, size_t m, size_t n, double alpha, const double* x, size_t incx,
                      const double* y, size_t incy, double* a, size_t lda, void* stream, rb_error* err);
rb_status rb_cgeru_dev(rb_layout layout, size_t m, size_t n, rb_complex32 alpha, const rb_complex32* x,
                       size_t incx, const rb_complex32* y, size_t incy, rb_complex32* a, size_t lda, void* stream,
                       rb_error* err);
rb_status rb_zgeru_dev(rb_layout layout, size_t m, size_t n, rb_complex64 alpha, const rb_complex64* x,
                       size_t incx, const rb_complex64* y, size_t incy, rb_complex64* a, size_t lda, void* stream,
                       rb_error* err);
rb_status rb_cgerc_dev(rb_layout layout, size_t m, size_t n, rb_complex32 alpha, const rb_complex32* x,
                       size_t incx, const rb_complex32* y, size_t incy, rb_complex32* a, size_t lda, void* stream,
                       rb_error* err);
rb_status rb_zgerc_dev(rb_layout layout, size_t m, size_t n, rb_complex64 alpha, const rb_complex64* x,
                       size_t incx, const rb_complex64* y, size_t incy, rb_complex64* a, size_t lda, void* stream,
                       rb_error* err);

/* Triangular multiply, B := alpha*op(A)*B (Left, A m x m) or alpha*B*op(A)
 * (Right, A n x n); A triangular (uplo, diag), column-major like trsm.
 * No counterpart in the reference: rblas lists trmm among its remaining
 * Level-3 routines (README.md roadmap); the arguments follow its trsm
 * (src/level3.rs:390-402) and standard BLAS trmm. op(A) is expanded to a
 * full matrix and multiplied in one plain GEMM. */
rb_status rb_strmm(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n,
                   float alpha, const float* a, size_t lda, size_t a_len, float* b, size_t ldb, size_t b_len,
                   rb_error* err);
rb_status rb_dtrmm(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n,
                   double alpha, const double* a, size_t lda, size_t a_len, double* b, size_t ldb, size_t b_len,
                   rb_error* err);
rb_status rb_ctrmm(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n,
                   rb_complex32 alpha, const rb_complex32* a, size_t lda, size_t a_len, rb_complex32* b,
                   size_t ldb, size_t b_len, rb_error* err);
rb_status rb_ztrmm(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n,
                   rb_complex64 alpha, const rb_complex64* a, size_t lda, size_t a_len, rb_complex64* b,
                   size_t ldb, size_t b_len, rb_error* err);
rb_status rb_dtrmm_dev(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n,
                       double alpha, const double* a, size_t lda, double* b, size_t ldb, void* stream,
                       rb_error* err);

/* Batched trsm on device pointers (no counterpart in the reference, which
 * solves one problem per call: trsm, src/level3.rs:390-520). Problem i solves
 * with A_i = a + i*stride_a and B_i = b + i*stride_b (elements), all sharing
 * side, uplo, trans, diag, m, n, alpha, lda, ldb; column-major like rblas.
 * One launch for the batch: each CTA keeps a slice of B_i's right-hand sides
 * in shared memory for the whole solve (32 right-hand sides per CTA up to
 * order 632 f64 / 1512 f32, 16 or 8 up to 2318 f64 / 5546 f32; larger orders
 * fall back to the single-problem path per member). The B_i must not
 * overlap. Enqueued on `stream`. */
rb_status rb_strsm_batched_dev(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m,
                               size_t n, float alpha, const float* a, size_t lda, size_t stride_a, float* b,
                               size_t ldb, size_t stride_b, size_t batch, void* stream, rb_error* err);
rb_status rb_dtrsm_batched_dev(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m,
                               size_t n, double alpha, const double* a, size_t lda, size_t stride_a,
                               double* b, size_t ldb, size_t stride_b, size_t batch, void* stream,
                               rb_error* err);

/* ---------------------------------------------------------------------------
 * Grouped GEMM and the serving loop (no counterpart in the reference: rblas
 * is a synchronous library; these are the batching and serving forms of its
 * gemm, level3::gemm src/level3.rs:32-62, on device-resident operands).
 * ------------------------------------------------------------------------- */

/* One GEMM of a group: C := alpha*op(A)*op(B) + beta*C with device pointers,
 * any layout / transposes, dtype 0 = f32, 1 = f64 (plain form). */
typedef struct {
    int32_t dtype;
    int32_t layout, transa, transb;
    size_t m, n, k;
    double alpha, beta;
    const void* a;
    size_t lda;
    const void* b;
    size_t ldb;
    void* c;
    size_t ldc;
} rb_gemm_problem;

/* Runs every problem of the table in one persistent launch (a device-side
 * problem table with per-problem TMA descriptors; tiles of all problems
 * stream through one pipeline per SM). Problems with m == 0 or n == 0 are
 * skipped; k == 0 or alpha == 0 only scale C. On a validation error
 * err->got is the index of the offending problem. Enqueued on `stream`. */
rb_status rb_gemm_grouped_dev(const rb_gemm_problem* problems, size_t count, void* stream,
                              rb_error* err);
/* The number of K ranges (split-K factor) the grouped kernel cuts this
 * problem into. It depends on the problem's own shape alone, and the K
 * partials are summed in a fixed order, so a problem's result is the same
 * whatever else shares the launch. 0 for an invalid problem. */
int rb_gemm_grouped_splits(const rb_gemm_problem* p);
/* Many f64 GEMMs in the Ozaki form (RB_PREC_OZAKI) in one grouped launch on
 * `stream` (no rblas counterpart; each entry stands for one
 * level3::gemm::<f64>, src/level3.rs:32-62): one exponent pass and one slice
 * pass over every operand, then one persistent tensor-core kernel over the
 * tiles of all problems, longest tiles first. Each result equals that
 * problem's own rb_dgemm_dev(..., RB_PREC_OZAKI, ...) bit for bit. Every
 * entry must be f64 (RB_ERR_UNSUPPORTED, err->got = its index, otherwise);
 * checks as rb_gemm_grouped_dev. Returns once the work is enqueued. */
rb_status rb_gemm_grouped_ozaki_dev(const rb_gemm_problem* problems, size_t count, void* stream,
                                    rb_error* err);
/* The same for f32 problems in a BF16-split form (form RB_PREC_BF16X3 or
 * RB_PREC_BF16X6; each entry one level3::gemm::<f32>): one split pass over
 * every operand, then one persistent tensor-core kernel over the tiles of all
 * problems. Each result equals that problem's own rb_sgemm_dev(..., form,
 * ...) bit for bit. Every entry must be f32 (RB_ERR_UNSUPPORTED, err->got =
 * its index, otherwise); another form is RB_ERR_INVALID_ARG. */
rb_status rb_gemm_grouped_bf16_dev(const rb_gemm_problem* problems, size_t count, rb_precision form,
                                   void* stream, rb_error* err);

/* A grouped launch frozen into a CUDA graph: the problem table (with its
 * TMA descriptors), the split-K workspace and any repack scratch are built
 * and allocated once; rb_gemm_grouped_plan_launch replays the graph on
 * `stream` (counter reset, repacks, the grouped kernel) with no host-side
 * table work. The problems' pointers are fixed at creation; the data they
 * point to may change between launches. Launches of one plan must not
 * overlap on the device (they share the workspace). On a validation error
 * err->got is the index of the offending problem. */
rb_status rb_gemm_grouped_plan_create(const rb_gemm_problem* problems, size_t count, void** plan,
                                      rb_error* err);
rb_status rb_gemm_grouped_plan_launch(void* plan, void* stream, rb_error* err);
rb_status rb_gemm_grouped_plan_destroy(void* plan);

/* Split-K autotuner of the grouped kernel. Times the candidate split
 * factors of every shape bucket (floor(log2) of m, n, k in 32..4096, per
 * dtype) on the current device, installs the winners process-wide and, if
 * cache_path is not NULL, writes them there; *buckets_tuned = buckets timed.
 * Takes seconds and about 1.5 GB of device memory while it runs. Launches
 * planned after the call use the table, so a problem's result depends on its
 * shape and the installed table only. */
rb_status rb_autotune_grouped(const char* cache_path, int* buckets_tuned);
/* Install a table written by rb_autotune_grouped on the same device model
 * (RB_ERR_INVALID_ARG if the file or its device line does not match). */
rb_status rb_autotune_load(const char* cache_path);
/* Back to the built-in split rule. */
rb_status rb_autotune_reset(void);

/* Per-request timestamps (CLOCK_MONOTONIC ns): submitted, admitted into a
 * batch (result memory reserved), finished (batch completion observed). */
typedef struct {
    uint64_t enqueue_ns, admit_ns, finish_ns;
} rb_request_times;

/* A serving loop on the current device. budget_bytes of HBM are reserved
 * up front for results; a request is admitted when its result fits the
 * budget and a batch slot is free (max_batch requests per launch).
 * grouped = 1 packs each admitted set into one grouped launch; grouped = 0
 * launches every request on its own (the per-request baseline). */
rb_status rb_server_create(size_t budget_bytes, int max_batch, int grouped, void** server);
/* Arithmetic forms for large requests: an f32 request of at least
 * f32_min_flop flop (2mnk) runs on its own in f32_form (RB_PREC_PLAIN,
 * RB_PREC_BF16X3 or RB_PREC_BF16X6), an f64 request of at least f64_min_flop
 * in f64_form (RB_PREC_PLAIN or RB_PREC_OZAKI); all other requests take the
 * plain path (grouped or one launch each). Applies to batches formed after
 * the call; default plain. The precision forms take their scratch (digit or
 * split planes) stream-ordered, outside the result budget. */
rb_status rb_server_set_forms(void* server, int f32_form, int f64_form, double f32_min_flop,
                              double f64_min_flop);
/* Queue D = alpha*op(A)*op(B) + beta*C0 where p->c is the device-resident
 * C0 (read only when beta != 0) and D is allocated by the server with C's
 * layout. Returns at once; RB_ERR_BUSY if D could never fit the budget. */
rb_status rb_server_submit(void* server, const rb_gemm_problem* p, uint64_t* id);
/* Wait for a request (timeout_us < 0: forever; 0: poll). On RB_OK, *d_out /
 * *ldd give the result in HBM (valid until rb_server_release). A request
 * whose batch saw the device error word set (a kernel's bounded wait gave up,
 * or a bounds check failed) finishes with RB_ERR_TIMEOUT / RB_ERR_DEVICE and
 * its result must not be used; the server clears the word and goes on. A
 * cancelled request finishes with RB_ERR_CANCELLED. RB_ERR_TIMEOUT is also
 * the answer when timeout_us runs out first (the request is then still
 * pending). */
rb_status rb_server_wait(void* server, uint64_t id, int64_t timeout_us, void** d_out, size_t* ldd,
                         rb_request_times* times);
/* Cancel a request that is still queued (not yet admitted): it never runs,
 * and rb_server_wait reports RB_ERR_CANCELLED for it (release it as usual).
 * RB_ERR_BUSY once it has been admitted (running or finished);
 * RB_ERR_INVALID_ARG for an unknown id. */
rb_status rb_server_cancel(void* server, uint64_t id);
/* Return a finished request's result memory to the budget. */
rb_status rb_server_release(void* server, uint64_t id);
rb_status rb_server_destroy(void* server);
/* Replay a trace: submit problems[i] at arrival_ns[i] after the call starts
 * (a native thread, so the arrival process is not limited by the caller),
 * release each result as it finishes, and fill times[i]. */
rb_status rb_server_run_trace(void* server, const rb_gemm_problem* problems,
                              const uint64_t* arrival_ns, size_t count, rb_request_times* times);

/* ---------------------------------------------------------------------------
 * Allocation-free DGEMM (no counterpart in the reference: rblas runs on the
 * CPU and never touches device memory).
 * ------------------------------------------------------------------------- */

/* Ozaki INT8 DGEMM on device pointers that never allocates: no cudaMalloc,
 * cudaMallocAsync, cudaFree or allocating library call, in this call or on
 * its behalf. For callers that cannot have a library allocate device memory:
 * a process that reserved all of the GPU's memory for its own pool up front,
 * or a latency-critical path where an allocation could block on the device
 * or fail in the middle of a run. All scratch (digit planes, exponents, the
 * kernels' status word) comes from one fixed 64 MiB + 64 KiB device array
 * that every GPU loading this library holds until the process exits.
 *   - Same arithmetic and result as rb_dgemm_dev(..., RB_PREC_OZAKI, ...)
 *     with the current rb_get_ozaki_slices() count; a, b, c, lda/ldb/ldc as
 *     there, enqueued on `stream` (NULL = legacy default stream).
 *   - Limit: 256 + (m+n)*4 + slices*(m+n)*round_up(k,16) bytes (each part
 *     rounded up to 256) must fit the array -- e.g. m = n = k = 2048 at 8
 *     slices; larger problems get RB_ERR_SCRATCH_LIMIT (err->got = bytes
 *     needed, err->min_or_need = bytes available) and touch nothing.
 *   - The first call on a device, with that device current, looks up the
 *     array's device address (cudaGetSymbolAddress), and so does the first
 *     call after that device's context was replaced (cudaDeviceReset); make
 *     that first call before any stream capture.
 *   - Null a or b (with k > 0) or null c: RB_ERR_INVALID_ARG, as for
 *     rb_dgemm_dev.
 *   - Every call shares the array and leaves its contents behind: calls whose
 *     work overlaps on the GPU (different streams, or different host threads)
 *     race on it. The call clears the status word it needs, and returns after
 *     its stream has finished the work, reporting RB_ERR_TIMEOUT /
 *     RB_ERR_DEVICE from the kernels' status word. */
rb_status rb_dgemm_ozaki_noalloc(rb_layout layout, rb_transpose transa, rb_transpose transb,
                                 size_t m, size_t n, size_t k, double alpha, const double* a,
                                 size_t lda, const double* b, size_t ldb, double beta, double* c,
                                 size_t ldc, void* stream, rb_error* err);

/* ---------------------------------------------------------------------------
 * Library state
 * ------------------------------------------------------------------------- */

/* Number of slices used by RB_PREC_OZAKI (2..12; default 8). Each scaled
 * row/column entry y in (-1/2, 1/2) is cut into signed 8-bit digits of
 * weight 2^-(7+8t) (the leading one in [-64, 64], the rest balanced in
 * [-128, 127]), so s slices carry about 7 + 8(s-1) bits; the s(s+1)/2 digit
 * products of weight index <= s-1 are computed. */
rb_status rb_set_ozaki_slices(int slices);
int rb_get_ozaki_slices(void);

/* Kernels this library has launched since load (all devices). */
uint64_t rb_launch_count(void);

/* Reads (and with clear != 0 resets) the current device's error word, set
 * by a kernel whose bounded wait gave up or whose own bounds check failed.
 * Synchronises the device. Returns RB_OK when no error was recorded. */
rb_status rb_device_error(int clear, uint32_t* detail);

/* Parallel width of the GEMM path: the current device's multiprocessor
 * count (each persistent GEMM kernel runs one CTA per SM); 1 when no device
 * is usable, so that like rayon's pool size it is never 0. Replaces
 * level3::num_threads (src/level3.rs:11-17), which reports the size of
 * rblas's rayon pool. */
size_t rb_num_threads(void);

/* Device allocations the library has requested since load, on all devices:
 * scratch-pool blocks, staging buffers, plan tables, serving pools, the
 * per-device error word (no rblas counterpart; rblas's only allocations are
 * its thread-local pack buffers, src/kernel/gemm.rs:58-84). */
uint64_t rb_device_alloc_count(void);

/* Host-side fault injection for tests of the error paths (no rblas
 * counterpart). Nothing here faults, traps or hangs a GPU.
 *   RB_INJECT_ALLOC: the next `count` device allocations the library
 *     requests fail as if the device were out of memory; the call that made
 *     them returns RB_ERR_ALLOC and leaves its outputs untouched. count 0
 *     clears any pending failures; `value` is ignored.
 *   RB_INJECT_DEVICE_WORD: waits for the current device to go idle, then
 *     writes `value` (nonzero, kind << 24 | site as the kernels write it)
 *     into its error word, as a kernel does when a bounded wait gives up.
 *     The next call or serving batch that reads the word reports it
 *     (RB_ERR_TIMEOUT for kind 1, else RB_ERR_DEVICE). `count` is ignored.
 * RB_ERR_INVALID_ARG for an unknown kind, a negative count or a zero word. */
typedef enum { RB_INJECT_ALLOC = 1, RB_INJECT_DEVICE_WORD = 2 } rb_inject_kind;
rb_status rb_debug_inject(int kind, uint32_t value, int count);

/* Self-test of the bounded device waits (no rblas counterpart). Launches one
 * kernel on the current device whose mbarrier wait cannot complete (one
 * arrival expected, none made). The wait gives up after its time limit (2 s)
 * and records the timeout in the device error word. The call clears the
 * word before the launch, reads and clears it afterwards, and returns
 * RB_ERR_TIMEOUT with *detail = the recorded code; any other status means
 * the bound did not work as designed. The device stays usable. */
rb_status rb_probe_wait_timeout(uint32_t* detail);

/* Per-kernel timing of the main GEMM kernels: while enabled, CUDA events are
 * recorded on the launching stream around each main kernel launch.
 * rb_kernel_timing_report synchronises those events, writes one line per
 * kernel ("<name> <launches> <total_ms> <total_work>\n", work in flop or
 * integer ops of the kernel's own pipe) into buf, clears the record and
 * returns the text length (-1 on error). */
void rb_kernel_timing_enable(int on);
int rb_kernel_timing_report(char* buf, size_t buf_len);

/* Releases the cached device/pinned staging buffers of the current device
 * and returns the scratch pool's free blocks to the driver. */
void rb_release_cached_memory(void);
/* Freed scratch (split/digit planes, repacks, problem tables) stays mapped
 * in the library's per-device pool up to this many bytes (default 8 GiB), so
 * that calls after a synchronisation do not map memory again. */
void rb_set_scratch_cache_bytes(size_t bytes);

/* Measures the current GPU's FMA throughput in TFLOP/s (is_f64: FP64 DFMA,
 * else FP32 FFMA; iters <= 0 picks a default). The roofline denominator of
 * the plain forms, which the tensor-core peaks do not cover. -1 on error. */
double rb_probe_fma_peak_tflops(int is_f64, int iters);

/* Measures the tcgen05 tensor-pipe throughput of back-to-back M=128 N=256
 * MMAs with shared-memory operands (no loads in the loop): is_i8 selects
 * kind::i8 (TOP/s) else kind::f16 with bf16 inputs (TFLOP/s). The roofline
 * denominator of the INT8 Ozaki form, for which no vendor-measured figure is
 * at hand. -1 on error. */
double rb_probe_tensor_peak_tflops(int is_i8, int iters);

#ifdef __cplusplus
}
#endif

#endif /* RBLAS_B200_H */
