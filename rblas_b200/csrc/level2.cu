// level2.cu -- Level-2 BLAS on the GPU: gemv (y := alpha*op(A)*x + beta*y)
// and the rank-1 updates ger / geru / gerc (A := alpha*x*y^T + A), real and
// complex (src/level2.rs:11-104, src/complex2.rs:11-145).
//
// Both read or write each element of A once, so they are bound by HBM
// bandwidth: gemv moves m*n elements, a rank-1 update 2*m*n. A is handled
// through its column-major view (R x C, leading dimension ld): a row-major
// A is the column-major view of its transpose, which swaps the two gemv
// kernels and the roles of x and y in the rank-1 update.
//   * "column sweep" gemv (y_r = sum_c A[r,c] x_c): one thread per row of
//     the view, consecutive threads on consecutive rows (coalesced), the
//     columns split into S ranges when there are too few rows to fill the
//     GPU; each range's partial sums go to a workspace.
//   * "column dot" gemv (y_c = sum_r A[r,c] x_r): one CTA per (column, row
//     range), 256 threads striding down the column, a fixed-order block
//     reduction.
//   * a finalize pass applies rblas's beta pass and alpha: partial sums are
//     added in range order, so results do not depend on timing.
// Within one range the terms are added in rblas's order (fma(a, x, acc) for
// real, acc + a*x with rblas's complex multiply for complex), so a call that
// needs a single range reproduces rblas's gemv for NoTrans column-major
// exactly; other shapes differ from rblas's order within rounding.
// The rank-1 update computes each element as rblas does (alpha*x_i rounded,
// then fma / complex multiply-add), so it matches rblas bit for bit.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/rblas_b200.h"
#include "rb_internal.h"

namespace rb {

namespace {

template <typename T> struct C2 { T re, im; };

__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

// rblas's complex multiply (src/complex.rs:101-111):
// re = fma(a.re, b.re, 0 - a.im*b.im), im = fma(a.re, b.im, a.im*b.re)
template <typename T>
__device__ __forceinline__ C2<T> cmul(C2<T> a, C2<T> b) {
    return {fma(a.re, b.re, sub_rn(T(0), mul_rn(a.im, b.im))), fma(a.re, b.im, mul_rn(a.im, b.re))};
}
template <typename T>
__device__ __forceinline__ C2<T> cadd(C2<T> a, C2<T> b) { return {add_rn(a.re, b.re), add_rn(a.im, b.im)}; }
template <typename T>
__device__ __forceinline__ C2<T> cconj(C2<T> a) { return {a.re, sub_rn(T(0), a.im)}; }

// Element access: real arrays of T, complex arrays of interleaved {re, im}.
template <typename T, bool CX> struct El { using type = T; };
template <typename T> struct El<T, true> { using type = C2<T>; };

template <typename T>
__device__ __forceinline__ T ld_el(const T* p) { return __ldg(p); }
// two scalar loads: a complex array is only guaranteed T's alignment
template <typename T>
__device__ __forceinline__ C2<T> ld_el(const C2<T>* p) {
    const T* q = reinterpret_cast<const T*>(p);
    return {__ldg(q), __ldg(q + 1)};
}

// acc + a*x in rblas's order for its type
template <typename T>
__device__ __forceinline__ T mac(T acc, T a, T x) { return fma(a, x, acc); }
template <typename T>
__device__ __forceinline__ C2<T> mac(C2<T> acc, C2<T> a, C2<T> x) { return cadd(acc, cmul(a, x)); }
template <typename T>
__device__ __forceinline__ T add_el(T a, T b) { return add_rn(a, b); }
template <typename T>
__device__ __forceinline__ C2<T> add_el(C2<T> a, C2<T> b) { return cadd(a, b); }
template <typename T>
__device__ __forceinline__ T conj_el(T a) { return a; }
template <typename T>
__device__ __forceinline__ C2<T> conj_el(C2<T> a) { return cconj(a); }
template <typename T>
__device__ __forceinline__ T zero_el(T*) { return T(0); }
template <typename T>
__device__ __forceinline__ C2<T> zero_el(C2<T>*) { return {T(0), T(0)}; }
template <typename T>
__device__ __forceinline__ T shfl_el(T v, int o) { return __shfl_down_sync(0xffffffffu, v, o); }
template <typename T>
__device__ __forceinline__ C2<T> shfl_el(C2<T> v, int o) {
    return {__shfl_down_sync(0xffffffffu, v.re, o), __shfl_down_sync(0xffffffffu, v.im, o)};
}

constexpr int kL2Threads = 256;

// y_r partial over columns [c0, c1) of range s: ws[s * R + r]. A CTA covers
// kSweepRows consecutive rows (each thread kRowsPerThread of them, 256 apart,
// so every warp load stays one contiguous 256-byte run and the CTA reads
// 8 KB contiguous per f64 column); the accumulators are independent.
constexpr int kRowsPerThread = 4;
constexpr int kSweepRows = kL2Threads * kRowsPerThread;

template <typename E>
__global__ void __launch_bounds__(kL2Threads)
    gemv_sweep_kernel(const E* __restrict__ A, size_t ld, int R, int C, const E* __restrict__ x, long long incx,
                      int conj, int cchunk, E* __restrict__ ws) {
    const int rbase = blockIdx.x * kSweepRows + threadIdx.x;
    const int s = blockIdx.y;
    const int c0 = s * cchunk, c1 = min(C, c0 + cchunk);
    E acc[kRowsPerThread];
    bool live[kRowsPerThread];
#pragma unroll
    for (int q = 0; q < kRowsPerThread; ++q) {
        acc[q] = zero_el(static_cast<E*>(nullptr));
        live[q] = rbase + q * kL2Threads < R;
    }
#pragma unroll 4
    for (int c = c0; c < c1; ++c) {
        const E xc = ld_el(x + static_cast<long long>(c) * incx);
        const E* col = A + static_cast<size_t>(c) * ld + rbase;
#pragma unroll
        for (int q = 0; q < kRowsPerThread; ++q) {
            if (live[q]) {
                E v = ld_el(col + q * kL2Threads);
                if (conj) v = conj_el(v);
                acc[q] = mac(acc[q], v, xc);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < kRowsPerThread; ++q)
        if (live[q]) ws[static_cast<size_t>(s) * R + rbase + q * kL2Threads] = acc[q];
}

// y_c partial over rows [r0, r1) of range s: ws[s * C + c]
template <typename E>
__global__ void __launch_bounds__(kL2Threads)
    gemv_dot_kernel(const E* __restrict__ A, size_t ld, int R, int C, const E* __restrict__ x, long long incx,
                    int conj, int rchunk, E* __restrict__ ws) {
    __shared__ E part[kL2Threads / 32];
    const int c = blockIdx.x, s = blockIdx.y;
    const int r0 = s * rchunk, r1 = min(R, r0 + rchunk);
    const E* a = A + static_cast<size_t>(c) * ld;
    E acc = zero_el(static_cast<E*>(nullptr));
#pragma unroll 8
    for (int r = r0 + threadIdx.x; r < r1; r += kL2Threads) {
        E v = ld_el(a + r);
        if (conj) v = conj_el(v);
        acc = mac(acc, v, ld_el(x + static_cast<long long>(r) * incx));
    }
    // fixed-order reduction: warp tree, then the warps' sums in warp order
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc = add_el(acc, shfl_el(acc, o));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) part[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        E t = part[0];
#pragma unroll
        for (int w = 1; w < kL2Threads / 32; ++w) t = add_el(t, part[w]);
        ws[static_cast<size_t>(s) * C + c] = t;
    }
}

// rblas's beta pass, then y += alpha * (sum of the S partials in range order).
// Real (src/level2.rs:91-104): beta == 1 leaves y, beta == 0 writes 0,
// else beta*y; then y = fma(alpha, acc, y). Complex (src/complex2.rs:31-43):
// the beta pass always runs (beta == 0 writes 0, else beta*y with the
// complex multiply); then y = y + alpha*acc. alpha == 0 stops after the
// beta pass.
// alpha_mode: 0 no alpha step; 1 add alpha * (sum of the S partials);
// 2 add alpha * 0 (rblas still runs the step on an empty sum).
template <typename T>
__global__ void gemv_finalize_real(T* y, long long incy, int len, const T* __restrict__ ws, int S, T alpha, T beta,
                                   int alpha_mode) {
    const int i = blockIdx.x * kL2Threads + threadIdx.x;
    if (i >= len) return;
    T* yp = y + static_cast<long long>(i) * incy;
    T yi = *yp;
    if (beta != T(1)) yi = (beta == T(0)) ? T(0) : mul_rn(beta, yi);
    if (alpha_mode != 0) {
        T acc = T(0);
        if (alpha_mode == 1) {
            acc = ws[i];
            for (int s = 1; s < S; ++s) acc = add_rn(acc, ws[static_cast<size_t>(s) * len + i]);
        }
        yi = fma(alpha, acc, yi);
    }
    *yp = yi;
}

template <typename T>
__global__ void gemv_finalize_cplx(C2<T>* y, long long incy, int len, const C2<T>* __restrict__ ws, int S,
                                   C2<T> alpha, C2<T> beta, int alpha_mode) {
    const int i = blockIdx.x * kL2Threads + threadIdx.x;
    if (i >= len) return;
    C2<T>* yp = y + static_cast<long long>(i) * incy;
    C2<T> yi = *yp;
    const bool beta_zero = beta.re == T(0) && beta.im == T(0);
    yi = beta_zero ? C2<T>{T(0), T(0)} : cmul(beta, yi);
    if (alpha_mode != 0) {
        C2<T> acc{T(0), T(0)};
        if (alpha_mode == 1) {
            acc = ws[i];
            for (int s = 1; s < S; ++s) acc = cadd(acc, ws[static_cast<size_t>(s) * len + i]);
        }
        yi = cadd(yi, cmul(alpha, acc));
    }
    *yp = yi;
}

// A[r, c] (column-major view) += alpha*x (.) y: the x index is the view's
// row when x_on_rows, else its column; y likewise on the other index.
// A CTA covers kSweepRows consecutive rows of a range of columns (each
// thread kRowsPerThread rows, 256 apart), the columns strided by gridDim.y.
template <typename T>
__global__ void __launch_bounds__(kL2Threads)
    ger_real_kernel(T* A, size_t ld, int R, int C, const T* __restrict__ x, long long incx, const T* __restrict__ y,
                    long long incy, T alpha, int x_on_rows) {
    const int rbase = blockIdx.x * kSweepRows + threadIdx.x;
    // the row-indexed factor (alpha*x_i, or y_j) does not depend on the
    // column: computed once per thread and row, with the same operations
    T rowv[kRowsPerThread];
#pragma unroll
    for (int q = 0; q < kRowsPerThread; ++q) {
        const int r = rbase + q * kL2Threads;
        rowv[q] = r < R ? (x_on_rows ? mul_rn(alpha, __ldg(x + static_cast<long long>(r) * incx))  // src/level2.rs:83
                                     : __ldg(y + static_cast<long long>(r) * incy))
                        : T(0);
    }
    // two columns per pass: 2 * kRowsPerThread loads of A in flight
    const int step = gridDim.y;
    for (int c = blockIdx.y; c < C; c += 2 * step) {
        const int c2 = c + step;
        const bool two = c2 < C;
        T* col = A + static_cast<size_t>(c) * ld;
        T* col2 = A + static_cast<size_t>(two ? c2 : c) * ld;
        const T colv = x_on_rows ? __ldg(y + static_cast<long long>(c) * incy)
                                 : mul_rn(alpha, __ldg(x + static_cast<long long>(c) * incx));
        const T colv2 = !two ? T(0)
                        : (x_on_rows ? __ldg(y + static_cast<long long>(c2) * incy)
                                     : mul_rn(alpha, __ldg(x + static_cast<long long>(c2) * incx)));
        T a1[kRowsPerThread], a2[kRowsPerThread];
#pragma unroll
        for (int q = 0; q < kRowsPerThread; ++q) {
            const int r = rbase + q * kL2Threads;
            a1[q] = r < R ? col[r] : T(0);
            a2[q] = (two && r < R) ? col2[r] : T(0);
        }
#pragma unroll
        for (int q = 0; q < kRowsPerThread; ++q) {
            const int r = rbase + q * kL2Threads;
            if (r < R) {
                // axi * y_j + a with axi = alpha*x_i (src/level2.rs:86)
                col[r] = x_on_rows ? fma(rowv[q], colv, a1[q]) : fma(colv, rowv[q], a1[q]);
                if (two) col2[r] = x_on_rows ? fma(rowv[q], colv2, a2[q]) : fma(colv2, rowv[q], a2[q]);
            }
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kL2Threads)
    ger_cplx_kernel(C2<T>* A, size_t ld, int R, int C, const C2<T>* __restrict__ x, long long incx,
                    const C2<T>* __restrict__ y, long long incy, C2<T> alpha, int x_on_rows, int conj) {
    const int rbase = blockIdx.x * kSweepRows + threadIdx.x;
    for (int c = blockIdx.y; c < C; c += gridDim.y) {
        C2<T>* col = A + static_cast<size_t>(c) * ld;
#pragma unroll
        for (int q = 0; q < kRowsPerThread; ++q) {
            const int r = rbase + q * kL2Threads;
            if (r < R) {
                const int xi = x_on_rows ? r : c, yj = x_on_rows ? c : r;
                const C2<T> axi = cmul(alpha, ld_el(x + static_cast<long long>(xi) * incx));  // src/complex2.rs:135
                C2<T> yv = ld_el(y + static_cast<long long>(yj) * incy);
                if (conj) yv = cconj(yv);                                              // src/complex2.rs:137-141
                col[r] = cadd(col[r], cmul(axi, yv));                                  // src/complex2.rs:143
            }
        }
    }
}

int blocks_for(long long n) { return static_cast<int>((n + kL2Threads - 1) / kL2Threads); }

int fail(cudaError_t e, int32_t* ce) {
    if (ce) *ce = static_cast<int32_t>(e);
    return RB_ERR_CUDA;
}

}  // namespace

template <typename T, bool CX>
int gemv_dev(int layout, int trans, size_t m, size_t n, T ar, T ai, const T* A, size_t lda, const T* x,
             long long incx, T br, T bi, T* y, long long incy, cudaStream_t st, int32_t* ce) {
    using E = typename El<T, CX>::type;
    const bool tr = trans != RB_NO_TRANS;
    const size_t leny = tr ? n : m;
    if (leny == 0) return RB_OK;
    if (m > 0x7fffffff || n > 0x7fffffff) return RB_ERR_INVALID_ARG;
    const bool alpha_zero = (ar == T(0)) && (!CX || ai == T(0));
    // column-major view R x C of A; y = view * x ("sweep") or view^T * x ("dot")
    const bool col = layout == RB_COL_MAJOR;
    const int R = static_cast<int>(col ? m : n), Cc = static_cast<int>(col ? n : m);
    const bool sweep = (col && !tr) || (!col && tr);
    const int conj = (CX && trans == RB_CONJ_TRANS) ? 1 : 0;
    const int len = static_cast<int>(leny);
    int S = 1, chunk = 0;
    const int target = 148 * 8;  // CTAs for a full GPU at 8 resident CTAs per SM
    bool have_work = !alpha_zero && R > 0 && Cc > 0;
    if (have_work) {
        if (sweep) {
            const int rb = (R + kSweepRows - 1) / kSweepRows;
            S = std::max(1, std::min((target + rb - 1) / rb, std::max(1, Cc / 16)));
            chunk = (Cc + S - 1) / S;
            S = (Cc + chunk - 1) / chunk;
        } else {
            S = std::max(1, std::min((target + Cc - 1) / Cc, std::max(1, R / 1024)));
            chunk = (R + S - 1) / S;
            S = (R + chunk - 1) / chunk;
        }
    }
    E* ws = nullptr;
    cudaError_t e;
    if (have_work) {
        if ((e = scratch_alloc(&ws, static_cast<size_t>(S) * len * sizeof(E), st)) != cudaSuccess) return fail(e, ce);
        const E* Av = reinterpret_cast<const E*>(A);
        const E* xv = reinterpret_cast<const E*>(x);
        if (sweep)
            gemv_sweep_kernel<E><<<dim3((R + kSweepRows - 1) / kSweepRows, S), kL2Threads, 0, st>>>(
                Av, lda, R, Cc, xv, incx, conj, chunk, ws);
        else
            gemv_dot_kernel<E><<<dim3(Cc, S), kL2Threads, 0, st>>>(Av, lda, R, Cc, xv, incx, conj, chunk, ws);
        count_launch();
    }
    // rblas runs the alpha step on an empty sum too, except for the real
    // Trans loop, which has no step when m == 0 (src/level2.rs:41-60,
    // src/complex2.rs:55-76)
    const int alpha_mode = alpha_zero ? 0 : (have_work ? 1 : ((!CX && tr) ? 0 : 2));
    if constexpr (CX)
        gemv_finalize_cplx<T><<<blocks_for(len), kL2Threads, 0, st>>>(
            reinterpret_cast<C2<T>*>(y), incy, len, reinterpret_cast<const C2<T>*>(ws), S, C2<T>{ar, ai},
            C2<T>{br, bi}, alpha_mode);
    else
        gemv_finalize_real<T><<<blocks_for(len), kL2Threads, 0, st>>>(y, incy, len, ws, S, ar, br, alpha_mode);
    count_launch();
    e = cudaGetLastError();
    if (ws) cudaFreeAsync(ws, st);
    return e == cudaSuccess ? RB_OK : fail(e, ce);
}

template <typename T, bool CX>
int ger_dev(int layout, size_t m, size_t n, T ar, T ai, const T* x, long long incx, const T* y, long long incy, T* A,
            size_t lda, int conj, cudaStream_t st, int32_t* ce) {
    if (m == 0 || n == 0) return RB_OK;
    if ((ar == T(0)) && (!CX || ai == T(0))) return RB_OK;  // src/level2.rs:77-79, src/complex2.rs:128-130
    if (m > 0x7fffffff || n > 0x7fffffff) return RB_ERR_INVALID_ARG;
    const bool col = layout == RB_COL_MAJOR;
    const int R = static_cast<int>(col ? m : n), Cc = static_cast<int>(col ? n : m);
    // about 8 CTAs per SM over the row blocks, each walking a slice of columns
    const int rblocks = (R + kSweepRows - 1) / kSweepRows;
    const dim3 grid(rblocks, std::max(1, std::min({Cc, 65535, (148 * 8 * 4 + rblocks - 1) / rblocks})));
    if constexpr (CX)
        ger_cplx_kernel<T><<<grid, kL2Threads, 0, st>>>(reinterpret_cast<C2<T>*>(A), lda, R, Cc,
                                                        reinterpret_cast<const C2<T>*>(x), incx,
                                                        reinterpret_cast<const C2<T>*>(y), incy, C2<T>{ar, ai},
                                                        col ? 1 : 0, conj);
    else
        ger_real_kernel<T><<<grid, kL2Threads, 0, st>>>(A, lda, R, Cc, x, incx, y, incy, ar, col ? 1 : 0);
    count_launch();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? RB_OK : fail(e, ce);
}

#define RB_L2_INST(T, CX)                                                                                           \
    template int gemv_dev<T, CX>(int, int, size_t, size_t, T, T, const T*, size_t, const T*, long long, T, T, T*, \
                                 long long, cudaStream_t, int32_t*);                                               \
    template int ger_dev<T, CX>(int, size_t, size_t, T, T, const T*, long long, const T*, long long, T*, size_t,   \
                                int, cudaStream_t, int32_t*);
RB_L2_INST(float, false)
RB_L2_INST(double, false)
RB_L2_INST(float, true)
RB_L2_INST(double, true)
#undef RB_L2_INST

}  // namespace rb

// ---- C ABI: device pointers, enqueued on `stream` ---------------------------
using namespace rb;

namespace {

rb_status l2_check(int layout, int trans, size_t m, size_t n, size_t lda, size_t incy_zero_len, rb_error* err) {
    if (err) *err = rb_error{0, 0, 0, 0, 0};
    if ((layout != RB_ROW_MAJOR && layout != RB_COL_MAJOR) || trans < RB_NO_TRANS || trans > RB_CONJ_TRANS) {
        if (err) err->code = RB_ERR_INVALID_ARG;
        return RB_ERR_INVALID_ARG;
    }
    const size_t min_lead = (layout == RB_ROW_MAJOR) ? n : m;
    if (m > 0 && n > 0 && lda < min_lead) {
        if (err) *err = rb_error{RB_ERR_INVALID_LEADING_DIM, 'a', lda, min_lead, 0};
        return RB_ERR_INVALID_LEADING_DIM;
    }
    if (incy_zero_len > 1) {
        if (err) *err = rb_error{RB_ERR_ZERO_STRIDE, 'y', 0, 0, 0};
        return RB_ERR_ZERO_STRIDE;
    }
    return RB_OK;
}

rb_status l2_done(int rc, int32_t ce, rb_error* err) {
    if (rc != RB_OK && err) {
        err->code = rc;
        err->cuda_error = ce;
    }
    return static_cast<rb_status>(rc);
}

template <typename T, bool CX>
rb_status gemv_c(int layout, int trans, size_t m, size_t n, T ar, T ai, const T* a, size_t lda, const T* x,
                 size_t incx, T br, T bi, T* y, size_t incy, void* stream, rb_error* err) {
    const size_t leny = (trans != RB_NO_TRANS) ? n : m;
    const rb_status v = l2_check(layout, trans, m, n, lda, incy == 0 ? leny : 0, err);
    if (v != RB_OK) return v;
    int32_t ce = 0;
    return l2_done(gemv_dev<T, CX>(layout, trans, m, n, ar, ai, a, lda, x, static_cast<long long>(incx), br, bi, y,
                                   static_cast<long long>(incy), static_cast<cudaStream_t>(stream), &ce),
                   ce, err);
}

template <typename T, bool CX>
rb_status ger_c(int layout, size_t m, size_t n, T ar, T ai, const T* x, size_t incx, const T* y, size_t incy, T* a,
                size_t lda, int conj, void* stream, rb_error* err) {
    const rb_status v = l2_check(layout, RB_NO_TRANS, m, n, lda, 0, err);
    if (v != RB_OK) return v;
    int32_t ce = 0;
    return l2_done(ger_dev<T, CX>(layout, m, n, ar, ai, x, static_cast<long long>(incx), y,
                                  static_cast<long long>(incy), a, lda, conj, static_cast<cudaStream_t>(stream), &ce),
                   ce, err);
}

}  // namespace

extern "C" {

rb_status rb_sgemv_dev(rb_layout layout, rb_transpose trans, size_t m, size_t n, float alpha, const float* a,
                       size_t lda, const float* x, size_t incx, float beta, float* y, size_t incy, void* stream,
                       rb_error* err) {
    return gemv_c<float, false>(layout, trans, m, n, alpha, 0.f, a, lda, x, incx, beta, 0.f, y, incy, stream, err);
}
rb_status rb_dgemv_dev(rb_layout layout, rb_transpose trans, size_t m, size_t n, double alpha, const double* a,
                       size_t lda, const double* x, size_t incx, double beta, double* y, size_t incy, void* stream,
                       rb_error* err) {
    return gemv_c<double, false>(layout, trans, m, n, alpha, 0.0, a, lda, x, incx, beta, 0.0, y, incy, stream, err);
}
rb_status rb_cgemv_dev(rb_layout layout, rb_transpose trans, size_t m, size_t n, rb_complex32 alpha,
                       const rb_complex32* a, size_t lda, const rb_complex32* x, size_t incx, rb_complex32 beta,
                       rb_complex32* y, size_t incy, void* stream, rb_error* err) {
    return gemv_c<float, true>(layout, trans, m, n, alpha.re, alpha.im, reinterpret_cast<const float*>(a), lda,
                               reinterpret_cast<const float*>(x), incx, beta.re, beta.im, reinterpret_cast<float*>(y),
                               incy, stream, err);
}
rb_status rb_zgemv_dev(rb_layout layout, rb_transpose trans, size_t m, size_t n, rb_complex64 alpha,
                       const rb_complex64* a, size_t lda, const rb_complex64* x, size_t incx, rb_complex64 beta,
                       rb_complex64* y, size_t incy, void* stream, rb_error* err) {
    return gemv_c<double, true>(layout, trans, m, n, alpha.re, alpha.im, reinterpret_cast<const double*>(a), lda,
                                reinterpret_cast<const double*>(x), incx, beta.re, beta.im,
                                reinterpret_cast<double*>(y), incy, stream, err);
}
rb_status rb_sger_dev(rb_layout layout, size_t m, size_t n, float alpha, const float* x, size_t incx, const float* y,
                      size_t incy, float* a, size_t lda, void* stream, rb_error* err) {
    return ger_c<float, false>(layout, m, n, alpha, 0.f, x, incx, y, incy, a, lda, 0, stream, err);
}
rb_status rb_dger_dev(rb_layout layout, size_t m, size_t n, double alpha, const double* x, size_t incx,
                      const double* y, size_t incy, double* a, size_t lda, void* stream, rb_error* err) {
    return ger_c<double, false>(layout, m, n, alpha, 0.0, x, incx, y, incy, a, lda, 0, stream, err);
}
#define RB_CGER_DEV(NAME, T, CT, CONJ)                                                                              \
    rb_status NAME(rb_layout layout, size_t m, size_t n, CT alpha, const CT* x, size_t incx, const CT* y,           \
                   size_t incy, CT* a, size_t lda, void* stream, rb_error* err) {                                   \
        return ger_c<T, true>(layout, m, n, alpha.re, alpha.im, reinterpret_cast<const T*>(x), incx,                \
                              reinterpret_cast<const T*>(y), incy, reinterpret_cast<T*>(a), lda, CONJ, stream, err);  \
    }
RB_CGER_DEV(rb_cgeru_dev, float, rb_complex32, 0)
RB_CGER_DEV(rb_zgeru_dev, double, rb_complex64, 0)
RB_CGER_DEV(rb_cgerc_dev, float, rb_complex32, 1)
RB_CGER_DEV(rb_zgerc_dev, double, rb_complex64, 1)
#undef RB_CGER_DEV

}  // extern "C"
