// level3_ops.cu -- the rest of rblas's Level-3 surface on the GPU, built on
// the library's GEMM kernels:
//
//   complex GEMM (complex3::gemm, src/complex3.rs:27-74): one real GEMM over
//     block operands instead of rblas's four. With op(A) = Ar + i*Ai and
//     op(B) = Br + i*Bi, the real 2m x 2k operand A' holds [[Ar, -Ai],
//     [Ai, Ar]] interleaved by rows and columns (A'[2i][2p] = Ar, A'[2i][2p+1]
//     = -Ai, A'[2i+1][2p] = Ai, A'[2i+1][2p+1] = Ar) and the 2k x n operand B'
//     is op(B) with re/im interleaved down each column -- for op(B) = B that
//     is B's own memory. P' = A' B' is then the interleaved complex product
//     (P'[2i][j] = Re, P'[2i+1][j] = Im): the four real products of the 4M
//     scheme share one pass over the operands; the flop count (8mnk) is the
//     same. A complex epilogue applies alpha/beta with rblas's complex
//     multiply (src/complex.rs:101-111).
//   syrk (src/level3.rs:236-294): the GEMM kernel restricted to the uplo
//     triangle: tiles outside it are skipped, half the work of rblas's full
//     product, and no n x n temporary.
//   symm / hemm (src/level3.rs:301-381, src/complex3.rs:130-247): the stored
//     triangle is mirrored into a full q x q operand on the device (conjugated
//     with a real diagonal for hemm), then GEMM.
//   trsm (src/level3.rs:390-520, src/complex3.rs:252-340): blocked, with
//     64-wide (32 complex) diagonal blocks solved by substitution and the
//     off-diagonal updates done as GEMMs (alpha = -1, beta = 1). rblas solves
//     by scalar substitution only.
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>

#include "../../include/rblas_b200.h"
#include "rb_device.cuh"
#include "rb_internal.h"

namespace rb {

namespace {

inline size_t rup(size_t x, size_t m) { return (x + m - 1) / m * m; }

template <typename T>
__device__ __forceinline__ T fma_t(T a, T b, T c) {
    return fma(a, b, c);
}

// rblas Complex arithmetic (src/complex.rs:101-111)
template <typename T>
__device__ __forceinline__ void cmul(T ar, T ai, T br, T bi, T& re, T& im) {
    re = fma_t(ar, br, T(0) - ai * bi);
    im = fma_t(ar, bi, ai * br);
}

// ---- complex block operands -------------------------------------------------

constexpr int kT = 32;

// A' (2m x 2k, col-major, ld = lda2) from op(A) (complex m x k): trans 0 = A
// stored m x k, 1 = A^T, 2 = A^H (stored k x m). 32 x 32 complex tiles go
// through shared memory so both the read and the write are coalesced.
template <typename T>
__global__ void cplx_expand_a_kernel(const T* __restrict__ a, size_t lda, int trans, int m, int k,
                                     T* __restrict__ out, size_t lda2) {
    __shared__ T re[kT][kT + 1], im[kT][kT + 1];
    const int i0 = blockIdx.x * kT, p0 = blockIdx.y * kT;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int yy = ty; yy < kT; yy += 8) {
        // stored element: NoTrans -> A[i0+tx, p0+yy]; Trans -> A[p0+tx, i0+yy]
        int i, p;
        if (trans == 0) { i = i0 + tx; p = p0 + yy; }
        else            { p = p0 + tx; i = i0 + yy; }
        T vr = T(0), vi = T(0);
        if (i < m && p < k) {
            const size_t off = (trans == 0) ? (static_cast<size_t>(i) + static_cast<size_t>(p) * lda)
                                            : (static_cast<size_t>(p) + static_cast<size_t>(i) * lda);
            vr = a[2 * off];
            vi = a[2 * off + 1];
            if (trans == 2) vi = T(0) - vi;
        }
        if (trans == 0) { re[tx][yy] = vr; im[tx][yy] = vi; }   // [i][p]
        else            { re[yy][tx] = vr; im[yy][tx] = vi; }
    }
    __syncthreads();
    // write: rows 2i, 2i+1 of columns 2p, 2p+1
    for (int yy = ty; yy < kT; yy += 8) {
        const int p = p0 + yy, i = i0 + tx;
        if (p >= k || i >= m) continue;
        const T r = re[tx][yy], v = im[tx][yy];
        T* c0 = out + static_cast<size_t>(2 * p) * lda2 + 2 * i;
        T* c1 = c0 + lda2;
        c0[0] = r;
        c0[1] = v;
        c1[0] = T(0) - v;
        c1[1] = r;
    }
}

// B' (2k x n, col-major, ld = ldb2) from op(B) (complex k x n) for op != NoTrans.
template <typename T>
__global__ void cplx_expand_b_kernel(const T* __restrict__ b, size_t ldb, int trans, int k, int n,
                                     T* __restrict__ out, size_t ldb2) {
    __shared__ T re[kT][kT + 1], im[kT][kT + 1];
    const int p0 = blockIdx.x * kT, j0 = blockIdx.y * kT;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int yy = ty; yy < kT; yy += 8) {
        // stored B is n x k: op(B)(p, j) = B[j, p] -> read along j (contiguous)
        const int j = j0 + tx, p = p0 + yy;
        T vr = T(0), vi = T(0);
        if (j < n && p < k) {
            const size_t off = static_cast<size_t>(j) + static_cast<size_t>(p) * ldb;
            vr = b[2 * off];
            vi = b[2 * off + 1];
            if (trans == 2) vi = T(0) - vi;
        }
        re[yy][tx] = vr;  // [p][j]
        im[yy][tx] = vi;
    }
    __syncthreads();
    for (int yy = ty; yy < kT; yy += 8) {
        const int j = j0 + yy, p = p0 + tx;
        if (j >= n || p >= k) continue;
        T* c = out + static_cast<size_t>(j) * ldb2 + 2 * p;
        c[0] = re[tx][yy];
        c[1] = im[tx][yy];
    }
}

// C = alpha * P + (beta == 0 ? 0 : beta * C), complex, P interleaved 2m x n.
template <typename T>
__global__ void cplx_epilogue_kernel(const T* __restrict__ P, size_t ldp, int m, int n, T ar, T ai,
                                     T br, T bi, T* __restrict__ C, size_t ldc) {
    const bool beta_zero = (br == T(0) && bi == T(0));
    const size_t total = static_cast<size_t>(m) * n;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t j = idx / m, i = idx - j * m;
        const T pr = P[2 * i + j * ldp], pi = P[2 * i + 1 + j * ldp];
        T* c = C + 2 * (i + j * ldc);
        T sr = T(0), si = T(0);
        if (!beta_zero) cmul(br, bi, c[0], c[1], sr, si);
        T qr, qi;
        cmul(ar, ai, pr, pi, qr, qi);
        c[0] = qr + sr;
        c[1] = qi + si;
    }
}

// ---- symmetric / Hermitian expansion ---------------------------------------

// full (q x q, ld = ldf) from the uplo triangle of A (src/level3.rs:359-381,
// src/complex3.rs:190-214). CX: complex interleaved; herm: conjugate mirror
// and real diagonal. One 32 x 32 tile of `full` per CTA (32 x 8 threads):
// the tile is staged from its stored counterpart in A (itself, or the
// transposed tile across the diagonal) with column reads, so both the global
// reads and the writes run down columns; the diagonal tile holds both halves.
constexpr int kSymTile = 32;

template <typename T, bool CX>
struct SymElem {
    T v;
};
template <typename T>
struct SymElem<T, true> {
    T re, im;
};

template <typename T, bool CX>
__global__ void __launch_bounds__(256) sym_expand_kernel(const T* __restrict__ a, size_t lda, int q, int uplo,
                                                         int herm, T* __restrict__ full, size_t ldf) {
    using E = SymElem<T, CX>;
    __shared__ E S[kSymTile][kSymTile + 1];  // S[c][r] = A(r0 + r, c0 + c)
    const int I = blockIdx.x, J = blockIdx.y, tx = threadIdx.x, ty = threadIdx.y;
    // the tile's own position is stored (or on the diagonal): stage it; else
    // stage the tile across the diagonal
    const bool same = (uplo == RB_UPPER) ? (I <= J) : (I >= J);
    const int r0 = (same ? I : J) * kSymTile, c0 = (same ? J : I) * kSymTile;
    for (int k = ty; k < kSymTile; k += 8) {
        const int r = r0 + tx, c = c0 + k;
        if (r < q && c < q) {
            const T* src = a + (CX ? 2 : 1) * (static_cast<size_t>(r) + static_cast<size_t>(c) * lda);
            if constexpr (CX) S[k][tx] = E{src[0], src[1]};
            else S[k][tx] = E{src[0]};
        }
    }
    __syncthreads();
    for (int k = ty; k < kSymTile; k += 8) {
        const int gi = I * kSymTile + tx, gj = J * kSymTile + k;
        if (gi >= q || gj >= q) continue;
        const bool stored = (uplo == RB_UPPER) ? (gi <= gj) : (gi >= gj);
        // A(gi, gj) when stored (own tile: S[k][tx]); else A(gj, gi) (S[tx][k]
        // in the own diagonal tile and in the tile across the diagonal alike)
        E v = (same && stored) ? S[k][tx] : S[tx][k];
        T* dst = full + (CX ? 2 : 1) * (static_cast<size_t>(gi) + static_cast<size_t>(gj) * ldf);
        if constexpr (CX) {
            if (herm) {
                if (gi == gj) v.im = T(0);
                else if (!stored) v.im = T(0) - v.im;
            }
            dst[0] = v.re;
            dst[1] = v.im;
        } else {
            dst[0] = v.v;
        }
    }
}

inline dim3 sym_grid(size_t q) {
    const unsigned t = static_cast<unsigned>((q + kSymTile - 1) / kSymTile);
    return dim3(t, t);
}

// ---- trsm pieces ------------------------------------------------------------

// B := alpha * B over m x n (complex with rblas's multiply).
template <typename T, bool CX>
__global__ void scale_b_kernel(T* __restrict__ b, size_t ldb, int m, int n, T ar, T ai) {
    const size_t total = static_cast<size_t>(m) * n;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t j = idx / m, i = idx - j * m;
        if constexpr (CX) {
            T* p = b + 2 * (i + j * ldb);
            T re, im;
            cmul(ar, ai, p[0], p[1], re, im);
            p[0] = re;
            p[1] = im;
        } else {
            b[i + j * ldb] *= ar;
        }
    }
}

// op(A) of a triangular A expanded to a full q x q column-major matrix:
// the referenced triangle of A (transposed for Trans / ConjTrans, conjugated
// for ConjTrans), zeros outside it, ones on the diagonal for Unit.
template <typename T, bool CX>
__global__ void tri_expand_kernel(const T* __restrict__ a, size_t lda, int q, int uplo, int trans, int diag,
                                  T* __restrict__ full, size_t ldf) {
    constexpr int W = CX ? 2 : 1;
    const size_t total = static_cast<size_t>(q) * q;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t j = idx / q, i = idx - j * q;
        const size_t r = trans ? j : i, c = trans ? i : j;  // stored position of op(A)[i, j]
        const bool stored = (uplo == RB_UPPER) ? (r <= c) : (r >= c);
        T re = T(0), im = T(0);
        if (r == c && diag == RB_UNIT) {
            re = T(1);
        } else if (stored) {
            re = a[W * (r + c * lda)];
            if constexpr (CX) im = (trans == RB_CONJ_TRANS) ? T(0) - a[W * (r + c * lda) + 1] : a[W * (r + c * lda) + 1];
        }
        full[W * (i + j * ldf)] = re;
        if constexpr (CX) full[W * (i + j * ldf) + 1] = im;
    }
}

constexpr int kNbCplx = 32;

// Solve one diagonal block of a complex trsm by substitution for `nvec`
// independent vectors, one thread per vector. The block of op(A) (nb x nb, origin (o, o) in op(A)
// coordinates) is staged in shared memory.
//   side Left : op(A)_blk x = v, v = B[o+t, j] (column j), t < nb.
//   side Right: x op(A)_blk = v, v = B[i, o+t] (row i).
// eff_upper: op(A) is upper triangular. Unit diagonal skips the division.
template <typename T, bool CX>
__global__ void trsm_diag_kernel(int side, int eff_upper, int trans, int diag, int nb, int o,
                                 const T* __restrict__ a, size_t lda, T* __restrict__ b, size_t ldb,
                                 int nvec) {
    constexpr int NB = kNbCplx;
    constexpr int W = CX ? 2 : 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* blk = reinterpret_cast<T*>(smem_raw);  // [r][c] of op(A)_blk, row-major, W components
    for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
        const int r = idx / nb, c = idx - r * nb;
        // op(A)[o+r, o+c] = trans ? A[o+c, o+r] (conj for 2) : A[o+r, o+c]
        const size_t src = trans ? (static_cast<size_t>(o + c) + static_cast<size_t>(o + r) * lda)
                                 : (static_cast<size_t>(o + r) + static_cast<size_t>(o + c) * lda);
        if constexpr (CX) {
            blk[2 * idx] = a[2 * src];
            blk[2 * idx + 1] = (trans == 2) ? T(0) - a[2 * src + 1] : a[2 * src + 1];
        } else {
            blk[idx] = a[src];
        }
    }
    __syncthreads();
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvec) return;
    T x[NB * W];
    // element t of this vector in B
    auto bptr = [&](int t) -> T* {
        const size_t off = (side == RB_LEFT) ? (static_cast<size_t>(o + t) + static_cast<size_t>(v) * ldb)
                                             : (static_cast<size_t>(v) + static_cast<size_t>(o + t) * ldb);
        return b + W * off;
    };
    for (int t = 0; t < nb; ++t) {
        const T* p = bptr(t);
        x[W * t] = p[0];
        if (CX) x[W * t + 1] = p[1];
    }
    // Left: rows of op(A) x = v; Right: x op(A) = v <=> op(A)^T x = v.
    // coef(t, s) is the matrix entry multiplying x_s in equation t.
    const bool forward = (side == RB_LEFT) ? !eff_upper : eff_upper;
    for (int step = 0; step < nb; ++step) {
        const int t = forward ? step : nb - 1 - step;
        T sr = x[W * t], si = CX ? x[W * t + 1] : T(0);
        const int s0 = forward ? 0 : t + 1, s1 = forward ? t : nb;
        for (int s = s0; s < s1; ++s) {
            const int e = (side == RB_LEFT) ? (t * nb + s) : (s * nb + t);
            if constexpr (CX) {
                T pr, pi;
                cmul(blk[2 * e], blk[2 * e + 1], x[2 * s], x[2 * s + 1], pr, pi);
                sr -= pr;
                si -= pi;
            } else {
                sr -= blk[e] * x[s];
            }
        }
        if (diag == RB_NON_UNIT) {
            const int e = t * nb + t;
            if constexpr (CX) {
                // cdiv: a * conj(d) / |d|^2   (src/complex3.rs:344-349)
                const T dr = blk[2 * e], di = blk[2 * e + 1];
                const T dd = fma_t(dr, dr, di * di);
                T nr, ni;
                cmul(sr, si, dr, T(0) - di, nr, ni);
                sr = nr / dd;
                si = ni / dd;
            } else {
                sr = sr / blk[e];
            }
        }
        x[W * t] = sr;
        if (CX) x[W * t + 1] = si;
    }
    for (int t = 0; t < nb; ++t) {
        T* p = bptr(t);
        p[0] = x[W * t];
        if (CX) p[1] = x[W * t + 1];
    }
}

int grid_for(size_t total) {
    size_t b = (total + 255) / 256;
    return static_cast<int>(std::min<size_t>(std::max<size_t>(b, 1), 148 * 32));
}

int fail(cudaError_t e, int32_t* ce) {
    if (ce) *ce = static_cast<int32_t>(e);
    return RB_ERR_CUDA;
}

}  // namespace

// ---------------------------------------------------------------------------
// complex GEMM
// ---------------------------------------------------------------------------
template <typename T>
int complex_gemm_dev(int transa, int transb, size_t m, size_t n, size_t k, T ar, T ai, const T* A,
                     size_t lda, const T* B, size_t ldb, T br, T bi, T* C, size_t ldc, int prec,
                     cudaStream_t st, int32_t* ce) {
    if (m == 0 || n == 0) return RB_OK;
    const size_t vec = 16 / sizeof(T);
    const size_t lda2 = rup(2 * m, vec), ldp = rup(2 * m, vec);
    const bool expand_b = transb != RB_NO_TRANS;
    const size_t ldb2 = expand_b ? rup(2 * k, vec) : 2 * ldb;
    const size_t a_bytes = rup(lda2 * 2 * std::max<size_t>(k, 1) * sizeof(T), 256);
    const size_t b_bytes = expand_b ? rup(ldb2 * n * sizeof(T), 256) : 0;
    const size_t p_bytes = ldp * n * sizeof(T);
    void* buf = nullptr;
    cudaError_t e = scratch_alloc(&buf, a_bytes + b_bytes + p_bytes, st);
    if (e != cudaSuccess) return fail(e, ce);
    T* Ap = static_cast<T*>(buf);
    T* Bp = expand_b ? reinterpret_cast<T*>(static_cast<uint8_t*>(buf) + a_bytes) : const_cast<T*>(B);
    T* P = reinterpret_cast<T*>(static_cast<uint8_t*>(buf) + a_bytes + b_bytes);
    int rc = RB_OK;
    if (k > 0) {
        dim3 blk(32, 8);
        cplx_expand_a_kernel<T><<<dim3((m + kT - 1) / kT, (k + kT - 1) / kT), blk, 0, st>>>(
            A, lda, transa, (int)m, (int)k, Ap, lda2);
        count_launch();
        if (expand_b) {
            cplx_expand_b_kernel<T><<<dim3((k + kT - 1) / kT, (n + kT - 1) / kT), blk, 0, st>>>(
                B, ldb, transb, (int)k, (int)n, Bp, ldb2);
            count_launch();
        }
        rc = gemm_colmajor_dev<T>(false, false, 2 * m, n, 2 * k, T(1), Ap, lda2, Bp, ldb2, T(0), P, ldp,
                                  prec, st, 0, ce);
    } else {
        e = cudaMemsetAsync(P, 0, p_bytes, st);
        if (e != cudaSuccess) rc = fail(e, ce);
    }
    if (rc == RB_OK) {
        cplx_epilogue_kernel<T><<<grid_for(m * n), 256, 0, st>>>(P, ldp, (int)m, (int)n, ar, ai, br, bi, C, ldc);
        count_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) rc = fail(e, ce);
    }
    cudaFreeAsync(buf, st);
    return rc;
}

// ---------------------------------------------------------------------------
// symm (real) and symm / hemm (complex)
// ---------------------------------------------------------------------------
template <typename T, bool CX>
int sym_full_dev(int herm, int uplo, size_t q, const T* A, size_t lda, T* full, size_t ldf, cudaStream_t st,
                 int32_t* ce) {
    if (q == 0) return RB_OK;
    sym_expand_kernel<T, CX><<<sym_grid(q), dim3(kSymTile, 8), 0, st>>>(A, lda, (int)q, uplo, herm, full, ldf);
    count_launch();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? RB_OK : fail(e, ce);
}

template <typename T>
int symm_dev(int side, int uplo, size_t m, size_t n, T alpha, const T* A, size_t lda, const T* B,
             size_t ldb, T beta, T* C, size_t ldc, int prec, cudaStream_t st, int32_t* ce) {
    const size_t q = (side == RB_LEFT) ? m : n;
    if (m == 0 || n == 0) return RB_OK;
    const size_t ldf = rup(q, 16 / sizeof(T));
    void* full = nullptr;
    cudaError_t e = scratch_alloc(&full, ldf * q * sizeof(T), st);
    if (e != cudaSuccess) return fail(e, ce);
    int rc = sym_full_dev<T, false>(0, uplo, q, A, lda, static_cast<T*>(full), ldf, st, ce);
    if (rc != RB_OK) {
        cudaFreeAsync(full, st);
        return rc;
    }
    if (side == RB_LEFT)
        rc = gemm_colmajor_dev<T>(false, false, m, n, m, alpha, static_cast<T*>(full), ldf, B, ldb, beta, C,
                                  ldc, prec, st, 0, ce);
    else
        rc = gemm_colmajor_dev<T>(false, false, m, n, n, alpha, B, ldb, static_cast<T*>(full), ldf, beta, C,
                                  ldc, prec, st, 0, ce);
    cudaFreeAsync(full, st);
    return rc;
}

template <typename T>
int hesy_dev(int herm, int side, int uplo, size_t m, size_t n, T ar, T ai, const T* A, size_t lda,
             const T* B, size_t ldb, T br, T bi, T* C, size_t ldc, int prec, cudaStream_t st,
             int32_t* ce) {
    if (m == 0 || n == 0) return RB_OK;  // src/complex3.rs:184-186
    const size_t q = (side == RB_LEFT) ? m : n;
    void* full = nullptr;
    cudaError_t e = scratch_alloc(&full, 2 * q * q * sizeof(T), st);
    if (e != cudaSuccess) return fail(e, ce);
    int rc = sym_full_dev<T, true>(herm, uplo, q, A, lda, static_cast<T*>(full), q, st, ce);
    if (rc != RB_OK) {
        cudaFreeAsync(full, st);
        return rc;
    }
    if (side == RB_LEFT)
        rc = complex_gemm_dev<T>(RB_NO_TRANS, RB_NO_TRANS, m, n, m, ar, ai, static_cast<T*>(full), q, B, ldb,
                                 br, bi, C, ldc, prec, st, ce);
    else
        rc = complex_gemm_dev<T>(RB_NO_TRANS, RB_NO_TRANS, m, n, n, ar, ai, B, ldb, static_cast<T*>(full), q,
                                 br, bi, C, ldc, prec, st, ce);
    cudaFreeAsync(full, st);
    return rc;
}

// ---------------------------------------------------------------------------
// trsm
// ---------------------------------------------------------------------------

// off-diagonal update B_target -= X * op(A)_sub or op(A)_sub * X, real or complex
template <typename T, bool CX>
static int update_gemm(bool a_first, size_t m, size_t n, size_t k, const T* X, size_t ldx,
                       const T* Asub, size_t lda, int a_trans, T* target, size_t ldt, cudaStream_t st,
                       int32_t* ce) {
    if (m == 0 || n == 0 || k == 0) return RB_OK;
    if constexpr (CX) {
        if (a_first)
            return complex_gemm_dev<T>(a_trans, RB_NO_TRANS, m, n, k, T(-1), T(0), Asub, lda, X, ldx, T(1),
                                       T(0), target, ldt, RB_PREC_PLAIN, st, ce);
        return complex_gemm_dev<T>(RB_NO_TRANS, a_trans, m, n, k, T(-1), T(0), X, ldx, Asub, lda, T(1), T(0),
                                   target, ldt, RB_PREC_PLAIN, st, ce);
    } else {
        if (a_first)
            return gemm_colmajor_dev<T>(a_trans != 0, false, m, n, k, T(-1), Asub, lda, X, ldx, T(1), target,
                                        ldt, RB_PREC_PLAIN, st, 0, ce);
        return gemm_colmajor_dev<T>(false, a_trans != 0, m, n, k, T(-1), X, ldx, Asub, lda, T(1), target, ldt,
                                    RB_PREC_PLAIN, st, 0, ce);
    }
}

// Blocked substitution over diagonal blocks of op(A) (src/level3.rs:390-520
// solves row by row; the blocking only regroups the same updates), the
// order halved recursively at whole blocks so that the off-diagonal updates
// are a few large GEMMs. The diagonal blocks:
//   real types    kTrsmDiagReal rows, each solved by the batched trsm with
//                 one member, whose grid spans the right-hand sides in 8-32
//                 wide slices (f64 on the FP64 tensor cores against inverted
//                 64 x 64 blocks);
//   complex types kNbCplx rows by trsm_diag_kernel, one thread per
//                 right-hand side.
constexpr size_t kTrsmDiagReal = 512;

template <typename T, bool CX>
int trsm_dev(int side, int uplo, int trans, int diag, size_t m, size_t n, T ar, T ai, const T* A,
             size_t lda, T* B, size_t ldb, cudaStream_t st, int32_t* ce) {
    constexpr int W = CX ? 2 : 1;
    constexpr size_t NB = CX ? static_cast<size_t>(kNbCplx) : kTrsmDiagReal;
    if (m == 0 || n == 0) return RB_OK;
    const bool alpha_one = (ar == T(1)) && (!CX || ai == T(0));
    if (!alpha_one) {  // src/level3.rs:403-409
        scale_b_kernel<T, CX><<<grid_for(m * n), 256, 0, st>>>(B, ldb, (int)m, (int)n, ar, ai);
        count_launch();
    }
    const bool tr = trans != RB_NO_TRANS;
    const bool eff_upper = (uplo == RB_UPPER) != tr;  // src/level3.rs:423-426
    const size_t q = (side == RB_LEFT) ? m : n;       // order of op(A)
    const size_t nvec = (side == RB_LEFT) ? n : m;
    if constexpr (CX) {
        static bool attr = false;
        if (!attr) {
            cudaFuncSetAttribute(trsm_diag_kernel<T, CX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(NB * NB * W * sizeof(T)));
            attr = true;
        }
    }
    // op(A)[r0:, c0:] as a stored sub-matrix and its transpose flag
    auto sub = [&](size_t r0, size_t c0) -> const T* {
        const size_t off = tr ? (c0 + r0 * lda) : (r0 + c0 * lda);
        return A + W * off;
    };
    const bool forward = (side == RB_LEFT) ? !eff_upper : eff_upper;
    // one diagonal block [o, o + nb) of op(A)'s order
    auto leaf = [&](size_t o, size_t nb) -> int {
        if constexpr (CX) {
            trsm_diag_kernel<T, CX><<<(int)((nvec + 127) / 128), 128, NB * NB * W * sizeof(T), st>>>(
                side, eff_upper, trans, diag, (int)nb, (int)o, A, lda, B, ldb, (int)nvec);
            count_launch();
            const cudaError_t le = cudaGetLastError();
            return le == cudaSuccess ? RB_OK : fail(le, ce);
        } else {
            // the diagonal block of op(A) is op() of A's diagonal block
            return trsm_batched_dev<T>(side, uplo, trans, diag, side == RB_LEFT ? nb : m, side == RB_LEFT ? n : nb,
                                       T(1), A + o + o * lda, lda, 0, side == RB_LEFT ? B + o : B + o * ldb, ldb, 0,
                                       1, st, ce, nullptr);
        }
    };
    // [o, o + len) split at o + h into P1 = [o, o + h) and P2 = [o + h, o + len):
    // forward solves P1, then B(P2) -= op(A)(P2, P1) X(P1) (Left) or
    // X(:, P1) op(A)(P1, P2) (Right), then P2; backward the mirror image.
    // Halving at whole blocks gives the same updates as a block-by-block
    // loop, grouped into a few GEMMs with K up to q / 2.
    std::function<int(size_t, size_t)> solve = [&](size_t o, size_t len) -> int {
        const size_t nblk = (len + NB - 1) / NB;
        if (nblk <= 1) return leaf(o, len);
        const size_t h = (nblk / 2) * NB, o2 = o + h, l2 = len - h;
        int rc = forward ? solve(o, h) : solve(o2, l2);
        if (rc != RB_OK) return rc;
        if (side == RB_LEFT) {
            rc = forward ? update_gemm<T, CX>(true, l2, n, h, B + W * o, ldb, sub(o2, o), lda, trans, B + W * o2,
                                              ldb, st, ce)
                         : update_gemm<T, CX>(true, h, n, l2, B + W * o2, ldb, sub(o, o2), lda, trans, B + W * o,
                                              ldb, st, ce);
        } else {
            rc = forward ? update_gemm<T, CX>(false, m, l2, h, B + W * o * ldb, ldb, sub(o, o2), lda, trans,
                                              B + W * o2 * ldb, ldb, st, ce)
                         : update_gemm<T, CX>(false, m, h, l2, B + W * o2 * ldb, ldb, sub(o2, o), lda, trans,
                                              B + W * o * ldb, ldb, st, ce);
        }
        if (rc != RB_OK) return rc;
        return forward ? solve(o2, l2) : solve(o, h);
    };
    return solve(0, q);
}

// B := alpha*op(A)*B (Left) or alpha*B*op(A) (Right), A triangular, in place.
// The order of op(A) is halved recursively at whole kTrmmLeaf blocks:
// with op(A) = [[T11, T12], [T21, T22]] (one of T12 / T21 zero) and B split
// to match, each half of B is multiplied by its diagonal block (recursion)
// before or after the off-diagonal product is added to it (a GEMM with
// beta = 1), in the order that reads the other half of B before it changes:
//   Left  lower: B2 := T22 B2; B2 += T21 B1; B1 := T11 B1
//   Left  upper: B1 := T11 B1; B1 += T12 B2; B2 := T22 B2
//   Right lower: B1 := B1 T11; B1 += B2 T21; B2 := B2 T22
//   Right upper: B2 := B2 T22; B2 += B1 T12; B1 := B1 T11
// A leaf block is expanded by tri_expand_kernel (the referenced triangle,
// zeros elsewhere, ones on a Unit diagonal) and multiplied by one GEMM into
// scratch, which is copied back into B. The unreferenced triangle and a Unit
// diagonal are never read. Only the T21 / T12 blocks and the leaves' squares
// are multiplied: about half the flops of one GEMM by the full op(A).
constexpr size_t kTrmmLeaf = 512;

template <typename T, bool CX>
int trmm_dev(int side, int uplo, int trans, int diag, size_t m, size_t n, T ar, T ai, const T* A, size_t lda, T* B,
             size_t ldb, cudaStream_t st, int32_t* ce) {
    if (m == 0 || n == 0) return RB_OK;
    constexpr int W = CX ? 2 : 1;
    const bool left = side == RB_LEFT;
    const size_t q = left ? m : n;
    const size_t L = std::min(q, kTrmmLeaf);
    const size_t vec = 16 / (W * sizeof(T)) > 0 ? 16 / (W * sizeof(T)) : 1;
    const size_t ldf = rup(L, vec), ldo = rup(left ? L : m, vec), out_cols = left ? n : L;
    const size_t full_bytes = rup(W * ldf * L * sizeof(T), 256);
    void* buf = nullptr;
    cudaError_t e = scratch_alloc(&buf, full_bytes + W * ldo * out_cols * sizeof(T), st);
    if (e != cudaSuccess) return fail(e, ce);
    T* full = static_cast<T*>(buf);
    T* out = reinterpret_cast<T*>(static_cast<uint8_t*>(buf) + full_bytes);
    const bool tr = trans != RB_NO_TRANS;
    const bool eff_upper = (uplo == RB_UPPER) != tr;
    // op(A)[r0:, c0:] as a stored sub-matrix (read through the GEMM's transpose)
    auto sub = [&](size_t r0, size_t c0) -> const T* { return A + W * (tr ? (c0 + r0 * lda) : (r0 + c0 * lda)); };
    auto bl = [&](size_t o) -> T* { return B + W * (left ? o : o * ldb); };  // B's rows / columns from o
    // target += alpha * op(A)(r0.., c0..) X (Left) or alpha * X op(A)(r0.., c0..) (Right)
    auto add = [&](size_t rows, size_t cols, size_t r0, size_t c0, const T* X, T* target) -> int {
        if constexpr (CX) {
            if (left)
                return complex_gemm_dev<T>(trans, RB_NO_TRANS, rows, n, cols, ar, ai, sub(r0, c0), lda, X, ldb, T(1),
                                           T(0), target, ldb, RB_PREC_PLAIN, st, ce);
            return complex_gemm_dev<T>(RB_NO_TRANS, trans, m, cols, rows, ar, ai, X, ldb, sub(r0, c0), lda, T(1),
                                       T(0), target, ldb, RB_PREC_PLAIN, st, ce);
        } else {
            if (left)
                return gemm_colmajor_dev<T>(tr, false, rows, n, cols, ar, sub(r0, c0), lda, X, ldb, T(1), target, ldb,
                                            RB_PREC_PLAIN, st, 0, ce);
            return gemm_colmajor_dev<T>(false, tr, m, cols, rows, ar, X, ldb, sub(r0, c0), lda, T(1), target, ldb,
                                        RB_PREC_PLAIN, st, 0, ce);
        }
    };
    auto leaf = [&](size_t o, size_t nb) -> int {
        tri_expand_kernel<T, CX><<<grid_for(nb * nb), 256, 0, st>>>(A + W * (o + o * lda), lda, static_cast<int>(nb),
                                                                     uplo, trans, diag, full, ldf);
        count_launch();
        const size_t rows = left ? nb : m, cols = left ? n : nb;
        int rc;
        if constexpr (CX) {
            rc = left ? complex_gemm_dev<T>(RB_NO_TRANS, RB_NO_TRANS, nb, n, nb, ar, ai, full, ldf, bl(o), ldb, T(0),
                                            T(0), out, ldo, RB_PREC_PLAIN, st, ce)
                      : complex_gemm_dev<T>(RB_NO_TRANS, RB_NO_TRANS, m, nb, nb, ar, ai, bl(o), ldb, full, ldf, T(0),
                                            T(0), out, ldo, RB_PREC_PLAIN, st, ce);
        } else {
            rc = left ? gemm_colmajor_dev<T>(false, false, nb, n, nb, ar, full, ldf, bl(o), ldb, T(0), out, ldo,
                                             RB_PREC_PLAIN, st, 0, ce)
                      : gemm_colmajor_dev<T>(false, false, m, nb, nb, ar, bl(o), ldb, full, ldf, T(0), out, ldo,
                                             RB_PREC_PLAIN, st, 0, ce);
        }
        if (rc != RB_OK) return rc;
        const cudaError_t ce2 = cudaMemcpy2DAsync(bl(o), W * ldb * sizeof(T), out, W * ldo * sizeof(T),
                                                  W * rows * sizeof(T), cols, cudaMemcpyDeviceToDevice, st);
        return ce2 == cudaSuccess ? RB_OK : fail(ce2, ce);
    };
    std::function<int(size_t, size_t)> mul = [&](size_t o, size_t len) -> int {
        const size_t nblk = (len + L - 1) / L;
        if (nblk <= 1) return leaf(o, len);
        const size_t h = (nblk / 2) * L, o2 = o + h, l2 = len - h;
        // the half whose product reads the other half's old values goes first
        const bool second_first = left ? !eff_upper : eff_upper;
        int rc = second_first ? mul(o2, l2) : mul(o, h);
        if (rc != RB_OK) return rc;
        if (left)
            rc = eff_upper ? add(h, l2, o, o2, bl(o2), bl(o)) : add(l2, h, o2, o, bl(o), bl(o2));
        else
            rc = eff_upper ? add(h, l2, o, o2, bl(o), bl(o2)) : add(l2, h, o2, o, bl(o2), bl(o));
        if (rc != RB_OK) return rc;
        return second_first ? mul(o, h) : mul(o2, l2);
    };
    const int rc = mul(0, q);
    cudaFreeAsync(buf, st);
    return rc;
}

template int trmm_dev<float, false>(int, int, int, int, size_t, size_t, float, float, const float*, size_t, float*,
                                    size_t, cudaStream_t, int32_t*);
template int trmm_dev<double, false>(int, int, int, int, size_t, size_t, double, double, const double*, size_t,
                                     double*, size_t, cudaStream_t, int32_t*);
template int trmm_dev<float, true>(int, int, int, int, size_t, size_t, float, float, const float*, size_t, float*,
                                   size_t, cudaStream_t, int32_t*);
template int trmm_dev<double, true>(int, int, int, int, size_t, size_t, double, double, const double*, size_t,
                                    double*, size_t, cudaStream_t, int32_t*);

template int complex_gemm_dev<float>(int, int, size_t, size_t, size_t, float, float, const float*, size_t,
                                     const float*, size_t, float, float, float*, size_t, int, cudaStream_t,
                                     int32_t*);
template int complex_gemm_dev<double>(int, int, size_t, size_t, size_t, double, double, const double*, size_t,
                                      const double*, size_t, double, double, double*, size_t, int,
                                      cudaStream_t, int32_t*);
template int sym_full_dev<float, false>(int, int, size_t, const float*, size_t, float*, size_t, cudaStream_t,
                                        int32_t*);
template int sym_full_dev<double, false>(int, int, size_t, const double*, size_t, double*, size_t, cudaStream_t,
                                         int32_t*);
template int sym_full_dev<float, true>(int, int, size_t, const float*, size_t, float*, size_t, cudaStream_t,
                                       int32_t*);
template int sym_full_dev<double, true>(int, int, size_t, const double*, size_t, double*, size_t, cudaStream_t,
                                        int32_t*);
template int symm_dev<float>(int, int, size_t, size_t, float, const float*, size_t, const float*, size_t,
                             float, float*, size_t, int, cudaStream_t, int32_t*);
template int symm_dev<double>(int, int, size_t, size_t, double, const double*, size_t, const double*,
                              size_t, double, double*, size_t, int, cudaStream_t, int32_t*);
template int hesy_dev<float>(int, int, int, size_t, size_t, float, float, const float*, size_t, const float*,
                             size_t, float, float, float*, size_t, int, cudaStream_t, int32_t*);
template int hesy_dev<double>(int, int, int, size_t, size_t, double, double, const double*, size_t,
                              const double*, size_t, double, double, double*, size_t, int, cudaStream_t,
                              int32_t*);
template int trsm_dev<float, false>(int, int, int, int, size_t, size_t, float, float, const float*, size_t,
                                    float*, size_t, cudaStream_t, int32_t*);
template int trsm_dev<double, false>(int, int, int, int, size_t, size_t, double, double, const double*,
                                     size_t, double*, size_t, cudaStream_t, int32_t*);
template int trsm_dev<float, true>(int, int, int, int, size_t, size_t, float, float, const float*, size_t,
                                   float*, size_t, cudaStream_t, int32_t*);
template int trsm_dev<double, true>(int, int, int, int, size_t, size_t, double, double, const double*,
                                    size_t, double*, size_t, cudaStream_t, int32_t*);

}  // namespace rb
