// rblas_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle). Never linked into
// the product library; only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg load it.
//
// Two things live here:
//
//  1. A CPU restatement of rblas's Level-3 GEMM path, written to reproduce the
//     reference's rounding on AVX2+FMA hosts:
//       - level3::gemm row-major swap            src/level3.rs:52-60
//       - level3::try_gemm / check_matrix        src/level3.rs:68-140
//       - gemm_colmajor / materialize            src/level3.rs:143-222
//       - gemm_contig early-outs + apply_beta    src/kernel/gemm.rs:185-230, 322-338
//       - gemm_band (KC/MC loops, packing)       src/kernel/gemm.rs:238-272, 343-400
//       - gemm_parallel column-chunk split       src/kernel/gemm.rs:277-313
//       - macrokernel                            src/kernel/gemm.rs:404-429
//       - micro_16x6_f32 / micro_8x6_f64 (AVX2)  src/kernel/gemm_avx2.rs:26-155
//       - micro_raw_scalar (no-AVX2 fallback)    src/kernel/gemm.rs:641-670
//       - syrk / symm / full_symmetric / trsm    src/level3.rs:236-520
//       - complex3::gemm (4M) / split_op / he_or_sy / trsm / cdiv
//                                                src/complex3.rs:27-349
//       - Complex mul / conj / norm_sqr          src/complex.rs:59-111
//     Built with -O3 -mavx2 -mfma -ffp-contract=off, so every fused
//     multiply-add here is an explicit fma and every unfused one stays two
//     roundings, as in the Rust source (Rust never contracts a*b+c).
//
//  2. An accuracy oracle: a compensated double-double GEMM (TwoProduct via fma,
//     TwoSum accumulation: the Dot2 scheme of Ogita, Rump & Oishi, "Accurate sum
//     and dot product", SIAM J. Sci. Comput. 26(6), 2005), optionally evaluated
//     on a row sample, returning the result as an unevaluated pair (hi, lo).
//
// Parity pin: rblas is Rust and cannot be compiled in this environment (no
// cargo/rustc); this restatement is pinned against the known-answer and
// tolerance assertions of the reference's own tests (tests/golden/).

#include <immintrin.h>
#include <pthread.h>
#include <stdint.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <atomic>
#include <cmath>
#include <utility>
#include <vector>
#include <thread>
#include <algorithm>

namespace {

// src/kernel/gemm.rs:173-175
constexpr size_t MC = 384;
constexpr size_t KC = 512;
constexpr size_t NC = 4096;

// src/kernel/gemm.rs:139-146 (x86-64 tile sizes)
template <typename T> struct Tile;
template <> struct Tile<float>  { static constexpr size_t MR = 16, NR = 6; };
template <> struct Tile<double> { static constexpr size_t MR = 8,  NR = 6; };

inline size_t round_up(size_t x, size_t m) { return (x + m - 1) / m * m; }

inline float  fmaT(float a, float b, float c)    { return fmaf(a, b, c); }
inline double fmaT(double a, double b, double c) { return fma(a, b, c); }

bool g_force_scalar = false;  // test hook: take the no-AVX2 microkernel

bool have_avx2_fma() {
    static int cached = -1;
    if (cached < 0) {
        __builtin_cpu_init();
        cached = (__builtin_cpu_supports("avx2") && __builtin_cpu_supports("fma")) ? 1 : 0;
    }
    return cached == 1 && !g_force_scalar;
}

// ---- microkernels ---------------------------------------------------------

// src/kernel/gemm_avx2.rs:26-85. fma accumulation in p order; full tile
// writes fma(alpha, acc, c); edge tile writes c + alpha*acc (two roundings).
__attribute__((target("avx2,fma")))
void micro_16x6_f32(size_t mr, size_t nr, size_t kc, float alpha, const float* ap,
                    const float* bp, float* c, size_t ldc, size_t ci, size_t cj) {
    __m256 lo[6], hi[6];
    for (int s = 0; s < 6; ++s) { lo[s] = _mm256_setzero_ps(); hi[s] = _mm256_setzero_ps(); }
    for (size_t p = 0; p < kc; ++p) {
        const float* a = ap + p * 16;
        const float* b = bp + p * 6;
        __m256 a_lo = _mm256_loadu_ps(a);
        __m256 a_hi = _mm256_loadu_ps(a + 8);
        for (int s = 0; s < 6; ++s) {
            __m256 bs = _mm256_broadcast_ss(b + s);
            lo[s] = _mm256_fmadd_ps(a_lo, bs, lo[s]);
            hi[s] = _mm256_fmadd_ps(a_hi, bs, hi[s]);
        }
    }
    // Every access to lo[] / hi[] uses a compile-time index, so the twelve
    // accumulators stay in registers through the k loop (a runtime index in
    // the edge path made the compiler store them to the stack every step).
    __m256 va = _mm256_set1_ps(alpha);
    if (mr == 16 && nr == 6) {
#pragma GCC unroll 6
        for (int s = 0; s < 6; ++s) {
            float* cptr = c + ci + (cj + s) * ldc;
            __m256 c_lo = _mm256_loadu_ps(cptr);
            __m256 c_hi = _mm256_loadu_ps(cptr + 8);
            _mm256_storeu_ps(cptr, _mm256_fmadd_ps(va, lo[s], c_lo));
            _mm256_storeu_ps(cptr + 8, _mm256_fmadd_ps(va, hi[s], c_hi));
        }
    } else {
        alignas(32) float buf[6][16];
#pragma GCC unroll 6
        for (int s = 0; s < 6; ++s) {
            _mm256_store_ps(buf[s], lo[s]);
            _mm256_store_ps(buf[s] + 8, hi[s]);
        }
        for (size_t s = 0; s < nr; ++s) {
            float* col = c + ci + (cj + s) * ldc;
            for (size_t r = 0; r < mr; ++r) {
                float t = alpha * buf[s][r];
                col[r] = col[r] + t;
            }
        }
    }
}

// src/kernel/gemm_avx2.rs:97-155
__attribute__((target("avx2,fma")))
void micro_8x6_f64(size_t mr, size_t nr, size_t kc, double alpha, const double* ap,
                   const double* bp, double* c, size_t ldc, size_t ci, size_t cj) {
    __m256d lo[6], hi[6];
    for (int s = 0; s < 6; ++s) { lo[s] = _mm256_setzero_pd(); hi[s] = _mm256_setzero_pd(); }
    for (size_t p = 0; p < kc; ++p) {
        const double* a = ap + p * 8;
        const double* b = bp + p * 6;
        __m256d a_lo = _mm256_loadu_pd(a);
        __m256d a_hi = _mm256_loadu_pd(a + 4);
        for (int s = 0; s < 6; ++s) {
            __m256d bs = _mm256_broadcast_sd(b + s);
            lo[s] = _mm256_fmadd_pd(a_lo, bs, lo[s]);
            hi[s] = _mm256_fmadd_pd(a_hi, bs, hi[s]);
        }
    }
    // compile-time indices only, as in micro_16x6_f32
    __m256d va = _mm256_set1_pd(alpha);
    if (mr == 8 && nr == 6) {
#pragma GCC unroll 6
        for (int s = 0; s < 6; ++s) {
            double* cptr = c + ci + (cj + s) * ldc;
            __m256d c_lo = _mm256_loadu_pd(cptr);
            __m256d c_hi = _mm256_loadu_pd(cptr + 4);
            _mm256_storeu_pd(cptr, _mm256_fmadd_pd(va, lo[s], c_lo));
            _mm256_storeu_pd(cptr + 4, _mm256_fmadd_pd(va, hi[s], c_hi));
        }
    } else {
        alignas(32) double buf[6][8];
#pragma GCC unroll 6
        for (int s = 0; s < 6; ++s) {
            _mm256_store_pd(buf[s], lo[s]);
            _mm256_store_pd(buf[s] + 4, hi[s]);
        }
        for (size_t s = 0; s < nr; ++s) {
            double* col = c + ci + (cj + s) * ldc;
            for (size_t r = 0; r < mr; ++r) {
                double t = alpha * buf[s][r];
                col[r] = col[r] + t;
            }
        }
    }
}

// src/kernel/gemm.rs:641-670: fma accumulation over the full MR x NR tile,
// writeback fma(alpha, acc, c) on every tile.
template <typename T>
void micro_raw_scalar(size_t mr, size_t nr, size_t kc, T alpha, const T* ap, const T* bp,
                      T* c, size_t ldc, size_t ci, size_t cj) {
    constexpr size_t MR = Tile<T>::MR, NR = Tile<T>::NR;
    T acc[MR][NR];
    for (size_t r = 0; r < MR; ++r)
        for (size_t s = 0; s < NR; ++s) acc[r][s] = T(0);
    for (size_t p = 0; p < kc; ++p) {
        for (size_t r = 0; r < MR; ++r) {
            T ar = ap[p * MR + r];
            for (size_t s = 0; s < NR; ++s) acc[r][s] = fmaT(ar, bp[p * NR + s], acc[r][s]);
        }
    }
    for (size_t s = 0; s < nr; ++s)
        for (size_t r = 0; r < mr; ++r) {
            T* cp = c + ci + r + (cj + s) * ldc;
            *cp = fmaT(alpha, acc[r][s], *cp);
        }
}

inline void micro(size_t mr, size_t nr, size_t kc, float alpha, const float* ap, const float* bp,
                  float* c, size_t ldc, size_t ci, size_t cj) {
    if (have_avx2_fma()) micro_16x6_f32(mr, nr, kc, alpha, ap, bp, c, ldc, ci, cj);
    else micro_raw_scalar<float>(mr, nr, kc, alpha, ap, bp, c, ldc, ci, cj);
}
inline void micro(size_t mr, size_t nr, size_t kc, double alpha, const double* ap, const double* bp,
                  double* c, size_t ldc, size_t ci, size_t cj) {
    if (have_avx2_fma()) micro_8x6_f64(mr, nr, kc, alpha, ap, bp, c, ldc, ci, cj);
    else micro_raw_scalar<double>(mr, nr, kc, alpha, ap, bp, c, ldc, ci, cj);
}

// ---- packing / blocking ---------------------------------------------------

// src/kernel/gemm.rs:343-371
template <typename T>
void pack_a_panel(size_t mc, size_t kc, const T* a, size_t lda, size_t ic, size_t pc, T* pack) {
    constexpr size_t MR = Tile<T>::MR;
    size_t dst = 0;
    for (size_t i = 0; i < mc; i += MR) {
        size_t mr = std::min(MR, mc - i);
        for (size_t p = 0; p < kc; ++p) {
            size_t acol = pc + p;
            for (size_t r = 0; r < mr; ++r) pack[dst++] = a[(ic + i + r) + acol * lda];
            for (size_t r = mr; r < MR; ++r) pack[dst++] = T(0);
        }
    }
}

// src/kernel/gemm.rs:374-400
template <typename T>
void pack_b_panel(size_t kc, size_t nc, const T* b, size_t ldb, size_t pc, size_t jc, T* pack) {
    constexpr size_t NR = Tile<T>::NR;
    size_t dst = 0;
    for (size_t j = 0; j < nc; j += NR) {
        size_t nr = std::min(NR, nc - j);
        for (size_t p = 0; p < kc; ++p) {
            size_t brow = pc + p;
            for (size_t s = 0; s < nr; ++s) pack[dst++] = b[brow + (jc + j + s) * ldb];
            for (size_t s = nr; s < NR; ++s) pack[dst++] = T(0);
        }
    }
}

// src/kernel/gemm.rs:404-429
template <typename T>
void macrokernel(size_t mc, size_t nc, size_t kc, T alpha, const T* pack_a, const T* pack_b,
                 T* c, size_t ldc, size_t ic, size_t jc) {
    constexpr size_t MR = Tile<T>::MR, NR = Tile<T>::NR;
    for (size_t j = 0; j < nc; j += NR) {
        size_t nr = std::min(NR, nc - j);
        const T* bp = pack_b + (j / NR) * (kc * NR);
        for (size_t i = 0; i < mc; i += MR) {
            size_t mr = std::min(MR, mc - i);
            const T* ap = pack_a + (i / MR) * (kc * MR);
            micro(mr, nr, kc, alpha, ap, bp, c, ldc, ic + i, jc + j);
        }
    }
}

// src/kernel/gemm.rs:238-272 (scratch is per call here; the reference keeps it
// thread-local, which changes nothing numerically: buffers are re-zeroed).
template <typename T>
void gemm_band(size_t m, size_t nc, size_t k, T alpha, const T* a, size_t lda, const T* b,
               size_t ldb, size_t j0, T* cband, size_t ldc) {
    constexpr size_t MR = Tile<T>::MR, NR = Tile<T>::NR;
    size_t a_cap = round_up(std::min(MC, m), MR) * std::min(KC, k);
    size_t b_cap = std::min(KC, k) * round_up(nc, NR);
    std::vector<T> pack_a(a_cap, T(0)), pack_b(b_cap, T(0));
    for (size_t pc = 0; pc < k; pc += KC) {
        size_t kc = std::min(KC, k - pc);
        pack_b_panel(kc, nc, b, ldb, pc, j0, pack_b.data());
        for (size_t ic = 0; ic < m; ic += MC) {
            size_t mc = std::min(MC, m - ic);
            pack_a_panel(mc, kc, a, lda, ic, pc, pack_a.data());
            macrokernel(mc, nc, kc, alpha, pack_a.data(), pack_b.data(), cband, ldc, ic, 0);
        }
    }
}

// src/kernel/gemm.rs:322-338
template <typename T>
void apply_beta(size_t m, size_t n, T beta, T* c, size_t ldc) {
    if (beta == T(1)) return;
    for (size_t j = 0; j < n; ++j) {
        T* col = c + j * ldc;
        if (beta == T(0)) {
            for (size_t i = 0; i < m; ++i) col[i] = T(0);
        } else {
            for (size_t i = 0; i < m; ++i) col[i] = beta * col[i];
        }
    }
}

// src/kernel/gemm.rs:277-313. Chunks are taken from a shared counter by
// `threads` workers (rayon's stealing order does not affect the result since
// chunks write disjoint columns). Chunks that would start at or beyond column
// n are not formed (the reference only forms them for C slices longer than
// (n-1)*ldc+m, where its `n - j0` would underflow).
template <typename T>
void gemm_parallel(size_t m, size_t n, size_t k, T alpha, const T* a, size_t lda, const T* b,
                   size_t ldb, T* c, size_t ldc, int threads) {
    constexpr size_t NR = Tile<T>::NR;
    size_t target_tasks = std::max<size_t>((size_t)threads * 4, 1);
    size_t chunk_cols = (n + target_tasks - 1) / target_tasks;
    chunk_cols = std::min(round_up(std::max(chunk_cols, NR), NR), NC);
    size_t nchunks = (n + chunk_cols - 1) / chunk_cols;
    std::atomic<size_t> next{0};
    auto worker = [&]() {
        for (;;) {
            size_t ci = next.fetch_add(1);
            if (ci >= nchunks) break;
            size_t j0 = ci * chunk_cols;
            size_t nc = std::min(chunk_cols, n - j0);
            gemm_band(m, nc, k, alpha, a, lda, b, ldb, j0, c + j0 * ldc, ldc);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
}

// src/kernel/gemm.rs:185-230. `threads` plays rayon::current_num_threads();
// threads <= 1 is the serial (no `threads` feature) build.
template <typename T>
void gemm_contig(size_t m, size_t n, size_t k, T alpha, const T* a, size_t lda, const T* b,
                 size_t ldb, T beta, T* c, size_t ldc, int threads) {
    constexpr size_t NR = Tile<T>::NR;
    if (m == 0 || n == 0) return;
    apply_beta(m, n, beta, c, ldc);
    if (k == 0 || alpha == T(0)) return;
    if (threads > 1) {
        bool big_enough = n >= 2 * NR && (m * n * k) >= ((size_t)1 << 18);
        if (big_enough) {
            gemm_parallel(m, n, k, alpha, a, lda, b, ldb, c, ldc, threads);
            return;
        }
    }
    for (size_t jc = 0; jc < n; jc += NC) {
        size_t nc = std::min(NC, n - jc);
        gemm_band(m, nc, k, alpha, a, lda, b, ldb, jc, c + jc * ldc, ldc);
    }
}

// src/level3.rs:179-222
template <typename T>
void materialize(bool ta, bool tb, size_t m, size_t n, size_t k, const T* a, size_t lda,
                 const T* b, size_t ldb, std::vector<T>& am, std::vector<T>& bm) {
    am.assign(m * k, T(0));
    bm.assign(k * n, T(0));
    for (size_t p = 0; p < k; ++p)
        for (size_t i = 0; i < m; ++i) am[i + p * m] = ta ? a[p + i * lda] : a[i + p * lda];
    for (size_t j = 0; j < n; ++j)
        for (size_t p = 0; p < k; ++p) bm[p + j * k] = tb ? b[j + p * ldb] : b[p + j * ldb];
}

// src/level3.rs:143-175
template <typename T>
void gemm_colmajor(bool ta, bool tb, size_t m, size_t n, size_t k, T alpha, const T* a,
                   size_t lda, const T* b, size_t ldb, T beta, T* c, size_t ldc, int threads) {
    if (!ta && !tb) {
        gemm_contig(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, threads);
    } else {
        std::vector<T> am, bm;
        materialize(ta, tb, m, n, k, a, lda, b, ldb, am, bm);
        gemm_contig(m, n, k, alpha, am.data(), m, bm.data(), k, beta, c, ldc, threads);
    }
}

// src/level3.rs:32-62. layout: 0 = RowMajor, 1 = ColMajor; trans: 0 None,
// 1 Trans, 2 ConjTrans (real: ConjTrans == Trans, src/types.rs:42-44).
template <typename T>
void gemm_any(int layout, int transa, int transb, size_t m, size_t n, size_t k, T alpha,
              const T* a, size_t lda, const T* b, size_t ldb, T beta, T* c, size_t ldc,
              int threads) {
    bool ta = transa != 0, tb = transb != 0;
    if (layout == 1)
        gemm_colmajor(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, threads);
    else
        gemm_colmajor(tb, ta, n, m, k, alpha, b, ldb, a, lda, beta, c, ldc, threads);
}

// ---- real syrk / symm / trsm (src/level3.rs:236-520) -------------------------

template <typename T>
void syrk_impl(int uplo, int trans, size_t n, size_t k, T alpha, const T* a, size_t lda, T beta,
               T* c, size_t ldc, int threads) {
    if (n == 0) return;
    bool t = trans != 0;
    std::vector<T> p(n * n, T(0));
    // op(A) op(A)^T: (Trans, None) when trans, else (None, Trans)  src/level3.rs:257-278
    gemm_any<T>(1, t ? 1 : 0, t ? 0 : 1, n, n, k, alpha, a, lda, a, lda, T(0), p.data(), n,
                threads);
    for (size_t j = 0; j < n; ++j) {
        size_t lo = (uplo == 0) ? 0 : j, hi = (uplo == 0) ? j + 1 : n;  // 0 = Upper
        for (size_t i = lo; i < hi; ++i) {
            size_t cij = i + j * ldc;
            T scaled = (beta == T(0)) ? T(0) : beta * c[cij];
            c[cij] = p[i + j * n] + scaled;
        }
    }
}

template <typename T>
std::vector<T> full_symmetric(int uplo, size_t q, const T* a, size_t lda) {
    std::vector<T> full(q * q, T(0));
    for (size_t j = 0; j < q; ++j)
        for (size_t i = 0; i < q; ++i) {
            bool stored = (uplo == 0) ? (i <= j) : (i >= j);
            full[i + j * q] = stored ? a[i + j * lda] : a[j + i * lda];
        }
    return full;
}

template <typename T>
void symm_impl(int side, int uplo, size_t m, size_t n, T alpha, const T* a, size_t lda,
               const T* b, size_t ldb, T beta, T* c, size_t ldc, int threads) {
    size_t q = (side == 0) ? m : n;  // 0 = Left
    std::vector<T> full = full_symmetric(uplo, q, a, lda);
    if (side == 0)
        gemm_any<T>(1, 0, 0, m, n, m, alpha, full.data(), q, b, ldb, beta, c, ldc, threads);
    else
        gemm_any<T>(1, 0, 0, m, n, n, alpha, b, ldb, full.data(), q, beta, c, ldc, threads);
}

template <typename T>
void trsm_impl(int side, int uplo, int trans, int diag, size_t m, size_t n, T alpha, const T* a,
               size_t lda, T* b, size_t ldb) {
    if (alpha != T(1))
        for (size_t j = 0; j < n; ++j)
            for (size_t i = 0; i < m; ++i) b[i + j * ldb] = alpha * b[i + j * ldb];
    bool tr = trans != 0;
    auto aop = [&](size_t r, size_t cc) -> T { return tr ? a[cc + r * lda] : a[r + cc * lda]; };
    bool eff_upper = (uplo == 0) != tr;  // src/level3.rs:423-426
    auto finish = [&](T s, T aii) -> T { return diag == 1 ? s : s / aii; };  // 1 = Unit
    // neg_mul_add(a, x, acc) = acc - a*x, unfused   src/level3.rs:509-512
    if (side == 0) {
        for (size_t j = 0; j < n; ++j) {
            size_t col = j * ldb;
            if (eff_upper) {
                for (size_t ii = m; ii-- > 0;) {
                    T s = b[ii + col];
                    for (size_t kk = ii + 1; kk < m; ++kk) { T t = aop(ii, kk) * b[kk + col]; s = s - t; }
                    b[ii + col] = finish(s, aop(ii, ii));
                }
            } else {
                for (size_t ii = 0; ii < m; ++ii) {
                    T s = b[ii + col];
                    for (size_t kk = 0; kk < ii; ++kk) { T t = aop(ii, kk) * b[kk + col]; s = s - t; }
                    b[ii + col] = finish(s, aop(ii, ii));
                }
            }
        }
    } else {
        for (size_t i = 0; i < m; ++i) {
            for (size_t t = 0; t < n; ++t) {
                size_t j = eff_upper ? t : n - 1 - t;
                T s = b[i + j * ldb];
                if (eff_upper) {
                    for (size_t kk = 0; kk < j; ++kk) { T u = b[i + kk * ldb] * aop(kk, j); s = s - u; }
                } else {
                    for (size_t kk = j + 1; kk < n; ++kk) { T u = b[i + kk * ldb] * aop(kk, j); s = s - u; }
                }
                b[i + j * ldb] = finish(s, aop(j, j));
            }
        }
    }
}

// ---- complex (src/complex.rs, src/complex3.rs) -------------------------------

template <typename T> struct Cx { T re, im; };

// src/complex.rs:101-111: re = fma(a.re, b.re, -(a.im*b.im)), im = fma(a.re, b.im, a.im*b.re)
template <typename T> inline Cx<T> cmul(Cx<T> a, Cx<T> b) {
    T t1 = a.im * b.im;
    T t2 = a.im * b.re;
    return {fmaT(a.re, b.re, T(0) - t1), fmaT(a.re, b.im, t2)};
}
template <typename T> inline Cx<T> cadd(Cx<T> a, Cx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <typename T> inline Cx<T> csub(Cx<T> a, Cx<T> b) { return {a.re - b.re, a.im - b.im}; }
template <typename T> inline Cx<T> cconj(Cx<T> a) { return {a.re, T(0) - a.im}; }
// src/complex3.rs:344-349; norm_sqr = fma(re, re, im*im)  src/complex.rs:68-70
template <typename T> inline Cx<T> cdiv(Cx<T> a, Cx<T> b) {
    T d = fmaT(b.re, b.re, b.im * b.im);
    Cx<T> num = cmul(a, cconj(b));
    return {num.re / d, num.im / d};
}

// src/complex3.rs:101-125
template <typename T>
void split_op(int trans, size_t rows, size_t cols, const Cx<T>* a, size_t lda, std::vector<T>& re,
              std::vector<T>& im) {
    re.assign(rows * cols, T(0));
    im.assign(rows * cols, T(0));
    bool conj = trans == 2, tr = trans != 0;
    for (size_t j = 0; j < cols; ++j)
        for (size_t i = 0; i < rows; ++i) {
            Cx<T> v = tr ? a[j + i * lda] : a[i + j * lda];
            if (conj) v = cconj(v);
            re[i + j * rows] = v.re;
            im[i + j * rows] = v.im;
        }
}

// src/complex3.rs:27-74 (4M: four real col-major NN gemms, then complex alpha/beta)
template <typename T>
void cgemm_impl(int transa, int transb, size_t m, size_t n, size_t k, Cx<T> alpha, const Cx<T>* a,
                size_t lda, const Cx<T>* b, size_t ldb, Cx<T> beta, Cx<T>* c, size_t ldc,
                int threads) {
    std::vector<T> ar, ai, br, bi;
    split_op(transa, m, k, a, lda, ar, ai);
    split_op(transb, k, n, b, ldb, br, bi);
    std::vector<T> pr(m * n, T(0)), pi(m * n, T(0));
    gemm_any<T>(1, 0, 0, m, n, k, T(1), ar.data(), m, br.data(), k, T(0), pr.data(), m, threads);
    gemm_any<T>(1, 0, 0, m, n, k, T(0) - T(1), ai.data(), m, bi.data(), k, T(1), pr.data(), m, threads);
    gemm_any<T>(1, 0, 0, m, n, k, T(1), ar.data(), m, bi.data(), k, T(0), pi.data(), m, threads);
    gemm_any<T>(1, 0, 0, m, n, k, T(1), ai.data(), m, br.data(), k, T(1), pi.data(), m, threads);
    bool beta_zero = beta.re == T(0) && beta.im == T(0);
    for (size_t j = 0; j < n; ++j)
        for (size_t i = 0; i < m; ++i) {
            Cx<T> p = {pr[i + j * m], pi[i + j * m]};
            size_t cij = i + j * ldc;
            Cx<T> scaled = beta_zero ? Cx<T>{T(0), T(0)} : cmul(beta, c[cij]);
            c[cij] = cadd(cmul(alpha, p), scaled);
        }
}

// src/complex3.rs:169-247
template <typename T>
void he_or_sy(int side, int uplo, size_t m, size_t n, Cx<T> alpha, const Cx<T>* a, size_t lda,
              const Cx<T>* b, size_t ldb, Cx<T> beta, Cx<T>* c, size_t ldc, bool hermitian,
              int threads) {
    if (m == 0 || n == 0) return;
    size_t q = (side == 0) ? m : n;
    std::vector<Cx<T>> full(q * q, Cx<T>{T(0), T(0)});
    for (size_t j = 0; j < q; ++j)
        for (size_t i = 0; i < q; ++i) {
            bool stored = (uplo == 0) ? (i <= j) : (i >= j);
            Cx<T> v;
            if (stored) {
                v = a[i + j * lda];
                if (hermitian && i == j) v.im = T(0);
            } else {
                v = a[j + i * lda];
                if (hermitian) v = cconj(v);
            }
            full[i + j * q] = v;
        }
    if (side == 0)
        cgemm_impl<T>(0, 0, m, n, m, alpha, full.data(), q, b, ldb, beta, c, ldc, threads);
    else
        cgemm_impl<T>(0, 0, m, n, n, alpha, b, ldb, full.data(), q, beta, c, ldc, threads);
}

// src/complex3.rs:252-340
template <typename T>
void ctrsm_impl(int side, int uplo, int trans, int diag, size_t m, size_t n, Cx<T> alpha,
                const Cx<T>* a, size_t lda, Cx<T>* b, size_t ldb) {
    if (!(alpha.re == T(1) && alpha.im == T(0)))
        for (size_t j = 0; j < n; ++j)
            for (size_t i = 0; i < m; ++i) b[i + j * ldb] = cmul(alpha, b[i + j * ldb]);
    bool conj = trans == 2, tr = trans != 0;
    auto aop = [&](size_t r, size_t cc) -> Cx<T> {
        Cx<T> v = tr ? a[cc + r * lda] : a[r + cc * lda];
        return conj ? cconj(v) : v;
    };
    bool eff_upper = (uplo == 0) != tr;
    auto finish = [&](Cx<T> s, Cx<T> aii) -> Cx<T> { return diag == 1 ? s : cdiv(s, aii); };
    if (side == 0) {
        for (size_t j = 0; j < n; ++j) {
            size_t col = j * ldb;
            if (eff_upper) {
                for (size_t ii = m; ii-- > 0;) {
                    Cx<T> s = b[ii + col];
                    for (size_t kk = ii + 1; kk < m; ++kk) s = csub(s, cmul(aop(ii, kk), b[kk + col]));
                    b[ii + col] = finish(s, aop(ii, ii));
                }
            } else {
                for (size_t ii = 0; ii < m; ++ii) {
                    Cx<T> s = b[ii + col];
                    for (size_t kk = 0; kk < ii; ++kk) s = csub(s, cmul(aop(ii, kk), b[kk + col]));
                    b[ii + col] = finish(s, aop(ii, ii));
                }
            }
        }
    } else {
        for (size_t i = 0; i < m; ++i)
            for (size_t t = 0; t < n; ++t) {
                size_t j = eff_upper ? t : n - 1 - t;
                Cx<T> s = b[i + j * ldb];
                if (eff_upper) {
                    for (size_t kk = 0; kk < j; ++kk) s = csub(s, cmul(b[i + kk * ldb], aop(kk, j)));
                } else {
                    for (size_t kk = j + 1; kk < n; ++kk) s = csub(s, cmul(b[i + kk * ldb], aop(kk, j)));
                }
                b[i + j * ldb] = finish(s, aop(j, j));
            }
    }
}

// ---- double-double accuracy oracle -------------------------------------------

inline void two_sum(double a, double b, double& s, double& e) {
    s = a + b;
    double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}
inline void two_prod(double a, double b, double& p, double& e) {
    p = a * b;
    e = fma(a, b, -p);
}

// Dot2-style compensated accumulation of one C column over a contiguous
// op(A) column panel. sh/sl carry the running (sum, compensation) per row.
void dd_column(size_t mrows, size_t k, const double* am, const double* bcol, double* sh, double* sl) {
    for (size_t i = 0; i < mrows; ++i) { sh[i] = 0.0; sl[i] = 0.0; }
    for (size_t p = 0; p < k; ++p) {
        const double bv = bcol[p];
        const double* acol = am + p * mrows;
        for (size_t i = 0; i < mrows; ++i) {
            double ph, pl, s, e;
            two_prod(acol[i], bv, ph, pl);
            two_sum(sh[i], ph, s, e);
            sh[i] = s;
            sl[i] += e + pl;
        }
    }
}

// C = alpha * op(A) op(B) + beta * C0, each op(.) given as a gather closure
// result materialised into double col-major panels. Output as (hi, lo) with
// hi + lo the double-double value, for every row listed in `rows`.
void dd_gemm_core(size_t nrows, size_t n, size_t k, double alpha, const double* am /* nrows x k */,
                  const double* bm /* k x n */, double beta, const double* c0 /* nrows x n or null */,
                  double* out_hi, double* out_lo, int threads) {
    std::atomic<size_t> next{0};
    auto worker = [&]() {
        std::vector<double> sh(nrows), sl(nrows);
        for (;;) {
            size_t j = next.fetch_add(1);
            if (j >= n) break;
            dd_column(nrows, k, am, bm + j * k, sh.data(), sl.data());
            for (size_t i = 0; i < nrows; ++i) {
                // normalise the column sum to a double-double (h, l)
                double h, l;
                two_sum(sh[i], sl[i], h, l);
                // alpha * (h + l)
                double ph, pl;
                two_prod(alpha, h, ph, pl);
                pl += alpha * l;
                // + beta * c0
                if (c0 && beta != 0.0) {
                    double qh, ql, s, e;
                    two_prod(beta, c0[i + j * nrows], qh, ql);
                    two_sum(ph, qh, s, e);
                    e += pl + ql;
                    two_sum(s, e, h, l);
                } else {
                    two_sum(ph, pl, h, l);
                }
                out_hi[i + j * nrows] = h;
                out_lo[i + j * nrows] = l;
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
}

template <typename T>
void dd_gemm_any(int layout, int transa, int transb, size_t m, size_t n, size_t k, double alpha,
                 const T* a, size_t lda, const T* b, size_t ldb, double beta, const T* c0,
                 size_t ldc, const int64_t* rows, size_t nrows, double* out_hi, double* out_lo,
                 int threads) {
    // Element accessors in the caller's layout (src/types.rs:20-25 strides).
    auto at = [&](size_t r, size_t cc, const T* x, size_t ld) -> double {
        return layout == 1 ? (double)x[r + cc * ld] : (double)x[r * ld + cc];
    };
    bool ta = transa != 0, tb = transb != 0;
    std::vector<double> am(nrows * k), bm(k * n), c0m;
    for (size_t p = 0; p < k; ++p)
        for (size_t ii = 0; ii < nrows; ++ii) {
            size_t i = rows ? (size_t)rows[ii] : ii;
            am[ii + p * nrows] = ta ? at(p, i, a, lda) : at(i, p, a, lda);
        }
    for (size_t j = 0; j < n; ++j)
        for (size_t p = 0; p < k; ++p) bm[p + j * k] = tb ? at(j, p, b, ldb) : at(p, j, b, ldb);
    if (c0 && beta != 0.0) {
        c0m.resize(nrows * n);
        for (size_t j = 0; j < n; ++j)
            for (size_t ii = 0; ii < nrows; ++ii) {
                size_t i = rows ? (size_t)rows[ii] : ii;
                c0m[ii + j * nrows] = at(i, j, c0, ldc);
            }
    }
    dd_gemm_core(nrows, n, k, alpha, am.data(), bm.data(), beta, c0m.empty() ? nullptr : c0m.data(),
                 out_hi, out_lo, threads);
}

}  // namespace

// ---- Level 1 (src/level1.rs, src/complex1.rs, src/kernel/{avx2,scalar}.rs) ----

// src/kernel/avx2.rs:30-56 / 104-130: two W-lane fma accumulators over
// blocks of 2W, then W, hsum of acc0+acc1 (hsum256_ps / hsum256_pd order),
// then the tail with scalar fma. src/kernel/scalar.rs: 4 accumulators.
template <typename T>
T dot_contig(size_t n, const T* x, const T* y) {
    if (have_avx2_fma()) {
        constexpr size_t W = sizeof(T) == 4 ? 8 : 4;
        T a0[W] = {}, a1[W] = {};
        size_t i = 0;
        for (; i + 2 * W <= n; i += 2 * W)
            for (size_t l = 0; l < W; ++l) {
                a0[l] = fmaT(x[i + l], y[i + l], a0[l]);
                a1[l] = fmaT(x[i + W + l], y[i + W + l], a1[l]);
            }
        for (; i + W <= n; i += W)
            for (size_t l = 0; l < W; ++l) a0[l] = fmaT(x[i + l], y[i + l], a0[l]);
        T v[W];
        for (size_t l = 0; l < W; ++l) v[l] = a0[l] + a1[l];
        T acc;
        if (W == 8) {  // lo + hi, then movehl, then lane 1
            T t[4];
            for (int k = 0; k < 4; ++k) t[k] = v[k] + v[k + 4];
            const T u0 = t[0] + t[2], u1 = t[1] + t[3];
            acc = u0 + u1;
        } else {
            const T t0 = v[0] + v[2], t1 = v[1] + v[3];
            acc = t0 + t1;
        }
        for (; i < n; ++i) acc = fmaT(x[i], y[i], acc);
        return acc;
    }
    T a0 = T(0), a1 = T(0), a2 = T(0), a3 = T(0);
    const size_t chunks = n / 4;
    for (size_t k = 0; k < chunks; ++k) {
        const size_t i = k * 4;
        a0 = fmaT(x[i], y[i], a0);
        a1 = fmaT(x[i + 1], y[i + 1], a1);
        a2 = fmaT(x[i + 2], y[i + 2], a2);
        a3 = fmaT(x[i + 3], y[i + 3], a3);
    }
    T acc = (a0 + a1) + (a2 + a3);
    for (size_t i = chunks * 4; i < n; ++i) acc = fmaT(x[i], y[i], acc);
    return acc;
}

// src/level1.rs:45-66
template <typename T>
T dot_impl(size_t n, const T* x, size_t incx, const T* y, size_t incy) {
    if (n == 0) return T(0);
    if (incx == 1 && incy == 1) return dot_contig(n, x, y);
    T acc = T(0);
    for (size_t q = 0; q < n; ++q) acc = fmaT(x[q * incx], y[q * incy], acc);
    return acc;
}

// src/level1.rs:96-124 (scaled sum of squares); complex: both components (src/complex1.rs:86-118)
template <typename T>
void nrm2_step(T xi, T& scale, T& ssq) {
    if (xi != T(0)) {
        const T a = std::fabs(xi);
        if (scale < a) {
            const T r = scale / a;
            ssq = T(1) + ssq * (r * r);
            scale = a;
        } else {
            const T r = a / scale;
            ssq = ssq + r * r;
        }
    }
}

// ---- trmm (no rblas counterpart: the textbook definition) ---------------------
// out = alpha * op(A) * B (Left) or alpha * B * op(A) (Right), op(A) the
// triangle of A (unit diagonal when diag), each output accumulated in index
// order with fma (real) or acc + a*b (complex); then B = out.
template <typename T>
inline T tri_at(const T* a, size_t lda, int uplo, int trans, int diag, size_t i, size_t j) {
    const size_t r = trans ? j : i, c = trans ? i : j;
    if (r == c && diag) return T(1);
    const bool stored = uplo == 0 ? r <= c : r >= c;
    return stored ? a[r + c * lda] : T(0);
}
template <typename T>
void trmm_impl(int side, int uplo, int trans, int diag, size_t m, size_t n, T alpha, const T* a, size_t lda, T* b,
               size_t ldb) {
    std::vector<T> out(m * n);
    for (size_t j = 0; j < n; ++j)
        for (size_t i = 0; i < m; ++i) {
            T acc = T(0);
            if (side == 0)
                for (size_t k = 0; k < m; ++k) acc = fmaT(tri_at(a, lda, uplo, trans, diag, i, k), b[k + j * ldb], acc);
            else
                for (size_t k = 0; k < n; ++k) acc = fmaT(b[i + k * ldb], tri_at(a, lda, uplo, trans, diag, k, j), acc);
            out[i + j * m] = alpha * acc;
        }
    for (size_t j = 0; j < n; ++j)
        for (size_t i = 0; i < m; ++i) b[i + j * ldb] = out[i + j * m];
}

// ---- Level 2 (src/level2.rs, src/complex2.rs) -------------------------------
// (rs, cs) = layout.strides(lda): RowMajor (lda, 1), ColMajor (1, lda)  src/types.rs:20-25

// src/level2.rs:91-104 (scale_y), 11-62 (gemv)
template <typename T>
void gemv_impl(int layout, int trans, size_t m, size_t n, T alpha, const T* a, size_t lda, const T* x,
               size_t incx, T beta, T* y, size_t incy) {
    const size_t rs = layout == 0 ? lda : 1, cs = layout == 0 ? 1 : lda;
    const bool tr = trans != 0;
    const size_t leny = tr ? n : m;
    if (beta != T(1)) {
        size_t iy = 0;
        for (size_t q = 0; q < leny; ++q) {
            y[iy] = (beta == T(0)) ? T(0) : beta * y[iy];
            iy += incy;
        }
    }
    if (alpha == T(0)) return;
    if (!tr) {
        for (size_t i = 0; i < m; ++i) {
            T acc = T(0);
            size_t jx = 0;
            for (size_t j = 0; j < n; ++j) {
                acc = fmaT(a[i * rs + j * cs], x[jx], acc);
                jx += incx;
            }
            y[i * incy] = fmaT(alpha, acc, y[i * incy]);
        }
    } else {
        for (size_t i = 0; i < m; ++i) {
            const T xi = alpha * x[i * incx];
            for (size_t j = 0; j < n; ++j) {
                const size_t yj = j * incy;
                y[yj] = fmaT(a[i * rs + j * cs], xi, y[yj]);
            }
        }
    }
}

// src/level2.rs:65-88
template <typename T>
void ger_impl(int layout, size_t m, size_t n, T alpha, const T* x, size_t incx, const T* y, size_t incy, T* a,
              size_t lda) {
    if (alpha == T(0)) return;
    const size_t rs = layout == 0 ? lda : 1, cs = layout == 0 ? 1 : lda;
    for (size_t i = 0; i < m; ++i) {
        const T axi = alpha * x[i * incx];
        for (size_t j = 0; j < n; ++j) {
            const size_t idx = i * rs + j * cs;
            a[idx] = fmaT(axi, y[j * incy], a[idx]);
        }
    }
}

// src/complex2.rs:11-77. The beta pass runs whenever beta is zero or not one,
// which is always ("!is_zero || != one"): beta == 1 still multiplies.
template <typename T>
void cgemv_impl(int layout, int trans, size_t m, size_t n, Cx<T> alpha, const Cx<T>* a, size_t lda, const Cx<T>* x,
                size_t incx, Cx<T> beta, Cx<T>* y, size_t incy) {
    const size_t rs = layout == 0 ? lda : 1, cs = layout == 0 ? 1 : lda;
    const bool conj = trans == 2, tr = trans != 0;
    const size_t leny = tr ? n : m;
    const bool beta_zero = beta.re == T(0) && beta.im == T(0);
    const bool beta_one = beta.re == T(1) && beta.im == T(0);
    if (!beta_zero || !beta_one) {
        size_t iy = 0;
        for (size_t q = 0; q < leny; ++q) {
            y[iy] = beta_zero ? Cx<T>{T(0), T(0)} : cmul(beta, y[iy]);
            iy += incy;
        }
    }
    if (alpha.re == T(0) && alpha.im == T(0)) return;
    auto aval = [&](size_t i, size_t j) {
        const Cx<T> v = a[i * rs + j * cs];
        return conj ? cconj(v) : v;
    };
    if (!tr) {
        for (size_t i = 0; i < m; ++i) {
            Cx<T> acc{T(0), T(0)};
            size_t jx = 0;
            for (size_t j = 0; j < n; ++j) {
                acc = cadd(acc, cmul(aval(i, j), x[jx]));
                jx += incx;
            }
            y[i * incy] = cadd(y[i * incy], cmul(alpha, acc));
        }
    } else {
        for (size_t j = 0; j < n; ++j) {
            Cx<T> acc{T(0), T(0)};
            size_t ix = 0;
            for (size_t i = 0; i < m; ++i) {
                acc = cadd(acc, cmul(aval(i, j), x[ix]));
                ix += incx;
            }
            y[j * incy] = cadd(y[j * incy], cmul(alpha, acc));
        }
    }
}

// src/complex2.rs:80-145 (geru conj = false, gerc conj = true)
template <typename T>
void crank1_impl(int layout, size_t m, size_t n, Cx<T> alpha, const Cx<T>* x, size_t incx, const Cx<T>* y,
                 size_t incy, Cx<T>* a, size_t lda, bool conj) {
    if (alpha.re == T(0) && alpha.im == T(0)) return;
    const size_t rs = layout == 0 ? lda : 1, cs = layout == 0 ? 1 : lda;
    for (size_t i = 0; i < m; ++i) {
        const Cx<T> axi = cmul(alpha, x[i * incx]);
        for (size_t j = 0; j < n; ++j) {
            const Cx<T> yj = conj ? cconj(y[j * incy]) : y[j * incy];
            const size_t idx = i * rs + j * cs;
            a[idx] = cadd(a[idx], cmul(axi, yj));
        }
    }
}

// ============================================================================
// extern "C" surface used by the test harness (ctypes). Integer enums follow
// the product header: layout 0=RowMajor 1=ColMajor; trans 0=None 1=Trans
// 2=ConjTrans; uplo 0=Upper 1=Lower; side 0=Left 1=Right; diag 0=NonUnit 1=Unit.
// ============================================================================

extern "C" {

struct or_error {
    int32_t code;   // 0 ok, 1 InvalidLeadingDim, 2 BufferTooSmall
    char which;     // 'a' | 'b' | 'c'
    uint64_t got;
    uint64_t min_or_need;
};

void or_set_force_scalar(int on) { g_force_scalar = on != 0; }

// The reference tests' dependency-free LCG (tests/correctness.rs:21-26 and
// tests/parallel.rs:9-14): s = s*6364136223846793005 + 1442695040888963407.
// mode 0: ((s>>33) as f32 / 2^31) - 1.0   (correctness.rs, U[-1,1))
// mode 1: ((s>>40) as f32 / 2^24) - 0.5   (parallel.rs, U[-0.5,0.5))
// Every f32 operation is a single IEEE rounding, as in the Rust expression.
uint64_t or_lcg_fill_f32(uint64_t seed, int mode, size_t n, float* out) {
    uint64_t s = seed;
    for (size_t i = 0; i < n; ++i) {
        s = s * 6364136223846793005ULL + 1442695040888963407ULL;
        if (mode == 0) {
            float v = (float)(s >> 33);
            out[i] = v / (float)(1ULL << 31) - 1.0f;
        } else {
            float v = (float)(s >> 40);
            out[i] = v / (float)(1ULL << 24) - 0.5f;
        }
    }
    return s;
}
int or_have_avx2_fma(void) { return have_avx2_fma() ? 1 : 0; }

// src/level3.rs:107-140
static int check_matrix(int layout, char which, size_t rows, size_t cols, size_t lead, size_t len,
                        or_error* err) {
    if (rows == 0 || cols == 0) return 0;
    size_t min_lead = layout == 0 ? cols : rows;
    size_t need = layout == 0 ? (rows - 1) * lead + cols : (cols - 1) * lead + rows;
    if (lead < min_lead) {
        if (err) *err = {1, which, lead, min_lead};
        return 1;
    }
    if (len < need) {
        if (err) *err = {2, which, len, need};
        return 2;
    }
    return 0;
}

// src/level3.rs:68-103 (validation only; returns the error code)
int or_check_gemm(int layout, int transa, int transb, size_t m, size_t n, size_t k, size_t lda,
                  size_t a_len, size_t ldb, size_t b_len, size_t ldc, size_t c_len, or_error* err) {
    if (err) *err = {0, 0, 0, 0};
    size_t ar = transa ? k : m, ac = transa ? m : k;
    size_t br = transb ? n : k, bc = transb ? k : n;
    int rc = check_matrix(layout, 'a', ar, ac, lda, a_len, err);
    if (rc) return rc;
    rc = check_matrix(layout, 'b', br, bc, ldb, b_len, err);
    if (rc) return rc;
    return check_matrix(layout, 'c', m, n, ldc, c_len, err);
}

void or_sgemm(int layout, int transa, int transb, size_t m, size_t n, size_t k, float alpha,
              const float* a, size_t lda, const float* b, size_t ldb, float beta, float* c,
              size_t ldc, int threads) {
    gemm_any<float>(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, threads);
}
void or_dgemm(int layout, int transa, int transb, size_t m, size_t n, size_t k, double alpha,
              const double* a, size_t lda, const double* b, size_t ldb, double beta, double* c,
              size_t ldc, int threads) {
    gemm_any<double>(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, threads);
}

void or_ssyrk(int uplo, int trans, size_t n, size_t k, float alpha, const float* a, size_t lda,
              float beta, float* c, size_t ldc, int threads) {
    syrk_impl<float>(uplo, trans, n, k, alpha, a, lda, beta, c, ldc, threads);
}
void or_dsyrk(int uplo, int trans, size_t n, size_t k, double alpha, const double* a, size_t lda,
              double beta, double* c, size_t ldc, int threads) {
    syrk_impl<double>(uplo, trans, n, k, alpha, a, lda, beta, c, ldc, threads);
}
void or_ssymm(int side, int uplo, size_t m, size_t n, float alpha, const float* a, size_t lda,
              const float* b, size_t ldb, float beta, float* c, size_t ldc, int threads) {
    symm_impl<float>(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, threads);
}
void or_dsymm(int side, int uplo, size_t m, size_t n, double alpha, const double* a, size_t lda,
              const double* b, size_t ldb, double beta, double* c, size_t ldc, int threads) {
    symm_impl<double>(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, threads);
}
void or_strsm(int side, int uplo, int trans, int diag, size_t m, size_t n, float alpha,
              const float* a, size_t lda, float* b, size_t ldb) {
    trsm_impl<float>(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb);
}
void or_dtrsm(int side, int uplo, int trans, int diag, size_t m, size_t n, double alpha,
              const double* a, size_t lda, double* b, size_t ldb) {
    trsm_impl<double>(side, uplo, trans, diag, m, n, alpha, a, lda, b, ldb);
}

// Complex: pointers to interleaved (re, im) pairs; alpha/beta as (re, im).
void or_cgemm(int transa, int transb, size_t m, size_t n, size_t k, float ar, float ai,
              const float* a, size_t lda, const float* b, size_t ldb, float br, float bi, float* c,
              size_t ldc, int threads) {
    cgemm_impl<float>(transa, transb, m, n, k, {ar, ai}, (const Cx<float>*)a, lda,
                      (const Cx<float>*)b, ldb, {br, bi}, (Cx<float>*)c, ldc, threads);
}
void or_zgemm(int transa, int transb, size_t m, size_t n, size_t k, double ar, double ai,
              const double* a, size_t lda, const double* b, size_t ldb, double br, double bi,
              double* c, size_t ldc, int threads) {
    cgemm_impl<double>(transa, transb, m, n, k, {ar, ai}, (const Cx<double>*)a, lda,
                       (const Cx<double>*)b, ldb, {br, bi}, (Cx<double>*)c, ldc, threads);
}
void or_chemm(int hermitian, int side, int uplo, size_t m, size_t n, float ar, float ai,
              const float* a, size_t lda, const float* b, size_t ldb, float br, float bi, float* c,
              size_t ldc, int threads) {
    he_or_sy<float>(side, uplo, m, n, {ar, ai}, (const Cx<float>*)a, lda, (const Cx<float>*)b, ldb,
                    {br, bi}, (Cx<float>*)c, ldc, hermitian != 0, threads);
}
void or_zhemm(int hermitian, int side, int uplo, size_t m, size_t n, double ar, double ai,
              const double* a, size_t lda, const double* b, size_t ldb, double br, double bi,
              double* c, size_t ldc, int threads) {
    he_or_sy<double>(side, uplo, m, n, {ar, ai}, (const Cx<double>*)a, lda, (const Cx<double>*)b,
                     ldb, {br, bi}, (Cx<double>*)c, ldc, hermitian != 0, threads);
}
void or_ctrsm(int side, int uplo, int trans, int diag, size_t m, size_t n, float ar, float ai,
              const float* a, size_t lda, float* b, size_t ldb) {
    ctrsm_impl<float>(side, uplo, trans, diag, m, n, {ar, ai}, (const Cx<float>*)a, lda,
                      (Cx<float>*)b, ldb);
}
void or_ztrsm(int side, int uplo, int trans, int diag, size_t m, size_t n, double ar, double ai,
              const double* a, size_t lda, double* b, size_t ldb) {
    ctrsm_impl<double>(side, uplo, trans, diag, m, n, {ar, ai}, (const Cx<double>*)a, lda,
                       (Cx<double>*)b, ldb);
}

// Double-double oracle for real GEMM in the caller's layout. `rows` (length
// nrows) selects output rows of C (null = all m rows, nrows must equal m).
// Output hi/lo are nrows x n col-major.
void or_dd_sgemm(int layout, int transa, int transb, size_t m, size_t n, size_t k, double alpha,
                 const float* a, size_t lda, const float* b, size_t ldb, double beta,
                 const float* c0, size_t ldc, const int64_t* rows, size_t nrows, double* hi,
                 double* lo, int threads) {
    (void)m;
    dd_gemm_any<float>(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c0, ldc, rows,
                       nrows, hi, lo, threads);
}
void or_dd_dgemm(int layout, int transa, int transb, size_t m, size_t n, size_t k, double alpha,
                 const double* a, size_t lda, const double* b, size_t ldb, double beta,
                 const double* c0, size_t ldc, const int64_t* rows, size_t nrows, double* hi,
                 double* lo, int threads) {
    (void)m;
    dd_gemm_any<double>(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c0, ldc,
                        rows, nrows, hi, lo, threads);
}

// Double-double oracle core on pre-materialised col-major panels (used by
// the complex oracle, which forms the real block operands in numpy).
void or_dd_core(size_t nrows, size_t n, size_t k, double alpha, const double* am, const double* bm,
                double beta, const double* c0, double* hi, double* lo, int threads) {
    dd_gemm_core(nrows, n, k, alpha, am, bm, beta, c0, hi, lo, threads);
}

void or_sgemv(int layout, int trans, size_t m, size_t n, float alpha, const float* a, size_t lda,
              const float* x, size_t incx, float beta, float* y, size_t incy) {
    gemv_impl<float>(layout, trans, m, n, alpha, a, lda, x, incx, beta, y, incy);
}
void or_dgemv(int layout, int trans, size_t m, size_t n, double alpha, const double* a, size_t lda,
              const double* x, size_t incx, double beta, double* y, size_t incy) {
    gemv_impl<double>(layout, trans, m, n, alpha, a, lda, x, incx, beta, y, incy);
}
void or_sger(int layout, size_t m, size_t n, float alpha, const float* x, size_t incx, const float* y, size_t incy,
             float* a, size_t lda) {
    ger_impl<float>(layout, m, n, alpha, x, incx, y, incy, a, lda);
}
void or_dger(int layout, size_t m, size_t n, double alpha, const double* x, size_t incx, const double* y,
             size_t incy, double* a, size_t lda) {
    ger_impl<double>(layout, m, n, alpha, x, incx, y, incy, a, lda);
}
void or_cgemv(int layout, int trans, size_t m, size_t n, float ar, float ai, const float* a, size_t lda,
              const float* x, size_t incx, float br, float bi, float* y, size_t incy) {
    cgemv_impl<float>(layout, trans, m, n, {ar, ai}, reinterpret_cast<const Cx<float>*>(a), lda,
                      reinterpret_cast<const Cx<float>*>(x), incx, {br, bi}, reinterpret_cast<Cx<float>*>(y), incy);
}
void or_zgemv(int layout, int trans, size_t m, size_t n, double ar, double ai, const double* a, size_t lda,
              const double* x, size_t incx, double br, double bi, double* y, size_t incy) {
    cgemv_impl<double>(layout, trans, m, n, {ar, ai}, reinterpret_cast<const Cx<double>*>(a), lda,
                       reinterpret_cast<const Cx<double>*>(x), incx, {br, bi}, reinterpret_cast<Cx<double>*>(y),
                       incy);
}
void or_cger(int layout, size_t m, size_t n, float ar, float ai, const float* x, size_t incx, const float* y,
             size_t incy, float* a, size_t lda, int conj) {
    crank1_impl<float>(layout, m, n, {ar, ai}, reinterpret_cast<const Cx<float>*>(x), incx,
                       reinterpret_cast<const Cx<float>*>(y), incy, reinterpret_cast<Cx<float>*>(a), lda, conj != 0);
}
void or_zger(int layout, size_t m, size_t n, double ar, double ai, const double* x, size_t incx, const double* y,
             size_t incy, double* a, size_t lda, int conj) {
    crank1_impl<double>(layout, m, n, {ar, ai}, reinterpret_cast<const Cx<double>*>(x), incx,
                        reinterpret_cast<const Cx<double>*>(y), incy, reinterpret_cast<Cx<double>*>(a), lda,
                        conj != 0);
}

void or_dtrmm(int side, int uplo, int trans, int diag, size_t m, size_t n, double alpha, const double* a,
              size_t lda, double* b, size_t ldb) {
    trmm_impl<double>(side, uplo, trans != 0, diag, m, n, alpha, a, lda, b, ldb);
}
void or_strmm(int side, int uplo, int trans, int diag, size_t m, size_t n, float alpha, const float* a, size_t lda,
              float* b, size_t ldb) {
    trmm_impl<float>(side, uplo, trans != 0, diag, m, n, alpha, a, lda, b, ldb);
}

// Level 1, real (src/level1.rs)
#define OR_L1_REAL(P, T)                                                                                           \
    void or_##P##axpy(size_t n, T alpha, const T* x, size_t incx, T* y, size_t incy) {                             \
        if (n == 0 || alpha == T(0)) return;                                                                       \
        for (size_t q = 0; q < n; ++q) y[q * incy] = fmaT(alpha, x[q * incx], y[q * incy]);                        \
    }                                                                                                              \
    T or_##P##dot(size_t n, const T* x, size_t incx, const T* y, size_t incy) { return dot_impl(n, x, incx, y, incy); } \
    void or_##P##scal(size_t n, T alpha, T* x, size_t incx) {                                                      \
        if (n == 0 || alpha == T(1)) return;                                                                       \
        for (size_t q = 0; q < n; ++q) x[q * incx] = alpha * x[q * incx];                                          \
    }                                                                                                              \
    T or_##P##nrm2(size_t n, const T* x, size_t incx) {                                                            \
        if (n == 0) return T(0);                                                                                   \
        T scale = T(0), ssq = T(1);                                                                                \
        for (size_t q = 0; q < n; ++q) nrm2_step(x[q * incx], scale, ssq);                                         \
        return scale * std::sqrt(ssq);                                                                             \
    }                                                                                                              \
    T or_##P##asum(size_t n, const T* x, size_t incx) {                                                            \
        T acc = T(0);                                                                                              \
        for (size_t q = 0; q < n; ++q) acc = acc + std::fabs(x[q * incx]);                                         \
        return acc;                                                                                                \
    }                                                                                                              \
    /* src/level1.rs:139-163: element by element in order (zero strides included) */                             \
    void or_##P##copy(size_t n, const T* x, size_t incx, T* y, size_t incy) {                                      \
        for (size_t q = 0; q < n; ++q) y[q * incy] = x[q * incx];                                                  \
    }                                                                                                              \
    void or_##P##swap(size_t n, T* x, size_t incx, T* y, size_t incy) {                                            \
        for (size_t q = 0; q < n; ++q) std::swap(x[q * incx], y[q * incy]);                                        \
    }
OR_L1_REAL(s, float)
OR_L1_REAL(d, double)
#undef OR_L1_REAL

// Level 1, complex (src/complex1.rs); results returned through out[2]
#define OR_L1_CPLX(P, T)                                                                                           \
    void or_##P##axpy(size_t n, T ar, T ai, const T* x, size_t incx, T* y, size_t incy) {                          \
        if (n == 0 || (ar == T(0) && ai == T(0))) return;                                                          \
        const Cx<T> al{ar, ai};                                                                                    \
        auto X = reinterpret_cast<const Cx<T>*>(x);                                                                \
        auto Y = reinterpret_cast<Cx<T>*>(y);                                                                      \
        for (size_t q = 0; q < n; ++q) Y[q * incy] = cadd(cmul(al, X[q * incx]), Y[q * incy]);                     \
    }                                                                                                              \
    void or_##P##dot(size_t n, const T* x, size_t incx, const T* y, size_t incy, int conj, T* out) {               \
        auto X = reinterpret_cast<const Cx<T>*>(x);                                                                \
        auto Y = reinterpret_cast<const Cx<T>*>(y);                                                                \
        Cx<T> acc{T(0), T(0)};                                                                                     \
        for (size_t q = 0; q < n; ++q) acc = cadd(acc, cmul(conj ? cconj(X[q * incx]) : X[q * incx], Y[q * incy])); \
        out[0] = acc.re;                                                                                           \
        out[1] = acc.im;                                                                                           \
    }                                                                                                              \
    void or_##P##scal(size_t n, T ar, T ai, T* x, size_t incx) {                                                   \
        const Cx<T> al{ar, ai};                                                                                    \
        auto X = reinterpret_cast<Cx<T>*>(x);                                                                      \
        for (size_t q = 0; q < n; ++q) X[q * incx] = cmul(al, X[q * incx]);                                        \
    }                                                                                                              \
    T or_##P##nrm2(size_t n, const T* x, size_t incx) {                                                            \
        if (n == 0) return T(0);                                                                                   \
        T scale = T(0), ssq = T(1);                                                                                \
        for (size_t q = 0; q < n; ++q) {                                                                           \
            nrm2_step(x[2 * q * incx], scale, ssq);                                                                \
            nrm2_step(x[2 * q * incx + 1], scale, ssq);                                                            \
        }                                                                                                          \
        return scale * std::sqrt(ssq);                                                                             \
    }
OR_L1_CPLX(c, float)
OR_L1_CPLX(z, double)
#undef OR_L1_CPLX

}  // extern "C"
