// level1.cu -- Level-1 BLAS on the GPU (src/level1.rs, src/complex1.rs).
//
// axpy, scal, copy and swap are elementwise and compute each element exactly
// as rblas does: fma(alpha, x, y) for real axpy (src/level1.rs:37 and the
// fused kernels of src/kernel/), alpha*x for scal, and rblas's complex
// multiply (src/complex.rs:101-111) for the complex forms. dot / dotu / dotc,
// asum and nrm2 are reductions in a fixed order: each thread folds a fixed
// strided set of elements in index order, a block folds its threads in a
// fixed tree, and one final block folds the block results in block order.
// The grid depends on n and on contiguity only (never on the device), so a
// result is the same bit for bit on every call; it differs from rblas's
// sequential sum within rounding. nrm2 is a scaled sum of squares like
// rblas's (src/level1.rs:96-124), so it neither overflows nor underflows,
// with the scale a power of two (see Nrm below) instead of the running
// maximum, which takes the division out of the per-element step.
//
// Every kernel here is bound by HBM bandwidth. Contiguous, 16-byte-aligned
// vectors move in 16-byte loads and stores, several per thread in flight;
// other strides take one element per thread per step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "../../include/rblas_b200.h"
#include "rb_internal.h"

namespace rb {

namespace {

constexpr int kL1Threads = 256;
// One wave on a B200 (148 SMs x 4 resident blocks of kL1Threads); a
// constant, so the reduction order depends on n only, never on the device.
constexpr int kL1BlocksPerSm = 4;
constexpr int kL1MaxBlocks = 148 * kL1BlocksPerSm;
constexpr int kUnroll = 4;

template <typename T> struct Z { T re, im; };

__device__ __forceinline__ float mulr(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mulr(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float addr(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double addr(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float subr(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double subr(double a, double b) { return __dsub_rn(a, b); }

// rblas's complex multiply: re = fma(a.re, b.re, 0 - a.im*b.im), im = fma(a.re, b.im, a.im*b.re)
template <typename T>
__device__ __forceinline__ Z<T> zmul(Z<T> a, Z<T> b) {
    return {fma(a.re, b.re, subr(T(0), mulr(a.im, b.im))), fma(a.re, b.im, mulr(a.im, b.re))};
}
template <typename T>
__device__ __forceinline__ Z<T> zadd(Z<T> a, Z<T> b) { return {addr(a.re, b.re), addr(a.im, b.im)}; }

// 16-byte vector moves: K scalars of T
template <typename T> constexpr int kVec = 16 / static_cast<int>(sizeof(T));

__device__ __forceinline__ void ld16nc(const float* p, float (&r)[4]) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    r[0] = v.x; r[1] = v.y; r[2] = v.z; r[3] = v.w;
}
__device__ __forceinline__ void ld16nc(const double* p, double (&r)[2]) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(p));
    r[0] = v.x; r[1] = v.y;
}
__device__ __forceinline__ void ld16(const float* p, float (&r)[4]) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    r[0] = v.x; r[1] = v.y; r[2] = v.z; r[3] = v.w;
}
__device__ __forceinline__ void ld16(const double* p, double (&r)[2]) {
    const double2 v = *reinterpret_cast<const double2*>(p);
    r[0] = v.x; r[1] = v.y;
}
__device__ __forceinline__ void st16(float* p, const float (&r)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(r[0], r[1], r[2], r[3]);
}
__device__ __forceinline__ void st16(double* p, const double (&r)[2]) {
    *reinterpret_cast<double2*>(p) = make_double2(r[0], r[1]);
}

// ---- elementwise -------------------------------------------------------------

// One element of op at x / y (complex: two scalars, {re, im}). SCAL scales y.
template <typename T, bool CX, int OP>
__device__ __forceinline__ void ew_elem(T* x, T* y, Z<T> al) {
    if constexpr (OP == L1_AXPY) {
        if constexpr (CX) {
            const Z<T> r = zadd(zmul(al, Z<T>{__ldg(x), __ldg(x + 1)}), Z<T>{y[0], y[1]});  // src/complex1.rs:23
            y[0] = r.re;
            y[1] = r.im;
        } else {
            *y = fma(al.re, __ldg(x), *y);  // src/level1.rs:37
        }
    } else if constexpr (OP == L1_SCAL) {
        if constexpr (CX) {
            const Z<T> r = zmul(al, Z<T>{y[0], y[1]});  // src/complex1.rs:78
            y[0] = r.re;
            y[1] = r.im;
        } else {
            *y = mulr(al.re, *y);  // src/level1.rs:82
        }
    } else if constexpr (OP == L1_COPY) {
        y[0] = x[0];
        if constexpr (CX) y[1] = x[1];
    } else {  // L1_SWAP
        const T t0 = x[0];
        x[0] = y[0];
        y[0] = t0;
        if constexpr (CX) {
            const T t1 = x[1];
            x[1] = y[1];
            y[1] = t1;
        }
    }
}

// The same op over K consecutive scalars held in registers.
template <typename T, bool CX, int OP, int K>
__device__ __forceinline__ void ew_vec(T (&xs)[K], T (&ys)[K], Z<T> al) {
    if constexpr (OP == L1_AXPY || OP == L1_SCAL) {
        if constexpr (CX) {
#pragma unroll
            for (int k = 0; k < K; k += 2) {
                const Z<T> r = OP == L1_AXPY ? zadd(zmul(al, Z<T>{xs[k], xs[k + 1]}), Z<T>{ys[k], ys[k + 1]})
                                             : zmul(al, Z<T>{ys[k], ys[k + 1]});
                ys[k] = r.re;
                ys[k + 1] = r.im;
            }
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) ys[k] = OP == L1_AXPY ? fma(al.re, xs[k], ys[k]) : mulr(al.re, ys[k]);
        }
    } else if constexpr (OP == L1_COPY) {
#pragma unroll
        for (int k = 0; k < K; ++k) ys[k] = xs[k];
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const T t = xs[k];
            xs[k] = ys[k];
            ys[k] = t;
        }
    }
}

// Contiguous, 16-byte-aligned vectors: block b owns the U*kL1Threads
// consecutive 16-byte vectors from b*U*kL1Threads (thread t takes t, t+256,
// ...: every load and store coalesced), and the grid covers the vector in
// waves. On B200 this tiling streams mixed read/write traffic faster than a
// persistent grid-stride loop (copy 6.9 vs 5.8 TB/s at 1 GiB). The last block
// also takes the ragged tail of whole elements after the last full vector.
template <typename T, bool CX, int OP, int U>
__global__ void __launch_bounds__(kL1Threads) ew_tile_kernel(size_t n, Z<T> al, T* x, T* y) {
    constexpr int K = kVec<T>;
    constexpr int E = CX ? 2 : 1;
    constexpr bool reads_x = OP != L1_SCAL, reads_y = OP != L1_COPY, writes_x = OP == L1_SWAP;
    const size_t nv = n * E / K;  // whole 16-byte vectors
    const size_t base = static_cast<size_t>(blockIdx.x) * (U * kL1Threads) + threadIdx.x;
    T xs[U][K], ys[U][K];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const size_t v = base + static_cast<size_t>(u) * kL1Threads;
        if (v < nv) {
            if constexpr (reads_x) {
                if constexpr (writes_x) ld16(x + v * K, xs[u]); else ld16nc(x + v * K, xs[u]);
            }
            if constexpr (reads_y) ld16(y + v * K, ys[u]);
        }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const size_t v = base + static_cast<size_t>(u) * kL1Threads;
        if (v < nv) {
            ew_vec<T, CX, OP, K>(xs[u], ys[u], al);
            st16(y + v * K, ys[u]);
            if constexpr (writes_x) st16(x + v * K, xs[u]);
        }
    }
    if (blockIdx.x == gridDim.x - 1) {
#pragma unroll 1
        for (size_t i = nv * K / E + threadIdx.x; i < n; i += kL1Threads)  // K is even: whole elements
            ew_elem<T, CX, OP>(reads_x ? x + i * E : nullptr, y + i * E, al);
    }
}

// Any other strides or alignment: one element per thread per step.
template <typename T, bool CX, int OP>
__global__ void __launch_bounds__(kL1Threads, kL1BlocksPerSm)
    ew_strided_kernel(size_t n, Z<T> al, T* x, size_t incx, T* y, size_t incy) {
    constexpr int E = CX ? 2 : 1;
    const size_t nth = static_cast<size_t>(gridDim.x) * kL1Threads;
#pragma unroll 1
    for (size_t i = static_cast<size_t>(blockIdx.x) * kL1Threads + threadIdx.x; i < n; i += nth)
        ew_elem<T, CX, OP>(OP != L1_SCAL ? x + i * incx * E : nullptr, y + i * incy * E, al);
}

// ---- reductions ----------------------------------------------------------------

// nrm2's partial state: the sum of squares of the finite elements seen, kept
// as ssq relative to 2^e, where 2^e is the smallest power of two above the
// largest magnitude (lim = 2^e, inv = 2^-e). Scaling by a power of two is
// exact, so an element costs a multiply and an fma, and a rescale is exact
// too (or flushes contributions far below the maximum to 0, as rblas's
// ratio does); there is no division. Neither overflow nor underflow: every
// scaled element is below 1, and e never drops below kMinExp, so the
// smallest subnormal still squares to a normal number. An empty state has
// e = kEmpty. Infinities are counted apart (ninf) so the result keeps
// rblas's outcome: one inf gives inf, two or more give NaN (its inf/inf
// rescale), a NaN gives NaN (it reaches ssq through the multiply).
template <typename T> struct Nrm {
    T ssq, lim, inv;
    int e, ninf;
};
template <typename T> struct NrmLimits;
template <> struct NrmLimits<float> { static constexpr int kMinExp = -100; };
template <> struct NrmLimits<double> { static constexpr int kMinExp = -1000; };
constexpr int kEmpty = -4096;

__device__ __forceinline__ float ldx(float v, int e) { return ldexpf(v, e); }
__device__ __forceinline__ double ldx(double v, int e) { return ldexp(v, e); }
__device__ __forceinline__ int exponent_above(float m) {  // 2^e > m >= 2^(e-1)
    int e;
    frexpf(m, &e);
    return e;
}
__device__ __forceinline__ int exponent_above(double m) {
    int e;
    frexp(m, &e);
    return e;
}

template <typename T>
__device__ __forceinline__ Nrm<T> nrm_zero() { return {T(1), T(0), T(0), kEmpty, 0}; }

// N scalars into a state: their largest finite magnitude may raise e first.
template <typename T, int N>
__device__ __forceinline__ void nrm_chunk(Nrm<T>& s, const T (&v)[N]) {
    T a[N];
    T m = T(0);
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const T ak = fabs(v[k]);
        const bool inf = isinf(ak);
        s.ninf += inf ? 1 : 0;
        a[k] = inf ? T(0) : v[k];
        m = fmax(m, inf ? T(0) : ak);  // a NaN is skipped here and reaches ssq below
    }
    if (m > T(0) && m >= s.lim) {
        const int e = max(exponent_above(m), NrmLimits<T>::kMinExp);
        const T inv = ldx(T(1), -e);
        const T f = mulr(s.lim, inv);  // 2^(e_old - e), exact or 0
        s.ssq = mulr(s.ssq, mulr(f, f));
        s.e = e;
        s.lim = ldx(T(1), e);  // inf for the top exponent: never reached again
        s.inv = inv;
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const T t = mulr(a[k], s.inv);
        s.ssq = fma(t, t, s.ssq);
    }
}

template <typename T>
__device__ __forceinline__ Nrm<T> nrm_merge(Nrm<T> a, Nrm<T> b) {
    const bool ah = a.e >= b.e;
    const Nrm<T>& hi = ah ? a : b;
    const Nrm<T>& lo = ah ? b : a;
    Nrm<T> r = hi;
    r.ssq = addr(hi.ssq, ldx(lo.ssq, 2 * (lo.e - hi.e)));  // exact scaling, or 0
    r.ninf = a.ninf + b.ninf;
    return r;
}

template <typename T>
__device__ __forceinline__ T nrm_finish(const Nrm<T>& s) {
    if (s.ninf > 1 || isnan(s.ssq)) return T(NAN);
    if (s.ninf == 1) return T(INFINITY);
    return ldx(sqrt(s.ssq), s.e);  // an empty state: 2^kEmpty underflows to 0
}

// Reduction ops: Acc, zero, merge, one element (pointers at it) and K
// consecutive scalars. RED: L1_DOT, L1_ASUM, L1_NRM2 (real, or complex as
// its components re, im in order), L1_DOTU, L1_DOTC.
template <typename T, bool CX, int RED> struct Rop;

template <typename T, bool CX> struct Rop<T, CX, L1_DOT> {
    using Acc = T;
    static constexpr bool uses_y = true;
    static __device__ Acc zero() { return T(0); }
    static __device__ Acc merge(Acc a, Acc b) { return addr(a, b); }
    static __device__ void elem(Acc& a, const T* x, const T* y) { a = fma(__ldg(x), __ldg(y), a); }
    template <int K>
    static __device__ void vec(Acc& a, const T (&xs)[K], const T (&ys)[K]) {
#pragma unroll
        for (int k = 0; k < K; ++k) a = fma(xs[k], ys[k], a);
    }
};
template <typename T, bool CX> struct Rop<T, CX, L1_ASUM> {
    using Acc = T;
    static constexpr bool uses_y = false;
    static __device__ Acc zero() { return T(0); }
    static __device__ Acc merge(Acc a, Acc b) { return addr(a, b); }
    static __device__ void elem(Acc& a, const T* x, const T*) { a = addr(a, fabs(__ldg(x))); }
    template <int K>
    static __device__ void vec(Acc& a, const T (&xs)[K], const T (&)[K]) {
#pragma unroll
        for (int k = 0; k < K; ++k) a = addr(a, fabs(xs[k]));
    }
};
template <typename T, bool CX> struct Rop<T, CX, L1_NRM2> {
    using Acc = Nrm<T>;
    static constexpr bool uses_y = false;
    static __device__ Acc zero() { return nrm_zero<T>(); }
    static __device__ Acc merge(Acc a, Acc b) { return nrm_merge(a, b); }
    static __device__ void elem(Acc& a, const T* x, const T*) {
        if constexpr (CX) {
            const T v[2] = {__ldg(x), __ldg(x + 1)};  // both components (src/complex1.rs:96)
            nrm_chunk<T, 2>(a, v);
        } else {
            const T v[1] = {__ldg(x)};
            nrm_chunk<T, 1>(a, v);
        }
    }
    template <int K>
    static __device__ void vec(Acc& a, const T (&xs)[K], const T (&)[K]) {
        nrm_chunk<T, K>(a, xs);
    }
};
template <typename T, bool CONJ> struct ZDotOp {
    using Acc = Z<T>;
    static constexpr bool uses_y = true;
    static __device__ Acc zero() { return {T(0), T(0)}; }
    static __device__ Acc merge(Acc a, Acc b) { return zadd(a, b); }
    static __device__ Z<T> xv(T re, T im) { return {re, CONJ ? subr(T(0), im) : im}; }
    static __device__ void elem(Acc& a, const T* x, const T* y) {  // src/complex1.rs:42 / 62
        a = zadd(a, zmul(xv(__ldg(x), __ldg(x + 1)), Z<T>{__ldg(y), __ldg(y + 1)}));
    }
    template <int K>
    static __device__ void vec(Acc& a, const T (&xs)[K], const T (&ys)[K]) {
#pragma unroll
        for (int k = 0; k < K; k += 2) a = zadd(a, zmul(xv(xs[k], xs[k + 1]), Z<T>{ys[k], ys[k + 1]}));
    }
};
template <typename T> struct Rop<T, true, L1_DOTU> : ZDotOp<T, false> {};
template <typename T> struct Rop<T, true, L1_DOTC> : ZDotOp<T, true> {};

template <typename R, typename Acc>
__device__ Acc block_fold(Acc a) {
    __shared__ Acc part[kL1Threads];
    part[threadIdx.x] = a;
    __syncthreads();
#pragma unroll
    for (int w = kL1Threads / 2; w > 0; w >>= 1) {  // a fixed tree
        if (threadIdx.x < w) part[threadIdx.x] = R::merge(part[threadIdx.x], part[threadIdx.x + w]);
        __syncthreads();
    }
    return part[0];
}

template <typename T, bool CX, int RED>
__global__ void __launch_bounds__(kL1Threads, kL1BlocksPerSm)
    reduce_partial_kernel(size_t n, const T* __restrict__ x, size_t incx, const T* __restrict__ y, size_t incy,
                          int contig, typename Rop<T, CX, RED>::Acc* part) {
    using R = Rop<T, CX, RED>;
    constexpr int K = kVec<T>;
    constexpr int E = CX ? 2 : 1;
    const size_t nth = static_cast<size_t>(gridDim.x) * kL1Threads;
    const size_t tid = static_cast<size_t>(blockIdx.x) * kL1Threads + threadIdx.x;
    typename R::Acc a = R::zero();
    size_t first_scalar_elem = 0;
    if (contig) {
        const size_t nv = n * E / K;
        size_t v = tid;
        for (; v + (kUnroll - 1) * nth < nv; v += kUnroll * nth) {
            T xs[kUnroll][K], ys[kUnroll][K];
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) {
                ld16nc(x + (v + u * nth) * K, xs[u]);
                if constexpr (R::uses_y) ld16nc(y + (v + u * nth) * K, ys[u]);
            }
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) R::template vec<K>(a, xs[u], ys[u]);
        }
#pragma unroll 1
        for (; v < nv; v += nth) {
            T xs[K], ys[K];
            ld16nc(x + v * K, xs);
            if constexpr (R::uses_y) ld16nc(y + v * K, ys);
            R::template vec<K>(a, xs, ys);
        }
        first_scalar_elem = nv * K / E;
        incx = incy = 1;
    }
#pragma unroll 1
    for (size_t i = first_scalar_elem + tid; i < n; i += nth)
        R::elem(a, x + i * incx * E, R::uses_y ? y + i * incy * E : nullptr);
    const typename R::Acc b = block_fold<R>(a);
    if (threadIdx.x == 0) part[blockIdx.x] = b;
}

template <typename T, bool CX, int RED>
__global__ void __launch_bounds__(kL1Threads)
    reduce_final_kernel(int nparts, const typename Rop<T, CX, RED>::Acc* part, T* out) {
    using R = Rop<T, CX, RED>;
    typename R::Acc a = R::zero();
    for (int i = threadIdx.x; i < nparts; i += kL1Threads) a = R::merge(a, part[i]);
    const typename R::Acc b = block_fold<R>(a);
    if (threadIdx.x == 0) {
        if constexpr (RED == L1_NRM2) {
            out[0] = nrm_finish(b);
        } else if constexpr (RED == L1_DOTU || RED == L1_DOTC) {
            out[0] = b.re;
            out[1] = b.im;
        } else {
            out[0] = b;
        }
    }
}

// Blocks for `units` work units (a 16-byte vector when contiguous, else an
// element): one unit per thread, at most kL1MaxBlocks.
int l1_blocks(size_t units) {
    const size_t b = (units + kL1Threads - 1) / kL1Threads;
    return static_cast<int>(std::max<size_t>(1, std::min<size_t>(b, kL1MaxBlocks)));
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int cuda_rc(cudaError_t e, int32_t* ce) {
    if (e == cudaSuccess) return RB_OK;
    if (ce) *ce = static_cast<int32_t>(e);
    return RB_ERR_CUDA;
}

template <typename T, bool CX, int RED>
int reduce_dev(size_t n, const T* x, size_t incx, const T* y, size_t incy, T* out, cudaStream_t st, int32_t* ce) {
    using Acc = typename Rop<T, CX, RED>::Acc;
    constexpr int E = CX ? 2 : 1;
    const bool contig = incx == 1 && aligned16(x) && (!Rop<T, CX, RED>::uses_y || (incy == 1 && aligned16(y)));
    const int nb = l1_blocks(contig ? (n * E + kVec<T> - 1) / kVec<T> : n);
    Acc* part = nullptr;
    cudaError_t e = scratch_alloc(&part, static_cast<size_t>(nb) * sizeof(Acc), st);
    if (e != cudaSuccess) return cuda_rc(e, ce);
    reduce_partial_kernel<T, CX, RED><<<nb, kL1Threads, 0, st>>>(n, x, incx, y, incy, contig ? 1 : 0, part);
    reduce_final_kernel<T, CX, RED><<<1, kL1Threads, 0, st>>>(nb, part, out);
    count_launch(2);
    e = cudaGetLastError();
    cudaFreeAsync(part, st);
    return cuda_rc(e, ce);
}

template <typename T, bool CX, int OP>
int elementwise_dev(size_t n, Z<T> al, T* x, size_t incx, T* y, size_t incy, cudaStream_t st, int32_t* ce) {
    constexpr int E = CX ? 2 : 1;
    const bool contig = incy == 1 && aligned16(y) && (OP == L1_SCAL || (incx == 1 && aligned16(x)));
    if (contig) {
        // vectors per block: swap moves four streams, so it keeps more in flight
        constexpr int U = OP == L1_SWAP ? 8 : 2;
        const size_t nv = n * E / kVec<T>;
        const size_t nb = std::max<size_t>(1, (nv + U * kL1Threads - 1) / (U * kL1Threads));
        if (nb > 0x7fffffffu) return RB_ERR_INVALID_ARG;
        ew_tile_kernel<T, CX, OP, U><<<static_cast<unsigned>(nb), kL1Threads, 0, st>>>(n, al, x, y);
    } else {
        ew_strided_kernel<T, CX, OP><<<l1_blocks(n), kL1Threads, 0, st>>>(n, al, x, incx, y, incy);
    }
    count_launch();
    return cuda_rc(cudaGetLastError(), ce);
}

}  // namespace

template <typename T, bool CX>
int l1_dev(int op, size_t n, T ar, T ai, const T* x, size_t incx, T* y, size_t incy, T* out, cudaStream_t st,
           int32_t* ce) {
    const Z<T> al{ar, ai};
    T* xm = const_cast<T*>(x);
    if (op >= L1_DOT) {
        if (n == 0) {
            const size_t cnt = (op == L1_DOTU || op == L1_DOTC) ? 2 : 1;
            return cuda_rc(cudaMemsetAsync(out, 0, cnt * sizeof(T), st), ce);
        }
        if constexpr (CX) {
            if (op == L1_DOTU) return reduce_dev<T, true, L1_DOTU>(n, x, incx, y, incy, out, st, ce);
            if (op == L1_DOTC) return reduce_dev<T, true, L1_DOTC>(n, x, incx, y, incy, out, st, ce);
            if (op == L1_NRM2) return reduce_dev<T, true, L1_NRM2>(n, x, incx, nullptr, 0, out, st, ce);
        } else {
            if (op == L1_DOT) return reduce_dev<T, false, L1_DOT>(n, x, incx, y, incy, out, st, ce);
            if (op == L1_ASUM) return reduce_dev<T, false, L1_ASUM>(n, x, incx, nullptr, 0, out, st, ce);
            if (op == L1_NRM2) return reduce_dev<T, false, L1_NRM2>(n, x, incx, nullptr, 0, out, st, ce);
        }
        return RB_ERR_INVALID_ARG;
    }
    if (n == 0) return RB_OK;
    switch (op) {
        case L1_AXPY: return elementwise_dev<T, CX, L1_AXPY>(n, al, xm, incx, y, incy, st, ce);
        case L1_SCAL: return elementwise_dev<T, CX, L1_SCAL>(n, al, nullptr, 0, y, incy, st, ce);
        case L1_COPY:
            // rblas's loop with incy == 0 leaves the last element in y[0]
            if (incy == 0 && n > 1) {
                xm += (n - 1) * incx * (CX ? 2 : 1);
                n = 1;
            }
            return elementwise_dev<T, CX, L1_COPY>(n, al, xm, incx, y, incy, st, ce);
        case L1_SWAP: return elementwise_dev<T, CX, L1_SWAP>(n, al, xm, incx, y, incy, st, ce);
        default: return RB_ERR_INVALID_ARG;
    }
}

template int l1_dev<float, false>(int, size_t, float, float, const float*, size_t, float*, size_t, float*,
                                  cudaStream_t, int32_t*);
template int l1_dev<double, false>(int, size_t, double, double, const double*, size_t, double*, size_t, double*,
                                   cudaStream_t, int32_t*);
template int l1_dev<float, true>(int, size_t, float, float, const float*, size_t, float*, size_t, float*,
                                 cudaStream_t, int32_t*);
template int l1_dev<double, true>(int, size_t, double, double, const double*, size_t, double*, size_t, double*,
                                  cudaStream_t, int32_t*);

// rblas's argument rules per routine, in its order: the early returns first
// (n == 0; real axpy with alpha == 0, real scal with alpha == 1), then the
// stride assertions (src/level1.rs:31, 53, 78, 100; src/complex1.rs:19, 75,
// 90) as ZeroStride, then the slice bounds as BufferTooSmall (have_len: the
// host entry points, which know the slices' lengths). copy, asum, dotu and
// dotc accept zero strides as rblas does; swap refuses a zero stride with
// n > 1 (rblas's loop then rotates elements one at a time, which has no
// parallel form). *noop: the call writes nothing (reductions return 0).
rb_status l1_check(int op, bool cx, size_t n, bool alpha_zero, bool alpha_one, size_t incx, size_t x_len,
                   size_t incy, size_t y_len, bool have_len, bool* noop, rb_error* err) {
    if (err) *err = rb_error{0, 0, 0, 0, 0};
    *noop = false;
    const bool uses_y = op == L1_AXPY || op == L1_COPY || op == L1_SWAP || op == L1_DOT || op == L1_DOTU ||
                        op == L1_DOTC;
    bool zero_ok = false;
    switch (op) {
        case L1_AXPY:
        case L1_DOT:
        case L1_SCAL:
        case L1_NRM2: break;
        case L1_ASUM:
        case L1_COPY:
        case L1_DOTU:
        case L1_DOTC: zero_ok = true; break;
        case L1_SWAP: zero_ok = n == 1; break;
        default:
            if (err) err->code = RB_ERR_INVALID_ARG;
            return RB_ERR_INVALID_ARG;
    }
    if (n == 0 || (op == L1_AXPY && alpha_zero) || (op == L1_SCAL && !cx && alpha_one)) {
        *noop = true;
        return RB_OK;
    }
    if (incx == 0 && !zero_ok) {
        if (err) *err = rb_error{RB_ERR_ZERO_STRIDE, 'x', 0, 0, 0};
        return RB_ERR_ZERO_STRIDE;
    }
    if (uses_y && incy == 0 && !zero_ok) {
        if (err) *err = rb_error{RB_ERR_ZERO_STRIDE, 'y', 0, 0, 0};
        return RB_ERR_ZERO_STRIDE;
    }
    if (have_len) {
        const size_t need_x = (n - 1) * incx + 1;
        if (x_len < need_x) {
            if (err) *err = rb_error{RB_ERR_BUFFER_TOO_SMALL, 'x', x_len, need_x, 0};
            return RB_ERR_BUFFER_TOO_SMALL;
        }
        const size_t need_y = (n - 1) * incy + 1;
        if (uses_y && y_len < need_y) {
            if (err) *err = rb_error{RB_ERR_BUFFER_TOO_SMALL, 'y', y_len, need_y, 0};
            return RB_ERR_BUFFER_TOO_SMALL;
        }
    }
    return RB_OK;
}

}  // namespace rb

using namespace rb;

namespace {

template <typename T, bool CX>
rb_status l1_dev_c(int op, size_t n, T ar, T ai, const T* x, size_t incx, T* y, size_t incy, T* out, void* stream,
                   rb_error* err) {
    bool noop = false;
    const rb_status v = l1_check(op, CX, n, ar == T(0) && ai == T(0), ar == T(1) && ai == T(0), incx, 0, incy, 0,
                                 false, &noop, err);
    if (v != RB_OK) return v;
    const bool red = op >= L1_DOT;
    if (red && !out) {
        if (err) err->code = RB_ERR_INVALID_ARG;
        return RB_ERR_INVALID_ARG;
    }
    if (noop && !red) return RB_OK;
    int32_t ce = 0;
    const int rc = l1_dev<T, CX>(op, n, ar, ai, x, incx, y, incy, out, static_cast<cudaStream_t>(stream), &ce);
    if (rc != RB_OK && err) {
        err->code = rc;
        err->cuda_error = ce;
    }
    return static_cast<rb_status>(rc);
}

}  // namespace

extern "C" {

// Real (src/level1.rs). scal's vector travels as y inside the library.
#define RB_L1_REAL_DEV(P, T)                                                                                        \
    rb_status rb_##P##axpy_dev(size_t n, T alpha, const T* x, size_t incx, T* y, size_t incy, void* stream,         \
                               rb_error* err) {                                                                     \
        return l1_dev_c<T, false>(L1_AXPY, n, alpha, T(0), x, incx, y, incy, nullptr, stream, err);                 \
    }                                                                                                               \
    rb_status rb_##P##scal_dev(size_t n, T alpha, T* x, size_t incx, void* stream, rb_error* err) {                 \
        return l1_dev_c<T, false>(L1_SCAL, n, alpha, T(0), nullptr, incx, x, incx, nullptr, stream, err);           \
    }                                                                                                               \
    rb_status rb_##P##copy_dev(size_t n, const T* x, size_t incx, T* y, size_t incy, void* stream, rb_error* err) { \
        return l1_dev_c<T, false>(L1_COPY, n, T(0), T(0), x, incx, y, incy, nullptr, stream, err);                  \
    }                                                                                                               \
    rb_status rb_##P##swap_dev(size_t n, T* x, size_t incx, T* y, size_t incy, void* stream, rb_error* err) {       \
        return l1_dev_c<T, false>(L1_SWAP, n, T(0), T(0), x, incx, y, incy, nullptr, stream, err);                  \
    }                                                                                                               \
    rb_status rb_##P##dot_dev(size_t n, const T* x, size_t incx, const T* y, size_t incy, T* result, void* stream,  \
                              rb_error* err) {                                                                      \
        return l1_dev_c<T, false>(L1_DOT, n, T(0), T(0), x, incx, const_cast<T*>(y), incy, result, stream, err);    \
    }                                                                                                               \
    rb_status rb_##P##asum_dev(size_t n, const T* x, size_t incx, T* result, void* stream, rb_error* err) {         \
        return l1_dev_c<T, false>(L1_ASUM, n, T(0), T(0), x, incx, nullptr, 0, result, stream, err);                \
    }                                                                                                               \
    rb_status rb_##P##nrm2_dev(size_t n, const T* x, size_t incx, T* result, void* stream, rb_error* err) {         \
        return l1_dev_c<T, false>(L1_NRM2, n, T(0), T(0), x, incx, nullptr, 0, result, stream, err);                \
    }
RB_L1_REAL_DEV(s, float)
RB_L1_REAL_DEV(d, double)
#undef RB_L1_REAL_DEV

// Complex (src/complex1.rs); dotu / dotc write {re, im}.
#define RB_L1_CPLX_DEV(P, N, T, CT)                                                                                 \
    rb_status rb_##P##axpy_dev(size_t n, CT alpha, const CT* x, size_t incx, CT* y, size_t incy, void* stream,      \
                               rb_error* err) {                                                                     \
        return l1_dev_c<T, true>(L1_AXPY, n, alpha.re, alpha.im, reinterpret_cast<const T*>(x), incx,               \
                                 reinterpret_cast<T*>(y), incy, nullptr, stream, err);                              \
    }                                                                                                               \
    rb_status rb_##P##scal_dev(size_t n, CT alpha, CT* x, size_t incx, void* stream, rb_error* err) {               \
        return l1_dev_c<T, true>(L1_SCAL, n, alpha.re, alpha.im, nullptr, incx, reinterpret_cast<T*>(x), incx,      \
                                 nullptr, stream, err);                                                             \
    }                                                                                                               \
    rb_status rb_##P##dotu_dev(size_t n, const CT* x, size_t incx, const CT* y, size_t incy, CT* result,            \
                               void* stream, rb_error* err) {                                                       \
        return l1_dev_c<T, true>(L1_DOTU, n, T(0), T(0), reinterpret_cast<const T*>(x), incx,                       \
                                 reinterpret_cast<T*>(const_cast<CT*>(y)), incy, reinterpret_cast<T*>(result),      \
                                 stream, err);                                                                      \
    }                                                                                                               \
    rb_status rb_##P##dotc_dev(size_t n, const CT* x, size_t incx, const CT* y, size_t incy, CT* result,            \
                               void* stream, rb_error* err) {                                                       \
        return l1_dev_c<T, true>(L1_DOTC, n, T(0), T(0), reinterpret_cast<const T*>(x), incx,                       \
                                 reinterpret_cast<T*>(const_cast<CT*>(y)), incy, reinterpret_cast<T*>(result),      \
                                 stream, err);                                                                      \
    }                                                                                                               \
    rb_status rb_##N##nrm2_dev(size_t n, const CT* x, size_t incx, T* result, void* stream, rb_error* err) {        \
        return l1_dev_c<T, true>(L1_NRM2, n, T(0), T(0), reinterpret_cast<const T*>(x), incx, nullptr, 0, result,   \
                                 stream, err);                                                                      \
    }
RB_L1_CPLX_DEV(c, sc, float, rb_complex32)
RB_L1_CPLX_DEV(z, dz, double, rb_complex64)
#undef RB_L1_CPLX_DEV

}  // extern "C"
