// trsm_batched.cu -- batched triangular solve, one launch for the batch.
//
// rblas's trsm (src/level3.rs:390-520) solves op(A) X = alpha*B (Left) or
// X op(A) = alpha*B (Right) for one problem by substitution. For a batch of
// same-shaped problems (uniform strides between the A_i and between the
// B_i) each problem is small -- the C4 case is 512 x 512 lower with 64
// right-hand sides, 16.8 Mflop -- so the single-problem path's blocked
// algorithm (a diagonal-block launch plus a GEMM launch per 64-row block)
// would pay ~15 launches per problem. Here every CTA owns RB right-hand
// sides of one problem: it keeps its q x RB slice of alpha*B in shared
// memory and runs a right-looking blocked forward substitution on it
// entirely on chip:
//   for each 64-row block: substitution inside the block, staged in shared
//   memory (each warp solves its own columns, rows in order, with a division
//   by the diagonal unless Unit), then
//   the trailing rows -= A[trailing, block] * X[block] as a register-tiled
//   SIMT GEMM (4 rows x RB/8 columns per thread) over 128-row panels of A
//   staged in shared memory.
// Right side is the transposed problem (B read through swapped strides);
// an upper-triangular op(A) is solved as a lower one with rows and columns
// reversed. Work per problem: q^2 * nrhs flop (q = order of A).
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/rblas_b200.h"
#include "rb_device.cuh"
#include "rb_internal.h"
#include "simt_tile.cuh"

namespace rb {

namespace {

constexpr int kTbNB = 64;      // diagonal block
constexpr int kTbPanel = 128;  // trailing rows per staged A panel
constexpr int kTbThreads = 256;

struct TbParams {
    int q, nrhs;
    int rev;    // solve the reversed (upper -> lower) system (B rows reversed)
    int unit;   // unit diagonal
    // op'(A)[r][c] (reversed when rev) at A_i + a_off + r*a_dr + c*a_dc
    long long a_off, a_dr, a_dc;
    size_t stride_a, ldb_rs, ldb_cs, stride_b;  // B element (i, j) of the solve at i*rs + j*cs
    // f64 tensor-core path: rows of op'(A) are unit stride and every even row
    // starts on 16 bytes (a_dr == 1, no offset, even lda and stride_a,
    // aligned base), so two adjacent rows load as one double2
    int vec_a;
};

template <typename T>
__device__ __forceinline__ const T* a_ptr(const T* __restrict__ A, const TbParams& p, int r, int c) {
    return A + (p.a_off + static_cast<long long>(r) * p.a_dr + static_cast<long long>(c) * p.a_dc);
}

// Asynchronous element copies global -> shared (cp.async, 4 or 8 bytes), so
// a thread's copies are all in flight at once instead of one load latency
// each; cp_wait() completes this thread's copies (a barrier must follow).
template <typename T>
__device__ __forceinline__ void cp_elem(T* dst, const T* src) {
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
// N consecutive elements from 16-byte-aligned shared memory in 16-byte loads.
template <typename T, int N>
__device__ __forceinline__ void ld_vec(const T* src, T (&v)[N]) {
    if constexpr (sizeof(T) == 8 && N % 2 == 0) {
#pragma unroll
        for (int i = 0; i < N; i += 2) {
            const double2 x = *reinterpret_cast<const double2*>(src + i);
            v[i] = x.x;
            v[i + 1] = x.y;
        }
    } else if constexpr (sizeof(T) == 4 && N % 4 == 0) {
#pragma unroll
        for (int i = 0; i < N; i += 4) {
            const float4 x = *reinterpret_cast<const float4*>(src + i);
            v[i] = x.x;
            v[i + 1] = x.y;
            v[i + 2] = x.z;
            v[i + 3] = x.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) v[i] = src[i];
    }
}

__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

template <typename T, int RB>
__global__ void __launch_bounds__(kTbThreads)
    trsm_batched_kernel(const T* __restrict__ A0, T* __restrict__ B0, T alpha, TbParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // Y: [q][YS], rows padded by one element so that a warp reading one
    // column down 32 rows touches distinct banks
    constexpr int YS = RB + 1;
    T* Y = reinterpret_cast<T*>(smem_raw);
    // P: [kTbNB][kTbPanel], 16-byte aligned for the vector loads (q*YS may be odd)
    T* P = Y + ((static_cast<size_t>(p.q) * YS + 3) & ~static_cast<size_t>(3));
    const int tid = threadIdx.x;
    const T* A = A0 + static_cast<size_t>(blockIdx.y) * p.stride_a;
    T* B = B0 + static_cast<size_t>(blockIdx.y) * p.stride_b;
    const int c0 = blockIdx.x * RB;
    const int ncols = min(RB, p.nrhs - c0);
    const int q = p.q;

    // Y = alpha * B slice (rows reversed when rev); consecutive threads walk
    // the unit-stride direction of B
    const bool rows_fast = p.ldb_rs == 1;
    for (int idx = tid; idx < q * RB; idx += kTbThreads) {
        const int i = rows_fast ? idx % q : idx / RB;
        const int j = rows_fast ? idx / q : idx % RB;
        T* dst = Y + (p.rev ? q - 1 - i : i) * YS + j;
        if (j < ncols) cp_elem(dst, B + (static_cast<size_t>(i) * p.ldb_rs + static_cast<size_t>(c0 + j) * p.ldb_cs));
        else *dst = T(0);
    }
    cp_wait();
    __syncthreads();
    if (alpha != T(1))  // B := alpha*B first (src/level3.rs:403-409)
        for (int idx = tid; idx < q * RB; idx += kTbThreads) Y[(idx / RB) * YS + idx % RB] *= alpha;
    __syncthreads();

    const int tr = (tid / 8) * 4;  // panel rows of this thread (32 groups of 4)
    const int tc = tid % 8;        // columns tc, tc+8, ... (RB/8 of them)
    constexpr int CW = RB / 8;
    for (int o = 0; o < q; o += kTbNB) {
        const int nb = min(kTbNB, q - o);
        // substitution inside the diagonal block, staged in shared memory
        // transposed (Dt[c][r] = op'(A)[o+r][o+c], r >= c). Each warp solves
        // RB/8 columns on its own, lane l holding rows l and l+32 of them:
        // at step t the lane owning row t divides it by the diagonal (unless
        // Unit), broadcasts it, and every lane folds it into its later rows.
        T* Dt = P;
        for (int idx = tid; idx < nb * nb; idx += kTbThreads) {
            const int r = idx % nb, c = idx / nb;
            if (r >= c) cp_elem(Dt + c * kTbNB + r, a_ptr(A, p, o + r, o + c));
        }
        cp_wait();
        __syncthreads();
        {
            constexpr int CWD = RB / 8;  // columns per warp
            const int warp = tid >> 5, lane = tid & 31;
            const int col0 = warp * CWD;
            T y0[CWD], y1[CWD];
#pragma unroll
            for (int c = 0; c < CWD; ++c) {
                y0[c] = (lane < nb) ? Y[(o + lane) * YS + col0 + c] : T(0);
                y1[c] = (lane + 32 < nb) ? Y[(o + lane + 32) * YS + col0 + c] : T(0);
            }
            for (int t = 0; t < nb; ++t) {
                const int owner = t & 31;
                const bool hi = t >= 32;  // warp-uniform
                T xt[CWD];
#pragma unroll
                for (int c = 0; c < CWD; ++c) xt[c] = __shfl_sync(0xffffffffu, hi ? y1[c] : y0[c], owner);
                if (!p.unit) {
                    // lane c divides column c's value, then broadcasts it
                    const T d = Dt[t * kTbNB + t];
                    T mine = xt[0];
#pragma unroll
                    for (int c = 1; c < CWD; ++c)
                        if (lane == c) mine = xt[c];
                    if (lane < CWD) mine = mine / d;
#pragma unroll
                    for (int c = 0; c < CWD; ++c) xt[c] = __shfl_sync(0xffffffffu, mine, c);
                    if (lane == owner) {
#pragma unroll
                        for (int c = 0; c < CWD; ++c) {
                            if (hi) y1[c] = xt[c];
                            else y0[c] = xt[c];
                        }
                    }
                }
                const T d0 = Dt[t * kTbNB + lane], d1 = Dt[t * kTbNB + lane + 32];
#pragma unroll
                for (int c = 0; c < CWD; ++c) {
                    if (lane > t) y0[c] = y0[c] - d0 * xt[c];
                    if (lane + 32 > t) y1[c] = y1[c] - d1 * xt[c];
                }
            }
#pragma unroll
            for (int c = 0; c < CWD; ++c) {
                if (lane < nb) Y[(o + lane) * YS + col0 + c] = y0[c];
                if (lane + 32 < nb) Y[(o + lane + 32) * YS + col0 + c] = y1[c];
            }
        }
        __syncthreads();
        // trailing update over 128-row panels
        for (int r0 = o + nb; r0 < q; r0 += kTbPanel) {
            const int pr = min(kTbPanel, q - r0);
            for (int idx = tid; idx < nb * kTbPanel; idx += kTbThreads) {
                const int r = idx % kTbPanel, s = idx / kTbPanel;
                if (r < pr) cp_elem(P + s * kTbPanel + r, a_ptr(A, p, r0 + r, o + s));
                else P[s * kTbPanel + r] = T(0);
            }
            cp_wait();
            __syncthreads();
            T acc[4][CW];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < CW; ++j) acc[i][j] = T(0);
#pragma unroll 4
            for (int s = 0; s < nb; ++s) {
                T a[4], y[CW];
                ld_vec<T, 4>(P + s * kTbPanel + tr, a);
#pragma unroll
                for (int j = 0; j < CW; ++j) y[j] = Y[(o + s) * YS + tc + 8 * j];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < CW; ++j) acc[i][j] = fma(a[i], y[j], acc[i][j]);
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (tr + i < pr)
#pragma unroll
                    for (int j = 0; j < CW; ++j) Y[(r0 + tr + i) * YS + tc + 8 * j] -= acc[i][j];
            __syncthreads();
        }
    }

    for (int idx = tid; idx < q * RB; idx += kTbThreads) {
        const int i = rows_fast ? idx % q : idx / RB;
        const int j = rows_fast ? idx / q : idx % RB;
        if (j < ncols)
            B[static_cast<size_t>(i) * p.ldb_rs + static_cast<size_t>(c0 + j) * p.ldb_cs] =
                Y[(p.rev ? q - 1 - i : i) * YS + j];
    }
}

template <typename T, int RB>
size_t tb_smem(int q) {
    return (((static_cast<size_t>(q) * (RB + 1) + 3) & ~static_cast<size_t>(3)) +
            static_cast<size_t>(kTbNB) * kTbPanel) * sizeof(T);
}

template <typename T, int RB>
cudaError_t tb_launch(const T* A, T* B, T alpha, const TbParams& p, size_t batch, cudaStream_t st) {
    const size_t smem = tb_smem<T, RB>(p.q);
    cudaError_t e = cudaFuncSetAttribute(trsm_batched_kernel<T, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    const dim3 grid((p.nrhs + RB - 1) / RB, static_cast<unsigned>(batch));
    KernelTimer tmr;
    kernel_timing_begin(sizeof(T) == 8 ? "trsm_batched_d" : "trsm_batched_s",
                        static_cast<double>(p.q) * p.q * p.nrhs * static_cast<double>(batch), st, &tmr);
    trsm_batched_kernel<T, RB><<<grid, kTbThreads, smem, st>>>(A, B, alpha, p);
    kernel_timing_end(&tmr, st);
    count_launch();
    return cudaGetLastError();
}

constexpr size_t kTbSmemMax = 227 * 1024;

// ---- f64 on the FP64 tensor cores ------------------------------------------------
//
// The substitution above runs 64 dependent steps (shuffle, divide, fold) per
// diagonal block on one CTA per SM; at the C4 shape it kept the FP64 pipe 17 %
// busy. The f64 path instead turns every step into a GEMM on DMMA
// (mma.sync m16n8k8 f64), blocked like the substitution:
//   1. trsm_inv_diag_kernel inverts every 64 x 64 diagonal block of every
//      member once, W_b = inv(L_bb), into a workspace, by recursive doubling:
//      the four 16 x 16 diagonal blocks by forward substitution, then
//      inv([[A, 0], [C, D]]) = [[inv A, 0], [-inv D * C * inv A, inv D]]
//      twice (16 -> 32 -> 64) with the products on DMMA (Unit takes the
//      diagonal as 1);
//   2. trsm_dmma_kernel keeps the member's q x RB slice Y = alpha*B in shared
//      memory and for each block b computes X_b = W_b * Y_b, then
//      Y_trailing -= L[trailing, b] * X_b. Both products read A and W as
//      DMMA fragments straight from global memory (L2: each member's A is
//      shared by its nrhs/RB CTAs) and Y from shared memory.
// Rounding differs from rblas's substitution (src/level3.rs:440-512: the
// blocks' inverses replace the divisions inside each block); the result
// stays within the normwise backward-error bound the tests state.
constexpr int kInvNB = 64;

// Column-major 64 x 64 f64 tiles in shared memory with columns padded to
// 68 doubles: the global loads of A's columns, the stores of W and the DMMA
// fragment reads below (a half-warp on rows g, k-columns t, or k-rows t,
// columns g, g and t < 4) then touch distinct banks.
constexpr int kInvLD = 68;
constexpr int kInvThreads = 128;
// L block and W (its inverse); the temporaries live in L's upper triangle,
// which is zero and never read (three CTAs per SM)
constexpr int kInvSmem = 2 * kInvNB * kInvLD * static_cast<int>(sizeof(double));

// C(16 x 16) += A(16 x K) * B(K x 16), A and B column-major in shared memory
// with column stride kInvLD; c[nb] holds columns 8 nb .. 8 nb + 7 in the DMMA
// accumulator layout (simt_tile.cuh, dmma_16x8x8).
template <int K>
__device__ __forceinline__ void inv_mm16(const double* As, const double* Bs, double (&c)[2][4], int g, int t) {
#pragma unroll
    for (int kk = 0; kk < K / 8; ++kk) {
        const int k = 8 * kk + t;
        const double a[4] = {As[k * kInvLD + g], As[k * kInvLD + g + 8], As[(k + 4) * kInvLD + g],
                             As[(k + 4) * kInvLD + g + 8]};
#pragma unroll
        for (int nb = 0; nb < 2; ++nb) {
            const double b[2] = {Bs[(8 * nb + g) * kInvLD + k], Bs[(8 * nb + g) * kInvLD + k + 4]};
            dmma_16x8x8(c[nb], a, b);
        }
    }
}

// D(16 x 16) = s * c, D column-major in shared memory with column stride kInvLD
__device__ __forceinline__ void inv_store16(double* Ds, const double (&c)[2][4], double s, int g, int t) {
#pragma unroll
    for (int nb = 0; nb < 2; ++nb) {
        const int col = 8 * nb + 2 * t;
        Ds[col * kInvLD + g] = s * c[nb][0];
        Ds[(col + 1) * kInvLD + g] = s * c[nb][1];
        Ds[col * kInvLD + g + 8] = s * c[nb][2];
        Ds[(col + 1) * kInvLD + g + 8] = s * c[nb][3];
    }
}

__global__ void __launch_bounds__(kInvThreads) trsm_inv_diag_kernel(const double* __restrict__ A0, TbParams p,
                                                                     double* __restrict__ W, int nblocks) {
    extern __shared__ __align__(16) unsigned char inv_smem[];
    // element (r, c) of a tile at [c * kInvLD + r]
    double* Ls = reinterpret_cast<double*>(inv_smem);  // L block (lower part read)
    double* Ws = Ls + kInvNB * kInvLD;                  // its inverse
    const int b = blockIdx.x, member = blockIdx.y;
    const double* A = A0 + static_cast<size_t>(member) * p.stride_a;
    const int o = b * kInvNB, nb = min(kInvNB, p.q - o);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;

    // L (lower part of the block; Unit puts 1 on the diagonal; rows and
    // columns past nb are the identity), W zero. Thread tid & 63 loads row r
    // of columns c = tid >> 6, +2, ...: 32 loads in flight.
    {
        const int r = tid & 63, c0 = tid >> 6;
        double v[kInvNB / 2];
#pragma unroll
        for (int i = 0; i < kInvNB / 2; ++i) {
            const int c = c0 + 2 * i;
            const bool in = r < nb && (c < r || (c == r && !p.unit));
            v[i] = in ? __ldg(a_ptr(A, p, o + r, o + c)) : (c == r ? 1.0 : 0.0);
        }
#pragma unroll
        for (int i = 0; i < kInvNB / 2; ++i) {
            Ls[(c0 + 2 * i) * kInvLD + r] = v[i];
            Ws[(c0 + 2 * i) * kInvLD + r] = 0.0;
        }
    }
    __syncthreads();
    // the four 16 x 16 diagonal blocks: thread (blk, c) solves column c of
    // block blk by forward substitution, the column held in registers
    if (tid < 64) {
        const int blk = tid >> 4, c = tid & 15, d = 16 * blk;
        double w[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            double acc[2] = {0.0, 0.0};
#pragma unroll
            for (int s = 0; s < r; ++s) acc[s & 1] = fma(Ls[(d + s) * kInvLD + d + r], w[s], acc[s & 1]);
            const double v = ((r == c) ? 1.0 : 0.0) - (acc[0] + acc[1]);
            w[r] = (r < c) ? 0.0 : v / Ls[(d + r) * kInvLD + d + r];
        }
#pragma unroll
        for (int r = 0; r < 16; ++r) Ws[(d + c) * kInvLD + d + r] = w[r];
    }
    __syncthreads();
    // 16 -> 32: warp h (0, 1) forms W[hi][lo] of the 32 x 32 diagonal block h
    // (lo, hi = its 16-row halves): T = L[hi][lo] * W[lo][lo], then
    // W[hi][lo] = -W[hi][hi] * T
    if (warp < 2) {
        const int lo = 32 * warp, hi = lo + 16;
        double* Tw = Ls + hi * kInvLD + lo;  // L[lo][hi]: upper, unused
        double c[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
        inv_mm16<16>(Ls + lo * kInvLD + hi, Ws + lo * kInvLD + lo, c, g, t);
        inv_store16(Tw, c, 1.0, g, t);
        __syncwarp();
        double e[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
        inv_mm16<16>(Ws + hi * kInvLD + hi, Tw, e, g, t);
        inv_store16(Ws + lo * kInvLD + hi, e, -1.0, g, t);
    }
    __syncthreads();
    // 32 -> 64: T = L[32:64][0:32] * W[0:32][0:32], then
    // W[32:64][0:32] = -W[32:64][32:64] * T; warp w takes the 16 x 16 tile
    // (mi, ni) = (w >> 1, w & 1) of each product
    {
        const int mi = warp >> 1, ni = warp & 1;
        double c[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
        double* Ts = Ls + 32 * kInvLD;  // L[0:32][32:64]: upper, unused
        inv_mm16<32>(Ls + 32 + 16 * mi, Ws + 16 * ni * kInvLD, c, g, t);
        inv_store16(Ts + 16 * ni * kInvLD + 16 * mi, c, 1.0, g, t);
        __syncthreads();
        double e[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
        inv_mm16<32>(Ws + 32 * kInvLD + 32 + 16 * mi, Ts + 16 * ni * kInvLD, e, g, t);
        inv_store16(Ws + 16 * ni * kInvLD + 32 + 16 * mi, e, -1.0, g, t);
    }
    __syncthreads();
    // W_b column-major, zero outside the block's nb x nb (coalesced stores)
    double* Wb = W + (static_cast<size_t>(member) * nblocks + b) * (kInvNB * kInvNB);
    for (int idx = tid; idx < kInvNB * kInvNB; idx += kInvThreads) {
        const int r = idx % kInvNB, c = idx / kInvNB;
        Wb[idx] = (r < nb && c < nb) ? Ws[c * kInvLD + r] : 0.0;
    }
}

// Y rows padded so that a DMMA B-fragment read (lanes 4g + t reading rows t
// and t+4, columns g) hits distinct banks: (2 * YS) % 32 must be 8 or 24.
template <int RB> struct TdCfg;
template <> struct TdCfg<16> { static constexpr int YS = 20; };
template <> struct TdCfg<8> { static constexpr int YS = 12; };

template <int RB>
__global__ void __launch_bounds__(kTbThreads, 2)
    trsm_dmma_kernel(const double* __restrict__ A0, double* __restrict__ B0, double alpha, TbParams p,
                     const double* __restrict__ W, int nblocks) {
    constexpr int YS = TdCfg<RB>::YS;
    constexpr int NBLK = RB / 8;  // DMMA n-blocks across the slice
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* Y = reinterpret_cast<double*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    const int member = blockIdx.y;
    const double* A = A0 + static_cast<size_t>(member) * p.stride_a;
    double* B = B0 + static_cast<size_t>(member) * p.stride_b;
    const double* Wm = W + static_cast<size_t>(member) * nblocks * (kInvNB * kInvNB);
    const int c0 = blockIdx.x * RB;
    const int ncols = min(RB, p.nrhs - c0);
    const int q = p.q;

    // Y = alpha * B slice (rows reversed when rev), one rounding per element
    // as rblas's B := alpha*B (src/level3.rs:403-409)
    // (eight loads in flight per thread before their stores)
    const bool rows_fast = p.ldb_rs == 1;
    constexpr int kYU = 8;
    for (int base = tid; base < q * RB; base += kTbThreads * kYU) {
        double v[kYU];
#pragma unroll
        for (int u = 0; u < kYU; ++u) {
            const int idx = base + u * kTbThreads;
            const int i = rows_fast ? idx % q : idx / RB;
            const int j = rows_fast ? idx / q : idx % RB;
            v[u] = (idx < q * RB && j < ncols)
                       ? B[static_cast<size_t>(i) * p.ldb_rs + static_cast<size_t>(c0 + j) * p.ldb_cs]
                       : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kYU; ++u) {
            const int idx = base + u * kTbThreads;
            if (idx < q * RB) {
                const int i = rows_fast ? idx % q : idx / RB;
                const int j = rows_fast ? idx / q : idx % RB;
                Y[(p.rev ? q - 1 - i : i) * YS + j] = (j < ncols && alpha != 1.0) ? alpha * v[u] : v[u];
            }
        }
    }
    __syncthreads();

    // Each warp walks a fixed sequence of 16 x 64 fragment tiles -- for every
    // block b, W_b's rows 16 xm.. (the X step, warps with an (xm, xn) pair)
    // and then A's rows r0 = o + nb + 16 warp, +128, ... of block b's
    // columns (the trailing update) -- in halves of four k-steps. A half's
    // loads are issued while the DMMAs of the half before it run, across the
    // block's barriers too: A and W do not depend on Y.
    const bool xw = warp < 4 * NBLK;
    const int xm = warp % 4, xn = warp / 4;
    // DMMA fragment rows g and g+8 take the adjacent rows 2g and 2g+1 of
    // the 16-row block (the output rows follow), so each pair is one
    // 16-byte load; the fragment layout is in simt_tile.cuh (dmma_16x8x8)
    auto first_trail = [&](int b) { return b * kInvNB + min(kInvNB, q - b * kInvNB) + 16 * warp; };
    // the tile after (kind, b, r0): kind 0 W_b, 1 A rows r0 of block b, 2 none
    auto next_tile = [&](int& kind, int& b, int& r0) {
        const int r = kind == 0 ? first_trail(b) : r0 + 16 * 8;
        if (r < q) {
            kind = 1;
            r0 = r;
            return;
        }
        for (int bb = b + 1; bb < nblocks; ++bb) {
            if (xw) {
                kind = 0;
                b = bb;
                return;
            }
            if (first_trail(bb) < q) {
                kind = 1;
                b = bb;
                r0 = first_trail(bb);
                return;
            }
        }
        kind = 2;
    };
    // k-steps 4h .. 4h+3 of a tile into f (W is column-major 64 x 64, zero
    // outside the block; A rows past q read as zero)
    auto load_half = [&](int kind, int b, int r0, int h, double (&f)[4][4]) {
        if (kind == 0) {
            const double* Wb = Wm + static_cast<size_t>(b) * (kInvNB * kInvNB) + 16 * xm + 2 * g;
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const int k = 8 * (4 * h + kk) + t;
                const double2 lo = __ldg(reinterpret_cast<const double2*>(Wb + 64 * k));
                const double2 hi = __ldg(reinterpret_cast<const double2*>(Wb + 64 * (k + 4)));
                f[kk][0] = lo.x;
                f[kk][1] = lo.y;
                f[kk][2] = hi.x;
                f[kk][3] = hi.y;
            }
        } else if (kind == 1) {
            const int o = b * kInvNB, ra = r0 + 2 * g, rb = ra + 1;
            if (p.vec_a && r0 + 16 <= q) {
                // r0 is even (o + 64 + 16 i), so every pair starts on 16 bytes
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) {
                    const int k = o + 8 * (4 * h + kk) + t;
                    const double2 lo = __ldg(reinterpret_cast<const double2*>(a_ptr(A, p, ra, k)));
                    const double2 hi = __ldg(reinterpret_cast<const double2*>(a_ptr(A, p, ra, k + 4)));
                    f[kk][0] = lo.x;
                    f[kk][1] = lo.y;
                    f[kk][2] = hi.x;
                    f[kk][3] = hi.y;
                }
            } else {
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) {
                    const int k = o + 8 * (4 * h + kk) + t;
                    f[kk][0] = (ra < q) ? __ldg(a_ptr(A, p, ra, k)) : 0.0;
                    f[kk][1] = (rb < q) ? __ldg(a_ptr(A, p, rb, k)) : 0.0;
                    f[kk][2] = (ra < q) ? __ldg(a_ptr(A, p, ra, k + 4)) : 0.0;
                    f[kk][3] = (rb < q) ? __ldg(a_ptr(A, p, rb, k + 4)) : 0.0;
                }
            }
        }
    };
    int kind = 0, tb = 0, tr0 = 0;      // W_0, or for a warp without X work
    if (!xw) next_tile(kind, tb, tr0);  // its first trailing tile
    double fa[4][4], fb[4][4];  // the current tile's halves
    load_half(kind, tb, tr0, 0, fa);

    for (int b = 0; b < nblocks; ++b) {
        const int o = b * kInvNB, nb = min(kInvNB, q - o);
        // ---- X_b = W_b * Y_b: 4 m-blocks x NBLK n-blocks, one (m, n) pair per warp
        double xacc[4] = {0.0, 0.0, 0.0, 0.0};
        if (xw) {  // the current tile is W_b
            load_half(kind, tb, tr0, 1, fb);
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const int k = 8 * kk + t;
                double bf[2];
                bf[0] = (k < nb) ? Y[(o + k) * YS + 8 * xn + g] : 0.0;
                bf[1] = (k + 4 < nb) ? Y[(o + k + 4) * YS + 8 * xn + g] : 0.0;
                dmma_16x8x8(xacc, fa[kk], bf);
            }
            next_tile(kind, tb, tr0);
            load_half(kind, tb, tr0, 0, fa);
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const int k = 8 * (4 + kk) + t;
                double bf[2];
                bf[0] = (k < nb) ? Y[(o + k) * YS + 8 * xn + g] : 0.0;
                bf[1] = (k + 4 < nb) ? Y[(o + k + 4) * YS + 8 * xn + g] : 0.0;
                dmma_16x8x8(xacc, fb[kk], bf);
            }
        }
        __syncthreads();  // every read of Y_b is done
        if (xw) {
            const int r = 16 * xm + 2 * g, c = 8 * xn + 2 * t;
            if (r < nb) {
                Y[(o + r) * YS + c] = xacc[0];
                Y[(o + r) * YS + c + 1] = xacc[1];
            }
            if (r + 1 < nb) {
                Y[(o + r + 1) * YS + c] = xacc[2];
                Y[(o + r + 1) * YS + c + 1] = xacc[3];
            }
        }
        __syncthreads();
        // ---- trailing rows -= L[trailing, block] * X_b, 16-row m-blocks dealt to the warps
        for (int r0 = first_trail(b); r0 < q; r0 += 16 * 8) {  // the current tile is A rows r0
            const int ra = r0 + 2 * g, rb = ra + 1;
            load_half(kind, tb, tr0, 1, fb);
            double acc[NBLK][4];
#pragma unroll
            for (int n = 0; n < NBLK; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.0;
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const int k = o + 8 * kk + t;
#pragma unroll
                for (int n = 0; n < NBLK; ++n) {
                    double bf[2] = {Y[k * YS + 8 * n + g], Y[(k + 4) * YS + 8 * n + g]};
                    dmma_16x8x8(acc[n], fa[kk], bf);
                }
            }
            next_tile(kind, tb, tr0);
            load_half(kind, tb, tr0, 0, fa);
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const int k = o + 8 * (4 + kk) + t;
#pragma unroll
                for (int n = 0; n < NBLK; ++n) {
                    double bf[2] = {Y[k * YS + 8 * n + g], Y[(k + 4) * YS + 8 * n + g]};
                    dmma_16x8x8(acc[n], fb[kk], bf);
                }
            }
#pragma unroll
            for (int n = 0; n < NBLK; ++n) {
                const int c = 8 * n + 2 * t;
                if (ra < q) {
                    Y[ra * YS + c] -= acc[n][0];
                    Y[ra * YS + c + 1] -= acc[n][1];
                }
                if (rb < q) {
                    Y[rb * YS + c] -= acc[n][2];
                    Y[rb * YS + c + 1] -= acc[n][3];
                }
            }
        }
        __syncthreads();
    }

    for (int idx = tid; idx < q * RB; idx += kTbThreads) {
        const int i = rows_fast ? idx % q : idx / RB;
        const int j = rows_fast ? idx / q : idx % RB;
        if (j < ncols)
            B[static_cast<size_t>(i) * p.ldb_rs + static_cast<size_t>(c0 + j) * p.ldb_cs] =
                Y[(p.rev ? q - 1 - i : i) * YS + j];
    }
}

template <int RB>
size_t td_smem(int q) {
    return static_cast<size_t>(q) * TdCfg<RB>::YS * sizeof(double);
}

// Workspace of the diagonal-block inverses is bounded: members go in chunks.
constexpr size_t kTdWorkspace = size_t(256) << 20;

template <int RB>
cudaError_t td_launch(const double* A, double* B, double alpha, const TbParams& p, size_t batch, cudaStream_t st,
                      bool* alloc_failed) {
    const size_t smem = td_smem<RB>(p.q);
    cudaError_t e = cudaFuncSetAttribute(trsm_dmma_kernel<RB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(trsm_inv_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kInvSmem);
    if (e != cudaSuccess) return e;
    const int nblocks = (p.q + kInvNB - 1) / kInvNB;
    const size_t per_member = static_cast<size_t>(nblocks) * kInvNB * kInvNB * sizeof(double);
    const size_t chunk = std::max<size_t>(1, std::min(batch, kTdWorkspace / per_member));
    double* W = nullptr;
    e = scratch_alloc(&W, chunk * per_member, st);
    if (e != cudaSuccess) {
        *alloc_failed = e == cudaErrorMemoryAllocation;
        return e;
    }
    KernelTimer tmr;
    kernel_timing_begin("trsm_batched_d", static_cast<double>(p.q) * p.q * p.nrhs * static_cast<double>(batch), st,
                        &tmr);
    for (size_t b0 = 0; b0 < batch && e == cudaSuccess; b0 += chunk) {
        const size_t nm = std::min(chunk, batch - b0);
        const double* Ac = A + b0 * p.stride_a;
        double* Bc = B + b0 * p.stride_b;
        trsm_inv_diag_kernel<<<dim3(nblocks, static_cast<unsigned>(nm)), kInvThreads, kInvSmem, st>>>(Ac, p, W,
                                                                                              nblocks);
        trsm_dmma_kernel<RB><<<dim3((p.nrhs + RB - 1) / RB, static_cast<unsigned>(nm)), kTbThreads, smem, st>>>(
            Ac, Bc, alpha, p, W, nblocks);
        count_launch(2);
        e = cudaGetLastError();
    }
    kernel_timing_end(&tmr, st);
    cudaFreeAsync(W, st);
    return e;
}

}  // namespace

template <typename T>
int trsm_batched_dev(int side, int uplo, int trans, int diag, size_t m, size_t n, T alpha, const T* A, size_t lda,
                     size_t stride_a, T* B, size_t ldb, size_t stride_b, size_t batch, cudaStream_t st,
                     int32_t* ce, rb_error* err) {
    if ((side != RB_LEFT && side != RB_RIGHT) || (uplo != RB_UPPER && uplo != RB_LOWER) || trans < 0 || trans > 2 ||
        (diag != RB_NON_UNIT && diag != RB_UNIT))
        return RB_ERR_INVALID_ARG;
    const size_t q = (side == RB_LEFT) ? m : n, nrhs = (side == RB_LEFT) ? n : m;
    // leading dimensions (check_matrix for a q x q A and an m x n B, column-major)
    if (q > 0 && lda < q) {
        if (err) *err = rb_error{RB_ERR_INVALID_LEADING_DIM, 'a', lda, q, 0};
        return RB_ERR_INVALID_LEADING_DIM;
    }
    if (m > 0 && n > 0 && ldb < m) {
        if (err) *err = rb_error{RB_ERR_INVALID_LEADING_DIM, 'b', ldb, m, 0};
        return RB_ERR_INVALID_LEADING_DIM;
    }
    if (m == 0 || n == 0 || batch == 0) return RB_OK;
    if (q > 0x7fffffff || nrhs > 0x7fffffff) return RB_ERR_INVALID_ARG;
    if (batch > 65535) {  // grid.y limit: launch in chunks
        for (size_t b0 = 0; b0 < batch; b0 += 65535) {
            const int rc = trsm_batched_dev<T>(side, uplo, trans, diag, m, n, alpha, A + b0 * stride_a, lda, stride_a,
                                               B + b0 * stride_b, ldb, stride_b, std::min<size_t>(65535, batch - b0),
                                               st, ce, err);
            if (rc != RB_OK) return rc;
        }
        return RB_OK;
    }
    const bool tr = trans != RB_NO_TRANS;
    // solve op'(A) Y = alpha Z: Left op' = op, Right op' = op^T (Z = B^T)
    const bool eff_tr = (side == RB_LEFT) ? tr : !tr;
    const bool eff_upper = (uplo == RB_UPPER) != eff_tr;
    TbParams p{};
    p.q = static_cast<int>(q);
    p.nrhs = static_cast<int>(nrhs);
    p.rev = eff_upper;
    p.unit = diag == RB_UNIT;
    // op'(A)[r][c] = eff_tr ? A[c + r*lda] : A[r + c*lda]; reversed: r -> q-1-r, c -> q-1-c
    const long long ld = static_cast<long long>(lda), qm = static_cast<long long>(q) - 1;
    const long long sr = eff_tr ? ld : 1, sc = eff_tr ? 1 : ld;
    p.a_off = eff_upper ? qm * (sr + sc) : 0;
    p.a_dr = eff_upper ? -sr : sr;
    p.a_dc = eff_upper ? -sc : sc;
    p.stride_a = stride_a;
    p.ldb_rs = (side == RB_LEFT) ? 1 : ldb;
    p.ldb_cs = (side == RB_LEFT) ? ldb : 1;
    p.stride_b = stride_b;
    p.vec_a = (p.a_dr == 1 && p.a_off == 0 && lda % 2 == 0 && stride_a % 2 == 0 &&
               reinterpret_cast<uintptr_t>(A) % 16 == 0) ? 1 : 0;
    cudaError_t e = cudaSuccess;
    bool alloc_failed = false;
    int td_rb = 0;  // f64: slice width of the tensor-core path (0: not used)
    if constexpr (sizeof(T) == 8) {
        // 16-wide slices while two CTAs fit an SM, then 8-wide, then one CTA per SM
        if (td_smem<16>(p.q) <= kTbSmemMax / 2) td_rb = 16;
        else if (td_smem<8>(p.q) <= kTbSmemMax / 2) td_rb = 8;
        else if (td_smem<16>(p.q) <= kTbSmemMax) td_rb = 16;
        else if (td_smem<8>(p.q) <= kTbSmemMax) td_rb = 8;
        if (td_rb == 16) e = td_launch<16>(reinterpret_cast<const double*>(A), reinterpret_cast<double*>(B), alpha, p,
                                           batch, st, &alloc_failed);
        else if (td_rb == 8) e = td_launch<8>(reinterpret_cast<const double*>(A), reinterpret_cast<double*>(B), alpha,
                                              p, batch, st, &alloc_failed);
    }
    if (td_rb) {
        // launched above
    } else if (tb_smem<T, 32>(p.q) <= kTbSmemMax) e = tb_launch<T, 32>(A, B, alpha, p, batch, st);
    else if (tb_smem<T, 16>(p.q) <= kTbSmemMax) e = tb_launch<T, 16>(A, B, alpha, p, batch, st);
    else if (tb_smem<T, 8>(p.q) <= kTbSmemMax) e = tb_launch<T, 8>(A, B, alpha, p, batch, st);
    else {
        // too large for one CTA's shared memory: the single-problem path per member
        for (size_t i = 0; i < batch; ++i) {
            const int rc = trsm_dev<T, false>(side, uplo, trans, diag, m, n, alpha, T(0), A + i * stride_a, lda,
                                              B + i * stride_b, ldb, st, ce);
            if (rc != RB_OK) return rc;
        }
        return RB_OK;
    }
    if (e != cudaSuccess) {
        if (ce) *ce = static_cast<int32_t>(e);
        if (alloc_failed) cudaGetLastError();
        return alloc_failed ? RB_ERR_ALLOC : RB_ERR_CUDA;
    }
    return RB_OK;
}

template int trsm_batched_dev<float>(int, int, int, int, size_t, size_t, float, const float*, size_t, size_t, float*,
                                     size_t, size_t, size_t, cudaStream_t, int32_t*, rb_error*);
template int trsm_batched_dev<double>(int, int, int, int, size_t, size_t, double, const double*, size_t, size_t,
                                      double*, size_t, size_t, size_t, cudaStream_t, int32_t*, rb_error*);

}  // namespace rb

using namespace rb;

extern "C" {

rb_status rb_strsm_batched_dev(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n,
                               float alpha, const float* a, size_t lda, size_t stride_a, float* b, size_t ldb,
                               size_t stride_b, size_t batch, void* stream, rb_error* err) {
    if (err) *err = rb_error{0, 0, 0, 0, 0};
    int32_t ce = 0;
    const int rc = trsm_batched_dev<float>(side, uplo, trans, diag, m, n, alpha, a, lda, stride_a, b, ldb, stride_b,
                                           batch, static_cast<cudaStream_t>(stream), &ce, err);
    if (rc != RB_OK && err) {
        err->code = rc;
        err->cuda_error = ce;
    }
    return static_cast<rb_status>(rc);
}

rb_status rb_dtrsm_batched_dev(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n,
                               double alpha, const double* a, size_t lda, size_t stride_a, double* b, size_t ldb,
                               size_t stride_b, size_t batch, void* stream, rb_error* err) {
    if (err) *err = rb_error{0, 0, 0, 0, 0};
    int32_t ce = 0;
    const int rc = trsm_batched_dev<double>(side, uplo, trans, diag, m, n, alpha, a, lda, stride_a, b, ldb, stride_b,
                                            batch, static_cast<cudaStream_t>(stream), &ce, err);
    if (rc != RB_OK && err) {
        err->code = rc;
        err->cuda_error = ce;
    }
    return static_cast<rb_status>(rc);
}

}  // extern "C"
