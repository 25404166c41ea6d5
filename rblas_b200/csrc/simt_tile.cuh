// simt_tile.cuh -- the plain GEMM tile pipeline, shared by the single-problem
// kernel (gemm_simt.cu) and the grouped persistent kernel (gemm_grouped.cu):
// true-FP32 SGEMM on FFMA, FP64 DGEMM on the FP64 tensor cores (mma.sync
// m16n8k8 f64, DMMA).
//
// One C tile = BM x BN. 8 compute warps (2 along M x 4 along N) consume a
// STAGES-deep ring of shared-memory stages that one producer lane fills with
// TMA. f32: each lane an 8 x TN register tile of FFMA. f64: each warp a
// 64 x 16 tile of 4 x 2 DMMA blocks (16 x 8 each, 4 accumulators per lane;
// the same 32 values per lane as an 8 x 4 register tile). A K-major operand
// tile lands as [mn][k] 128-byte rows with the hardware 128-byte swizzle; an
// MN-major tile as [k][mn] rows, unswizzled. All read patterns are
// bank-conflict free.
// The ring's mbarrier phases run on a counter `it` that continues across
// tiles, so a persistent CTA streams tile after tile through one ring.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "rb_device.cuh"

namespace rb {

// Tile shape per element type; V = 1 is the narrow f32 tile.
template <typename T, int V = 0> struct SimtCfg;
// f32: 128x128 C tile, 8x8 per thread, BK = 32 (one 128-byte swizzle row).
template <> struct SimtCfg<float, 0> { static constexpr int BM = 128, BN = 128, BK = 32, TN = 8, STAGES = 4; };
// f32 narrow: 128x64 C tile, 8x4 per thread, for problems whose 128 x 128
// tiles leave SMs idle (twice the tiles; 96 KiB of stages, two CTAs per SM).
template <> struct SimtCfg<float, 1> { static constexpr int BM = 128, BN = 64, BK = 32, TN = 4, STAGES = 4; };
// f64: 128x64 C tile, 8x4 per thread, BK = 16 (one 128-byte swizzle row).
template <> struct SimtCfg<double, 0> { static constexpr int BM = 128, BN = 64, BK = 16, TN = 4, STAGES = 4; };

constexpr int kSimtComputeWarps = 8;
constexpr int kSimtThreads = (kSimtComputeWarps + 1) * 32;

template <typename T> struct Vec16;
template <> struct Vec16<float> { using type = float4; static constexpr int N = 4; };
template <> struct Vec16<double> { using type = double2; static constexpr int N = 2; };

template <typename T>
__device__ __forceinline__ void lds16(const uint8_t* p, T (&v)[Vec16<T>::N]) {
    const typename Vec16<T>::type x = *reinterpret_cast<const typename Vec16<T>::type*>(p);
    if constexpr (Vec16<T>::N == 4) {
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    } else {
        v[0] = x.x; v[1] = x.y;
    }
}

template <typename T, int V = 0>
constexpr int simt_smem_bytes() {
    using Cfg = SimtCfg<T, V>;
    return Cfg::STAGES * (Cfg::BM + Cfg::BN) * Cfg::BK * (int)sizeof(T) + 2 * Cfg::STAGES * 8 + 1024;
}

// An MN-major f64 A tile lands as BM/16 boxes of 16 m x BK k, each [k][16 m]
// with the 128-byte swizzle (2 KiB apiece), so that the DMMA fragment reads
// below are bank-conflict free; every other MN-major tile is one unswizzled
// [k][mn] box. Box rows (mn) of the A tensor map and its swizzle, by element size.
__host__ __device__ constexpr uint32_t simt_mn_a_box(size_t elem) { return elem == 8 ? 16u : 128u; }
__host__ __device__ constexpr bool simt_mn_a_swizzled(size_t elem) { return elem == 8; }

// Byte offsets of the A and B tiles inside a stage.
template <typename T, int V = 0>
__host__ __device__ constexpr int simt_a_bytes() { return SimtCfg<T, V>::BM * SimtCfg<T, V>::BK * (int)sizeof(T); }
template <typename T, int V = 0>
__host__ __device__ constexpr int simt_stage_bytes() {
    return (SimtCfg<T, V>::BM + SimtCfg<T, V>::BN) * SimtCfg<T, V>::BK * (int)sizeof(T);
}

// Producer lane: issue the num_kt K-tile loads (starting at K-tile kt0) of
// the tile at (m0, n0) on ring iterations it, it+1, ... Returns false (after
// letting its own copies land) if a wait gave up.
template <typename T, bool A_K, bool B_K, int V = 0>
__device__ __forceinline__ bool simt_produce(const CUtensorMap* tmA, const CUtensorMap* tmB, int m0, int n0,
                                             int kt0, int num_kt, uint8_t* smem, int stage_stride, uint64_t* full,
                                             uint64_t* empty, uint32_t& it, uint32_t* err) {
    using Cfg = SimtCfg<T, V>;
    constexpr int ST = Cfg::STAGES, BK = Cfg::BK;
    constexpr int A_BYTES = simt_a_bytes<T, V>();
    constexpr uint32_t TX = simt_stage_bytes<T, V>();
    for (int kt = 0; kt < num_kt; ++kt, ++it) {
        const int s = it % ST;
        if (it >= ST && !mbar_wait(&empty[s], ((it / ST) - 1) & 1, err, 0x101)) {
            const uint32_t first = it > (uint32_t)ST ? it - ST : 0;
            for (uint32_t j = first; j < it; ++j) mbar_wait_drain(&full[j % ST], (j / ST) & 1);
            return false;
        }
        uint8_t* sa = smem + s * stage_stride;
        uint8_t* sb = sa + A_BYTES;
        mbar_arrive_expect_tx(&full[s], TX);
        const int k0 = (kt0 + kt) * BK;
        if constexpr (A_K) {
            tma_load_2d(sa, tmA, &full[s], k0, m0);
        } else if constexpr (simt_mn_a_swizzled(sizeof(T))) {
#pragma unroll
            for (int c = 0; c < Cfg::BM / 16; ++c) tma_load_2d(sa + c * 2048, tmA, &full[s], m0 + 16 * c, k0);
        } else {
            tma_load_2d(sa, tmA, &full[s], m0, k0);
        }
        if (B_K) tma_load_2d(sb, tmB, &full[s], k0, n0);
        else     tma_load_2d(sb, tmB, &full[s], n0, k0);
    }
    return true;
}

// Epilogue data of one tile: C = alpha*acc + beta*Cin, written to c (cin
// may equal c).
template <typename T>
struct SimtOut {
    T* c;
    size_t ldc;
    const T* cin;
    size_t ldcin;
    int m, n;
    T alpha, beta;
    int beta_mode;  // 0: beta == 0 (C not read), 1: beta == 1, 2: general
    int tri;        // 0 full C; 1 upper triangle only (row <= col); 2 lower (row >= col)
};

// ---- f64 on the tensor cores (DMMA) -------------------------------------------
// mma.sync m16n8k8 f64, lane = 4g + t:
//   a = {A[g][t], A[g+8][t], A[g][t+4], A[g+8][t+4]}   (16 x 8, row-major)
//   b = {B[t][g], B[t+4][g]}                             (8 x 8, col-major)
//   c = {C[g][2t], C[g][2t+1], C[g+8][2t], C[g+8][2t+1]} (16 x 8)
__device__ __forceinline__ void dmma_16x8x8(double (&c)[4], const double (&a)[4], const double (&b)[2]) {
    asm("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}
__device__ __forceinline__ double lds64(const uint8_t* p) { return *reinterpret_cast<const double*>(p); }
__device__ __forceinline__ double2 lds128d(const uint8_t* p) { return *reinterpret_cast<const double2*>(p); }
// byte offset of element k of row `row` in a 128-byte-swizzled [row][16 doubles] tile
__device__ __forceinline__ int swz64(int row, int k) { return row * 128 + ((((k >> 1) ^ (row & 7))) << 4) + ((k & 1) << 3); }

// Which C element DMMA accumulator q of block (mb, nb) holds, in the warp's
// 64 x 16 tile. K-major operands keep the fragment's natural rows / columns.
// An MN-major operand is read 16 bytes at a time: fragment rows g and g+8 of
// an A block are the adjacent rows 2g, 2g+1, and fragment column j of B
// block nb is column 2j + nb, so each lane's load brings both values.
// With an MN-major A the fragment's k slots t and t+4 also take the physical
// k rows 2t and 2t+1 (for A and B alike; the k order of a sum of exact
// products changes nothing): a quarter-warp's A reads then fall on 8
// distinct swizzle chunks of the [k][16 m] boxes, one wavefront.
template <bool A_K>
__device__ __forceinline__ int dmma_row(int mb, int q, int g) {
    const int hi = q >> 1;  // q = 2, 3: fragment row g + 8
    return mb * 16 + (A_K ? g + 8 * hi : 2 * g + hi);
}
template <bool B_K>
__device__ __forceinline__ int dmma_col(int nb, int q, int t) {
    const int j = 2 * t + (q & 1);
    return B_K ? nb * 8 + j : 2 * j + nb;
}

template <bool A_K, bool B_K>
__device__ __forceinline__ bool dmma_mainloop(double (&acc)[8][4], int num_kt, const uint8_t* smem, int stage_stride,
                                              uint64_t* full, uint64_t* empty, uint32_t& it, uint32_t* err,
                                              int warp, int lane) {
    using Cfg = SimtCfg<double>;
    constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK, ST = Cfg::STAGES;
    constexpr int A_BYTES = simt_a_bytes<double>();
    static_assert(BK == 16 && BM == 128 && BN == 64, "the DMMA tile assumes 128 x 64 x 16");
    const int wm0 = (warp & 1) * 64, wn0 = (warp >> 1) * 16;
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[i][q] = 0.0;

    for (int kt = 0; kt < num_kt; ++kt, ++it) {
        const int s = it % ST;
        if (!mbar_wait(&full[s], (it / ST) & 1, err, 0x102)) return false;
        const uint8_t* sa = smem + s * stage_stride;
        const uint8_t* sb = sa + A_BYTES;
#pragma unroll
        for (int ks = 0; ks < BK; ks += 8) {
            double a[4][4], b[2][2];
#pragma unroll
            for (int mb = 0; mb < 4; ++mb) {
                if constexpr (A_K) {
                    const int row = wm0 + mb * 16 + g;  // row & 7 == g: the 8 rows' chunks differ
                    a[mb][0] = lds64(sa + swz64(row, ks + t));
                    a[mb][1] = lds64(sa + swz64(row + 8, ks + t));
                    a[mb][2] = lds64(sa + swz64(row, ks + t + 4));
                    a[mb][3] = lds64(sa + swz64(row + 8, ks + t + 4));
                } else {
                    // box (wm0 + 16 mb) / 16, rows k = ks + 2t, ks + 2t + 1, chunk g (m = 2g, 2g + 1)
                    const uint8_t* box = sa + ((wm0 >> 4) + mb) * 2048;
                    const int k0r = ks + 2 * t, k1r = k0r + 1;
                    const double2 v0 = lds128d(box + k0r * 128 + ((g ^ (k0r & 7)) << 4));
                    const double2 v1 = lds128d(box + k1r * 128 + ((g ^ (k1r & 7)) << 4));
                    a[mb][0] = v0.x; a[mb][1] = v0.y; a[mb][2] = v1.x; a[mb][3] = v1.y;
                }
            }
            // B follows A's k slots: t, t+4 (K-major A) or 2t, 2t+1 (MN-major A)
            if constexpr (B_K) {
#pragma unroll
                for (int nb = 0; nb < 2; ++nb) {
                    const int row = wn0 + nb * 8 + g;
                    if constexpr (A_K) {
                        b[nb][0] = lds64(sb + swz64(row, ks + t));
                        b[nb][1] = lds64(sb + swz64(row, ks + t + 4));
                    } else {
                        const double2 v = lds128d(sb + swz64(row, ks + 2 * t));  // k = ks+2t, ks+2t+1
                        b[nb][0] = v.x;
                        b[nb][1] = v.y;
                    }
                }
            } else {
                const int n = wn0 + 2 * g;
                const int k0r = A_K ? ks + t : ks + 2 * t, k1r = A_K ? ks + t + 4 : ks + 2 * t + 1;
                const double2 v0 = lds128d(sb + (k0r * BN + n) * 8);
                const double2 v1 = lds128d(sb + (k1r * BN + n) * 8);
                b[0][0] = v0.x; b[1][0] = v0.y; b[0][1] = v1.x; b[1][1] = v1.y;
            }
#pragma unroll
            for (int mb = 0; mb < 4; ++mb)
#pragma unroll
                for (int nb = 0; nb < 2; ++nb) dmma_16x8x8(acc[mb * 2 + nb], a[mb], b[nb]);
        }
        // every lane's shared-memory reads of the stage are ordered before
        // the warp's release (lane 0's arrive orders only its own accesses,
        // and __syncwarp alone did not keep in-flight reads ahead of the
        // producer's next TMA write into the stage)
        __threadfence_block();
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
    return true;
}

// Compute warps: consume num_kt stages from ring iteration it into the
// thread's 8 x TN accumulator. Returns false if a wait gave up.
template <typename T, bool A_K, bool B_K, int V = 0>
__device__ __forceinline__ bool simt_mainloop(T (&acc)[8][SimtCfg<T, V>::TN], int num_kt, const uint8_t* smem,
                                              int stage_stride, uint64_t* full, uint64_t* empty, uint32_t& it,
                                              uint32_t* err, int warp, int lane) {
    if constexpr (sizeof(T) == 8) {
        return dmma_mainloop<A_K, B_K>(acc, num_kt, smem, stage_stride, full, empty, it, err, warp, lane);
    }
    using Cfg = SimtCfg<T, V>;
    constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK, TN = Cfg::TN, ST = Cfg::STAGES;
    constexpr int VEC = Vec16<T>::N;  // elements per 16-byte load
    constexpr int A_BYTES = simt_a_bytes<T, V>();
    static_assert(BK * sizeof(T) == 128, "a K-major tile row must be one 128-byte swizzle row");
    static_assert(A_BYTES % 1024 == 0, "swizzled tiles need 1 KiB alignment");
    const int wm = warp & 1, wn = warp >> 1;          // 2 x 4 warps
    const int lane_m = lane & 7, lane_n = lane >> 3;  // 8 x 4 lanes
    const int wm0 = wm * 64, wn0 = wn * (4 * TN);

#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = T(0);

    for (int kt = 0; kt < num_kt; ++kt, ++it) {
        const int s = it % ST;
        if (!mbar_wait(&full[s], (it / ST) & 1, err, 0x102)) return false;
        const uint8_t* sa = smem + s * stage_stride;
        const uint8_t* sb = sa + A_BYTES;
#pragma unroll
        for (int kk = 0; kk < BK; kk += VEC) {
            T a[VEC][8];
            T b[VEC][TN];
            const int chunk = kk / VEC;  // 16-byte chunk along k within a 128-byte row
            if constexpr (A_K) {
                // [m][k] swizzled: a quarter-warp (same lane_n, lane_m 0..7)
                // touches 8 rows whose swizzled chunks chunk^lane_m differ.
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    const int row = wm0 + lane_m + 8 * r;
                    T v[VEC];
                    lds16<T>(sa + row * 128 + ((chunk ^ (row & 7)) << 4), v);
#pragma unroll
                    for (int q = 0; q < VEC; ++q) a[q][r] = v[q];
                }
            } else {
                // [k][m]: a quarter-warp reads 8 consecutive 16-byte chunks of one row.
#pragma unroll
                for (int q = 0; q < VEC; ++q)
#pragma unroll
                    for (int g = 0; g < 8 / VEC; ++g) {
                        const int col = wm0 + g * 8 * VEC + lane_m * VEC;
                        T v[VEC];
                        lds16<T>(sa + ((kk + q) * BM + col) * sizeof(T), v);
#pragma unroll
                        for (int e = 0; e < VEC; ++e) a[q][g * VEC + e] = v[e];
                    }
            }
            if constexpr (B_K) {
                // [n][k] swizzled: a quarter-warp shares lane_n -> one address (broadcast).
#pragma unroll
                for (int j = 0; j < TN; ++j) {
                    const int row = wn0 + lane_n * TN + j;
                    T v[VEC];
                    lds16<T>(sb + row * 128 + ((chunk ^ (row & 7)) << 4), v);
#pragma unroll
                    for (int q = 0; q < VEC; ++q) b[q][j] = v[q];
                }
            } else {
#pragma unroll
                for (int q = 0; q < VEC; ++q)
#pragma unroll
                    for (int g = 0; g < TN / VEC; ++g) {
                        const int col = wn0 + g * 4 * VEC + lane_n * VEC;
                        T v[VEC];
                        lds16<T>(sb + ((kk + q) * BN + col) * sizeof(T), v);
#pragma unroll
                        for (int e = 0; e < VEC; ++e) b[q][g * VEC + e] = v[e];
                    }
            }
#pragma unroll
            for (int q = 0; q < VEC; ++q)
#pragma unroll
                for (int i = 0; i < 8; ++i)
#pragma unroll
                    for (int j = 0; j < TN; ++j) acc[i][j] = fma(a[q][i], b[q][j], acc[i][j]);
        }
        // every lane's shared-memory reads of the stage are ordered before
        // the warp's release (lane 0's arrive orders only its own accesses,
        // and __syncwarp alone did not keep in-flight reads ahead of the
        // producer's next TMA write into the stage)
        __threadfence_block();
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
    return true;
}

// Compute warps: C = alpha*acc + beta*Cin for the tile at (m0, n0).
template <typename T, bool A_K, bool B_K, int V = 0>
__device__ __forceinline__ void simt_epilogue(const SimtOut<T>& o, const T (&acc)[8][SimtCfg<T, V>::TN], int m0,
                                              int n0, int warp, int lane) {
    constexpr int TN = SimtCfg<T, V>::TN;
    constexpr int VEC = Vec16<T>::N;
    const int wm = warp & 1, wn = warp >> 1;
    if constexpr (sizeof(T) == 8) {
        // DMMA accumulators: acc[mb * 2 + nb][q], placed by dmma_row / dmma_col
        const int g = lane >> 2, tq = lane & 3;
        const int wm0 = wm * 64, wn0 = wn * 16;
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = m0 + wm0 + dmma_row<A_K>(i >> 1, q, g);
                const int cidx = n0 + wn0 + dmma_col<B_K>(i & 1, q, tq);
                if (r >= o.m || cidx >= o.n) continue;
                if ((o.tri == 1 && r > cidx) || (o.tri == 2 && r < cidx)) continue;
                T* cp = o.c + r + static_cast<size_t>(cidx) * o.ldc;
                T tv = T(0);
                if (o.beta_mode != 0) {
                    const T cv = o.cin[r + static_cast<size_t>(cidx) * o.ldcin];
                    tv = (o.beta_mode == 1) ? cv : o.beta * cv;
                }
                *cp = fma(o.alpha, acc[i][q], tv);
            }
        return;
    }
    const int lane_m = lane & 7, lane_n = lane >> 3;
    const int wm0 = wm * 64, wn0 = wn * (4 * TN);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int r = m0 + (A_K ? (wm0 + lane_m + 8 * i)
                                : (wm0 + (i / VEC) * 8 * VEC + lane_m * VEC + (i % VEC)));
        if (r >= o.m) continue;
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int cidx = n0 + (B_K ? (wn0 + lane_n * TN + j)
                                       : (wn0 + (j / VEC) * 4 * VEC + lane_n * VEC + (j % VEC)));
            if (cidx >= o.n) continue;
            if ((o.tri == 1 && r > cidx) || (o.tri == 2 && r < cidx)) continue;
            T* cp = o.c + r + static_cast<size_t>(cidx) * o.ldc;
            T t = T(0);
            if (o.beta_mode != 0) {
                const T cv = o.cin[r + static_cast<size_t>(cidx) * o.ldcin];
                t = (o.beta_mode == 1) ? cv : o.beta * cv;
            }
            *cp = fma(o.alpha, acc[i][j], t);
        }
    }
}

// Mainloop then epilogue: one whole tile.
template <typename T, bool A_K, bool B_K, int V = 0>
__device__ __forceinline__ bool simt_consume(const SimtOut<T>& o, int m0, int n0, int num_kt, uint8_t* smem,
                                             int stage_stride, uint64_t* full, uint64_t* empty, uint32_t& it,
                                             uint32_t* err, int warp, int lane) {
    T acc[8][SimtCfg<T, V>::TN];
    if (!simt_mainloop<T, A_K, B_K, V>(acc, num_kt, smem, stage_stride, full, empty, it, err, warp, lane))
        return false;
    simt_epilogue<T, A_K, B_K, V>(o, acc, m0, n0, warp, lane);
    return true;
}

}  // namespace rb
