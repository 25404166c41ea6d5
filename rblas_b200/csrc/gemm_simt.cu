// gemm_simt.cu -- the plain GEMM forms: true-FP32 SGEMM and FP64 DGEMM on the
// CUDA cores (FFMA / DFMA), fed by TMA.
//
// Replaces rblas's CPU blocking driver, packing and microkernels
// (src/kernel/gemm.rs:185-429, src/kernel/gemm_avx2.rs:26-155). sm_100's
// tensor cores have no FP32xFP32 product and tcgen05 has no f64 kind, so the
// plain (drop-in) forms run here; the tensor-core forms live elsewhere.
//
// Structure (one CTA per C tile, 8 compute warps + 1 TMA producer warp):
//   producer lane 0: for each K tile, wait `empty[s]`, arm `full[s]` with the
//     stage's byte count and issue two cp.async.bulk.tensor loads (A, B).
//   compute warps: wait `full[s]`, run the register-tiled FMA loop over the
//     stage, arrive on `empty[s]`; after the last stage apply alpha/beta and
//     store C.
// Transposes are absorbed into the tensor maps: a K-major operand tile lands
// in shared memory as [mn][k] rows of 128 bytes with the hardware 128-byte
// swizzle; an MN-major tile lands as [k][mn] rows, unswizzled. Both read
// patterns below are bank-conflict free (see the per-layout notes).
#include <cuda.h>
#include <cuda_runtime.h>

#include "rb_device.cuh"
#include "rb_internal.h"

namespace rb {

template <typename T> struct SimtCfg;
// f32: 128x128 C tile, 8x8 per thread, BK = 32 (one 128-byte swizzle row).
template <> struct SimtCfg<float> { static constexpr int BM = 128, BN = 128, BK = 32, TN = 8, STAGES = 4; };
// f64: 128x64 C tile, 8x4 per thread, BK = 16 (one 128-byte swizzle row).
template <> struct SimtCfg<double> { static constexpr int BM = 128, BN = 64, BK = 16, TN = 4, STAGES = 4; };

constexpr int kSimtComputeWarps = 8;
constexpr int kSimtThreads = (kSimtComputeWarps + 1) * 32;

template <typename T>
struct SimtParams {
    int m, n, k;
    int tiles_m, tiles_n;
    T alpha, beta;
    int beta_mode;  // 0: beta == 0 (C not read), 1: beta == 1, 2: general
    int tri;        // 0 full C; 1 upper triangle only (row <= col); 2 lower (row >= col)
    T* c;
    size_t ldc;
    uint32_t* err;
};

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

template <typename T>
constexpr int simt_smem_bytes() {
    using Cfg = SimtCfg<T>;
    return Cfg::STAGES * (Cfg::BM + Cfg::BN) * Cfg::BK * (int)sizeof(T) + 2 * Cfg::STAGES * 8 + 1024;
}

template <typename T, bool A_K, bool B_K>
__global__ void __launch_bounds__(kSimtThreads, 1)
    simt_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                     const SimtParams<T> p) {
    using Cfg = SimtCfg<T>;
    constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK, TN = Cfg::TN, ST = Cfg::STAGES;
    constexpr int VEC = Vec16<T>::N;                 // elements per 16-byte load
    constexpr int A_BYTES = BM * BK * sizeof(T);
    constexpr int B_BYTES = BN * BK * sizeof(T);
    constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
    static_assert(BK * sizeof(T) == 128, "a K-major tile row must be one 128-byte swizzle row");
    static_assert(A_BYTES % 1024 == 0 && B_BYTES % 1024 == 0, "swizzled tiles need 1 KiB alignment");

    extern __shared__ uint8_t smem_raw[];
    // Align by offsetting the __shared__ array itself (not through an integer
    // cast) so every access below stays a shared-window load.
    uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + ST * STAGE_BYTES);
    uint64_t* empty = full + ST;

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    int tm, tn;
    raster_tile(blockIdx.x, p.tiles_m, p.tiles_n, tm, tn);
    const int m0 = tm * BM, n0 = tn * BN;
    const int num_kt = (p.k + BK - 1) / BK;
    // syrk: tiles wholly outside the referenced triangle do nothing
    if ((p.tri == 1 && m0 > n0 + BN - 1) || (p.tri == 2 && m0 + BM - 1 < n0)) return;

    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kSimtComputeWarps);
        }
        fence_barrier_init();
    }
    __syncthreads();

    if (warp == kSimtComputeWarps) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            prefetch_tmap(&tmA);
            prefetch_tmap(&tmB);
            int kt = 0;
            bool ok = true;
            for (; kt < num_kt; ++kt) {
                const int s = kt % ST;
                if (kt >= ST && !mbar_wait(&empty[s], ((kt / ST) - 1) & 1, p.err, 0x101)) {
                    ok = false;
                    break;
                }
                uint8_t* sa = smem + s * STAGE_BYTES;
                uint8_t* sb = sa + A_BYTES;
                mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
                const int k0 = kt * BK;
                if (A_K) tma_load_2d(sa, &tmA, &full[s], k0, m0);
                else     tma_load_2d(sa, &tmA, &full[s], m0, k0);
                if (B_K) tma_load_2d(sb, &tmB, &full[s], k0, n0);
                else     tma_load_2d(sb, &tmB, &full[s], n0, k0);
            }
            if (!ok) {
                // let this CTA's own copies land before it exits
                for (int j = (kt > ST ? kt - ST : 0); j < kt; ++j) mbar_wait_drain(&full[j % ST], (j / ST) & 1);
            }
        }
        return;
    }

    // ---------------- compute warps ----------------
    const int wm = warp & 1, wn = warp >> 1;         // 2 x 4 warps
    const int lane_m = lane & 7, lane_n = lane >> 3; // 8 x 4 lanes
    const int wm0 = wm * 64, wn0 = wn * (4 * TN);

    T acc[8][TN];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = T(0);

    bool ok = true;
    for (int kt = 0; kt < num_kt; ++kt) {
        const int s = kt % ST;
        if (!mbar_wait(&full[s], (kt / ST) & 1, p.err, 0x102)) {
            ok = false;
            break;
        }
        const uint8_t* sa = smem + s * STAGE_BYTES;
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
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
    if (!ok) return;

    // ---------------- epilogue: C = alpha*acc + beta*C ----------------
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int r = m0 + (A_K ? (wm0 + lane_m + 8 * i)
                                : (wm0 + (i / VEC) * 8 * VEC + lane_m * VEC + (i % VEC)));
        if (r >= p.m) continue;
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int cidx = n0 + (B_K ? (wn0 + lane_n * TN + j)
                                       : (wn0 + (j / VEC) * 4 * VEC + lane_n * VEC + (j % VEC)));
            if (cidx >= p.n) continue;
            if ((p.tri == 1 && r > cidx) || (p.tri == 2 && r < cidx)) continue;
            T* cp = p.c + r + static_cast<size_t>(cidx) * p.ldc;
            T t = T(0);
            if (p.beta_mode == 1) t = *cp;
            else if (p.beta_mode == 2) t = p.beta * *cp;
            *cp = fma(p.alpha, acc[i][j], t);
        }
    }
}

template <typename T>
__global__ void scale_c_kernel(int m, int n, T beta, T* c, size_t ldc, int tri) {
    const size_t total = static_cast<size_t>(m) * n;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t j = idx / m, i = idx - j * m;
        if ((tri == 1 && i > j) || (tri == 2 && i < j)) continue;
        T* cp = c + i + j * ldc;
        *cp = (beta == T(0)) ? T(0) : beta * *cp;
    }
}

template <typename T>
cudaError_t launch_scale_c(int m, int n, T beta, T* C, size_t ldc, cudaStream_t st, int tri) {
    if (beta == T(1) || m == 0 || n == 0) return cudaSuccess;
    const size_t total = static_cast<size_t>(m) * n;
    int blocks = static_cast<int>((total + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    scale_c_kernel<T><<<blocks, 256, 0, st>>>(m, n, beta, C, ldc, tri);
    count_launch();
    return cudaGetLastError();
}

template <typename T>
static CUtensorMapDataType tmap_dtype();
template <> CUtensorMapDataType tmap_dtype<float>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT32; }
template <> CUtensorMapDataType tmap_dtype<double>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT64; }

template <typename T, bool A_K, bool B_K>
static cudaError_t launch_variant(const CUtensorMap& ta, const CUtensorMap& tb, const SimtParams<T>& p,
                                  cudaStream_t st) {
    auto kern = simt_gemm_kernel<T, A_K, B_K>;
    constexpr int smem = simt_smem_bytes<T>();
    static bool attr_set = false;  // per instantiation; benign race (idempotent)
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    const int grid = p.tiles_m * p.tiles_n;
    KernelTimer tm;
    kernel_timing_begin(sizeof(T) == 4 ? "simt_sgemm" : "simt_dgemm", 2.0 * p.m * p.n * p.k, st, &tm);
    kern<<<grid, kSimtThreads, smem, st>>>(ta, tb, p);
    kernel_timing_end(&tm, st);
    count_launch();
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_simt_gemm(bool a_kmajor, bool b_kmajor, int m, int n, int k, T alpha,
                             const T* A, size_t lda, const T* B, size_t ldb, T beta, T* C,
                             size_t ldc, cudaStream_t st, CUresult* cu_err, int tri) {
    using Cfg = SimtCfg<T>;
    CUtensorMap ta, tb;
    CUresult r;
    // op(A) is m x k: K-major when stored k x m (Trans), else stored m x k.
    if (a_kmajor)
        r = make_tmap_2d(&ta, A, tmap_dtype<T>(), sizeof(T), k, m, lda, Cfg::BK, Cfg::BM, true);
    else
        r = make_tmap_2d(&ta, A, tmap_dtype<T>(), sizeof(T), m, k, lda, Cfg::BM, Cfg::BK, false);
    if (r != CUDA_SUCCESS) { if (cu_err) *cu_err = r; return cudaErrorInvalidValue; }
    // op(B) is k x n: K-major when stored k x n (NoTrans), else stored n x k.
    if (b_kmajor)
        r = make_tmap_2d(&tb, B, tmap_dtype<T>(), sizeof(T), k, n, ldb, Cfg::BK, Cfg::BN, true);
    else
        r = make_tmap_2d(&tb, B, tmap_dtype<T>(), sizeof(T), n, k, ldb, Cfg::BN, Cfg::BK, false);
    if (r != CUDA_SUCCESS) { if (cu_err) *cu_err = r; return cudaErrorInvalidValue; }

    SimtParams<T> p;
    p.m = m; p.n = n; p.k = k;
    p.tiles_m = (m + Cfg::BM - 1) / Cfg::BM;
    p.tiles_n = (n + Cfg::BN - 1) / Cfg::BN;
    p.alpha = alpha; p.beta = beta;
    p.beta_mode = (beta == T(0)) ? 0 : (beta == T(1) ? 1 : 2);
    p.tri = tri;
    p.c = C; p.ldc = ldc;
    p.err = device_error_word();
    if (!p.err) return cudaErrorMemoryAllocation;
    if (a_kmajor) {
        if (b_kmajor) return launch_variant<T, true, true>(ta, tb, p, st);
        return launch_variant<T, true, false>(ta, tb, p, st);
    }
    if (b_kmajor) return launch_variant<T, false, true>(ta, tb, p, st);
    return launch_variant<T, false, false>(ta, tb, p, st);
}

template cudaError_t launch_simt_gemm<float>(bool, bool, int, int, int, float, const float*, size_t,
                                             const float*, size_t, float, float*, size_t, cudaStream_t,
                                             CUresult*, int);
template cudaError_t launch_simt_gemm<double>(bool, bool, int, int, int, double, const double*, size_t,
                                              const double*, size_t, double, double*, size_t,
                                              cudaStream_t, CUresult*, int);
template cudaError_t launch_scale_c<float>(int, int, float, float*, size_t, cudaStream_t, int);
template cudaError_t launch_scale_c<double>(int, int, double, double*, size_t, cudaStream_t, int);

}  // namespace rb
