// gemm_simt.cu -- the plain GEMM forms, fed by TMA: true-FP32 SGEMM on the
// CUDA cores (FFMA) and FP64 DGEMM on the FP64 tensor cores (mma.sync f64;
// the tile code is in simt_tile.cuh).
//
// Replaces rblas's CPU blocking driver, packing and microkernels
// (src/kernel/gemm.rs:185-429, src/kernel/gemm_avx2.rs:26-155). sm_100's
// tcgen05 has no FP32xFP32 product and no f64 kind, so the plain (drop-in)
// forms run here; the tcgen05 precision forms live elsewhere.
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
#include "simt_tile.cuh"

namespace rb {

template <typename T>
struct SimtParams {
    int m, n, k;
    int tiles_m, tiles_n;
    T alpha, beta;
    int beta_mode;  // 0: beta == 0 (C not read), 1: beta == 1, 2: general
    int tri;        // 0 full C; 1 upper triangle only (row <= col); 2 lower (row >= col)
    T* c;
    size_t ldc;
    const T* cin;  // C0 read for beta != 0 (== c for the in-place update)
    size_t ldcin;
    uint32_t* err;
};

template <typename T, bool A_K, bool B_K, int V>
__global__ void __launch_bounds__(kSimtThreads, V == 1 ? 2 : 1)
    simt_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                     const SimtParams<T> p) {
    using Cfg = SimtCfg<T, V>;
    constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK, ST = Cfg::STAGES;
    constexpr int STAGE_BYTES = simt_stage_bytes<T, V>();

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

    uint32_t it = 0;
    if (warp == kSimtComputeWarps) {
        if (lane == 0) {
            prefetch_tmap(&tmA);
            prefetch_tmap(&tmB);
            simt_produce<T, A_K, B_K, V>(&tmA, &tmB, m0, n0, 0, num_kt, smem, STAGE_BYTES, full, empty, it,
                                         p.err);
        }
        return;
    }
    const SimtOut<T> o{p.c, p.ldc, p.cin, p.ldcin, p.m, p.n, p.alpha, p.beta, p.beta_mode, p.tri};
    simt_consume<T, A_K, B_K, V>(o, m0, n0, num_kt, smem, STAGE_BYTES, full, empty, it, p.err, warp, lane);
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

template <typename T, bool A_K, bool B_K, int V>
static cudaError_t launch_variant(const CUtensorMap& ta, const CUtensorMap& tb, const SimtParams<T>& p,
                                  cudaStream_t st) {
    auto kern = simt_gemm_kernel<T, A_K, B_K, V>;
    constexpr int smem = simt_smem_bytes<T, V>();
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

template <typename T, int V>
static cudaError_t launch_simt_tiles(bool a_kmajor, bool b_kmajor, int m, int n, int k, T alpha,
                                     const T* A, size_t lda, const T* B, size_t ldb, T beta, T* C,
                                     size_t ldc, cudaStream_t st, CUresult* cu_err, int tri, const T* Cin,
                                     size_t ldcin) {
    using Cfg = SimtCfg<T, V>;
    CUtensorMap ta, tb;
    CUresult r;
    // op(A) is m x k: K-major when stored k x m (Trans), else stored m x k.
    if (a_kmajor)
        r = make_tmap_2d(&ta, A, tmap_dtype<T>(), sizeof(T), k, m, lda, Cfg::BK, Cfg::BM, true);
    else
        r = make_tmap_2d(&ta, A, tmap_dtype<T>(), sizeof(T), m, k, lda, simt_mn_a_box(sizeof(T)), Cfg::BK,
                         simt_mn_a_swizzled(sizeof(T)));
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
    p.cin = Cin ? Cin : C;
    p.ldcin = Cin ? ldcin : ldc;
    p.err = device_error_word();
    if (!p.err) return cudaErrorMemoryAllocation;
    if (a_kmajor) {
        if (b_kmajor) return launch_variant<T, true, true, V>(ta, tb, p, st);
        return launch_variant<T, true, false, V>(ta, tb, p, st);
    }
    if (b_kmajor) return launch_variant<T, false, true, V>(ta, tb, p, st);
    return launch_variant<T, false, false, V>(ta, tb, p, st);
}

bool simt_narrow_f32(size_t m, size_t n) {
    static int sms = 0;  // benign race: every thread stores the same value
    if (!sms) {
        int dev = 0, v = 148;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0)
            sms = v;
        else
            return false;
    }
    const size_t tm = (m + 127) / 128;
    const size_t wide = tm * ((n + 127) / 128), narrow = tm * ((n + 63) / 64);
    return wide < static_cast<size_t>(sms) && 4 * narrow >= 3 * static_cast<size_t>(sms);
}

template <typename T>
cudaError_t launch_simt_gemm(bool a_kmajor, bool b_kmajor, int m, int n, int k, T alpha,
                             const T* A, size_t lda, const T* B, size_t ldb, T beta, T* C,
                             size_t ldc, cudaStream_t st, CUresult* cu_err, int tri, const T* Cin,
                             size_t ldcin) {
    if constexpr (sizeof(T) == 4) {
        if (simt_narrow_f32(m, n))
            return launch_simt_tiles<T, 1>(a_kmajor, b_kmajor, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, st,
                                           cu_err, tri, Cin, ldcin);
    }
    return launch_simt_tiles<T, 0>(a_kmajor, b_kmajor, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, st, cu_err,
                                   tri, Cin, ldcin);
}

template cudaError_t launch_simt_gemm<float>(bool, bool, int, int, int, float, const float*, size_t,
                                             const float*, size_t, float, float*, size_t, cudaStream_t,
                                             CUresult*, int, const float*, size_t);
template cudaError_t launch_simt_gemm<double>(bool, bool, int, int, int, double, const double*, size_t,
                                              const double*, size_t, double, double*, size_t,
                                              cudaStream_t, CUresult*, int, const double*, size_t);
template cudaError_t launch_scale_c<float>(int, int, float, float*, size_t, cudaStream_t, int);
template cudaError_t launch_scale_c<double>(int, int, double, double*, size_t, cudaStream_t, int);

}  // namespace rb
