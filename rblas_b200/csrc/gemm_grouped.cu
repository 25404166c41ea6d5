// gemm_grouped.cu -- grouped GEMM: many problems with their own m, n, k,
// transposes, alpha/beta and dtype (f32 / f64, plain form) in one launch.
//
// The host builds a device-side problem table: per problem two TMA tensor
// maps (in global memory, 64-byte aligned), the epilogue description, the
// tile grid and the problem's first index in the concatenated tile space.
// A persistent grid (one CTA per SM) walks that space round-robin; each
// CTA's producer lane and compute warps follow the same tile sequence, find
// the problem by binary search, and run the same tile pipeline as the
// single-problem kernel (simt_tile.cuh) through one continuous mbarrier ring,
// so tiles of different problems stream back to back without a launch.
// Work per problem: 2mnk flop.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/rblas_b200.h"
#include "rb_device.cuh"
#include "rb_internal.h"
#include "simt_tile.cuh"

namespace rb {

namespace {

constexpr int kGroupStage = 32768;  // max(f32 32 KiB, f64 24 KiB) stage
constexpr int kGroupSmem = SimtCfg<float>::STAGES * kGroupStage + 2 * SimtCfg<float>::STAGES * 8 + 1024;
static_assert(SimtCfg<float>::STAGES == SimtCfg<double>::STAGES, "one ring for both dtypes");

struct alignas(64) GroupProblem {
    CUtensorMap tmA;
    CUtensorMap tmB;
    void* c;
    const void* cin;
    uint64_t ldc, ldcin;
    double alpha, beta;
    int m, n, num_kt;
    int variant;  // dtype * 4 + a_kmajor * 2 + b_kmajor
    int tiles_m, tiles_n;
    int beta_mode;
    int pad;
};

__device__ __forceinline__ int find_problem(const int* __restrict__ starts, int nprob, int t) {
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(starts + mid) <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <typename T, bool A_K, bool B_K>
__device__ __noinline__ bool produce_v(const GroupProblem* p, int tm, int tn, uint8_t* smem, uint64_t* full,
                                          uint64_t* empty, uint32_t& it, uint32_t* err) {
    return simt_produce<T, A_K, B_K>(&p->tmA, &p->tmB, tm * SimtCfg<T>::BM, tn * SimtCfg<T>::BN, p->num_kt, smem,
                                     kGroupStage, full, empty, it, err);
}

template <typename T, bool A_K, bool B_K>
__device__ __noinline__ bool consume_v(const GroupProblem* p, int tm, int tn, uint8_t* smem, uint64_t* full,
                                          uint64_t* empty, uint32_t& it, uint32_t* err, int warp, int lane) {
    const SimtOut<T> o{static_cast<T*>(p->c), p->ldc, static_cast<const T*>(p->cin), p->ldcin, p->m, p->n,
                       static_cast<T>(p->alpha), static_cast<T>(p->beta), p->beta_mode, 0};
    return simt_consume<T, A_K, B_K>(o, tm * SimtCfg<T>::BM, tn * SimtCfg<T>::BN, p->num_kt, smem, kGroupStage,
                                     full, empty, it, err, warp, lane);
}

__global__ void __launch_bounds__(kSimtThreads, 1)
    grouped_gemm_kernel(const GroupProblem* __restrict__ probs, const int* __restrict__ starts, int nprob,
                        int total_tiles, uint32_t* err) {
    constexpr int ST = SimtCfg<float>::STAGES;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + ST * kGroupStage);
    uint64_t* empty = full + ST;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kSimtComputeWarps);
        }
        fence_barrier_init();
    }
    __syncthreads();
    uint32_t it = 0;
    const bool producer = (warp == kSimtComputeWarps);
    if (producer && lane != 0) return;
    for (int t = blockIdx.x; t < total_tiles; t += gridDim.x) {
        const int pi = find_problem(starts, nprob, t);
        const GroupProblem* p = probs + pi;
        int tm, tn;
        raster_tile(t - __ldg(starts + pi), p->tiles_m, p->tiles_n, tm, tn);
        bool ok;
        if (producer) {
            switch (p->variant) {
                case 0: ok = produce_v<float, false, false>(p, tm, tn, smem, full, empty, it, err); break;
                case 1: ok = produce_v<float, false, true>(p, tm, tn, smem, full, empty, it, err); break;
                case 2: ok = produce_v<float, true, false>(p, tm, tn, smem, full, empty, it, err); break;
                case 3: ok = produce_v<float, true, true>(p, tm, tn, smem, full, empty, it, err); break;
                case 4: ok = produce_v<double, false, false>(p, tm, tn, smem, full, empty, it, err); break;
                case 5: ok = produce_v<double, false, true>(p, tm, tn, smem, full, empty, it, err); break;
                case 6: ok = produce_v<double, true, false>(p, tm, tn, smem, full, empty, it, err); break;
                default: ok = produce_v<double, true, true>(p, tm, tn, smem, full, empty, it, err); break;
            }
        } else {
            switch (p->variant) {
                case 0: ok = consume_v<float, false, false>(p, tm, tn, smem, full, empty, it, err, warp, lane); break;
                case 1: ok = consume_v<float, false, true>(p, tm, tn, smem, full, empty, it, err, warp, lane); break;
                case 2: ok = consume_v<float, true, false>(p, tm, tn, smem, full, empty, it, err, warp, lane); break;
                case 3: ok = consume_v<float, true, true>(p, tm, tn, smem, full, empty, it, err, warp, lane); break;
                case 4: ok = consume_v<double, false, false>(p, tm, tn, smem, full, empty, it, err, warp, lane); break;
                case 5: ok = consume_v<double, false, true>(p, tm, tn, smem, full, empty, it, err, warp, lane); break;
                case 6: ok = consume_v<double, true, false>(p, tm, tn, smem, full, empty, it, err, warp, lane); break;
                default: ok = consume_v<double, true, true>(p, tm, tn, smem, full, empty, it, err, warp, lane); break;
            }
        }
        if (!ok) return;
    }
}

inline size_t rup(size_t x, size_t m) { return (x + m - 1) / m * m; }

bool tma_aligned(const void* p, size_t ld, size_t elem) {
    return (reinterpret_cast<uintptr_t>(p) % 16 == 0) && ((ld * elem) % 16 == 0);
}

}  // namespace

int validate_problem(const rb_gemm_problem& q) {
    if ((q.dtype != 0 && q.dtype != 1) || (q.layout != RB_ROW_MAJOR && q.layout != RB_COL_MAJOR) ||
        q.transa < 0 || q.transa > 2 || q.transb < 0 || q.transb > 2)
        return RB_ERR_INVALID_ARG;
    const bool ta = q.transa != RB_NO_TRANS, tb = q.transb != RB_NO_TRANS;
    // leading dimensions (check_matrix, src/level3.rs:107-140)
    struct Chk { size_t rows, cols, ld; } chk[3] = {
        {ta ? q.k : q.m, ta ? q.m : q.k, q.lda}, {tb ? q.n : q.k, tb ? q.k : q.n, q.ldb}, {q.m, q.n, q.ldc}};
    for (const Chk& c : chk) {
        if (c.rows == 0 || c.cols == 0) continue;
        if (c.ld < ((q.layout == RB_ROW_MAJOR) ? c.cols : c.rows)) return RB_ERR_INVALID_LEADING_DIM;
    }
    // tile indices are 32-bit
    if (q.m > 0x7fffffff || q.n > 0x7fffffff || q.k > 0x7fffffff) return RB_ERR_INVALID_ARG;
    return RB_OK;
}

size_t grouped_table_bytes(size_t count) { return count * (sizeof(GroupProblem) + sizeof(int)); }

int grouped_gemm_dev(const rb_gemm_problem* probs, size_t count, const void* const* cin, const size_t* ldcin,
                     cudaStream_t st, int32_t* ce, size_t* bad_index, const GroupStaging* staging) {
    std::vector<GroupProblem> table;
    std::vector<int> starts;
    table.reserve(count);
    size_t scratch = 0;
    int total = 0;
    // first pass: validate and normalise (row-major -> column-major by swapping the operands)
    struct Norm { bool ta, tb; size_t m, n, k; const void* a; size_t lda; const void* b; size_t ldb; };
    std::vector<Norm> norm(count);
    for (size_t i = 0; i < count; ++i) {
        const rb_gemm_problem& q = probs[i];
        const int v = validate_problem(q);
        if (v != RB_OK) {
            if (bad_index) *bad_index = i;
            return v;
        }
        const bool ta = q.transa != RB_NO_TRANS, tb = q.transb != RB_NO_TRANS;
        if (q.layout == RB_COL_MAJOR) norm[i] = {ta, tb, q.m, q.n, q.k, q.a, q.lda, q.b, q.ldb};
        else norm[i] = {tb, ta, q.n, q.m, q.k, q.b, q.ldb, q.a, q.lda};
    }
    // second pass: scratch for operands TMA cannot address directly
    const size_t elem_of[2] = {4, 8};
    std::vector<std::pair<size_t, size_t>> rp_a(count, {SIZE_MAX, 0}), rp_b(count, {SIZE_MAX, 0});
    for (size_t i = 0; i < count; ++i) {
        const Norm& nm = norm[i];
        const size_t el = elem_of[probs[i].dtype];
        if (nm.m == 0 || nm.n == 0 || nm.k == 0 || probs[i].alpha == 0.0) continue;
        const size_t vec = 16 / el;
        if (!tma_aligned(nm.a, nm.lda, el)) {
            const size_t rows = nm.ta ? nm.k : nm.m, cols = nm.ta ? nm.m : nm.k, ld2 = rup(rows, vec);
            rp_a[i] = {scratch, ld2};
            scratch += rup(ld2 * cols * el, 256);
        }
        if (!tma_aligned(nm.b, nm.ldb, el)) {
            const size_t rows = nm.tb ? nm.n : nm.k, cols = nm.tb ? nm.k : nm.n, ld2 = rup(rows, vec);
            rp_b[i] = {scratch, ld2};
            scratch += rup(ld2 * cols * el, 256);
        }
    }
    uint8_t* sbuf = nullptr;
    cudaError_t e;
    if (scratch) {
        e = cudaMallocAsync(reinterpret_cast<void**>(&sbuf), scratch, st);
        if (e != cudaSuccess) { if (ce) *ce = e; return RB_ERR_CUDA; }
    }
    for (size_t i = 0; i < count; ++i) {
        const rb_gemm_problem& q = probs[i];
        Norm nm = norm[i];
        if (nm.m == 0 || nm.n == 0) continue;
        const size_t el = elem_of[q.dtype];
        const bool f64 = q.dtype == 1;
        const bool skip_ab = (nm.k == 0 || q.alpha == 0.0);
        if (rp_a[i].first != SIZE_MAX) {
            const size_t rows = nm.ta ? nm.k : nm.m, cols = nm.ta ? nm.m : nm.k;
            e = cudaMemcpy2DAsync(sbuf + rp_a[i].first, rp_a[i].second * el, nm.a, nm.lda * el, rows * el, cols,
                                  cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) { if (ce) *ce = e; cudaFreeAsync(sbuf, st); return RB_ERR_CUDA; }
            nm.a = sbuf + rp_a[i].first;
            nm.lda = rp_a[i].second;
        }
        if (rp_b[i].first != SIZE_MAX) {
            const size_t rows = nm.tb ? nm.n : nm.k, cols = nm.tb ? nm.k : nm.n;
            e = cudaMemcpy2DAsync(sbuf + rp_b[i].first, rp_b[i].second * el, nm.b, nm.ldb * el, rows * el, cols,
                                  cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) { if (ce) *ce = e; cudaFreeAsync(sbuf, st); return RB_ERR_CUDA; }
            nm.b = sbuf + rp_b[i].first;
            nm.ldb = rp_b[i].second;
        }
        GroupProblem g{};
        const int BM = 128, BN = f64 ? SimtCfg<double>::BN : SimtCfg<float>::BN;
        const int BK = f64 ? SimtCfg<double>::BK : SimtCfg<float>::BK;
        const CUtensorMapDataType dt = f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
        const bool a_k = nm.ta, b_k = !nm.tb;
        CUresult r = CUDA_SUCCESS;
        if (!skip_ab) {
            r = a_k ? make_tmap_2d(&g.tmA, nm.a, dt, el, nm.k, nm.m, nm.lda, BK, BM, true)
                    : make_tmap_2d(&g.tmA, nm.a, dt, el, nm.m, nm.k, nm.lda, BM, BK, false);
            if (r == CUDA_SUCCESS)
                r = b_k ? make_tmap_2d(&g.tmB, nm.b, dt, el, nm.k, nm.n, nm.ldb, BK, BN, true)
                        : make_tmap_2d(&g.tmB, nm.b, dt, el, nm.n, nm.k, nm.ldb, BN, BK, false);
        }
        if (r != CUDA_SUCCESS) {
            if (ce) *ce = static_cast<int32_t>(r);
            if (bad_index) *bad_index = i;
            if (sbuf) cudaFreeAsync(sbuf, st);
            return RB_ERR_CUDA;
        }
        g.c = q.c;
        g.ldc = q.ldc;
        g.cin = cin ? cin[i] : q.c;
        g.ldcin = ldcin ? ldcin[i] : q.ldc;
        g.alpha = q.alpha;
        g.beta = q.beta;
        g.m = static_cast<int>(nm.m);
        g.n = static_cast<int>(nm.n);
        g.num_kt = skip_ab ? 0 : static_cast<int>((nm.k + BK - 1) / BK);  // k == 0 || alpha == 0: C = beta*Cin
        g.variant = (f64 ? 4 : 0) + (a_k ? 2 : 0) + (b_k ? 1 : 0);
        g.tiles_m = static_cast<int>((nm.m + BM - 1) / BM);
        g.tiles_n = static_cast<int>((nm.n + BN - 1) / BN);
        g.beta_mode = (q.beta == 0.0) ? 0 : (q.beta == 1.0 ? 1 : 2);
        starts.push_back(total);
        total += g.tiles_m * g.tiles_n;
        table.push_back(g);
    }
    if (table.empty()) {
        if (sbuf) cudaFreeAsync(sbuf, st);
        return RB_OK;
    }
    const size_t tbytes = table.size() * sizeof(GroupProblem);
    const size_t all_bytes = tbytes + starts.size() * sizeof(int);
    void* dev = nullptr;
    const bool staged = staging && staging->host && staging->dev && all_bytes <= staging->bytes;
    if (staged) {
        // pinned source: one truly asynchronous copy, no allocation
        std::memcpy(staging->host, table.data(), tbytes);
        std::memcpy(static_cast<uint8_t*>(staging->host) + tbytes, starts.data(), starts.size() * sizeof(int));
        dev = staging->dev;
        e = cudaMemcpyAsync(dev, staging->host, all_bytes, cudaMemcpyHostToDevice, st);
    } else {
        e = cudaMallocAsync(&dev, all_bytes, st);
        if (e != cudaSuccess) { if (ce) *ce = e; if (sbuf) cudaFreeAsync(sbuf, st); return RB_ERR_CUDA; }
        // pageable sources: the copies are staged before the calls return
        e = cudaMemcpyAsync(dev, table.data(), tbytes, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(static_cast<uint8_t*>(dev) + tbytes, starts.data(), starts.size() * sizeof(int),
                                cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess) {
        static bool attr = false;
        if (!attr) {
            e = cudaFuncSetAttribute(grouped_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kGroupSmem);
            attr = (e == cudaSuccess);
        }
    }
    if (e == cudaSuccess) {
        int dev_id = 0, sms = 148;
        cudaGetDevice(&dev_id);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_id);
        double work = 0;
        for (size_t i = 0; i < count; ++i) work += 2.0 * probs[i].m * probs[i].n * static_cast<double>(probs[i].k);
        KernelTimer tmr;
        kernel_timing_begin("grouped_gemm", work, st, &tmr);
        grouped_gemm_kernel<<<std::min(total, sms), kSimtThreads, kGroupSmem, st>>>(
            static_cast<const GroupProblem*>(dev),
            reinterpret_cast<const int*>(static_cast<uint8_t*>(dev) + tbytes), static_cast<int>(table.size()), total,
            device_error_word());
        kernel_timing_end(&tmr, st);
        count_launch();
        e = cudaGetLastError();
    }
    if (!staged) cudaFreeAsync(dev, st);
    if (sbuf) cudaFreeAsync(sbuf, st);
    if (e != cudaSuccess) { if (ce) *ce = e; return RB_ERR_CUDA; }
    return RB_OK;
}

int single_gemm_dev(const rb_gemm_problem* prob, const void* cin, size_t ldcin, cudaStream_t st, int32_t* ce) {
    const rb_gemm_problem& q = *prob;
    const int v = validate_problem(q);
    if (v != RB_OK) return v;
    const bool ta = q.transa != RB_NO_TRANS, tb = q.transb != RB_NO_TRANS;
    const bool col = q.layout == RB_COL_MAJOR;
    const size_t el = q.dtype ? 8 : 4;
    const size_t m = col ? q.m : q.n, n = col ? q.n : q.m;
    const void* a = col ? q.a : q.b;
    const void* b = col ? q.b : q.a;
    const size_t lda = col ? q.lda : q.ldb, ldb = col ? q.ldb : q.lda;
    const bool nta = col ? ta : tb, ntb = col ? tb : ta;
    // the single kernel needs TMA-addressable operands and a real product;
    // everything else goes through the one-problem table path
    if (m == 0 || n == 0 || q.k == 0 || q.alpha == 0.0 || !tma_aligned(a, lda, el) || !tma_aligned(b, ldb, el))
        return grouped_gemm_dev(prob, 1, &cin, &ldcin, st, ce, nullptr);
    CUresult cr = CUDA_SUCCESS;
    cudaError_t e;
    if (q.dtype == 1)
        e = launch_simt_gemm<double>(nta, !ntb, (int)m, (int)n, (int)q.k, q.alpha, static_cast<const double*>(a),
                                     lda, static_cast<const double*>(b), ldb, q.beta, static_cast<double*>(q.c),
                                     q.ldc, st, &cr, 0, static_cast<const double*>(cin), ldcin);
    else
        e = launch_simt_gemm<float>(nta, !ntb, (int)m, (int)n, (int)q.k, (float)q.alpha,
                                    static_cast<const float*>(a), lda, static_cast<const float*>(b), ldb,
                                    (float)q.beta, static_cast<float*>(q.c), q.ldc, st, &cr, 0,
                                    static_cast<const float*>(cin), ldcin);
    if (e != cudaSuccess) {
        if (ce) *ce = (cr != CUDA_SUCCESS) ? static_cast<int32_t>(cr) : static_cast<int32_t>(e);
        return RB_ERR_CUDA;
    }
    return RB_OK;
}

}  // namespace rb
