// gemm_umma.cu -- the split-precision GEMM forms on the 5th-generation tensor
// cores (tcgen05.mma, accumulators in TMEM):
//
//   BF16X3 (SGEMM): x = hi + lo with hi = bf16(x), lo = bf16(x - hi);
//     C = alpha * (Ah*Bh + Ah*Bl + Al*Bh) + beta * C, FP32 accumulation.
//   OZAKI (DGEMM): Ozaki-scheme INT8 slice emulation (Ozaki, Ogita, Oishi &
//     Rump, "Error-free transformations of matrix multiplication by using
//     fast routines of matrix multiplication and its applications", Numer.
//     Algorithms 59, 2012; Ootomo, Ozaki & Yokota, "DGEMM on integer matrix
//     multiplication unit", IJHPCA 2024). Each row of op(A) / column of op(B)
//     is scaled by a power of two 2^-e so |x| < 1, then cut into `s` signed
//     7-bit slices: x * 2^-e = sum_t sigma_t 2^-7(t+1). Slice products are
//     exact in INT32; the products of equal weight (t+u = d) share one TMEM
//     accumulator, and C = alpha * 2^(e_i+f_j) sum_d 2^-7(d+2) S_d + beta * C
//     is summed in FP64 from the smallest weight up. Pairs with t+u >= s are
//     dropped (the scheme's truncation).
//
// Both replace rblas's CPU blocking/packing/microkernel path
// (src/kernel/gemm.rs:185-429) for the precision forms that rblas does not
// have; the plain forms live in gemm_simt.cu.
//
// Kernel structure (persistent, one CTA per SM, 6 warps):
//   warp 0 lane 0  TMA producer: K-major operand tiles (128-byte rows, 128-byte
//                  swizzle) into a STAGES-deep shared-memory ring.
//   warp 1         allocates 512 TMEM columns; lane 0 issues tcgen05.mma
//                  (M=128, N=256) into one of two 256-column accumulators and
//                  commits each stage back to the producer.
//   warps 2..5     epilogue: tcgen05.ld the accumulator (warp w reads TMEM
//                  lanes 32*(w%4)..+31 = tile rows), apply the form's
//                  scaling and alpha/beta, store C coalesced; release the
//                  accumulator so the next unit's MMAs overlap this drain.
// Operands are first rewritten by a pre-pass into K-major bf16 hi/lo planes
// or int8 slice planes (this also absorbs every transpose and layout).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>
#include <type_traits>

#include "../../include/rblas_b200.h"
#include "rb_device.cuh"
#include "rb_internal.h"

namespace rb {

namespace {

constexpr int kUM = 128;
constexpr int kRowBytes = 128;                  // K bytes per tile row (one swizzle row)
constexpr int kATile = kUM * kRowBytes;         // 16 KiB
constexpr int kExpSentinel = -(1 << 30);        // row exponent of an all-zero row

enum { kModeBf16x3 = 0, kModeBf16x6 = 1 };

// Per BF16 form: tile N, operand planes per stage, ring depth, and the plane
// products issued per UMMA K step (smallest weights first).
template <int MODE> struct UCfg;
template <> struct UCfg<kModeBf16x3> {
    static constexpr int UN = 128, NA = 2, NB = 2, STAGES = 3, NPROD = 3, THREADS = 192;
    // lo*hi, hi*lo, hi*hi
    __host__ __device__ static constexpr int pa(int q) { return q == 0 ? 1 : 0; }
    __host__ __device__ static constexpr int pb(int q) { return q == 1 ? 1 : 0; }
};
template <> struct UCfg<kModeBf16x6> {
    static constexpr int UN = 128, NA = 3, NB = 3, STAGES = 2, NPROD = 6, THREADS = 192;
    // weight 2 (lo*hi, mid*mid, hi*lo), weight 1 (mid*hi, hi*mid), weight 0 (hi*hi)
    __host__ __device__ static constexpr int pa(int q) { return q == 0 ? 2 : (q == 1 || q == 3) ? 1 : 0; }
    __host__ __device__ static constexpr int pb(int q) { return q == 2 ? 2 : (q == 1 || q == 4) ? 1 : 0; }
};

template <int MODE>
constexpr int umma_smem_bytes() {
    using C = UCfg<MODE>;
    return C::STAGES * (C::NA * kATile + C::NB * C::UN * kRowBytes) + 256 + 1024;
}

struct UParams {
    int m, n, k;
    int tiles_m, tiles_n, num_tiles;
    int num_kt;        // 128-byte K tiles over the whole K
    int kt_per_chunk;  // K tiles per accumulation unit (FP32 promotion interval)
    int kchunks;
    int beta_mode;     // 0 beta == 0, 1 beta == 1, 2 general
    float alpha_f, beta_f;
    float* c;
    size_t ldc;
    const float* cin;  // C0, read for beta != 0: c itself, or a separate input with c's leading dimension
    uint32_t* err;
};

constexpr int kMaxStages = 8;  // mbarrier pairs in Bar: every kernel's ring must fit

struct Bar {
    uint64_t full[kMaxStages], empty[kMaxStages], acc_full[2], acc_empty[2], drain;
    uint32_t tmem_base;
};
static_assert(sizeof(Bar) <= 256, "the kernels reserve 256 bytes of shared memory for Bar");

// One problem of a grouped BF16-split launch: its plane tensor maps (64-byte
// aligned for TMA) and parameters.
struct alignas(64) UGroupEntry {
    CUtensorMap tmA, tmB;
    UParams p;
};

struct UWork {
    const UParams* p;
    const CUtensorMap* ta;
    const CUtensorMap* tb;
    int t;  // tile of the problem
};

// The single-problem kernel's tiles, one problem.
struct USingleSrc {
    const UParams* p;
    const CUtensorMap* ta;
    const CUtensorMap* tb;
    __device__ __forceinline__ uint32_t* err() const { return p->err; }
    __device__ __forceinline__ int items() const { return p->num_tiles; }
    __device__ __forceinline__ UWork get(int item) const { return UWork{p, ta, tb, item}; }
};

// Grouped: item i is tile i - starts[j] of problem j (starts[j] <= i <
// starts[j+1]); problems ordered by K, longest first.
struct UGroupSrc {
    const UGroupEntry* tab;
    const int* starts;
    int nprob;
    uint32_t* error;
    __device__ __forceinline__ uint32_t* err() const { return error; }
    __device__ __forceinline__ int items() const { return __ldg(starts + nprob); }
    __device__ __forceinline__ UWork get(int item) const {
        int lo = 0, hi = nprob - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(starts + mid) <= item) lo = mid;
            else hi = mid - 1;
        }
        const UGroupEntry* g = tab + lo;
        return UWork{&g->p, &g->tmA, &g->tmB, item - __ldg(starts + lo)};
    }
};

// Work of one tile is a sequence of accumulation units: unit c covers K
// tiles [c*G, (c+1)*G) with all plane products, and the epilogue promotes
// each unit's FP32 partial into FP32 registers (tcgen05's accumulation
// truncates; short units keep that error small).
template <int MODE, class Src>
__device__ __forceinline__ void umma_body(const Src& src) {
    using Cfg = UCfg<MODE>;
    constexpr int UN = Cfg::UN, NA = Cfg::NA, NB = Cfg::NB, ST = Cfg::STAGES;
    static_assert(ST <= kMaxStages, "Bar holds kMaxStages stages");
    constexpr int BTILE = UN * kRowBytes;
    constexpr int STAGE_BYTES = NA * kATile + NB * BTILE;
    constexpr int KSTEPS = 4;  // UMMA K steps of 32 bytes per 128-byte tile row
    constexpr uint32_t IDESC = umma_idesc(1, 1, kUM, UN);  // f32 <- bf16
    // BF16X6 keeps hi*hi apart from the five smaller products: tcgen05's FP32
    // accumulation truncates, so each of its roundings costs up to one ulp of
    // the accumulator it adds into. In an accumulator of their own the small
    // products' roundings are ~2^-8 of hi*hi's, and hi*hi's own are one per
    // instruction instead of one per product. (At K ~ 400 the shared
    // accumulator left BF16X6 at up to 4x plain SGEMM's error.)
    constexpr bool SPLIT_ACC = (MODE == kModeBf16x6);
    constexpr uint32_t ACC_COLS = SPLIT_ACC ? 2 * UN : UN;  // per accumulator buffer
    constexpr uint32_t TMEM_COLS = 2 * ACC_COLS;
    static_assert(TMEM_COLS <= 512, "two buffers must fit the SM's TMEM");

    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    Bar* bar = reinterpret_cast<Bar*>(smem + ST * STAGE_BYTES);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; ++s) {
            mbar_init(&bar->full[s], 1);
            mbar_init(&bar->empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&bar->acc_full[b], 1);
            mbar_init(&bar->acc_empty[b], 4);
        }
        mbar_init(&bar->drain, 1);
        fence_barrier_init();
    }
    if (warp == 1) {
        tmem_alloc(&bar->tmem_base, TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = bar->tmem_base;
    const int items = src.items();
    uint32_t* const err = src.err();
    bool ok = true;

    if (warp == 0 && lane == 0) {
        // ------------------------------ TMA producer ------------------------------
        uint32_t it = 0;
        const CUtensorMap* fetched = nullptr;
        for (int item = blockIdx.x; ok && item < items; item += gridDim.x) {
            const UWork w = src.get(item);
            const UParams& p = *w.p;
            if (w.ta != fetched) {
                prefetch_tmap(w.ta);
                prefetch_tmap(w.tb);
                fetched = w.ta;
            }
            int tm, tn;
            raster_tile(w.t, p.tiles_m, p.tiles_n, tm, tn);
            const int m0 = tm * kUM, n0 = tn * UN;
            for (int kt = 0; kt < p.num_kt; ++kt, ++it) {
                const int s = it % ST;
                if (it >= ST && !mbar_wait(&bar->empty[s], ((it / ST) - 1) & 1, err, 0x201)) {
                    ok = false;
                    break;
                }
                uint8_t* sa = smem + s * STAGE_BYTES;
                uint8_t* sb = sa + NA * kATile;
                mbar_arrive_expect_tx(&bar->full[s], STAGE_BYTES);
                const int k0 = kt * 64;  // bf16 elements per 128-byte row
#pragma unroll
                for (int q = 0; q < NA; ++q) tma_load_3d(sa + q * kATile, w.ta, &bar->full[s], k0, m0, q);
#pragma unroll
                for (int q = 0; q < NB; ++q) tma_load_3d(sb + q * BTILE, w.tb, &bar->full[s], k0, n0, q);
            }
        }
        if (!ok) {
            const uint32_t first = it > (uint32_t)ST ? it - ST : 0;
            for (uint32_t j = first; j < it; ++j) mbar_wait_drain(&bar->full[j % ST], (j / ST) & 1);
        }
    } else if (warp == 1 && lane == 0) {
        // ------------------------------ MMA issuer ------------------------------
        uint32_t it = 0, uc = 0;
        for (int item = blockIdx.x; ok && item < items; item += gridDim.x) {
            const UWork w = src.get(item);
            const UParams& p = *w.p;
            const int units = p.kchunks;
            for (int u = 0; ok && u < units; ++u, ++uc) {
                const int kt0 = u * p.kt_per_chunk, kt1 = min(p.num_kt, kt0 + p.kt_per_chunk);
                const uint32_t b = uc & 1;
                if (uc >= 2 && !mbar_wait(&bar->acc_empty[b], ((uc >> 1) - 1) & 1, err, 0x202)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d_tmem = tmem_base + b * ACC_COLS;        // the products (all, or all but hi*hi)
                const uint32_t d_big = SPLIT_ACC ? d_tmem + UN : d_tmem;  // hi*hi
                uint32_t accumulate = 0;
                for (int kt = kt0; kt < kt1; ++kt, ++it) {
                    const int s = it % ST;
                    if (!mbar_wait(&bar->full[s], (it / ST) & 1, err, 0x203)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sa = smem_u32(smem + s * STAGE_BYTES);
                    const uint32_t sb = sa + NA * kATile;
#pragma unroll
                    for (int kk = 0; kk < KSTEPS; ++kk) {
#pragma unroll
                        for (int q = 0; q < Cfg::NPROD; ++q) {
                            const bool big = SPLIT_ACC && q == Cfg::NPROD - 1;
                            umma_f16(big ? d_big : d_tmem, sw128_kmajor_desc(sa + Cfg::pa(q) * kATile) + 2 * kk,
                                     sw128_kmajor_desc(sb + Cfg::pb(q) * BTILE) + 2 * kk, IDESC,
                                     (q == 0 || big) ? accumulate : 1u);
                        }
                        accumulate = 1;
                    }
                    tc_commit(&bar->empty[s]);  // stage free once these MMAs complete
                }
                if (ok) tc_commit(&bar->acc_full[b]);
            }
        }
        // make sure nothing of ours is still in flight before TMEM is released
        tc_commit(&bar->drain);
        mbar_wait_drain(&bar->drain, 0);
    } else if (warp >= 2) {
        // ------------------------------ epilogue ------------------------------
        const int quarter = warp & 3;
        const int row_in_tile = quarter * 32 + lane;
        uint32_t uc = 0;
        for (int item = blockIdx.x; ok && item < items; item += gridDim.x) {
            const UWork w = src.get(item);
            const UParams& p = *w.p;
            const int units = p.kchunks;
            int tm, tn;
            raster_tile(w.t, p.tiles_m, p.tiles_n, tm, tn);
            const int m0 = tm * kUM, n0 = tn * UN;
            const int r = m0 + row_in_tile;
            const bool row_ok = r < p.m;
            float sum[UN];
#pragma unroll
            for (int j = 0; j < UN; ++j) sum[j] = 0.f;
            for (int u = 0; ok && u < units; ++u, ++uc) {
                const uint32_t b = uc & 1;
                if (!mbar_wait(&bar->acc_full[b], (uc >> 1) & 1, err, 0x204)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t taddr = tmem_base + (static_cast<uint32_t>(quarter * 32) << 16) + b * ACC_COLS;
                // the smaller products first, then hi*hi (SPLIT_ACC)
#pragma unroll
                for (int part = 0; part < (SPLIT_ACC ? 2 : 1); ++part) {
#pragma unroll
                    for (int ch = 0; ch < UN / 32; ++ch) {
                        uint32_t v[32];
                        tmem_ld32(taddr + part * UN + ch * 32, v);
                        tmem_ld_wait();
#pragma unroll
                        for (int j = 0; j < 32; ++j) sum[ch * 32 + j] += __uint_as_float(v[j]);
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&bar->acc_empty[b]);
            }
            if (ok && row_ok) {
                // C0 read 16 values at a time, all requested before use, so
                // the loads' latencies overlap instead of adding up
#pragma unroll
                for (int g = 0; g < UN / 16; ++g) {
                    float cv[16];
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj) {
                        const int col = n0 + g * 16 + jj;
                        cv[jj] = (p.beta_mode != 0 && col < p.n) ? p.cin[r + static_cast<size_t>(col) * p.ldc] : 0.f;
                    }
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj) {
                        const int col = n0 + g * 16 + jj;
                        if (col < p.n) {
                            const float tb = (p.beta_mode == 2) ? p.beta_f * cv[jj] : cv[jj];
                            p.c[r + static_cast<size_t>(col) * p.ldc] = fmaf(p.alpha_f, sum[g * 16 + jj], tb);
                        }
                    }
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, TMEM_COLS);
    }
}

template <int MODE>
__global__ void __launch_bounds__(UCfg<MODE>::THREADS, 1)
    umma_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                     const __grid_constant__ UParams p) {
    umma_body<MODE>(USingleSrc{&p, &tmA, &tmB});
}

// Many f32 problems in one persistent launch (the serving loop's BF16-split
// batches): the same tiles and epilogue as umma_gemm_kernel.
template <int MODE>
__global__ void __launch_bounds__(UCfg<MODE>::THREADS, 1)
    umma_grouped_kernel(const UGroupEntry* __restrict__ tab, const int* __restrict__ starts, int nprob,
                        uint32_t* err) {
    umma_body<MODE>(UGroupSrc{tab, starts, nprob, err});
}

// ------------------------------------------------------------------------------
// The BF16-split forms with A split inside the GEMM (A rows contiguous:
// NoTrans).
//
// Two passes read A, write its planes and read the planes again: about three
// times A's bytes, which is most of the time of a tall-skinny product
// (65536 x 128 x 8192: A is 2.1 GB, the GEMM itself ~0.3 ms of tensor work in
// 3xBF16). Here TMA brings 128 x 64 f32 tiles of A (128 contiguous rows per K
// column) into shared memory, and the epilogue warps split them, between
// their accumulator promotions, into the planes (hi, lo for 3xBF16; hi, mid,
// lo for BF16X6) in the 128-byte-swizzled K-major layout the UMMA
// descriptors read: row r's 16-byte chunk c at r * 128 + ((c ^ (r & 7)) *
// 16), the layout a TMA load of the planes produces. The split is the split
// pass's (hi = rn(x), then each next plane rn of what is left) and the
// products, their order, the accumulators and the promotions are
// umma_gemm_kernel<MODE>'s, so the results are the two-pass form's bit for
// bit. B's planes come from the split pass (B is small). Rings: A's f32
// tiles (released as soon as the splitters hold them in registers), A's
// planes (released by the MMAs), B's planes. BF16X6's three-plane stages
// leave room for one f32 stage only; its refill overlaps the conversion and
// the wait for a free plane stage.
// Warps: 0 TMA producer, 1 TMEM owner / MMA issuer, 2..9 splitter and
// epilogue: tile row quarter * 32 + lane (quarter = warp % 4, the TMEM lane
// quarter the warp may read) in both roles, and one half of the tile -- K
// chunks 4h..4h+3 of each 64-column K tile to split, columns 64h..64h+63 to
// promote and write -- for h = (warp - 2) / 4. Two such warps per scheduler
// hide each other's latencies, and 64 running sums per thread leave
// registers for the split.
// ------------------------------------------------------------------------------
template <int MODE> struct FzCfg;
template <> struct FzCfg<kModeBf16x3> { static constexpr int FS = 3, PS = 2, BS = 2; };
template <> struct FzCfg<kModeBf16x6> { static constexpr int FS = 1, PS = 2, BS = 2; };
constexpr int kFzMaxStages = 3;
constexpr int kFzThreads = 320;
constexpr int kFzEpiWarps = 8;
constexpr int kFzF32Tile = kUM * 64 * 4;  // 64 K columns of 128 f32 rows: 32 KiB
template <int MODE>
constexpr int fz_smem_bytes() {
    using F = FzCfg<MODE>;
    // f32 stages, then A's and B's plane stages (NA planes of one 128 x 64 tile each)
    return F::FS * kFzF32Tile + (F::PS + F::BS) * UCfg<MODE>::NA * kATile + 256 + 1024;
}
static_assert(fz_smem_bytes<kModeBf16x3>() <= 232448 && fz_smem_bytes<kModeBf16x6>() <= 232448,
              "the fused kernels' rings must fit one CTA's shared memory");

struct FzBar {
    uint64_t f_full[kFzMaxStages], f_empty[kFzMaxStages];
    uint64_t a_full[kFzMaxStages], a_empty[kFzMaxStages];
    uint64_t b_full[kFzMaxStages], b_empty[kFzMaxStages];
    uint64_t acc_full[2], acc_empty[2], drain;
    uint32_t tmem_base;
};
static_assert(sizeof(FzBar) <= 256, "the fused kernels reserve 256 bytes of shared memory for their barriers");

template <int MODE>
__global__ void __launch_bounds__(kFzThreads, 1)
    umma_split_fused_kernel(const __grid_constant__ CUtensorMap tmA32, const __grid_constant__ CUtensorMap tmB,
                            const __grid_constant__ UParams p) {
    using Cfg = UCfg<MODE>;
    constexpr int UN = Cfg::UN, NP = Cfg::NA;
    constexpr int FS = FzCfg<MODE>::FS, PS = FzCfg<MODE>::PS, BS = FzCfg<MODE>::BS;
    static_assert(FS <= kFzMaxStages && PS <= kFzMaxStages && BS <= kFzMaxStages, "FzBar holds the rings");
    static_assert(Cfg::NB == NP, "A and B have the same planes");
    constexpr int PLANES = NP * kATile;  // one plane stage: NP planes of a 128 x 64 tile
    constexpr int KSTEPS = 4;
    constexpr uint32_t IDESC = umma_idesc(1, 1, kUM, UN);  // f32 <- bf16
    // BF16X6 keeps hi*hi in an accumulator of its own, as umma_body does
    constexpr bool SPLIT_ACC = (MODE == kModeBf16x6);
    constexpr uint32_t ACC_COLS = SPLIT_ACC ? 2 * UN : UN;  // per accumulator buffer
    constexpr uint32_t TMEM_COLS = 2 * ACC_COLS;
    static_assert(TMEM_COLS <= 512, "two buffers must fit the SM's TMEM");
    static_assert(UN * kRowBytes == kATile, "B plane tiles are as large as A's");

    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint8_t* f32s = smem;                        // FS x 32 KiB, [k][row] f32
    uint8_t* aps = f32s + FS * kFzF32Tile;       // PS x NP planes, swizzled K-major
    uint8_t* bps = aps + PS * PLANES;            // BS x NP planes, by TMA
    FzBar* bar = reinterpret_cast<FzBar*>(bps + BS * PLANES);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < FS; ++s) {
            mbar_init(&bar->f_full[s], 1);
            mbar_init(&bar->f_empty[s], kFzEpiWarps);
        }
        for (int s = 0; s < PS; ++s) {
            mbar_init(&bar->a_full[s], kFzEpiWarps);
            mbar_init(&bar->a_empty[s], 1);
        }
        for (int s = 0; s < BS; ++s) {
            mbar_init(&bar->b_full[s], 1);
            mbar_init(&bar->b_empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&bar->acc_full[b], 1);
            mbar_init(&bar->acc_empty[b], kFzEpiWarps);
        }
        mbar_init(&bar->drain, 1);
        fence_barrier_init();
    }
    if (warp == 1) {
        tmem_alloc(&bar->tmem_base, TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = bar->tmem_base;
    const int items = p.num_tiles;
    uint32_t* const err = p.err;
    bool ok = true;

    if (warp == 0 && lane == 0) {
        // ------------------------------ TMA producer ------------------------------
        prefetch_tmap(&tmA32);
        prefetch_tmap(&tmB);
        uint32_t nf = 0, nb = 0;  // f32 tiles and B plane tiles issued
        for (int item = blockIdx.x; ok && item < items; item += gridDim.x) {
            int tm, tn;
            raster_tile(item, p.tiles_m, p.tiles_n, tm, tn);
            const int m0 = tm * kUM, n0 = tn * UN;
            for (int kt = 0; kt < p.num_kt; ++kt) {
                const int fs = nf % FS;
                if (nf >= FS && !mbar_wait(&bar->f_empty[fs], ((nf / FS) - 1) & 1, err, 0x211)) {
                    ok = false;
                    break;
                }
                mbar_arrive_expect_tx(&bar->f_full[fs], kFzF32Tile);
                tma_load_2d(f32s + fs * kFzF32Tile, &tmA32, &bar->f_full[fs], m0, kt * 64);
                ++nf;
                const int bs = nb % BS;
                if (nb >= BS && !mbar_wait(&bar->b_empty[bs], ((nb / BS) - 1) & 1, err, 0x212)) {
                    ok = false;
                    break;
                }
                mbar_arrive_expect_tx(&bar->b_full[bs], PLANES);
#pragma unroll
                for (int q = 0; q < NP; ++q)
                    tma_load_3d(bps + bs * PLANES + q * kATile, &tmB, &bar->b_full[bs], kt * 64, n0, q);
                ++nb;
            }
        }
        if (!ok) {  // this CTA's copies land before it exits
            for (uint32_t j = nf > (uint32_t)FS ? nf - FS : 0; j < nf; ++j)
                mbar_wait_drain(&bar->f_full[j % FS], (j / FS) & 1);
            for (uint32_t j = nb > (uint32_t)BS ? nb - BS : 0; j < nb; ++j)
                mbar_wait_drain(&bar->b_full[j % BS], (j / BS) & 1);
        }
    } else if (warp == 1 && lane == 0) {
        // ------------------------------ MMA issuer ------------------------------
        uint32_t it = 0, uc = 0;
        for (int item = blockIdx.x; ok && item < items; item += gridDim.x) {
            for (int u = 0; ok && u < p.kchunks; ++u, ++uc) {
                const int kt0 = u * p.kt_per_chunk, kt1 = min(p.num_kt, kt0 + p.kt_per_chunk);
                const uint32_t b = uc & 1;
                if (uc >= 2 && !mbar_wait(&bar->acc_empty[b], ((uc >> 1) - 1) & 1, err, 0x213)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d_tmem = tmem_base + b * ACC_COLS;        // the products (all, or all but hi*hi)
                const uint32_t d_big = SPLIT_ACC ? d_tmem + UN : d_tmem;  // hi*hi
                uint32_t accumulate = 0;
                for (int kt = kt0; kt < kt1; ++kt, ++it) {
                    const int ps = it % PS, bs = it % BS;
                    if (!mbar_wait(&bar->a_full[ps], (it / PS) & 1, err, 0x214) ||
                        !mbar_wait(&bar->b_full[bs], (it / BS) & 1, err, 0x215)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sa = smem_u32(aps + ps * PLANES);
                    const uint32_t sb = smem_u32(bps + bs * PLANES);
#pragma unroll
                    for (int kk = 0; kk < KSTEPS; ++kk) {
#pragma unroll
                        for (int q = 0; q < Cfg::NPROD; ++q) {
                            const bool big = SPLIT_ACC && q == Cfg::NPROD - 1;
                            umma_f16(big ? d_big : d_tmem, sw128_kmajor_desc(sa + Cfg::pa(q) * kATile) + 2 * kk,
                                     sw128_kmajor_desc(sb + Cfg::pb(q) * kATile) + 2 * kk, IDESC,
                                     (q == 0 || big) ? accumulate : 1u);
                        }
                        accumulate = 1;
                    }
                    tc_commit(&bar->a_empty[ps]);  // plane stages free once these MMAs complete
                    tc_commit(&bar->b_empty[bs]);
                }
                if (ok) tc_commit(&bar->acc_full[b]);
            }
        }
        tc_commit(&bar->drain);
        mbar_wait_drain(&bar->drain, 0);
    } else if (warp >= 2) {
        // ------------------------- splitter and epilogue -------------------------
        constexpr int HC = UN / 2;  // columns per warp
        const int quarter = warp & 3, half = (warp - 2) >> 2;
        const int row = quarter * 32 + lane;  // tile row: TMEM lane and split row
        uint32_t it = 0, uc = 0;
        for (int item = blockIdx.x; ok && item < items; item += gridDim.x) {
            int tm, tn;
            raster_tile(item, p.tiles_m, p.tiles_n, tm, tn);
            const int m0 = tm * kUM, n0 = tn * UN + half * HC;
            const int r = m0 + row;
            const bool row_ok = r < p.m;
            float sum[HC];
#pragma unroll
            for (int j = 0; j < HC; ++j) sum[j] = 0.f;
            int promoted = 0;
            // add unit `promoted`'s FP32 partial (TMEM) into sum, as umma_body does
            auto promote = [&]() -> bool {
                const uint32_t b = uc & 1;
                if (!mbar_wait(&bar->acc_full[b], (uc >> 1) & 1, err, 0x216)) return false;
                tc_fence_after();
                const uint32_t taddr =
                    tmem_base + (static_cast<uint32_t>(quarter * 32) << 16) + b * ACC_COLS + half * HC;
                // the smaller products first, then hi*hi (SPLIT_ACC)
#pragma unroll
                for (int part = 0; part < (SPLIT_ACC ? 2 : 1); ++part) {
#pragma unroll
                    for (int ch = 0; ch < HC / 32; ++ch) {
                        uint32_t v[32];
                        tmem_ld32(taddr + part * UN + ch * 32, v);
                        tmem_ld_wait();
#pragma unroll
                        for (int j = 0; j < 32; ++j) sum[ch * 32 + j] += __uint_as_float(v[j]);
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&bar->acc_empty[b]);
                ++uc;
                ++promoted;
                return true;
            };
            for (int kt = 0; kt < p.num_kt; ++kt, ++it) {
                const int fs = it % FS, ps = it % PS;
                if (!mbar_wait(&bar->f_full[fs], (it / FS) & 1, err, 0x218)) {
                    ok = false;
                    break;
                }
                // this warp's half of the row's 64 K values, split into NP
                // planes of packed bf16 pairs: pl[q][c4][j] holds plane q of K
                // values 8 c4 + 2 j (low half) and 8 c4 + 2 j + 1 (high half)
                uint32_t pl[NP][4][4];
                {
                    const float* F = reinterpret_cast<const float*>(f32s + fs * kFzF32Tile);  // F[k * 128 + row]
                    float v[32];
#pragma unroll
                    for (int e = 0; e < 32; ++e) v[e] = F[(half * 32 + e) * kUM + row];
#pragma unroll
                    for (int c4 = 0; c4 < 4; ++c4)
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            float v0 = v[c4 * 8 + 2 * j], v1 = v[c4 * 8 + 2 * j + 1];
#pragma unroll
                            for (int q = 0; q < NP; ++q) {
                                const __nv_bfloat162 hb = __floats2bfloat162_rn(v0, v1);  // rn(v0) low, rn(v1) high
                                pl[q][c4][j] = *reinterpret_cast<const uint32_t*>(&hb);
                                if (q + 1 < NP) {
                                    v0 -= __low2float(hb);
                                    v1 -= __high2float(hb);
                                }
                            }
                        }
                }
                // the f32 stage is free once every lane's reads have been used
                __threadfence_block();
                __syncwarp();
                if (lane == 0) mbar_arrive(&bar->f_empty[fs]);
                if (it >= PS && !mbar_wait(&bar->a_empty[ps], ((it / PS) - 1) & 1, err, 0x217)) {
                    ok = false;
                    break;
                }
                uint8_t* dst = aps + ps * PLANES;
#pragma unroll
                for (int c4 = 0; c4 < 4; ++c4) {
                    const int c = half * 4 + c4;
                    const uint32_t off = static_cast<uint32_t>(row) * kRowBytes + ((c ^ (row & 7)) << 4);
#pragma unroll
                    for (int q = 0; q < NP; ++q)
                        *reinterpret_cast<uint4*>(dst + q * kATile + off) =
                            make_uint4(pl[q][c4][0], pl[q][c4][1], pl[q][c4][2], pl[q][c4][3]);
                }
                fence_proxy_async_smem();  // the planes' generic stores, visible to the tensor cores
                __syncwarp();
                if (lane == 0) mbar_arrive(&bar->a_full[ps]);
                // once unit u's last tile is split, unit u - 1 is promoted: the
                // MMAs of unit u + 1 wait for that buffer, and the split of
                // unit u + 1's tiles waits for unit u's MMAs
                if ((kt + 1) % p.kt_per_chunk == 0 || kt + 1 == p.num_kt) {
                    if (kt / p.kt_per_chunk >= 1 && !promote()) {
                        ok = false;
                        break;
                    }
                }
            }
            while (ok && promoted < p.kchunks)
                if (!promote()) ok = false;
            if (ok && row_ok) {
#pragma unroll
                for (int g = 0; g < HC / 16; ++g) {
                    float cv[16];
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj) {
                        const int col = n0 + g * 16 + jj;
                        cv[jj] = (p.beta_mode != 0 && col < p.n) ? p.cin[r + static_cast<size_t>(col) * p.ldc] : 0.f;
                    }
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj) {
                        const int col = n0 + g * 16 + jj;
                        if (col < p.n) {
                            const float tb = (p.beta_mode == 2) ? p.beta_f * cv[jj] : cv[jj];
                            p.c[r + static_cast<size_t>(col) * p.ldc] = fmaf(p.alpha_f, sum[g * 16 + jj], tb);
                        }
                    }
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, TMEM_COLS);
    }
}

// ------------------------------------------------------------------------------
// Ozaki GEMM kernel.
//
// Slice products of equal weight (t + u = d: digit t has weight 2^-(7+8t))
// form diagonal d; S_d = sum_{t+u=d} A_t B_u^T is exact in INT32 over a K
// chunk. Diagonals are processed two at a time ("units" {d0, d1 = d0+1})
// with both accumulators in TMEM (2 x 256 columns). For each K tile the
// stages walk the A slices i = d1 .. 0, stage i holding A_i and B_{d1-i}:
// S_d1 takes A_i x B_{d1-i} from the stage, S_d0 takes A_i x B_{d0-i}, which
// is the B tile of the previous stage. So every stage brings one new A and
// one new B tile (48 KiB) for two MMAs, and a stage is released once the
// next one's MMAs have been issued. (The order of the INT32 additions does
// not change the exact sums.) The epilogue folds the unit exactly,
// S_d0 * 2^8 + S_d1 (< 2^40), scales by alpha * 2^(e_i + f_j + 2 - 14 -
// 8 d1) and accumulates into C in FP64; units run from the smallest weight
// up, the first one adding beta*C0.
// Warps: 0 TMA producer, 1 TMEM owner / MMA issuer, 2..17 epilogue (four
// warps per TMEM lane quarter, UN/4 columns each). With the 128 x 256 tile a
// unit's two accumulators fill TMEM, so the tensor cores wait while the
// epilogue drains them; the epilogue is written for that latency: 16 warps,
// a per-warp table of the tile's column scales in shared memory, and the
// first chunk's C values requested before the accumulator wait. The
// 128 x 128 tile keeps two sets of accumulators and alternates them, so its
// drain overlaps the next unit's MMAs.
// ------------------------------------------------------------------------------

constexpr int kOzEpiWarps = 16;
constexpr int kOzThreads = 64 + 32 * kOzEpiWarps;
constexpr int kOzColTab = 64 * (8 + 4);             // per epilogue warp: 2^fc (double) and fc (int), 64 columns
// Per tile width UN (256, or 128 for narrow problems): stages of
// (B_{d1-i}, A_i), their bytes, the columns each epilogue warp drains, and
// the dynamic shared memory.
template <int UN>
struct OzCfg {
    static_assert(UN == 256 || UN == 128, "Ozaki tiles are 128 x 256 or 128 x 128");
    static constexpr int ST = UN == 256 ? 4 : 6;
    static_assert(ST <= kMaxStages, "Bar holds kMaxStages stages");
    static constexpr int BTILE = UN * kRowBytes;
    static constexpr int STAGE = kATile + BTILE;  // 48 KiB / 32 KiB
    static constexpr int CW = UN / 4;             // four epilogue warps per TMEM lane quarter
    static constexpr int SMEM = ST * STAGE + 256 + kOzEpiWarps * kOzColTab + 1024;
    // accumulator sets of 2 x UN columns in TMEM's 512: the 128-wide tile
    // keeps two, so the MMAs of the next unit run while this one drains
    static constexpr int NBUF = 512 / (2 * UN);
};
// Tile rows per rasterisation group. A wave of 148 tiles walks R row panels
// of A and C column panels of B, each once per diagonal-pair unit; B panels
// (256 columns) are twice the A panels (128 rows), so R ~ 2C (16 x ~9)
// moves fewer digit-plane bytes through L2 than the 8 x ~18 of the plain
// kernels.
constexpr int kOzRaster = 16;

struct OzParams {
    int m, n, k;
    int tiles_m, tiles_n, num_tiles;
    int num_kt;        // 128-byte K tiles
    int slices;
    int kt_per_chunk;  // exact-INT32 K chunk
    int kchunks;
    int beta_mode;
    double alpha, beta;
    double* c;
    size_t ldc;
    const double* cin;  // C0, read for beta != 0: c itself, or a separate input with c's leading dimension
    const int* row_exp;
    const int* col_exp;
    uint32_t* err;
    // Split tail: the last tail_tiles tiles (in raster order) run as one work
    // item per (tile, unit). Such an item's epilogue writes the unit's exact
    // FP64 terms to its own plane of ws (kUM * un doubles per tile and unit,
    // element (row, col) of the tile at row + col * kUM), and
    // ozaki_reduce_kernel folds the planes into C in unit order afterwards:
    // the same operations as the fused epilogue, so the same bits. Used where
    // whole tiles would leave SMs idle (a partial last wave, or fewer tiles
    // than SMs). 0: every tile fused.
    double* ws;
    int tail_tiles;
    int un;  // tile width (256 or 128): the split tail's plane size and the reduce kernel's tiling
};

// 2^x for x in [-1022, 1023]
__device__ __forceinline__ double pow2_normal(int x) {
    return __longlong_as_double(static_cast<long long>(x + 1023) << 52);
}

// v * 2^x: one multiply by an exactly representable power of two (the same
// single rounding as scalbn), scalbn only where 2^x is not a double.
__device__ __forceinline__ double scale_pow2(double v, int x) {
    if (x >= -1022 && x <= 1023) return v * __longlong_as_double(static_cast<long long>(x + 1023) << 52);
    if (x >= -1074 && x < -1022) return v * __longlong_as_double(1LL << (x + 1074));
    return scalbn(v, x);
}

// unit u (0-based) of a chunk covers diagonals d0 and d1 = d0 + 1 (d1 < 0
// when absent); units go from the highest diagonals down.
__host__ __device__ __forceinline__ void oz_unit(int slices, int u, int& d0, int& d1) {
    const int units = (slices + 1) / 2;
    d0 = 2 * (units - 1 - u);
    d1 = (d0 + 1 < slices) ? d0 + 1 : -1;
}

// Work item -> tile t and units [u_lo, u_hi). Items below the fused count are
// whole tiles (tt = -1). The others are single units of the tail tiles (tt:
// index among them), ranked by cost -- pair 0 of a chunk, the highest
// diagonals, has the most products -- and dealt to the CTAs in a snake, so
// a CTA that took an expensive unit in one pass takes a cheap one in the
// next. G is the grid size; any G gives a bijection, the balance assumes the
// fused count is a multiple of G.
__host__ __device__ __forceinline__ void oz_item(int num_tiles, int tail_tiles, int kchunks, int upc, int G,
                                                 int item, int& t, int& u_lo, int& u_hi, int& tt) {
    const int fused = num_tiles - tail_tiles;
    if (item < fused) {
        t = item;
        u_lo = 0;
        u_hi = kchunks * upc;
        tt = -1;
        return;
    }
    const int j = item - fused;
    const int total = tail_tiles * kchunks * upc;
    const int pass = j / G, q = j - pass * G;
    const int len = (total - pass * G < G) ? total - pass * G : G;
    const int rank = (pass & 1) ? pass * G + (len - 1 - q) : j;
    const int per_pair = tail_tiles * kchunks;
    const int pair = rank / per_pair, rest = rank - pair * per_pair;
    const int chunk = rest / tail_tiles;
    tt = rest - chunk * tail_tiles;
    t = fused + tt;
    u_lo = chunk * upc + pair;
    u_hi = u_lo + 1;
}

// One problem of a grouped Ozaki launch: its digit-plane tensor maps (TMA
// reads them from global memory: 64-byte aligned) and its parameters.
struct alignas(64) OzGroupEntry {
    CUtensorMap tmA, tmB;
    OzParams p;
};

// One work item as a CTA sees it: its problem, tile and units (oz_item).
struct OzWork {
    const OzParams* p;
    const CUtensorMap* ta;
    const CUtensorMap* tb;
    int t, u_lo, u_hi, tt;
};

// Work of the single-problem kernel: whole tiles, then the split tail's
// units (oz_item).
struct OzSingleSrc {
    const OzParams* p;
    const CUtensorMap* ta;
    const CUtensorMap* tb;
    __device__ __forceinline__ uint32_t* err() const { return p->err; }
    __device__ __forceinline__ int items() const {
        const int units = p->kchunks * ((p->slices + 1) / 2);
        return p->num_tiles + p->tail_tiles * (units - 1);
    }
    __device__ __forceinline__ OzWork get(int item) const {
        OzWork w{p, ta, tb, 0, 0, 0, -1};
        oz_item(p->num_tiles, p->tail_tiles, p->kchunks, (p->slices + 1) / 2, gridDim.x, item, w.t, w.u_lo, w.u_hi,
                w.tt);
        return w;
    }
};

// Work of the grouped kernel: item i is one whole tile (fused epilogue, every
// unit) of problem j, where starts[j] <= i < starts[j+1]. The host orders the
// problems by the cost of one tile, largest first, so the CTAs' strided walk
// over the items deals the long tiles out first.
struct OzGroupSrc {
    const OzGroupEntry* tab;
    const int* starts;
    int nprob;
    uint32_t* error;
    __device__ __forceinline__ uint32_t* err() const { return error; }
    __device__ __forceinline__ int items() const { return __ldg(starts + nprob); }
    __device__ __forceinline__ OzWork get(int item) const {
        int lo = 0, hi = nprob - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(starts + mid) <= item) lo = mid;
            else hi = mid - 1;
        }
        const OzGroupEntry* g = tab + lo;
        OzWork w{&g->p, &g->tmA, &g->tmB, item - __ldg(starts + lo), 0, 0, -1};
        w.u_hi = g->p.kchunks * ((g->p.slices + 1) / 2);
        return w;
    }
};

template <int UN, class Src>
__device__ __forceinline__ void ozaki_body(const Src& src) {
    using Cfg = OzCfg<UN>;
    constexpr int ST = Cfg::ST, CW = Cfg::CW, NCH = CW / 8;
    constexpr int TILE_ELEMS = kUM * UN;
    constexpr int KSTEPS = 4;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    Bar* bar = reinterpret_cast<Bar*>(smem + ST * Cfg::STAGE);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; ++s) {
            mbar_init(&bar->full[s], 1);
            mbar_init(&bar->empty[s], 1);
        }
        for (int b = 0; b < Cfg::NBUF; ++b) {
            mbar_init(&bar->acc_full[b], 1);
            mbar_init(&bar->acc_empty[b], kOzEpiWarps);
        }
        mbar_init(&bar->drain, 1);
        fence_barrier_init();
    }
    if (warp == 1) {
        tmem_alloc(&bar->tmem_base, 512);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = bar->tmem_base;
    const int items = src.items();
    uint32_t* const err = src.err();
    bool ok = true;

    if (warp == 0 && lane == 0) {
        // ------------------------------ TMA producer ------------------------------
        uint32_t it = 0;
        const CUtensorMap* fetched = nullptr;
        for (int item = blockIdx.x; ok && item < items; item += gridDim.x) {
            const OzWork w = src.get(item);
            const OzParams& p = *w.p;
            if (w.ta != fetched) {
                prefetch_tmap(w.ta);
                prefetch_tmap(w.tb);
                fetched = w.ta;
            }
            const int upc = (p.slices + 1) / 2;
            int tm, tn;
            raster_tile<kOzRaster>(w.t, p.tiles_m, p.tiles_n, tm, tn);
            const int m0 = tm * kUM, n0 = tn * UN;
            for (int u = w.u_lo; ok && u < w.u_hi; ++u) {
                int d0, d1;
                oz_unit(p.slices, u % upc, d0, d1);
                const int kt0 = (u / upc) * p.kt_per_chunk, kt1 = min(p.num_kt, kt0 + p.kt_per_chunk);
                const int top = d1 >= 0 ? d1 : d0;
                for (int kt = kt0; ok && kt < kt1; ++kt) {
                    const int k0 = kt * 128;
                    for (int i = top; ok && i >= 0; --i, ++it) {  // stage: A_i and B_{top-i}
                        const int s = it % ST;
                        if (it >= ST && !mbar_wait(&bar->empty[s], ((it / ST) - 1) & 1, err, 0x301)) {
                            ok = false;
                            break;
                        }
                        uint8_t* sb = smem + s * Cfg::STAGE;
                        uint8_t* sa = sb + Cfg::BTILE;
                        mbar_arrive_expect_tx(&bar->full[s], Cfg::BTILE + kATile);
                        tma_load_3d(sb, w.tb, &bar->full[s], k0, n0, top - i);
                        tma_load_3d(sa, w.ta, &bar->full[s], k0, m0, i);
                    }
                }
            }
        }
        if (!ok) {
            const uint32_t first = it > (uint32_t)ST ? it - ST : 0;
            for (uint32_t j = first; j < it; ++j) mbar_wait_drain(&bar->full[j % ST], (j / ST) & 1);
        }
    } else if (warp == 1 && lane == 0) {
        // ------------------------------ MMA issuer ------------------------------
        uint32_t it = 0, uc = 0;
        for (int item = blockIdx.x; ok && item < items; item += gridDim.x) {
            const OzWork w = src.get(item);
            const OzParams& p = *w.p;
            const int upc = (p.slices + 1) / 2;
            for (int u = w.u_lo; ok && u < w.u_hi; ++u, ++uc) {
                int d0, d1;
                oz_unit(p.slices, u % upc, d0, d1);
                const int kt0 = (u / upc) * p.kt_per_chunk, kt1 = min(p.num_kt, kt0 + p.kt_per_chunk);
                const int bsel = static_cast<int>(uc % Cfg::NBUF);
                if (uc >= static_cast<uint32_t>(Cfg::NBUF) &&
                    !mbar_wait(&bar->acc_empty[bsel], ((uc / Cfg::NBUF) - 1) & 1, err, 0x302)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                // S_top (d1, or d0 alone) at acc + UN for a pair, acc otherwise;
                // S_d0 of a pair at acc (the epilogue's layout)
                const uint32_t acc = tmem_base + bsel * (2 * UN);
                const bool pair = d1 >= 0;
                const int top = pair ? d1 : d0;
                const uint32_t acc_top = pair ? acc + UN : acc;
                constexpr uint32_t idesc = umma_idesc(2, 1, kUM, UN);  // s32 <- s8 x s8
                uint32_t f_top = 0, f_low = 0;
                for (int kt = kt0; ok && kt < kt1; ++kt) {
                    int prev_s = -1;
                    for (int i = top; ok && i >= 0; --i, ++it) {
                        const int s = it % ST;
                        if (!mbar_wait(&bar->full[s], (it / ST) & 1, err, 0x303)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t sb = smem_u32(smem + s * Cfg::STAGE);
                        const uint32_t sa = sb + Cfg::BTILE;
                        const bool low = pair && prev_s >= 0;  // A_i x B_{d0-i}: the previous stage's B
                        const uint32_t pb = low ? smem_u32(smem + prev_s * Cfg::STAGE) : 0u;
#pragma unroll
                        for (int kk = 0; kk < KSTEPS; ++kk) {
                            const uint64_t ad = sw128_kmajor_desc(sa) + 2 * kk;
                            umma_i8(acc_top, ad, sw128_kmajor_desc(sb) + 2 * kk, idesc, f_top);
                            f_top = 1;
                            if (low) {
                                umma_i8(acc, ad, sw128_kmajor_desc(pb) + 2 * kk, idesc, f_low);
                                f_low = 1;
                            }
                        }
                        // the previous stage is consumed once these MMAs complete;
                        // without a pair the stage itself is
                        if (pair) {
                            if (prev_s >= 0) tc_commit(&bar->empty[prev_s]);
                            prev_s = s;
                        } else {
                            tc_commit(&bar->empty[s]);
                        }
                    }
                    if (pair && prev_s >= 0) tc_commit(&bar->empty[prev_s]);
                }
                if (ok) tc_commit(&bar->acc_full[bsel]);
            }
        }
        tc_commit(&bar->drain);
        mbar_wait_drain(&bar->drain, 0);
    } else if (warp >= 2) {
        // ------------------------------ epilogue ------------------------------
        const int quarter = warp & 3;      // TMEM lanes 32*quarter.. (the warp's rank in its warpgroup)
        const int cq = (warp - 2) >> 2;    // columns CW*cq .. CW*cq+CW-1 of the tile
        const int row_in_tile = quarter * 32 + lane;
        // this warp's column table: 2^fc where fc is in [-1022, 1023], else 0
        // (a zero or absent column, or an exponent outside the normal range),
        // and fc itself
        uint8_t* tab = smem + ST * Cfg::STAGE + 256 + (warp - 2) * kOzColTab;
        double* col_scale = reinterpret_cast<double*>(tab);
        int* col_e = reinterpret_cast<int*>(tab + 64 * sizeof(double));
        const uint32_t lanebase = tmem_base + (static_cast<uint32_t>(quarter * 32) << 16);
        // C between the units of a tile stays in L2 (the tiles in flight hold
        // ~38 MB of it) while the digit planes stream past; C0's read and the
        // last unit's write are the tile's final touches
        uint32_t uc = 0;
        for (int item = blockIdx.x; ok && item < items; item += gridDim.x) {
            const OzWork w = src.get(item);
            const OzParams& p = *w.p;
            const int upc = (p.slices + 1) / 2;
            const int units = p.kchunks * upc;
            const bool split = w.tt >= 0;
            int tm, tn;
            raster_tile<kOzRaster>(w.t, p.tiles_m, p.tiles_n, tm, tn);
            const int m0 = tm * kUM, n0 = tn * UN;
            const int r = m0 + row_in_tile;
            const bool row_ok = r < p.m;
            const int er = row_ok ? p.row_exp[r] : kExpSentinel;
            __syncwarp();  // the previous item's reads of the table are done
            // bit j of colmask: column j of the warp's CW has a nonzero table
            // scale (so it also lies inside C)
            uint64_t colmask = 0;
#pragma unroll
            for (int h = 0; h < CW / 32; ++h) {
                const int j = lane + 32 * h;
                const int col = n0 + cq * CW + j;
                const int fc = col < p.n ? __ldg(p.col_exp + col) : kExpSentinel;
                const bool normal = fc != kExpSentinel && fc >= -1022 && fc <= 1023;
                col_e[j] = fc;
                col_scale[j] = normal ? pow2_normal(fc) : 0.0;
                colmask |= static_cast<uint64_t>(__ballot_sync(0xffffffffu, normal)) << (32 * h);
            }
            __syncwarp();
            double* const crow = p.c + (row_ok ? r : 0);
            const double* const c0row = p.cin + (row_ok ? r : 0);
            const size_t ldc = p.ldc;
            for (int u = w.u_lo; ok && u < w.u_hi; ++u, ++uc) {
                int d0, d1;
                oz_unit(p.slices, u % upc, d0, d1);
                const bool first_unit = (u == 0);
                const uint64_t pol_ld = first_unit ? l2_evict_first_policy() : l2_evict_last_policy();
                const uint64_t pol_st = (u == units - 1) ? l2_evict_first_policy() : l2_evict_last_policy();
                // the first unit reads C0 (beta * C0), the later ones the running sum in C
                const double* const srow = first_unit ? c0row : crow;
                // digits of both operands are scaled by 2^-(e+1): weight 2^-(14+8d) per diagonal
                const int wexp = 14 + 8 * (d1 >= 0 ? d1 : d0) - 2;
                // the row's part of the scale first: sv * 2^(er - wexp) is exact
                // (a nonzero integer below 2^40 times a power of two, landing in
                // [2^-1022, 2^1000)), so the second multiply, by 2^fc, is the only
                // rounding -- the same single rounding as scale_pow2(sv, er+fc-wexp)
                const int ra = er - wexp;
                const bool row_fast = er != kExpSentinel && ra >= -1022 && ra <= 960;
                const double rs = row_fast ? pow2_normal(ra) : 0.0;
                // C is read (beta*C0 on the first unit, the running sum after)
                // (a split item: the unit's terms go to its workspace plane, C is untouched)
                const bool read_c = !split && (!first_unit || p.beta_mode != 0);
                const bool live = row_ok && (split || !(er == kExpSentinel && !first_unit));
                // every live row of the warp takes the two-multiply scaling
                const bool warp_fast = __all_sync(0xffffffffu, row_fast || !live);
                double* wplane =
                    split ? p.ws + (static_cast<size_t>(w.tt) * units + u) * TILE_ELEMS + row_in_tile : nullptr;
                // chunk ch's C values are requested one chunk ahead (the first
                // chunk's before the accumulator wait), so a chunk's L2 round
                // trip overlaps the previous chunk's arithmetic
                double cv[8];
#pragma unroll
                for (int jj = 0; jj < 8; ++jj) {
                    const int cbase = n0 + cq * CW;
                    cv[jj] = (live && read_c && cbase + jj < p.n)
                                 ? ld_l2hint(srow + static_cast<size_t>(cbase + jj) * ldc, pol_ld) : 0.0;
                }
                const int bsel = static_cast<int>(uc % Cfg::NBUF);
                const uint32_t accbase = lanebase + bsel * (2 * UN);
                {
                    const bool got = mbar_wait(&bar->acc_full[bsel], (uc / Cfg::NBUF) & 1, err, 0x304);
                    if (!__all_sync(0xffffffffu, got)) {  // the whole warp goes on, or the whole warp stops
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                }
#pragma unroll 1
                for (int ch = 0; ch < NCH; ++ch) {
                    // 8 columns at a time
                    const int j0 = ch * 8;
                    const int col0 = cq * CW + j0;
                    const int cbase = n0 + col0;
                    double* const cp = crow + static_cast<size_t>(cbase) * ldc;
                    const double* const sp = srow + static_cast<size_t>(cbase) * ldc;
                    double cn[8];
#pragma unroll
                    for (int jj = 0; jj < 8; ++jj)
                        cn[jj] = (live && read_c && ch < NCH - 1 && cbase + 8 + jj < p.n)
                                     ? ld_l2hint(sp + static_cast<size_t>(8 + jj) * ldc, pol_ld) : 0.0;
                    uint32_t v0[8], v1[8];
                    tmem_ld8(accbase + col0, v0);
                    if (d1 >= 0) tmem_ld8(accbase + UN + col0, v1);
                    tmem_ld_wait();
                    if (live) {
                        if (warp_fast && ((colmask >> j0) & 0xffu) == 0xffu) {
                            // branch-free: eight independent chains the compiler can interleave
#pragma unroll
                            for (int jj = 0; jj < 8; ++jj) {
                                double sv = static_cast<double>(static_cast<int32_t>(v0[jj]));
                                if (d1 >= 0) sv = fma(sv, 256.0, static_cast<double>(static_cast<int32_t>(v1[jj])));
                                const double term = (sv * rs) * col_scale[j0 + jj];
                                if (wplane) {
                                    wplane[static_cast<size_t>(col0 + jj) * kUM] = term;
                                } else {
                                    double acc = cv[jj];
                                    if (first_unit && p.beta_mode == 2) acc = p.beta * acc;
                                    st_l2hint(cp + static_cast<size_t>(jj) * ldc, fma(p.alpha, term, acc), pol_st);
                                }
                            }
                        } else {
#pragma unroll
                            for (int jj = 0; jj < 8; ++jj) {
                                if (cbase + jj < p.n) {
                                    double sv = static_cast<double>(static_cast<int32_t>(v0[jj]));
                                    if (d1 >= 0)
                                        sv = fma(sv, 256.0, static_cast<double>(static_cast<int32_t>(v1[jj])));
                                    const double cs = col_scale[j0 + jj];
                                    double term;
                                    if (row_fast && cs != 0.0) {
                                        term = (sv * rs) * cs;
                                    } else {
                                        const int fc = col_e[j0 + jj];
                                        term = (er != kExpSentinel && fc != kExpSentinel)
                                                   ? scale_pow2(sv, er + fc - wexp) : 0.0;
                                    }
                                    if (wplane) {
                                        wplane[static_cast<size_t>(col0 + jj) * kUM] = term;
                                    } else {
                                        double acc = cv[jj];
                                        if (first_unit && p.beta_mode == 2) acc = p.beta * acc;
                                        st_l2hint(cp + static_cast<size_t>(jj) * ldc, fma(p.alpha, term, acc),
                                                  pol_st);
                                    }
                                }
                            }
                        }
                    }
#pragma unroll
                    for (int jj = 0; jj < 8; ++jj) cv[jj] = cn[jj];
                }
                if (!ok) break;
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&bar->acc_empty[bsel]);
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, 512);
    }
}

template <int UN>
__global__ void __launch_bounds__(kOzThreads, 1)
    ozaki_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                      const __grid_constant__ OzParams p) {
    ozaki_body<UN>(OzSingleSrc{&p, &tmA, &tmB});
}

// Many f64 problems in one persistent launch (the serving loop's Ozaki
// batches): the same tiles and epilogue as ozaki_gemm_kernel, whole tiles only.
template <int UN>
__global__ void __launch_bounds__(kOzThreads, 1)
    ozaki_grouped_kernel(const OzGroupEntry* __restrict__ tab, const int* __restrict__ starts, int nprob,
                         uint32_t* err) {
    ozaki_body<UN>(OzGroupSrc{tab, starts, nprob, err});
}

// Split tail: C of the tail tiles = the fused epilogue's sequence over the
// unit planes, element by element -- acc = beta-pass(C0) for the first unit,
// then acc = fma(alpha, term_u, acc) in unit order; rows with a zero exponent
// take only the first unit's step, as in the fused epilogue. Consecutive
// threads take consecutive rows of a tile column (coalesced C and planes).
__global__ void ozaki_reduce_kernel(const OzParams p, int units) {
    const int fused = p.num_tiles - p.tail_tiles;
    const int tile_elems = kUM * p.un;
    const size_t total = static_cast<size_t>(p.tail_tiles) * tile_elems;
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int tt = static_cast<int>(idx / tile_elems);
        const int local = static_cast<int>(idx - static_cast<size_t>(tt) * tile_elems);
        int tm, tn;
        raster_tile<kOzRaster>(fused + tt, p.tiles_m, p.tiles_n, tm, tn);
        const int r = tm * kUM + local % kUM, col = tn * p.un + local / kUM;
        if (r >= p.m || col >= p.n) continue;
        double* cp = p.c + r + static_cast<size_t>(col) * p.ldc;
        const double c0 = p.beta_mode ? p.cin[r + static_cast<size_t>(col) * p.ldc] : 0.0;
        double acc = 0.0;
        if (p.beta_mode == 1) acc = c0;
        else if (p.beta_mode == 2) acc = p.beta * c0;
        const double* w = p.ws + static_cast<size_t>(tt) * units * tile_elems + local;
        const int last = (p.row_exp[r] == kExpSentinel) ? 1 : units;
        for (int u = 0; u < last; ++u) acc = fma(p.alpha, w[static_cast<size_t>(u) * tile_elems], acc);
        *cp = acc;
    }
}

// ------------------------------------------------------------------------------
// Pre-pass kernels. An operand is viewed as R x K with element (r, p) at
// x[r*rs + p*ps]; outputs are K-major planes [plane][R][kp] (kp = padded K).
// ------------------------------------------------------------------------------

__device__ __forceinline__ int frexp_exp(double x) {
    // exponent e with |x| in [2^(e-1), 2^e); x != 0
    const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(x));
    const int f = static_cast<int>((bits >> 52) & 0x7FF);
    if (f != 0) return f - 1022;
    int e;
    frexp(x, &e);
    return e;
}

__global__ void fill_int_kernel(int* p, int n, int v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

// e[r] = max over p of frexp_exp(x(r,p)) (kExpSentinel if the row is zero);
// atomicMax merges the K slabs. frexp_exp is non-decreasing in |x|, and the
// bit patterns of non-negative doubles (subnormals, inf and NaN included)
// order as their values, so the row's exponent is frexp_exp of the largest
// |x| bit pattern: one mask and one 64-bit max per element (0 for a zero row).
__device__ __forceinline__ long long abs_bits(double v) {
    return __double_as_longlong(v) & 0x7FFFFFFFFFFFFFFFLL;
}
// K-contiguous view: one warp per row (8 rows per 256-thread block), a
// 1024-wide K slab per block row by.
__device__ __forceinline__ void row_exp_kcontig(const double* __restrict__ x, size_t rs, int R, int K,
                                                int* __restrict__ e, int bx, int by) {
    const int r = bx * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (r >= R) return;
    const int p0 = by * 1024, p1 = min(K, p0 + 1024);
    long long best = 0;
#pragma unroll 8
    for (int q = p0 + (threadIdx.x & 31); q < p1; q += 32) best = max(best, abs_bits(x[static_cast<size_t>(r) * rs + q]));
    for (int o = 16; o; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0 && best != 0) atomicMax(e + r, frexp_exp(__longlong_as_double(best)));
}
// R-contiguous view: one thread per row (coalesced across the warp), a
// 32-wide K slab per block row by so the grid covers the whole matrix.
__device__ __forceinline__ void row_exp_rcontig(const double* __restrict__ x, size_t ps, int R, int K,
                                                int* __restrict__ e, int bx, int by) {
    const int r = bx * blockDim.x + threadIdx.x;
    if (r >= R) return;
    const int p0 = by * 32, p1 = min(K, p0 + 32);
    long long best = 0;
#pragma unroll 8
    for (int q = p0; q < p1; ++q) best = max(best, abs_bits(x[r + static_cast<size_t>(q) * ps]));
    if (best != 0) atomicMax(e + r, frexp_exp(__longlong_as_double(best)));
}
__global__ void row_exp_kcontig_kernel(const double* __restrict__ x, size_t rs, int R, int K,
                                       int* __restrict__ e) {
    row_exp_kcontig(x, rs, R, K, e, blockIdx.x, blockIdx.y);
}
__global__ void row_exp_rcontig_kernel(const double* __restrict__ x, size_t ps, int R, int K,
                                       int* __restrict__ e) {
    row_exp_rcontig(x, ps, R, K, e, blockIdx.x, blockIdx.y);
}

constexpr int kTile = 64;

// Load a 64 x 64 tile of the R x K view into shared memory (coalesced along
// the view's contiguous dimension); out-of-range elements read as 0. Blocks
// of 256 threads: each thread issues its 16 loads before the first store, so
// the loads are in flight together instead of one latency each.
constexpr int kTileThreads = 256;
template <typename T>
__device__ __forceinline__ void load_tile(const T* __restrict__ x, size_t rs, size_t ps, int R, int K,
                                          int r0, int p0, T (*tile)[kTile + 1]) {
    constexpr int PER = kTile * kTile / kTileThreads;
    const bool kcontig = (ps == 1);
    T v[PER];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const int idx = threadIdx.x + i * kTileThreads;
        const int a = idx % kTile, b = idx / kTile;
        const int r = kcontig ? b : a;
        const int q = kcontig ? a : b;
        v[i] = (r0 + r < R && p0 + q < K) ? x[static_cast<size_t>(r0 + r) * rs + static_cast<size_t>(p0 + q) * ps]
                                          : T(0);
    }
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const int idx = threadIdx.x + i * kTileThreads;
        const int a = idx % kTile, b = idx / kTile;
        tile[kcontig ? b : a][kcontig ? a : b] = v[i];
    }
}

// Ozaki slicing. With e[r] the row exponent (|x| < 2^e), y = x * 2^-(e+1)
// lies in (-1/2, 1/2). For s slices let N = 7 + 8(s-1) and
//   Y = floor(y * 2^N) = floor(x * 2^(N-e-1)),
// computed exactly from x's bits (x = m * 2^q with an integer m of at most
// 53 bits: Y = m << (q+N-e-1), or an arithmetic right shift -- a floor --
// when that exponent is negative; |Y| < 2^(N-1) <= 2^94 fits an __int128).
// Its base-256 digits, the top one signed, are
//   d_0 = floor(y * 2^7) in [-64, 63],  d_t = floor(y * 2^(7+8t)) mod 256,
// which are then balanced from the least significant up: d_t >= 128 becomes
// d_t - 256 with a carry of 1 into d_{t-1} (d_0 <= 64 after the carry). The
// result: signed 8-bit digits with y = sum_t d_t 2^-(7+8t) + rem,
// 0 <= rem < 2^-N, and tail digits symmetric about zero, so the dropped cross
// products do not accumulate a bias along K. No floating-point rounding
// occurs anywhere in the extraction (slices: 2 to 12).

// floor(x * 2^n) for |x * 2^n| < 2^94 (Int = __int128) or < 2^62 (long long)
template <typename Int>
__device__ __forceinline__ Int floor_scaled(double x, int n) {
    const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(x));
    const int ex = static_cast<int>((bits >> 52) & 0x7FF);
    long long m = static_cast<long long>(bits & ((1ull << 52) - 1));
    if (ex != 0) m |= (1ll << 52);
    if (m == 0) return 0;
    if (bits >> 63) m = -m;
    const int sh = (ex == 0 ? 1 : ex) - 1075 + n;  // x = m * 2^((ex|1) - 1075)
    if (sh >= 0) return static_cast<Int>(m) << sh;
    if (sh <= -63) return m < 0 ? -1 : 0;
    return static_cast<Int>(m >> (-sh));  // arithmetic shift: floor
}

// S slices known at compile time: up to 8 digits the integer fits 64 bits.
// One 64 x 64 tile of the R x K view per 256-thread block: K tile bx, row
// tile by.
// The slice pass's tile: rows of kSliceLD doubles (1 mod 16), and every
// 16-column group shifted by 4 more, so that the reads below (a half-warp on
// rows r and groups c, tid = 4r + c) and the loads' stores both touch
// distinct banks; with 65-double rows the four groups of a row shared theirs.
constexpr int kSliceLD = 81;
__device__ __forceinline__ int slice_col(int col) { return col + (col >> 4) * 4; }

__device__ __forceinline__ void load_tile_sliced(const double* __restrict__ x, size_t rs, size_t ps, int R, int K,
                                                 int r0, int p0, double (*tile)[kSliceLD]) {
    constexpr int PER = kTile * kTile / kTileThreads;
    const bool kcontig = (ps == 1);
    double v[PER];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const int idx = threadIdx.x + i * kTileThreads;
        const int a = idx % kTile, b = idx / kTile;
        const int r = kcontig ? b : a;
        const int q = kcontig ? a : b;
        v[i] = (r0 + r < R && p0 + q < K) ? x[static_cast<size_t>(r0 + r) * rs + static_cast<size_t>(p0 + q) * ps]
                                          : 0.0;
    }
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const int idx = threadIdx.x + i * kTileThreads;
        const int a = idx % kTile, b = idx / kTile;
        if (kcontig) tile[b][slice_col(a)] = v[i];
        else         tile[a][slice_col(b)] = v[i];
    }
}

template <int S>
__device__ __forceinline__ void ozaki_slice_tile(const double* __restrict__ x, size_t rs, size_t ps, int R, int K,
                                                 const int* __restrict__ e, int8_t* __restrict__ out, size_t kp,
                                                 size_t plane, int bx, int by) {
    using Int = typename std::conditional<(S <= 8), long long, __int128>::type;
    constexpr int slices = S;
    __shared__ double tile[kTile][kSliceLD];
    const int r0 = by * kTile, p0 = bx * kTile;
    load_tile_sliced(x, rs, ps, R, K, r0, p0, tile);
    __syncthreads();
    const int r = threadIdx.x >> 2, c = threadIdx.x & 3;  // 64 rows x 4 chunks of 16
    if (r0 + r >= R) return;
    if (p0 + c * 16 >= static_cast<int>(kp)) return;
    const int er = e[r0 + r];
    const int n = 7 + 8 * (slices - 1) - er - 1;  // Y = floor(x * 2^n)
    uint32_t w[S][4];
    if constexpr (S <= 8) {
        // Balancing by bytes: adding 0x80 to each of the S-1 low bytes of Y
        // makes the carries of the loop below (a byte >= 128 becomes byte-256
        // and carries 1 upward); flipping those bytes back (xor 0x80) leaves
        // each balanced digit as a two's-complement byte, and byte S-1 (the
        // top digit, carry included) is already one. So digit t is byte
        // S-1-t of Z = (Y + B) ^ B, and four elements' digit t pack into one
        // word with byte permutes.
        constexpr unsigned long long B = 0x0080808080808080ull >> (8 * (8 - S));
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            uint32_t lo[4], hi[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const long long Y = (er == kExpSentinel) ? 0LL : floor_scaled<long long>(tile[r][slice_col(c * 16 + g * 4 + q)], n);
                const unsigned long long Z = (static_cast<unsigned long long>(Y) + B) ^ B;
                lo[q] = static_cast<uint32_t>(Z);
                hi[q] = static_cast<uint32_t>(Z >> 32);
            }
#pragma unroll
            for (int t = 0; t < S; ++t) {
                const int b = S - 1 - t;  // byte of Z holding digit t
                const uint32_t* src = b < 4 ? lo : hi;
                const uint32_t sel = static_cast<uint32_t>((b & 3) | (((b & 3) + 4) << 4));
                const uint32_t x01 = __byte_perm(src[0], src[1], sel);
                const uint32_t x23 = __byte_perm(src[2], src[3], sel);
                w[t][g] = __byte_perm(x01, x23, 0x5410);
            }
        }
    } else {
#pragma unroll
    for (int t = 0; t < S; ++t) w[t][0] = w[t][1] = w[t][2] = w[t][3] = 0u;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const Int Y = (er == kExpSentinel) ? Int(0) : floor_scaled<Int>(tile[r][slice_col(c * 16 + i)], n);
        int d[S];
#pragma unroll
        for (int t = 0; t < S; ++t) {
            const int sh = 8 * (S - 1 - t);
            d[t] = (t == 0) ? static_cast<int>(Y >> sh) : static_cast<int>((Y >> sh) & 0xFF);
        }
#pragma unroll
        for (int t = S - 1; t >= 1; --t) {
            if (d[t] >= 128) {
                d[t] -= 256;
                d[t - 1] += 1;
            }
        }
#pragma unroll
        for (int t = 0; t < S; ++t) w[t][i >> 2] |= (static_cast<uint32_t>(d[t]) & 0xFFu) << (8 * (i & 3));
    }
    }
    const size_t off = static_cast<size_t>(r0 + r) * kp + p0 + c * 16;
#pragma unroll
    for (int t = 0; t < S; ++t)
        *reinterpret_cast<uint4*>(out + t * plane + off) = make_uint4(w[t][0], w[t][1], w[t][2], w[t][3]);
}

template <int S>
__global__ void __launch_bounds__(256) ozaki_slice_kernel(const double* __restrict__ x, size_t rs, size_t ps,
                                                          int R, int K, const int* __restrict__ e,
                                                          int8_t* __restrict__ out, size_t kp, size_t plane) {
    ozaki_slice_tile<S>(x, rs, ps, R, K, e, out, kp, plane, blockIdx.x, blockIdx.y);
}

// ---- grouped pre-pass: one launch per pass over every operand of a batch ------

// One operand of a grouped Ozaki launch, viewed as R x K (element (r, p) at
// x[r*rs + p*ps]): its exponents e[R] and digit planes out[slices][R][kp].
// exp_blocks / slice_blocks: the blocks it takes in each pass (the grid's
// blocks are dealt to operands by the prefix sums exp_start / slice_start).
struct OzOperand {
    const double* x;
    size_t rs, ps;
    int R, K;
    int* e;
    int8_t* out;
    size_t kp, plane;
    int exp_gx, slice_gx;  // blocks along R (exponent pass) / along K (slice pass)
    int exp_start, slice_start;
};

__device__ __forceinline__ int oz_find_operand(const OzOperand* ops, int nops, int b, bool slice) {
    int lo = 0, hi = nops - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((slice ? ops[mid].slice_start : ops[mid].exp_start) <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// The exponent pass of every operand (grid = total exponent blocks; e
// pre-filled with the zero-row sentinel).
__global__ void __launch_bounds__(256) ozaki_exp_grouped_kernel(const OzOperand* __restrict__ ops, int nops) {
    const OzOperand& o = ops[oz_find_operand(ops, nops, blockIdx.x, false)];
    const int b = blockIdx.x - o.exp_start;
    const int bx = b % o.exp_gx, by = b / o.exp_gx;
    if (o.ps == 1) row_exp_kcontig(o.x, o.rs, o.R, o.K, o.e, bx, by);
    else           row_exp_rcontig(o.x, o.ps, o.R, o.K, o.e, bx, by);
}

// The slice pass of every operand (grid = total slice tiles).
template <int S>
__global__ void __launch_bounds__(256) ozaki_slice_grouped_kernel(const OzOperand* __restrict__ ops, int nops) {
    const OzOperand& o = ops[oz_find_operand(ops, nops, blockIdx.x, true)];
    const int b = blockIdx.x - o.slice_start;
    ozaki_slice_tile<S>(o.x, o.rs, o.ps, o.R, o.K, o.e, o.out, o.kp, o.plane, b % o.slice_gx, b / o.slice_gx);
}

// Host dispatch on the slice count (2 .. 12).
void launch_ozaki_slices(dim3 grid, cudaStream_t st, const double* x, size_t rs, size_t ps, int R, int K,
                         const int* e, int slices, int8_t* out, size_t kp, size_t plane) {
    switch (slices) {
#define RB_SLICES(S) \
    case S: ozaki_slice_kernel<S><<<grid, 256, 0, st>>>(x, rs, ps, R, K, e, out, kp, plane); break;
        RB_SLICES(2) RB_SLICES(3) RB_SLICES(4) RB_SLICES(5) RB_SLICES(6) RB_SLICES(7) RB_SLICES(8)
        RB_SLICES(9) RB_SLICES(10) RB_SLICES(11) RB_SLICES(12)
#undef RB_SLICES
        default: break;
    }
}

// BF16 split into `planes` (2 or 3) planes: out[0] = bf16(x),
// out[1] = bf16(x - out[0]), out[2] = bf16(x - out[0] - out[1]); every
// difference is exact in FP32.
// One 64 x 64 tile of the R x K view per 256-thread block (K tile bx, row tile by).
// The f32 tile loader with 16-byte loads along the view's contiguous
// dimension when its lines start on 16 bytes (4 loads per thread instead of
// 16); the element loader otherwise.
__device__ __forceinline__ void load_tile_f32(const float* __restrict__ x, size_t rs, size_t ps, int R, int K,
                                              int r0, int p0, float (*tile)[kTile + 1]) {
    const bool kcontig = (ps == 1);
    const size_t ld = kcontig ? rs : ps;         // between the contiguous lines
    const int L = kcontig ? R : K, E = kcontig ? K : R;
    const int l0 = kcontig ? r0 : p0, e0 = kcontig ? p0 : r0;
    if ((!kcontig && rs != 1) || (reinterpret_cast<uintptr_t>(x) & 15) != 0 || (ld & 3) != 0) {
        load_tile<float>(x, rs, ps, R, K, r0, p0, tile);
        return;
    }
    constexpr int PER = kTile * kTile / 4 / kTileThreads;  // float4 per thread
    float4 v[PER];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const int idx = threadIdx.x + i * kTileThreads;
        const int l = l0 + idx / (kTile / 4), e = e0 + 4 * (idx % (kTile / 4));
        const float* src = x + static_cast<size_t>(l) * ld + e;
        if (l < L && e + 3 < E) {
            v[i] = __ldg(reinterpret_cast<const float4*>(src));
        } else {
            v[i].x = (l < L && e < E) ? src[0] : 0.f;
            v[i].y = (l < L && e + 1 < E) ? src[1] : 0.f;
            v[i].z = (l < L && e + 2 < E) ? src[2] : 0.f;
            v[i].w = (l < L && e + 3 < E) ? src[3] : 0.f;
        }
    }
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const int idx = threadIdx.x + i * kTileThreads;
        const int ln = idx / (kTile / 4), el = 4 * (idx % (kTile / 4));
        const float w[4] = {v[i].x, v[i].y, v[i].z, v[i].w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (kcontig) tile[ln][el + j] = w[j];  // row = line, column = k
            else         tile[el + j][ln] = w[j];  // row = contiguous index, column = line (k)
        }
    }
}

// VEC: the 16-byte loader (the single-problem pass over large operands);
// the grouped pass keeps the element loader, whose kernel stays at five CTAs
// per SM
template <bool VEC>
__device__ __forceinline__ void bf16_split_tile(const float* __restrict__ x, size_t rs, size_t ps, int R, int K,
                                                int planes, __nv_bfloat16* __restrict__ out, size_t kp, size_t plane,
                                                int bx, int by) {
    __shared__ float tile[kTile][kTile + 1];
    const int r0 = by * kTile, p0 = bx * kTile;
    if constexpr (VEC) load_tile_f32(x, rs, ps, R, K, r0, p0, tile);
    else               load_tile<float>(x, rs, ps, R, K, r0, p0, tile);
    __syncthreads();
    for (int job = threadIdx.x; job < kTile * 8; job += blockDim.x) {
        const int r = job >> 3, c = job & 7;  // 64 rows x 8 chunks of 8
        if (r0 + r >= R || p0 + c * 8 >= static_cast<int>(kp)) continue;
        __align__(16) __nv_bfloat16 h[3][8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            // hi, then the rest rounded again (mid / lo); the single-problem
            // pass skips the third plane when the 3xBF16 form does not write
            // it (the grouped pass, branch-free, measured faster without the test)
            float v = tile[r][c * 8 + i];
            h[0][i] = __float2bfloat16_rn(v);
            v = v - __bfloat162float(h[0][i]);
            h[1][i] = __float2bfloat16_rn(v);
            if (!VEC || planes > 2) {
                v = v - __bfloat162float(h[1][i]);
                h[2][i] = __float2bfloat16_rn(v);
            }
        }
        const size_t off = static_cast<size_t>(r0 + r) * kp + p0 + c * 8;
        for (int q = 0; q < planes; ++q)
            *reinterpret_cast<uint4*>(out + q * plane + off) = *reinterpret_cast<const uint4*>(h[q]);
    }
}

__global__ void __launch_bounds__(256) bf16_split_kernel(const float* __restrict__ x, size_t rs, size_t ps,
                                                         int R, int K, int planes,
                                                         __nv_bfloat16* __restrict__ out, size_t kp,
                                                         size_t plane) {
    bf16_split_tile<true>(x, rs, ps, R, K, planes, out, kp, plane, blockIdx.x, blockIdx.y);
}

// One operand of a grouped BF16-split launch, viewed as R x K, and its
// planes out[planes][R][kp]; gx K tiles per row tile, `start` its first block.
struct BsOperand {
    const float* x;
    size_t rs, ps;
    int R, K, planes;
    __nv_bfloat16* out;
    size_t kp, plane;
    int gx, start;
};

// The split pass over every operand of a batch (grid = all their tiles).
__global__ void __launch_bounds__(256) bf16_split_grouped_kernel(const BsOperand* __restrict__ ops, int nops) {
    int lo = 0, hi = nops - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (ops[mid].start <= static_cast<int>(blockIdx.x)) lo = mid;
        else hi = mid - 1;
    }
    const BsOperand& o = ops[lo];
    const int b = blockIdx.x - o.start;
    bf16_split_tile<false>(o.x, o.rs, o.ps, o.R, o.K, o.planes, o.out, o.kp, o.plane, b % o.gx, b / o.gx);
}

CUresult make_tmap_planes(CUtensorMap* map, const void* base, CUtensorMapDataType dtype, size_t elem,
                          uint64_t k, uint64_t rows, uint64_t planes, uint64_t kp, uint32_t box_rows) {
    return make_tmap_3d(map, base, dtype, elem, k, rows, planes, kp, kp * rows, kRowBytes / elem,
                        box_rows, 1, true);
}

template <int MODE>
cudaError_t launch_umma(const CUtensorMap& ta, const CUtensorMap& tb, const UParams& p, cudaStream_t st) {
    auto kern = umma_gemm_kernel<MODE>;
    constexpr int smem = umma_smem_bytes<MODE>();
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = p.num_tiles < sms ? p.num_tiles : sms;
    const double work = 2.0 * p.m * p.n * static_cast<double>(p.k) * UCfg<MODE>::NPROD;
    const char* name = (MODE == kModeBf16x3) ? "umma_bf16x3" : "umma_bf16x6";
    KernelTimer tm;
    kernel_timing_begin(name, work, st, &tm);
    kern<<<grid, UCfg<MODE>::THREADS, smem, st>>>(ta, tb, p);
    kernel_timing_end(&tm, st);
    count_launch();
    return cudaGetLastError();
}

inline size_t round_up(size_t x, size_t m) { return (x + m - 1) / m * m; }

// Tensor-pipe throughput probe: one CTA per SM, smem operands filled once
// with a fixed bit pattern, thread 0 issues `iters` back-to-back MMAs
// (M=128, N=256, one 32-byte K step) into a TMEM accumulator.
template <bool I8>
__global__ void __launch_bounds__(128, 1) umma_peak_kernel(int iters, uint32_t* err) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t* done = reinterpret_cast<uint64_t*>(smem + kATile + 256 * kRowBytes);
    uint32_t* tbase = reinterpret_cast<uint32_t*>(done + 1);
    for (int i = threadIdx.x; i < (kATile + 256 * kRowBytes) / 4; i += blockDim.x)
        reinterpret_cast<uint32_t*>(smem)[i] = 0x3c003c00u ^ (i * 2654435761u & 0x00ff00ffu);
    fence_proxy_async_smem();
    if (threadIdx.x == 0) {
        mbar_init(done, 1);
        fence_barrier_init();
    }
    if ((threadIdx.x >> 5) == 0) {
        tmem_alloc(tbase, 256);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tbase;
    if (threadIdx.x == 0) {
        const uint32_t sa = smem_u32(smem), sb = sa + kATile;
        constexpr uint32_t idesc = I8 ? umma_idesc(2, 1, kUM, 256) : umma_idesc(1, 1, kUM, 256);
        for (int i = 0; i < iters; ++i) {
            const uint64_t a = sw128_kmajor_desc(sa) + 2 * (i & 3), b = sw128_kmajor_desc(sb) + 2 * (i & 3);
            if (I8) umma_i8(tmem, a, b, idesc, i > 0);
            else    umma_f16(tmem, a, b, idesc, i > 0);
        }
        tc_commit(done);
        mbar_wait(done, 0, err, 0x2f0);
    }
    tc_fence_before();
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, 256);
    }
}

}  // namespace

double probe_umma_peak(int i8, int iters) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int smem = kATile + 256 * kRowBytes + 64 + 1024;
    auto k0 = umma_peak_kernel<false>;
    auto k1 = umma_peak_kernel<true>;
    auto kern = i8 ? k1 : k0;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return -1.0;
    uint32_t* err = device_error_word();
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    kern<<<sms, 128, smem>>>(iters / 8 + 1, err);  // warm-up
    cudaEventRecord(e0);
    kern<<<sms, 128, smem>>>(iters, err);
    cudaEventRecord(e1);
    count_launch(2);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return -1.0;
    const double per_mma = 2.0 * kUM * 256 * (i8 ? 32 : 16);
    return per_mma * iters * sms / (ms * 1e-3) / 1e12;
}

// op(A) viewed as m x k: (i,p) at A[i + p*lda] (NoTrans) or A[p + i*lda] (Trans).
// op(B)^T viewed as n x k: (j,p) at B[p + j*ldb] (NoTrans) or B[j + p*ldb] (Trans).
static void operand_views(bool ta, bool tb, size_t lda, size_t ldb, size_t& ars, size_t& aps,
                          size_t& brs, size_t& bps) {
    if (!ta) { ars = 1; aps = lda; } else { ars = lda; aps = 1; }
    if (!tb) { brs = ldb; bps = 1; } else { brs = 1; bps = ldb; }
}

// The BF16-split forms split A inside the GEMM (umma_split_fused_kernel) when
// A's rows are contiguous (NoTrans, 16-byte aligned base and column stride)
// and C has at most two 128-wide column tiles, so the f32 tiles TMA brings
// are read about once: there the split pass's read and write of A cost more
// than the GEMM. Wider products keep the two passes (their GEMM is
// compute-bound and the deeper plane ring of the two-pass kernel feeds it
// better).
bool bf16_fused_a(bool ta, int n, const float* A, size_t lda) {
    return !ta && n <= 256 && (reinterpret_cast<uintptr_t>(A) & 15) == 0 && (lda & 3) == 0;
}

template <int MODE>
cudaError_t launch_bf16_fused(const CUtensorMap& ta32, const CUtensorMap& tb, const UParams& p, cudaStream_t st) {
    auto kern = umma_split_fused_kernel<MODE>;
    constexpr int smem = fz_smem_bytes<MODE>();
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = p.num_tiles < sms ? p.num_tiles : sms;
    const char* name = (MODE == kModeBf16x3) ? "umma_bf16x3" : "umma_bf16x6";
    KernelTimer tm;
    kernel_timing_begin(name, 2.0 * p.m * p.n * static_cast<double>(p.k) * UCfg<MODE>::NPROD, st, &tm);
    kern<<<grid, kFzThreads, smem, st>>>(ta32, tb, p);
    kernel_timing_end(&tm, st);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_bf16_split_gemm(int planes, bool ta, bool tb, int m, int n, int k, float alpha,
                                   const float* A, size_t lda, const float* B, size_t ldb, float beta,
                                   float* C, size_t ldc, cudaStream_t st, CUresult* cu_err) {
    constexpr int UN = 128;
    const bool fused = bf16_fused_a(ta, n, A, lda);
    const size_t kp = round_up(static_cast<size_t>(k), 8);  // 16-byte rows of bf16
    const size_t pa = fused ? 0 : static_cast<size_t>(m) * kp, pb = static_cast<size_t>(n) * kp;
    void* buf = nullptr;
    const size_t a_bytes = round_up(planes * pa * sizeof(__nv_bfloat16), 256);
    cudaError_t e = scratch_alloc(&buf, a_bytes + planes * pb * sizeof(__nv_bfloat16), st);
    if (e != cudaSuccess) return e;
    __nv_bfloat16* sa = static_cast<__nv_bfloat16*>(buf);
    __nv_bfloat16* sb = reinterpret_cast<__nv_bfloat16*>(static_cast<uint8_t*>(buf) + a_bytes);
    size_t ars, aps, brs, bps;
    operand_views(ta, tb, lda, ldb, ars, aps, brs, bps);
    const dim3 ga((k + kTile - 1) / kTile, (m + kTile - 1) / kTile);
    const dim3 gb((k + kTile - 1) / kTile, (n + kTile - 1) / kTile);
    if (!fused) {
        bf16_split_kernel<<<ga, 256, 0, st>>>(A, ars, aps, m, k, planes, sa, kp, pa);
        count_launch();
    }
    bf16_split_kernel<<<gb, 256, 0, st>>>(B, brs, bps, n, k, planes, sb, kp, pb);
    count_launch();
    CUtensorMap tma, tmb;
    // fused: A itself as an m x k f32 tensor, 128-row x 64-column boxes
    CUresult r = fused ? make_tmap_2d(&tma, A, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, sizeof(float), m, k, lda, kUM, 64,
                                      false)
                       : make_tmap_planes(&tma, sa, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, k, m, planes, kp, kUM);
    if (r == CUDA_SUCCESS) r = make_tmap_planes(&tmb, sb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, k, n, planes, kp, UN);
    if (r != CUDA_SUCCESS) {
        if (cu_err) *cu_err = r;
        cudaFreeAsync(buf, st);
        return cudaErrorInvalidValue;
    }
    UParams p{};
    p.m = m; p.n = n; p.k = k;
    p.tiles_m = (m + kUM - 1) / kUM;
    p.tiles_n = (n + UN - 1) / UN;
    p.num_tiles = p.tiles_m * p.tiles_n;
    p.num_kt = static_cast<int>((k + 63) / 64);
    p.kt_per_chunk = 2;  // FP32 promotion every 128 elements of K
    p.kchunks = (p.num_kt + p.kt_per_chunk - 1) / p.kt_per_chunk;
    p.beta_mode = (beta == 0.f) ? 0 : (beta == 1.f ? 1 : 2);
    p.alpha_f = alpha; p.beta_f = beta;
    p.c = C; p.ldc = ldc;
    p.cin = C;
    p.err = device_error_word();
    if (fused)
        e = (planes == 2) ? launch_bf16_fused<kModeBf16x3>(tma, tmb, p, st)
                          : launch_bf16_fused<kModeBf16x6>(tma, tmb, p, st);
    else
        e = (planes == 2) ? launch_umma<kModeBf16x3>(tma, tmb, p, st) : launch_umma<kModeBf16x6>(tma, tmb, p, st);
    cudaFreeAsync(buf, st);
    return e;
}

// Many f32 GEMMs in a BF16-split form (planes 2: 3xBF16, 3: BF16X6) with two
// launches for the whole batch: one split pass over every operand, then one
// persistent umma_grouped_kernel over every problem's tiles. C0 of problem i
// comes from cin[i] (leading dimension ldcin[i]) or probs[i].c. Each result
// equals that problem's own rb_sgemm_dev(..., form, ...) bit for bit.
int bf16_grouped_dev(int planes, const rb_gemm_problem* probs, size_t count, const void* const* cin,
                     const size_t* ldcin, cudaStream_t st, int32_t* ce) {
    constexpr int UN = 128;
    struct Job {
        bool ta, tb;
        int m, n, k;
        const float *a, *b;
        size_t lda, ldb;
        float* c;
        const float* c0;
        size_t ldc;
        float alpha, beta;
        size_t kp, off_a, off_b;
        int num_kt;
    };
    std::vector<Job> jobs;
    jobs.reserve(count);
    size_t elems = 0;  // bf16 plane elements, every operand 256-byte aligned
    cudaError_t e = cudaSuccess;
    for (size_t i = 0; i < count; ++i) {
        const rb_gemm_problem& q = probs[i];
        if (q.dtype != 0) return RB_ERR_UNSUPPORTED;
        const int v = validate_problem(q);
        if (v != RB_OK) return v;
        const bool col = q.layout == RB_COL_MAJOR;
        const size_t m = col ? q.m : q.n, n = col ? q.n : q.m;
        if (m == 0 || n == 0) continue;
        if (m > 0x7fffffff || n > 0x7fffffff || q.k > 0x7fffffff) return RB_ERR_INVALID_ARG;
        float* c = static_cast<float*>(q.c);
        const float* c0 = cin ? static_cast<const float*>(cin[i]) : c;
        const size_t ldc0 = cin ? ldcin[i] : q.ldc;
        const float beta = static_cast<float>(q.beta), alpha = static_cast<float>(q.alpha);
        if (beta != 0.f && c0 != c && ldc0 != q.ldc) {
            // the kernels read C0 with C's leading dimension: bring it into C first
            e = cudaMemcpy2DAsync(c, q.ldc * 4, c0, ldc0 * 4, m * 4, n, cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) break;
            c0 = c;
        }
        if (q.k == 0 || alpha == 0.f) {  // C = beta * C0 only (gemm_contig's early out)
            if (beta != 0.f && c0 != c) {
                e = cudaMemcpy2DAsync(c, q.ldc * 4, c0, q.ldc * 4, m * 4, n, cudaMemcpyDeviceToDevice, st);
                if (e != cudaSuccess) break;
            }
            e = launch_scale_c<float>(static_cast<int>(m), static_cast<int>(n), beta, c, q.ldc, st);
            if (e != cudaSuccess) break;
            continue;
        }
        Job j{};
        const bool ta = q.transa != RB_NO_TRANS, tb = q.transb != RB_NO_TRANS;
        j.ta = col ? ta : tb;
        j.tb = col ? tb : ta;
        j.m = static_cast<int>(m);
        j.n = static_cast<int>(n);
        j.k = static_cast<int>(q.k);
        j.a = static_cast<const float*>(col ? q.a : q.b);
        j.b = static_cast<const float*>(col ? q.b : q.a);
        j.lda = col ? q.lda : q.ldb;
        j.ldb = col ? q.ldb : q.lda;
        j.c = c;
        j.c0 = c0;
        j.ldc = q.ldc;
        j.alpha = alpha;
        j.beta = beta;
        j.kp = round_up(q.k, 8);  // 16-byte rows of bf16
        j.num_kt = static_cast<int>((q.k + 63) / 64);
        j.off_a = elems;
        elems += round_up(planes * m * j.kp, 128);
        j.off_b = elems;
        elems += round_up(planes * n * j.kp, 128);
        jobs.push_back(j);
    }
    if (e != cudaSuccess) {
        if (ce) *ce = e;
        return RB_ERR_CUDA;
    }
    if (jobs.empty()) return RB_OK;
    // longest tiles first: the CTAs walk the items with a stride of the grid
    std::stable_sort(jobs.begin(), jobs.end(), [](const Job& x, const Job& y) { return x.num_kt > y.num_kt; });
    const int np = static_cast<int>(jobs.size());
    // device image: [entries][starts][operands], then the planes
    const size_t ent_bytes = round_up(np * sizeof(UGroupEntry), 256);
    const size_t starts_bytes = round_up((np + 1) * sizeof(int), 256);
    const size_t ops_bytes = round_up(2 * np * sizeof(BsOperand), 256);
    const size_t img_bytes = ent_bytes + starts_bytes + ops_bytes;
    uint8_t* mem = nullptr;
    e = scratch_alloc(reinterpret_cast<void**>(&mem), img_bytes + elems * sizeof(__nv_bfloat16), st);
    if (e != cudaSuccess) {
        if (ce) *ce = e;
        if (e == cudaErrorMemoryAllocation) cudaGetLastError();
        return e == cudaErrorMemoryAllocation ? RB_ERR_ALLOC : RB_ERR_CUDA;
    }
    std::vector<uint8_t> img(img_bytes, 0);
    int* starts = reinterpret_cast<int*>(img.data() + ent_bytes);
    BsOperand* ops = reinterpret_cast<BsOperand*>(img.data() + ent_bytes + starts_bytes);
    __nv_bfloat16* dplanes = reinterpret_cast<__nv_bfloat16*>(mem + img_bytes);
    uint32_t* err_word = device_error_word();
    int tiles = 0, split_blocks = 0;
    double work = 0;
    CUresult r = CUDA_SUCCESS;
    for (int i = 0; i < np && r == CUDA_SUCCESS; ++i) {
        const Job& j = jobs[i];
        __nv_bfloat16* sa = dplanes + j.off_a;
        __nv_bfloat16* sb = dplanes + j.off_b;
        size_t ars, aps, brs, bps;
        operand_views(j.ta, j.tb, j.lda, j.ldb, ars, aps, brs, bps);
        const int gx = (j.k + kTile - 1) / kTile;
        const struct { const float* x; size_t rs, ps; int R; __nv_bfloat16* out; } od[2] = {
            {j.a, ars, aps, j.m, sa}, {j.b, brs, bps, j.n, sb}};
        for (int h = 0; h < 2; ++h) {
            BsOperand& o = ops[2 * i + h];
            o.x = od[h].x; o.rs = od[h].rs; o.ps = od[h].ps;
            o.R = od[h].R; o.K = j.k; o.planes = planes;
            o.out = od[h].out;
            o.kp = j.kp; o.plane = static_cast<size_t>(od[h].R) * j.kp;
            o.gx = gx;
            o.start = split_blocks;
            split_blocks += gx * ((o.R + kTile - 1) / kTile);
        }
        UGroupEntry g{};  // 64-byte aligned here; copied into the image below
        r = make_tmap_planes(&g.tmA, sa, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, j.k, j.m, planes, j.kp, kUM);
        if (r == CUDA_SUCCESS)
            r = make_tmap_planes(&g.tmB, sb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, j.k, j.n, planes, j.kp, UN);
        UParams& p = g.p;
        p.m = j.m; p.n = j.n; p.k = j.k;
        p.tiles_m = (j.m + kUM - 1) / kUM;
        p.tiles_n = (j.n + UN - 1) / UN;
        p.num_tiles = p.tiles_m * p.tiles_n;
        p.num_kt = j.num_kt;
        p.kt_per_chunk = 2;  // FP32 promotion every 128 elements of K
        p.kchunks = (p.num_kt + p.kt_per_chunk - 1) / p.kt_per_chunk;
        p.beta_mode = (j.beta == 0.f) ? 0 : (j.beta == 1.f ? 1 : 2);
        p.alpha_f = j.alpha; p.beta_f = j.beta;
        p.c = j.c; p.ldc = j.ldc;
        p.cin = j.c0;
        p.err = err_word;
        std::memcpy(img.data() + i * sizeof(UGroupEntry), &g, sizeof(UGroupEntry));
        starts[i] = tiles;
        tiles += p.num_tiles;
        work += 2.0 * j.m * j.n * static_cast<double>(j.k) * (planes == 2 ? 3 : 6);
    }
    starts[np] = tiles;
    if (r != CUDA_SUCCESS) {
        if (ce) *ce = static_cast<int32_t>(r);
        cudaFreeAsync(mem, st);
        return RB_ERR_CUDA;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = tiles < sms ? tiles : sms;
    // a pageable source: the driver has staged the image when the call returns
    e = cudaMemcpyAsync(mem, img.data(), img_bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        bf16_split_grouped_kernel<<<split_blocks, 256, 0, st>>>(
            reinterpret_cast<const BsOperand*>(mem + ent_bytes + starts_bytes), 2 * np);
        const UGroupEntry* dtab = reinterpret_cast<const UGroupEntry*>(mem);
        const int* dstarts = reinterpret_cast<const int*>(mem + ent_bytes);
        KernelTimer tmr;
        if (planes == 2) {
            constexpr int smem = umma_smem_bytes<kModeBf16x3>();
            static bool attr3 = false;
            if (!attr3) {
                e = cudaFuncSetAttribute(umma_grouped_kernel<kModeBf16x3>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
                attr3 = e == cudaSuccess;
            }
            kernel_timing_begin("umma_bf16x3_grouped", work, st, &tmr);
            if (e == cudaSuccess)
                umma_grouped_kernel<kModeBf16x3><<<grid, UCfg<kModeBf16x3>::THREADS, smem, st>>>(dtab, dstarts, np,
                                                                                                 err_word);
        } else {
            constexpr int smem = umma_smem_bytes<kModeBf16x6>();
            static bool attr6 = false;
            if (!attr6) {
                e = cudaFuncSetAttribute(umma_grouped_kernel<kModeBf16x6>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
                attr6 = e == cudaSuccess;
            }
            kernel_timing_begin("umma_bf16x6_grouped", work, st, &tmr);
            if (e == cudaSuccess)
                umma_grouped_kernel<kModeBf16x6><<<grid, UCfg<kModeBf16x6>::THREADS, smem, st>>>(dtab, dstarts, np,
                                                                                                 err_word);
        }
        kernel_timing_end(&tmr, st);
        count_launch(2);
        if (e == cudaSuccess) e = cudaGetLastError();
    }
    cudaFreeAsync(mem, st);
    if (e != cudaSuccess) {
        if (ce) *ce = e;
        return RB_ERR_CUDA;
    }
    return RB_OK;
}

// Tail tiles to run unit by unit (OzParams::tail_tiles): the tiles of the
// partial last wave (all tiles when there are fewer than SMs), when dealing
// their units as oz_item does finishes clearly before one more whole tile
// would, counting the reduce pass over their planes and C; else 0. Times are
// modelled from the products per unit (a diagonal d has d + 1) at the B200's
// INT8 rate per SM and its copy rate; only their ratio matters.
// Dynamic shared memory of both Ozaki tile widths, set once per process.
cudaError_t ozaki_kernel_attributes() {
    static std::once_flag once;
    static cudaError_t result = cudaSuccess;
    std::call_once(once, [] {
        result = cudaFuncSetAttribute(ozaki_gemm_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      OzCfg<256>::SMEM);
        if (result == cudaSuccess)
            result = cudaFuncSetAttribute(ozaki_gemm_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          OzCfg<128>::SMEM);
        if (result == cudaSuccess)
            result = cudaFuncSetAttribute(ozaki_grouped_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          OzCfg<256>::SMEM);
        if (result == cudaSuccess)
            result = cudaFuncSetAttribute(ozaki_grouped_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          OzCfg<128>::SMEM);
    });
    return result;
}

int ozaki_tail_tiles(int num_tiles, int slices, int kchunks, int k, int sms, int un) {
    const int upc = (slices + 1) / 2;
    if (kchunks != 1 || upc < 2 || sms < 1) return 0;
    const int full = num_tiles / sms;
    const int tail = num_tiles - full * sms;
    if (tail == 0) return 0;
    const int total = tail * upc;
    const int G = full > 0 ? sms : std::min(total, sms);
    std::vector<int> load(G, 0);
    for (int j = 0; j < total; ++j) {
        int t, lo, hi, tt, d0, d1;
        oz_item(num_tiles, tail, 1, upc, G, num_tiles - tail + j, t, lo, hi, tt);
        oz_unit(slices, lo % upc, d0, d1);
        load[(num_tiles - tail + j) % G] += (d0 + 1) + (d1 >= 0 ? d1 + 1 : 0);
    }
    const int max_load = *std::max_element(load.begin(), load.end());
    const double tile_elems = static_cast<double>(kUM) * un;
    const double product_s = 2.0 * tile_elems * static_cast<double>(k) / (4.4e15 / 148);
    const double whole_tile_s = product_s * slices * (slices + 1) / 2;
    const double reduce_s = 4e-6 + tail * (upc + 2.0) * tile_elems * sizeof(double) / 6.5e12;
    const bool fits = tail * upc * tile_elems * sizeof(double) <= static_cast<double>(size_t(512) << 20);
    return (fits && product_s * max_load + reduce_s < 0.9 * whole_tile_s) ? tail : 0;
}

cudaError_t launch_ozaki_gemm(bool ta, bool tb, int m, int n, int k, double alpha, const double* A,
                              size_t lda, const double* B, size_t ldb, double beta, double* C,
                              size_t ldc, int slices, cudaStream_t st, CUresult* cu_err) {
    const size_t kp = round_up(static_cast<size_t>(k), 16);
    const size_t pa = static_cast<size_t>(m) * kp, pb = static_cast<size_t>(n) * kp;
    void* buf = nullptr;
    const size_t exps = round_up((static_cast<size_t>(m) + n) * sizeof(int), 256);
    const size_t a_bytes = round_up(slices * pa, 256);
    // the partial last wave runs unit by unit when that pays (see OzParams)
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int un = ozaki_tile_n(m, n, k);
    const int num_tiles = ((m + kUM - 1) / kUM) * ((n + un - 1) / un);
    const int upc = (slices + 1) / 2;
    const long long kt_chunk = 2147483647LL / (static_cast<long long>(slices) * 128 * 128) / 128;
    const long long ktc = std::max(kt_chunk, 1LL);
    const int kchunks = static_cast<int>(((k + 127) / 128 + ktc - 1) / ktc);
    const int tail_tiles = ozaki_tail_tiles(num_tiles, slices, kchunks, k, sms, un);
    const size_t b_bytes = round_up(slices * pb, 256);
    const size_t w_bytes = static_cast<size_t>(tail_tiles) * upc * kUM * un * sizeof(double);
    cudaError_t e = scratch_alloc(&buf, exps + a_bytes + b_bytes + w_bytes, st);
    if (e != cudaSuccess) return e;
    int* ea = static_cast<int*>(buf);
    int* eb = ea + m;
    int8_t* sla = reinterpret_cast<int8_t*>(static_cast<uint8_t*>(buf) + exps);
    int8_t* slb = sla + a_bytes;
    size_t ars, aps, brs, bps;
    operand_views(ta, tb, lda, ldb, ars, aps, brs, bps);
    fill_int_kernel<<<64, 256, 0, st>>>(ea, m + n, kExpSentinel);
    const int kb = (k + 1023) / 1024, k32 = (k + 31) / 32;
    if (aps == 1) row_exp_kcontig_kernel<<<dim3((m + 7) / 8, kb), 256, 0, st>>>(A, ars, m, k, ea);
    else          row_exp_rcontig_kernel<<<dim3((m + 255) / 256, k32), 256, 0, st>>>(A, aps, m, k, ea);
    if (bps == 1) row_exp_kcontig_kernel<<<dim3((n + 7) / 8, kb), 256, 0, st>>>(B, brs, n, k, eb);
    else          row_exp_rcontig_kernel<<<dim3((n + 255) / 256, k32), 256, 0, st>>>(B, bps, n, k, eb);
    const dim3 ga((kp + kTile - 1) / kTile, (m + kTile - 1) / kTile);
    const dim3 gb((kp + kTile - 1) / kTile, (n + kTile - 1) / kTile);
    launch_ozaki_slices(ga, st, A, ars, aps, m, k, ea, slices, sla, kp, pa);
    launch_ozaki_slices(gb, st, B, brs, bps, n, k, eb, slices, slb, kp, pb);
    count_launch(5);
    CUtensorMap tma, tmb;
    CUresult r = make_tmap_planes(&tma, sla, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, k, m, slices, kp, kUM);
    if (r == CUDA_SUCCESS) r = make_tmap_planes(&tmb, slb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, k, n, slices, kp, un);
    if (r != CUDA_SUCCESS) {
        if (cu_err) *cu_err = r;
        cudaFreeAsync(buf, st);
        return cudaErrorInvalidValue;
    }
    OzParams p{};
    p.m = m; p.n = n; p.k = k;
    p.un = un;
    p.tiles_m = (m + kUM - 1) / kUM;
    p.tiles_n = (n + un - 1) / un;
    p.num_tiles = p.tiles_m * p.tiles_n;
    p.num_kt = static_cast<int>((k + 127) / 128);
    p.slices = slices;
    // exact INT32: a diagonal has <= slices products of |d_t d_u| <= 128*128 per K element
    const long long max_k = 2147483647LL / (static_cast<long long>(slices) * 128 * 128);
    p.kt_per_chunk = static_cast<int>(max_k / 128);
    if (p.kt_per_chunk < 1) p.kt_per_chunk = 1;
    p.kchunks = (p.num_kt + p.kt_per_chunk - 1) / p.kt_per_chunk;
    p.beta_mode = (beta == 0.0) ? 0 : (beta == 1.0 ? 1 : 2);
    p.alpha = alpha; p.beta = beta;
    p.c = C; p.ldc = ldc;
    p.cin = C;
    p.row_exp = ea; p.col_exp = eb;
    p.err = device_error_word();
    if (tail_tiles > 0) {
        p.tail_tiles = tail_tiles;
        p.ws = reinterpret_cast<double*>(static_cast<uint8_t*>(buf) + exps + a_bytes + b_bytes);
    }

    e = ozaki_kernel_attributes();
    if (e != cudaSuccess) { cudaFreeAsync(buf, st); return e; }
    const int items = p.num_tiles + p.tail_tiles * (p.kchunks * upc - 1);
    const int grid = items < sms ? items : sms;
    KernelTimer tmr;
    kernel_timing_begin("umma_ozaki_i8", 2.0 * m * n * static_cast<double>(k) * slices * (slices + 1) / 2, st, &tmr);
    if (un == 256) ozaki_gemm_kernel<256><<<grid, kOzThreads, OzCfg<256>::SMEM, st>>>(tma, tmb, p);
    else           ozaki_gemm_kernel<128><<<grid, kOzThreads, OzCfg<128>::SMEM, st>>>(tma, tmb, p);
    kernel_timing_end(&tmr, st);
    count_launch();
    if (p.tail_tiles > 0) {
        const size_t elems = static_cast<size_t>(p.tail_tiles) * kUM * un;
        const size_t blocks = std::min<size_t>((elems + 255) / 256, static_cast<size_t>(sms) * 16);
        ozaki_reduce_kernel<<<static_cast<unsigned>(blocks), 256, 0, st>>>(p, p.kchunks * upc);
        count_launch();
    }
    e = cudaGetLastError();
    cudaFreeAsync(buf, st);
    return e;
}

// Many f64 GEMMs in the Ozaki form with three launches for the whole batch:
// one exponent pass and one slice pass over every operand, then one
// persistent ozaki_grouped_kernel over every problem's tiles. probs[i] is
// column-major or row-major like rb_gemm_problem; its C0 is read from
// cin[i] (leading dimension ldcin[i]; probs[i].c itself when cin is null) and
// the result goes to probs[i].c. Every tile runs the fused epilogue of
// ozaki_gemm_kernel, so each result equals that problem's own
// rb_dgemm_dev(..., RB_PREC_OZAKI, ...) bit for bit.
int ozaki_grouped_dev(const rb_gemm_problem* probs, size_t count, const void* const* cin, const size_t* ldcin,
                      cudaStream_t st, int32_t* ce) {
    const int slices = rb_get_ozaki_slices();
    const long long kt_chunk = std::max(2147483647LL / (static_cast<long long>(slices) * 128 * 128) / 128, 1LL);
    struct Job {
        bool ta, tb;
        int m, n, k;
        const double *a, *b;
        size_t lda, ldb;
        double* c;
        const double* c0;
        size_t ldc;
        double alpha, beta;
        size_t kp, off_exp, off_a, off_b;
        int num_kt;
        int un;  // tile width
    };
    std::vector<Job> jobs;
    jobs.reserve(count);
    size_t exps = 0, planes = 0;
    cudaError_t e = cudaSuccess;
    for (size_t i = 0; i < count; ++i) {
        const rb_gemm_problem& q = probs[i];
        if (q.dtype != 1) return RB_ERR_UNSUPPORTED;
        const int v = validate_problem(q);
        if (v != RB_OK) return v;
        const bool col = q.layout == RB_COL_MAJOR;
        const size_t m = col ? q.m : q.n, n = col ? q.n : q.m;
        if (m == 0 || n == 0) continue;
        if (m > 0x7fffffff || n > 0x7fffffff || q.k > 0x7fffffff) return RB_ERR_INVALID_ARG;
        double* c = static_cast<double*>(q.c);
        const double* c0 = cin ? static_cast<const double*>(cin[i]) : c;
        const size_t ldc0 = cin ? ldcin[i] : q.ldc;
        if (q.beta != 0.0 && c0 != c && ldc0 != q.ldc) {
            // the kernels read C0 with C's leading dimension: bring it into C first
            e = cudaMemcpy2DAsync(c, q.ldc * 8, c0, ldc0 * 8, m * 8, n, cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) break;
            c0 = c;
        }
        if (q.k == 0 || q.alpha == 0.0) {  // C = beta * C0 only (gemm_contig's early out)
            if (q.beta != 0.0 && c0 != c) {
                e = cudaMemcpy2DAsync(c, q.ldc * 8, c0, q.ldc * 8, m * 8, n, cudaMemcpyDeviceToDevice, st);
                if (e != cudaSuccess) break;
            }
            e = launch_scale_c<double>(static_cast<int>(m), static_cast<int>(n), q.beta, c, q.ldc, st);
            if (e != cudaSuccess) break;
            continue;
        }
        Job j{};
        const bool ta = q.transa != RB_NO_TRANS, tb = q.transb != RB_NO_TRANS;
        j.ta = col ? ta : tb;
        j.tb = col ? tb : ta;
        j.m = static_cast<int>(m);
        j.n = static_cast<int>(n);
        j.k = static_cast<int>(q.k);
        j.a = static_cast<const double*>(col ? q.a : q.b);
        j.b = static_cast<const double*>(col ? q.b : q.a);
        j.lda = col ? q.lda : q.ldb;
        j.ldb = col ? q.ldb : q.lda;
        j.c = c;
        j.c0 = c0;
        j.ldc = q.ldc;
        j.alpha = q.alpha;
        j.beta = q.beta;
        j.kp = round_up(q.k, 16);
        j.num_kt = static_cast<int>((q.k + 127) / 128);
        j.un = ozaki_tile_n(j.m, j.n, j.k);
        j.off_exp = exps;
        exps += m + n;
        j.off_a = planes;
        planes += round_up(slices * m * j.kp, 256);
        j.off_b = planes;
        planes += round_up(slices * n * j.kp, 256);
        jobs.push_back(j);
    }
    if (e != cudaSuccess) {
        if (ce) *ce = e;
        return RB_ERR_CUDA;
    }
    if (jobs.empty()) return RB_OK;
    // one launch per tile width, wide tiles first; inside each, longest tiles
    // first: the CTAs walk the items with a stride of the grid
    std::stable_sort(jobs.begin(), jobs.end(), [](const Job& x, const Job& y) {
        return x.un != y.un ? x.un > y.un : x.num_kt > y.num_kt;
    });
    const int np = static_cast<int>(jobs.size());
    // device image: [entries][starts][operands] then exponents, then planes
    const size_t ent_bytes = round_up(np * sizeof(OzGroupEntry), 256);
    const size_t starts_bytes = round_up((np + 2) * sizeof(int), 256);  // starts of each width's table
    const size_t ops_bytes = round_up(2 * np * sizeof(OzOperand), 256);
    const size_t img_bytes = ent_bytes + starts_bytes + ops_bytes;
    const size_t exp_bytes = round_up(exps * sizeof(int), 256);
    uint8_t* mem = nullptr;
    e = scratch_alloc(reinterpret_cast<void**>(&mem), img_bytes + exp_bytes + planes, st);
    if (e != cudaSuccess) {
        if (ce) *ce = e;
        if (e == cudaErrorMemoryAllocation) cudaGetLastError();
        return e == cudaErrorMemoryAllocation ? RB_ERR_ALLOC : RB_ERR_CUDA;
    }
    std::vector<uint8_t> img(img_bytes, 0);
    int* starts = reinterpret_cast<int*>(img.data() + ent_bytes);
    OzOperand* ops = reinterpret_cast<OzOperand*>(img.data() + ent_bytes + starts_bytes);
    int* dexp = reinterpret_cast<int*>(mem + img_bytes);
    int8_t* dplanes = reinterpret_cast<int8_t*>(mem + img_bytes + exp_bytes);
    uint32_t* err_word = device_error_word();
    int tiles = 0, exp_blocks = 0, slice_blocks = 0;
    int n_wide = 0, tiles_wide = 0;  // the problems (and their tiles) of the 256-wide launch
    double work = 0;
    CUresult r = CUDA_SUCCESS;
    for (int i = 0; i < np && r == CUDA_SUCCESS; ++i) {
        const Job& j = jobs[i];
        int* ea = dexp + j.off_exp;
        int* eb = ea + j.m;
        int8_t* sla = dplanes + j.off_a;
        int8_t* slb = dplanes + j.off_b;
        size_t ars, aps, brs, bps;
        operand_views(j.ta, j.tb, j.lda, j.ldb, ars, aps, brs, bps);
        const int kb = (j.k + 1023) / 1024, k32 = (j.k + 31) / 32;
        const int skb = static_cast<int>((j.kp + kTile - 1) / kTile);
        const struct { const double* x; size_t rs, ps; int R; int* e; int8_t* out; } od[2] = {
            {j.a, ars, aps, j.m, ea, sla}, {j.b, brs, bps, j.n, eb, slb}};
        for (int h = 0; h < 2; ++h) {
            OzOperand& o = ops[2 * i + h];
            o.x = od[h].x; o.rs = od[h].rs; o.ps = od[h].ps;
            o.R = od[h].R; o.K = j.k;
            o.e = od[h].e; o.out = od[h].out;
            o.kp = j.kp; o.plane = static_cast<size_t>(od[h].R) * j.kp;
            o.exp_gx = (o.ps == 1) ? (o.R + 7) / 8 : (o.R + 255) / 256;
            o.slice_gx = skb;
            o.exp_start = exp_blocks;
            o.slice_start = slice_blocks;
            exp_blocks += o.exp_gx * ((o.ps == 1) ? kb : k32);
            slice_blocks += skb * ((o.R + kTile - 1) / kTile);
        }
        OzGroupEntry g{};  // 64-byte aligned here; copied into the image below
        r = make_tmap_planes(&g.tmA, sla, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, j.k, j.m, slices, j.kp, kUM);
        if (r == CUDA_SUCCESS)
            r = make_tmap_planes(&g.tmB, slb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, j.k, j.n, slices, j.kp, j.un);
        OzParams& p = g.p;
        p.m = j.m; p.n = j.n; p.k = j.k;
        p.un = j.un;
        p.tiles_m = (j.m + kUM - 1) / kUM;
        p.tiles_n = (j.n + j.un - 1) / j.un;
        p.num_tiles = p.tiles_m * p.tiles_n;
        p.num_kt = j.num_kt;
        p.slices = slices;
        p.kt_per_chunk = static_cast<int>(kt_chunk);
        p.kchunks = (p.num_kt + p.kt_per_chunk - 1) / p.kt_per_chunk;
        p.beta_mode = (j.beta == 0.0) ? 0 : (j.beta == 1.0 ? 1 : 2);
        p.alpha = j.alpha; p.beta = j.beta;
        p.c = j.c; p.ldc = j.ldc;
        p.cin = j.c0;
        p.row_exp = ea; p.col_exp = eb;
        p.err = err_word;
        std::memcpy(img.data() + i * sizeof(OzGroupEntry), &g, sizeof(OzGroupEntry));
        // the wide launch's starts at [0, n_wide], the narrow launch's at
        // [n_wide + 1, np + 1], each counting from its own first tile
        if (j.un == 256) {
            starts[i] = tiles;
            n_wide = i + 1;
            tiles_wide = tiles + p.num_tiles;
        } else {
            starts[i + 1] = tiles - tiles_wide;
        }
        tiles += p.num_tiles;
        work += 2.0 * j.m * j.n * static_cast<double>(j.k) * slices * (slices + 1) / 2;
    }
    starts[n_wide] = tiles_wide;        // end of the wide table
    starts[np + 1] = tiles - tiles_wide;  // end of the narrow table (at n_wide + 1 .. np + 1)
    if (r != CUDA_SUCCESS) {
        if (ce) *ce = static_cast<int32_t>(r);
        cudaFreeAsync(mem, st);
        return RB_ERR_CUDA;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e = ozaki_kernel_attributes();
    // a pageable source: the driver has staged the image when the call returns
    if (e == cudaSuccess) e = cudaMemcpyAsync(mem, img.data(), img_bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        const OzOperand* dops = reinterpret_cast<const OzOperand*>(mem + ent_bytes + starts_bytes);
        fill_int_kernel<<<static_cast<unsigned>(std::min<size_t>((exps + 255) / 256, 1024)), 256, 0, st>>>(
            dexp, static_cast<int>(exps), kExpSentinel);
        ozaki_exp_grouped_kernel<<<exp_blocks, 256, 0, st>>>(dops, 2 * np);
        switch (slices) {
#define RB_SLICES(S) \
    case S: ozaki_slice_grouped_kernel<S><<<slice_blocks, 256, 0, st>>>(dops, 2 * np); break;
            RB_SLICES(2) RB_SLICES(3) RB_SLICES(4) RB_SLICES(5) RB_SLICES(6) RB_SLICES(7) RB_SLICES(8)
            RB_SLICES(9) RB_SLICES(10) RB_SLICES(11) RB_SLICES(12)
#undef RB_SLICES
            default: break;
        }
        KernelTimer tmr;
        kernel_timing_begin("umma_ozaki_grouped_i8", work, st, &tmr);
        const OzGroupEntry* dtab = reinterpret_cast<const OzGroupEntry*>(mem);
        const int* dstarts = reinterpret_cast<const int*>(mem + ent_bytes);
        const int tiles_narrow = tiles - tiles_wide;
        // with both widths, the narrow launch goes on a forked stream: its
        // CTAs take the SMs that the wide launch's CTAs leave as they finish
        // (each persistent CTA holds a whole SM), instead of waiting for the
        // wide launch's last tile
        ForkedStream fk;
        const bool fork = n_wide > 0 && np > n_wide && fork_stream(st, &fk) == cudaSuccess;
        if (n_wide > 0)
            ozaki_grouped_kernel<256><<<std::min(tiles_wide, sms), kOzThreads, OzCfg<256>::SMEM, st>>>(
                dtab, dstarts, n_wide, err_word);
        if (np > n_wide)
            ozaki_grouped_kernel<128><<<std::min(tiles_narrow, sms), kOzThreads, OzCfg<128>::SMEM,
                                        fork ? fk.s : st>>>(dtab + n_wide, dstarts + n_wide + 1, np - n_wide,
                                                            err_word);
        e = cudaGetLastError();
        if (fork) {
            const cudaError_t je = join_stream(st, &fk);
            if (e == cudaSuccess) e = je;
        }
        kernel_timing_end(&tmr, st);
        count_launch(3 + (n_wide > 0) + (np > n_wide));
        if (e == cudaSuccess) e = cudaGetLastError();
    }
    cudaFreeAsync(mem, st);
    if (e != cudaSuccess) {
        if (ce) *ce = e;
        return RB_ERR_CUDA;
    }
    return RB_OK;
}

}  // namespace rb

// ==============================================================================
// Allocation-free Ozaki DGEMM.
//
// Some callers cannot let a library call cudaMalloc: a serving process that
// has handed all of the GPU's memory to its own pool up front, or code on a
// latency-critical path where an allocation could block on the device or fail
// halfway through a run. For them, rb_dgemm_ozaki_noalloc runs the same
// Ozaki kernels as rb_dgemm_dev(..., RB_PREC_OZAKI, ...) with every scratch
// buffer (digit planes, exponents, the device status word) carved out of the
// fixed array below. The array is a file-scope __device__ object: every GPU
// that loads this library holds its 64 MiB + 64 KiB until the process exits.
// In host code `g_noalloc_scratch` is only a host-side stand-in for the
// symbol, so its device address is looked up with cudaGetSymbolAddress, once
// per device, on the first call made with that device current (and again
// if that device's context has been replaced since, e.g. after a
// cudaDeviceReset, since the old address then belongs to a dead context).
// ==============================================================================

namespace rb {
namespace {

constexpr size_t kNoAllocScratchBytes = (64u << 20) + (64u << 10);
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
struct NoAllocAddr {
    void* ptr;
    unsigned long long ctx;  // the context the address was looked up in (0: unknown)
};
NoAllocAddr g_noalloc_addr[64] = {};

// Bytes of the array one problem uses: the status word, the exponents and
// both digit planes. Returns false (nothing computed) when that exceeds
// `cap`; each step is checked before it can wrap, since m, n and k may each
// be up to 2^31 - 1.
bool noalloc_bytes_needed(size_t m, size_t n, size_t kp, int slices, size_t cap, size_t* need) {
    *need = cap + 1;
    if (m > cap || n > cap || kp > cap) return false;
    const size_t per_k = static_cast<size_t>(slices) * (m + n);  // < 12 * 2^33
    if (kp != 0 && per_k > cap / kp) return false;
    *need = 256 + round_up((m + n) * sizeof(int), 256) + round_up(slices * m * kp, 256) + slices * n * kp;
    return *need <= cap;
}

}  // namespace
}  // namespace rb

extern "C" rb_status rb_dgemm_ozaki_noalloc(rb_layout layout, rb_transpose transa, rb_transpose transb,
                                            size_t m, size_t n, size_t k, double alpha, const double* a,
                                            size_t lda, const double* b, size_t ldb, double beta, double* c,
                                            size_t ldc, void* stream, rb_error* err) {
    using namespace rb;
    auto fail = [&](rb_status s, uint64_t got = 0, uint64_t need = 0, int32_t ce = 0, char which = 0) {
        if (err) {
            err->code = s;
            err->which = which;
            err->got = got;
            err->min_or_need = need;
            err->cuda_error = ce;
        }
        return s;
    };
    if (err) *err = rb_error{0, 0, 0, 0, 0};
    if ((layout != RB_ROW_MAJOR && layout != RB_COL_MAJOR) || transa < RB_NO_TRANS || transa > RB_CONJ_TRANS ||
        transb < RB_NO_TRANS || transb > RB_CONJ_TRANS)
        return fail(RB_ERR_INVALID_ARG);
    // leading dimensions, as check_matrix (src/level3.rs:107-140)
    const bool ta = transa != RB_NO_TRANS, tb = transb != RB_NO_TRANS;
    struct Chk { char w; size_t rows, cols, ld; } chk[3] = {
        {'a', ta ? k : m, ta ? m : k, lda}, {'b', tb ? n : k, tb ? k : n, ldb}, {'c', m, n, ldc}};
    for (const Chk& q : chk) {
        if (q.rows == 0 || q.cols == 0) continue;
        const size_t min_lead = (layout == RB_ROW_MAJOR) ? q.cols : q.rows;
        if (q.ld < min_lead) return fail(RB_ERR_INVALID_LEADING_DIM, q.ld, min_lead, 0, q.w);
    }
    if (m == 0 || n == 0) return RB_OK;
    // row-major -> column-major by swapping operands (src/level3.rs:52-60)
    bool cta = ta, ctb = tb;
    size_t cm = m, cn = n, clda = lda, cldb = ldb;
    const double* ca = a;
    const double* cb = b;
    if (layout == RB_ROW_MAJOR) {
        cta = tb; ctb = ta;
        cm = n; cn = m;
        ca = b; cb = a;
        clda = ldb; cldb = lda;
    }
    if ((k > 0 && (!a || !b)) || !c) return fail(RB_ERR_INVALID_ARG);
    if (cm > 0x7fffffff || cn > 0x7fffffff || k > 0x7fffffff) return fail(RB_ERR_INVALID_ARG);
    const int slices = rb_get_ozaki_slices();
    const size_t kp = round_up(k, 16);
    size_t need = 0;
    if (!noalloc_bytes_needed(cm, cn, kp, slices, kNoAllocScratchBytes, &need))
        return fail(RB_ERR_SCRATCH_LIMIT, need, kNoAllocScratchBytes);

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) return fail(RB_ERR_CUDA, 0, 0, e);
    uint8_t* base;
    {
        // set-up, once per device (and context): the array's device address
        unsigned long long ctx = 0;
        const bool have_ctx = current_context_id(&ctx);
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        NoAllocAddr& s = g_noalloc_addr[dev];
        if (!s.ptr || !have_ctx || s.ctx != ctx) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) return fail(RB_ERR_CUDA, 0, 0, e);
            s.ptr = p;
            // without a context id the lookup is simply repeated on every call
            if (!have_ctx) current_context_id(&ctx);
            s.ctx = ctx;
        }
        base = static_cast<uint8_t*>(s.ptr);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint32_t* status = reinterpret_cast<uint32_t*>(base);
    e = cudaMemsetAsync(status, 0, sizeof(uint32_t), st);  // the previous call's word is stale
    if (e != cudaSuccess) return fail(RB_ERR_CUDA, 0, 0, e);

    if (k == 0 || alpha == 0.0) {
        e = launch_scale_c<double>(static_cast<int>(cm), static_cast<int>(cn), beta, c, ldc, st);
    } else {
        const int M = static_cast<int>(cm), N = static_cast<int>(cn), K = static_cast<int>(k);
        const size_t exps = round_up((cm + cn) * sizeof(int), 256);
        const size_t pa = cm * kp, pb = cn * kp;
        int* ea = reinterpret_cast<int*>(base + 256);
        int* eb = ea + cm;
        int8_t* sla = reinterpret_cast<int8_t*>(base + 256 + exps);
        int8_t* slb = sla + round_up(slices * pa, 256);
        size_t ars, aps, brs, bps;
        operand_views(cta, ctb, clda, cldb, ars, aps, brs, bps);
        fill_int_kernel<<<64, 256, 0, st>>>(ea, M + N, kExpSentinel);
        const int kb = (K + 1023) / 1024, k32 = (K + 31) / 32;
        if (aps == 1) row_exp_kcontig_kernel<<<dim3((M + 7) / 8, kb), 256, 0, st>>>(ca, ars, M, K, ea);
        else          row_exp_rcontig_kernel<<<dim3((M + 255) / 256, k32), 256, 0, st>>>(ca, aps, M, K, ea);
        if (bps == 1) row_exp_kcontig_kernel<<<dim3((N + 7) / 8, kb), 256, 0, st>>>(cb, brs, N, K, eb);
        else          row_exp_rcontig_kernel<<<dim3((N + 255) / 256, k32), 256, 0, st>>>(cb, bps, N, K, eb);
        const dim3 ga((kp + kTile - 1) / kTile, (M + kTile - 1) / kTile);
        const dim3 gb((kp + kTile - 1) / kTile, (N + kTile - 1) / kTile);
        launch_ozaki_slices(ga, st, ca, ars, aps, M, K, ea, slices, sla, kp, pa);
        launch_ozaki_slices(gb, st, cb, brs, bps, N, K, eb, slices, slb, kp, pb);
        count_launch(5);
        CUtensorMap tma, tmb;
        CUresult r = make_tmap_planes(&tma, sla, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, K, M, slices, kp, kUM);
        if (r == CUDA_SUCCESS) r = make_tmap_planes(&tmb, slb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, K, N, slices, kp, 256);
        if (r != CUDA_SUCCESS) return fail(RB_ERR_CUDA, 0, 0, static_cast<int32_t>(r));
        OzParams p{};
        p.m = M; p.n = N; p.k = K;
        p.un = 256;  // always the wide tile, and never the split tail: its scratch is sized for that
        p.tiles_m = (M + kUM - 1) / kUM;
        p.tiles_n = (N + 255) / 256;
        p.num_tiles = p.tiles_m * p.tiles_n;
        p.num_kt = (K + 127) / 128;
        p.slices = slices;
        const long long max_k = 2147483647LL / (static_cast<long long>(slices) * 128 * 128);
        p.kt_per_chunk = static_cast<int>(max_k / 128) > 0 ? static_cast<int>(max_k / 128) : 1;
        p.kchunks = (p.num_kt + p.kt_per_chunk - 1) / p.kt_per_chunk;
        p.beta_mode = (beta == 0.0) ? 0 : (beta == 1.0 ? 1 : 2);
        p.alpha = alpha; p.beta = beta;
        p.c = c; p.ldc = ldc;
        p.cin = c;
        p.row_exp = ea; p.col_exp = eb;
        p.err = status;
        e = ozaki_kernel_attributes();
        if (e != cudaSuccess) return fail(RB_ERR_CUDA, 0, 0, e);
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        ozaki_gemm_kernel<256><<<p.num_tiles < sms ? p.num_tiles : sms, kOzThreads, OzCfg<256>::SMEM, st>>>(
            tma, tmb, p);
        count_launch();
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return fail(RB_ERR_CUDA, 0, 0, e);
    // The call returns once its work has finished, with the kernels' status word read back.
    uint32_t word = 0;
    e = cudaMemcpyAsync(&word, status, sizeof(word), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(RB_ERR_CUDA, 0, 0, e);
    if (word != 0) return fail((word >> 24) == (RB_DEVERR_TIMEOUT >> 24) ? RB_ERR_TIMEOUT : RB_ERR_DEVICE, word);
    return RB_OK;
}
