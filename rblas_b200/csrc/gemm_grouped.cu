// gemm_grouped.cu -- grouped GEMM: many problems with their own m, n, k,
// transposes, alpha/beta and dtype (f32 / f64, plain form) in one launch.
//
// The host builds a device-side problem table: per problem two TMA tensor
// maps (in global memory, 64-byte aligned), the epilogue description, the
// tile grid, the split-K factor and the problem's first index in the
// concatenated work-item space (item = one K range of one C tile). Problems
// are ordered longest item first. A persistent grid (one CTA per SM) takes
// items from an atomic counter (greedy longest-first scheduling); the
// producer lane claims each item and hands it to the compute warps through a
// two-slot mbarrier ring, then all of them run the same tile pipeline as the
// single-problem kernel (simt_tile.cuh) through one continuous stage ring, so
// tiles of different problems stream back to back without a launch.
//
// Split-K is deterministic: each of a tile's S items stores its partial
// accumulator to a 64 KiB workspace slot; the item that arrives last on the
// tile's counter sums the S slots in index order and runs the epilogue, so a
// problem's result depends only on its own shape (which fixes S), never on
// the other problems in the launch or on timing.
// Work per problem: 2mnk flop.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <vector>

#include "../../include/rblas_b200.h"
#include "rb_device.cuh"
#include "rb_internal.h"
#include "simt_tile.cuh"

namespace rb {

namespace {

constexpr int kGroupStage = 32768;  // max(f32 32 KiB, f64 24 KiB) stage
constexpr int kGroupST = SimtCfg<float>::STAGES;
// stages, then full/empty stage barriers, item ring barriers, compute barrier, item slots, reduce flag
constexpr int kGroupCtl = 2 * kGroupST * 8 + 4 * 8 + 8 + 2 * 4 + 4;
constexpr int kGroupSmem = kGroupST * kGroupStage + 128 + 1024;
static_assert(kGroupCtl <= 128, "control block");
static_assert(SimtCfg<float>::STAGES == SimtCfg<double>::STAGES, "one ring for both dtypes");
constexpr int kSlotElems = SimtCfg<float>::BM * SimtCfg<float>::BN;  // per-slot f32 elements (64 KiB)
static_assert(kSlotElems * 4 == SimtCfg<double>::BM * SimtCfg<double>::BN * 8, "one slot size for both dtypes");
constexpr size_t kSlotBytes = kSlotElems * 4;

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
    int splits;       // S: items per C tile
    int kt_per_split; // K-tiles per item (the last item of a tile may have fewer)
    int ws_slot;      // first workspace slot (S > 1)
    int sem;          // first tile counter (S > 1)
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

// An item's tile and K range.
struct Item {
    int tm, tn, tile, split, kt0, nkt;
};

__device__ __forceinline__ Item decode_item(const GroupProblem* p, int r) {
    Item w;
    w.tile = r / p->splits;
    w.split = r - w.tile * p->splits;
    raster_tile(w.tile, p->tiles_m, p->tiles_n, w.tm, w.tn);
    w.kt0 = w.split * p->kt_per_split;
    w.nkt = min(p->kt_per_split, p->num_kt - w.kt0);
    return w;
}

// Barrier of the 8 compute warps on an mbarrier (count 8, one arrival per
// warp), so that the wait is bounded like every other wait in the kernel.
__device__ __forceinline__ bool compute_sync(uint64_t* cbar, uint32_t& cph, uint32_t* err, int lane) {
    __syncwarp();
    if (lane == 0) mbar_arrive(cbar);
    const bool ok = mbar_wait(cbar, cph & 1, err, 0x113);
    ++cph;
    return ok;
}

template <typename T, bool A_K, bool B_K>
__device__ __noinline__ bool produce_v(const GroupProblem* p, int r, uint8_t* smem, uint64_t* full,
                                       uint64_t* empty, uint32_t& it, uint32_t* err) {
    const Item w = decode_item(p, r);
    return simt_produce<T, A_K, B_K>(&p->tmA, &p->tmB, w.tm * SimtCfg<T>::BM, w.tn * SimtCfg<T>::BN, w.kt0, w.nkt,
                                     smem, kGroupStage, full, empty, it, err);
}

template <typename T, bool A_K, bool B_K>
__device__ __noinline__ bool consume_v(const GroupProblem* p, int r, uint8_t* smem, uint64_t* full, uint64_t* empty,
                                       uint32_t& it, uint32_t* err, int warp, int lane, float* ws, int* sems,
                                       volatile int* red_flag, uint64_t* cbar, uint32_t& cph) {
    constexpr int TN = SimtCfg<T>::TN;
    const Item w = decode_item(p, r);
    T acc[8][TN];
    if (!simt_mainloop<T, A_K, B_K>(acc, w.nkt, smem, kGroupStage, full, empty, it, err, warp, lane)) return false;
    const SimtOut<T> o{static_cast<T*>(p->c), p->ldc, static_cast<const T*>(p->cin), p->ldcin, p->m, p->n,
                       static_cast<T>(p->alpha), static_cast<T>(p->beta), p->beta_mode, 0};
    const int m0 = w.tm * SimtCfg<T>::BM, n0 = w.tn * SimtCfg<T>::BN;
    if (p->splits == 1) {
        simt_epilogue<T, A_K, B_K>(o, acc, m0, n0, warp, lane);
        return true;
    }
    // split-K: partial to this item's slot, element (i, j) of thread t at
    // [(i * TN + j) * 256 + t] so every warp store is 32 consecutive values
    constexpr int NT = kSimtComputeWarps * 32;
    const int t = warp * 32 + lane;
    T* base = reinterpret_cast<T*>(ws + static_cast<size_t>(p->ws_slot + w.tile * p->splits) * kSlotElems);
    T* mine = base + static_cast<size_t>(w.split) * (kSlotBytes / sizeof(T));
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) __stcg(mine + (i * TN + j) * NT + t, acc[i][j]);
    __threadfence();
    if (!compute_sync(cbar, cph, err, lane)) return false;
    if (t == 0) *red_flag = (atomicAdd(sems + p->sem + w.tile, 1) == p->splits - 1);
    if (!compute_sync(cbar, cph, err, lane)) return false;
    const bool last = *red_flag;
    // every thread has read the flag before the next item may rewrite it
    if (!compute_sync(cbar, cph, err, lane)) return false;
    if (!last) return true;
    __threadfence();
    // the last item of the tile sums the S partials in slot order
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = __ldcg(base + (i * TN + j) * NT + t);
    for (int s = 1; s < p->splits; ++s) {
        const T* src = base + static_cast<size_t>(s) * (kSlotBytes / sizeof(T));
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < TN; ++j) acc[i][j] += __ldcg(src + (i * TN + j) * NT + t);
    }
    simt_epilogue<T, A_K, B_K>(o, acc, m0, n0, warp, lane);
    return true;
}

// ctl layout: [0] item counter, then one counter per split tile (zeroed by
// the host with the table upload).
__global__ void __launch_bounds__(kSimtThreads, 1)
    grouped_gemm_kernel(const GroupProblem* __restrict__ probs, const int* __restrict__ starts, int nprob,
                        int total_items, int* ctl, float* ws, uint32_t* err) {
    constexpr int ST = kGroupST;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + ST * kGroupStage);
    uint64_t* empty = full + ST;
    uint64_t* item_full = empty + ST;
    uint64_t* item_empty = item_full + 2;
    uint64_t* cbar = item_empty + 2;
    volatile int* item_slot = reinterpret_cast<volatile int*>(cbar + 1);
    volatile int* red_flag = item_slot + 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kSimtComputeWarps);
        }
        for (int s = 0; s < 2; ++s) {
            mbar_init(&item_full[s], 1);
            mbar_init(&item_empty[s], kSimtComputeWarps);
        }
        mbar_init(cbar, kSimtComputeWarps);
        fence_barrier_init();
    }
    __syncthreads();
    uint32_t it = 0, cph = 0;
    const bool producer = (warp == kSimtComputeWarps);
    if (producer && lane != 0) return;
    int* sems = ctl + 1;
    for (uint32_t q = 0;; ++q) {
        const int slot = q & 1;
        int item;
        if (producer) {
            item = atomicAdd(ctl, 1);
            if (item >= total_items) item = -1;
            if (q >= 2 && !mbar_wait(&item_empty[slot], ((q >> 1) - 1) & 1, err, 0x111)) {
                const uint32_t first = it > (uint32_t)ST ? it - ST : 0;
                for (uint32_t j = first; j < it; ++j) mbar_wait_drain(&full[j % ST], (j / ST) & 1);
                return;
            }
            item_slot[slot] = item;
            mbar_arrive(&item_full[slot]);
        } else {
            if (!mbar_wait(&item_full[slot], (q >> 1) & 1, err, 0x112)) return;
            item = item_slot[slot];
            __threadfence_block();  // each lane's read of the slot precedes the release
            __syncwarp();
            if (lane == 0) mbar_arrive(&item_empty[slot]);
        }
        if (item < 0) return;
        const int pi = find_problem(starts, nprob, item);
        const GroupProblem* p = probs + pi;
        const int r = item - __ldg(starts + pi);
        bool ok;
        if (producer) {
            switch (p->variant) {
                case 0: ok = produce_v<float, false, false>(p, r, smem, full, empty, it, err); break;
                case 1: ok = produce_v<float, false, true>(p, r, smem, full, empty, it, err); break;
                case 2: ok = produce_v<float, true, false>(p, r, smem, full, empty, it, err); break;
                case 3: ok = produce_v<float, true, true>(p, r, smem, full, empty, it, err); break;
                case 4: ok = produce_v<double, false, false>(p, r, smem, full, empty, it, err); break;
                case 5: ok = produce_v<double, false, true>(p, r, smem, full, empty, it, err); break;
                case 6: ok = produce_v<double, true, false>(p, r, smem, full, empty, it, err); break;
                default: ok = produce_v<double, true, true>(p, r, smem, full, empty, it, err); break;
            }
        } else {
#define RB_CONSUME(T, AK, BK) consume_v<T, AK, BK>(p, r, smem, full, empty, it, err, warp, lane, ws, sems, red_flag, cbar, cph)
            switch (p->variant) {
                case 0: ok = RB_CONSUME(float, false, false); break;
                case 1: ok = RB_CONSUME(float, false, true); break;
                case 2: ok = RB_CONSUME(float, true, false); break;
                case 3: ok = RB_CONSUME(float, true, true); break;
                case 4: ok = RB_CONSUME(double, false, false); break;
                case 5: ok = RB_CONSUME(double, false, true); break;
                case 6: ok = RB_CONSUME(double, true, false); break;
                default: ok = RB_CONSUME(double, true, true); break;
            }
#undef RB_CONSUME
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

namespace {

// Split-K policy: a function of the problem's own shape only, so a result
// never depends on what else shares the launch. A problem with fewer C tiles
// than SMs and a long K is cut into up to kMaxSplit K ranges of at least
// kMinSplitKt K-tiles, aiming at about one wave of items for the problem.
constexpr int kMinSplitKt = 16;
constexpr int kMaxSplit = 16;
constexpr int kWaveItems = 148;

struct Plan {
    size_t m, n, k;  // column-major (normalised)
    bool ta, tb;
    int tiles_m, tiles_n, num_kt, splits, kt_per_split;
};

// Tuned split factors per shape bucket (floor(log2) of the column-major m, n
// and of k, per dtype), installed by the autotuner or from its cache file.
// Readers take a snapshot; a problem's split depends on its shape and on the
// table installed when its launch was planned.
std::mutex g_tune_mu;
std::shared_ptr<const std::map<uint32_t, int>> g_tuned;
thread_local int t_forced_splits = 0;  // autotuner candidates

int log2_bucket(size_t x) {
    int b = 0;
    while (x > 1 && b < 31) {
        x >>= 1;
        ++b;
    }
    return b;
}

}  // namespace

uint32_t tune_key(int dtype, size_t m, size_t n, size_t k) {
    return (static_cast<uint32_t>(dtype & 1) << 24) | (static_cast<uint32_t>(log2_bucket(m)) << 16) |
           (static_cast<uint32_t>(log2_bucket(n)) << 8) | static_cast<uint32_t>(log2_bucket(k));
}

void set_tuned_splits(std::shared_ptr<const std::map<uint32_t, int>> table) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned = std::move(table);
}

void force_grouped_splits(int s) { t_forced_splits = s; }

// Tuned Ozaki tile widths per shape bucket (the f64 buckets of tune_key),
// installed alongside the split factors.
namespace {
std::shared_ptr<const std::map<uint32_t, int>> g_tuned_oz;
thread_local int t_forced_oz_width = 0;
}  // namespace

void set_tuned_ozaki_widths(std::shared_ptr<const std::map<uint32_t, int>> table) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned_oz = std::move(table);
}

void force_ozaki_width(int w) { t_forced_oz_width = w; }

int ozaki_tile_n(size_t m, size_t n, size_t k) {
    if (t_forced_oz_width) return t_forced_oz_width;
    std::shared_ptr<const std::map<uint32_t, int>> t;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        t = g_tuned_oz;
    }
    if (t) {
        auto it = t->find(tune_key(1, m, n, k));
        if (it != t->end()) return it->second;
    }
    return n <= 128 ? 128 : 256;  // one narrow tile column: no padding to 256
}

namespace {

std::shared_ptr<const std::map<uint32_t, int>> tuned_snapshot() {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    return g_tuned;
}

Plan plan_problem(const rb_gemm_problem& q, const std::map<uint32_t, int>* tuned = nullptr) {
    Plan pl{};
    const bool ta = q.transa != RB_NO_TRANS, tb = q.transb != RB_NO_TRANS;
    const bool col = q.layout == RB_COL_MAJOR;
    pl.m = col ? q.m : q.n;
    pl.n = col ? q.n : q.m;
    pl.k = q.k;
    pl.ta = col ? ta : tb;
    pl.tb = col ? tb : ta;
    const bool f64 = q.dtype == 1;
    const int BN = f64 ? SimtCfg<double>::BN : SimtCfg<float>::BN;
    const int BK = f64 ? SimtCfg<double>::BK : SimtCfg<float>::BK;
    pl.tiles_m = static_cast<int>((pl.m + 127) / 128);
    pl.tiles_n = static_cast<int>((pl.n + BN - 1) / BN);
    const bool skip_ab = (pl.k == 0 || q.alpha == 0.0);
    pl.num_kt = skip_ab ? 0 : static_cast<int>((pl.k + BK - 1) / BK);
    pl.splits = 1;
    pl.kt_per_split = std::max(pl.num_kt, 1);
    const long tiles = static_cast<long>(pl.tiles_m) * pl.tiles_n;
    if (!pl.m || !pl.n || pl.num_kt < 2) return pl;
    int s = 1;
    if (t_forced_splits > 0) {
        s = t_forced_splits;
    } else {
        auto it = tuned ? tuned->find(tune_key(q.dtype, pl.m, pl.n, pl.k)) : std::map<uint32_t, int>::const_iterator();
        if (tuned && it != tuned->end()) {
            s = it->second;
        } else if (tiles < kWaveItems && pl.num_kt >= 2 * kMinSplitKt) {
            s = static_cast<int>(std::min<long>({static_cast<long>(pl.num_kt / kMinSplitKt),
                                                 static_cast<long>(kMaxSplit), (kWaveItems + tiles - 1) / tiles}));
        }
    }
    s = std::max(1, std::min({s, kMaxSplit, pl.num_kt}));
    if (s > 1) {
        pl.kt_per_split = (pl.num_kt + s - 1) / s;
        pl.splits = (pl.num_kt + pl.kt_per_split - 1) / pl.kt_per_split;
    }
    return pl;
}

size_t plan_slots(const Plan& pl) {
    return pl.splits > 1 ? static_cast<size_t>(pl.tiles_m) * pl.tiles_n * pl.splits : 0;
}

}  // namespace

size_t grouped_table_bytes(size_t count, size_t sems) {
    return rup(count * sizeof(GroupProblem) + count * sizeof(int) + (1 + sems) * sizeof(int), 256);
}

size_t grouped_ws_slots(const rb_gemm_problem& q) {
    if (validate_problem(q) != RB_OK) return 0;
    return plan_slots(plan_problem(q, tuned_snapshot().get()));
}

size_t grouped_slot_bytes() { return kSlotBytes; }

int grouped_splits(const rb_gemm_problem& q) {
    if (validate_problem(q) != RB_OK) return 0;
    return plan_problem(q, tuned_snapshot().get()).splits;
}

namespace {

// Host side of one grouped launch: validation, ordering, the split plan,
// the repacks of operands TMA cannot address, and the device image (table,
// item starts, zeroed counters). Used by the one-shot path and by plans.
class GroupBuilder {
public:
    struct Repack {
        const void* src;
        size_t spitch, dst_off, dpitch, width, height;
    };
    size_t n = 0, total = 0, slots = 0, sems = 0, tbytes = 0, ctl_off = 0, all_bytes = 0, scratch = 0;
    double work = 0;
    std::vector<Repack> repacks;

    // validate and size everything; *bad = first invalid problem
    int plan(const rb_gemm_problem* probs, size_t count, size_t* bad) {
        probs_ = probs;
        plan_.resize(count);
        const auto tuned = tuned_snapshot();
        for (size_t i = 0; i < count; ++i) {
            const int v = validate_problem(probs[i]);
            if (v != RB_OK) {
                if (bad) *bad = i;
                return v;
            }
            plan_[i] = plan_problem(probs[i], tuned.get());
        }
        // order: longest item first (greedy longest-processing-time
        // scheduling through the kernel's atomic item counter); estimated
        // time per K-tile of an item, f32 : f64 about 15 : 8
        order_.clear();
        for (size_t i = 0; i < count; ++i)
            if (plan_[i].m && plan_[i].n) order_.push_back(i);
        auto cost = [&](size_t i) {
            return static_cast<long>(std::min(plan_[i].kt_per_split, std::max(plan_[i].num_kt, 1))) *
                   (probs[i].dtype ? 8 : 15);
        };
        std::stable_sort(order_.begin(), order_.end(), [&](size_t x, size_t y) { return cost(x) > cost(y); });
        rp_a_.assign(count, {SIZE_MAX, 0});
        rp_b_.assign(count, {SIZE_MAX, 0});
        scratch = slots = sems = total = 0;
        work = 0;
        for (size_t i : order_) {
            const Plan& pl = plan_[i];
            const rb_gemm_problem& q = probs[i];
            const size_t el = q.dtype ? 8 : 4, vec = 16 / el;
            work += 2.0 * q.m * q.n * static_cast<double>(q.k);
            if (pl.splits > 1) {
                slots += plan_slots(pl);
                sems += static_cast<size_t>(pl.tiles_m) * pl.tiles_n;
            }
            total += static_cast<size_t>(pl.tiles_m) * pl.tiles_n * pl.splits;
            if (pl.num_kt == 0) continue;
            const bool col = q.layout == RB_COL_MAJOR;
            if (!tma_aligned(col ? q.a : q.b, col ? q.lda : q.ldb, el)) {
                const size_t rows = pl.ta ? pl.k : pl.m, cols = pl.ta ? pl.m : pl.k, ld2 = rup(rows, vec);
                rp_a_[i] = {scratch, ld2};
                scratch += rup(ld2 * cols * el, 256);
            }
            if (!tma_aligned(col ? q.b : q.a, col ? q.ldb : q.lda, el)) {
                const size_t rows = pl.tb ? pl.n : pl.k, cols = pl.tb ? pl.k : pl.n, ld2 = rup(rows, vec);
                rp_b_[i] = {scratch, ld2};
                scratch += rup(ld2 * cols * el, 256);
            }
        }
        if (total > 0x7fffffff || slots > 0x7fffffff) return RB_ERR_INVALID_ARG;
        n = order_.size();
        tbytes = n * sizeof(GroupProblem);
        ctl_off = tbytes + n * sizeof(int);
        all_bytes = grouped_table_bytes(n, sems);
        return RB_OK;
    }

    // write the device image (all_bytes) into `image`, tensor maps pointing
    // at `scratch_base` for repacked operands; fills `repacks`
    int encode(const void* const* cin, const size_t* ldcin, uint8_t* scratch_base, uint8_t* image, size_t* bad,
               int32_t* ce) {
        repacks.clear();
        std::vector<int> starts;
        starts.reserve(n);
        size_t slot = 0, sem = 0, item = 0, row = 0;
        for (size_t i : order_) {
            const rb_gemm_problem& q = probs_[i];
            const Plan& pl = plan_[i];
            const size_t el = q.dtype ? 8 : 4;
            const bool f64 = q.dtype == 1;
            const bool col = q.layout == RB_COL_MAJOR;
            const void* a = col ? q.a : q.b;
            const void* b = col ? q.b : q.a;
            size_t lda = col ? q.lda : q.ldb, ldb = col ? q.ldb : q.lda;
            if (rp_a_[i].first != SIZE_MAX) {
                const size_t rows = pl.ta ? pl.k : pl.m, cols = pl.ta ? pl.m : pl.k;
                repacks.push_back({a, lda * el, rp_a_[i].first, rp_a_[i].second * el, rows * el, cols});
                a = scratch_base + rp_a_[i].first;
                lda = rp_a_[i].second;
            }
            if (rp_b_[i].first != SIZE_MAX) {
                const size_t rows = pl.tb ? pl.n : pl.k, cols = pl.tb ? pl.k : pl.n;
                repacks.push_back({b, ldb * el, rp_b_[i].first, rp_b_[i].second * el, rows * el, cols});
                b = scratch_base + rp_b_[i].first;
                ldb = rp_b_[i].second;
            }
            GroupProblem g{};
            const int BM = 128, BN = f64 ? SimtCfg<double>::BN : SimtCfg<float>::BN;
            const int BK = f64 ? SimtCfg<double>::BK : SimtCfg<float>::BK;
            const CUtensorMapDataType dt = f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
            const bool a_k = pl.ta, b_k = !pl.tb;
            CUresult r = CUDA_SUCCESS;
            if (pl.num_kt > 0) {
                r = a_k ? make_tmap_2d(&g.tmA, a, dt, el, pl.k, pl.m, lda, BK, BM, true)
                        : make_tmap_2d(&g.tmA, a, dt, el, pl.m, pl.k, lda, simt_mn_a_box(el), BK,
                                       simt_mn_a_swizzled(el));
                if (r == CUDA_SUCCESS)
                    r = b_k ? make_tmap_2d(&g.tmB, b, dt, el, pl.k, pl.n, ldb, BK, BN, true)
                            : make_tmap_2d(&g.tmB, b, dt, el, pl.n, pl.k, ldb, BN, BK, false);
            }
            if (r != CUDA_SUCCESS) {
                if (ce) *ce = static_cast<int32_t>(r);
                if (bad) *bad = i;
                return RB_ERR_CUDA;
            }
            g.c = q.c;
            g.ldc = q.ldc;
            g.cin = cin ? cin[i] : q.c;
            g.ldcin = ldcin ? ldcin[i] : q.ldc;
            // k == 0 or alpha == 0: C = beta*Cin exactly (alpha*0 would turn an inf alpha into NaN)
            g.alpha = pl.num_kt ? q.alpha : 0.0;
            g.beta = q.beta;
            g.m = static_cast<int>(pl.m);
            g.n = static_cast<int>(pl.n);
            g.num_kt = pl.num_kt;
            g.variant = (f64 ? 4 : 0) + (a_k ? 2 : 0) + (b_k ? 1 : 0);
            g.tiles_m = pl.tiles_m;
            g.tiles_n = pl.tiles_n;
            g.beta_mode = (q.beta == 0.0) ? 0 : (q.beta == 1.0 ? 1 : 2);
            g.splits = pl.splits;
            g.kt_per_split = pl.kt_per_split;
            g.ws_slot = static_cast<int>(slot);
            g.sem = static_cast<int>(sem);
            if (pl.splits > 1) {
                slot += plan_slots(pl);
                sem += static_cast<size_t>(pl.tiles_m) * pl.tiles_n;
            }
            starts.push_back(static_cast<int>(item));
            item += static_cast<size_t>(pl.tiles_m) * pl.tiles_n * pl.splits;
            std::memcpy(image + row * sizeof(GroupProblem), &g, sizeof(GroupProblem));
            ++row;
        }
        std::memcpy(image + tbytes, starts.data(), n * sizeof(int));
        std::memset(image + ctl_off, 0, all_bytes - ctl_off);
        return RB_OK;
    }

    cudaError_t enqueue_repacks(uint8_t* scratch_base, cudaStream_t st) const {
        for (const Repack& r : repacks) {
            const cudaError_t e = cudaMemcpy2DAsync(scratch_base + r.dst_off, r.dpitch, r.src, r.spitch, r.width,
                                                    r.height, cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }

    // the kernel over a device image already in place (counters zeroed)
    cudaError_t launch(uint8_t* dev_image, float* ws, cudaStream_t st, bool timed) const {
        static bool attr = false;
        if (!attr) {
            const cudaError_t e =
                cudaFuncSetAttribute(grouped_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kGroupSmem);
            if (e != cudaSuccess) return e;
            attr = true;
        }
        int dev_id = 0, sms = 148;
        cudaGetDevice(&dev_id);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_id);
        KernelTimer tmr;
        if (timed) kernel_timing_begin("grouped_gemm", work, st, &tmr);
        grouped_gemm_kernel<<<static_cast<int>(std::min<size_t>(total, sms)), kSimtThreads, kGroupSmem, st>>>(
            reinterpret_cast<const GroupProblem*>(dev_image), reinterpret_cast<const int*>(dev_image + tbytes),
            static_cast<int>(n), static_cast<int>(total), reinterpret_cast<int*>(dev_image + ctl_off), ws,
            device_error_word());
        if (timed) kernel_timing_end(&tmr, st);
        if (timed) count_launch();  // a captured launch is counted at each replay
        return cudaGetLastError();
    }

private:
    const rb_gemm_problem* probs_ = nullptr;
    std::vector<Plan> plan_;
    std::vector<size_t> order_;
    std::vector<std::pair<size_t, size_t>> rp_a_, rp_b_;
};

}  // namespace

int grouped_gemm_dev(const rb_gemm_problem* probs, size_t count, const void* const* cin, const size_t* ldcin,
                     cudaStream_t st, int32_t* ce, size_t* bad_index, const GroupStaging* staging) {
    GroupBuilder gb;
    int rc = gb.plan(probs, count, bad_index);
    if (rc != RB_OK || gb.n == 0) return rc;
    if (!device_error_word()) return RB_ERR_ALLOC;
    const size_t ws_bytes = gb.slots * kSlotBytes;
    const bool staged = staging && staging->host && staging->dev && gb.all_bytes <= staging->bytes &&
                        (ws_bytes == 0 || (staging->ws && ws_bytes <= staging->ws_bytes));
    uint8_t* host = nullptr;
    std::vector<uint8_t> pageable;
    uint8_t* dev = nullptr;
    float* ws = nullptr;
    cudaError_t e;
    // one stream-ordered allocation for what staging does not cover: [image][workspace][repack scratch]
    const size_t own = (staged ? 0 : gb.all_bytes + ws_bytes) + gb.scratch;
    uint8_t* mem = nullptr;
    if (own) {
        e = scratch_alloc(reinterpret_cast<void**>(&mem), own, st);
        if (e != cudaSuccess) {
            if (ce) *ce = e;
            if (e == cudaErrorMemoryAllocation) cudaGetLastError();
            return e == cudaErrorMemoryAllocation ? RB_ERR_ALLOC : RB_ERR_CUDA;
        }
    }
    if (staged) {
        host = static_cast<uint8_t*>(staging->host);
        dev = static_cast<uint8_t*>(staging->dev);
        ws = static_cast<float*>(staging->ws);
    } else {
        pageable.resize(gb.all_bytes);
        host = pageable.data();
        dev = mem;
        if (ws_bytes) ws = reinterpret_cast<float*>(mem + gb.all_bytes);
    }
    uint8_t* scratch = gb.scratch ? mem + (staged ? 0 : gb.all_bytes + ws_bytes) : nullptr;
    rc = gb.encode(cin, ldcin, scratch, host, bad_index, ce);
    if (rc == RB_OK) {
        // a pinned source copies asynchronously; a pageable one is staged by
        // the driver before the call returns
        e = gb.enqueue_repacks(scratch, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dev, host, gb.all_bytes, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = gb.launch(dev, ws, st, true);
        if (e != cudaSuccess) {
            if (ce) *ce = e;
            rc = RB_ERR_CUDA;
        }
    }
    if (mem) cudaFreeAsync(mem, st);
    return rc;
}

// A grouped launch frozen into a CUDA graph: table, workspace and repack
// scratch allocated once; each replay re-zeroes the counters, redoes the
// repacks (operand contents may change between replays) and runs the kernel.
struct GroupedPlan {
    uint8_t* mem = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~GroupedPlan() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (mem) cudaFree(mem);
    }
};

int grouped_plan_create(const rb_gemm_problem* probs, size_t count, void** out, int32_t* ce, size_t* bad) {
    GroupBuilder gb;
    int rc = gb.plan(probs, count, bad);
    if (rc != RB_OK) return rc;
    if (!device_error_word()) return RB_ERR_ALLOC;
    GroupedPlan* pl = new GroupedPlan();
    const size_t ws_bytes = gb.slots * kSlotBytes;
    const size_t total = rup(gb.all_bytes, 256) + ws_bytes + gb.scratch;
    cudaError_t e = cudaSuccess;
    if (total) e = dev_alloc(reinterpret_cast<void**>(&pl->mem), total);
    if (e != cudaSuccess) {
        if (ce) *ce = e;
        delete pl;
        return RB_ERR_ALLOC;
    }
    uint8_t* dev = pl->mem;
    float* ws = ws_bytes ? reinterpret_cast<float*>(pl->mem + rup(gb.all_bytes, 256)) : nullptr;
    uint8_t* scratch = gb.scratch ? pl->mem + rup(gb.all_bytes, 256) + ws_bytes : nullptr;
    std::vector<uint8_t> image(gb.all_bytes);
    if (gb.n) rc = gb.encode(nullptr, nullptr, scratch, image.data(), bad, ce);
    if (rc == RB_OK && gb.n) e = cudaMemcpy(dev, image.data(), gb.all_bytes, cudaMemcpyHostToDevice);
    cudaStream_t cs = nullptr;
    if (rc == RB_OK && e == cudaSuccess) e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (rc == RB_OK && e == cudaSuccess) {
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t e2 = cudaSuccess;
            if (gb.n) {
                e2 = cudaMemsetAsync(dev + gb.ctl_off, 0, gb.all_bytes - gb.ctl_off, cs);
                if (e2 == cudaSuccess) e2 = gb.enqueue_repacks(scratch, cs);
                if (e2 == cudaSuccess) e2 = gb.launch(dev, ws, cs, false);
            }
            e = cudaStreamEndCapture(cs, &pl->graph);
            if (e == cudaSuccess) e = e2;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&pl->exec, pl->graph, 0);
    }
    if (cs) cudaStreamDestroy(cs);
    if (rc == RB_OK && e != cudaSuccess) {
        if (ce) *ce = e;
        rc = RB_ERR_CUDA;
    }
    if (rc != RB_OK) {
        delete pl;
        return rc;
    }
    *out = pl;
    return RB_OK;
}

int grouped_plan_launch(void* plan, cudaStream_t st, int32_t* ce) {
    GroupedPlan* pl = static_cast<GroupedPlan*>(plan);
    const cudaError_t e = cudaGraphLaunch(pl->exec, st);
    count_launch();
    if (e != cudaSuccess) {
        if (ce) *ce = e;
        return RB_ERR_CUDA;
    }
    return RB_OK;
}

void grouped_plan_destroy(void* plan) { delete static_cast<GroupedPlan*>(plan); }

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
