// rb_api.cu -- the extern "C" boundary (include/rblas_b200.h).
//
// Host entry points mirror rblas's slice-based Level-3 functions: argument
// order, validation order and error fields follow level3::try_gemm and
// check_matrix (src/level3.rs:68-140); the math follows level3::gemm
// (src/level3.rs:32-62) and gemm_contig's early-outs (src/kernel/gemm.rs:
// 185-205): m == 0 || n == 0 returns before touching C; otherwise C is scaled
// by beta (beta == 0 writes zeros without reading C, so NaNs in C vanish) and
// k == 0 || alpha == 0 stops there.
#include <cuda.h>
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/rblas_b200.h"
#include "rb_internal.h"
#include "rb_device.cuh"

namespace rb {

// ---- library scratch pool (one per device) ---------------------------------
namespace {
std::mutex g_pool_mu;
constexpr int kPoolDevices = 64;
cudaMemPool_t g_pools[kPoolDevices] = {};
std::atomic<uint64_t> g_scratch_cache{uint64_t(8) << 30};

cudaMemPool_t pool_for_current(cudaError_t* err) {
    int dev = 0;
    *err = cudaGetDevice(&dev);
    if (*err != cudaSuccess || dev < 0 || dev >= kPoolDevices) return nullptr;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        *err = cudaMemPoolCreate(&g_pools[dev], &props);
        if (*err != cudaSuccess) {
            g_pools[dev] = nullptr;
            return nullptr;
        }
        uint64_t thr = g_scratch_cache.load();
        cudaMemPoolSetAttribute(g_pools[dev], cudaMemPoolAttrReleaseThreshold, &thr);
    }
    return g_pools[dev];
}
}  // namespace

namespace {
std::atomic<uint64_t> g_device_allocs{0};
std::atomic<int64_t> g_inject_alloc{0};  // pending injected allocation failures
}  // namespace

void count_device_alloc() { g_device_allocs.fetch_add(1, std::memory_order_relaxed); }

bool take_injected_alloc_failure() {
    int64_t n = g_inject_alloc.load();
    while (n > 0)
        if (g_inject_alloc.compare_exchange_weak(n, n - 1)) return true;
    return false;
}

cudaError_t dev_alloc(void** p, size_t bytes) {
    count_device_alloc();
    if (take_injected_alloc_failure()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMalloc(p, bytes);
}

cudaError_t scratch_alloc_raw(void** p, size_t bytes, cudaStream_t st) {
    count_device_alloc();
    if (take_injected_alloc_failure()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    cudaError_t e;
    cudaMemPool_t pool = pool_for_current(&e);
    if (!pool) return e == cudaSuccess ? cudaErrorMemoryAllocation : e;
    return cudaMallocFromPoolAsync(p, bytes, pool, st);
}

void scratch_reserve(size_t bytes) {
    cudaError_t e;
    cudaMemPool_t pool = pool_for_current(&e);
    if (!pool || bytes == 0) return;
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return;
    void* p = nullptr;
    if (cudaMallocFromPoolAsync(&p, bytes, pool, st) == cudaSuccess) cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
}

void scratch_trim() {
    cudaError_t e;
    cudaMemPool_t pool = pool_for_current(&e);
    if (pool) cudaMemPoolTrimTo(pool, 0);
}

void set_scratch_cache_bytes(size_t bytes) {
    g_scratch_cache.store(bytes);
    std::lock_guard<std::mutex> lk(g_pool_mu);
    uint64_t thr = bytes;
    for (auto& pl : g_pools)
        if (pl) cudaMemPoolSetAttribute(pl, cudaMemPoolAttrReleaseThreshold, &thr);
}

}  // namespace rb

namespace rb {

std::atomic<uint64_t> g_launches{0};

// ---- kernel timing registry ---------------------------------------------------
namespace {
struct TimedLaunch {
    std::string name;
    double work;
    cudaEvent_t e0, e1;
    int dev;
};
std::mutex g_timing_mu;
std::atomic<bool> g_timing_on{false};
std::vector<TimedLaunch*> g_timed;
// events of reported launches, reused per device: creating two per launch
// cost more host time than a short kernel runs, so the timed region starved
// the GPU
std::map<int, std::vector<cudaEvent_t>> g_event_pool;

cudaEvent_t pooled_event(int dev) {
    {
        std::lock_guard<std::mutex> lk(g_timing_mu);
        std::vector<cudaEvent_t>& v = g_event_pool[dev];
        if (!v.empty()) {
            cudaEvent_t e = v.back();
            v.pop_back();
            return e;
        }
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}
}  // namespace

bool kernel_timing_on() { return g_timing_on.load(std::memory_order_relaxed); }

void kernel_timing_begin(const char* name, double work, cudaStream_t st, KernelTimer* t) {
    t->slot = nullptr;
    if (!kernel_timing_on()) return;
    int dev = 0;
    cudaGetDevice(&dev);
    TimedLaunch* L = new TimedLaunch{name, work, pooled_event(dev), pooled_event(dev), dev};
    cudaEventRecord(L->e0, st);
    t->slot = L;
}

void kernel_timing_end(KernelTimer* t, cudaStream_t st) {
    if (!t->slot) return;
    TimedLaunch* L = static_cast<TimedLaunch*>(t->slot);
    cudaEventRecord(L->e1, st);
    std::lock_guard<std::mutex> lk(g_timing_mu);
    g_timed.push_back(L);
}
static std::atomic<int> g_ozaki_slices{8};
static int ozaki_slices() { return g_ozaki_slices.load(); }

namespace {

constexpr int kMaxDevices = 64;

// Per-device state for host-slice calls: an internal stream, grow-only
// staging buffers for A, B, C, and the device error word.
constexpr int kHostSplit = 8;                   // panels of a large host-slice call, by width
constexpr int kHostPanels = kHostSplit + 1;     // the last one split in two

struct DeviceCtx {
    std::mutex mu;
    bool init = false;
    cudaStream_t stream = nullptr;
    cudaStream_t pstream[kHostPanels] = {};  // one per panel of a pipelined host call
    cudaEvent_t a_ready = nullptr, pdone[kHostPanels] = {};
    uint32_t* err_word = nullptr;
    void* buf[3] = {nullptr, nullptr, nullptr};
    size_t cap[3] = {0, 0, 0};
};
DeviceCtx g_ctx[kMaxDevices];
std::mutex g_init_mu;

int current_device() {
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess) return -1;
    return d;
}

DeviceCtx* ctx_for_current(cudaError_t* e) {
    const int d = current_device();
    if (d < 0 || d >= kMaxDevices) {
        *e = cudaErrorInvalidDevice;
        return nullptr;
    }
    DeviceCtx& c = g_ctx[d];
    std::lock_guard<std::mutex> lk(g_init_mu);
    if (!c.init) {
        *e = cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking);
        if (*e != cudaSuccess) return nullptr;
        count_device_alloc();
        *e = cudaMalloc(&c.err_word, 64);
        if (*e != cudaSuccess) return nullptr;
        *e = cudaMemset(c.err_word, 0, 64);
        if (*e != cudaSuccess) return nullptr;
        *e = cudaEventCreateWithFlags(&c.a_ready, cudaEventDisableTiming);
        for (int i = 0; i < kHostPanels && *e == cudaSuccess; ++i) {
            *e = cudaStreamCreateWithFlags(&c.pstream[i], cudaStreamNonBlocking);
            if (*e == cudaSuccess) *e = cudaEventCreateWithFlags(&c.pdone[i], cudaEventDisableTiming);
        }
        if (*e != cudaSuccess) return nullptr;
        c.init = true;
    }
    *e = cudaSuccess;
    return &c;
}

// Panels of a pipelined host call along `extent`: widths of a multiple of
// 256 (every kernel's tile width divides 256, and offsets stay 16-byte
// aligned) giving at most kHostSplit panels; the last one, when at least 512
// wide, is split in two, so the GEMM and download that wait behind the last
// upload are half as long. Returns the number of panels.
int panel_plan(size_t extent, size_t* lens) {
    const size_t width = std::max<size_t>(256, (extent + kHostSplit * 256 - 1) / (kHostSplit * 256) * 256);
    int np = 0;
    for (size_t off = 0; off < extent; off += lens[np++]) lens[np] = std::min(width, extent - off);
    if (np > 0 && np < kHostPanels && lens[np - 1] >= 512) {
        const size_t first = (lens[np - 1] / 2 + 255) / 256 * 256;
        lens[np] = lens[np - 1] - first;
        lens[np - 1] = first;
        ++np;
    }
    return np;
}

cudaError_t ensure_buf(DeviceCtx* c, int slot, size_t bytes) {
    if (bytes <= c->cap[slot]) return cudaSuccess;
    if (c->buf[slot]) cudaFree(c->buf[slot]);
    c->buf[slot] = nullptr;
    c->cap[slot] = 0;
    size_t want = std::max(bytes, c->cap[slot] * 2);
    cudaError_t e = dev_alloc(&c->buf[slot], want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (want == bytes) return e;
        e = dev_alloc(&c->buf[slot], bytes);
        if (e != cudaSuccess) return e;
        want = bytes;
    }
    c->cap[slot] = want;
    return cudaSuccess;
}

void set_err(rb_error* err, int32_t code, char which = 0, uint64_t got = 0, uint64_t need = 0,
             int32_t cuda_error = 0) {
    if (err) {
        err->code = code;
        err->which = which;
        err->got = got;
        err->min_or_need = need;
        err->cuda_error = cuda_error;
    }
}

// A failed CUDA call; an out-of-memory one is RB_ERR_ALLOC (cuda_error keeps
// the CUDA code either way).
rb_status cuda_fail(rb_error* err, cudaError_t e) {
    const rb_status s = (e == cudaErrorMemoryAllocation) ? RB_ERR_ALLOC : RB_ERR_CUDA;
    if (s == RB_ERR_ALLOC) cudaGetLastError();  // not sticky: clear it for the next call
    set_err(err, s, 0, 0, 0, static_cast<int32_t>(e));
    return s;
}

// src/level3.rs:107-140. Zero dims are valid; InvalidLeadingDim before
// BufferTooSmall. check_len == false skips the length check (device calls).
rb_status check_matrix(rb_layout layout, char which, size_t rows, size_t cols, size_t lead,
                       size_t len, bool check_len, rb_error* err) {
    if (rows == 0 || cols == 0) return RB_OK;
    const size_t min_lead = (layout == RB_ROW_MAJOR) ? cols : rows;
    if (lead < min_lead) {
        set_err(err, RB_ERR_INVALID_LEADING_DIM, which, lead, min_lead);
        return RB_ERR_INVALID_LEADING_DIM;
    }
    const size_t need = (layout == RB_ROW_MAJOR) ? (rows - 1) * lead + cols : (cols - 1) * lead + rows;
    if (check_len && len < need) {
        set_err(err, RB_ERR_BUFFER_TOO_SMALL, which, len, need);
        return RB_ERR_BUFFER_TOO_SMALL;
    }
    return RB_OK;
}

bool valid_layout(int v) { return v == RB_ROW_MAJOR || v == RB_COL_MAJOR; }
bool valid_trans(int v) { return v >= RB_NO_TRANS && v <= RB_CONJ_TRANS; }
bool valid_prec(int v) { return v >= RB_PREC_PLAIN && v <= RB_PREC_BF16X6; }

// A GEMM problem after row-major normalisation (src/level3.rs:52-60):
// column-major, C is m x n; op(A) m x k; op(B) k x n.
template <typename T>
struct ColProblem {
    bool ta, tb;
    size_t m, n, k;
    T alpha, beta;
    const T* a; size_t lda;
    const T* b; size_t ldb;
    T* c; size_t ldc;
    int tri = 0;  // syrk: restrict C to one triangle
    bool split_ok = true;  // the plain form may take the grouped kernel's split-K
};

// The plain problem as one grouped-kernel entry; true when the grouped
// kernel's shape rule splits its K (fewer C tiles than SMs and a long K).
template <typename T>
bool plain_split(const ColProblem<T>& p, rb_gemm_problem* q) {
    *q = rb_gemm_problem{};
    q->dtype = sizeof(T) == 8 ? 1 : 0;
    q->layout = RB_COL_MAJOR;
    q->transa = p.ta ? RB_TRANS : RB_NO_TRANS;
    q->transb = p.tb ? RB_TRANS : RB_NO_TRANS;
    q->m = p.m; q->n = p.n; q->k = p.k;
    q->alpha = static_cast<double>(p.alpha);
    q->beta = static_cast<double>(p.beta);
    q->a = p.a; q->lda = p.lda;
    q->b = p.b; q->ldb = p.ldb;
    q->c = p.c; q->ldc = p.ldc;
    // an f32 problem the narrow tile fills the GPU with runs unsplit
    if (sizeof(T) == 4 && simt_narrow_f32(p.m, p.n)) return false;
    return !p.tri && grouped_splits(*q) > 1;
}

template <typename T>
ColProblem<T> normalise(rb_layout layout, rb_transpose transa, rb_transpose transb, size_t m,
                        size_t n, size_t k, T alpha, const T* a, size_t lda, const T* b, size_t ldb,
                        T beta, T* c, size_t ldc) {
    ColProblem<T> p;
    if (layout == RB_COL_MAJOR) {
        p = {transa != RB_NO_TRANS, transb != RB_NO_TRANS, m, n, k, alpha, beta, a, lda, b, ldb, c, ldc};
    } else {
        // C^T = alpha * op(B)^T op(A)^T + beta * C^T: swap A<->B, m<->n, trans flags.
        p = {transb != RB_NO_TRANS, transa != RB_NO_TRANS, n, m, k, alpha, beta, b, ldb, a, lda, c, ldc};
    }
    return p;
}

constexpr size_t kMaxDim = 0x7fffffff;

template <typename T>
bool tma_ok(const T* p, size_t ld) {
    return (reinterpret_cast<uintptr_t>(p) % 16 == 0) && ((ld * sizeof(T)) % 16 == 0);
}

// The split-precision forms: BF16X3 for f32, OZAKI for f64. Their pre-pass
// reads the operands with plain loads, so no TMA alignment repack is needed.
template <typename T>
rb_status run_precision_form(const ColProblem<T>& p, rb_precision prec, cudaStream_t st, rb_error* err) {
    cudaError_t e;
    CUresult cu = CUDA_SUCCESS;
    if constexpr (sizeof(T) == 4) {
        if (prec != RB_PREC_BF16X3 && prec != RB_PREC_BF16X6) {
            set_err(err, RB_ERR_UNSUPPORTED);
            return RB_ERR_UNSUPPORTED;
        }
        e = launch_bf16_split_gemm(prec == RB_PREC_BF16X3 ? 2 : 3, p.ta, p.tb, (int)p.m, (int)p.n, (int)p.k,
                                   p.alpha, p.a, p.lda, p.b, p.ldb, p.beta, p.c, p.ldc, st, &cu);
    } else {
        if (prec != RB_PREC_OZAKI) {
            set_err(err, RB_ERR_UNSUPPORTED);
            return RB_ERR_UNSUPPORTED;
        }
        e = launch_ozaki_gemm(p.ta, p.tb, (int)p.m, (int)p.n, (int)p.k, p.alpha, p.a, p.lda, p.b, p.ldb,
                              p.beta, p.c, p.ldc, ozaki_slices(), st, &cu);
    }
    if (cu != CUDA_SUCCESS) {
        set_err(err, RB_ERR_CUDA, 0, 0, 0, static_cast<int32_t>(cu));
        return RB_ERR_CUDA;
    }
    return e == cudaSuccess ? RB_OK : cuda_fail(err, e);
}

// Enqueue the column-major problem on `st` with device operands. Operands
// that TMA cannot address directly (unaligned base or leading dimension) are
// repacked into stream-ordered scratch first.
template <typename T>
rb_status run_dev(const ColProblem<T>& p, rb_precision prec, cudaStream_t st, rb_error* err) {
    if (p.m == 0 || p.n == 0) return RB_OK;
    if (p.m > kMaxDim || p.n > kMaxDim || p.k > kMaxDim) {
        set_err(err, RB_ERR_INVALID_ARG);
        return RB_ERR_INVALID_ARG;
    }
    cudaError_t e;
    if (p.k == 0 || p.alpha == T(0)) {
        e = launch_scale_c<T>((int)p.m, (int)p.n, p.beta, p.c, p.ldc, st, p.tri);
        return e == cudaSuccess ? RB_OK : cuda_fail(err, e);
    }
    if (prec != RB_PREC_PLAIN) {
        if (p.tri) {
            set_err(err, RB_ERR_UNSUPPORTED);
            return RB_ERR_UNSUPPORTED;
        }
        return run_precision_form(p, prec, st, err);
    }
    // Fewer C tiles than SMs and a long K (the 1024^3 SGEMM: 64 tiles): the
    // grouped kernel's deterministic split-K fills the GPU. The factor
    // depends on the shape alone, so a call's bits repeat from call to call.
    rb_gemm_problem gq;
    if (p.split_ok && plain_split(p, &gq)) {
        int32_t ce = 0;
        const int rc = grouped_gemm_dev(&gq, 1, nullptr, nullptr, st, &ce, nullptr);
        if (rc != RB_OK) set_err(err, rc, 0, 0, 0, ce);
        return static_cast<rb_status>(rc);
    }
    const T* A = p.a;
    const T* B = p.b;
    size_t lda = p.lda, ldb = p.ldb;
    void* scratch[2] = {nullptr, nullptr};
    const size_t vec = 16 / sizeof(T);
    // stored extents (column-major)
    const size_t a_rows = p.ta ? p.k : p.m, a_cols = p.ta ? p.m : p.k;
    const size_t b_rows = p.tb ? p.n : p.k, b_cols = p.tb ? p.k : p.n;
    if (!tma_ok(A, lda)) {
        const size_t ld2 = (a_rows + vec - 1) / vec * vec;
        e = scratch_alloc(&scratch[0], ld2 * a_cols * sizeof(T), st);
        if (e != cudaSuccess) return cuda_fail(err, e);
        e = cudaMemcpy2DAsync(scratch[0], ld2 * sizeof(T), A, lda * sizeof(T), a_rows * sizeof(T),
                              a_cols, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return cuda_fail(err, e);
        A = static_cast<const T*>(scratch[0]);
        lda = ld2;
    }
    if (!tma_ok(B, ldb)) {
        const size_t ld2 = (b_rows + vec - 1) / vec * vec;
        e = scratch_alloc(&scratch[1], ld2 * b_cols * sizeof(T), st);
        if (e != cudaSuccess) return cuda_fail(err, e);
        e = cudaMemcpy2DAsync(scratch[1], ld2 * sizeof(T), B, ldb * sizeof(T), b_rows * sizeof(T),
                              b_cols, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return cuda_fail(err, e);
        B = static_cast<const T*>(scratch[1]);
        ldb = ld2;
    }
    CUresult cu = CUDA_SUCCESS;
    // op(A): Trans -> stored k x m, k-contiguous; op(B): NoTrans -> stored k x n, k-contiguous.
    e = launch_simt_gemm<T>(p.ta, !p.tb, (int)p.m, (int)p.n, (int)p.k, p.alpha, A, lda, B, ldb,
                            p.beta, p.c, p.ldc, st, &cu, p.tri);
    for (void* s : scratch)
        if (s) cudaFreeAsync(s, st);
    if (cu != CUDA_SUCCESS) {
        set_err(err, RB_ERR_CUDA, 0, 0, 0, static_cast<int32_t>(cu));
        return RB_ERR_CUDA;
    }
    return e == cudaSuccess ? RB_OK : cuda_fail(err, e);
}

rb_status check_device_word(DeviceCtx* c, rb_error* err) {
    uint32_t w = 0;
    cudaError_t e = cudaMemcpyAsync(&w, c->err_word, sizeof(w), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(err, e);
    if (w != 0) {
        cudaMemsetAsync(c->err_word, 0, sizeof(uint32_t), c->stream);
        cudaStreamSynchronize(c->stream);
        const rb_status s = ((w >> 24) == (RB_DEVERR_TIMEOUT >> 24)) ? RB_ERR_TIMEOUT : RB_ERR_DEVICE;
        set_err(err, s, 0, w, 0);
        return s;
    }
    return RB_OK;
}

// Host-slice GEMM: validate (try_gemm), stage into device buffers with padded
// leading dimensions, run, copy C back, report any device error.
template <typename T>
rb_status host_gemm(rb_layout layout, rb_transpose transa, rb_transpose transb, size_t m, size_t n,
                    size_t k, T alpha, const T* a, size_t lda, size_t a_len, const T* b, size_t ldb,
                    size_t b_len, T beta, T* c, size_t ldc, size_t c_len, rb_precision prec,
                    rb_error* err) {
    set_err(err, RB_OK);
    if (!valid_layout(layout) || !valid_trans(transa) || !valid_trans(transb) ||
        !valid_prec(prec)) {
        set_err(err, RB_ERR_INVALID_ARG);
        return RB_ERR_INVALID_ARG;
    }
    // src/level3.rs:86-98: stored shapes, then a, b, c in that order.
    const bool ta = transa != RB_NO_TRANS, tb = transb != RB_NO_TRANS;
    const size_t ar = ta ? k : m, ac = ta ? m : k;
    const size_t br = tb ? n : k, bc = tb ? k : n;
    rb_status s;
    if ((s = check_matrix(layout, 'a', ar, ac, lda, a_len, true, err)) != RB_OK) return s;
    if ((s = check_matrix(layout, 'b', br, bc, ldb, b_len, true, err)) != RB_OK) return s;
    if ((s = check_matrix(layout, 'c', m, n, ldc, c_len, true, err)) != RB_OK) return s;
    if (m == 0 || n == 0) return RB_OK;  // src/kernel/gemm.rs:198-200
    if ((k > 0 && (!a || !b)) || !c) {
        set_err(err, RB_ERR_INVALID_ARG);
        return RB_ERR_INVALID_ARG;
    }

    cudaError_t e;
    DeviceCtx* ctx = ctx_for_current(&e);
    if (!ctx) return cuda_fail(err, e);
    std::lock_guard<std::mutex> lk(ctx->mu);

    ColProblem<T> p = normalise<T>(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
    const size_t vec = 16 / sizeof(T);
    const bool need_ab = p.k > 0 && p.alpha != T(0);
    const bool read_c = p.beta != T(0);
    // column-major stored extents after normalisation
    const size_t a_rows = p.ta ? p.k : p.m, a_cols = p.ta ? p.m : p.k;
    const size_t b_rows = p.tb ? p.n : p.k, b_cols = p.tb ? p.k : p.n;
    const size_t lda_d = (a_rows + vec - 1) / vec * vec;
    const size_t ldb_d = (b_rows + vec - 1) / vec * vec;
    const size_t ldc_d = (p.m + vec - 1) / vec * vec;

    if (need_ab) {
        if ((e = ensure_buf(ctx, 0, lda_d * a_cols * sizeof(T))) != cudaSuccess) return cuda_fail(err, e);
        if ((e = ensure_buf(ctx, 1, ldb_d * b_cols * sizeof(T))) != cudaSuccess) return cuda_fail(err, e);
    }
    if ((e = ensure_buf(ctx, 2, ldc_d * p.n * sizeof(T))) != cudaSuccess) return cuda_fail(err, e);
    T* dA = static_cast<T*>(ctx->buf[0]);
    T* dB = static_cast<T*>(ctx->buf[1]);
    T* dC = static_cast<T*>(ctx->buf[2]);
    cudaStream_t st = ctx->stream;

    // Large calls run as column panels of C (and of op(B)), each on its own
    // stream, after A has been uploaded once: one panel's upload, GEMM and
    // download overlap the others' (host-to-device and device-to-host copies
    // use separate engines). Every element of C is computed from the same
    // operands in the same order as in one whole call, so results are the
    // same bit for bit. Panels start at multiples of 256 columns
    // (panel_plan).
    const size_t el = sizeof(T);
    const size_t total_bytes = (need_ab ? (a_rows * a_cols + b_rows * b_cols) * el : 0) +
                               p.m * p.n * el * (read_c ? 2 : 1);
    // a plain call whose whole shape takes split-K runs whole (a panel's
    // split could differ, and with it the summation order), and so does one
    // whose C the narrow f32 tile spreads over the SMs (its panels would not)
    rb_gemm_problem whole;
    const bool whole_call = prec == RB_PREC_PLAIN &&
                            (plain_split(p, &whole) || (sizeof(T) == 4 && simt_narrow_f32(p.m, p.n)));
    if (total_bytes >= (size_t(64) << 20) && p.n >= 2 * 256 && !whole_call) {
        size_t lens[kHostPanels];
        const int np = panel_plan(p.n, lens);
        if (need_ab) {
            e = cudaMemcpy2DAsync(dA, lda_d * el, p.a, p.lda * el, a_rows * el, a_cols, cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) return cuda_fail(err, e);
        }
        if ((e = cudaEventRecord(ctx->a_ready, st)) != cudaSuccess) return cuda_fail(err, e);
        rb_status ps = RB_OK;
        int used = 0;
        for (size_t j0 = 0; used < np && ps == RB_OK; j0 += lens[used], ++used) {
            const size_t jn = lens[used];
            cudaStream_t sp = ctx->pstream[used];
            e = cudaStreamWaitEvent(sp, ctx->a_ready, 0);
            if (e == cudaSuccess && need_ab) {
                if (p.tb)  // op(B) columns j0.. are rows j0.. of the stored n x k B
                    e = cudaMemcpy2DAsync(dB + j0, ldb_d * el, p.b + j0, p.ldb * el, jn * el, b_cols,
                                          cudaMemcpyHostToDevice, sp);
                else
                    e = cudaMemcpy2DAsync(dB + j0 * ldb_d, ldb_d * el, p.b + j0 * p.ldb, p.ldb * el, b_rows * el, jn,
                                          cudaMemcpyHostToDevice, sp);
            }
            if (e == cudaSuccess && read_c)
                e = cudaMemcpy2DAsync(dC + j0 * ldc_d, ldc_d * el, p.c + j0 * p.ldc, p.ldc * el, p.m * el, jn,
                                      cudaMemcpyHostToDevice, sp);
            if (e != cudaSuccess) {
                ps = cuda_fail(err, e);
                break;
            }
            ColProblem<T> q = p;
            q.n = jn;
            q.split_ok = false;  // as in the whole call
            q.a = dA; q.lda = lda_d;
            q.b = p.tb ? dB + j0 : dB + j0 * ldb_d; q.ldb = ldb_d;
            q.c = dC + j0 * ldc_d; q.ldc = ldc_d;
            ps = run_dev<T>(q, prec, sp, err);
            if (ps != RB_OK) break;
            e = cudaMemcpy2DAsync(p.c + j0 * p.ldc, p.ldc * el, dC + j0 * ldc_d, ldc_d * el, p.m * el, jn,
                                  cudaMemcpyDeviceToHost, sp);
            if (e == cudaSuccess) e = cudaEventRecord(ctx->pdone[used], sp);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ctx->pdone[used], 0);
            if (e != cudaSuccess) ps = cuda_fail(err, e);
        }
        if (ps != RB_OK) {
            for (int i = 0; i < used + 1 && i < kHostPanels; ++i) cudaStreamSynchronize(ctx->pstream[i]);
            return ps;
        }
        return check_device_word(ctx, err);
    }

    if (need_ab) {
        e = cudaMemcpy2DAsync(dA, lda_d * sizeof(T), p.a, p.lda * sizeof(T), a_rows * sizeof(T), a_cols,
                              cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(dB, ldb_d * sizeof(T), p.b, p.ldb * sizeof(T), b_rows * sizeof(T),
                                  b_cols, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return cuda_fail(err, e);
    }
    if (read_c) {
        e = cudaMemcpy2DAsync(dC, ldc_d * sizeof(T), p.c, p.ldc * sizeof(T), p.m * sizeof(T), p.n,
                              cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return cuda_fail(err, e);
    }
    ColProblem<T> q = p;
    q.a = dA; q.lda = lda_d;
    q.b = dB; q.ldb = ldb_d;
    q.c = dC; q.ldc = ldc_d;
    // beta == 0: C is never uploaded nor read (apply_beta writes zeros).
    s = run_dev<T>(q, prec, st, err);
    if (s != RB_OK) return s;
    e = cudaMemcpy2DAsync(p.c, p.ldc * sizeof(T), dC, ldc_d * sizeof(T), p.m * sizeof(T), p.n,
                          cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return cuda_fail(err, e);
    return check_device_word(ctx, err);
}

template <typename T>
rb_status dev_gemm(rb_layout layout, rb_transpose transa, rb_transpose transb, size_t m, size_t n,
                   size_t k, T alpha, const T* a, size_t lda, const T* b, size_t ldb, T beta, T* c,
                   size_t ldc, rb_precision prec, void* stream, rb_error* err) {
    set_err(err, RB_OK);
    if (!valid_layout(layout) || !valid_trans(transa) || !valid_trans(transb) ||
        !valid_prec(prec)) {
        set_err(err, RB_ERR_INVALID_ARG);
        return RB_ERR_INVALID_ARG;
    }
    const bool ta = transa != RB_NO_TRANS, tb = transb != RB_NO_TRANS;
    rb_status s;
    if ((s = check_matrix(layout, 'a', ta ? k : m, ta ? m : k, lda, 0, false, err)) != RB_OK) return s;
    if ((s = check_matrix(layout, 'b', tb ? n : k, tb ? k : n, ldb, 0, false, err)) != RB_OK) return s;
    if ((s = check_matrix(layout, 'c', m, n, ldc, 0, false, err)) != RB_OK) return s;
    if (m == 0 || n == 0) return RB_OK;
    if ((k > 0 && (!a || !b)) || !c) {
        set_err(err, RB_ERR_INVALID_ARG);
        return RB_ERR_INVALID_ARG;
    }
    cudaError_t e;
    if (!ctx_for_current(&e)) return cuda_fail(err, e);
    ColProblem<T> p = normalise<T>(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
    return run_dev<T>(p, prec, static_cast<cudaStream_t>(stream), err);
}

// A host buffer holding a stored rows x cols column-major matrix (`elem`
// bytes per element) with leading dimension ld.
struct HostMat {
    const void* src;  // host pointer read (may be null when !in)
    void* dst;        // host pointer written back (null when !out)
    size_t rows, cols, ld, elem;
    bool in, out;
};

// Stage up to three matrices into the device context's buffers (leading
// dimensions padded to 16 bytes), run `body(dev_ptrs, dev_lds, stream,
// &cuda_err)` on the internal stream, copy results back, and report any
// device-side error word.
template <typename F>
rb_status host_run(HostMat* mats, int nm, rb_error* err, F&& body) {
    cudaError_t e;
    DeviceCtx* ctx = ctx_for_current(&e);
    if (!ctx) return cuda_fail(err, e);
    std::lock_guard<std::mutex> lk(ctx->mu);
    void* dptr[3] = {nullptr, nullptr, nullptr};
    size_t dld[3] = {0, 0, 0};
    for (int i = 0; i < nm; ++i) {
        HostMat& h = mats[i];
        const size_t per16 = (h.elem >= 16) ? 1 : 16 / h.elem;
        dld[i] = std::max<size_t>((h.rows + per16 - 1) / per16 * per16, per16);
        const size_t bytes = dld[i] * std::max<size_t>(h.cols, 1) * h.elem;
        if ((e = ensure_buf(ctx, i, bytes)) != cudaSuccess) return cuda_fail(err, e);
        dptr[i] = ctx->buf[i];
        if (h.in && h.rows && h.cols) {
            e = cudaMemcpy2DAsync(dptr[i], dld[i] * h.elem, h.src, h.ld * h.elem, h.rows * h.elem, h.cols,
                                  cudaMemcpyHostToDevice, ctx->stream);
            if (e != cudaSuccess) return cuda_fail(err, e);
        }
    }
    int32_t ce = 0;
    const int rc = body(dptr, dld, ctx->stream, &ce);
    if (rc != RB_OK) {
        cudaStreamSynchronize(ctx->stream);
        set_err(err, rc, 0, 0, 0, ce);
        return static_cast<rb_status>(rc);
    }
    for (int i = 0; i < nm; ++i) {
        HostMat& h = mats[i];
        if (h.out && h.rows && h.cols) {
            e = cudaMemcpy2DAsync(h.dst, h.ld * h.elem, dptr[i], dld[i] * h.elem, h.rows * h.elem, h.cols,
                                  cudaMemcpyDeviceToHost, ctx->stream);
            if (e != cudaSuccess) return cuda_fail(err, e);
        }
    }
    return check_device_word(ctx, err);
}

// A Level-3 host call whose first matrix (the triangular or symmetric A) is
// needed whole and whose other matrices (B, and C) split into independent
// panels along `extent`: columns (by_cols) or rows. A is uploaded once and
// `prologue(dA, ldA, stream, &cuda_err)` runs on it on the internal stream;
// then each panel's slices of the other matrices are uploaded, computed by
// `panel(dA, ldA, dev_ptrs, dev_lds, offset, length, stream, &cuda_err)`
// (dev_ptrs at the panel's first row / column) and downloaded on a panel
// stream of its own, so the copies of different panels overlap each other
// and the kernels (uploads and downloads use separate copy engines);
// `finish(stream)` runs on the internal stream after every panel. Calls
// under 64 MB, or too narrow for two 256-wide panels, run whole through
// host_run.
template <typename Pro, typename Pan, typename Fin>
rb_status host_run_split(HostMat* mats, int nm, bool by_cols, size_t extent, rb_error* err, Pro&& prologue,
                         Pan&& panel, Fin&& finish) {
    size_t total = 0;
    for (int i = 0; i < nm; ++i)
        total += mats[i].rows * mats[i].cols * mats[i].elem * ((mats[i].in ? 1 : 0) + (mats[i].out ? 1 : 0));
    if (total < (size_t(64) << 20) || extent < 2 * 256) {
        return host_run(mats, nm, err, [&](void** d, size_t* ld, cudaStream_t st, int32_t* ce) {
            int rc = prologue(d[0], ld[0], st, ce);
            if (rc == RB_OK) rc = panel(d[0], ld[0], d + 1, ld + 1, size_t(0), extent, st, ce);
            finish(st);
            return rc;
        });
    }
    cudaError_t e;
    DeviceCtx* ctx = ctx_for_current(&e);
    if (!ctx) return cuda_fail(err, e);
    std::lock_guard<std::mutex> lk(ctx->mu);
    void* dptr[3] = {nullptr, nullptr, nullptr};
    size_t dld[3] = {0, 0, 0};
    for (int i = 0; i < nm; ++i) {
        const HostMat& h = mats[i];
        const size_t per16 = (h.elem >= 16) ? 1 : 16 / h.elem;
        dld[i] = std::max<size_t>((h.rows + per16 - 1) / per16 * per16, per16);
        if ((e = ensure_buf(ctx, i, dld[i] * std::max<size_t>(h.cols, 1) * h.elem)) != cudaSuccess)
            return cuda_fail(err, e);
        dptr[i] = ctx->buf[i];
    }
    cudaStream_t st = ctx->stream;
    const HostMat& a = mats[0];
    e = cudaMemcpy2DAsync(dptr[0], dld[0] * a.elem, a.src, a.ld * a.elem, a.rows * a.elem, a.cols,
                          cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(err, e);
    int32_t ce = 0;
    int rc = prologue(dptr[0], dld[0], st, &ce);
    if (rc != RB_OK) {
        finish(st);
        cudaStreamSynchronize(st);
        set_err(err, rc, 0, 0, 0, ce);
        return static_cast<rb_status>(rc);
    }
    if ((e = cudaEventRecord(ctx->a_ready, st)) != cudaSuccess) return cuda_fail(err, e);
    // the slice [off, off + len) of matrix i along the split, on the host and on the device
    auto copy = [&](int i, size_t off, size_t len, bool up, cudaStream_t sp) -> cudaError_t {
        const HostMat& h = mats[i];
        const size_t el = h.elem;
        uint8_t* dev = static_cast<uint8_t*>(dptr[i]) + (by_cols ? off * dld[i] : off) * el;
        const size_t hoff = (by_cols ? off * h.ld : off) * el;
        const size_t width = (by_cols ? h.rows : len) * el, height = by_cols ? len : h.cols;
        if (up)
            return cudaMemcpy2DAsync(dev, dld[i] * el, static_cast<const uint8_t*>(h.src) + hoff, h.ld * el, width,
                                     height, cudaMemcpyHostToDevice, sp);
        return cudaMemcpy2DAsync(static_cast<uint8_t*>(h.dst) + hoff, h.ld * el, dev, dld[i] * el, width, height,
                                 cudaMemcpyDeviceToHost, sp);
    };
    size_t lens[kHostPanels];
    const int np = panel_plan(extent, lens);
    rb_status ps = RB_OK;
    int used = 0;
    for (size_t off = 0; used < np && ps == RB_OK; off += lens[used], ++used) {
        const size_t len = lens[used];
        cudaStream_t sp = ctx->pstream[used];
        e = cudaStreamWaitEvent(sp, ctx->a_ready, 0);
        for (int i = 1; i < nm && e == cudaSuccess; ++i)
            if (mats[i].in) e = copy(i, off, len, true, sp);
        if (e != cudaSuccess) {
            ps = cuda_fail(err, e);
            break;
        }
        void* pp[2] = {nullptr, nullptr};
        for (int i = 1; i < nm; ++i)
            pp[i - 1] = static_cast<uint8_t*>(dptr[i]) + (by_cols ? off * dld[i] : off) * mats[i].elem;
        rc = panel(dptr[0], dld[0], pp, dld + 1, off, len, sp, &ce);
        if (rc != RB_OK) {
            set_err(err, rc, 0, 0, 0, ce);
            ps = static_cast<rb_status>(rc);
            break;
        }
        for (int i = 1; i < nm && e == cudaSuccess; ++i)
            if (mats[i].out) e = copy(i, off, len, false, sp);
        if (e == cudaSuccess) e = cudaEventRecord(ctx->pdone[used], sp);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ctx->pdone[used], 0);
        if (e != cudaSuccess) ps = cuda_fail(err, e);
    }
    if (ps != RB_OK) {
        for (int i = 0; i < used + 1 && i < kHostPanels; ++i) cudaStreamSynchronize(ctx->pstream[i]);
        finish(st);
        cudaStreamSynchronize(st);
        return ps;
    }
    finish(st);
    return check_device_word(ctx, err);
}

bool valid_uplo(int v) { return v == RB_UPPER || v == RB_LOWER; }
bool valid_side(int v) { return v == RB_LEFT || v == RB_RIGHT; }
bool valid_diag(int v) { return v == RB_NON_UNIT || v == RB_UNIT; }

rb_status invalid(rb_error* err) {
    set_err(err, RB_ERR_INVALID_ARG);
    return RB_ERR_INVALID_ARG;
}

}  // namespace

template <typename T>
int gemm_colmajor_dev(bool ta, bool tb, size_t m, size_t n, size_t k, T alpha, const T* A,
                      size_t lda, const T* B, size_t ldb, T beta, T* C, size_t ldc, int prec,
                      cudaStream_t st, int tri, int32_t* cuda_err) {
    ColProblem<T> p{ta, tb, m, n, k, alpha, beta, A, lda, B, ldb, C, ldc, tri};
    rb_error e{};
    const rb_status s = run_dev<T>(p, static_cast<rb_precision>(prec), st, &e);
    if (cuda_err) *cuda_err = e.cuda_error;
    return s;
}
template int gemm_colmajor_dev<float>(bool, bool, size_t, size_t, size_t, float, const float*, size_t,
                                      const float*, size_t, float, float*, size_t, int, cudaStream_t,
                                      int, int32_t*);
template int gemm_colmajor_dev<double>(bool, bool, size_t, size_t, size_t, double, const double*,
                                       size_t, const double*, size_t, double, double*, size_t, int,
                                       cudaStream_t, int, int32_t*);

uint32_t* device_error_word() {
    cudaError_t e;
    DeviceCtx* c = ctx_for_current(&e);
    return c ? c->err_word : nullptr;
}

namespace {
constexpr int kAuxStreams = 4;
struct AuxSlot {
    std::mutex mu;
    bool init = false;
    cudaStream_t s = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};
AuxSlot g_aux[kMaxDevices][kAuxStreams];
}  // namespace

cudaError_t fork_stream(cudaStream_t st, ForkedStream* f) {
    const int d = current_device();
    if (d < 0 || d >= kMaxDevices) return cudaErrorInvalidDevice;
    const int slot = static_cast<int>((reinterpret_cast<uintptr_t>(st) >> 4) % kAuxStreams);
    AuxSlot& a = g_aux[d][slot];
    a.mu.lock();
    cudaError_t e = cudaSuccess;
    if (!a.init) {
        e = cudaStreamCreateWithFlags(&a.s, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&a.fork, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&a.join, cudaEventDisableTiming);
        a.init = e == cudaSuccess;
    }
    if (e == cudaSuccess) e = cudaEventRecord(a.fork, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(a.s, a.fork, 0);
    if (e != cudaSuccess) {
        a.mu.unlock();
        return e;
    }
    f->s = a.s;
    f->slot = d * kAuxStreams + slot;
    return cudaSuccess;
}

cudaError_t join_stream(cudaStream_t st, ForkedStream* f) {
    if (f->slot < 0) return cudaSuccess;
    AuxSlot& a = g_aux[f->slot / kAuxStreams][f->slot % kAuxStreams];
    cudaError_t e = cudaEventRecord(a.join, a.s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, a.join, 0);
    f->slot = -1;
    f->s = nullptr;
    a.mu.unlock();
    return e;
}

namespace {
// One thread waits on an mbarrier that expects one arrival and never gets
// it (the flag nothing sets): the bounded wait gives up after
// RB_WAIT_LIMIT_NS and records RB_DEVERR_TIMEOUT | kProbeWaitSite.
constexpr uint32_t kProbeWaitSite = 0x7F0;
__global__ void wait_timeout_probe_kernel(uint32_t* err, uint32_t* completed) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
        *completed = mbar_wait(&bar, 0, err, kProbeWaitSite) ? 1u : 0u;
    }
}
}  // namespace

}  // namespace rb

using namespace rb;

extern "C" {

const char* rb_status_string(int32_t status) {
    switch (status) {
        case RB_OK: return "ok";
        case RB_ERR_INVALID_LEADING_DIM: return "invalid leading dimension";
        case RB_ERR_BUFFER_TOO_SMALL: return "buffer too small";
        case RB_ERR_ZERO_STRIDE: return "stride must be positive (got 0)";
        case RB_ERR_INVALID_ARG: return "invalid argument";
        case RB_ERR_UNSUPPORTED: return "unsupported precision form for this operation";
        case RB_ERR_CUDA: return "CUDA error";
        case RB_ERR_ALLOC: return "allocation failed";
        case RB_ERR_TIMEOUT: return "device wait timed out";
        case RB_ERR_DEVICE: return "device-side error";
        case RB_ERR_BUSY: return "admission refused";
        case RB_ERR_CANCELLED: return "cancelled";
        case RB_ERR_SCRATCH_LIMIT: return "problem exceeds the fixed scratch of the allocation-free entry point";
        default: return "unknown status";
    }
}

rb_status rb_sgemm(rb_layout layout, rb_transpose transa, rb_transpose transb, size_t m, size_t n,
                   size_t k, float alpha, const float* a, size_t lda, size_t a_len, const float* b,
                   size_t ldb, size_t b_len, float beta, float* c, size_t ldc, size_t c_len,
                   rb_error* err) {
    return host_gemm<float>(layout, transa, transb, m, n, k, alpha, a, lda, a_len, b, ldb, b_len,
                            beta, c, ldc, c_len, RB_PREC_PLAIN, err);
}

rb_status rb_dgemm(rb_layout layout, rb_transpose transa, rb_transpose transb, size_t m, size_t n,
                   size_t k, double alpha, const double* a, size_t lda, size_t a_len,
                   const double* b, size_t ldb, size_t b_len, double beta, double* c, size_t ldc,
                   size_t c_len, rb_error* err) {
    return host_gemm<double>(layout, transa, transb, m, n, k, alpha, a, lda, a_len, b, ldb, b_len,
                             beta, c, ldc, c_len, RB_PREC_PLAIN, err);
}

rb_status rb_sgemm_prec(rb_layout layout, rb_transpose transa, rb_transpose transb, size_t m,
                        size_t n, size_t k, float alpha, const float* a, size_t lda, size_t a_len,
                        const float* b, size_t ldb, size_t b_len, float beta, float* c,
                        size_t ldc, size_t c_len, rb_precision prec, rb_error* err) {
    return host_gemm<float>(layout, transa, transb, m, n, k, alpha, a, lda, a_len, b, ldb, b_len,
                            beta, c, ldc, c_len, prec, err);
}

rb_status rb_dgemm_prec(rb_layout layout, rb_transpose transa, rb_transpose transb, size_t m,
                        size_t n, size_t k, double alpha, const double* a, size_t lda,
                        size_t a_len, const double* b, size_t ldb, size_t b_len, double beta,
                        double* c, size_t ldc, size_t c_len, rb_precision prec, rb_error* err) {
    return host_gemm<double>(layout, transa, transb, m, n, k, alpha, a, lda, a_len, b, ldb, b_len,
                             beta, c, ldc, c_len, prec, err);
}

rb_status rb_sgemm_dev(rb_layout layout, rb_transpose transa, rb_transpose transb, size_t m,
                       size_t n, size_t k, float alpha, const float* a, size_t lda,
                       const float* b, size_t ldb, float beta, float* c, size_t ldc,
                       rb_precision prec, void* stream, rb_error* err) {
    return dev_gemm<float>(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                           prec, stream, err);
}

rb_status rb_dgemm_dev(rb_layout layout, rb_transpose transa, rb_transpose transb, size_t m,
                       size_t n, size_t k, double alpha, const double* a, size_t lda,
                       const double* b, size_t ldb, double beta, double* c, size_t ldc,
                       rb_precision prec, void* stream, rb_error* err) {
    return dev_gemm<double>(layout, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc,
                            prec, stream, err);
}


rb_status rb_set_ozaki_slices(int slices) {
    if (slices < 2 || slices > 12) return RB_ERR_INVALID_ARG;
    g_ozaki_slices.store(slices);
    return RB_OK;
}

int rb_get_ozaki_slices(void) { return g_ozaki_slices.load(); }

uint64_t rb_launch_count(void) { return g_launches.load(); }

rb_status rb_device_error(int clear, uint32_t* detail) {
    cudaError_t e;
    DeviceCtx* c = ctx_for_current(&e);
    if (!c) return RB_ERR_CUDA;
    if (cudaDeviceSynchronize() != cudaSuccess) return RB_ERR_CUDA;
    uint32_t w = 0;
    if (cudaMemcpy(&w, c->err_word, sizeof(w), cudaMemcpyDeviceToHost) != cudaSuccess) return RB_ERR_CUDA;
    if (detail) *detail = w;
    if (clear && w) cudaMemset(c->err_word, 0, sizeof(uint32_t));
    if (w == 0) return RB_OK;
    return ((w >> 24) == (RB_DEVERR_TIMEOUT >> 24)) ? RB_ERR_TIMEOUT : RB_ERR_DEVICE;
}

size_t rb_num_threads(void) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();  // no usable device: leave no sticky error
        return 1;            // like rayon's pool size, never 0 (callers divide by it)
    }
    return sms > 0 ? static_cast<size_t>(sms) : 1;
}

uint64_t rb_device_alloc_count(void) { return g_device_allocs.load(); }

rb_status rb_debug_inject(int kind, uint32_t value, int count) {
    switch (kind) {
        case RB_INJECT_ALLOC:
            if (count < 0) return RB_ERR_INVALID_ARG;
            g_inject_alloc.store(count);
            return RB_OK;
        case RB_INJECT_DEVICE_WORD: {
            if (value == 0) return RB_ERR_INVALID_ARG;
            cudaError_t e;
            DeviceCtx* c = ctx_for_current(&e);
            if (!c) return RB_ERR_CUDA;
            // ordered after the work already queued on the device's streams
            // that use the word, like a kernel setting it
            if (cudaDeviceSynchronize() != cudaSuccess) return RB_ERR_CUDA;
            if (cudaMemcpy(c->err_word, &value, sizeof(value), cudaMemcpyHostToDevice) != cudaSuccess)
                return RB_ERR_CUDA;
            return RB_OK;
        }
        default:
            return RB_ERR_INVALID_ARG;
    }
}

rb_status rb_probe_wait_timeout(uint32_t* detail) {
    if (detail) *detail = 0;
    uint32_t* err = device_error_word();
    if (!err) return RB_ERR_CUDA;
    if (rb_device_error(1, nullptr) == RB_ERR_CUDA) return RB_ERR_CUDA;  // start from a clear word
    uint32_t* done = nullptr;
    if (dev_alloc(reinterpret_cast<void**>(&done), sizeof(uint32_t)) != cudaSuccess) return RB_ERR_ALLOC;
    wait_timeout_probe_kernel<<<1, 32>>>(err, done);
    count_launch();
    uint32_t completed = 1;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(&completed, done, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    cudaFree(done);
    if (e != cudaSuccess) return RB_ERR_CUDA;
    const rb_status st = rb_device_error(1, detail);  // reads and clears the word
    return completed ? RB_ERR_DEVICE : st;  // a wait that completed means the probe itself is broken
}

void rb_kernel_timing_enable(int on) { g_timing_on.store(on != 0); }

int rb_kernel_timing_report(char* buf, size_t buf_len) {
    std::vector<TimedLaunch*> items;
    {
        std::lock_guard<std::mutex> lk(g_timing_mu);
        items.swap(g_timed);
    }
    std::map<std::string, std::pair<uint64_t, std::pair<double, double>>> agg;
    int status = 0;
    for (TimedLaunch* L : items) {
        float ms = 0.f;
        if (cudaEventSynchronize(L->e1) != cudaSuccess || cudaEventElapsedTime(&ms, L->e0, L->e1) != cudaSuccess)
            status = -1;
        auto& a = agg[L->name];
        a.first += 1;
        a.second.first += ms;
        a.second.second += L->work;
        {
            std::lock_guard<std::mutex> lk(g_timing_mu);
            g_event_pool[L->dev].push_back(L->e0);
            g_event_pool[L->dev].push_back(L->e1);
        }
        delete L;
    }
    std::string out;
    for (auto& kv : agg) {
        char line[256];
        snprintf(line, sizeof line, "%s %llu %.6f %.6e\n", kv.first.c_str(),
                 static_cast<unsigned long long>(kv.second.first), kv.second.second.first,
                 kv.second.second.second);
        out += line;
    }
    if (buf && buf_len) {
        const size_t n = std::min(buf_len - 1, out.size());
        memcpy(buf, out.data(), n);
        buf[n] = 0;
    }
    return status == 0 ? static_cast<int>(out.size()) : -1;
}

void rb_release_cached_memory(void) {
    cudaError_t e;
    DeviceCtx* c = ctx_for_current(&e);
    if (!c) return;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaStreamSynchronize(c->stream);
    for (int i = 0; i < 3; ++i) {
        if (c->buf[i]) cudaFree(c->buf[i]);
        c->buf[i] = nullptr;
        c->cap[i] = 0;
    }
    scratch_trim();
}

void rb_set_scratch_cache_bytes(size_t bytes) { rb::set_scratch_cache_bytes(bytes); }

}  // extern "C"

// ============================================================================
// Complex GEMM, syrk, symm/hemm, trsm (host slices and device pointers)
// ============================================================================
namespace rb {
namespace {

template <typename T>
rb_status cgemm_host(rb_transpose ta, rb_transpose tb, size_t m, size_t n, size_t k, T ar, T ai,
                     const T* a, size_t lda, size_t a_len, const T* b, size_t ldb, size_t b_len, T br,
                     T bi, T* c, size_t ldc, size_t c_len, rb_precision prec, rb_error* err) {
    set_err(err, RB_OK);
    if (!valid_trans(ta) || !valid_trans(tb) || !valid_prec(prec)) return invalid(err);
    const bool tra = ta != RB_NO_TRANS, trb = tb != RB_NO_TRANS;
    rb_status s;
    if ((s = check_matrix(RB_COL_MAJOR, 'a', tra ? k : m, tra ? m : k, lda, a_len, true, err))) return s;
    if ((s = check_matrix(RB_COL_MAJOR, 'b', trb ? n : k, trb ? k : n, ldb, b_len, true, err))) return s;
    if ((s = check_matrix(RB_COL_MAJOR, 'c', m, n, ldc, c_len, true, err))) return s;
    if (m == 0 || n == 0) return RB_OK;
    const bool beta0 = (br == T(0) && bi == T(0));
    HostMat mats[3] = {{a, nullptr, tra ? k : m, tra ? m : k, lda, 2 * sizeof(T), k > 0, false},
                       {b, nullptr, trb ? n : k, trb ? k : n, ldb, 2 * sizeof(T), k > 0, false},
                       {c, c, m, n, ldc, 2 * sizeof(T), !beta0, true}};
    return host_run(mats, 3, err, [&](void** d, size_t* ld, cudaStream_t st, int32_t* ce) {
        return complex_gemm_dev<T>(ta, tb, m, n, k, ar, ai, static_cast<const T*>(d[0]), ld[0],
                                   static_cast<const T*>(d[1]), ld[1], br, bi, static_cast<T*>(d[2]), ld[2],
                                   prec, st, ce);
    });
}

template <typename T>
rb_status syrk_host(rb_uplo uplo, rb_transpose trans, size_t n, size_t k, T alpha, const T* a, size_t lda,
                    size_t a_len, T beta, T* c, size_t ldc, size_t c_len, rb_error* err) {
    set_err(err, RB_OK);
    if (!valid_uplo(uplo) || !valid_trans(trans)) return invalid(err);
    const bool t = trans != RB_NO_TRANS;
    rb_status s;
    if ((s = check_matrix(RB_COL_MAJOR, 'a', t ? k : n, t ? n : k, lda, a_len, true, err))) return s;
    if ((s = check_matrix(RB_COL_MAJOR, 'c', n, n, ldc, c_len, true, err))) return s;
    if (n == 0) return RB_OK;
    // the other triangle of C is preserved, so C is always staged in. Column
    // panels of C are independent: panel [j0, j0 + len) of the lower triangle
    // is rows j0.. (one triangle-masked product whose origin is on the
    // diagonal); of the upper, rows ..j0 (a plain product) above the masked
    // diagonal block.
    HostMat mats[2] = {{a, nullptr, t ? k : n, t ? n : k, lda, sizeof(T), k > 0, false},
                       {c, c, n, n, ldc, sizeof(T), true, true}};
    return host_run_split(
        mats, 2, true, n, err, [](void*, size_t, cudaStream_t, int32_t*) { return static_cast<int>(RB_OK); },
        [&](void* dA, size_t ldA, void** d, size_t* ld, size_t j0, size_t len, cudaStream_t sp, int32_t* ce) {
            const T* A = static_cast<const T*>(dA);
            auto rows = [&](size_t r) { return t ? A + r * ldA : A + r; };  // op(A) from row r
            T* Cp = static_cast<T*>(d[0]);                                  // C(0, j0)
            if (uplo == RB_LOWER)
                return gemm_colmajor_dev<T>(t, !t, n - j0, len, k, alpha, rows(j0), ldA, rows(j0), ldA, beta, Cp + j0,
                                            ld[0], RB_PREC_PLAIN, sp, 2, ce);
            if (j0 > 0) {
                const int rc = gemm_colmajor_dev<T>(t, !t, j0, len, k, alpha, rows(0), ldA, rows(j0), ldA, beta, Cp,
                                                    ld[0], RB_PREC_PLAIN, sp, 0, ce);
                if (rc != RB_OK) return rc;
            }
            return gemm_colmajor_dev<T>(t, !t, len, len, k, alpha, rows(j0), ldA, rows(j0), ldA, beta, Cp + j0, ld[0],
                                        RB_PREC_PLAIN, sp, 1, ce);
        },
        [](cudaStream_t) {});
}

template <typename T, bool CX>
rb_status symm_host(int herm, rb_side side, rb_uplo uplo, size_t m, size_t n, T ar, T ai, const T* a,
                    size_t lda, size_t a_len, const T* b, size_t ldb, size_t b_len, T br, T bi, T* c,
                    size_t ldc, size_t c_len, rb_precision prec, rb_error* err) {
    set_err(err, RB_OK);
    if (!valid_side(side) || !valid_uplo(uplo) || !valid_prec(prec)) return invalid(err);
    const size_t q = (side == RB_LEFT) ? m : n;
    rb_status s;
    if ((s = check_matrix(RB_COL_MAJOR, 'a', q, q, lda, a_len, true, err))) return s;
    if ((s = check_matrix(RB_COL_MAJOR, 'b', m, n, ldb, b_len, true, err))) return s;
    if ((s = check_matrix(RB_COL_MAJOR, 'c', m, n, ldc, c_len, true, err))) return s;
    if (m == 0 || n == 0) return RB_OK;
    const size_t el = (CX ? 2 : 1) * sizeof(T);
    const bool beta0 = (br == T(0) && (!CX || bi == T(0)));
    const bool left = side == RB_LEFT;
    HostMat mats[3] = {{a, nullptr, q, q, lda, el, true, false},
                       {b, nullptr, m, n, ldb, el, true, false},
                       {c, c, m, n, ldc, el, !beta0, true}};
    // the full operand is mirrored once; panels of B and C (columns for
    // Left, rows for Right) are independent GEMMs against it
    const size_t ldf = CX ? q : (q + 16 / sizeof(T) - 1) / (16 / sizeof(T)) * (16 / sizeof(T));
    T* full = nullptr;
    return host_run_split(
        mats, 3, left, left ? n : m, err,
        [&](void* dA, size_t ldA, cudaStream_t st, int32_t* ce) {
            void* f = nullptr;
            const cudaError_t e = scratch_alloc(&f, ldf * q * el, st);
            if (e != cudaSuccess) {
                if (ce) *ce = static_cast<int32_t>(e);
                return static_cast<int>(e == cudaErrorMemoryAllocation ? RB_ERR_ALLOC : RB_ERR_CUDA);
            }
            full = static_cast<T*>(f);
            return sym_full_dev<T, CX>(herm, uplo, q, static_cast<const T*>(dA), ldA, full, ldf, st, ce);
        },
        [&](void*, size_t, void** d, size_t* ld, size_t, size_t len, cudaStream_t sp, int32_t* ce) {
            const T* B = static_cast<const T*>(d[0]);
            T* C = static_cast<T*>(d[1]);
            const size_t pm = left ? m : len, pn = left ? len : n;
            if constexpr (CX) {
                return left ? complex_gemm_dev<T>(RB_NO_TRANS, RB_NO_TRANS, pm, pn, q, ar, ai, full, ldf, B, ld[0], br,
                                                  bi, C, ld[1], prec, sp, ce)
                            : complex_gemm_dev<T>(RB_NO_TRANS, RB_NO_TRANS, pm, pn, q, ar, ai, B, ld[0], full, ldf, br,
                                                  bi, C, ld[1], prec, sp, ce);
            } else {
                return left ? gemm_colmajor_dev<T>(false, false, pm, pn, q, ar, full, ldf, B, ld[0], br, C, ld[1],
                                                   prec, sp, 0, ce)
                            : gemm_colmajor_dev<T>(false, false, pm, pn, q, ar, B, ld[0], full, ldf, br, C, ld[1],
                                                   prec, sp, 0, ce);
            }
        },
        [&](cudaStream_t st) {
            if (full) cudaFreeAsync(full, st);
        });
}

template <typename T, bool CX>
rb_status trsm_host(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n, T ar,
                    T ai, const T* a, size_t lda, size_t a_len, T* b, size_t ldb, size_t b_len, rb_error* err) {
    set_err(err, RB_OK);
    if (!valid_side(side) || !valid_uplo(uplo) || !valid_trans(trans) || !valid_diag(diag)) return invalid(err);
    const size_t q = (side == RB_LEFT) ? m : n;
    rb_status s;
    if ((s = check_matrix(RB_COL_MAJOR, 'a', q, q, lda, a_len, true, err))) return s;
    if ((s = check_matrix(RB_COL_MAJOR, 'b', m, n, ldb, b_len, true, err))) return s;
    if (m == 0 || n == 0) return RB_OK;
    const size_t el = (CX ? 2 : 1) * sizeof(T);
    const bool left = side == RB_LEFT;
    HostMat mats[2] = {{a, nullptr, q, q, lda, el, true, false}, {b, b, m, n, ldb, el, true, true}};
    // columns of B (Left) or rows (Right) are independent solves
    return host_run_split(
        mats, 2, left, left ? n : m, err, [](void*, size_t, cudaStream_t, int32_t*) { return static_cast<int>(RB_OK); },
        [&](void* dA, size_t ldA, void** d, size_t* ld, size_t, size_t len, cudaStream_t sp, int32_t* ce) {
            return trsm_dev<T, CX>(side, uplo, trans, diag, left ? m : len, left ? len : n, ar, ai,
                                   static_cast<const T*>(dA), ldA, static_cast<T*>(d[0]), ld[0], sp, ce);
        },
        [](cudaStream_t) {});
}

// trmm: no rblas counterpart (its README lists trmm as remaining Level 3);
// the argument checks follow trsm's (src/level3.rs:390-402 shapes).
template <typename T, bool CX>
rb_status trmm_host(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n, T ar, T ai,
                    const T* a, size_t lda, size_t a_len, T* b, size_t ldb, size_t b_len, rb_error* err) {
    set_err(err, RB_OK);
    if (!valid_side(side) || !valid_uplo(uplo) || !valid_trans(trans) || !valid_diag(diag)) return invalid(err);
    const size_t q = (side == RB_LEFT) ? m : n;
    rb_status s;
    if ((s = check_matrix(RB_COL_MAJOR, 'a', q, q, lda, a_len, true, err))) return s;
    if ((s = check_matrix(RB_COL_MAJOR, 'b', m, n, ldb, b_len, true, err))) return s;
    if (m == 0 || n == 0) return RB_OK;
    const size_t el = (CX ? 2 : 1) * sizeof(T);
    const bool left = side == RB_LEFT;
    HostMat mats[2] = {{a, nullptr, q, q, lda, el, true, false}, {b, b, m, n, ldb, el, true, true}};
    // columns of B (Left) or rows (Right) are independent products
    return host_run_split(
        mats, 2, left, left ? n : m, err, [](void*, size_t, cudaStream_t, int32_t*) { return static_cast<int>(RB_OK); },
        [&](void* dA, size_t ldA, void** d, size_t* ld, size_t, size_t len, cudaStream_t sp, int32_t* ce) {
            return trmm_dev<T, CX>(side, uplo, trans, diag, left ? m : len, left ? len : n, ar, ai,
                                   static_cast<const T*>(dA), ldA, static_cast<T*>(d[0]), ld[0], sp, ce);
        },
        [](cudaStream_t) {});
}

rb_status dev_status(int rc, int32_t ce, rb_error* err) {
    if (rc != RB_OK) set_err(err, rc, 0, 0, 0, ce);
    return static_cast<rb_status>(rc);
}


// ---- Level 2 host slices (src/level2.rs, src/complex2.rs) --------------------

// A strided vector of len elements must reach element (len-1)*inc.
rb_status check_vector(char which, size_t len, size_t inc, size_t buf_len, rb_error* err) {
    if (len == 0) return RB_OK;
    const size_t need = (len - 1) * inc + 1;
    if (buf_len < need) {
        set_err(err, RB_ERR_BUFFER_TOO_SMALL, which, buf_len, need);
        return RB_ERR_BUFFER_TOO_SMALL;
    }
    return RB_OK;
}

// A vector staged as a 1 x len block with pitch inc (inc 0: one element).
HostMat vec_mat(const void* src, void* dst, size_t len, size_t inc, size_t elem, bool in, bool out) {
    return HostMat{src, dst, 1, inc == 0 ? (len ? 1 : 0) : len, inc == 0 ? 1 : inc, elem, in, out};
}

template <typename T, bool CX>
rb_status gemv_host(rb_layout layout, rb_transpose trans, size_t m, size_t n, T ar, T ai, const T* a, size_t lda,
                    size_t a_len, const T* x, size_t incx, size_t x_len, T br, T bi, T* y, size_t incy, size_t y_len,
                    rb_error* err) {
    set_err(err, RB_OK);
    if (!valid_layout(layout) || !valid_trans(trans)) return invalid(err);
    const bool tr = trans != RB_NO_TRANS;
    const size_t lenx = tr ? m : n, leny = tr ? n : m;
    rb_status s;
    if ((s = check_matrix(layout, 'a', m, n, lda, a_len, true, err)) != RB_OK) return s;
    if ((s = check_vector('x', lenx, incx, x_len, err)) != RB_OK) return s;
    if ((s = check_vector('y', leny, incy, y_len, err)) != RB_OK) return s;
    if (incy == 0 && leny > 1) {  // every output on one element: no parallel form
        set_err(err, RB_ERR_ZERO_STRIDE, 'y', 0, 0);
        return RB_ERR_ZERO_STRIDE;
    }
    if (leny == 0) return RB_OK;
    const size_t el = sizeof(T) * (CX ? 2 : 1);
    const bool col = layout == RB_COL_MAJOR;
    HostMat mats[3] = {{a, nullptr, col ? m : n, col ? n : m, lda, el, m > 0 && n > 0, false},
                       vec_mat(x, nullptr, lenx, incx, el, lenx > 0, false),
                       vec_mat(y, y, leny, incy, el, true, true)};
    return host_run(mats, 3, err, [&](void** d, size_t* ld, cudaStream_t st, int32_t* ce) {
        return gemv_dev<T, CX>(layout, trans, m, n, ar, ai, static_cast<const T*>(d[0]), ld[0],
                               static_cast<const T*>(d[1]), incx == 0 ? 0 : static_cast<long long>(ld[1]), br, bi,
                               static_cast<T*>(d[2]), static_cast<long long>(ld[2]), st, ce);
    });
}

template <typename T, bool CX>
rb_status ger_host(rb_layout layout, size_t m, size_t n, T ar, T ai, const T* x, size_t incx, size_t x_len,
                   const T* y, size_t incy, size_t y_len, T* a, size_t lda, size_t a_len, int conj, rb_error* err) {
    set_err(err, RB_OK);
    if (!valid_layout(layout)) return invalid(err);
    rb_status s;
    if ((s = check_vector('x', m, incx, x_len, err)) != RB_OK) return s;
    if ((s = check_vector('y', n, incy, y_len, err)) != RB_OK) return s;
    if ((s = check_matrix(layout, 'a', m, n, lda, a_len, true, err)) != RB_OK) return s;
    if (m == 0 || n == 0 || (ar == T(0) && (!CX || ai == T(0)))) return RB_OK;  // nothing is written
    const size_t el = sizeof(T) * (CX ? 2 : 1);
    const bool col = layout == RB_COL_MAJOR;
    HostMat mats[3] = {vec_mat(x, nullptr, m, incx, el, true, false), vec_mat(y, nullptr, n, incy, el, true, false),
                       {a, a, col ? m : n, col ? n : m, lda, el, true, true}};
    return host_run(mats, 3, err, [&](void** d, size_t* ld, cudaStream_t st, int32_t* ce) {
        return ger_dev<T, CX>(layout, m, n, ar, ai, static_cast<const T*>(d[0]),
                              incx == 0 ? 0 : static_cast<long long>(ld[0]), static_cast<const T*>(d[1]),
                              incy == 0 ? 0 : static_cast<long long>(ld[1]), static_cast<T*>(d[2]), ld[2], conj, st,
                              ce);
    });
}

// ---- Level 1 host slices (src/level1.rs, src/complex1.rs) --------------------
// Each vector travels as the contiguous span from its first to its last
// strided element (one copy at full speed; the kernels keep the stride), so
// elements between the strided ones come back unchanged. scal's vector is x;
// reductions write *result (T, or {re, im} for dotu / dotc).
template <typename T, bool CX>
rb_status l1_host(int op, size_t n, T ar, T ai, const T* x, size_t incx, size_t x_len, T* y, size_t incy,
                  size_t y_len, T* result, rb_error* err) {
    set_err(err, RB_OK);
    bool noop = false;
    const rb_status s = l1_check(op, CX, n, ar == T(0) && ai == T(0), ar == T(1) && ai == T(0), incx, x_len, incy,
                                 y_len, true, &noop, err);
    if (s != RB_OK) return s;
    const bool red = op >= L1_DOT;
    const size_t nres = red ? ((op == L1_DOTU || op == L1_DOTC) ? 2 : 1) : 0;
    if (red && !result) return invalid(err);
    if (noop) {
        for (size_t r = 0; r < nres; ++r) result[r] = T(0);
        return RB_OK;
    }
    const bool uses_y = op == L1_AXPY || op == L1_COPY || op == L1_SWAP || op == L1_DOT || op == L1_DOTU ||
                        op == L1_DOTC;
    if (!x || (uses_y && !y)) return invalid(err);
    const size_t el = sizeof(T) * (CX ? 2 : 1);
    const size_t sx = incx == 0 ? 1 : (n - 1) * incx + 1, sy = incy == 0 ? 1 : (n - 1) * incy + 1;
    const bool x_out = op == L1_SCAL || op == L1_SWAP, y_out = op == L1_AXPY || op == L1_COPY || op == L1_SWAP;
    HostMat mats[3];
    int nm = 0;
    mats[nm++] = HostMat{x, x_out ? const_cast<T*>(x) : nullptr, sx, 1, sx, el, true, x_out};
    if (uses_y) mats[nm++] = HostMat{y, y_out ? y : nullptr, sy, 1, sy, el, op != L1_COPY || incy > 1, y_out};
    if (red) mats[nm++] = HostMat{nullptr, result, nres, 1, nres, sizeof(T), false, true};
    return host_run(mats, nm, err, [&](void** d, size_t*, cudaStream_t st, int32_t* ce) {
        T* dx = static_cast<T*>(d[0]);
        T* dy = uses_y ? static_cast<T*>(d[1]) : nullptr;
        T* dr = red ? static_cast<T*>(d[nm - 1]) : nullptr;
        if (op == L1_SCAL) return l1_dev<T, CX>(op, n, ar, ai, nullptr, 0, dx, incx, nullptr, st, ce);
        return l1_dev<T, CX>(op, n, ar, ai, dx, incx, dy, incy, dr, st, ce);
    });
}

}  // namespace
}  // namespace rb

extern "C" {

rb_status rb_cgemm(rb_transpose transa, rb_transpose transb, size_t m, size_t n, size_t k, rb_complex32 alpha,
                   const rb_complex32* a, size_t lda, size_t a_len, const rb_complex32* b, size_t ldb,
                   size_t b_len, rb_complex32 beta, rb_complex32* c, size_t ldc, size_t c_len,
                   rb_precision prec, rb_error* err) {
    return cgemm_host<float>(transa, transb, m, n, k, alpha.re, alpha.im, reinterpret_cast<const float*>(a), lda,
                             a_len, reinterpret_cast<const float*>(b), ldb, b_len, beta.re, beta.im,
                             reinterpret_cast<float*>(c), ldc, c_len, prec, err);
}
rb_status rb_zgemm(rb_transpose transa, rb_transpose transb, size_t m, size_t n, size_t k, rb_complex64 alpha,
                   const rb_complex64* a, size_t lda, size_t a_len, const rb_complex64* b, size_t ldb,
                   size_t b_len, rb_complex64 beta, rb_complex64* c, size_t ldc, size_t c_len,
                   rb_precision prec, rb_error* err) {
    return cgemm_host<double>(transa, transb, m, n, k, alpha.re, alpha.im, reinterpret_cast<const double*>(a),
                              lda, a_len, reinterpret_cast<const double*>(b), ldb, b_len, beta.re, beta.im,
                              reinterpret_cast<double*>(c), ldc, c_len, prec, err);
}
rb_status rb_cgemm_dev(rb_transpose transa, rb_transpose transb, size_t m, size_t n, size_t k,
                       rb_complex32 alpha, const rb_complex32* a, size_t lda, const rb_complex32* b, size_t ldb,
                       rb_complex32 beta, rb_complex32* c, size_t ldc, rb_precision prec, void* stream,
                       rb_error* err) {
    set_err(err, RB_OK);
    if (!valid_trans(transa) || !valid_trans(transb) || !valid_prec(prec)) return invalid(err);
    int32_t ce = 0;
    const int rc = complex_gemm_dev<float>(transa, transb, m, n, k, alpha.re, alpha.im,
                                           reinterpret_cast<const float*>(a), lda, reinterpret_cast<const float*>(b),
                                           ldb, beta.re, beta.im, reinterpret_cast<float*>(c), ldc, prec,
                                           static_cast<cudaStream_t>(stream), &ce);
    return dev_status(rc, ce, err);
}
rb_status rb_zgemm_dev(rb_transpose transa, rb_transpose transb, size_t m, size_t n, size_t k,
                       rb_complex64 alpha, const rb_complex64* a, size_t lda, const rb_complex64* b, size_t ldb,
                       rb_complex64 beta, rb_complex64* c, size_t ldc, rb_precision prec, void* stream,
                       rb_error* err) {
    set_err(err, RB_OK);
    if (!valid_trans(transa) || !valid_trans(transb) || !valid_prec(prec)) return invalid(err);
    int32_t ce = 0;
    const int rc = complex_gemm_dev<double>(transa, transb, m, n, k, alpha.re, alpha.im,
                                            reinterpret_cast<const double*>(a), lda,
                                            reinterpret_cast<const double*>(b), ldb, beta.re, beta.im,
                                            reinterpret_cast<double*>(c), ldc, prec,
                                            static_cast<cudaStream_t>(stream), &ce);
    return dev_status(rc, ce, err);
}

rb_status rb_ssyrk(rb_uplo uplo, rb_transpose trans, size_t n, size_t k, float alpha, const float* a, size_t lda,
                   size_t a_len, float beta, float* c, size_t ldc, size_t c_len, rb_error* err) {
    return syrk_host<float>(uplo, trans, n, k, alpha, a, lda, a_len, beta, c, ldc, c_len, err);
}
rb_status rb_dsyrk(rb_uplo uplo, rb_transpose trans, size_t n, size_t k, double alpha, const double* a,
                   size_t lda, size_t a_len, double beta, double* c, size_t ldc, size_t c_len, rb_error* err) {
    return syrk_host<double>(uplo, trans, n, k, alpha, a, lda, a_len, beta, c, ldc, c_len, err);
}

rb_status rb_ssymm(rb_side side, rb_uplo uplo, size_t m, size_t n, float alpha, const float* a, size_t lda,
                   size_t a_len, const float* b, size_t ldb, size_t b_len, float beta, float* c, size_t ldc,
                   size_t c_len, rb_error* err) {
    return symm_host<float, false>(0, side, uplo, m, n, alpha, 0.f, a, lda, a_len, b, ldb, b_len, beta, 0.f, c,
                                   ldc, c_len, RB_PREC_PLAIN, err);
}
rb_status rb_dsymm(rb_side side, rb_uplo uplo, size_t m, size_t n, double alpha, const double* a, size_t lda,
                   size_t a_len, const double* b, size_t ldb, size_t b_len, double beta, double* c, size_t ldc,
                   size_t c_len, rb_error* err) {
    return symm_host<double, false>(0, side, uplo, m, n, alpha, 0.0, a, lda, a_len, b, ldb, b_len, beta, 0.0, c,
                                    ldc, c_len, RB_PREC_PLAIN, err);
}
rb_status rb_csymm(rb_side side, rb_uplo uplo, size_t m, size_t n, rb_complex32 alpha, const rb_complex32* a,
                   size_t lda, size_t a_len, const rb_complex32* b, size_t ldb, size_t b_len, rb_complex32 beta,
                   rb_complex32* c, size_t ldc, size_t c_len, rb_error* err) {
    return symm_host<float, true>(0, side, uplo, m, n, alpha.re, alpha.im, reinterpret_cast<const float*>(a), lda,
                                  a_len, reinterpret_cast<const float*>(b), ldb, b_len, beta.re, beta.im,
                                  reinterpret_cast<float*>(c), ldc, c_len, RB_PREC_PLAIN, err);
}
rb_status rb_zsymm(rb_side side, rb_uplo uplo, size_t m, size_t n, rb_complex64 alpha, const rb_complex64* a,
                   size_t lda, size_t a_len, const rb_complex64* b, size_t ldb, size_t b_len, rb_complex64 beta,
                   rb_complex64* c, size_t ldc, size_t c_len, rb_error* err) {
    return symm_host<double, true>(0, side, uplo, m, n, alpha.re, alpha.im, reinterpret_cast<const double*>(a),
                                   lda, a_len, reinterpret_cast<const double*>(b), ldb, b_len, beta.re, beta.im,
                                   reinterpret_cast<double*>(c), ldc, c_len, RB_PREC_PLAIN, err);
}
rb_status rb_chemm(rb_side side, rb_uplo uplo, size_t m, size_t n, rb_complex32 alpha, const rb_complex32* a,
                   size_t lda, size_t a_len, const rb_complex32* b, size_t ldb, size_t b_len, rb_complex32 beta,
                   rb_complex32* c, size_t ldc, size_t c_len, rb_error* err) {
    return symm_host<float, true>(1, side, uplo, m, n, alpha.re, alpha.im, reinterpret_cast<const float*>(a), lda,
                                  a_len, reinterpret_cast<const float*>(b), ldb, b_len, beta.re, beta.im,
                                  reinterpret_cast<float*>(c), ldc, c_len, RB_PREC_PLAIN, err);
}
rb_status rb_zhemm(rb_side side, rb_uplo uplo, size_t m, size_t n, rb_complex64 alpha, const rb_complex64* a,
                   size_t lda, size_t a_len, const rb_complex64* b, size_t ldb, size_t b_len, rb_complex64 beta,
                   rb_complex64* c, size_t ldc, size_t c_len, rb_error* err) {
    return symm_host<double, true>(1, side, uplo, m, n, alpha.re, alpha.im, reinterpret_cast<const double*>(a),
                                   lda, a_len, reinterpret_cast<const double*>(b), ldb, b_len, beta.re, beta.im,
                                   reinterpret_cast<double*>(c), ldc, c_len, RB_PREC_PLAIN, err);
}

rb_status rb_strsm(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n, float alpha,
                   const float* a, size_t lda, size_t a_len, float* b, size_t ldb, size_t b_len, rb_error* err) {
    return trsm_host<float, false>(side, uplo, trans, diag, m, n, alpha, 0.f, a, lda, a_len, b, ldb, b_len, err);
}
rb_status rb_dtrsm(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n, double alpha,
                   const double* a, size_t lda, size_t a_len, double* b, size_t ldb, size_t b_len, rb_error* err) {
    return trsm_host<double, false>(side, uplo, trans, diag, m, n, alpha, 0.0, a, lda, a_len, b, ldb, b_len, err);
}
rb_status rb_ctrsm(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n,
                   rb_complex32 alpha, const rb_complex32* a, size_t lda, size_t a_len, rb_complex32* b, size_t ldb,
                   size_t b_len, rb_error* err) {
    return trsm_host<float, true>(side, uplo, trans, diag, m, n, alpha.re, alpha.im, reinterpret_cast<const float*>(a),
                                  lda, a_len, reinterpret_cast<float*>(b), ldb, b_len, err);
}
rb_status rb_ztrsm(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n,
                   rb_complex64 alpha, const rb_complex64* a, size_t lda, size_t a_len, rb_complex64* b, size_t ldb,
                   size_t b_len, rb_error* err) {
    return trsm_host<double, true>(side, uplo, trans, diag, m, n, alpha.re, alpha.im,
                                   reinterpret_cast<const double*>(a), lda, a_len, reinterpret_cast<double*>(b), ldb,
                                   b_len, err);
}

rb_status rb_dtrsm_dev(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n,
                       double alpha, const double* a, size_t lda, double* b, size_t ldb, void* stream, rb_error* err) {
    set_err(err, RB_OK);
    if (!valid_side(side) || !valid_uplo(uplo) || !valid_trans(trans) || !valid_diag(diag)) return invalid(err);
    int32_t ce = 0;
    const int rc = trsm_dev<double, false>(side, uplo, trans, diag, m, n, alpha, 0.0, a, lda, b, ldb,
                                           static_cast<cudaStream_t>(stream), &ce);
    return dev_status(rc, ce, err);
}


// ---- Level 2 (src/level2.rs:11-88, src/complex2.rs:11-145) ------------------
rb_status rb_sgemv(rb_layout layout, rb_transpose trans, size_t m, size_t n, float alpha, const float* a, size_t lda,
                   size_t a_len, const float* x, size_t incx, size_t x_len, float beta, float* y, size_t incy,
                   size_t y_len, rb_error* err) {
    return gemv_host<float, false>(layout, trans, m, n, alpha, 0.f, a, lda, a_len, x, incx, x_len, beta, 0.f, y, incy,
                                   y_len, err);
}
rb_status rb_dgemv(rb_layout layout, rb_transpose trans, size_t m, size_t n, double alpha, const double* a,
                   size_t lda, size_t a_len, const double* x, size_t incx, size_t x_len, double beta, double* y,
                   size_t incy, size_t y_len, rb_error* err) {
    return gemv_host<double, false>(layout, trans, m, n, alpha, 0.0, a, lda, a_len, x, incx, x_len, beta, 0.0, y,
                                    incy, y_len, err);
}
rb_status rb_cgemv(rb_layout layout, rb_transpose trans, size_t m, size_t n, rb_complex32 alpha,
                   const rb_complex32* a, size_t lda, size_t a_len, const rb_complex32* x, size_t incx, size_t x_len,
                   rb_complex32 beta, rb_complex32* y, size_t incy, size_t y_len, rb_error* err) {
    return gemv_host<float, true>(layout, trans, m, n, alpha.re, alpha.im, reinterpret_cast<const float*>(a), lda,
                                  a_len, reinterpret_cast<const float*>(x), incx, x_len, beta.re, beta.im,
                                  reinterpret_cast<float*>(y), incy, y_len, err);
}
rb_status rb_zgemv(rb_layout layout, rb_transpose trans, size_t m, size_t n, rb_complex64 alpha,
                   const rb_complex64* a, size_t lda, size_t a_len, const rb_complex64* x, size_t incx, size_t x_len,
                   rb_complex64 beta, rb_complex64* y, size_t incy, size_t y_len, rb_error* err) {
    return gemv_host<double, true>(layout, trans, m, n, alpha.re, alpha.im, reinterpret_cast<const double*>(a), lda,
                                   a_len, reinterpret_cast<const double*>(x), incx, x_len, beta.re, beta.im,
                                   reinterpret_cast<double*>(y), incy, y_len, err);
}
rb_status rb_sger(rb_layout layout, size_t m, size_t n, float alpha, const float* x, size_t incx, size_t x_len,
                  const float* y, size_t incy, size_t y_len, float* a, size_t lda, size_t a_len, rb_error* err) {
    return ger_host<float, false>(layout, m, n, alpha, 0.f, x, incx, x_len, y, incy, y_len, a, lda, a_len, 0, err);
}
rb_status rb_dger(rb_layout layout, size_t m, size_t n, double alpha, const double* x, size_t incx, size_t x_len,
                  const double* y, size_t incy, size_t y_len, double* a, size_t lda, size_t a_len, rb_error* err) {
    return ger_host<double, false>(layout, m, n, alpha, 0.0, x, incx, x_len, y, incy, y_len, a, lda, a_len, 0, err);
}
#define RB_CGER(NAME, T, CT, CONJ)                                                                                  \
    rb_status NAME(rb_layout layout, size_t m, size_t n, CT alpha, const CT* x, size_t incx, size_t x_len,          \
                   const CT* y, size_t incy, size_t y_len, CT* a, size_t lda, size_t a_len, rb_error* err) {       \
        return ger_host<T, true>(layout, m, n, alpha.re, alpha.im, reinterpret_cast<const T*>(x), incx, x_len,      \
                                 reinterpret_cast<const T*>(y), incy, y_len, reinterpret_cast<T*>(a), lda, a_len,   \
                                 CONJ, err);                                                                        \
    }
RB_CGER(rb_cgeru, float, rb_complex32, 0)
RB_CGER(rb_zgeru, double, rb_complex64, 0)
RB_CGER(rb_cgerc, float, rb_complex32, 1)
RB_CGER(rb_zgerc, double, rb_complex64, 1)
#undef RB_CGER


// ---- trmm (no rblas counterpart) ----------------------------------------------
rb_status rb_strmm(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n, float alpha,
                   const float* a, size_t lda, size_t a_len, float* b, size_t ldb, size_t b_len, rb_error* err) {
    return trmm_host<float, false>(side, uplo, trans, diag, m, n, alpha, 0.f, a, lda, a_len, b, ldb, b_len, err);
}
rb_status rb_dtrmm(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n, double alpha,
                   const double* a, size_t lda, size_t a_len, double* b, size_t ldb, size_t b_len, rb_error* err) {
    return trmm_host<double, false>(side, uplo, trans, diag, m, n, alpha, 0.0, a, lda, a_len, b, ldb, b_len, err);
}
rb_status rb_ctrmm(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n,
                   rb_complex32 alpha, const rb_complex32* a, size_t lda, size_t a_len, rb_complex32* b, size_t ldb,
                   size_t b_len, rb_error* err) {
    return trmm_host<float, true>(side, uplo, trans, diag, m, n, alpha.re, alpha.im, reinterpret_cast<const float*>(a),
                                  lda, a_len, reinterpret_cast<float*>(b), ldb, b_len, err);
}
rb_status rb_ztrmm(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n,
                   rb_complex64 alpha, const rb_complex64* a, size_t lda, size_t a_len, rb_complex64* b, size_t ldb,
                   size_t b_len, rb_error* err) {
    return trmm_host<double, true>(side, uplo, trans, diag, m, n, alpha.re, alpha.im,
                                   reinterpret_cast<const double*>(a), lda, a_len, reinterpret_cast<double*>(b), ldb,
                                   b_len, err);
}
rb_status rb_dtrmm_dev(rb_side side, rb_uplo uplo, rb_transpose trans, rb_diag diag, size_t m, size_t n,
                       double alpha, const double* a, size_t lda, double* b, size_t ldb, void* stream, rb_error* err) {
    set_err(err, RB_OK);
    if (!valid_side(side) || !valid_uplo(uplo) || !valid_trans(trans) || !valid_diag(diag)) return invalid(err);
    int32_t ce = 0;
    const int rc = trmm_dev<double, false>(side, uplo, trans, diag, m, n, alpha, 0.0, a, lda, b, ldb,
                                           static_cast<cudaStream_t>(stream), &ce);
    return dev_status(rc, ce, err);
}

// Level 1 over host slices, real (src/level1.rs)
#define RB_L1_REAL_HOST(P, T)                                                                                      \
    rb_status rb_##P##axpy(size_t n, T alpha, const T* x, size_t incx, size_t x_len, T* y, size_t incy,            \
                           size_t y_len, rb_error* err) {                                                          \
        return l1_host<T, false>(L1_AXPY, n, alpha, T(0), x, incx, x_len, y, incy, y_len, nullptr, err);           \
    }                                                                                                              \
    rb_status rb_##P##scal(size_t n, T alpha, T* x, size_t incx, size_t x_len, rb_error* err) {                    \
        return l1_host<T, false>(L1_SCAL, n, alpha, T(0), x, incx, x_len, nullptr, 0, 0, nullptr, err);            \
    }                                                                                                              \
    rb_status rb_##P##copy(size_t n, const T* x, size_t incx, size_t x_len, T* y, size_t incy, size_t y_len,       \
                           rb_error* err) {                                                                        \
        return l1_host<T, false>(L1_COPY, n, T(0), T(0), x, incx, x_len, y, incy, y_len, nullptr, err);            \
    }                                                                                                              \
    rb_status rb_##P##swap(size_t n, T* x, size_t incx, size_t x_len, T* y, size_t incy, size_t y_len,             \
                           rb_error* err) {                                                                        \
        return l1_host<T, false>(L1_SWAP, n, T(0), T(0), x, incx, x_len, y, incy, y_len, nullptr, err);            \
    }                                                                                                              \
    rb_status rb_##P##dot(size_t n, const T* x, size_t incx, size_t x_len, const T* y, size_t incy, size_t y_len,  \
                          T* result, rb_error* err) {                                                              \
        return l1_host<T, false>(L1_DOT, n, T(0), T(0), x, incx, x_len, const_cast<T*>(y), incy, y_len, result,    \
                                 err);                                                                             \
    }                                                                                                              \
    rb_status rb_##P##asum(size_t n, const T* x, size_t incx, size_t x_len, T* result, rb_error* err) {            \
        return l1_host<T, false>(L1_ASUM, n, T(0), T(0), x, incx, x_len, nullptr, 0, 0, result, err);              \
    }                                                                                                              \
    rb_status rb_##P##nrm2(size_t n, const T* x, size_t incx, size_t x_len, T* result, rb_error* err) {            \
        return l1_host<T, false>(L1_NRM2, n, T(0), T(0), x, incx, x_len, nullptr, 0, 0, result, err);              \
    }
RB_L1_REAL_HOST(s, float)
RB_L1_REAL_HOST(d, double)
#undef RB_L1_REAL_HOST

// Level 1 over host slices, complex (src/complex1.rs)
#define RB_L1_CPLX_HOST(P, N, T, CT)                                                                               \
    rb_status rb_##P##axpy(size_t n, CT alpha, const CT* x, size_t incx, size_t x_len, CT* y, size_t incy,         \
                           size_t y_len, rb_error* err) {                                                          \
        return l1_host<T, true>(L1_AXPY, n, alpha.re, alpha.im, reinterpret_cast<const T*>(x), incx, x_len,        \
                                reinterpret_cast<T*>(y), incy, y_len, nullptr, err);                               \
    }                                                                                                              \
    rb_status rb_##P##scal(size_t n, CT alpha, CT* x, size_t incx, size_t x_len, rb_error* err) {                  \
        return l1_host<T, true>(L1_SCAL, n, alpha.re, alpha.im, reinterpret_cast<T*>(x), incx, x_len, nullptr, 0,  \
                                0, nullptr, err);                                                                  \
    }                                                                                                              \
    rb_status rb_##P##dotu(size_t n, const CT* x, size_t incx, size_t x_len, const CT* y, size_t incy,             \
                           size_t y_len, CT* result, rb_error* err) {                                              \
        return l1_host<T, true>(L1_DOTU, n, T(0), T(0), reinterpret_cast<const T*>(x), incx, x_len,                \
                                reinterpret_cast<T*>(const_cast<CT*>(y)), incy, y_len,                             \
                                reinterpret_cast<T*>(result), err);                                                \
    }                                                                                                              \
    rb_status rb_##P##dotc(size_t n, const CT* x, size_t incx, size_t x_len, const CT* y, size_t incy,             \
                           size_t y_len, CT* result, rb_error* err) {                                              \
        return l1_host<T, true>(L1_DOTC, n, T(0), T(0), reinterpret_cast<const T*>(x), incx, x_len,                \
                                reinterpret_cast<T*>(const_cast<CT*>(y)), incy, y_len,                             \
                                reinterpret_cast<T*>(result), err);                                                \
    }                                                                                                              \
    rb_status rb_##N##nrm2(size_t n, const CT* x, size_t incx, size_t x_len, T* result, rb_error* err) {           \
        return l1_host<T, true>(L1_NRM2, n, T(0), T(0), reinterpret_cast<const T*>(x), incx, x_len, nullptr, 0, 0, \
                                result, err);                                                                      \
    }
RB_L1_CPLX_HOST(c, sc, float, rb_complex32)
RB_L1_CPLX_HOST(z, dz, double, rb_complex64)
#undef RB_L1_CPLX_HOST

}  // extern "C"
