// rb_server.cu -- the serving loop: GEMM requests accepted as they arrive,
// operands resident in HBM, admission against an HBM budget, continuous
// batching into the grouped kernel, per-request timestamps.
//
// A request names its device-resident inputs A, B (and C0 when beta != 0)
// and asks for D = alpha*op(A)op(B) + beta*C0. D is allocated from the
// server's own HBM pool (the budget) when the request is admitted and stays
// resident until the client releases it. One worker thread:
//   1. retires finished batches (event polled), marking their requests done;
//   2. admits queued requests in arrival order while the in-flight batch
//      count, the per-batch slot count and the pool allow (memory freed by
//      released results makes room for the next ones);
//   3. launches the admitted set as one grouped kernel on the next of two
//      streams, so a batch starts while the previous one drains.
// In per-request mode (grouped = 0) every admitted request is launched at
// once as its own single-problem kernel, alternating between the two
// streams -- the baseline the grouped mode is measured against.
#include <cuda_runtime.h>
#include <time.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/rblas_b200.h"
#include "rb_internal.h"

namespace rb {

namespace {

uint64_t now_ns() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return static_cast<uint64_t>(ts.tv_sec) * 1000000000ull + static_cast<uint64_t>(ts.tv_nsec);
}

size_t rup(size_t x, size_t m) { return (x + m - 1) / m * m; }

// First-fit allocator over one device allocation (offsets, 256-byte granules).
class Pool {
public:
    bool init(size_t bytes, cudaError_t* e) {
        *e = dev_alloc(&base_, bytes);
        if (*e != cudaSuccess) return false;
        size_ = bytes;
        free_[0] = bytes;
        return true;
    }
    void release_all() {
        if (base_) cudaFree(base_);
        base_ = nullptr;
    }
    void* alloc(size_t bytes) {
        bytes = rup(std::max<size_t>(bytes, 1), 256);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= bytes) {
                const size_t off = it->first, len = it->second;
                free_.erase(it);
                if (len > bytes) free_[off + bytes] = len - bytes;
                used_ += bytes;
                sizes_[off] = bytes;
                return static_cast<uint8_t*>(base_) + off;
            }
        }
        return nullptr;
    }
    void free(void* p) {
        const size_t off = static_cast<uint8_t*>(p) - static_cast<uint8_t*>(base_);
        auto s = sizes_.find(off);
        if (s == sizes_.end()) return;
        size_t len = s->second;
        sizes_.erase(s);
        used_ -= len;
        size_t start = off;
        auto next = free_.lower_bound(off);
        if (next != free_.end() && next->first == off + len) {
            len += next->second;
            free_.erase(next);
        }
        auto prev = free_.lower_bound(off);
        if (prev != free_.begin()) {
            --prev;
            if (prev->first + prev->second == off) {
                start = prev->first;
                len += prev->second;
                free_.erase(prev);
            }
        }
        free_[start] = len;
    }
    size_t capacity() const { return size_; }

private:
    void* base_ = nullptr;
    size_t size_ = 0, used_ = 0;
    std::map<size_t, size_t> free_;
    std::unordered_map<size_t, size_t> sizes_;
};

struct Request {
    uint64_t id;
    rb_gemm_problem prob;  // prob.c = C0 (input); the output D is server-owned
    size_t d_bytes, ldd;
    size_t ws_slots;       // split-K workspace slots of the grouped kernel
    void* d = nullptr;
    int status = -1;  // -1 queued, -2 in flight, else rb_status
    rb_request_times t{};
};

struct Batch {
    std::vector<Request*> reqs;
    cudaEvent_t done;
    int stream;
    int word;            // slot in the pinned status words: the device error word after the batch
    int form[2];         // forms and thresholds in force when the batch formed
    double min_flop[2];
};

class Server {
public:
    size_t budget;
    int max_batch;
    int grouped;
    // arithmetic forms for large requests (rb_server_set_forms): requests of
    // at least min_flop[dtype] flop run in form[dtype] (a batch's requests of
    // one form in one grouped launch when there are several); the rest take
    // the plain path (grouped or single)
    int form[2] = {RB_PREC_PLAIN, RB_PREC_PLAIN};
    double min_flop[2] = {0.0, 0.0};
    int device = 0;
    Pool pool;
    cudaStream_t streams[2] = {nullptr, nullptr};
    // the precision-form launches go round-robin over these, so they share
    // the GPU with the batch's plain launch instead of running after it
    static constexpr int kFormStreams = 4;
    cudaStream_t form_streams[kFormStreams] = {};
    cudaEvent_t form_events[kFormStreams] = {};  // re-recorded per use; a wait takes the latest record
    int next_form_stream = 0;
    // per stream: pinned host + device problem table of max_batch entries and
    // a split-K workspace, rewritten only after that stream's previous batch
    // has retired (grouped mode keeps at most one batch per stream in flight)
    static constexpr size_t kWsBytes = size_t(256) << 20;
    GroupStaging staging[2] = {{nullptr, nullptr, 0, nullptr, 0}, {nullptr, nullptr, 0, nullptr, 0}};
    size_t ws_slot_cap = 0;
    std::vector<cudaEvent_t> free_events;
    // Per batch, a pinned copy of the device error word taken on the batch's
    // stream after its kernels (before its completion event), so a kernel
    // that gave up a bounded wait fails the requests of its batch.
    static constexpr int kWordSlots = 4096 + 64;
    uint32_t* words = nullptr;     // pinned host, kWordSlots
    uint32_t* dev_word = nullptr;  // the device's error word
    std::vector<int> free_words;
    // A batch saw the word set. Kernels that find it set give up their waits,
    // so every batch in flight alongside may hold a partial result: they all
    // fail (the word stays set until they have retired), no new batch starts,
    // and the word is cleared once nothing is in flight.
    bool poisoned = false;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> queue;
    std::unordered_map<uint64_t, Request*> reqs;
    std::deque<Batch> inflight[2];  // per stream, in launch order
    std::vector<uint64_t> completed;  // ids finished since the trace player last looked
    bool track_completed = false;
    std::atomic<uint64_t> next_id{1};
    std::thread worker;
    bool stop = false;
    int next_stream = 0;

    rb_status start(cudaError_t* e) {
        *e = cudaGetDevice(&device);
        if (*e != cudaSuccess) return RB_ERR_CUDA;
        if (!pool.init(budget, e)) return RB_ERR_ALLOC;
        dev_word = device_error_word();
        if (!dev_word) {
            *e = cudaErrorInitializationError;
            return RB_ERR_CUDA;
        }
        *e = cudaMallocHost(&words, kWordSlots * sizeof(uint32_t));
        if (*e != cudaSuccess) return RB_ERR_ALLOC;
        for (int i = kWordSlots - 1; i >= 0; --i) {
            words[i] = 0;
            free_words.push_back(i);
        }
        for (auto& s : streams) {
            *e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
            if (*e != cudaSuccess) return RB_ERR_CUDA;
        }
        for (int i = 0; i < kFormStreams; ++i) {
            *e = cudaStreamCreateWithFlags(&form_streams[i], cudaStreamNonBlocking);
            if (*e == cudaSuccess) *e = cudaEventCreateWithFlags(&form_events[i], cudaEventDisableTiming);
            if (*e != cudaSuccess) return RB_ERR_CUDA;
        }
        if (grouped) {
            ws_slot_cap = kWsBytes / grouped_slot_bytes();
            const size_t tb = grouped_table_bytes(static_cast<size_t>(max_batch), ws_slot_cap);
            for (auto& g : staging) {
                *e = cudaMallocHost(&g.host, tb);
                if (*e != cudaSuccess) return RB_ERR_ALLOC;
                *e = dev_alloc(&g.dev, tb + kWsBytes);
                if (*e != cudaSuccess) return RB_ERR_ALLOC;
                g.bytes = tb;
                g.ws = static_cast<uint8_t*>(g.dev) + tb;
                g.ws_bytes = kWsBytes;
            }
        }
        worker = std::thread([this] { loop(); });
        return RB_OK;
    }

    void shutdown() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv_work.notify_all();
        if (worker.joinable()) worker.join();
        for (auto& s : streams)
            if (s) cudaStreamSynchronize(s);
        for (auto& s : form_streams)
            if (s) cudaStreamSynchronize(s);
        for (auto& q : inflight)
            for (auto& b : q) cudaEventDestroy(b.done);
        for (auto ev : free_events) cudaEventDestroy(ev);
        for (auto& s : streams)
            if (s) cudaStreamDestroy(s);
        for (int i = 0; i < kFormStreams; ++i) {
            if (form_streams[i]) cudaStreamDestroy(form_streams[i]);
            if (form_events[i]) cudaEventDestroy(form_events[i]);
        }
        for (auto& g : staging) {
            if (g.host) cudaFreeHost(g.host);
            if (g.dev) cudaFree(g.dev);
            g = GroupStaging{nullptr, nullptr, 0, nullptr, 0};
        }
        for (auto& kv : reqs) delete kv.second;
        if (words) cudaFreeHost(words);
        words = nullptr;
        pool.release_all();
    }

    cudaEvent_t get_event() {
        if (!free_events.empty()) {
            cudaEvent_t e = free_events.back();
            free_events.pop_back();
            return e;
        }
        cudaEvent_t e;
        cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        return e;
    }

    size_t inflight_count() const { return inflight[0].size() + inflight[1].size(); }

    int take_word() {
        const int w = free_words.back();
        free_words.pop_back();
        return w;
    }

    // retire finished batches, in order per stream (caller holds mu)
    bool retire() {
        bool any = false;
        for (auto& q : inflight) {
            while (!q.empty() && cudaEventQuery(q.front().done) == cudaSuccess) {
                Batch& b = q.front();
                const uint64_t t = now_ns();
                // the device error word as the batch's stream saw it after its kernels
                const uint32_t w = words[b.word];
                int st = RB_OK;
                if (w != 0) {
                    st = ((w >> 24) == (RB_DEVERR_TIMEOUT >> 24)) ? RB_ERR_TIMEOUT : RB_ERR_DEVICE;
                    words[b.word] = 0;
                    poisoned = true;
                }
                for (Request* r : b.reqs) {
                    if (r->status < 0) r->status = st;
                    r->t.finish_ns = t;
                    if (track_completed) completed.push_back(r->id);
                }
                free_words.push_back(b.word);
                free_events.push_back(b.done);
                q.pop_front();
                any = true;
            }
        }
        return any;
    }

    // Enqueue a batch (worker thread, without the lock); returns the status.
    int launch(const Batch& b) {
        cudaStream_t st = streams[b.stream];
        int32_t ce = 0;
        std::vector<rb_gemm_problem> probs;
        std::vector<const void*> cin;
        std::vector<size_t> ldcin;
        probs.reserve(b.reqs.size());
        for (Request* r : b.reqs) {
            rb_gemm_problem q = r->prob;
            cin.push_back(q.c);  // C0 is read, D written
            ldcin.push_back(q.ldc);
            q.c = r->d;
            q.ldc = r->ldd;
            probs.push_back(q);
        }
        int rc = RB_OK;
        // large requests take a precision form; the rest stay plain
        std::vector<size_t> alone;
        std::vector<rb_gemm_problem> plain;
        std::vector<const void*> plain_cin;
        std::vector<size_t> plain_ldcin;
        for (size_t i = 0; i < probs.size(); ++i) {
            const rb_gemm_problem& q = probs[i];
            const int f = b.form[q.dtype & 1];
            const double flop = 2.0 * q.m * q.n * static_cast<double>(q.k);
            if (f != RB_PREC_PLAIN && flop >= b.min_flop[q.dtype & 1] && flop > 0 && q.alpha != 0.0) {
                alone.push_back(i);
            } else {
                plain.push_back(q);
                plain_cin.push_back(cin[i]);
                plain_ldcin.push_back(ldcin[i]);
            }
        }
        if (grouped) {
            if (!plain.empty())
                rc = grouped_gemm_dev(plain.data(), plain.size(), plain_cin.data(), plain_ldcin.data(), st, &ce,
                                      nullptr, &staging[b.stream]);
        } else {
            for (size_t i = 0; i < plain.size() && rc == RB_OK; ++i)
                rc = single_gemm_dev(&plain[i], plain_cin[i], plain_ldcin[i], st, &ce);
        }
        // the batch's f64 requests in the Ozaki form: one grouped launch when
        // there are several (a lone one takes the single-problem kernel,
        // whose unit-split tail keeps every SM busy on a few tiles)
        std::vector<rb_gemm_problem> oz;
        std::vector<const void*> oz_cin;
        std::vector<size_t> oz_ldcin;
        size_t n_oz = 0, n_bf = 0;
        for (size_t i : alone) {
            n_oz += (probs[i].dtype == 1);
            n_bf += (probs[i].dtype == 0);
        }
        const bool group_oz = n_oz >= 2, group_bf = n_bf >= 2;
        for (size_t i : alone)
            if (group_oz && probs[i].dtype == 1) {
                oz.push_back(probs[i]);
                oz_cin.push_back(cin[i]);
                oz_ldcin.push_back(ldcin[i]);
            }
        if (!oz.empty() && rc == RB_OK) {
            const int f = next_form_stream;
            next_form_stream = (next_form_stream + 1) % kFormStreams;
            rc = ozaki_grouped_dev(oz.data(), oz.size(), oz_cin.data(), oz_ldcin.data(), form_streams[f], &ce);
            if (rc == RB_OK) {
                cudaEventRecord(form_events[f], form_streams[f]);
                cudaStreamWaitEvent(st, form_events[f], 0);
            }
        }
        // the f32 ones in the batch's BF16-split form: one grouped launch too
        std::vector<rb_gemm_problem> bf;
        std::vector<const void*> bf_cin;
        std::vector<size_t> bf_ldcin;
        for (size_t i : alone)
            if (group_bf && probs[i].dtype == 0) {
                bf.push_back(probs[i]);
                bf_cin.push_back(cin[i]);
                bf_ldcin.push_back(ldcin[i]);
            }
        if (!bf.empty() && rc == RB_OK) {
            const int f = next_form_stream;
            next_form_stream = (next_form_stream + 1) % kFormStreams;
            rc = bf16_grouped_dev(b.form[0] == RB_PREC_BF16X3 ? 2 : 3, bf.data(), bf.size(), bf_cin.data(),
                                  bf_ldcin.data(), form_streams[f], &ce);
            if (rc == RB_OK) {
                cudaEventRecord(form_events[f], form_streams[f]);
                cudaStreamWaitEvent(st, form_events[f], 0);
            }
        }
        for (size_t i = 0; i < alone.size() && rc == RB_OK; ++i) {
            if (group_oz && probs[alone[i]].dtype == 1) continue;  // in the grouped launch
            if (group_bf && probs[alone[i]].dtype == 0) continue;
            // on a form stream; the batch's stream then waits for it, so the
            // batch's completion event covers the request
            const int f = next_form_stream;
            next_form_stream = (next_form_stream + 1) % kFormStreams;
            rc = precision_request(probs[alone[i]], cin[alone[i]], ldcin[alone[i]],
                                   b.form[probs[alone[i]].dtype & 1], form_streams[f], &ce);
            if (rc == RB_OK) {
                cudaEventRecord(form_events[f], form_streams[f]);
                cudaStreamWaitEvent(st, form_events[f], 0);
            }
        }
        cudaMemcpyAsync(&words[b.word], dev_word, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        cudaEventRecord(b.done, st);
        return rc;
    }

    // D = alpha*op(A)op(B) + beta*C0 in a precision form: C0 copied into D
    // (beta != 0), then the library's in-place column-major GEMM on D
    static int precision_request(const rb_gemm_problem& q, const void* c0, size_t ldc0, int prec, cudaStream_t st,
                                 int32_t* ce) {
        const bool col = q.layout == RB_COL_MAJOR;
        const size_t el = q.dtype ? 8 : 4;
        const size_t m = col ? q.m : q.n, n = col ? q.n : q.m;  // column-major view
        if (q.beta != 0.0) {
            const cudaError_t e = cudaMemcpy2DAsync(q.c, q.ldc * el, c0, ldc0 * el, m * el, n,
                                                    cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) {
                if (ce) *ce = e;
                return RB_ERR_CUDA;
            }
        }
        const bool ta = (col ? q.transa : q.transb) != RB_NO_TRANS;
        const bool tb = (col ? q.transb : q.transa) != RB_NO_TRANS;
        const void* a = col ? q.a : q.b;
        const void* b = col ? q.b : q.a;
        const size_t lda = col ? q.lda : q.ldb, ldb = col ? q.ldb : q.lda;
        if (q.dtype)
            return gemm_colmajor_dev<double>(ta, tb, m, n, q.k, q.alpha, static_cast<const double*>(a), lda,
                                             static_cast<const double*>(b), ldb, q.beta, static_cast<double*>(q.c),
                                             q.ldc, prec, st, 0, ce);
        return gemm_colmajor_dev<float>(ta, tb, m, n, q.k, static_cast<float>(q.alpha), static_cast<const float*>(a),
                                        lda, static_cast<const float*>(b), ldb, static_cast<float>(q.beta),
                                        static_cast<float*>(q.c), q.ldc, prec, st, 0, ce);
    }

    void loop() {
        cudaSetDevice(device);
        std::unique_lock<std::mutex> lk(mu);
        while (!stop) {
            if (retire()) cv_done.notify_all();
            if (poisoned) {
                if (inflight_count()) {
                    lk.unlock();
                    std::this_thread::sleep_for(std::chrono::microseconds(10));
                    lk.lock();
                    continue;
                }
                // nothing in flight can still read the word: clear it, then go on
                cudaMemsetAsync(dev_word, 0, sizeof(uint32_t), streams[0]);
                cudaStreamSynchronize(streams[0]);
                poisoned = false;
            }
            if (grouped) {
                // continuous batching: one batch running, one queued behind it;
                // everything that arrived meanwhile forms the next batch
                std::vector<Request*> batch;
                // a stream whose previous batch has retired (its staging is free)
                const int s = inflight[next_stream].empty() ? next_stream
                              : (inflight[next_stream ^ 1].empty() ? (next_stream ^ 1) : -1);
                if (!queue.empty() && s >= 0) {
                    size_t slots = 0;
                    while (!queue.empty() && static_cast<int>(batch.size()) < max_batch) {
                        Request* r = queue.front();
                        if (slots + r->ws_slots > ws_slot_cap) break;  // next batch
                        void* d = pool.alloc(r->d_bytes);
                        if (!d) break;  // wait for results to be released
                        r->d = d;
                        r->status = -2;
                        r->t.admit_ns = now_ns();
                        slots += r->ws_slots;
                        queue.pop_front();
                        batch.push_back(r);
                    }
                }
                if (!batch.empty()) {
                    inflight[s].push_back(Batch{std::move(batch), get_event(), s, take_word(), {form[0], form[1]},
                                                {min_flop[0], min_flop[1]}});
                    next_stream = s ^ 1;
                    const Batch& b = inflight[s].back();
                    lk.unlock();
                    const int rc = launch(b);
                    lk.lock();
                    if (rc != RB_OK)
                        for (Request* r : b.reqs) r->status = rc;
                    continue;
                }
            } else {
                // per request: launch every admitted request at once
                std::vector<Batch*> fresh;
                while (!queue.empty() && inflight_count() < kMaxInflightRequests) {
                    Request* r = queue.front();
                    void* d = pool.alloc(r->d_bytes);
                    if (!d) break;
                    r->d = d;
                    r->status = -2;
                    r->t.admit_ns = now_ns();
                    queue.pop_front();
                    const int s = next_stream;
                    next_stream ^= 1;
                    inflight[s].push_back(Batch{std::vector<Request*>{r}, get_event(), s, take_word(),
                                                {form[0], form[1]}, {min_flop[0], min_flop[1]}});
                    fresh.push_back(&inflight[s].back());
                }
                if (!fresh.empty()) {
                    // only this thread changes `inflight`, so the entries stay put while unlocked
                    lk.unlock();
                    std::vector<int> rcs(fresh.size());
                    for (size_t i = 0; i < fresh.size(); ++i) rcs[i] = launch(*fresh[i]);
                    lk.lock();
                    for (size_t i = 0; i < fresh.size(); ++i)
                        if (rcs[i] != RB_OK) fresh[i]->reqs[0]->status = rcs[i];
                    continue;
                }
            }
            if (inflight_count()) {
                lk.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(10));
                lk.lock();
            } else {
                cv_work.wait_for(lk, std::chrono::milliseconds(2));
            }
        }
    }
    static constexpr size_t kMaxInflightRequests = 4096;
    // per-request mode keeps at most kMaxInflightRequests batches in flight, grouped mode two
    static_assert(kWordSlots >= kMaxInflightRequests + 2, "a status word per batch in flight");
};

}  // namespace

}  // namespace rb

using namespace rb;

extern "C" {

rb_status rb_gemm_grouped_dev(const rb_gemm_problem* problems, size_t count, void* stream, rb_error* err) {
    if (err) *err = rb_error{0, 0, 0, 0, 0};
    if (count && !problems) {
        if (err) err->code = RB_ERR_INVALID_ARG;
        return RB_ERR_INVALID_ARG;
    }
    int32_t ce = 0;
    size_t bad = 0;
    const int rc = grouped_gemm_dev(problems, count, nullptr, nullptr, static_cast<cudaStream_t>(stream), &ce, &bad);
    if (rc != RB_OK && err) {
        err->code = rc;
        err->got = bad;
        err->cuda_error = ce;
    }
    return static_cast<rb_status>(rc);
}

int rb_gemm_grouped_splits(const rb_gemm_problem* p) { return p ? grouped_splits(*p) : 0; }

rb_status rb_gemm_grouped_bf16_dev(const rb_gemm_problem* problems, size_t count, rb_precision form, void* stream,
                                   rb_error* err) {
    if (err) *err = rb_error{0, 0, 0, 0, 0};
    if ((form != RB_PREC_BF16X3 && form != RB_PREC_BF16X6) || (count && !problems)) {
        if (err) err->code = RB_ERR_INVALID_ARG;
        return RB_ERR_INVALID_ARG;
    }
    for (size_t i = 0; i < count; ++i) {
        const rb_gemm_problem& q = problems[i];
        const int v = q.dtype != 0 ? RB_ERR_UNSUPPORTED : validate_problem(q);
        const bool null_ptr = q.m && q.n && (!q.c || (q.k && q.alpha != 0.0 && (!q.a || !q.b)));
        if (v != RB_OK || null_ptr) {
            if (err) {
                err->code = v != RB_OK ? v : RB_ERR_INVALID_ARG;
                err->got = i;
            }
            return static_cast<rb_status>(v != RB_OK ? v : RB_ERR_INVALID_ARG);
        }
    }
    int32_t ce = 0;
    const int rc = bf16_grouped_dev(form == RB_PREC_BF16X3 ? 2 : 3, problems, count, nullptr, nullptr,
                                    static_cast<cudaStream_t>(stream), &ce);
    if (rc != RB_OK && err) {
        err->code = rc;
        err->cuda_error = ce;
    }
    return static_cast<rb_status>(rc);
}

rb_status rb_gemm_grouped_ozaki_dev(const rb_gemm_problem* problems, size_t count, void* stream, rb_error* err) {
    if (err) *err = rb_error{0, 0, 0, 0, 0};
    if (count && !problems) {
        if (err) err->code = RB_ERR_INVALID_ARG;
        return RB_ERR_INVALID_ARG;
    }
    for (size_t i = 0; i < count; ++i) {
        const rb_gemm_problem& q = problems[i];
        const int v = q.dtype != 1 ? RB_ERR_UNSUPPORTED : validate_problem(q);
        const bool null_ptr = q.m && q.n && (!q.c || (q.k && q.alpha != 0.0 && (!q.a || !q.b)));
        if (v != RB_OK || null_ptr) {
            if (err) {
                err->code = v != RB_OK ? v : RB_ERR_INVALID_ARG;
                err->got = i;
            }
            return static_cast<rb_status>(v != RB_OK ? v : RB_ERR_INVALID_ARG);
        }
    }
    int32_t ce = 0;
    const int rc = ozaki_grouped_dev(problems, count, nullptr, nullptr, static_cast<cudaStream_t>(stream), &ce);
    if (rc != RB_OK && err) {
        err->code = rc;
        err->cuda_error = ce;
    }
    return static_cast<rb_status>(rc);
}

rb_status rb_gemm_grouped_plan_create(const rb_gemm_problem* problems, size_t count, void** plan, rb_error* err) {
    if (err) *err = rb_error{0, 0, 0, 0, 0};
    if (!plan || (count && !problems)) {
        if (err) err->code = RB_ERR_INVALID_ARG;
        return RB_ERR_INVALID_ARG;
    }
    int32_t ce = 0;
    size_t bad = 0;
    const int rc = grouped_plan_create(problems, count, plan, &ce, &bad);
    if (rc != RB_OK && err) {
        err->code = rc;
        err->got = bad;
        err->cuda_error = ce;
    }
    return static_cast<rb_status>(rc);
}

rb_status rb_gemm_grouped_plan_launch(void* plan, void* stream, rb_error* err) {
    if (err) *err = rb_error{0, 0, 0, 0, 0};
    if (!plan) {
        if (err) err->code = RB_ERR_INVALID_ARG;
        return RB_ERR_INVALID_ARG;
    }
    int32_t ce = 0;
    const int rc = grouped_plan_launch(plan, static_cast<cudaStream_t>(stream), &ce);
    if (rc != RB_OK && err) {
        err->code = rc;
        err->cuda_error = ce;
    }
    return static_cast<rb_status>(rc);
}

rb_status rb_gemm_grouped_plan_destroy(void* plan) {
    if (!plan) return RB_ERR_INVALID_ARG;
    grouped_plan_destroy(plan);
    return RB_OK;
}

rb_status rb_server_create(size_t budget_bytes, int max_batch, int grouped, void** server) {
    if (!server || max_batch < 1 || budget_bytes < 256) return RB_ERR_INVALID_ARG;
    Server* s = new Server();
    s->budget = budget_bytes;
    s->max_batch = max_batch;
    s->grouped = grouped;
    cudaError_t e;
    const rb_status st = s->start(&e);
    if (st != RB_OK) {
        s->shutdown();
        delete s;
        return st;
    }
    *server = s;
    return RB_OK;
}

rb_status rb_server_set_forms(void* server, int f32_form, int f64_form, double f32_min_flop, double f64_min_flop) {
    Server* s = static_cast<Server*>(server);
    if (!s || (f32_form != RB_PREC_PLAIN && f32_form != RB_PREC_BF16X3 && f32_form != RB_PREC_BF16X6) ||
        (f64_form != RB_PREC_PLAIN && f64_form != RB_PREC_OZAKI) || !(f32_min_flop >= 0) || !(f64_min_flop >= 0))
        return RB_ERR_INVALID_ARG;
    // precision requests take their planes from the scratch pool on several
    // streams at once: map its working set now rather than in the middle of
    // a run (growing a pool under load stalled the serving loop)
    if (f32_form != RB_PREC_PLAIN || f64_form != RB_PREC_PLAIN) {
        cudaSetDevice(s->device);
        scratch_reserve(size_t(6) << 30);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->form[0] = f32_form;
    s->form[1] = f64_form;
    s->min_flop[0] = f32_min_flop;
    s->min_flop[1] = f64_min_flop;
    return RB_OK;
}

rb_status rb_server_submit(void* server, const rb_gemm_problem* p, uint64_t* id) {
    Server* s = static_cast<Server*>(server);
    if (!s || !p || !id) return RB_ERR_INVALID_ARG;
    const int v = validate_problem(*p);
    if (v != RB_OK) return static_cast<rb_status>(v);
    Request* r = new Request();
    r->prob = *p;
    const size_t el = p->dtype ? 8 : 4;
    // D mirrors C's layout with a compact leading dimension padded to 16 bytes
    const size_t rows = (p->layout == RB_COL_MAJOR) ? p->m : p->n;
    const size_t cols = (p->layout == RB_COL_MAJOR) ? p->n : p->m;
    r->ldd = std::max<size_t>(rup(rows, 16 / el), 16 / el);
    r->d_bytes = r->ldd * std::max<size_t>(cols, 1) * el;
    r->ws_slots = s->grouped ? grouped_ws_slots(*p) : 0;
    if (r->d_bytes > s->pool.capacity()) {
        delete r;
        return RB_ERR_BUSY;  // can never be admitted under this budget
    }
    r->t.enqueue_ns = now_ns();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = s->next_id++;
        s->reqs[r->id] = r;
        s->queue.push_back(r);
    }
    s->cv_work.notify_one();
    *id = r->id;
    return RB_OK;
}

rb_status rb_server_wait(void* server, uint64_t id, int64_t timeout_us, void** d_out, size_t* ldd,
                         rb_request_times* times) {
    Server* s = static_cast<Server*>(server);
    if (!s) return RB_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return RB_ERR_INVALID_ARG;
    Request* r = it->second;
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::microseconds(timeout_us < 0 ? 0 : timeout_us);
    while (r->status < 0) {
        if (timeout_us >= 0 && std::chrono::steady_clock::now() >= deadline) return RB_ERR_TIMEOUT;
        s->cv_done.wait_for(lk, std::chrono::microseconds(200));
    }
    if (d_out) *d_out = r->d;
    if (ldd) *ldd = r->ldd;
    if (times) *times = r->t;
    return static_cast<rb_status>(r->status);
}

rb_status rb_server_cancel(void* server, uint64_t id) {
    Server* s = static_cast<Server*>(server);
    if (!s) return RB_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(id);
        if (it == s->reqs.end()) return RB_ERR_INVALID_ARG;
        Request* r = it->second;
        if (r->status != -1) return RB_ERR_BUSY;  // admitted: running or finished
        auto q = std::find(s->queue.begin(), s->queue.end(), r);
        if (q != s->queue.end()) s->queue.erase(q);
        r->status = RB_ERR_CANCELLED;
        r->t.finish_ns = now_ns();
        if (s->track_completed) s->completed.push_back(r->id);
    }
    s->cv_done.notify_all();
    return RB_OK;
}

rb_status rb_server_release(void* server, uint64_t id) {
    Server* s = static_cast<Server*>(server);
    if (!s) return RB_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(id);
        if (it == s->reqs.end()) return RB_ERR_INVALID_ARG;
        Request* r = it->second;
        if (r->status < 0) return RB_ERR_BUSY;  // still queued or running
        if (r->d) s->pool.free(r->d);
        s->reqs.erase(it);
        delete r;
    }
    s->cv_work.notify_one();
    return RB_OK;
}

rb_status rb_server_destroy(void* server) {
    Server* s = static_cast<Server*>(server);
    if (!s) return RB_ERR_INVALID_ARG;
    s->shutdown();
    delete s;
    return RB_OK;
}

rb_status rb_server_run_trace(void* server, const rb_gemm_problem* problems, const uint64_t* arrival_ns,
                              size_t count, rb_request_times* times) {
    Server* s = static_cast<Server*>(server);
    if (!s || (count && (!problems || !arrival_ns || !times))) return RB_ERR_INVALID_ARG;
    std::unordered_map<uint64_t, size_t> index;  // request id -> trace position
    rb_status first_err = RB_OK;
    for (size_t i = 0; i < count; ++i) times[i] = rb_request_times{0, 0, 0};
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->completed.clear();
        s->track_completed = true;
    }
    const uint64_t t0 = now_ns();
    size_t next = 0, finished = 0;
    std::vector<uint64_t> got;
    while (finished < count) {
        // submit every request whose arrival time has passed
        const uint64_t now = now_ns();
        while (next < count && t0 + arrival_ns[next] <= now) {
            uint64_t id = 0;
            const rb_status st = rb_server_submit(server, &problems[next], &id);
            if (st != RB_OK) {
                ++finished;
                if (first_err == RB_OK) first_err = st;
            } else {
                index[id] = next;
            }
            ++next;
        }
        // collect finished requests and release their results
        {
            std::lock_guard<std::mutex> lk(s->mu);
            got.swap(s->completed);
        }
        for (uint64_t id : got) {
            auto it = index.find(id);
            if (it == index.end()) continue;
            rb_request_times t;
            const rb_status st = rb_server_wait(server, id, 0, nullptr, nullptr, &t);
            times[it->second] = t;
            if (st != RB_OK && first_err == RB_OK) first_err = st;
            rb_server_release(server, id);
            index.erase(it);
            ++finished;
        }
        got.clear();
        if (next < count) {
            const uint64_t due = t0 + arrival_ns[next];
            const uint64_t n2 = now_ns();
            if (due > n2 + 20000)
                std::this_thread::sleep_for(std::chrono::nanoseconds(std::min<uint64_t>(due - n2 - 10000, 100000)));
        } else {
            std::this_thread::sleep_for(std::chrono::microseconds(10));
        }
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->track_completed = false;
        s->completed.clear();
    }
    return first_err;
}

}  // extern "C"
