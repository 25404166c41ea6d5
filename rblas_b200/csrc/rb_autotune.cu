// rb_autotune.cu -- autotuner of the GEMM kernels' per-shape parameters,
// with a cache file.
//
// Two parameters are tuned per shape bucket (floor(log2) of the
// column-major m, n and of k, for 32 <= m, n, k <= 4096):
//   - the split-K factor of the grouped plain kernel, per dtype. Its tile is
//     fixed per dtype (128 x 128 f32, 128 x 64 f64: the register budget of
//     the 8-warp SIMT tile) and it runs without clusters. Every candidate
//     factor is timed on the bucket's representative shape (each dimension
//     1.41x its bucket floor) launched alone through the grouped path; a
//     larger factor must win by 3% to be kept. Buckets with a full wave of C
//     tiles, or too short a K for two ranges of four K-tiles, are left to
//     the built-in rule.
//   - the tile width of the Ozaki tensor-core kernels, 128 x 256 or
//     128 x 128 (f64 buckets with n below 2048): the narrow tile pads less
//     and deals more tiles to the SMs, the wide one lands fewer operand bytes
//     per MAC. The narrow one must win by 3%. The width changes no result
//     bit.
// The table is written as text:
//
//   rblas_b200 grouped autotune v2
//   device <name with spaces replaced by _> <sm count>
//   <kind> <log2 m> <log2 n> <log2 k> <value>
//   ...
//
// kind 0 / 1: split factor of an f32 / f64 bucket; kind 2: Ozaki tile width
// of an f64 bucket. Files written by the first version ("... split-k v1",
// split lines only) still load. The tables are installed process-wide;
// loading checks the device line.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/rblas_b200.h"
#include "rb_internal.h"

namespace rb {

namespace {

std::string device_tag() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, dev);
    sms = prop.multiProcessorCount;
    std::string name = prop.name;
    for (char& c : name)
        if (c == ' ') c = '_';
    return name + " " + std::to_string(sms);
}

constexpr int kLoBucket = 5, kHiBucket = 12;  // 32 .. 4096

}  // namespace

}  // namespace rb

using namespace rb;

extern "C" {

rb_status rb_autotune_grouped(const char* cache_path, int* buckets_tuned) {
    if (buckets_tuned) *buckets_tuned = 0;
    const size_t maxdim = size_t(1) << (kHiBucket + 1);  // representative shapes stay below 2^13
    const size_t maxel = maxdim * maxdim;
    void *A = nullptr, *B = nullptr, *Cm = nullptr;
    cudaError_t e = dev_alloc(&A, maxel * 8);
    if (e == cudaSuccess) e = dev_alloc(&B, maxel * 8);
    if (e == cudaSuccess) e = dev_alloc(&Cm, maxel * 8);
    if (e == cudaSuccess) e = cudaMemset(A, 0, maxel * 8);
    if (e == cudaSuccess) e = cudaMemset(B, 0, maxel * 8);
    if (e == cudaSuccess) e = cudaMemset(Cm, 0, maxel * 8);
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&ev1);
    auto cleanup = [&] {
        force_grouped_splits(0);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (st) cudaStreamDestroy(st);
        if (A) cudaFree(A);
        if (B) cudaFree(B);
        if (Cm) cudaFree(Cm);
    };
    if (e != cudaSuccess) {
        cleanup();
        return RB_ERR_ALLOC;
    }
    auto table = std::make_shared<std::map<uint32_t, int>>();
    int tuned = 0;
    rb_status status = RB_OK;
    for (int dt = 0; dt < 2 && status == RB_OK; ++dt) {
        const int BN = dt ? 64 : 128, BK = dt ? 16 : 32;
        for (int lm = kLoBucket; lm <= kHiBucket && status == RB_OK; ++lm)
            for (int ln = kLoBucket; ln <= kHiBucket && status == RB_OK; ++ln)
                for (int lk = kLoBucket; lk <= kHiBucket && status == RB_OK; ++lk) {
                    const size_t m = static_cast<size_t>(std::ldexp(1.41, lm));
                    const size_t n = static_cast<size_t>(std::ldexp(1.41, ln));
                    const size_t k = static_cast<size_t>(std::ldexp(1.41, lk));
                    const long tiles = static_cast<long>((m + 127) / 128) * static_cast<long>((n + BN - 1) / BN);
                    const int num_kt = static_cast<int>((k + BK - 1) / BK);
                    if (tiles >= 148 || num_kt < 8) continue;
                    rb_gemm_problem q{};
                    q.dtype = dt;
                    q.layout = RB_COL_MAJOR;
                    q.transa = RB_NO_TRANS;
                    q.transb = RB_NO_TRANS;
                    q.m = m;
                    q.n = n;
                    q.k = k;
                    q.alpha = 1.0;
                    q.beta = 0.0;
                    q.a = A;
                    q.lda = m;
                    q.b = B;
                    q.ldb = k;
                    q.c = Cm;
                    q.ldc = m;
                    int best_s = 1;
                    float best_ms = 0;
                    for (int s : {1, 2, 3, 4, 6, 8, 12, 16}) {
                        if (s > kGroupedMaxSplit || num_kt / s < 4) break;
                        force_grouped_splits(s);
                        int32_t ce = 0;
                        int rc = grouped_gemm_dev(&q, 1, nullptr, nullptr, st, &ce, nullptr);  // warm-up
                        float ms = 0;
                        if (rc == RB_OK) {
                            cudaEventRecord(ev0, st);
                            for (int r = 0; r < 3 && rc == RB_OK; ++r)
                                rc = grouped_gemm_dev(&q, 1, nullptr, nullptr, st, &ce, nullptr);
                            cudaEventRecord(ev1, st);
                            if (cudaEventSynchronize(ev1) != cudaSuccess) rc = RB_ERR_CUDA;
                            cudaEventElapsedTime(&ms, ev0, ev1);
                        }
                        if (rc != RB_OK) {
                            status = static_cast<rb_status>(rc);
                            break;
                        }
                        if (s == 1 || ms < best_ms * 0.97f) {
                            best_ms = ms;
                            best_s = s;
                        }
                    }
                    force_grouped_splits(0);
                    (*table)[tune_key(dt, m, n, k)] = best_s;
                    ++tuned;
                }
    }
    // Ozaki tile width per f64 bucket (n below 2048)
    auto oz_table = std::make_shared<std::map<uint32_t, int>>();
    for (int lm = kLoBucket; lm <= kHiBucket && status == RB_OK; ++lm)
        for (int ln = kLoBucket; ln <= 10 && status == RB_OK; ++ln)
            for (int lk = kLoBucket; lk <= kHiBucket && status == RB_OK; ++lk) {
                const int m = static_cast<int>(std::ldexp(1.41, lm));
                const int n = static_cast<int>(std::ldexp(1.41, ln));
                const int k = static_cast<int>(std::ldexp(1.41, lk));
                float ms[2] = {0, 0};
                for (int w = 0; w < 2 && status == RB_OK; ++w) {
                    force_ozaki_width(w == 0 ? 256 : 128);
                    CUresult cu = CUDA_SUCCESS;
                    cudaError_t ce = launch_ozaki_gemm(false, false, m, n, k, 1.0, static_cast<const double*>(A), m,
                                                       static_cast<const double*>(B), k, 0.0,
                                                       static_cast<double*>(Cm), m, rb_get_ozaki_slices(), st, &cu);
                    if (ce == cudaSuccess) cudaEventRecord(ev0, st);
                    for (int r = 0; r < 3 && ce == cudaSuccess; ++r)
                        ce = launch_ozaki_gemm(false, false, m, n, k, 1.0, static_cast<const double*>(A), m,
                                               static_cast<const double*>(B), k, 0.0, static_cast<double*>(Cm), m,
                                               rb_get_ozaki_slices(), st, &cu);
                    if (ce == cudaSuccess) ce = cudaEventRecord(ev1, st);
                    if (ce == cudaSuccess) ce = cudaEventSynchronize(ev1);
                    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms[w], ev0, ev1);
                    if (ce != cudaSuccess || cu != CUDA_SUCCESS) status = RB_ERR_CUDA;
                }
                force_ozaki_width(0);
                if (status != RB_OK) break;
                (*oz_table)[tune_key(1, m, n, k)] = (ms[1] < 0.97f * ms[0]) ? 128 : 256;
                ++tuned;
            }
    force_ozaki_width(0);
    if (status == RB_OK) {
        if (cache_path && *cache_path) {
            std::ofstream out(cache_path);
            if (!out) {
                status = RB_ERR_INVALID_ARG;
            } else {
                out << "rblas_b200 grouped autotune v2\n";
                out << "device " << device_tag() << "\n";
                for (const auto& kv : *table)
                    out << ((kv.first >> 24) & 1) << ' ' << ((kv.first >> 16) & 255) << ' ' << ((kv.first >> 8) & 255)
                        << ' ' << (kv.first & 255) << ' ' << kv.second << "\n";
                for (const auto& kv : *oz_table)
                    out << 2 << ' ' << ((kv.first >> 16) & 255) << ' ' << ((kv.first >> 8) & 255) << ' '
                        << (kv.first & 255) << ' ' << kv.second << "\n";
            }
        }
        set_tuned_splits(table);
        set_tuned_ozaki_widths(oz_table);
        if (buckets_tuned) *buckets_tuned = tuned;
    }
    cleanup();
    return status;
}

rb_status rb_autotune_load(const char* cache_path) {
    if (!cache_path) return RB_ERR_INVALID_ARG;
    std::ifstream in(cache_path);
    if (!in) return RB_ERR_INVALID_ARG;
    std::string line;
    if (!std::getline(in, line)) return RB_ERR_INVALID_ARG;
    const bool v2 = line == "rblas_b200 grouped autotune v2";
    if (!v2 && line != "rblas_b200 grouped split-k v1") return RB_ERR_INVALID_ARG;
    if (!std::getline(in, line) || line != "device " + device_tag()) return RB_ERR_INVALID_ARG;
    auto table = std::make_shared<std::map<uint32_t, int>>();
    auto oz_table = std::make_shared<std::map<uint32_t, int>>();
    while (std::getline(in, line)) {
        if (line.empty()) continue;
        std::istringstream ls(line);
        int kind, lm, ln, lk, v;
        if (!(ls >> kind >> lm >> ln >> lk >> v) || kind < 0 || kind > (v2 ? 2 : 1) || lm < 0 || lm > 31 || ln < 0 ||
            ln > 31 || lk < 0 || lk > 31)
            return RB_ERR_INVALID_ARG;
        const size_t m = size_t(1) << lm, n = size_t(1) << ln, k = size_t(1) << lk;
        if (kind == 2) {
            if (v != 128 && v != 256) return RB_ERR_INVALID_ARG;
            (*oz_table)[tune_key(1, m, n, k)] = v;
        } else {
            if (v < 1 || v > kGroupedMaxSplit) return RB_ERR_INVALID_ARG;
            (*table)[tune_key(kind, m, n, k)] = v;
        }
    }
    set_tuned_splits(table);
    set_tuned_ozaki_widths(oz_table);
    return RB_OK;
}

rb_status rb_autotune_reset(void) {
    set_tuned_splits(nullptr);
    set_tuned_ozaki_widths(nullptr);
    return RB_OK;
}

}  // extern "C"
