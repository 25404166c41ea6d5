// rb_internal.h -- host-side declarations shared by the library's translation
// units: tensor-map encoding, kernel launchers and the per-device context.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <atomic>
#include <map>
#include <memory>
#include <mutex>

#include "../../include/rblas_b200.h"

// Device error word layout: [31:24] kind, [23:0] site.
#define RB_DEVERR_TIMEOUT 0x01000000u
#define RB_DEVERR_BOUNDS 0x02000000u
#define RB_DEVERR_ARG 0x03000000u

namespace rb {

// ---- tensor maps --------------------------------------------------------------

// 2-D tiled tensor map over a column-major matrix whose contiguous extent is
// `rows` elements and which has `cols` lines `ld` elements apart; the box is
// box_rows x box_cols. swizzle128: 128-byte swizzle (box_rows*elem == 128).
// Returns CUDA_SUCCESS or the driver error.
CUresult make_tmap_2d(CUtensorMap* map, const void* base, CUtensorMapDataType dtype, size_t elem,
                      uint64_t rows, uint64_t cols, uint64_t ld, uint32_t box_rows,
                      uint32_t box_cols, bool swizzle128);

// 3-D tiled tensor map: dims d0 (contiguous), d1, d2; strides s1, s2 in
// elements between consecutive d1 / d2 indices; box b0 x b1 x b2.
CUresult make_tmap_3d(CUtensorMap* map, const void* base, CUtensorMapDataType dtype, size_t elem,
                      uint64_t d0, uint64_t d1, uint64_t d2, uint64_t s1, uint64_t s2,
                      uint32_t b0, uint32_t b1, uint32_t b2, bool swizzle128);

// ---- launch bookkeeping ----------------------------------------------------------

extern std::atomic<uint64_t> g_launches;
inline void count_launch(uint64_t n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// Optional per-kernel timing of the main GEMM kernels (CUDA events recorded
// on the launching stream around each launch; off unless enabled).
struct KernelTimer {
    void* slot = nullptr;  // opaque
};
bool kernel_timing_on();
void kernel_timing_begin(const char* name, double work, cudaStream_t st, KernelTimer* t);
void kernel_timing_end(KernelTimer* t, cudaStream_t st);

// Stream-ordered scratch (split and digit planes, repacks, tables) from the
// library's own per-device memory pool. Freed blocks stay mapped in the pool
// up to a release threshold (default 8 GiB, rb_set_scratch_cache_bytes), so
// a call after a synchronisation does not map fresh memory again; free with
// cudaFreeAsync on the stream.
cudaError_t scratch_alloc_raw(void** p, size_t bytes, cudaStream_t st);
template <typename T>
inline cudaError_t scratch_alloc(T** p, size_t bytes, cudaStream_t st) {
    return scratch_alloc_raw(reinterpret_cast<void**>(p), bytes, st);
}
void scratch_trim();
// Map `bytes` into the scratch pool now (allocated and freed at once), so
// that later allocations within the release threshold find it mapped.
void scratch_reserve(size_t bytes);
void set_scratch_cache_bytes(size_t bytes);

// Per-device error word (device memory, zero when healthy).
uint32_t* device_error_word();

// A second stream for work that may overlap the caller's stream st: after
// fork_stream, f->s starts behind everything queued on st so far; after
// join_stream, st waits for everything queued on f->s. The pair holds one
// of a few per-device auxiliary streams (picked by st) locked in between,
// so concurrent callers never interleave their fork and join records.
// Both also work while st is being captured into a CUDA graph.
struct ForkedStream {
    cudaStream_t s = nullptr;
    int slot = -1;
};
cudaError_t fork_stream(cudaStream_t st, ForkedStream* f);
cudaError_t join_stream(cudaStream_t st, ForkedStream* f);

// ---- device allocations ---------------------------------------------------------
// Every device allocation the library makes outside the pool (staging
// buffers, plan tables, serving pools) goes through dev_alloc; it and
// scratch_alloc_raw count into rb_device_alloc_count and fail with
// cudaErrorMemoryAllocation while an injected failure is pending
// (rb_debug_inject(RB_INJECT_ALLOC, ...)).
cudaError_t dev_alloc(void** p, size_t bytes);
// True (and one pending failure consumed) when an injected allocation
// failure is due; callers that allocate by other means use it directly.
bool take_injected_alloc_failure();
void count_device_alloc();

// The driver's unique id of the calling thread's current context (0 and
// false when there is none or the driver lacks cuCtxGetId).
bool current_context_id(unsigned long long* id);

// ---- launchers (all operands column-major after row-major normalisation) ------

// Plain SIMT GEMM, C = alpha*op(A)op(B) + beta*C. a_kmajor: op(A) is stored
// k-contiguous (Trans); otherwise m-contiguous (NoTrans). b_kmajor: op(B) is
// stored k-contiguous (NoTrans); otherwise n-contiguous (Trans).
// Requirements: A/B 16-byte aligned with lda/ldb*sizeof(T) % 16 == 0.
// tri: 0 whole C; 1 only the upper triangle (row <= col); 2 only the lower.
// Cin (optional): a separate C0 read for beta != 0, the result going to C.
// f32 problems whose 128 x 128 tiles leave SMs idle while 128 x 64 tiles
// fill at least three quarters of them run the narrow tile.
template <typename T>
cudaError_t launch_simt_gemm(bool a_kmajor, bool b_kmajor, int m, int n, int k, T alpha,
                             const T* A, size_t lda, const T* B, size_t ldb, T beta, T* C,
                             size_t ldc, cudaStream_t st, CUresult* cu_err, int tri = 0,
                             const T* Cin = nullptr, size_t ldcin = 0);
bool simt_narrow_f32(size_t m, size_t n);

// C := beta*C over an m x n column-major block (beta == 0 writes zeros
// without reading; beta == 1 is a no-op and launches nothing); tri as above.
template <typename T>
cudaError_t launch_scale_c(int m, int n, T beta, T* C, size_t ldc, cudaStream_t st, int tri = 0);

// The library's column-major GEMM on device pointers, used by every Level-3
// routine built on it: C = alpha*op(A)op(B) + beta*C (op = transpose when
// ta/tb), `prec` an rb_precision value, `tri` as above (plain form only).
// Returns an rb_status value; *cuda_err receives the CUDA/driver code.
template <typename T>
int gemm_colmajor_dev(bool ta, bool tb, size_t m, size_t n, size_t k, T alpha, const T* A,
                      size_t lda, const T* B, size_t ldb, T beta, T* C, size_t ldc, int prec,
                      cudaStream_t st, int tri, int32_t* cuda_err);

// BF16-split SGEMM on tcgen05 (kind::f16): planes == 2 is 3xBF16
// (hi*hi + hi*lo + lo*hi), planes == 3 is the 6-product form over hi/mid/lo.
// Operands may have any alignment (a pre-pass rewrites them into bf16 planes
// in stream-ordered scratch).
cudaError_t launch_bf16_split_gemm(int planes, bool ta, bool tb, int m, int n, int k, float alpha,
                                   const float* A, size_t lda, const float* B, size_t ldb, float beta,
                                   float* C, size_t ldc, cudaStream_t st, CUresult* cu_err);

// Ozaki INT8-slice DGEMM on tcgen05 (kind::i8, exact INT32 in TMEM, FP64
// summation and alpha/beta epilogue).
cudaError_t launch_ozaki_gemm(bool ta, bool tb, int m, int n, int k, double alpha, const double* A,
                              size_t lda, const double* B, size_t ldb, double beta, double* C,
                              size_t ldc, int slices, cudaStream_t st, CUresult* cu_err);

// Many f64 problems in the Ozaki form in one grouped launch (plus one
// exponent and one slice pass over all operands). cin / ldcin (optional)
// name each problem's C0 when it is not probs[i].c. Results equal each
// problem's own Ozaki call bit for bit. Returns an rb_status value.
int ozaki_grouped_dev(const rb_gemm_problem* probs, size_t count, const void* const* cin, const size_t* ldcin,
                      cudaStream_t st, int32_t* ce);
// Many f32 problems in a BF16-split form (planes 2: 3xBF16, 3: BF16X6) in
// one grouped launch plus one split pass; results equal each problem's own
// call in that form bit for bit. Returns an rb_status value.
int bf16_grouped_dev(int planes, const rb_gemm_problem* probs, size_t count, const void* const* cin,
                     const size_t* ldcin, cudaStream_t st, int32_t* ce);

// ---- Level-3 routines on device pointers (all column-major; complex
// operands interleaved {re, im}; return rb_status values) -------------------
template <typename T>
int complex_gemm_dev(int transa, int transb, size_t m, size_t n, size_t k, T ar, T ai, const T* A,
                     size_t lda, const T* B, size_t ldb, T br, T bi, T* C, size_t ldc, int prec,
                     cudaStream_t st, int32_t* ce);
// The full q x q operand of symm / hemm (ld = ldf) from the uplo triangle of A
// (complex: interleaved; herm: conjugate mirror and real diagonal).
template <typename T, bool CX>
int sym_full_dev(int herm, int uplo, size_t q, const T* A, size_t lda, T* full, size_t ldf, cudaStream_t st,
                 int32_t* ce);
template <typename T>
int symm_dev(int side, int uplo, size_t m, size_t n, T alpha, const T* A, size_t lda, const T* B,
             size_t ldb, T beta, T* C, size_t ldc, int prec, cudaStream_t st, int32_t* ce);
template <typename T>
int hesy_dev(int herm, int side, int uplo, size_t m, size_t n, T ar, T ai, const T* A, size_t lda,
             const T* B, size_t ldb, T br, T bi, T* C, size_t ldc, int prec, cudaStream_t st,
             int32_t* ce);
template <typename T, bool CX>
int trsm_dev(int side, int uplo, int trans, int diag, size_t m, size_t n, T ar, T ai, const T* A,
             size_t lda, T* B, size_t ldb, cudaStream_t st, int32_t* ce);

// Staging for the grouped kernel: a pinned host buffer and a device buffer
// of `bytes` each for the problem table and its counters, and a split-K
// workspace of ws_bytes, owned by the caller and reused once the previous
// launch that used them has finished (the serving loop keeps one set per
// stream). Without it every launch allocates stream-ordered.
struct GroupStaging {
    void* host;
    void* dev;
    size_t bytes;
    void* ws;
    size_t ws_bytes;
};
// Table bytes for `count` problems of which split ones hold `sems` C tiles.
size_t grouped_table_bytes(size_t count, size_t sems);
// Split-K workspace slots (grouped_slot_bytes() each) one problem needs.
size_t grouped_ws_slots(const rb_gemm_problem& q);
size_t grouped_slot_bytes();
int grouped_splits(const rb_gemm_problem& q);
// Split-K autotuning: bucket key of a (column-major) shape, the installed
// table of tuned factors (nullptr: the built-in rule), and a per-thread
// forced factor for timing candidates (0: off).
uint32_t tune_key(int dtype, size_t m, size_t n, size_t k);
void set_tuned_splits(std::shared_ptr<const std::map<uint32_t, int>> table);
void force_grouped_splits(int s);
constexpr int kGroupedMaxSplit = 16;
// Tile width (256 or 128 columns) of the Ozaki kernels for a column-major
// m x n x k problem: the installed autotuner table's choice for its bucket,
// else 128 when n <= 128 and 256 otherwise. The width changes no result
// bit, only the speed. force_ozaki_width(w) fixes it on this thread (0: off).
int ozaki_tile_n(size_t m, size_t n, size_t k);
void set_tuned_ozaki_widths(std::shared_ptr<const std::map<uint32_t, int>> table);
void force_ozaki_width(int w);

// rblas's argument checks for one table entry (dtype, layout, transposes,
// leading dimensions) plus the 32-bit tile-index limit; an rb_status value.
int validate_problem(const rb_gemm_problem& q);

// Grouped plain GEMM over a problem table (see rb_gemm_grouped_dev). cin /
// ldcin (optional, per problem) name a separate input C0 read for beta != 0
// while the result goes to problems[i].c. *bad_index: first invalid problem.
int grouped_gemm_dev(const rb_gemm_problem* probs, size_t count, const void* const* cin, const size_t* ldcin,
                     cudaStream_t st, int32_t* ce, size_t* bad_index, const GroupStaging* staging = nullptr);

// Level 2 on device pointers (rb_?gemv_dev, rb_?ger*_dev): complex arrays
// are interleaved {re, im}; alpha/beta given as (re, im) (im ignored for
// real). conj (rank-1 update) conjugates y. incx/incy in elements.
template <typename T, bool CX>
int gemv_dev(int layout, int trans, size_t m, size_t n, T ar, T ai, const T* A, size_t lda, const T* x,
             long long incx, T br, T bi, T* y, long long incy, cudaStream_t st, int32_t* ce);
template <typename T, bool CX>
int ger_dev(int layout, size_t m, size_t n, T ar, T ai, const T* x, long long incx, const T* y, long long incy, T* A,
            size_t lda, int conj, cudaStream_t st, int32_t* ce);

// Level 1 (rb_?axpy ... rb_?nrm2 and their _dev forms). Reductions come
// after L1_DOT; scal's vector is passed as y.
enum L1Op : int { L1_AXPY = 0, L1_SCAL, L1_COPY, L1_SWAP, L1_DOT, L1_ASUM, L1_NRM2, L1_DOTU, L1_DOTC };
// Device pointers; out (reductions) receives T, or {re, im} for dotu / dotc.
template <typename T, bool CX>
int l1_dev(int op, size_t n, T ar, T ai, const T* x, size_t incx, T* y, size_t incy, T* out, cudaStream_t st,
           int32_t* ce);
// rblas's argument rules for op; *noop when the call writes nothing.
rb_status l1_check(int op, bool cx, size_t n, bool alpha_zero, bool alpha_one, size_t incx, size_t x_len,
                   size_t incy, size_t y_len, bool have_len, bool* noop, rb_error* err);

// Triangular multiply B := alpha*op(A)*B (Left) / alpha*B*op(A) (Right) through one GEMM.
template <typename T, bool CX>
int trmm_dev(int side, int uplo, int trans, int diag, size_t m, size_t n, T ar, T ai, const T* A, size_t lda, T* B,
             size_t ldb, cudaStream_t st, int32_t* ce);

// Batched triangular solve over uniformly strided A_i / B_i (rb_?trsm_batched_dev).
template <typename T>
int trsm_batched_dev(int side, int uplo, int trans, int diag, size_t m, size_t n, T alpha, const T* A, size_t lda,
                     size_t stride_a, T* B, size_t ldb, size_t stride_b, size_t batch, cudaStream_t st,
                     int32_t* ce, rb_error* err);

// Grouped launch frozen into a CUDA graph (rb_gemm_grouped_plan_*).
int grouped_plan_create(const rb_gemm_problem* probs, size_t count, void** plan, int32_t* ce, size_t* bad);
int grouped_plan_launch(void* plan, cudaStream_t st, int32_t* ce);
void grouped_plan_destroy(void* plan);

// One problem of the serving loop's per-request mode: the single-problem
// plain kernel (one launch), result to probs->c, C0 read from cin.
int single_gemm_dev(const rb_gemm_problem* prob, const void* cin, size_t ldcin, cudaStream_t st, int32_t* ce);

// Tensor-pipe throughput (TFLOP/s or TOP/s) of back-to-back M128 N256 UMMAs
// on every SM: i8 != 0 -> kind::i8, else kind::f16 (bf16).
double probe_umma_peak(int i8, int iters);

}  // namespace rb
