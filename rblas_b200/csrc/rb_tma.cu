// rb_tma.cu -- tensor-map encoding through the driver entry point (the
// library links only the CUDA runtime; libcuda is reached at run time).
#include <cudaTypedefs.h>

#include <mutex>

#include "rb_internal.h"

namespace rb {

namespace {
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

void load_encode() {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault,
                                         &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
}
}  // namespace

CUresult make_tmap_2d(CUtensorMap* map, const void* base, CUtensorMapDataType dtype, size_t elem,
                      uint64_t rows, uint64_t cols, uint64_t ld, uint32_t box_rows,
                      uint32_t box_cols, bool swizzle128) {
    std::call_once(g_encode_once, load_encode);
    if (!g_encode) return CUDA_ERROR_NOT_FOUND;
    cuuint64_t dims[2] = {rows, cols};
    cuuint64_t strides[1] = {ld * elem};
    cuuint32_t box[2] = {box_rows, box_cols};
    cuuint32_t estr[2] = {1, 1};
    return g_encode(map, dtype, 2, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE,
                    swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}

CUresult make_tmap_3d(CUtensorMap* map, const void* base, CUtensorMapDataType dtype, size_t elem,
                      uint64_t d0, uint64_t d1, uint64_t d2, uint64_t s1, uint64_t s2,
                      uint32_t b0, uint32_t b1, uint32_t b2, bool swizzle128) {
    std::call_once(g_encode_once, load_encode);
    if (!g_encode) return CUDA_ERROR_NOT_FOUND;
    cuuint64_t dims[3] = {d0, d1, d2};
    cuuint64_t strides[2] = {s1 * elem, s2 * elem};
    cuuint32_t box[3] = {b0, b1, b2};
    cuuint32_t estr[3] = {1, 1, 1};
    return g_encode(map, dtype, 3, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE,
                    swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}

namespace {
PFN_cuCtxGetCurrent_v4000 g_ctx_current = nullptr;
PFN_cuCtxGetId_v12000 g_ctx_id = nullptr;
std::once_flag g_ctx_once;

void load_ctx_fns() {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &fn, 4000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_ctx_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(fn);
    fn = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &fn, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_ctx_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(fn);
}
}  // namespace

bool current_context_id(unsigned long long* id) {
    *id = 0;
    std::call_once(g_ctx_once, load_ctx_fns);
    if (!g_ctx_current || !g_ctx_id) return false;
    CUcontext ctx = nullptr;
    if (g_ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
    return g_ctx_id(ctx, id) == CUDA_SUCCESS;
}

}  // namespace rb
