// rb_device.cuh -- device-side building blocks shared by every kernel:
// inline-PTX wrappers for mbarriers, TMA (cp.async.bulk.tensor) and tcgen05,
// the device error word, and bounded waits.
//
// Every spin on an mbarrier is bounded: after RB_WAIT_LIMIT_NS of
// %globaltimer the waiting thread records RB_DEVERR_TIMEOUT|site in the
// device error word and returns false; every other waiter polls that word and
// gives up as soon as it is set, so one stuck CTA ends the whole grid quickly.
// Kernels then drain their own in-flight copies (again bounded), release any
// TMEM they hold, and return. The host reads the word after the call.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#ifndef RB_WAIT_LIMIT_NS
#define RB_WAIT_LIMIT_NS 2000000000ull  // 2 s: far above any legitimate stage wait
#endif

#include "rb_internal.h"

namespace rb {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool dev_aborted(const uint32_t* err) {
    return *reinterpret_cast<const volatile uint32_t*>(err) != 0u;
}

__device__ __forceinline__ void dev_raise(uint32_t* err, uint32_t code) {
    atomicCAS(err, 0u, code);
}

// ---- mbarrier ----------------------------------------------------------------

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase with the given parity. Returns false (and makes
// sure the error word is set) if it gave up.
__device__ __noinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t* err,
                                       uint32_t site) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer();
    for (uint32_t it = 1;; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 31u) == 0u) {
            if (dev_aborted(err)) return false;
            if (globaltimer() - t0 > RB_WAIT_LIMIT_NS) {
                dev_raise(err, RB_DEVERR_TIMEOUT | site);
                return false;
            }
        }
    }
}

// Wait used only on the error path to let this CTA's own copies land before
// it exits: ignores the abort flag, bounded by time alone.
__device__ __noinline__ bool mbar_wait_drain(uint64_t* bar, uint32_t parity) {
    const uint64_t t0 = globaltimer();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (globaltimer() - t0 > RB_WAIT_LIMIT_NS) return false;
    }
}

// ---- TMA ---------------------------------------------------------------------

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// 2-D tiled load into this CTA's shared memory, completing on `bar`.
// c0 is the innermost (contiguous) coordinate; c0 * elemsize must be a
// multiple of 16 bytes (callers pass tile-aligned coordinates).
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int32_t c0, int32_t c1) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int32_t c0, int32_t c1, int32_t c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

// ---- grid rasterisation --------------------------------------------------------

// Linear block id -> (tile_m, tile_n), walking tile columns in groups of G
// tile rows so concurrently resident CTAs share A rows and B columns in L2.
__device__ __forceinline__ void raster_tile(int bid, int tiles_m, int tiles_n, int& tm, int& tn) {
    constexpr int G = 8;
    const int per_group = G * tiles_n;
    const int group = bid / per_group;
    const int first_m = group * G;
    const int gsz = min(tiles_m - first_m, G);
    const int in_group = bid - group * per_group;
    tm = first_m + in_group % gsz;
    tn = in_group / gsz;
}

}  // namespace rb
