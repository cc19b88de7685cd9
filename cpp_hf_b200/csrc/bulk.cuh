// Bulk asynchronous copies (cp.async.bulk, the TMA engine's untiled form) into
// shared memory with mbarrier completion, plus bounded waits.
//
// Only global -> shared::cta copies of this GPU's own memory; no multicast.
// Every wait is bounded: after kMbarSpinLimit polls it ORs a code into the
// library's device error word (the pointer every launch with such waits is
// given; see wait_error_word()) and returns false so the kernel can stop
// instead of hanging.
#pragma once

#include "common.cuh"

#include <cuda.h>

namespace cpphf {

constexpr long long kMbarSpinLimit = 2000000LL;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// arrive (count 1) and add `bytes` to the expected transaction count
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// plain arrive (count 1, no transaction bytes)
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// orders this thread's generic-proxy global accesses with later async-proxy
// (TMA) accesses and vice versa
__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// global -> shared bulk copy; dst, src 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// 3-D tiled TMA load (no multicast) of the box at coordinates {x, y, z}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// Host: encode a 3-D tiled tensor map (dims innermost first, strides in bytes
// for dims 1 and 2).  Returns false if the driver rejects it.
bool make_tensor_map_3d(CUtensorMap* map, const void* base, CUtensorMapDataType dt, unsigned long long d0,
                        unsigned long long d1, unsigned long long d2, unsigned long long stride1_bytes,
                        unsigned long long stride2_bytes, unsigned b0, unsigned b1, unsigned b2);

// Bounded wait for phase `parity`; false (and kWaitErrMbar ORed into *err) on timeout.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, unsigned* err) {
    long long spins = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (++spins > kMbarSpinLimit) {
            if (err) atomicOr(err, kWaitErrMbar);
            return false;
        }
    }
    return true;
}

}  // namespace cpphf
