// sw_tma.cuh -- TMA tile loads and mbarrier pipelines for sm_100a.
//
// A producer thread issues 2-D tensor copies (cp.async.bulk.tensor, no
// multicast) of row chunks into a ring of shared-memory slots; consumers wait
// on the slot's "full" mbarrier and hand it back through its "empty"
// mbarrier.  Every wait is bounded: after the limit the kernel records
// SW_ERR_TIMEOUT in the device status and returns instead of spinning on.
#pragma once
#include <cuda.h>
#include <stdint.h>

#include "sw_common.cuh"

namespace swb {

// polls of a bounded mbarrier wait (each poll suspends in hardware, then
// sleeps briefly): well above any real wait, well below a hang.  Kernels take
// the limit as an argument (this is the default), so a test can shorten it.
constexpr uint32_t MBAR_SPIN_LIMIT = 1u << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase with the given parity to complete, at most
// `limit` polls.  Returns false (and records a timeout) if it does not.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, DevStatus* st, uint32_t limit) {
    for (uint32_t it = 0; it < limit; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (it > 16) __nanosleep(64);
    }
    atomicCAS(&st->error, 0, (int)SW_ERR_TIMEOUT);
    atomicExch(&st->stop, 1);
    return false;
}

// 2-D tile load, completing on an mbarrier.  x (the innermost coordinate) must
// be a multiple of 16 bytes / element size; the callers only use x = multiples
// of 4 elements.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

}  // namespace swb
