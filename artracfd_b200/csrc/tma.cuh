// TMA (cp.async.bulk.tensor) and mbarrier helpers for sm_100a, written as
// inline PTX.  Only plain tile loads into the issuing CTA's own shared memory
// are used: no cluster multicast anywhere.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace acfd {
namespace tma {

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    // make the initialised barrier visible to the async (TMA) proxy
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// invalidate a barrier that no thread or copy uses any more, so that its
// memory may hold a new barrier (mbarrier.init on a valid barrier is
// undefined)
__device__ __forceinline__ void mbar_inval(uint64_t *bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// plain arrival (count 1) on a barrier
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// one non-blocking probe of phase `parity`; true once the phase completed
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// 5-D tiled load of one box into shared memory, completion counted on `bar`.
// c0 (innermost, x) must be even for FP64 data (16-byte rule); the other
// coordinates may be negative or beyond the extent (zero fill).
__device__ __forceinline__ void load_5d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3, int c4,
                                        uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_addr(bar))
        : "memory");
}

// Bounded wait: every thread polls the barrier at most `limit` times.  On
// time-out the caller's status word gets `code` and false is returned; the
// caller must then not read the buffer.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int *status, int code,
                                                  long long limit)
{
    for (long long it = 0; it < limit; ++it) {
        if (mbar_try_wait(bar, parity)) {
            return true;
        }
    }
    atomicExch(status, code);
    return false;
}

}  // namespace tma
}  // namespace acfd
