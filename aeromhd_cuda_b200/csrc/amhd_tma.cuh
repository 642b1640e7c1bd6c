// amhd_tma.cuh -- Tensor Memory Accelerator staging of the state tile + halo.
//
// One thread issues cp.async.bulk.tensor.3d for the box [10 planes][tile_x+4
// rows][36 columns] of a state buffer into shared memory; completion is
// tracked by a CTA-local mbarrier (expect_tx / complete_tx).  The wait is
// bounded: if the transfer has not completed within kTmaWaitNs (read from
// %globaltimer; kTmaWaitIters polls as a backstop) the caller gets `false`
// back, records AMHD_FLAG_TIMEOUT and the CTA leaves.
// Every CTA loads its own box, from this GPU's memory only.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace amhd {
namespace tma {

constexpr uint32_t kTmaWaitIters = 1u << 22;
constexpr uint64_t kTmaWaitNs = 1000000000ull;  // 1 s

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// order this thread's earlier generic shared-memory accesses before later async-proxy writes
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// 3-D tiled load; coordinates innermost first (column, row, plane)
__device__ __forceinline__ void load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// wait for the phase `parity` of the barrier to complete, at most limit_ns
// nanoseconds and max_iters polls (try_wait may suspend the thread between
// polls); false when it gave up
__device__ __forceinline__ bool wait_for(uint64_t *bar, uint32_t parity, uint64_t limit_ns, uint32_t max_iters)
{
    const uint32_t a = smem_addr(bar);
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t it = 0; it < max_iters; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 63u) == 63u && globaltimer_ns() - t0 > limit_ns) return false;
    }
    return false;
}

__device__ __forceinline__ bool wait(uint64_t *bar, uint32_t parity)
{
    return wait_for(bar, parity, kTmaWaitNs, kTmaWaitIters);
}

}  // namespace tma
}  // namespace amhd
