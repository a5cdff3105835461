// device_util.cuh -- shared-memory staging primitives for the sm_100a kernels:
// cp.async (16-byte LDGSTS), TMA bulk copies completing on mbarriers, and
// bounded mbarrier waits (a copy that never lands must not hang the GPU).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace aab200 {
namespace dev {

__device__ __forceinline__ void cp_async16(void *smem_ptr, const void *gptr)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_ptr));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gptr) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ unsigned smem_addr(const void *p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity)
{
    unsigned done;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}\n"
                 : "=r"(done)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return done != 0;
}

// Wait of at most `limit` polls; false when the phase did not complete.
__device__ __forceinline__ bool mbar_wait_limit(unsigned bar, unsigned parity, int limit)
{
    for (int i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity))
            return true;
    return false;
}

// Bounded wait (about a second at the try_wait suspend time); false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity)
{
    return mbar_wait_limit(bar, parity, 1 << 22);
}

// Orders earlier generic-proxy accesses of shared memory before later
// async-proxy (TMA) writes to it.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// 1-D TMA copy global -> shared; dst/src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void tma_load_1d(unsigned dst, const void *src, unsigned bytes, unsigned bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

} // namespace dev
} // namespace aab200
