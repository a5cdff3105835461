// selftest.cu -- checks of the library's failure handling that need no fault:
// a bounded wait that is made to run out, and the host-side injection
// counter (fault.hpp).
#include <atomic>

#include <cuda_runtime.h>

#include "aa_b200.h"
#include "ddtr_kernels.cuh"
#include "device_util.cuh"
#include "fault.hpp"

namespace aab200 {

namespace {

std::atomic<long long> g_countdown{0};

// An mbarrier that expects two arrivals and gets one: its phase never
// completes, so the bounded wait gives up after `limit` polls and the kernel
// reports DERR_TIMEOUT, exactly as the staged kernels do when a copy does not
// land.  No copy is in flight and nothing else waits on the barrier.
__global__ void k_wait_probe(int *err, int limit)
{
    __shared__ __align__(8) unsigned long long bar;
    const unsigned b = dev::smem_addr(&bar);
    if (threadIdx.x == 0) {
        dev::mbar_init(b, 2);
        dev::mbar_init_fence();
    }
    __syncthreads();
    if (threadIdx.x == 0)
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(b) : "memory");
    const bool ok = dev::mbar_wait_limit(b, 0, limit);
    if (!ok && threadIdx.x == 0)
        atomicOr(err, DERR_TIMEOUT);
}

} // namespace

void arm_injected_failure(long long n) { g_countdown.store(n > 0 ? n : 0); }

bool injected_failure_now()
{
    long long c = g_countdown.load();
    while (c > 0) {
        if (g_countdown.compare_exchange_weak(c, c - 1))
            return c == 1;
    }
    return false;
}

long long injected_failure_countdown() { return g_countdown.load(); }

} // namespace aab200

extern "C" {

int aa_b200_selftest_bounded_wait(int limit, int *status)
{
    using namespace aab200;
    if (limit < 1 || limit > (1 << 22) || !status)
        return 1;
    int *d_err = nullptr;
    if (cudaMalloc(&d_err, sizeof(int)) != cudaSuccess)
        return 1;
    int rc = 0;
    if (cudaMemset(d_err, 0, sizeof(int)) != cudaSuccess)
        rc = 1;
    if (!rc) {
        k_wait_probe<<<1, 32>>>(d_err, limit);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
            cudaMemcpy(status, d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = 1;
    }
    cudaFree(d_err);
    return rc;
}

int aa_b200_binary_version(int *version)
{
    if (!version)
        return 1;
    cudaFuncAttributes a{};
    if (cudaFuncGetAttributes(&a, aab200::k_wait_probe) != cudaSuccess)
        return 1;
    *version = a.binaryVersion;
    return 0;
}

void aa_b200_debug_fail_after(long long n) { aab200::arm_injected_failure(n); }

long long aa_b200_debug_fail_countdown(void) { return aab200::injected_failure_countdown(); }

} // extern "C"
