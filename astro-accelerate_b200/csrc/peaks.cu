// peaks.cu -- measured ceiling of the shared-memory load pipe on this GPU.
//
// The channel-quad dedispersion kernel adds four one-byte channel samples per
// 32-bit shared-memory load, so its binding roof is the rate at which an SM
// can return 32-bit shared loads.  This microbenchmark measures that rate:
// every warp issues conflict-free 32-bit loads (32 consecutive words per
// warp-wide load, i.e. one 128-byte wavefront each) from an 8 KB array, with
// no dependence between loads and one integer add per load to keep them
// alive; two 1024-thread CTAs per SM.  The result is thread-loads per second
// over the whole GPU, timed with CUDA events on the caller's stream.
#include <cstdint>

#include <cuda_runtime.h>

#include "aa_b200.h"

namespace aab200 {
namespace {

constexpr int PK_THREADS = 1024;
constexpr int PK_WORDS = 2048; // 8 KB: 128 words x 16 offsets
constexpr int PK_UNROLL = 16;

// loads U, U+1, ... PK_UNROLL-1 of one pass (the offsets are immediates)
template <int U> struct LoadPass {
    static __device__ __forceinline__ void run(unsigned a, unsigned &acc0, unsigned &acc1)
    {
        unsigned v0, v1;
        // volatile: every pass loads again (a plain load of an unchanged
        // address would be hoisted out of the loop)
        asm volatile("ld.volatile.shared.b32 %0, [%1+%2];" : "=r"(v0) : "r"(a), "n"(512 * U));
        asm volatile("ld.volatile.shared.b32 %0, [%1+%2];" : "=r"(v1) : "r"(a), "n"(512 * (U + 1)));
        acc0 += v0;
        acc1 += v1;
        LoadPass<U + 2>::run(a, acc0, acc1);
    }
};
template <> struct LoadPass<PK_UNROLL> {
    static __device__ __forceinline__ void run(unsigned, unsigned &, unsigned &) {}
};

__global__ void __launch_bounds__(PK_THREADS, 2) k_smem_load_rate(int iters, unsigned *sink)
{
    __shared__ uint32_t buf[PK_WORDS];
    for (int i = threadIdx.x; i < PK_WORDS; i += PK_THREADS)
        buf[i] = static_cast<uint32_t>(i * 2654435761u);
    __syncthreads();
    // word (threadIdx.x mod 128) + 128 u (u < 16): the lanes of a warp read 32
    // consecutive words, one register holds the address, the rest is an
    // immediate offset
    const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(buf)) + 4u * (threadIdx.x & 127u);
    unsigned acc0 = 0, acc1 = 0;
    for (int it = 0; it < iters; ++it)
        LoadPass<0>::run(a, acc0, acc1);
    if ((acc0 ^ acc1) == 0x9E3779B9u) // practically never true; keeps the sums alive
        sink[blockIdx.x] = acc0;
}

} // namespace
} // namespace aab200

extern "C" int aa_b200_smem_load_rate(int iters, void *stream, double *loads_per_s, float *ms_out)
{
    using namespace aab200;
    if (iters < 1 || iters > (1 << 20) || !loads_per_s)
        return 1;
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 1;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int grid = 2 * nsm;
    unsigned *sink = nullptr;
    if (cudaMalloc(&sink, sizeof(unsigned) * grid) != cudaSuccess)
        return 1;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = 0;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        rc = 1;
    float ms = 0.f;
    if (!rc) {
        k_smem_load_rate<<<grid, PK_THREADS, 0, st>>>(iters, sink); // warm-up
        cudaEventRecord(e0, st);
        k_smem_load_rate<<<grid, PK_THREADS, 0, st>>>(iters, sink);
        cudaEventRecord(e1, st);
        if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess || ms <= 0.f)
            rc = 1;
    }
    if (!rc) {
        const double loads = static_cast<double>(grid) * PK_THREADS * static_cast<double>(iters) * PK_UNROLL;
        *loads_per_s = loads / (ms * 1e-3);
        if (ms_out)
            *ms_out = ms;
    }
    if (e0)
        cudaEventDestroy(e0);
    if (e1)
        cudaEventDestroy(e1);
    cudaFree(sink);
    return rc;
}
