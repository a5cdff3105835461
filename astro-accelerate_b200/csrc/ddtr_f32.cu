// ddtr_f32.cu -- dedispersion of two-byte samples (16-bit and rescaled 32-bit
// filterbanks) with TMA-staged channel rows and fp32 sums in channel order,
// one launch per (time chunk, DM range).  The per-CTA work is
// body::f32_body (ddtr_bodies.cuh).
#include "ddtr_bodies.cuh"

namespace aab200 {

namespace {

using namespace dev;

constexpr int F32_M = 16; // outputs per lane per DM trial (tile of 512 samples)

__global__ void __launch_bounds__(body::NTHREADS, 1) k_ddtr_f32(const DdtrLaunch p, const F32Launch F)
{
    extern __shared__ __align__(16) uint32_t sm[];
    const unsigned bar0 = smem_addr(sm);
    body::init_barriers(bar0);
    __syncthreads();
    unsigned stage_ctr = 0;
    body::f32_body<F32_M>(p, F, blockIdx.x, static_cast<long long>(blockIdx.y) * (32 * F32_M), sm + body::BAR_WORDS,
                          bar0, stage_ctr);
}

} // namespace

F32Geometry f32_geometry(int span, int group_dms, int nchans, int cs)
{
    F32Geometry G{};
    G.f.W = (span + 32 * F32_M + 3) & ~3;
    G.f.rawh = (G.f.W + 8 + 7) & ~7;
    G.f.nch_pad = (nchans + 3) & ~3;
    const int cands[] = {16, 8, 4};
    for (int c : cands) {
        if (cs > 0 && c != cs)
            continue;
        const size_t bytes = 4 * (body::BAR_WORDS + body::f32_body_words(c, group_dms, G.f.rawh, G.f.nch_pad, G.f.W));
        if (bytes <= kStagedSmemLimit) {
            G.f.cs = c;
            G.smem_bytes = bytes;
            return G;
        }
    }
    G.smem_bytes = 0;
    return G;
}

cudaError_t launch_ddtr_f32(const DdtrLaunch &p, const F32Launch &f, cudaStream_t st)
{
    if (p.group_dms != 64 || (f.cs != 4 && f.cs != 8 && f.cs != 16 && f.cs != 32) || (f.W & 3) || (f.rawh & 7) ||
        f.rawh < f.W + 8 || f.W < p.span + 32 * F32_M)
        return cudaErrorInvalidValue;
    const size_t smem = 4 * (body::BAR_WORDS + body::f32_body_words(f.cs, p.group_dms, f.rawh, f.nch_pad, f.W));
    cudaError_t e = cudaFuncSetAttribute(k_ddtr_f32, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess)
        return e;
    const long long tile = 32LL * F32_M;
    dim3 grid(p.ndms / p.group_dms, static_cast<unsigned>((p.tp + tile - 1) / tile));
    k_ddtr_f32<<<grid, body::NTHREADS, smem, st>>>(p, f);
    return cudaGetLastError();
}

} // namespace aab200
