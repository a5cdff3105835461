// ddtr_batch.cu -- persistent dedispersion over many beams in one launch.
//
// The grid is sized to the GPU (SMs x resident CTAs); every CTA takes work
// items from a device counter until the table is exhausted.  An item is one
// output tile (64 DM trials x 512 samples) of one (beam, chunk, range) job;
// the jobs are ordered heaviest first on the host, so the items that finish
// last are the cheap ones.  Consecutive items are the DM groups of one time
// tile, so the input rows they stage are fetched from HBM once and served
// from L2 to the others.  The tile itself is computed by the same device
// bodies as the one-launch-per-job kernels (ddtr_bodies.cuh), so every beam's
// output is bit-identical to its plain run.
//
// Shared memory: [mbarriers][job descriptor][body area], the body area sized
// for the largest job.  The mbarriers are initialised once; running stage
// counters carry their phases from item to item (one for the TMA ring of
// the bodies of the instance, one for the split-phase quad body's barriers).
#include "ddtr_bodies.cuh"

namespace aab200 {

namespace {

using namespace dev;

constexpr int JD_WORDS = 72; // shared-memory words kept for the job descriptor
static_assert(sizeof(BatchJobDev) <= 4 * JD_WORDS, "job descriptor larger than its shared-memory slot");
static_assert(sizeof(BatchJobDev) % 4 == 0, "job descriptor is copied word by word");
static_assert((body::BAR_WORDS + JD_WORDS) % 4 == 0, "the body area must start on a 16-byte boundary");
constexpr int BATCH_M = 16;

// Body sets, one kernel instance each, so that every instance's bodies fit
// the 128 registers a thread has at 512 threads without spilling:
// PSET_QUAD the channel-quad and fp32 bodies, PSET_SP those and the
// split-phase quad body (jobs of variant 6), PSET_SUB the subband body alone
// (jobs of variant 4; with the quad bodies in one instance it spilled).
template <int SET>
__global__ void __launch_bounds__(body::NTHREADS, 1)
    k_ddtr_persistent(const BatchJobDev *__restrict__ jobs, int njobs, long long total_items,
                      unsigned long long *__restrict__ counter)
{
    extern __shared__ __align__(16) uint32_t sm[];
    __shared__ long long s_item;
    __shared__ int s_job;
    const int tid = threadIdx.x;
    const unsigned bar0 = smem_addr(sm);
    uint32_t *jd_words = sm + body::BAR_WORDS;
    const BatchJobDev &jd = *reinterpret_cast<const BatchJobDev *>(jd_words);
    uint32_t *area = sm + body::BAR_WORDS + JD_WORDS;
    body::init_barriers(bar0);
    unsigned stage_ctr = 0; // phases of the TMA ring barriers (the subband ring in PSET_SUB)
    unsigned sp_ctr = 0;    // phases of the split-phase quad body's barriers
    int jcur = 0; // thread 0: job of the last item (items arrive in increasing order)
    for (;;) {
        if (tid == 0) {
            const long long item = static_cast<long long>(atomicAdd(counter, 1ull));
            if (item < total_items)
                while (jcur + 1 < njobs && jobs[jcur + 1].item0 <= item)
                    ++jcur;
            s_item = item;
            s_job = jcur;
        }
        __syncthreads();
        const long long item = s_item;
        if (item >= total_items)
            break;
        const uint32_t *src = reinterpret_cast<const uint32_t *>(jobs + s_job);
        if (tid < static_cast<int>(sizeof(BatchJobDev) / 4))
            jd_words[tid] = src[tid];
        __syncthreads();
        const long long li = item - jd.item0;
        const int g = static_cast<int>(li % jd.groups);
        const long long t0 = (li / jd.groups) * (32 * BATCH_M);
        bool ok = false; // stays false for a job this instance has no body for (the host never issues one)
        if (SET == PSET_SUB) {
            if (jd.variant == 4)
                ok = body::sub_body(jd.p, jd.s, g, t0, area, bar0, stage_ctr);
        } else if (jd.variant == 2 && jd.q.flavour == 7) {
            ok = body::quad_body<BATCH_M, 4, false, true, true, true>(jd.p, jd.q, g, t0, area, bar0, stage_ctr);
        } else if (jd.variant == 2) {
            ok = body::quad_body<BATCH_M, 4>(jd.p, jd.q, g, t0, area, bar0, stage_ctr);
        } else if (SET == PSET_SP && jd.variant == 6) {
            ok = body::quad_sp_body<BATCH_M>(jd.p, jd.q, g, t0, area, bar0, sp_ctr);
        } else if (jd.variant == 3) {
            ok = body::f32_body<BATCH_M>(jd.p, jd.f, g, t0, area, bar0, stage_ctr);
        }
        fence_proxy_async();
        // a tile whose copies timed out ends this CTA (the flag is set); the
        // decision is block-wide so that no thread is left at a barrier
        if (__syncthreads_or(!ok))
            break;
    }
}

} // namespace

size_t persistent_job_smem(const BatchJobDev &j)
{
    size_t words;
    if (j.variant == 2)
        words = body::quad_body_words(j.q.qs, j.p.group_dms, j.q.raww, j.q.nq_pad, j.q.npool, j.q.W);
    else if (j.variant == 6)
        words = body::quad_sp_body_words(j.q.qs, j.q.raww, j.q.nq_pad, j.q.npool, j.q.W);
    else if (j.variant == 4)
        words = body::sub_body_words(j.s.raww, j.s.nsub_pad, j.s.nqrow, j.s.wq, j.s.npat, j.s.W);
    else
        words = body::f32_body_words(j.f.cs, j.p.group_dms, j.f.rawh, j.f.nch_pad, j.f.W);
    return 4 * (body::BAR_WORDS + JD_WORDS + words);
}

template <int SET> const void *persistent_fn() { return reinterpret_cast<const void *>(k_ddtr_persistent<SET>); }

const void *persistent_fn_of(int set)
{
    return (set == PSET_SP) ? persistent_fn<PSET_SP>() : (set == PSET_SUB) ? persistent_fn<PSET_SUB>()
                                                                           : persistent_fn<PSET_QUAD>();
}

int persistent_blocks_per_sm(size_t smem_bytes, int set)
{
    const void *fn = persistent_fn_of(set);
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem_bytes)) !=
        cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, body::NTHREADS, smem_bytes) != cudaSuccess)
        return 0;
    return n;
}

cudaError_t launch_ddtr_persistent(const BatchJobDev *jobs, int njobs, long long total_items,
                                   unsigned long long *counter, size_t smem_bytes, int grid, int set, cudaStream_t st)
{
    if (njobs <= 0 || total_items <= 0)
        return cudaSuccess;
    if (grid <= 0 || smem_bytes > 227 * 1024 || set < PSET_QUAD || set > PSET_SUB)
        return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(persistent_fn_of(set), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem_bytes));
    if (e != cudaSuccess)
        return e;
    if (set == PSET_SP)
        k_ddtr_persistent<PSET_SP><<<grid, body::NTHREADS, smem_bytes, st>>>(jobs, njobs, total_items, counter);
    else if (set == PSET_SUB)
        k_ddtr_persistent<PSET_SUB><<<grid, body::NTHREADS, smem_bytes, st>>>(jobs, njobs, total_items, counter);
    else
        k_ddtr_persistent<PSET_QUAD><<<grid, body::NTHREADS, smem_bytes, st>>>(jobs, njobs, total_items, counter);
    return cudaGetLastError();
}

} // namespace aab200
