// ddtr_quad.cu -- dedispersion of one-byte samples with channel-quad rows
// pre-skewed per delay pattern and 4-channel byte dot products (IDP4A).
//
// For four adjacent channels c..c+3 and one DM trial, the delays differ by a
// small "skew" (d1, d2, d3) = (D[c+1]-D[c], D[c+2]-D[c], D[c+3]-D[c]).  Within a
// group of 64 DM trials only a few distinct skews occur (at most 4 in every
// range of the survey plan).  For each of them the kernel builds, in shared
// memory, a row of 32-bit words
//     P[tau] = (x[c][tau], x[c+1][tau+d1], x[c+2][tau+d2], x[c+3][tau+d3])
// so that one 32-bit load at tau = t + D[c] - window start gives the four
// samples the DM trial adds at output t, and one __dp4a with 0x01010101 adds
// them into a 32-bit accumulator.  Lanes of a warp own outputs t0 + lane + 32m,
// so the loads are conflict-free and need no alignment phases.
//
// Delays are the table of k_delay_table (smallest delay over the reference's
// thread classes + class mask).  A (quad, DM) whose channels have class
// exceptions, a skew outside [0, 255] or no pattern slot left takes a per-byte
// path that applies every class delay exactly; it never occurs in the survey
// plan.  Sums are exact integers, so the result is bit-identical to the other
// kernels.
#include "ddtr_bodies.cuh"

namespace aab200 {

namespace {

using namespace dev;

constexpr int QMAXPAT = 15;

// One thread per (channel quad, DM group): distinct skews, window start.
__global__ void k_quad_patterns(const int32_t *__restrict__ table, int nch_used, int ndms, int group_dms, int nquads,
                                int nq_pad, int32_t *__restrict__ qpat, int32_t *__restrict__ qwin,
                                int32_t *__restrict__ qtmp, int *__restrict__ stats)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int g = blockIdx.y;
    if (q >= nquads)
        return;
    const int c0 = 4 * q;
    const int dm0 = g * group_dms;
    int lo = 0x7fffffff;
    for (int j = 0; j < group_dms; ++j)
        lo = min(lo, table[static_cast<size_t>(c0) * ndms + dm0 + j] & 0xFFFFFF);
    int pats[QMAXPAT];
    int cnt = 0, maxtau = 0, maxd = 0, nbyte = 0;
    for (int j = 0; j < group_dms; ++j) {
        const int dm = dm0 + j;
        const int e0 = table[static_cast<size_t>(c0) * ndms + dm];
        const int d0 = e0 & 0xFFFFFF;
        bool bad = (static_cast<unsigned>(e0) >> 24) != 0u;
        int pw = 0;
#pragma unroll
        for (int i = 1; i < 4; ++i) {
            const int c = c0 + i;
            if (c < nch_used) {
                const int ei = table[static_cast<size_t>(c) * ndms + dm];
                const int di = (ei & 0xFFFFFF) - d0;
                if ((static_cast<unsigned>(ei) >> 24) != 0u || di < 0 || di > 255)
                    bad = true;
                else
                    pw |= di << (8 * (i - 1));
                if (di > maxd)
                    maxd = di;
            }
        }
        const int tau = d0 - lo;
        maxtau = max(maxtau, tau);
        int slot = -1;
        if (!bad) {
            for (int k = 0; k < cnt; ++k)
                if (pats[k] == pw)
                    slot = k;
            if (slot < 0 && cnt < QMAXPAT) {
                pats[cnt] = pw;
                slot = cnt++;
            }
        }
        qtmp[static_cast<size_t>(q) * ndms + dm] = (slot < 0) ? -1 : ((slot << 24) | tau);
        if (slot < 0)
            ++nbyte;
    }
    int32_t *pr = qpat + (static_cast<size_t>(g) * nquads + q) * 16;
    for (int k = 0; k < QMAXPAT; ++k)
        pr[k] = (k < cnt) ? pats[k] : 0;
    pr[15] = cnt;
    qwin[static_cast<size_t>(g) * nq_pad + q] = lo;
    atomicMax(stats + 0, maxtau);
    atomicMax(stats + 1, maxd);
    atomicMax(stats + 2, cnt);
    if (nbyte)
        atomicAdd(stats + 3, nbyte); // (quad, DM) entries that need the per-byte path
}

// pairs = 0: slot*W + tau (words of a pre-skewed row); pairs = 1: the pair
// body's offsets slot*W + (tau&1)*W/2 + tau/2 (E half for even tau, O half
// for odd tau)
__global__ void k_quad_offsets(const int32_t *__restrict__ qtmp, size_t n, int W, int pairs,
                               int32_t *__restrict__ qoff)
{
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int v = qtmp[i];
    const int tau = v & 0xFFFFFF;
    qoff[i] = (v < 0) ? -1 : ((v >> 24) * W + (pairs ? (tau & 1) * (W >> 1) + (tau >> 1) : tau));
}

// M = 16: 16 warps x 4 DM trials, one CTA per SM (127 registers);
// M = 8: 8 warps x 8 DM trials, two CTAs per SM, so that one CTA issues
// while the other waits at its stage barrier.
template <int M, int DW, bool SWITCH, int MINB, bool LOADALL = false, bool NOSLOW = false, bool ASM = false>
__global__ void __launch_bounds__(32 * 64 / DW, MINB) k_ddtr_quad(const DdtrLaunch p, const QuadLaunch Q)
{
    extern __shared__ __align__(16) uint32_t sm[];
    const unsigned bar0 = smem_addr(sm);
    body::init_barriers(bar0);
    __syncthreads();
    unsigned stage_ctr = 0;
    body::quad_body<M, DW, SWITCH, LOADALL, NOSLOW, ASM>(p, Q, blockIdx.x,
                                                         static_cast<long long>(blockIdx.y) * (32 * M),
                                                         sm + body::BAR_WORDS, bar0, stage_ctr);
}

// 16 consumer + WS_PROD producer warps (body::quad_ws_body); five warps per
// scheduler leave 96 registers a thread.
__global__ void __launch_bounds__(body::WS_THREADS, 1) k_ddtr_quadws(const DdtrLaunch p, const QuadLaunch Q)
{
    extern __shared__ __align__(16) uint32_t sm[];
    const unsigned bar0 = smem_addr(sm);
    body::init_barriers(bar0);
    __syncthreads();
    unsigned stage_ctr = 0;
    body::quad_ws_body(p, Q, blockIdx.x, static_cast<long long>(blockIdx.y) * 512, sm + body::BAR_WORDS, bar0,
                       stage_ctr);
}

// Channel-quad pair kernel (body::quad_pair_body): 16 warps x 4 DM trials x
// 256 output pairs, one CTA per SM.
__global__ void __launch_bounds__(512, 1) k_ddtr_quadpair(const DdtrLaunch p, const QuadLaunch Q)
{
    extern __shared__ __align__(16) uint32_t sm[];
    const unsigned bar0 = smem_addr(sm);
    body::init_barriers(bar0);
    __syncthreads();
    unsigned stage_ctr = 0;
    body::quad_pair_body<8>(p, Q, blockIdx.x, static_cast<long long>(blockIdx.y) * 512, sm + body::BAR_WORDS, bar0,
                            stage_ctr);
}

// Split-phase channel-quad kernel (body::quad_sp_body): 16 warps x 4 DM
// trials x 512 samples, one CTA per SM.
__global__ void __launch_bounds__(32 * body::SP_WARPS, 1) k_ddtr_quadsp(const DdtrLaunch p, const QuadLaunch Q)
{
    extern __shared__ __align__(16) uint32_t sm[];
    const unsigned bar0 = smem_addr(sm);
    body::init_barriers(bar0);
    __syncthreads();
    unsigned sp_ctr = 0;
    body::quad_sp_body<16>(p, Q, blockIdx.x, static_cast<long long>(blockIdx.y) * 512, sm + body::BAR_WORDS, bar0,
                           sp_ctr);
}

} // namespace

size_t quadsp_smem_bytes(const QuadLaunch &q)
{
    return 4 * (body::BAR_WORDS + body::quad_sp_body_words(q.qs, q.raww, q.nq_pad, q.npool, q.W));
}

cudaError_t launch_ddtr_quadsp(const DdtrLaunch &p, const QuadLaunch &q, cudaStream_t st)
{
    if (p.group_dms != 64 || q.qs < 1 || q.qs > 8 || q.M != 16)
        return cudaErrorInvalidValue;
    const size_t smem = quadsp_smem_bytes(q);
    if (smem > 227 * 1024)
        return cudaErrorInvalidValue;
    cudaError_t e =
        cudaFuncSetAttribute(k_ddtr_quadsp, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess)
        return e;
    dim3 grid(p.ndms / p.group_dms, static_cast<unsigned>((p.tp + 511) / 512));
    k_ddtr_quadsp<<<grid, 32 * body::SP_WARPS, smem, st>>>(p, q);
    return cudaGetLastError();
}

size_t quadws_smem_bytes(const QuadLaunch &q)
{
    return 4 * (body::BAR_WORDS + body::quad_ws_body_words(q.qs, q.raww, q.nq_pad, q.npool, q.W));
}

cudaError_t launch_ddtr_quadws(const DdtrLaunch &p, const QuadLaunch &q, cudaStream_t st)
{
    if (p.group_dms != 64 || q.qs < 1 || q.qs > 8 || q.M != 16)
        return cudaErrorInvalidValue;
    const size_t smem = quadws_smem_bytes(q);
    if (smem > 227 * 1024)
        return cudaErrorInvalidValue;
    cudaError_t e =
        cudaFuncSetAttribute(k_ddtr_quadws, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess)
        return e;
    dim3 grid(p.ndms / p.group_dms, static_cast<unsigned>((p.tp + 511) / 512));
    k_ddtr_quadws<<<grid, body::WS_THREADS, smem, st>>>(p, q);
    return cudaGetLastError();
}

cudaError_t launch_quad_patterns(const int32_t *table, int nch_used, int ndms, int group_dms, int nquads, int nq_pad,
                                 int32_t *qpat, int32_t *qwin, int32_t *qtmp, int *stats, cudaStream_t st)
{
    dim3 grid((nquads + 127) / 128, ndms / group_dms);
    k_quad_patterns<<<grid, 128, 0, st>>>(table, nch_used, ndms, group_dms, nquads, nq_pad, qpat, qwin, qtmp, stats);
    return cudaGetLastError();
}

cudaError_t launch_quad_offsets(const int32_t *qtmp, size_t n, int W, int32_t *qoff, cudaStream_t st, int pairs)
{
    k_quad_offsets<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(qtmp, n, W, pairs, qoff);
    return cudaGetLastError();
}

QuadGeometry quad_geometry(int span, int dmax, int maxcnt, int group_dms, int nquads, int out_words, int qs, int npool)
{
    QuadGeometry G;
    G.M = out_words;
    G.W = ((span + 32 * out_words) + 3) & ~3;
    G.raww = ((((15 + G.W + dmax + 3) >> 2) + 2) + 3) & ~3;
    G.qs = qs;
    G.npool = npool > 0 ? npool : qs * (maxcnt > 0 ? maxcnt : 1);
    G.nq_pad = (nquads + 3) & ~3;
    G.smem_bytes = 4 * (body::BAR_WORDS + body::quad_body_words(qs, group_dms, G.raww, G.nq_pad, G.npool, G.W));
    return G;
}

template <typename K>
static cudaError_t launch_quad_instance(K kernel, int threads, const DdtrLaunch &p, const QuadLaunch &q, size_t smem,
                                        cudaStream_t st)
{
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess)
        return e;
    const long long tile = 32LL * q.M;
    dim3 grid(p.ndms / p.group_dms, static_cast<unsigned>((p.tp + tile - 1) / tile));
    kernel<<<grid, threads, smem, st>>>(p, q);
    return cudaGetLastError();
}

cudaError_t launch_ddtr_quad(const DdtrLaunch &p, const QuadLaunch &q, cudaStream_t st)
{
    if (p.group_dms != 64 || q.qs < 1 || q.qs > 8)
        return cudaErrorInvalidValue;
    const size_t smem = 4 * (body::BAR_WORDS + body::quad_body_words(q.qs, p.group_dms, q.raww, q.nq_pad, q.npool, q.W));
    if (q.M == 16 && q.flavour == 3)
        return launch_quad_instance(k_ddtr_quadpair, 512, p, q, smem, st);
    if (q.M == 16 && q.flavour == 4)
        return launch_quad_instance(k_ddtr_quad<16, 4, false, 1, true>, 512, p, q, smem, st);
    if (q.M == 16 && q.flavour == 5)
        return launch_quad_instance(k_ddtr_quad<16, 4, false, 1, false, true>, 512, p, q, smem, st);
    if (q.M == 16 && q.flavour == 6)
        return launch_quad_instance(k_ddtr_quad<16, 4, false, 1, true, true>, 512, p, q, smem, st);
    if (q.M == 16 && q.flavour == 7)
        return launch_quad_instance(k_ddtr_quad<16, 4, false, 1, true, true, true>, 512, p, q, smem, st);
    if (q.M == 8 && q.flavour == 2)
        return launch_quad_instance(k_ddtr_quad<8, 4, true, 2>, 512, p, q, smem, st);
    if (q.M == 8)
        return launch_quad_instance(k_ddtr_quad<8, 8, false, 2>, 256, p, q, smem, st);
    if (q.M == 16 && q.flavour == 1)
        return launch_quad_instance(k_ddtr_quad<16, 4, true, 1>, 512, p, q, smem, st);
    if (q.M == 16)
        return launch_quad_instance(k_ddtr_quad<16, 4, false, 1>, 512, p, q, smem, st);
    return cudaErrorInvalidValue;
}

} // namespace aab200
