// ddtr_sub.cu -- two-level dedispersion of one-byte samples over 16-channel
// subbands (tables and launcher; the per-CTA work is body::sub_body in
// ddtr_bodies.cuh).
//
// For a subband of 16 channels c0..c0+15 (four channel quads i = 0..3) and a
// DM trial, the delays split exactly as
//     D[c0 + 4i + k] = D[c0] + off_i + d_ik,
// off_i = D[c0+4i] - D[c0] (quad offset), d_ik = D[c0+4i+k] - D[c0+4i] (skew
// inside the quad).  Within a group of 64 DM trials a subband shows only a
// few distinct (off_1..3, skews) combinations -- its patterns (about 6-11 in
// the survey plan, at most 16 here).  Per pattern p the kernel builds the
// 16-channel partial sums
//     P_p[tau] = sum_i sum_k x[c0+4i+k][w0 + tau + off_i + d_ik]
// (at most 16 * 255, 12 bits) from the quads' pre-skewed rows with IDP4A, and
// a DM trial then adds P_p[t + tau_dm] for its outputs t, two outputs per
// 32-bit add in 16-bit lanes.  Sums are exact integers: the result is
// bit-identical to every other kernel.
//
// Tables per range:
//   sblk [group][nsub][128] int32: pattern block of a (subband, group):
//        [0] patterns, [1..4] distinct quad skews per quad, [8 + 8i + k] skew
//        word k of quad i (d1 | d2<<8 | d3<<16), [40 + p] quad skew indices of
//        pattern p (4 bits per quad), [56 + 3p + i - 1] off_i of pattern p
//   swin [group][nsub_pad] int32: smallest delay of channel c0 over the group
//   stmp [nsub][ndms] int32: pattern << 24 | tau, or -1 (no exact pattern)
//   soff [nsub][ndms] int32: pattern * W + tau (samples), or -1
#include "ddtr_bodies.cuh"

namespace aab200 {

namespace {

// One thread per (subband, DM group).  stats: [0] max tau, [1] max off_i,
// [2] max skew, [3] max patterns, [4] max quad rows (sum of distinct skews),
// [5] number of (subband, DM) without an exact pattern.
__global__ void k_sub_patterns(const int32_t *__restrict__ table, int nch_used, int ndms, int nsub, int nsub_pad,
                               int32_t *__restrict__ sblk, int32_t *__restrict__ swin, int32_t *__restrict__ stmp,
                               int *__restrict__ stats)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    const int g = blockIdx.y;
    if (b >= nsub)
        return;
    const int c0 = 16 * b;
    const int dm0 = 64 * g;
    int32_t *blk = sblk + (static_cast<size_t>(g) * nsub + b) * SUB_BLK_WORDS;
    for (int w = 0; w < SUB_BLK_WORDS; ++w)
        blk[w] = 0;
    int lo = 0x7fffffff;
    for (int j = 0; j < 64; ++j)
        lo = min(lo, table[static_cast<size_t>(c0) * ndms + dm0 + j] & 0xFFFFFF);
    int qcnt[4] = {0, 0, 0, 0};
    int npat = 0, maxtau = 0, maxoff = 0, maxd = 0, fails = 0;
    for (int j = 0; j < 64; ++j) {
        const int dm = dm0 + j;
        const int e0 = table[static_cast<size_t>(c0) * ndms + dm];
        const int d0 = e0 & 0xFFFFFF;
        bool bad = (static_cast<unsigned>(e0) >> 24) != 0u;
        int qidx[4] = {0, 0, 0, 0};
        int off[4] = {0, 0, 0, 0};
        for (int i = 0; i < 4 && !bad; ++i) {
            const int cq = c0 + 4 * i;
            if (cq >= nch_used)
                break;
            const int eq = table[static_cast<size_t>(cq) * ndms + dm];
            const int dq = eq & 0xFFFFFF;
            off[i] = dq - d0;
            if ((static_cast<unsigned>(eq) >> 24) != 0u || off[i] < 0 || off[i] > SUB_MAX_OFF) {
                bad = true;
                break;
            }
            int pw = 0;
            for (int k = 1; k < 4; ++k) {
                const int c = cq + k;
                if (c >= nch_used)
                    break;
                const int ek = table[static_cast<size_t>(c) * ndms + dm];
                const int dk = (ek & 0xFFFFFF) - dq;
                if ((static_cast<unsigned>(ek) >> 24) != 0u || dk < 0 || dk > 255) {
                    bad = true;
                    break;
                }
                maxd = max(maxd, dk);
                pw |= dk << (8 * (k - 1));
            }
            if (bad)
                break;
            int slot = -1;
            for (int k = 0; k < qcnt[i]; ++k)
                if (blk[8 + 8 * i + k] == pw)
                    slot = k;
            if (slot < 0) {
                if (qcnt[i] == SUB_MAX_QPAT) {
                    bad = true;
                    break;
                }
                blk[8 + 8 * i + qcnt[i]] = pw;
                slot = qcnt[i]++;
            }
            qidx[i] = slot;
            maxoff = max(maxoff, off[i]);
        }
        int p = -1;
        if (!bad) {
            const int key = qidx[0] | (qidx[1] << 4) | (qidx[2] << 8) | (qidx[3] << 12);
            for (int k = 0; k < npat && p < 0; ++k)
                if (blk[40 + k] == key && blk[56 + 3 * k] == off[1] && blk[57 + 3 * k] == off[2] &&
                    blk[58 + 3 * k] == off[3])
                    p = k;
            if (p < 0 && npat < SUB_MAX_PAT) {
                blk[40 + npat] = key;
                blk[56 + 3 * npat] = off[1];
                blk[57 + 3 * npat] = off[2];
                blk[58 + 3 * npat] = off[3];
                p = npat++;
            }
        }
        const int tau = d0 - lo;
        if (p < 0) {
            ++fails;
            stmp[static_cast<size_t>(b) * ndms + dm] = -1;
        } else {
            maxtau = max(maxtau, tau);
            stmp[static_cast<size_t>(b) * ndms + dm] = (p << 24) | tau;
        }
    }
    blk[0] = npat;
    for (int i = 0; i < 4; ++i)
        blk[1 + i] = qcnt[i];
    swin[static_cast<size_t>(g) * nsub_pad + b] = lo;
    atomicMax(stats + 0, maxtau);
    atomicMax(stats + 1, maxoff);
    atomicMax(stats + 2, maxd);
    atomicMax(stats + 3, npat);
    atomicMax(stats + 4, qcnt[0] + qcnt[1] + qcnt[2] + qcnt[3]);
    if (fails)
        atomicAdd(stats + 5, fails);
}

__global__ void k_sub_offsets(const int32_t *__restrict__ stmp, size_t n, int W, int32_t *__restrict__ soff)
{
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int v = stmp[i];
    soff[i] = (v < 0) ? -1 : ((v >> 24) * W + (v & 0xFFFFFF));
}

__global__ void __launch_bounds__(body::NTHREADS, 1) k_ddtr_sub(const DdtrLaunch p, const SubLaunch S)
{
    extern __shared__ __align__(16) uint32_t sm[];
    const unsigned bar0 = dev::smem_addr(sm);
    body::init_barriers(bar0);
    __syncthreads();
    unsigned stage_ctr = 0;
    body::sub_body(p, S, blockIdx.x, static_cast<long long>(blockIdx.y) * 512, sm + body::BAR_WORDS, bar0, stage_ctr);
}

} // namespace

cudaError_t launch_sub_patterns(const int32_t *table, int nch_used, int ndms, int nsub, int nsub_pad, int32_t *sblk,
                                int32_t *swin, int32_t *stmp, int *stats, cudaStream_t st)
{
    dim3 grid((nsub + 127) / 128, ndms / 64);
    k_sub_patterns<<<grid, 128, 0, st>>>(table, nch_used, ndms, nsub, nsub_pad, sblk, swin, stmp, stats);
    return cudaGetLastError();
}

cudaError_t launch_sub_offsets(const int32_t *stmp, size_t n, int W, int32_t *soff, cudaStream_t st)
{
    k_sub_offsets<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(stmp, n, W, soff);
    return cudaGetLastError();
}

SubGeometry sub_geometry(int maxtau, int maxoff, int maxd, int maxpat, int maxqrows, int nsub)
{
    SubGeometry G{};
    G.W = (maxtau + 514 + 1) & ~1;                        // samples per partial-sum row (even)
    G.wq = ((G.W + maxoff + 4) + 3) & ~3;                 // samples per quad-sum row (16-bit pairs)
    G.raww = ((((15 + G.wq + maxd + 3) >> 2) + 2) + 3) & ~3; // words per staged raw row
    G.npat = maxpat;
    G.nqrow = maxqrows;
    G.nsub_pad = (nsub + 3) & ~3;
    G.smem_bytes = 4 * (body::BAR_WORDS + body::sub_body_words(G.raww, G.nsub_pad, G.nqrow, G.wq, G.npat, G.W));
    return G;
}

cudaError_t launch_ddtr_sub(const DdtrLaunch &p, const SubLaunch &s, cudaStream_t st)
{
    if (p.group_dms != 64 || s.npat < 1 || s.npat > SUB_MAX_PAT || s.nqrow < 1 || s.nqrow > 4 * SUB_MAX_QPAT ||
        (s.W & 1) || (s.wq & 3) || (s.raww & 3))
        return cudaErrorInvalidValue;
    const size_t smem = 4 * (body::BAR_WORDS + body::sub_body_words(s.raww, s.nsub_pad, s.nqrow, s.wq, s.npat, s.W));
    if (smem > kStagedSmemLimit)
        return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k_ddtr_sub, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess)
        return e;
    dim3 grid(p.ndms / 64, static_cast<unsigned>((p.tp + 511) / 512));
    k_ddtr_sub<<<grid, body::NTHREADS, smem, st>>>(p, s);
    return cudaGetLastError();
}

} // namespace aab200
