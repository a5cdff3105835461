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
#include "ddtr_kernels.cuh"
#include "device_util.cuh"

namespace aab200 {

namespace {

using namespace dev;

constexpr int QNSTAGE = 3; // TMA ring depth
constexpr int QDMW = 4;    // DM trials per warp
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
    int cnt = 0, maxtau = 0, maxd = 0;
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
    }
    int32_t *pr = qpat + (static_cast<size_t>(g) * nquads + q) * 16;
    for (int k = 0; k < QMAXPAT; ++k)
        pr[k] = (k < cnt) ? pats[k] : 0;
    pr[15] = cnt;
    qwin[static_cast<size_t>(g) * nq_pad + q] = lo;
    atomicMax(stats + 0, maxtau);
    atomicMax(stats + 1, maxd);
    atomicMax(stats + 2, cnt);
}

__global__ void k_quad_offsets(const int32_t *__restrict__ qtmp, size_t n, int W, int32_t *__restrict__ qoff)
{
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int v = qtmp[i];
    qoff[i] = (v < 0) ? -1 : ((v >> 24) * W + (v & 0xFFFFFF));
}

__device__ __forceinline__ int output_class(int kind, long long t)
{
    return (kind == KIND_SHARED4) ? static_cast<int>((t & 31) >> 2) : static_cast<int>((t & 15) >> 1);
}

template <int M>
__global__ void __launch_bounds__(512, (M <= 8) ? 2 : 1) k_ddtr_quad(const DdtrLaunch p, const QuadLaunch Q)
{
    extern __shared__ __align__(16) uint32_t sm[];
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int nwarps = blockDim.x >> 5;
    const int GD = p.group_dms;
    const int g = blockIdx.x;
    const int dm0 = g * GD;
    const long long t0 = static_cast<long long>(blockIdx.y) * (32 * M);
    const int W = Q.W, RAWW = Q.raww, QS = Q.qs;
    const unsigned char *in = static_cast<const unsigned char *>(p.in);
    const int nstages = (Q.nquads + QS - 1) / QS;

    // word offsets of the shared-memory areas
    const int o_raw = 0;
    const int o_ent = o_raw + QNSTAGE * QS * 4 * RAWW;
    const int o_pat = o_ent + QNSTAGE * QS * GD;
    const int o_rsh = o_pat + QNSTAGE * QS * 16;
    const int o_bar = o_rsh + QNSTAGE * QS * 4;
    const int o_qw = o_bar + 2 * QNSTAGE + 2;
    const int o_P = ((o_qw + Q.nq_pad) + 3) & ~3;
    const unsigned bar0 = smem_addr(&sm[o_bar]);

    for (int i = tid; i < (Q.nq_pad >> 2); i += blockDim.x)
        cp_async16(&sm[o_qw + 4 * i], Q.qwin + static_cast<size_t>(g) * Q.nq_pad + 4 * i);
    cp_async_commit();
    if (tid == 0)
        for (int i = 0; i < QNSTAGE; ++i)
            mbar_init(bar0 + 8 * i, 1);
    cp_async_wait<0>();
    mbar_init_fence();
    __syncthreads();

    // warp 0: raw rows of the stage's channels, their DM offsets, patterns
    auto issue = [&](int s) {
        if (warp != 0 || s >= nstages)
            return;
        const int slot = s % QNSTAGE;
        const int q0 = s * QS;
        const int nq = min(QS, Q.nquads - q0);
        const int c0 = 4 * q0;
        const int nrows = max(0, min(4 * nq, p.nch_used - c0));
        const unsigned bar = bar0 + 8 * slot;
        fence_proxy_async();
        if (lane == 0)
            mbar_expect_tx(bar, static_cast<unsigned>(nrows * RAWW * 4 + nq * GD * 4 + nq * 64));
        __syncwarp();
        if (lane < 4 * nq) {
            const int c = c0 + lane;
            if (lane < nrows) {
                const int w0 = static_cast<int>(sm[o_qw + q0 + (lane >> 2)]);
                const uintptr_t a = reinterpret_cast<uintptr_t>(in + static_cast<long long>(c) * p.stride + t0 + w0);
                sm[o_rsh + slot * QS * 4 + lane] = static_cast<uint32_t>(a & 15);
                tma_load_1d(smem_addr(&sm[o_raw + (slot * QS * 4 + lane) * RAWW]),
                            reinterpret_cast<const void *>(a & ~static_cast<uintptr_t>(15)),
                            static_cast<unsigned>(RAWW * 4), bar);
            } else {
                sm[o_rsh + slot * QS * 4 + lane] = 0xFFFFFFFFu; // channel contributes nothing
            }
        }
        if (lane < nq)
            tma_load_1d(smem_addr(&sm[o_ent + (slot * QS + lane) * GD]),
                        Q.qoff + static_cast<size_t>(q0 + lane) * p.ndms + dm0, static_cast<unsigned>(GD * 4), bar);
        if (lane == 0)
            tma_load_1d(smem_addr(&sm[o_pat + slot * QS * 16]), Q.qpat + (static_cast<size_t>(g) * Q.nquads + q0) * 16,
                        static_cast<unsigned>(nq * 64), bar);
    };

    bool ok = true;
    // pre-skewed quad rows of stage s into P buffer b
    auto build = [&](int s, int b) {
        const int slot = s % QNSTAGE;
        if (!mbar_wait_bounded(bar0 + 8 * slot, static_cast<unsigned>((s / QNSTAGE) & 1))) {
            if (ok)
                atomicOr(p.err, DERR_TIMEOUT);
            ok = false;
        }
        const int q0 = s * QS;
        const int nq = min(QS, Q.nquads - q0);
        int total = 0;
        for (int q = 0; q < nq; ++q)
            total += static_cast<int>(sm[o_pat + (slot * QS + q) * 16 + 15]);
        total = min(total, Q.npool);
        // one warp per pattern row; the lanes walk the row four words at a time
        const int n4 = W >> 2;
        int q = 0, base = 0;
        int cnt_q = (nq > 0) ? static_cast<int>(sm[o_pat + (slot * QS) * 16 + 15]) : 0;
        for (int r = warp; r < total; r += nwarps) {
            while (r >= base + cnt_q && q + 1 < nq) {
                base += cnt_q;
                ++q;
                cnt_q = static_cast<int>(sm[o_pat + (slot * QS + q) * 16 + 15]);
            }
            const unsigned pw = sm[o_pat + (slot * QS + q) * 16 + (r - base)];
            int d[4], rs[4], rb[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                d[i] = (i == 0) ? 0 : static_cast<int>((pw >> (8 * (i - 1))) & 255u);
                rs[i] = static_cast<int>(sm[o_rsh + slot * QS * 4 + 4 * q + i]);
                rb[i] = o_raw + (slot * QS * 4 + 4 * q + i) * RAWW;
            }
            const int prow = o_P + (b * Q.npool + r) * W;
            for (int t4 = lane; t4 < n4; t4 += 32) {
                const int tau = 4 * t4;
                uint32_t a[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    if (rs[i] < 0) {
                        a[i] = 0u;
                    } else {
                        const int bb = rs[i] + tau + d[i];
                        const int wi = rb[i] + (bb >> 2);
                        a[i] = __funnelshift_r(sm[wi], sm[wi + 1], 8u * static_cast<unsigned>(bb & 3));
                    }
                }
                // 4x4 byte transpose: word k of the result holds sample tau+k of the four channels
                const uint32_t lo01 = __byte_perm(a[0], a[1], 0x5140), hi01 = __byte_perm(a[0], a[1], 0x7362);
                const uint32_t lo23 = __byte_perm(a[2], a[3], 0x5140), hi23 = __byte_perm(a[2], a[3], 0x7362);
                uint4 v;
                v.x = __byte_perm(lo01, lo23, 0x5410);
                v.y = __byte_perm(lo01, lo23, 0x7632);
                v.z = __byte_perm(hi01, hi23, 0x5410);
                v.w = __byte_perm(hi01, hi23, 0x7632);
                *reinterpret_cast<uint4 *>(&sm[prow + tau]) = v;
            }
        }
    };

    uint32_t acc[QDMW][M];
#pragma unroll
    for (int j = 0; j < QDMW; ++j)
#pragma unroll
        for (int m = 0; m < M; ++m)
            acc[j][m] = 0u;

    // per-byte path for one (quad, DM trial): every channel with its own class delays
    auto slow = [&](int j, int slot, int q0, int q) {
        const int dm = dm0 + warp * QDMW + j;
        const int lo = static_cast<int>(sm[o_qw + q0 + q]);
#pragma unroll 1
        for (int i = 0; i < 4; ++i) {
            const int c = 4 * (q0 + q) + i;
            const int rs = static_cast<int>(sm[o_rsh + slot * QS * 4 + 4 * q + i]);
            if (c >= p.nch_used || rs < 0)
                continue;
            const int rb = o_raw + (slot * QS * 4 + 4 * q + i) * RAWW;
            const int ee = p.table[static_cast<size_t>(c) * p.ndms + dm];
            const int dd = (ee & 0xFFFFFF) - lo;
            const unsigned mask = static_cast<unsigned>(ee) >> 24;
#pragma unroll
            for (int m = 0; m < M; ++m) {
                const int tl = lane + 32 * m;
                const int o = dd + static_cast<int>((mask >> output_class(p.kind, t0 + tl)) & 1u) + tl;
                const int bb = rs + o;
                if (o < 0 || bb >= RAWW * 4) {
                    atomicOr(p.err, DERR_WINDOW);
                    continue;
                }
                acc[j][m] += (sm[rb + (bb >> 2)] >> (8u * static_cast<unsigned>(bb & 3))) & 255u;
            }
        }
    };

#pragma unroll
    for (int s = 0; s < QNSTAGE - 1; ++s)
        issue(s);
    __syncthreads(); // raw-row shifts written by warp 0 become visible
    build(0, 0);
    __syncthreads();
    issue(QNSTAGE - 1);

    for (int s = 0; s < nstages; ++s) {
        if (s + 1 < nstages)
            build(s + 1, (s + 1) & 1);
        const int slot = s % QNSTAGE;
        const int q0 = s * QS;
        const int nq = min(QS, Q.nquads - q0);
        if (ok) {
            int rbase = 0;
            for (int q = 0; q < nq; ++q) {
                const int4 e4 = *reinterpret_cast<const int4 *>(&sm[o_ent + (slot * QS + q) * GD + warp * QDMW]);
                const int prow = o_P + ((s & 1) * Q.npool + rbase) * W + lane;
                const int ej[QDMW] = {e4.x, e4.y, e4.z, e4.w};
                if ((e4.x | e4.y | e4.z | e4.w) >= 0) {
#pragma unroll
                    for (int j = 0; j < QDMW; ++j) {
                        uint32_t w[M];
#pragma unroll
                        for (int m = 0; m < M; ++m)
                            w[m] = sm[prow + ej[j] + 32 * m];
#pragma unroll
                        for (int m = 0; m < M; ++m)
                            acc[j][m] = __dp4a(w[m], 0x01010101u, acc[j][m]);
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < QDMW; ++j) {
                        if (ej[j] >= 0) {
#pragma unroll
                            for (int m = 0; m < M; ++m)
                                acc[j][m] = __dp4a(sm[prow + ej[j] + 32 * m], 0x01010101u, acc[j][m]);
                        } else {
                            slow(j, slot, q0, q);
                        }
                    }
                }
                rbase += static_cast<int>(sm[o_pat + (slot * QS + q) * 16 + 15]);
            }
        }
        __syncthreads();
        issue(s + QNSTAGE);
    }
    if (!ok)
        return;

    // (float)S / nchans / bin, the reference's expression (4-bit: / nchans)
#pragma unroll
    for (int j = 0; j < QDMW; ++j) {
        const int dm = dm0 + warp * QDMW + j;
        if (dm >= p.ndms)
            continue;
        float *orow = p.out + static_cast<long long>(dm) * p.out_pitch;
#pragma unroll
        for (int m = 0; m < M; ++m) {
            const long long t = t0 + lane + 32 * m;
            if (t < p.tp) {
                const float v = static_cast<float>(static_cast<int>(acc[j][m]));
                orow[t] = p.divide_by_bin ? (v / p.nchans_f / p.bin_f) : (v / p.nchans_f);
            }
        }
    }
}

size_t quad_smem_words(int qs, int group_dms, int raww, int nq_pad, int npool, int W)
{
    int o = QNSTAGE * qs * 4 * raww;
    o += QNSTAGE * qs * group_dms;
    o += QNSTAGE * qs * 16;
    o += QNSTAGE * qs * 4;
    o += 2 * QNSTAGE + 2;
    o += nq_pad;
    o = (o + 3) & ~3;
    o += 2 * npool * W;
    return static_cast<size_t>(o);
}

} // namespace

cudaError_t launch_quad_patterns(const int32_t *table, int nch_used, int ndms, int group_dms, int nquads, int nq_pad,
                                 int32_t *qpat, int32_t *qwin, int32_t *qtmp, int *stats, cudaStream_t st)
{
    dim3 grid((nquads + 127) / 128, ndms / group_dms);
    k_quad_patterns<<<grid, 128, 0, st>>>(table, nch_used, ndms, group_dms, nquads, nq_pad, qpat, qwin, qtmp, stats);
    return cudaGetLastError();
}

cudaError_t launch_quad_offsets(const int32_t *qtmp, size_t n, int W, int32_t *qoff, cudaStream_t st)
{
    k_quad_offsets<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(qtmp, n, W, qoff);
    return cudaGetLastError();
}

QuadGeometry quad_geometry(int span, int dmax, int maxcnt, int group_dms, int nquads, int out_words, int qs)
{
    QuadGeometry G;
    G.M = out_words;
    G.W = ((span + 32 * out_words) + 3) & ~3;
    G.raww = ((((15 + G.W + dmax + 3) >> 2) + 2) + 3) & ~3;
    G.qs = qs;
    G.npool = qs * (maxcnt > 0 ? maxcnt : 1);
    G.nq_pad = (nquads + 3) & ~3;
    G.smem_bytes = 4 * quad_smem_words(qs, group_dms, G.raww, G.nq_pad, G.npool, G.W);
    return G;
}

cudaError_t launch_ddtr_quad(const DdtrLaunch &p, const QuadLaunch &q, cudaStream_t st)
{
    if ((p.group_dms % QDMW) || p.group_dms > 64 || q.qs < 1 || q.qs > 8)
        return cudaErrorInvalidValue;
    const size_t smem = 4 * quad_smem_words(q.qs, p.group_dms, q.raww, q.nq_pad, q.npool, q.W);
    const int threads = 32 * (p.group_dms / QDMW);
    const long long tile = 32LL * q.M;
    dim3 grid(p.ndms / p.group_dms, static_cast<unsigned>((p.tp + tile - 1) / tile));
    cudaError_t e;
    switch (q.M) {
    case 8:
        e = cudaFuncSetAttribute(k_ddtr_quad<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess)
            return e;
        k_ddtr_quad<8><<<grid, threads, smem, st>>>(p, q);
        break;
    case 16:
        e = cudaFuncSetAttribute(k_ddtr_quad<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess)
            return e;
        k_ddtr_quad<16><<<grid, threads, smem, st>>>(p, q);
        break;
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

} // namespace aab200
