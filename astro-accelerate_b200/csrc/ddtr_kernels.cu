// ddtr_kernels.cu -- sm_100a kernels of the B200 brute-force dedispersion path.
//
// Replaces, for the drop-in seam of AstroAccelerate v1.3.1:
//   corner_turn_SM_inplace   src/aa_corner_turn.cpp:118-121
//   bin_gpu                  src/aa_bin_gpu.cpp:8-44
//   dedisperse() + kernels   src/aa_dedisperse.cpp:5-163,
//                            src/aa_device_dedispersion_kernel.cu:16-477
//
// Design (B200-first, not a translation):
//  * The input is narrowed to one byte per sample for nbits <= 8 while it is
//    corner-turned, halving every later HBM pass.
//  * Every delay the reference computes inside its kernels (two-level
//    truncated delay of the shared kernels, including the per-thread-class
//    rounding of shift_one*dm_shifts[c]+findex, or the single delay of the
//    cache kernel) is evaluated once per range with explicit IEEE intrinsics
//    into a table [c][dm].  The table stores the smallest delay over the
//    reference's thread classes plus a bit mask of the classes that read one
//    sample later, so the hot loop needs one delay per (channel, DM) and a
//    warp-uniform branch for the rare classes that differ.
//  * The hot kernel stages channel rows of a (DM group x time tile) window
//    into shared memory with cp.async, expands each row into four byte-phase
//    copies so that every warp-uniform delay becomes an aligned 32-bit load,
//    and accumulates two 16-bit lanes per 32-bit add (flushed to 32-bit
//    accumulators every 256 channels).  Lanes of a warp cover consecutive time
//    words of one DM trial, so delays, class exceptions and window checks are
//    warp-uniform.
#include "ddtr_kernels.cuh"
#include "device_util.cuh"

#include <algorithm>
#include <cstdio>

namespace aab200 {

namespace {

using namespace dev;

constexpr int CS = 16;      // channels per shared-memory stage
constexpr int NSTAGE = 3;   // depth of the staging ring
constexpr int DMW = 4;      // DM trials per warp
constexpr int MAX_NCH = 16384;


__device__ __forceinline__ int findex_of(int kind, int tx)
{
    return kind == KIND_SHARED8 ? 2 * tx + 1 : (kind == KIND_SHARED16 ? 2 * tx : 4 * tx + 3);
}

// ---------------------------------------------------------------------------
// Delay table.  One thread per (channel, DM trial).
//   shared kernels: src/aa_device_dedispersion_kernel.cu:196-197 (shift_two,
//   shift_one), :206 (per-block base), :211 (per-thread shift); cache kernel
//   :430 and :440.  fma_mode selects the fused or unfused evaluation of each
//   contractible expression.
// ---------------------------------------------------------------------------
__global__ void k_delay_table(const float *__restrict__ dmshifts, int nchans, int ndms, int kind,
                              int fma_mode, float mstartdm, float mdmstep,
                              int32_t *__restrict__ table, int *__restrict__ err)
{
    const int dm = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (dm >= ndms || c >= nchans)
        return;
    const float dms = dmshifts[c];
    int dmin, mask = 0;
    bool bad = false;
    if (kind == KIND_CACHE) {
        const float dmf = __uint2float_rn(static_cast<unsigned>(dm));
        const float sh = (fma_mode & FMA_CACHE) ? __fmaf_rn(dmf, mdmstep, mstartdm)
                                                : __fadd_rn(mstartdm, __fmul_rn(dmf, mdmstep));
        dmin = __float2int_rz(__fmul_rn(dms, sh));
    } else {
        const float two = __fmul_rn(__int2float_rz(dm >> 6), 64.0f);
        const float shift_two = (fma_mode & FMA_TWO) ? __fmaf_rn(two, mdmstep, mstartdm)
                                                     : __fadd_rn(mstartdm, __fmul_rn(two, mdmstep));
        const float shift_one = __fmul_rn(__int2float_rz(dm & 63), mdmstep);
        const int base = __float2int_rz(__fmul_rn(dms, shift_two));
        int d[8];
#pragma unroll
        for (int tx = 0; tx < 8; ++tx) {
            const int f = findex_of(kind, tx);
            const float ff = static_cast<float>(f);
            const float s = (fma_mode & FMA_ONE) ? __fmaf_rn(shift_one, dms, ff)
                                                 : __fadd_rn(__fmul_rn(shift_one, dms), ff);
            d[tx] = base + __float2int_rz(s) - f;
        }
        dmin = d[0];
#pragma unroll
        for (int tx = 1; tx < 8; ++tx)
            dmin = min(dmin, d[tx]);
#pragma unroll
        for (int tx = 0; tx < 8; ++tx) {
            if (d[tx] == dmin + 1)
                mask |= 1 << tx;
            else if (d[tx] != dmin)
                bad = true;
        }
    }
    if (dmin < 0 || dmin >= (1 << 24) - 2)
        bad = true;
    if (bad) {
        atomicOr(err, DERR_DELAY_RANGE);
        dmin = 0;
        mask = 0;
    }
    table[static_cast<size_t>(c) * ndms + dm] = dmin | (mask << 24);
}

// Per (DM group, channel): smallest base delay (window start) and the largest
// span (max delay incl. class step minus window start) over all groups.
__global__ void k_group_windows(const int32_t *__restrict__ table, int nchans, int nch_pad, int ndms,
                                int group_dms, int32_t *__restrict__ wmin, int *__restrict__ span_max,
                                int *__restrict__ delay_max)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int g = blockIdx.y;
    if (c >= nch_pad)
        return;
    if (c >= nchans) {
        wmin[static_cast<size_t>(g) * nch_pad + c] = 0;
        return;
    }
    const int32_t *row = table + static_cast<size_t>(c) * ndms + static_cast<size_t>(g) * group_dms;
    int lo = 0x7fffffff, hi = 0;
    for (int j = 0; j < group_dms; ++j) {
        const int e = row[j];
        const int d = e & 0xFFFFFF;
        lo = min(lo, d);
        hi = max(hi, d + ((static_cast<unsigned>(e) >> 24) ? 1 : 0));
    }
    wmin[static_cast<size_t>(g) * nch_pad + c] = lo;
    atomicMax(span_max, hi - lo);
    atomicMax(delay_max, hi);
}

// Word offset of every (c, dm) inside the staged four-phase window, or -1 for
// entries that need the per-class path.
__global__ void k_offset_table(const int32_t *__restrict__ table, const int32_t *__restrict__ wmin,
                               int nchans, int nch_pad, int ndms, int group_dms, int rw, int span,
                               int32_t *__restrict__ offtab)
{
    const int dm = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (dm >= ndms || c >= nchans)
        return;
    const size_t i = static_cast<size_t>(c) * ndms + dm;
    const int e = table[i];
    const int o = (e & 0xFFFFFF) - wmin[static_cast<size_t>(dm / group_dms) * nch_pad + c];
    const bool fast = ((static_cast<unsigned>(e) >> 24) == 0u) && o >= 0 && o <= span;
    offtab[i] = fast ? ((o & 3) * rw + (o >> 2)) : -1;
}

// ---------------------------------------------------------------------------
// Corner turn [t][c] uint16 -> [c][stride] (uint8 or uint16), with a range
// check of every sample against the bit depth.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_corner_turn(const uint16_t *__restrict__ in, T *__restrict__ out,
                                                     int nchans, long long nsamp, long long stride,
                                                     int max_value, int *__restrict__ err)
{
    __shared__ uint16_t tile[64][65];
    const long long t0 = static_cast<long long>(blockIdx.x) * 64;
    const int c0 = blockIdx.y * 64;
    const int tx = threadIdx.x & 63, ty = threadIdx.x >> 6;
    bool over = false;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int tt = ty + 4 * i;
        const long long t = t0 + tt;
        const int c = c0 + tx;
        uint16_t v = 0;
        if (t < nsamp && c < nchans) {
            v = in[t * nchans + c];
            over |= (v > max_value);
        }
        tile[tt][tx] = v;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int cc = ty + 4 * i;
        const int c = c0 + cc;
        const long long t = t0 + tx;
        if (t < nsamp && c < nchans)
            out[static_cast<long long>(c) * stride + t] = static_cast<T>(tile[tx][cc]);
    }
    if (over)
        atomicOr(err, DERR_INPUT_RANGE);
}

// Sample c of one stored SIGPROC record: 4-bit high nibble first, 2-bit most
// significant pair first, 1-bit least significant bit first.
template <int NBITS>
__device__ __forceinline__ uint16_t packed_sample(const uint8_t *__restrict__ rec, int c)
{
    if constexpr (NBITS == 16) {
        return reinterpret_cast<const uint16_t *>(rec)[c];
    } else if constexpr (NBITS == 8) {
        return rec[c];
    } else if constexpr (NBITS == 4) {
        const unsigned b = rec[c >> 1];
        return static_cast<uint16_t>((c & 1) ? (b & 15u) : (b >> 4));
    } else if constexpr (NBITS == 2) {
        const unsigned b = rec[c >> 2];
        return static_cast<uint16_t>((b >> (6 - 2 * (c & 3))) & 3u);
    } else {
        const unsigned b = rec[c >> 3];
        return static_cast<uint16_t>((b >> (c & 7)) & 1u);
    }
}

// Unpack + corner turn in one pass: the H2D copy carries the stored bytes
// (1/2, 1/4, 1/8 or 1/16 of the unsigned-short input) and the transpose
// tile is filled from them.
template <int NBITS, typename T>
__global__ void __launch_bounds__(256) k_corner_turn_packed(const uint8_t *__restrict__ in, T *__restrict__ out,
                                                            int nchans, long long nsamp, long long stride)
{
    __shared__ uint16_t tile[64][65];
    const long long t0 = static_cast<long long>(blockIdx.x) * 64;
    const int c0 = blockIdx.y * 64;
    const int tx = threadIdx.x & 63, ty = threadIdx.x >> 6;
    const long long rec = static_cast<long long>(nchans) * NBITS / 8;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int tt = ty + 4 * i;
        const long long t = t0 + tt;
        const int c = c0 + tx;
        tile[tt][tx] = (t < nsamp && c < nchans) ? packed_sample<NBITS>(in + t * rec, c) : uint16_t(0);
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int cc = ty + 4 * i;
        const int c = c0 + cc;
        const long long t = t0 + tx;
        if (t < nsamp && c < nchans)
            out[static_cast<long long>(c) * stride + t] = static_cast<T>(tile[tx][cc]);
    }
}

// ---------------------------------------------------------------------------
// Reference x2 binning as it acts on the flat buffer (bin + swap,
// src/aa_device_binning_kernel.cu:33-45, src/aa_device_corner_turn_kernel.cu:91-98):
// (a+b)/2.0f truncated back to the integer type is (a+b)>>1.
// When nchans and nsamp are multiples of 32 the reference's grids cover the
// whole buffer: dst[0, nchans*nsamp/2) = binned, dst[.., nchans*nsamp) = 0,
// and rows of the binned output start on 8-element boundaries, so each thread
// writes 8 elements of one row.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_bin_flat(const T *__restrict__ src, T *__restrict__ dst, long long nchans,
                           long long nsamp)
{
    const long long half = nsamp / 2;
    const long long nout = nchans * half;
    const long long ntot = nchans * nsamp;
    const long long i0 = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) * 8;
    if (i0 >= ntot)
        return;
    T v[8];
    if (i0 < nout) {
        const long long c = i0 / half;
        const long long t = i0 - c * half;
        const T *s = src + c * nsamp + 2 * t;
#pragma unroll
        for (int k = 0; k < 8; ++k)
            v[k] = static_cast<T>((static_cast<unsigned>(s[2 * k]) + static_cast<unsigned>(s[2 * k + 1])) >> 1);
    } else {
#pragma unroll
        for (int k = 0; k < 8; ++k)
            v[k] = 0;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k)
        dst[i0 + k] = v[k];
}

// The general case, one element per thread.  The reference's bin kernel runs
// on a grid of 32-channel x 8-sample blocks, (nsamp+1)/16 blocks in time and
// nchans/32 in frequency (src/aa_bin_gpu.cpp:10-14), so it bins channels
// c < 32*floor(nchans/32) and output samples t < 8*floor((nsamp+1)/16) into a
// zeroed float buffer; its swap kernel runs on 32 x 8 blocks
// (src/aa_bin_gpu.cpp:25-28) and copies that buffer back, in place, only for
// flat positions c*nsamp + t with c < 8*floor(nchans/8) and
// t < 32*floor(nsamp/32).  Positions the swap does not reach keep the
// unbinned input.  nsamp must be even (the runner's lengths always are).
template <typename T>
__global__ void k_bin_flat_general(const T *__restrict__ src, T *__restrict__ dst, long long nchans,
                                   long long nsamp)
{
    const long long n = nchans * nsamp;
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const long long half = nsamp / 2;
    const long long c = i / nsamp;
    const long long t = i - c * nsamp;
    T v;
    if (c < 8 * (nchans / 8) && t < 32 * (nsamp / 32)) {
        const long long c2 = i / half;
        const long long t2 = i - c2 * half;
        v = 0;
        if (c2 < 32 * (nchans / 32) && t2 < 8 * ((nsamp + 1) / 16)) {
            const long long s0 = c2 * nsamp + 2 * t2;
            if (s0 + 1 < n)
                v = static_cast<T>((static_cast<unsigned>(src[s0]) + static_cast<unsigned>(src[s0 + 1])) >> 1);
        }
    } else {
        v = src[i];
    }
    dst[i] = v;
}

// ---------------------------------------------------------------------------
// Hot kernel, one-byte samples, exact integer sums.
//   grid  = (ndms / group_dms, ceil(tp / (128*K))): the DM groups of one time
//           tile are adjacent in launch order, so the tile's input rows are
//           fetched from HBM once and served from L2 to the other groups.
//   block = 32 * group_dms / 4; lane l of warp w accumulates DM trial w*4+j of
//           the group at time words l + 32k, i.e. outputs t0+128k+4l+{0,1,2,3}.
// Pipeline per stage of CS channels:
//   * one warp issues TMA bulk copies (cp.async.bulk) of the CS raw channel
//     windows and of their DM offsets into a ring of NSTAGE slots, completing
//     on an mbarrier per slot;
//   * all threads wait on the mbarrier (bounded: a copy that never lands sets
//     DERR_TIMEOUT and the thread stops accumulating), expand the rows of the
//     next stage into four byte-phase copies (double buffered), accumulate
//     the current stage, and meet at one barrier.
// Shared memory is addressed in 32-bit words from one extern array.
// ---------------------------------------------------------------------------
struct U8Smem {
    int rw;      // words per phase row (multiple of 4)
    int raww;    // words per staged raw row (multiple of 4)
    int nch_pad; // channels rounded up to 4
    int o_ent, o_wtab, o_bar, o_wrow, o_ph; // word offsets
    size_t total;                           // bytes
};

__host__ __device__ inline U8Smem u8_layout(int span, int group_dms, int tile_words, int nchans)
{
    U8Smem L;
    L.rw = (((span >> 2) + 32 * tile_words + 1) + 3) & ~3;
    L.raww = (L.rw + 8 + 3) & ~3;
    L.nch_pad = (nchans + 3) & ~3;
    int o = NSTAGE * CS * L.raww;
    L.o_ent = o;
    o += NSTAGE * CS * group_dms;
    L.o_wtab = o;
    o += NSTAGE * CS * 2;
    o = (o + 3) & ~3;
    L.o_bar = o;
    o += 2 * NSTAGE;
    o = (o + 3) & ~3;
    L.o_wrow = o;
    o += L.nch_pad;
    o = (o + 3) & ~3;
    L.o_ph = o;
    o += 2 * CS * 4 * L.rw;
    L.total = static_cast<size_t>(o) * 4;
    return L;
}

template <int K>
__global__ void __launch_bounds__(512, 1) k_ddtr_u8(const DdtrLaunch p, const int32_t *__restrict__ offtab,
                                                    const U8Smem L, const uint32_t one)
{
    extern __shared__ __align__(16) uint32_t sm[];
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int nwarps = blockDim.x >> 5;
    const int GD = p.group_dms;
    const int g = blockIdx.x;
    const int dm0 = g * GD;
    const long long t0 = static_cast<long long>(blockIdx.y) * (128 * K);
    const int RW = L.rw, RAWW = L.raww;
    const unsigned char *in = static_cast<const unsigned char *>(p.in);
    const int nstages = (p.nch_used + CS - 1) / CS;
    const unsigned bar0 = smem_addr(&sm[L.o_bar]);

    // window starts of this DM group for every channel, and the barriers
    for (int q = tid; q < (L.nch_pad >> 2); q += blockDim.x)
        cp_async16(&sm[L.o_wrow + 4 * q], p.wmin + static_cast<size_t>(g) * L.nch_pad + 4 * q);
    cp_async_commit();
    if (tid == 0)
        for (int i = 0; i < NSTAGE; ++i)
            mbar_init(bar0 + 8 * i, 1);
    cp_async_wait<0>();
    mbar_init_fence();
    __syncthreads();

    // warp 0 stages stage s: lane cl copies channel cl's raw window and offsets
    auto issue = [&](int s) {
        if (warp != 0 || s >= nstages)
            return;
        const int slot = s % NSTAGE;
        const int ncl = min(CS, p.nch_used - s * CS);
        const unsigned bar = bar0 + 8 * slot;
        // the slot was last read through the generic proxy; order those reads
        // before the async-proxy writes of the copies
        fence_proxy_async();
        if (lane == 0)
            mbar_expect_tx(bar, static_cast<unsigned>(ncl) * static_cast<unsigned>(RAWW * 4 + GD * 4));
        __syncwarp();
        if (lane < ncl) {
            const int c = s * CS + lane;
            const int w0 = static_cast<int>(sm[L.o_wrow + c]);
            const unsigned char *src = in + static_cast<long long>(c) * p.stride + t0 + w0;
            const uintptr_t a = reinterpret_cast<uintptr_t>(src);
            sm[L.o_wtab + (slot * CS + lane) * 2 + 0] = static_cast<uint32_t>(w0);
            sm[L.o_wtab + (slot * CS + lane) * 2 + 1] = static_cast<uint32_t>(a & 15);
            tma_load_1d(smem_addr(&sm[(slot * CS + lane) * RAWW]),
                        reinterpret_cast<const void *>(a & ~static_cast<uintptr_t>(15)),
                        static_cast<unsigned>(RAWW * 4), bar);
            tma_load_1d(smem_addr(&sm[L.o_ent + (slot * CS + lane) * GD]),
                        offtab + static_cast<size_t>(c) * p.ndms + dm0, static_cast<unsigned>(GD * 4), bar);
        }
    };

    bool ok = true;
    // expand stage s (raw slot) into phase buffer b: phase q word j = raw bytes
    // [sh + q + 4j, +4); each warp takes channels, lanes take (phase, 4 words)
    auto build = [&](int s, int b) {
        const int slot = s % NSTAGE;
        if (!mbar_wait_bounded(bar0 + 8 * slot, static_cast<unsigned>((s / NSTAGE) & 1))) {
            if (ok)
                atomicOr(p.err, DERR_TIMEOUT);
            ok = false;
        }
        const int ncl = min(CS, p.nch_used - s * CS);
        const int n4 = RW >> 2;
        for (int cl = warp; cl < ncl; cl += nwarps) {
            const int sh = static_cast<int>(sm[L.o_wtab + (slot * CS + cl) * 2 + 1]) & 15;
            const int rbase = (slot * CS + cl) * RAWW;
            const int pbase = L.o_ph + (b * CS + cl) * 4 * RW;
            for (int idx = lane; idx < 4 * n4; idx += 32) {
                const int q = idx & 3, j4 = idx >> 2;
                const int a = sh + q;
                const int rb = rbase + 4 * j4 + (a >> 2);
                const unsigned amt = 8u * static_cast<unsigned>(a & 3);
                const uint32_t r0 = sm[rb], r1 = sm[rb + 1], r2 = sm[rb + 2], r3 = sm[rb + 3], r4 = sm[rb + 4];
                uint4 v;
                v.x = __funnelshift_r(r0, r1, amt);
                v.y = __funnelshift_r(r1, r2, amt);
                v.z = __funnelshift_r(r2, r3, amt);
                v.w = __funnelshift_r(r3, r4, amt);
                *reinterpret_cast<uint4 *>(&sm[pbase + q * RW + 4 * j4]) = v;
            }
        }
    };

    uint32_t a16[DMW][K][2];
    uint32_t a32[DMW][K][4];
#pragma unroll
    for (int j = 0; j < DMW; ++j)
#pragma unroll
        for (int k = 0; k < K; ++k) {
            a16[j][k][0] = a16[j][k][1] = 0u;
            a32[j][k][0] = a32[j][k][1] = a32[j][k][2] = a32[j][k][3] = 0u;
        }

#pragma unroll
    for (int s = 0; s < NSTAGE - 1; ++s)
        issue(s);
    __syncthreads(); // window shifts written by warp 0 become visible
    build(0, 0);
    __syncthreads();
    issue(NSTAGE - 1);

    int since_flush = 0;
    for (int s = 0; s < nstages; ++s) {
        if (s + 1 < nstages)
            build(s + 1, (s + 1) & 1);
        const int slot = s % NSTAGE;
        const int ncl = min(CS, p.nch_used - s * CS);
        const int ebase = L.o_ent + slot * CS * GD + warp * DMW;
        const int phb = L.o_ph + (s & 1) * CS * 4 * RW + lane;
        if (ok) {
            for (int cl = 0; cl < ncl; ++cl) {
                const int4 e4 = *reinterpret_cast<const int4 *>(&sm[ebase + cl * GD]);
                const int prow = phb + cl * 4 * RW;
                if ((e4.x | e4.y | e4.z | e4.w) >= 0) {
                    const int ej[DMW] = {e4.x, e4.y, e4.z, e4.w};
#pragma unroll
                    for (int h = 0; h < DMW; h += 2) {
                        uint32_t w[2][K];
#pragma unroll
                        for (int j = 0; j < 2; ++j)
#pragma unroll
                            for (int k = 0; k < K; ++k)
                                w[j][k] = sm[prow + ej[h + j] + 32 * k];
#pragma unroll
                        for (int j = 0; j < 2; ++j)
#pragma unroll
                            for (int k = 0; k < K; ++k) {
                                a16[h + j][k][0] = (w[j][k] & 0x00FF00FFu) * one + a16[h + j][k][0];
                                a16[h + j][k][1] = __byte_perm(w[j][k], 0u, 0x4341) * one + a16[h + j][k][1];
                            }
                    }
                } else {
                    // per-class path (rare): some thread classes read one sample
                    // later, or a delay falls outside the window
                    const int c = s * CS + cl;
                    const int wmin = static_cast<int>(sm[L.o_wtab + (slot * CS + cl) * 2 + 0]);
#pragma unroll
                    for (int j = 0; j < DMW; ++j) {
                        const int dm = dm0 + warp * DMW + j;
                        const int ee = p.table[static_cast<size_t>(c) * p.ndms + dm];
                        const int o = (ee & 0xFFFFFF) - wmin;
                        const unsigned mask = static_cast<unsigned>(ee) >> 24;
                        int dA, dB;
                        if (p.kind == KIND_SHARED4) {
                            dA = dB = (mask >> (lane & 7)) & 1;
                        } else {
                            dA = (mask >> (2 * (lane & 3))) & 1;
                            dB = (mask >> (2 * (lane & 3) + 1)) & 1;
                        }
                        const int oA = o + dA, oB = o + dB;
                        if (oA < 0 || oB < 0 || oA > p.span || oB > p.span) {
                            if (lane == 0)
                                atomicOr(p.err, DERR_WINDOW);
                            continue;
                        }
                        const int pa = prow - lane + (oA & 3) * RW + (oA >> 2) + lane;
                        const int pb = prow - lane + (oB & 3) * RW + (oB >> 2) + lane;
#pragma unroll
                        for (int k = 0; k < K; ++k) {
                            const uint32_t wa = sm[pa + 32 * k], wb = sm[pb + 32 * k];
                            a16[j][k][0] += (wa & 0x000000FFu) | (wb & 0x00FF0000u);
                            a16[j][k][1] += ((wa >> 8) & 0x000000FFu) | ((wb >> 8) & 0x00FF0000u);
                        }
                    }
                }
            }
        }
        since_flush += ncl;
        if (since_flush > 256 - CS) {
#pragma unroll
            for (int j = 0; j < DMW; ++j)
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    a32[j][k][0] += a16[j][k][0] & 0xFFFFu;
                    a32[j][k][2] += a16[j][k][0] >> 16;
                    a32[j][k][1] += a16[j][k][1] & 0xFFFFu;
                    a32[j][k][3] += a16[j][k][1] >> 16;
                    a16[j][k][0] = a16[j][k][1] = 0u;
                }
            since_flush = 0;
        }
        __syncthreads();
        issue(s + NSTAGE);
    }
#pragma unroll
    for (int j = 0; j < DMW; ++j)
#pragma unroll
        for (int k = 0; k < K; ++k) {
            a32[j][k][0] += a16[j][k][0] & 0xFFFFu;
            a32[j][k][2] += a16[j][k][0] >> 16;
            a32[j][k][1] += a16[j][k][1] & 0xFFFFu;
            a32[j][k][3] += a16[j][k][1] >> 16;
        }
    if (!ok)
        return;

    // epilogue: (float)S / nchans / bin, the reference's expression
#pragma unroll
    for (int j = 0; j < DMW; ++j) {
        const int dm = dm0 + warp * DMW + j;
        if (dm >= p.ndms)
            continue;
        float *orow = p.out + static_cast<long long>(dm) * p.out_pitch;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const long long t = t0 + 128 * k + 4 * lane;
            if (t < p.tp) {
                float4 v;
                if (p.divide_by_bin) {
                    v.x = static_cast<float>(static_cast<int>(a32[j][k][0])) / p.nchans_f / p.bin_f;
                    v.y = static_cast<float>(static_cast<int>(a32[j][k][1])) / p.nchans_f / p.bin_f;
                    v.z = static_cast<float>(static_cast<int>(a32[j][k][2])) / p.nchans_f / p.bin_f;
                    v.w = static_cast<float>(static_cast<int>(a32[j][k][3])) / p.nchans_f / p.bin_f;
                } else {
                    v.x = static_cast<float>(static_cast<int>(a32[j][k][0])) / p.nchans_f;
                    v.y = static_cast<float>(static_cast<int>(a32[j][k][1])) / p.nchans_f;
                    v.z = static_cast<float>(static_cast<int>(a32[j][k][2])) / p.nchans_f;
                    v.w = static_cast<float>(static_cast<int>(a32[j][k][3])) / p.nchans_f;
                }
                *reinterpret_cast<float4 *>(orow + t) = v;
            }
        }
    }
}
// ---------------------------------------------------------------------------
// Two-byte samples (16/32-bit data): fp32 sums in ascending channel order,
// as shared_dedisperse_kernel_16 and the cache kernel accumulate them
// (src/aa_device_dedispersion_kernel.cu:344-350, :433-443).  One thread per
// four consecutive outputs of one DM trial.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_ddtr_u16(const DdtrLaunch p)
{
    const int dm = blockIdx.y;
    const long long t = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) * 4;
    if (t >= p.tp || dm >= p.ndms)
        return;
    const uint16_t *in = static_cast<const uint16_t *>(p.in);
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    int cls[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int tt = static_cast<int>((t + i) & 31);
        cls[i] = (p.kind == KIND_SHARED4) ? (tt >> 2) : ((tt & 15) >> 1);
    }
    for (int c = 0; c < p.nch_used; ++c) {
        const int e = __ldg(p.table + static_cast<size_t>(c) * p.ndms + dm);
        const int d = e & 0xFFFFFF;
        const unsigned mask = static_cast<unsigned>(e) >> 24;
        const uint16_t *row = in + static_cast<long long>(c) * p.stride + t + d;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int extra = (mask >> cls[i]) & 1;
            acc[i] = __fadd_rn(acc[i], static_cast<float>(__ldg(row + i + extra)));
        }
    }
    float *orow = p.out + static_cast<long long>(dm) * p.out_pitch + t;
#pragma unroll
    for (int i = 0; i < 4; ++i)
        orow[i] = p.divide_by_bin ? (acc[i] / p.nchans_f / p.bin_f) : (acc[i] / p.nchans_f);
}

} // namespace

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
cudaError_t launch_delay_table(const float *dmshifts, int nchans, int ndms, int kind, int fma_mode,
                               float mstartdm, float mdmstep, int32_t *table, int *err, cudaStream_t st)
{
    dim3 grid((ndms + 127) / 128, nchans);
    k_delay_table<<<grid, 128, 0, st>>>(dmshifts, nchans, ndms, kind, fma_mode, mstartdm, mdmstep,
                                        table, err);
    return cudaGetLastError();
}

cudaError_t launch_group_windows(const int32_t *table, int nchans, int ndms, int group_dms,
                                 int32_t *wmin, int *span_max, int *delay_max, cudaStream_t st)
{
    const int nch_pad = (nchans + 3) & ~3;
    dim3 grid((nch_pad + 127) / 128, ndms / group_dms);
    k_group_windows<<<grid, 128, 0, st>>>(table, nchans, nch_pad, ndms, group_dms, wmin, span_max,
                                          delay_max);
    return cudaGetLastError();
}

cudaError_t launch_offset_table(const int32_t *table, const int32_t *wmin, int nchans, int ndms,
                                int group_dms, int rw, int span, int32_t *offtab, cudaStream_t st)
{
    const int nch_pad = (nchans + 3) & ~3;
    dim3 grid((ndms + 127) / 128, nchans);
    k_offset_table<<<grid, 128, 0, st>>>(table, wmin, nchans, nch_pad, ndms, group_dms, rw, span, offtab);
    return cudaGetLastError();
}

cudaError_t launch_corner_turn(const uint16_t *in_tc, void *out_ct, int elem_bytes, int nchans,
                               long long nsamp, long long out_stride, int max_value, int *err,
                               cudaStream_t st)
{
    dim3 grid(static_cast<unsigned>((nsamp + 63) / 64), (nchans + 63) / 64);
    if (elem_bytes == 1)
        k_corner_turn<uint8_t><<<grid, 256, 0, st>>>(in_tc, static_cast<uint8_t *>(out_ct), nchans, nsamp,
                                                     out_stride, max_value, err);
    else
        k_corner_turn<uint16_t><<<grid, 256, 0, st>>>(in_tc, static_cast<uint16_t *>(out_ct), nchans, nsamp,
                                                      out_stride, max_value, err);
    return cudaGetLastError();
}

cudaError_t launch_corner_turn_packed(const uint8_t *in_rec, int nbits, void *out_ct, int nchans, long long nsamp,
                                      long long out_stride, cudaStream_t st)
{
    if (nchans < 1 || nsamp < 0 || (static_cast<long long>(nchans) * nbits) % 8)
        return cudaErrorInvalidValue;
    if (nbits == 16 && (reinterpret_cast<uintptr_t>(in_rec) & 1))
        return cudaErrorInvalidValue;
    if (nsamp == 0)
        return cudaSuccess;
    dim3 grid(static_cast<unsigned>((nsamp + 63) / 64), (nchans + 63) / 64);
    uint8_t *o8 = static_cast<uint8_t *>(out_ct);
    switch (nbits) {
    case 1:
        k_corner_turn_packed<1, uint8_t><<<grid, 256, 0, st>>>(in_rec, o8, nchans, nsamp, out_stride);
        break;
    case 2:
        k_corner_turn_packed<2, uint8_t><<<grid, 256, 0, st>>>(in_rec, o8, nchans, nsamp, out_stride);
        break;
    case 4:
        k_corner_turn_packed<4, uint8_t><<<grid, 256, 0, st>>>(in_rec, o8, nchans, nsamp, out_stride);
        break;
    case 8:
        k_corner_turn_packed<8, uint8_t><<<grid, 256, 0, st>>>(in_rec, o8, nchans, nsamp, out_stride);
        break;
    case 16:
        k_corner_turn_packed<16, uint16_t><<<grid, 256, 0, st>>>(in_rec, static_cast<uint16_t *>(out_ct), nchans,
                                                                  nsamp, out_stride);
        break;
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_bin_flat(const void *src, void *dst, int elem_bytes, int nchans, long long nsamp,
                            cudaStream_t st)
{
    const long long ntot = static_cast<long long>(nchans) * nsamp;
    if (nsamp < 2 || (nsamp & 1) || nchans < 1)
        return cudaErrorInvalidValue;
    if ((nsamp % 32) || (nchans % 32)) {
        const unsigned b = static_cast<unsigned>((ntot + 255) / 256);
        if (elem_bytes == 1)
            k_bin_flat_general<uint8_t><<<b, 256, 0, st>>>(static_cast<const uint8_t *>(src),
                                                            static_cast<uint8_t *>(dst), nchans, nsamp);
        else
            k_bin_flat_general<uint16_t><<<b, 256, 0, st>>>(static_cast<const uint16_t *>(src),
                                                             static_cast<uint16_t *>(dst), nchans, nsamp);
        return cudaGetLastError();
    }
    const long long nthreads = (ntot + 7) / 8;
    const unsigned blocks = static_cast<unsigned>((nthreads + 255) / 256);
    if (elem_bytes == 1)
        k_bin_flat<uint8_t><<<blocks, 256, 0, st>>>(static_cast<const uint8_t *>(src), static_cast<uint8_t *>(dst),
                                                     nchans, nsamp);
    else
        k_bin_flat<uint16_t><<<blocks, 256, 0, st>>>(static_cast<const uint16_t *>(src),
                                                      static_cast<uint16_t *>(dst), nchans, nsamp);
    return cudaGetLastError();
}

size_t ddtr_u8_smem_bytes(int span, int group_dms, int tile_words, int nchans)
{
    return u8_layout(span, group_dms, tile_words, nchans).total;
}

int ddtr_u8_rw(int span, int tile_words)
{
    return (((span >> 2) + 32 * tile_words + 1) + 3) & ~3;
}

cudaError_t launch_ddtr_u8(const DdtrLaunch &p, const int32_t *offtab, int tile_words, cudaStream_t st)
{
    if (p.nchans > MAX_NCH || (p.group_dms & 3) || p.group_dms > 64 || p.group_dms < 4)
        return cudaErrorInvalidValue;
    const U8Smem L = u8_layout(p.span, p.group_dms, tile_words, p.nchans);
    const int threads = 32 * (p.group_dms / DMW);
    const long long tile = 128LL * tile_words;
    dim3 grid(p.ndms / p.group_dms, static_cast<unsigned>((p.tp + tile - 1) / tile));
    cudaError_t e;
    switch (tile_words) {
    case 2:
        e = cudaFuncSetAttribute(k_ddtr_u8<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(L.total));
        if (e != cudaSuccess)
            return e;
        k_ddtr_u8<2><<<grid, threads, L.total, st>>>(p, offtab, L, 1u);
        break;
    case 4:
        e = cudaFuncSetAttribute(k_ddtr_u8<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(L.total));
        if (e != cudaSuccess)
            return e;
        k_ddtr_u8<4><<<grid, threads, L.total, st>>>(p, offtab, L, 1u);
        break;
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_ddtr_u16(const DdtrLaunch &p, cudaStream_t st)
{
    dim3 grid(static_cast<unsigned>((p.tp / 4 + 255) / 256), p.ndms);
    k_ddtr_u16<<<grid, 256, 0, st>>>(p);
    return cudaGetLastError();
}

} // namespace aab200
