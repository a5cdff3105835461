// spd.cu -- kernels of the single-pulse detection (see spd.cuh).  Each keeps
// the arithmetic of the reference kernel it corresponds to (cited per
// kernel): the streaming mean/variance updates and pairwise merges in float,
// the merge trees of its thread blocks, the boxcar partial sums exchanged
// between threads through shared memory, the fast divisions, and the
// neighbourhood rules of the peak finder.
#include "spd.cuh"

#include <atomic>
#include <cmath>

namespace aab200 {

namespace {
std::atomic<long long> g_spd_launches{0};
}

long long spd_kernel_launches() { return g_spd_launches.load(); }

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int MSD_BATCH = 8; // rows loaded ahead per thread in the MSD passes

// ---------------------------------------------------------------------------
// Streaming statistics (include/aa_device_MSD_shared_kernel_functions.cuh:13-35)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void st_first(float &M, float &S, float &j, float e)
{
    M = e;
    S = 0;
    j = 1.0f;
}

__device__ __forceinline__ void st_add(float &M, float &S, float &j, float e)
{
    float ftemp;
    j = j + 1.0f;
    M = M + e;
    ftemp = (j * e - M);
    S = S + 1.0f / (j * (j - 1.0f)) * ftemp * ftemp;
}

__device__ __forceinline__ void st_merge(float &AM, float &AS, float &Aj, float BM, float BS, float Bj)
{
    float ftemp;
    ftemp = (Bj / Aj) * AM - BM;
    AS = AS + BS + (Aj / (Bj * (Aj + Bj))) * ftemp * ftemp;
    AM = AM + BM;
    Aj = Aj + Bj;
}

// Block tree over s[3][bd] (M, S, j) down to 32 values, skipping empty ones
// (:36-66); then the warp tree (:120-139).
__device__ __forceinline__ void tree_sm(float &M, float &S, float &j, float *s)
{
    const int t = threadIdx.x, bd = blockDim.x;
    M = s[t];
    S = s[bd + t];
    j = s[2 * bd + t];
    for (int i = (bd >> 1); i > 16; i >>= 1) {
        if (t < i) {
            const float jv = s[2 * bd + i + t];
            if (((int)jv) != 0) {
                if (j == 0) {
                    S = s[bd + i + t];
                    M = s[i + t];
                    j = jv;
                } else {
                    st_merge(M, S, j, s[i + t], s[bd + i + t], jv);
                }
            }
            s[t] = M;
            s[bd + t] = S;
            s[2 * bd + t] = j;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ void tree_warp(float &M, float &S, float &j)
{
    for (int q = 16; q > 0; q >>= 1) {
        const float BM = __shfl_down_sync(FULL, M, q);
        const float BS = __shfl_down_sync(FULL, S, q);
        const float Bj = __shfl_down_sync(FULL, j, q);
        if (Bj > 0) {
            if (j == 0) {
                S = BS;
                M = BM;
                j = Bj;
            } else {
                st_merge(M, S, j, BM, BS, Bj);
            }
        }
    }
}

// with running maxima and minima (:67-119, :140-169; the reference keeps
// the larger of the two minima in the warp tree, reproduced)
__device__ __forceinline__ void tree_sm_max(float &M, float &S, float &j, float &mx, float &mn, float *s)
{
    const int t = threadIdx.x, bd = blockDim.x;
    M = s[t];
    S = s[bd + t];
    j = s[2 * bd + t];
    mx = s[3 * bd + t];
    mn = s[4 * bd + t];
    for (int i = (bd >> 1); i > 16; i >>= 1) {
        if (t < i) {
            const int jv = (int)s[2 * bd + i + t];
            if (jv != 0) {
                if (j == 0) {
                    M = s[i + t];
                    S = s[bd + i + t];
                    mx = s[3 * bd + i + t];
                    mn = s[4 * bd + i + t];
                    j = (float)jv;
                } else {
                    st_merge(M, S, j, s[i + t], s[bd + i + t], (float)jv);
                    mx = fmaxf(mx, s[3 * bd + i + t]);
                    mn = fminf(mn, s[4 * bd + i + t]);
                }
            }
            s[t] = M;
            s[bd + t] = S;
            s[2 * bd + t] = j;
            s[3 * bd + t] = mx;
            s[4 * bd + t] = mn;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ void tree_warp_max(float &M, float &S, float &j, float &mx, float &mn)
{
    for (int q = 16; q > 0; q >>= 1) {
        const float BM = __shfl_down_sync(FULL, M, q);
        const float BS = __shfl_down_sync(FULL, S, q);
        const float Bmx = __shfl_down_sync(FULL, mx, q);
        const float Bmn = __shfl_down_sync(FULL, mn, q);
        const float Bj = __shfl_down_sync(FULL, j, q);
        if (Bj > 0) {
            if (j == 0) {
                S = BS;
                M = BM;
                j = Bj;
                mx = Bmx;
                mn = Bmn;
            } else {
                st_merge(M, S, j, BM, BS, Bj);
                mx = fmaxf(mx, Bmx);
                mn = fmaxf(mn, Bmn);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Partial statistics per block of 512 columns x y_steps rows
// (src/aa_device_MSD_normal_kernel.cu:10-47,
//  src/aa_device_MSD_outlier_rejection_kernel.cu:11-115)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(SPD_NTHREADS) k_msd_partials(const float *__restrict__ in, float *__restrict__ part,
                                                               int y_steps, long long nT, long long offset)
{
    __shared__ float s[3 * SPD_NTHREADS];
    float M = 0, S = 0, j = 0;
    const long long spos = static_cast<long long>(blockIdx.x) * SPD_NTHREADS + threadIdx.x;
    long long g = static_cast<long long>(blockIdx.y) * y_steps * nT + spos;
    if (spos < nT - offset) {
        // loads batched ahead of the (sequential) updates: same order of
        // arithmetic, more loads in flight per thread
        const float *p = in + g;
        st_first(M, S, j, __ldg(p));
        int y = 1;
        for (; y + MSD_BATCH <= y_steps; y += MSD_BATCH) {
            float e[MSD_BATCH];
#pragma unroll
            for (int k = 0; k < MSD_BATCH; ++k)
                e[k] = __ldg(p + static_cast<long long>(y + k) * nT);
#pragma unroll
            for (int k = 0; k < MSD_BATCH; ++k)
                st_add(M, S, j, e[k]);
        }
        for (; y < y_steps; ++y)
            st_add(M, S, j, __ldg(p + static_cast<long long>(y) * nT));
    }
    s[threadIdx.x] = M;
    s[blockDim.x + threadIdx.x] = S;
    s[2 * blockDim.x + threadIdx.x] = j;
    __syncthreads();
    tree_sm(M, S, j, s);
    tree_warp(M, S, j);
    if (threadIdx.x == 0) {
        const long long b = static_cast<long long>(blockIdx.y) * gridDim.x + blockIdx.x;
        part[5 * b] = M;
        part[5 * b + 1] = S;
        part[5 * b + 2] = j;
    }
}

__global__ void __launch_bounds__(SPD_NTHREADS) k_msd_partials_minmax(const float *__restrict__ in,
                                                                      float *__restrict__ part, int y_steps,
                                                                      long long nT, long long offset)
{
    __shared__ float s[5 * SPD_NTHREADS];
    float M = 0, S = 0, j = 0, mx = 0, mn = 0;
    const long long spos = static_cast<long long>(blockIdx.x) * SPD_NTHREADS + threadIdx.x;
    long long g = static_cast<long long>(blockIdx.y) * y_steps * nT + spos;
    if (spos < nT - offset) {
        const float *p = in + g;
        const float e0 = __ldg(p);
        st_first(M, S, j, e0);
        mx = e0;
        mn = e0;
        int y = 1;
        for (; y + MSD_BATCH <= y_steps; y += MSD_BATCH) {
            float e[MSD_BATCH];
#pragma unroll
            for (int k = 0; k < MSD_BATCH; ++k)
                e[k] = __ldg(p + static_cast<long long>(y + k) * nT);
#pragma unroll
            for (int k = 0; k < MSD_BATCH; ++k) {
                mx = fmaxf(mx, e[k]);
                mn = fminf(mn, e[k]);
                st_add(M, S, j, e[k]);
            }
        }
        for (; y < y_steps; ++y) {
            const float e = __ldg(p + static_cast<long long>(y) * nT);
            mx = fmaxf(mx, e);
            mn = fminf(mn, e);
            st_add(M, S, j, e);
        }
    }
    s[threadIdx.x] = M;
    s[blockDim.x + threadIdx.x] = S;
    s[2 * blockDim.x + threadIdx.x] = j;
    s[3 * blockDim.x + threadIdx.x] = mx;
    s[4 * blockDim.x + threadIdx.x] = mn;
    __syncthreads();
    tree_sm_max(M, S, j, mx, mn, s);
    tree_warp_max(M, S, j, mx, mn);
    if (threadIdx.x == 0) {
        const long long b = static_cast<long long>(blockIdx.y) * gridDim.x + blockIdx.x;
        part[5 * b] = M;
        part[5 * b + 1] = S;
        part[5 * b + 2] = j;
        part[5 * b + 3] = mx;
        part[5 * b + 4] = mn;
    }
}

// A block whose previous extremes lie inside the cut keeps its partials.
__global__ void __launch_bounds__(SPD_NTHREADS) k_msd_partials_rejection(const float *__restrict__ in,
                                                                         float *__restrict__ part,
                                                                         const float *__restrict__ msd, int y_steps,
                                                                         long long nT, long long offset, float sigma)
{
    __shared__ float s[5 * SPD_NTHREADS];
    const float limit_down = msd[0] - sigma * msd[1];
    const float limit_up = msd[0] + sigma * msd[1];
    const long long b = static_cast<long long>(blockIdx.y) * gridDim.x + blockIdx.x;
    float mx = part[5 * b + 3];
    float mn = part[5 * b + 4];
    if ((mn > limit_down) && (mx < limit_up))
        return; // the whole block
    float M = 0, S = 0, j = 0;
    mx = 0;
    mn = 0;
    const long long spos = static_cast<long long>(blockIdx.x) * SPD_NTHREADS + threadIdx.x;
    long long g = static_cast<long long>(blockIdx.y) * y_steps * nT + spos;
    if (spos < nT - offset) {
        const float *p = in + g;
        auto take = [&](float e) {
            if ((e > limit_down) && (e < limit_up)) {
                if (j == 0) {
                    st_first(M, S, j, e);
                    mx = e;
                    mn = e;
                } else {
                    st_add(M, S, j, e);
                    mx = fmaxf(mx, e);
                    mn = fminf(mn, e);
                }
            }
        };
        int y = 0;
        for (; y + MSD_BATCH <= y_steps; y += MSD_BATCH) {
            float e[MSD_BATCH];
#pragma unroll
            for (int k = 0; k < MSD_BATCH; ++k)
                e[k] = __ldg(p + static_cast<long long>(y + k) * nT);
#pragma unroll
            for (int k = 0; k < MSD_BATCH; ++k)
                take(e[k]);
        }
        for (; y < y_steps; ++y)
            take(__ldg(p + static_cast<long long>(y) * nT));
    }
    s[threadIdx.x] = M;
    s[blockDim.x + threadIdx.x] = S;
    s[2 * blockDim.x + threadIdx.x] = j;
    s[3 * blockDim.x + threadIdx.x] = mx;
    s[4 * blockDim.x + threadIdx.x] = mn;
    __syncthreads();
    tree_sm_max(M, S, j, mx, mn, s);
    tree_warp_max(M, S, j, mx, mn);
    if (threadIdx.x == 0) {
        part[5 * b] = M;
        part[5 * b + 1] = S;
        part[5 * b + 2] = j;
        part[5 * b + 3] = mx;
        part[5 * b + 4] = mn;
    }
}

// ---------------------------------------------------------------------------
// Merging the partials in one block (src/aa_device_MSD_shared_kernel_functions.cu:7-85
// with include/aa_device_MSD_shared_kernel_functions.cuh:81-240).  "Regular"
// partials are all non-empty and are merged unconditionally; "non-regular"
// ones (after outlier rejection) skip empty partials -- and, below one
// partial per thread, also skip partial 0, as the reference does.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void sum_regular(float &M, float &S, float &j, const float *p, float *s, int size)
{
    const int t = threadIdx.x, bd = blockDim.x;
    int pos = t;
    if (size > bd) {
        M = p[5 * pos];
        S = p[5 * pos + 1];
        j = p[5 * pos + 2];
        pos += bd;
        while (pos < size) {
            st_merge(M, S, j, p[5 * pos], p[5 * pos + 1], p[5 * pos + 2]);
            pos += bd;
        }
        s[t] = M;
        s[bd + t] = S;
        s[2 * bd + t] = j;
        __syncthreads();
        M = s[t];
        S = s[bd + t];
        j = s[2 * bd + t];
        for (int i = (bd >> 1); i > 16; i >>= 1) {
            if (t < i) {
                st_merge(M, S, j, s[i + t], s[bd + i + t], s[2 * bd + i + t]);
                s[t] = M;
                s[bd + t] = S;
                s[2 * bd + t] = j;
            }
            __syncthreads();
        }
        for (int q = 16; q > 0; q >>= 1)
            st_merge(M, S, j, __shfl_down_sync(FULL, M, q), __shfl_down_sync(FULL, S, q),
                     __shfl_down_sync(FULL, j, q));
    } else if (t == 0) {
        M = p[0];
        S = p[1];
        j = p[2];
        for (pos = 1; pos < size; ++pos)
            st_merge(M, S, j, p[5 * pos], p[5 * pos + 1], p[5 * pos + 2]);
    }
}

__device__ __forceinline__ void sum_nonregular(float &M, float &S, float &j, const float *p, float *s, int size)
{
    const int t = threadIdx.x, bd = blockDim.x;
    int pos = t;
    if (size > bd) {
        M = 0;
        S = 0;
        j = 0;
        while (pos < size) {
            const float jv = p[5 * pos + 2];
            if (((int)jv) > 0) {
                if ((int)j == 0) {
                    M = p[5 * pos];
                    S = p[5 * pos + 1];
                    j = jv;
                } else {
                    st_merge(M, S, j, p[5 * pos], p[5 * pos + 1], jv);
                }
            }
            pos += bd;
        }
        s[t] = M;
        s[bd + t] = S;
        s[2 * bd + t] = j;
        __syncthreads();
        tree_sm(M, S, j, s);
        tree_warp(M, S, j);
    } else if (t == 0) {
        M = 0;
        S = 0;
        j = 0;
        for (pos = 1; pos < size; ++pos) {
            const float jv = p[5 * pos + 2];
            if (((int)jv) != 0) {
                if ((int)j == 0) {
                    M = p[5 * pos];
                    S = p[5 * pos + 1];
                    j = jv;
                } else {
                    st_merge(M, S, j, p[5 * pos], p[5 * pos + 1], jv);
                }
            }
        }
    }
}

// d_msd = (M / j, sqrt(S / j), j); with d_pp, earlier (M, S, j) are merged
// in first and the merged totals kept in d_pp.
__global__ void k_msd_final(const float *__restrict__ p, float *__restrict__ msd, float *pp, int size, int regular)
{
    __shared__ float s[3 * 32 * 32];
    float M, S, j;
    if (regular)
        sum_regular(M, S, j, p, s, size);
    else
        sum_nonregular(M, S, j, p, s, size);
    if (pp && pp[2] > 0)
        st_merge(M, S, j, pp[0], pp[1], pp[2]);
    if (threadIdx.x == 0) {
        msd[0] = M / j;
        msd[1] = sqrt(S / j);
        msd[2] = j;
        if (pp) {
            pp[0] = M;
            pp[1] = S;
            pp[2] = j;
        }
    }
}

// src/aa_device_binning_kernel.cu:48-64 (rows 0 .. 2*(nDMs/2)-1)
__global__ void k_dit_pairs(const float *__restrict__ in, float *__restrict__ out, int rows, long long nT, long long dts)
{
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (y >= rows || 2 * i + 1 >= nT)
        return;
    out[y * dts + i] = in[y * nT + 2 * i] + in[y * nT + 2 * i + 1];
}

// The same sums for even rows on an 8-byte aligned input: one float2 load per pair.
__global__ void k_dit_pairs2(const float2 *__restrict__ in, float *__restrict__ out, int rows, long long dts)
{
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (y >= rows || i >= dts)
        return;
    const float2 v = __ldg(in + y * dts + i);
    out[y * dts + i] = v.x + v.y;
}

// src/aa_device_single_FIR_kernel.cu:95-107
__global__ void k_fir_rows(const float *__restrict__ in, float *__restrict__ out, int nTaps, long long nT)
{
    const long long x = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long long y = blockIdx.y;
    if (x < nT - nTaps + 1) {
        float f = 0;
        for (int t = 0; t < nTaps; ++t)
            f += __ldg(in + y * nT + x + t);
        out[y * nT + x] = f;
    }
}

// src/aa_device_MSD_shared_kernel_functions.cu:86-120
__global__ void k_msd_interpolate(const float *__restrict__ dit, float *__restrict__ out, const int *__restrict__ dw,
                                  int n_dit, const int *__restrict__ widths, int max_width_performed)
{
    const int tid = threadIdx.x;
    if (widths[tid] <= max_width_performed) {
        const int desired = widths[tid];
        const int position = (int)floorf(log2f((float)desired));
        const float width1 = dw[position];
        const float mean1 = dit[position * 3];
        const float sd1 = dit[position * 3 + 1];
        if (position == n_dit - 1 && width1 == (int)desired) {
            out[tid * 2] = mean1;
            out[tid * 2 + 1] = sd1;
        } else {
            const float width2 = dw[position + 1];
            const float distance_in_width = width2 - width1;
            const float mean2 = dit[(position + 1) * 3];
            const float distance_in_mean = mean2 - mean1;
            const float sd2 = dit[(position + 1) * 3 + 1];
            const float distance_in_sd = sd2 - sd1;
            out[tid * 2] = mean1 + (distance_in_mean / distance_in_width) * ((float)desired - width1);
            out[tid * 2 + 1] = sd1 + (distance_in_sd / distance_in_width) * ((float)desired - width1);
        }
    }
}

// ---------------------------------------------------------------------------
// Boxcar S/N planes: for every start sample u of a DM trial and every width
// w = 1..nBoxcars the boxcar sum B(u, w), its S/N and the best S/N over w with
// its width; plus the half-resolution pair sums (the next iteration's input)
// and the full-width boxcar values at even starts (the next iteration's
// running values).  src/aa_device_SPS_long_kernel.cu:42-283 defines what is
// computed; the association of every sum and the order of every comparison
// below reproduce its values bit for bit:
//   * w = 4q + k + 1 (k = 0..3): B(u, w) = P_k(u + 4q) + S4(u + 4q - 4) + ...
//     + S4(u), added left to right, where P_k(v) = ((x[v] + x[v+1]) + x[v+2])
//     + x[v+3] truncated to k+1 terms and S4 = P_3; a pair of samples (2p,
//     2p+1) whose even sample has fewer than 4 samples after it counts as
//     zeros;
//   * S/N = (B - mean_w) / sd_w (later iterations: (bv(u) + (B - mean_w)) /
//     sd_w with the running value bv at the start) by the fast division;
//   * per q the best of its four widths (a later width only when strictly
//     better, the pair of pairs likewise), at q = 0 the second pair on a
//     tie; over q a later group only when strictly better.
//
// Design: one warp per window of 32 x PPL consecutive positions v of one DM
// trial, PPL consecutive positions per lane (PPL = 4 or 8).  The sum for
// start u and group q is built where v = u + 4q sits: it starts from P_k(v)
// and adds S4(v - 4), S4(v - 8), ... one group per step, each S4 taken from
// a register of the same lane or, 4q positions back, by a shuffle from a
// lane below; the group's best S/N then moves to the position u the same
// way, which folds it into its running best.  No shared memory and no block
// barrier; a window yields 32 PPL - 4(Q-1) starts (Q = nBoxcars / 4), its
// last 4(Q-1) positions only feed the others, so wider windows waste less.
// ---------------------------------------------------------------------------
constexpr int SNR_WARPS = 8;
#ifndef SPD_BOXCAR_PPL
#define SPD_BOXCAR_PPL 4
#endif

// Lane offset and register of the position 'a' positions from a lane's
// register p (a may be negative): floor division by PPL.
template <int PPL>
__host__ __device__ constexpr int pos_lane(int a)
{
    return (a >= 0) ? a / PPL : -((-a + PPL - 1) / PPL);
}
template <int PPL>
__host__ __device__ constexpr int pos_reg(int a)
{
    return a - PPL * pos_lane<PPL>(a);
}

template <int NB, bool NTH, int PPL>
__global__ void __launch_bounds__(32 * SNR_WARPS, PPL == 4 ? 4 : 1) k_boxcar_snr(const float *__restrict__ in,
                                                               const float *__restrict__ bv_in, float *bv_out,
                                                               float *dec, float *snr_out, uint16_t *taps_out,
                                                               const SnrMsd msd, int nT, int startTaps,
                                                               int dit_value, int dtm)
{
    constexpr int Q = NB / 4;
    constexpr int OUT = 32 * PPL - 4 * (Q - 1); // starts per window
    static_assert(OUT > 0 && OUT % 2 == 0, "window too short for the widths");
    const int lane = threadIdx.x & 31;
    const long long window = static_cast<long long>(blockIdx.x) * SNR_WARPS + (threadIdx.x >> 5);
    const long long wbase = window * OUT;
    if (wbase >= nT)
        return;
    const long long row = static_cast<long long>(blockIdx.y) * nT;
    const float *x = in + row;
    const long long v0 = wbase + PPL * lane; // this lane's first position (even)

    // samples v0 .. v0+PPL+2 (the last three from the next lane)
    float xs[PPL + 3];
#pragma unroll
    for (int j = 0; j < PPL; ++j)
        xs[j] = (v0 + j < nT) ? __ldg(x + v0 + j) : 0.f;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const float nx = __shfl_down_sync(0xffffffffu, xs[j], 1);
        xs[PPL + j] = (lane == 31) ? ((v0 + PPL + j < nT) ? __ldg(x + v0 + PPL + j) : 0.f) : nx;
    }
    // partial sums P_k(v) of the positions; zeros for pairs without four
    // samples after their even sample
    float acc[PPL][4], s4[PPL], bv[PPL], pair[PPL];
#pragma unroll
    for (int p = 0; p < PPL; ++p) {
        const long long v = v0 + p;
        const bool ok = ((v & ~1LL) + 4) < nT;
        const float a1 = xs[p] + xs[p + 1];
        const float a2 = a1 + xs[p + 2];
        const float a3 = a2 + xs[p + 3];
        acc[p][0] = ok ? xs[p] : 0.f;
        acc[p][1] = ok ? a1 : 0.f;
        acc[p][2] = ok ? a2 : 0.f;
        acc[p][3] = ok ? a3 : 0.f;
        s4[p] = acc[p][3];
        pair[p] = acc[p][1];
        bv[p] = 0.f;
        if (NTH && ok)
            bv[p] = __ldg(bv_in + row + v);
    }
    auto snr = [&](float b, float bvu, int w) -> float {
        const float2 st = msd.v[w];
        return NTH ? __fdividef(bvu + (b - st.x), st.y) : __fdividef(b - st.x, st.y);
    };
    float best[PPL];
    int taps[PPL];
    float full[PPL]; // B(u, NB) of this lane's starts (bv_out at even starts)
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        float fq[PPL];
        int tq[PPL];
#pragma unroll
        for (int p = 0; p < PPL; ++p) {
            // the start u = v - 4q: its S4 joins the sum, its running value
            // enters the S/N
            const int dl = pos_lane<PPL>(p - 4 * q), pr = pos_reg<PPL>(p - 4 * q);
            float bvq = 0.f;
            if (q > 0) {
                const float sv = (dl == 0) ? s4[pr] : __shfl_up_sync(0xffffffffu, s4[pr], -dl);
                acc[p][0] = acc[p][0] + sv;
                acc[p][1] = acc[p][1] + sv;
                acc[p][2] = acc[p][2] + sv;
                acc[p][3] = acc[p][3] + sv;
            }
            if (NTH)
                bvq = (dl == 0) ? bv[pr] : __shfl_up_sync(0xffffffffu, bv[pr], -dl);
            const int d = 4 * q;
            float f1 = snr(acc[p][0], bvq, d);
            float f2 = snr(acc[p][1], bvq, d + 1);
            int t1, t2;
            if (f2 > f1) {
                f1 = f2;
                t1 = d + 2;
            } else {
                t1 = d + 1;
            }
            f2 = snr(acc[p][2], bvq, d + 2);
            const float f3 = snr(acc[p][3], bvq, d + 3);
            if (f3 > f2) {
                f2 = f3;
                t2 = d + 4;
            } else {
                t2 = d + 3;
            }
            if (q == 0) {
                if (f1 > f2) {
                    best[p] = f1;
                    taps[p] = t1;
                } else {
                    best[p] = f2;
                    taps[p] = t2;
                }
            } else {
                if (f2 > f1) {
                    f1 = f2;
                    t1 = t2;
                }
                fq[p] = f1;
                tq[p] = t1;
            }
        }
        if (q > 0) {
            // position u takes the group computed 4q positions ahead
#pragma unroll
            for (int p = 0; p < PPL; ++p) {
                const int dl = pos_lane<PPL>(p + 4 * q), pr = pos_reg<PPL>(p + 4 * q);
                const float c = (dl == 0) ? fq[pr] : __shfl_down_sync(0xffffffffu, fq[pr], dl);
                const int ct = (dl == 0) ? tq[pr] : __shfl_down_sync(0xffffffffu, tq[pr], dl);
                if (c > best[p]) {
                    best[p] = c;
                    taps[p] = ct;
                }
            }
        }
        if (q == Q - 1) {
#pragma unroll
            for (int p = 0; p < PPL; ++p) {
                const int dl = pos_lane<PPL>(p + 4 * (Q - 1)), pr = pos_reg<PPL>(p + 4 * (Q - 1));
                full[p] = (dl == 0) ? acc[pr][3] : __shfl_down_sync(0xffffffffu, acc[pr][3], dl);
            }
        }
    }
#pragma unroll
    for (int p = 0; p < PPL; ++p) {
        const long long u = v0 + p;
        if (PPL * lane + p >= OUT || u >= nT)
            break;
        snr_out[row + u] = best[p];
        taps_out[row + u] = static_cast<uint16_t>(NTH ? startTaps + taps[p] * dit_value : taps[p]);
        if ((p & 1) == 0 && (u >> 1) < dtm) {
            const long long o = static_cast<long long>(blockIdx.y) * dtm + (u >> 1);
            dec[o] = pair[p];
            bv_out[o] = NTH ? bv[p] + full[p] : full[p];
        }
    }
}

// ---------------------------------------------------------------------------
// Candidates.  Peak finding (src/aa_device_peak_find_kernel.cu:72-156 with
// include/aa_device_peak_find_shared_kernel_functions.cuh): a sample is a
// candidate when it is above the cut and equal to the maximum of its
// neighbourhood -- 3 x 3 inside, the rows or columns that exist at the
// edges, 2 x 2 at the corners, where the last processed column
// (width - offset - 1) counts as the right edge.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float max_rows(const float *in, int x0, int x1, int y0, int y1, int width)
{
    // same maximum as the reference's fmaxf chains (order does not matter
    // for fmaxf except with NaN, which the planes do not hold)
    float m = __ldg(in + static_cast<long long>(y0) * width + x0);
    for (int y = y0; y <= y1; ++y)
        for (int x = x0; x <= x1; ++x)
            m = fmaxf(m, __ldg(in + static_cast<long long>(y) * width + x));
    return m;
}

__global__ void k_peak_find(const float *__restrict__ in, const uint16_t *__restrict__ taps, unsigned *c_dm,
                            unsigned *c_ts, float *c_snr, unsigned *c_bw, int width, int height, int offset,
                            float threshold, int max_cands, int *count, int shift, int dit_value)
{
    const int x = blockDim.x * blockIdx.x + threadIdx.x;
    const int y = blockDim.y * blockIdx.y + threadIdx.y;
    if (x >= width - offset || y >= height)
        return;
    const int last = width - offset - 1;
    float my, dil;
    if (width == 1 && (y == 0 || y == height - 1)) {
        my = dil = in[static_cast<long long>(y) * width];
    } else if ((y == 0 || y == height - 1) && (x == 0 || x == last)) {
        const int xa = (x == 0) ? 0 : width - offset - 2;
        const int ya = (y == 0) ? 0 : height - 2;
        dil = max_rows(in, xa, xa + 1, ya, ya + 1, width);
        my = __ldg(in + static_cast<long long>(y) * width + x);
    } else {
        const int x0 = (x == 0) ? x : x - 1, x1 = (x == last) ? x : x + 1;
        const int y0 = (y == 0) ? y : y - 1, y1 = (y == height - 1) ? y : y + 1;
        dil = max_rows(in, x0, x1, y0, y1, width);
        my = __ldg(in + static_cast<long long>(y) * width + x);
    }
    if (my > threshold && my == dil) {
        const int pos = atomicAdd(count, 1);
        if (pos < max_cands) {
            const unsigned tp = taps[static_cast<long long>(y) * width + x];
            c_dm[pos] = y + shift;
            c_ts[pos] = x * dit_value + tp / 2;
            c_snr[pos] = my;
            c_bw[pos] = tp;
        }
    }
}

// The same rule over strips of rows: a thread owns one column of
// SPD_PF_ROWS rows plus the row above and below the strip, loads them all
// first (many loads in flight), takes each row's horizontal maximum with its
// neighbour columns by warp shuffles (the two halo columns of a warp loaded
// by lanes 0 and 31), then tests each row against the maxima of the rows
// above, at and below it.  The window is the 3 x 3 neighbourhood clipped to
// columns 0..last and rows 0..height-1, which is the reference's rule
// whenever last >= 1 and height >= 2 (corners included); other shapes use
// k_peak_find.  Which samples pass does not depend on the thread layout, only
// the order in which they enter the list does (atomics, as in the reference).
constexpr int SPD_PF_ROWS = 8;
constexpr int SPD_PF_THREADS = 128;

__global__ void __launch_bounds__(SPD_PF_THREADS) k_peak_find_strips(const float *__restrict__ in,
                                                                      const uint16_t *__restrict__ taps,
                                                                      unsigned *c_dm, unsigned *c_ts, float *c_snr,
                                                                      unsigned *c_bw, int width, int height, int last,
                                                                      float threshold, int max_cands, int *count,
                                                                      int shift, int dit_value)
{
    constexpr int K = SPD_PF_ROWS + 2;
    const int x = blockIdx.x * SPD_PF_THREADS + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int y0 = blockIdx.y * SPD_PF_ROWS;
    const bool xin = x <= last;
    const bool left_halo = lane == 0 && x >= 1 && x - 1 <= last;
    const bool right_halo = lane == 31 && x + 1 <= last;
    float own[K], h[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int y = y0 - 1 + k;
        const bool yin = y >= 0 && y < height;
        const float *row = in + static_cast<long long>(y) * width;
        own[k] = (yin && xin) ? __ldg(row + x) : -INFINITY;
        h[k] = -INFINITY;
        if (yin && left_halo)
            h[k] = __ldg(row + x - 1);
        else if (yin && right_halo)
            h[k] = __ldg(row + x + 1);
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
        float left = __shfl_up_sync(FULL, own[k], 1);
        float right = __shfl_down_sync(FULL, own[k], 1);
        if (lane == 0)
            left = h[k];
        if (lane == 31)
            right = h[k];
        h[k] = fmaxf(own[k], fmaxf(left, right));
    }
#pragma unroll
    for (int r = 0; r < SPD_PF_ROWS; ++r) {
        const int y = y0 + r;
        const float v = own[r + 1];
        if (xin && y < height && v > threshold && v == fmaxf(h[r], fmaxf(h[r + 1], h[r + 2]))) {
            const int pos = atomicAdd(count, 1);
            if (pos < max_cands) {
                const unsigned tp = taps[static_cast<long long>(y) * width + x];
                c_dm[pos] = y + shift;
                c_ts[pos] = x * dit_value + tp / 2;
                c_snr[pos] = v;
                c_bw[pos] = tp;
            }
        }
    }
}

// Peak filtering, first stage (src/aa_device_peak_find_kernel.cu:10-70): a
// sample of the interior (rows 3..height-4, columns 3..width-4) that no
// sample of its 7 x 7 neighbourhood exceeds and that is above the cut.  The
// record's width is the width plane's first element, as in the reference;
// its sample uses the sample's own width.  Row maxima over 7 columns, then
// the maximum over 7 rows, over strips of SPD_PF7_ROWS rows.
constexpr int SPD_PF7_ROWS = 8;

__global__ void __launch_bounds__(128) k_peak_find_7x7(const float *__restrict__ in, const uint16_t *__restrict__ taps,
                                                       unsigned *c_dm, unsigned *c_ts, float *c_snr, unsigned *c_bw,
                                                       int width, int height, float threshold, int max_cands,
                                                       int *count, int shift, int dit_value)
{
    constexpr int K = SPD_PF7_ROWS + 6;
    const int x = blockIdx.x * 128 + threadIdx.x;
    const int y0 = 3 + blockIdx.y * SPD_PF7_ROWS; // first output row of the strip
    const bool xin = x >= 3 && x <= width - 4;
    float h[K], own[SPD_PF7_ROWS];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int y = y0 - 3 + k;
        h[k] = -INFINITY;
        if (xin && y < height) {
            const float *r = in + static_cast<long long>(y) * width + x;
            float m = __ldg(r - 3);
#pragma unroll
            for (int i = -2; i <= 3; ++i)
                m = fmaxf(m, __ldg(r + i));
            h[k] = m;
            if (k >= 3 && k < 3 + SPD_PF7_ROWS)
                own[k - 3] = __ldg(r);
        }
    }
    if (!xin)
        return;
#pragma unroll
    for (int r = 0; r < SPD_PF7_ROWS; ++r) {
        const int y = y0 + r;
        if (y > height - 4)
            break;
        float m = h[r];
#pragma unroll
        for (int i = 1; i < 7; ++i)
            m = fmaxf(m, h[r + i]);
        const float c = own[r];
        if (c == m && c > threshold) {
            const int pos = atomicAdd(count, 1);
            if (pos < max_cands) {
                c_dm[pos] = y + shift;
                c_ts[pos] = x * dit_value + taps[static_cast<long long>(y) * width + x] / 2;
                c_snr[pos] = c;
                c_bw[pos] = taps[0];
            }
        }
    }
}

// Peak filtering, second stage (src/aa_device_peak_find_kernel.cu:391-486):
// a candidate is dropped when another one with at least its S/N lies closer
// than max_distance (squared, in DM trials and samples) but not at distance
// 0.  One thread per candidate, the others staged through shared memory.
constexpr int SPD_FILTER_THREADS = 256;

__global__ void __launch_bounds__(SPD_FILTER_THREADS) k_filter_peaks(
    const unsigned *__restrict__ dm, const unsigned *__restrict__ ts, const unsigned *__restrict__ bw,
    const float *__restrict__ snr, int n, unsigned max_distance, unsigned *o_dm, unsigned *o_ts, unsigned *o_bw,
    float *o_snr, int max_cands, int *count)
{
    __shared__ int s_dm[SPD_FILTER_THREADS], s_ts[SPD_FILTER_THREADS];
    __shared__ float s_snr[SPD_FILTER_THREADS];
    const int p = blockIdx.x * SPD_FILTER_THREADS + threadIdx.x;
    const bool have = p < n;
    const int d = have ? static_cast<int>(dm[p]) : 0;
    const int t = have ? static_cast<int>(ts[p]) : 0;
    const float sp = have ? snr[p] : 0.f;
    bool keep = have;
    for (int base = 0; base < n; base += SPD_FILTER_THREADS) {
        const int q = base + threadIdx.x;
        __syncthreads();
        s_dm[threadIdx.x] = q < n ? static_cast<int>(dm[q]) : 0;
        s_ts[threadIdx.x] = q < n ? static_cast<int>(ts[q]) : 0;
        s_snr[threadIdx.x] = q < n ? snr[q] : -1000.f;
        __syncthreads();
        if (keep) {
            for (int k = 0; k < SPD_FILTER_THREADS; ++k) {
                if (s_snr[k] >= sp) {
                    const float fs = static_cast<float>(s_dm[k]) - static_cast<float>(d);
                    const float fd = static_cast<float>(s_ts[k]) - static_cast<float>(t);
                    const float distance = (fd * fd + fs * fs);
                    if ((distance < static_cast<float>(max_distance)) && (distance != 0)) {
                        keep = false;
                        break;
                    }
                }
            }
        }
    }
    if (keep) {
        const int pos = atomicAdd(count, 1);
        if (pos < max_cands) {
            o_dm[pos] = dm[p];
            o_ts[pos] = ts[p];
            o_bw[pos] = bw[p];
            o_snr[pos] = snr[p];
        }
    }
}

// Thresholding (src/aa_device_threshold_kernel.cu:10-41): every sample of
// the rows 0 .. 4*floor(nDMs/4)-1 and columns < offset above the cut.
// A block of 256 threads covers 1024 columns of one row, four per thread.
__global__ void __launch_bounds__(256) k_threshold(const float *__restrict__ in, const uint16_t *__restrict__ taps,
                                                   unsigned *c_dm, unsigned *c_ts, float *c_snr, unsigned *c_bw,
                                                   int *count, float threshold, int nT, int offset, int shift,
                                                   int max_cands, int dit_value)
{
    const int y = blockIdx.y;
    const float *row = in + static_cast<long long>(y) * nT;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int x = blockIdx.x * 1024 + k * 256 + threadIdx.x;
        if (x >= offset)
            break;
        const float R = __ldg(row + x);
        if (R > threshold) {
            const int pos = atomicAdd(count, 1);
            if (pos < max_cands) {
                const unsigned tp = taps[static_cast<long long>(y) * nT + x];
                c_dm[pos] = y + shift;
                c_ts[pos] = dit_value * x + tp / 2;
                c_snr[pos] = R;
                c_bw[pos] = tp;
            }
        }
    }
}

} // namespace

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
MsdConf msd_conf(long long nTimesamples, long long nDMs, long long offset)
{
    // include/aa_device_MSD_Configuration.hpp:33-99
    MsdConf c{};
    c.nTimesamples = nTimesamples;
    c.nDMs = nDMs;
    c.offset = offset;
    const int nsx = SPD_NTHREADS;
    c.nBlocks_x = static_cast<int>((nTimesamples - offset) / nsx);
    if ((nTimesamples - offset) - static_cast<long long>(c.nBlocks_x) * nsx > 0)
        c.nBlocks_x++;
    // largest product of small prime factors of nDMs not above 64
    {
        const int seive[12] = {2, 3, 4, 5, 7, 11, 13, 17, 19, 23, 29, 31};
        int number = static_cast<int>(nDMs), N = 1, N_accepted = 1;
        do {
            N = 1;
            for (int f = 0; f < 12; ++f) {
                const int nb = number / seive[f];
                if (number - nb * seive[f] == 0) {
                    N = seive[f];
                    N_accepted *= N;
                    break;
                }
            }
            number /= N;
        } while (N_accepted <= 64 && N > 1);
        c.nSteps_y = N_accepted / N;
    }
    c.nBlocks_y = static_cast<int>(nDMs / c.nSteps_y);
    c.nBlocks_total = c.nBlocks_x * c.nBlocks_y;
    int nThreads = 2048, itemp = 0;
    while (itemp == 0 && nThreads > 32) {
        nThreads >>= 1;
        itemp = c.nBlocks_total / (nThreads * 32);
    }
    c.final_threads = nThreads < 32 ? 32 : nThreads;
    return c;
}

cudaError_t msd_plane(float *d_msd, const float *d_input, float *d_partials, const MsdConf &c, bool outlier_rejection,
                      float sigma, float *d_pp, cudaStream_t st)
{
    if (c.nBlocks_x < 1 || c.nBlocks_y < 1)
        return cudaErrorInvalidValue;
    const dim3 grid(c.nBlocks_x, c.nBlocks_y);
    if (!outlier_rejection) {
        k_msd_partials<<<grid, SPD_NTHREADS, 0, st>>>(d_input, d_partials, c.nSteps_y, c.nTimesamples, c.offset);
        ++g_spd_launches;
        k_msd_final<<<1, c.final_threads, 0, st>>>(d_partials, d_msd, d_pp, c.nBlocks_total, 1);
        ++g_spd_launches;
        return cudaGetLastError();
    }
    // src/aa_device_MSD.cu:110-196
    k_msd_partials_minmax<<<grid, SPD_NTHREADS, 0, st>>>(d_input, d_partials, c.nSteps_y, c.nTimesamples, c.offset);
    ++g_spd_launches;
    k_msd_final<<<1, c.final_threads, 0, st>>>(d_partials, d_msd, nullptr, c.nBlocks_total, 1);
    ++g_spd_launches;
    for (int i = 0; i < 5; ++i) {
        k_msd_partials_rejection<<<grid, SPD_NTHREADS, 0, st>>>(d_input, d_partials, d_msd, c.nSteps_y, c.nTimesamples,
                                                                c.offset, sigma);
        ++g_spd_launches;
        k_msd_final<<<1, c.final_threads, 0, st>>>(d_partials, d_msd, nullptr, c.nBlocks_total, 0);
        ++g_spd_launches;
    }
    if (d_pp) {
        k_msd_final<<<1, c.final_threads, 0, st>>>(d_partials, d_msd, d_pp, c.nBlocks_total, 0);
        ++g_spd_launches;
    }
    return cudaGetLastError();
}

cudaError_t dit_pairs(const float *d_in, float *d_out, int nDMs, int nT, cudaStream_t st)
{
    const long long dts = nT >> 1;
    if (dts == 0)
        return cudaErrorInvalidValue;
    const int rows = (nDMs / 2) * 2;
    if (rows == 0)
        return cudaSuccess;
    const dim3 grid(static_cast<unsigned>((dts + 255) / 256), rows);
    if (nT % 2 == 0 && (reinterpret_cast<uintptr_t>(d_in) & 7) == 0)
        k_dit_pairs2<<<grid, 256, 0, st>>>(reinterpret_cast<const float2 *>(d_in), d_out, rows, dts);
    else
        k_dit_pairs<<<grid, 256, 0, st>>>(d_in, d_out, rows, nT, dts);
    ++g_spd_launches;
    return cudaGetLastError();
}

cudaError_t fir_rows(const float *d_in, float *d_out, int nDMs, int nT, int nTaps, cudaStream_t st)
{
    const int n = nT - nTaps + 1;
    if (n <= 0 || nDMs <= 0)
        return cudaErrorInvalidValue;
    k_fir_rows<<<dim3((n + 255) / 256, nDMs), 256, 0, st>>>(d_in, d_out, nTaps, nT);
    ++g_spd_launches;
    return cudaGetLastError();
}

cudaError_t msd_interpolate(const float *d_msd_dit, float *d_msd_interp, const int *d_dit_widths, int n_dit,
                            const int *d_widths, int n_widths, int max_width_performed, cudaStream_t st)
{
    if (n_widths < 1 || n_widths > 1024)
        return cudaErrorInvalidValue;
    k_msd_interpolate<<<1, n_widths, 0, st>>>(d_msd_dit, d_msd_interp, d_dit_widths, n_dit, d_widths,
                                              max_width_performed);
    ++g_spd_launches;
    return cudaGetLastError();
}

// nBlocks: the plan's count of the reference's 512-thread blocks, 0 when the
// plane is too short to be searched at this iteration (then nothing is
// written); otherwise every start sample of every DM trial is covered
template <bool NTH>
static cudaError_t launch_boxcar_snr(const float *in, const float *bv_in, float *bv_out, float *dec, float *snr,
                                     uint16_t *taps, const SnrMsd &msd, int nT, int nBoxcars, int startTaps,
                                     int dit_value, int dtm, int nBlocks, int nDMs, cudaStream_t st)
{
    if (nBlocks <= 0 || nT <= 0)
        return cudaSuccess;
    // positions per lane: 8 where the widths span several lanes' positions
    const int ppl = (nBoxcars >= 16) ? SPD_BOXCAR_PPL : 4;
    const int out = 32 * ppl - 4 * (nBoxcars / 4 - 1);
    const long long windows = (static_cast<long long>(nT) + out - 1) / out;
    const dim3 grid(static_cast<unsigned>((windows + SNR_WARPS - 1) / SNR_WARPS), nDMs);
    switch (nBoxcars) {
    case 32:
        k_boxcar_snr<32, NTH, SPD_BOXCAR_PPL><<<grid, 32 * SNR_WARPS, 0, st>>>(in, bv_in, bv_out, dec, snr, taps, msd,
                                                                              nT, startTaps, dit_value, dtm);
        break;
    case 16:
        k_boxcar_snr<16, NTH, SPD_BOXCAR_PPL><<<grid, 32 * SNR_WARPS, 0, st>>>(in, bv_in, bv_out, dec, snr, taps, msd,
                                                                              nT, startTaps, dit_value, dtm);
        break;
    case 8:
        k_boxcar_snr<8, NTH, 4><<<grid, 32 * SNR_WARPS, 0, st>>>(in, bv_in, bv_out, dec, snr, taps, msd, nT,
                                                                startTaps, dit_value, dtm);
        break;
    default:
        return cudaErrorInvalidValue;
    }
    ++g_spd_launches;
    return cudaGetLastError();
}

cudaError_t spdt_first_plane(const float *d_input, float *d_bv_out, float *d_decimated, float *d_snr, uint16_t *d_taps,
                             const SnrMsd &msd, int nTimesamples, int nBoxcars, int dtm, int nBlocks, int nDMs,
                             cudaStream_t st)
{
    return launch_boxcar_snr<false>(d_input, nullptr, d_bv_out, d_decimated, d_snr, d_taps, msd, nTimesamples,
                                    nBoxcars, 0, 1, dtm, nBlocks, nDMs, st);
}

cudaError_t spdt_nth_plane(const float *d_input, const float *d_bv_in, float *d_bv_out, float *d_decimated,
                           float *d_snr, uint16_t *d_taps, const SnrMsd &msd, int nTimesamples, int nBoxcars,
                           int startTaps, int dit_value, int dtm, int nBlocks, int nDMs, cudaStream_t st)
{
    return launch_boxcar_snr<true>(d_input, d_bv_in, d_bv_out, d_decimated, d_snr, d_taps, msd, nTimesamples,
                                   nBoxcars, startTaps, dit_value, dtm, nBlocks, nDMs, st);
}

cudaError_t spd_peak_find(const float *d_snr, const uint16_t *d_taps, unsigned *d_dm, unsigned *d_ts, float *d_csnr,
                          unsigned *d_bw, int width, int height, int offset, float threshold, int max_cands,
                          int *d_count, int shift, int dit_value, cudaStream_t st)
{
    if (width - offset - 1 <= 0)
        return cudaSuccess;
    const int last = width - offset - 1;
    if (height >= 2) {
        const dim3 grid((last + SPD_PF_THREADS) / SPD_PF_THREADS, (height + SPD_PF_ROWS - 1) / SPD_PF_ROWS);
        k_peak_find_strips<<<grid, SPD_PF_THREADS, 0, st>>>(d_snr, d_taps, d_dm, d_ts, d_csnr, d_bw, width, height,
                                                             last, threshold, max_cands, d_count, shift, dit_value);
        ++g_spd_launches;
        return cudaGetLastError();
    }
    const dim3 block(32, 2);
    const dim3 grid(1 + (width - offset - 1) / 32, 1 + (height - 1) / 2);
    k_peak_find<<<grid, block, 0, st>>>(d_snr, d_taps, d_dm, d_ts, d_csnr, d_bw, width, height, offset, threshold,
                                        max_cands, d_count, shift, dit_value);
    ++g_spd_launches;
    return cudaGetLastError();
}

cudaError_t spd_peak_find_7x7(const float *d_snr, const uint16_t *d_taps, unsigned *d_dm, unsigned *d_ts, float *d_csnr,
                              unsigned *d_bw, int width, int height, int offset, float threshold, int max_cands,
                              int *d_count, int shift, int dit_value, cudaStream_t st)
{
    // launched when the iteration has searched columns; the stencil itself
    // covers the whole interior, the unprocessed tail included
    if (width - offset - 1 <= 0 || width < 7 || height < 7)
        return cudaSuccess;
    const dim3 grid((width + 127) / 128, (height - 6 + SPD_PF7_ROWS - 1) / SPD_PF7_ROWS);
    k_peak_find_7x7<<<grid, 128, 0, st>>>(d_snr, d_taps, d_dm, d_ts, d_csnr, d_bw, width, height, threshold,
                                          max_cands, d_count, shift, dit_value);
    ++g_spd_launches;
    return cudaGetLastError();
}

cudaError_t spd_filter_peaks(const unsigned *d_dm, const unsigned *d_ts, const unsigned *d_bw, const float *d_snr,
                             int n, unsigned max_distance, unsigned *o_dm, unsigned *o_ts, unsigned *o_bw,
                             float *o_snr, int max_cands, int *d_count, cudaStream_t st)
{
    if (n <= 0)
        return cudaSuccess;
    k_filter_peaks<<<(n + SPD_FILTER_THREADS - 1) / SPD_FILTER_THREADS, SPD_FILTER_THREADS, 0, st>>>(
        d_dm, d_ts, d_bw, d_snr, n, max_distance, o_dm, o_ts, o_bw, o_snr, max_cands, d_count);
    ++g_spd_launches;
    return cudaGetLastError();
}

cudaError_t spd_threshold(const float *d_snr, const uint16_t *d_taps, unsigned *d_dm, unsigned *d_ts, float *d_csnr,
                          unsigned *d_bw, int *d_count, float threshold, int nTimesamples, int offset, int shift,
                          int max_cands, int dit_value, int nDMs, cudaStream_t st)
{
    const int rows = (nDMs / 4) * 4;
    if (offset <= 0 || rows == 0)
        return cudaSuccess;
    // every column < offset of the rows below 4 * floor(nDMs / 4)
    const int nb = (offset + 1023) / 1024;
    k_threshold<<<dim3(nb, rows), 256, 0, st>>>(d_snr, d_taps, d_dm, d_ts, d_csnr, d_bw, d_count, threshold,
                                                nTimesamples, offset, shift, max_cands, dit_value);
    ++g_spd_launches;
    return cudaGetLastError();
}

} // namespace aab200
