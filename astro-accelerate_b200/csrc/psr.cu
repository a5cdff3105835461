// psr.cu -- periodicity building blocks (see psr.cuh).
#include "psr.cuh"

#include <atomic>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

namespace aab200 {

namespace {

std::atomic<long long> g_psr_launches{0};

// ---------------------------------------------------------------------------
// Power and interbin spectra.  One thread per pair of bins (2i, 2i+1) of one
// spectrum; the pair's right neighbour (bin 2i+2, needed by the interbin
// value of bin 2i+1) is the next lane's first bin, passed by a shuffle (the
// last lane of a warp loads it).  Per bin the values follow
// src/aa_device_power_kernel.cu:19-41: X / norm component-wise (the fast
// division), |X|^2, and 0.616850275 |X_k - X_{k+1}|^2; bin 0 and the bins
// at and above nT/2 give zeros.  Four consecutive interbin entries are one
// 16-byte store when the row length allows it.
// ---------------------------------------------------------------------------
constexpr int PSR_PAIR_THREADS = 256;

// How the contractible expressions below are evaluated.  The values must
// round exactly as the reference build's (nvcc with --use_fast_math, which
// fuses a multiply into a following add); each form is spelled out with
// intrinsics so that the result does not depend on the compiler's choice in
// this file's context.  Form 0 leaves the choice to the compiler.
// The forms used are those that give the reference's bits on the golden
// spectra (tests/golden/psr_golden.json).
#ifndef PSR_POWER_FORM
#define PSR_POWER_FORM 2 // power spectra x*x + y*y: 1 fma(x,x,y*y), 2 fma(y,y,x*x), 3 unfused, 0 compiler's choice
#endif
#ifndef PSR_MEDIAN_POWER_FORM
#define PSR_MEDIAN_POWER_FORM 1 // powers of the whitening medians, the same choices
#endif
#ifndef PSR_INTERP_FORM
#define PSR_INTERP_FORM 1 // mean + slope*i: 1 fma, 2 unfused, 0 compiler's choice
#endif
#ifndef PSR_SCAL_FORM
#define PSR_SCAL_FORM 1 // scalloping correction in double: 1 nested fma, 2 unfused, 0 compiler's choice
#endif
#ifndef PSR_PP_FORM
#define PSR_PP_FORM 1 // PRESTO-plus bin f*frac + 0.5 in double: 1 fma, 2 unfused, 0 compiler's choice
#endif
#ifndef PSR_DIV_FORM
#define PSR_DIV_FORM 4 // X / norm of the power spectra: 1 __fdividef, 2 x * (1/norm), 3 IEEE, 4 x * rcp_rn(norm),
                       // 0 the division operator (fast-math build)
#endif

template <int FORM> __device__ __forceinline__ float psr_sq2(float x, float y)
{
    if (FORM == 1)
        return fmaf(x, x, __fmul_rn(y, y));
    if (FORM == 2)
        return fmaf(y, y, __fmul_rn(x, x));
    if (FORM == 3)
        return __fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y));
    return x * x + y * y;
}

__device__ __forceinline__ float psr_div(float x, float norm)
{
#if PSR_DIV_FORM == 1
    return __fdividef(x, norm);
#elif PSR_DIV_FORM == 2
    return x * (1.0f / norm);
#elif PSR_DIV_FORM == 3
    return __fdiv_rn(x, norm);
#elif PSR_DIV_FORM == 4
    return __fmul_rn(x, __frcp_rn(norm));
#else
    return x / norm;
#endif
}

__device__ __forceinline__ float2 psr_scaled(float2 a, float norm) { return make_float2(psr_div(a.x, norm), psr_div(a.y, norm)); }
__device__ __forceinline__ float psr_power(float2 a) { return psr_sq2<PSR_POWER_FORM>(a.x, a.y); }
__device__ __forceinline__ float psr_interbin(float2 a, float2 b)
{
    return 0.616850275f * psr_sq2<PSR_POWER_FORM>(a.x - b.x, a.y - b.y);
}

template <bool VEC4>
__global__ void __launch_bounds__(PSR_PAIR_THREADS) k_power_pairs(const float2 *__restrict__ in, float *power,
                                                                  float *interbin, int nT, float norm)
{
    const int half = nT >> 1;
    const long long r = blockIdx.y;
    const float2 *spec = in + r * (half + 1);
    const int k0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    const float2 zero = make_float2(0.f, 0.f);
    const float2 x0 = (k0 <= half) ? spec[k0] : zero;
    const float2 x1 = (k0 + 1 <= half) ? spec[k0 + 1] : zero;
    float2 x2;
    x2.x = __shfl_down_sync(0xffffffffu, x0.x, 1);
    x2.y = __shfl_down_sync(0xffffffffu, x0.y, 1);
    if ((threadIdx.x & 31) == 31)
        x2 = (k0 + 2 <= half) ? spec[k0 + 2] : zero;
    // bin k0 (zero at k0 = 0) and bin k0 + 1
    const float2 a = (k0 > 0) ? psr_scaled(x0, norm) : zero;
    const float2 b = (k0 > 0) ? psr_scaled(x1, norm) : zero;
    const float2 c = psr_scaled(x1, norm);
    const float2 d = psr_scaled(x2, norm);
    const float pa = psr_power(a), pc = psr_power(c);
    const float ia = psr_interbin(a, b), ic = psr_interbin(c, d);
    float *prow = power + r * half;
    float *irow = interbin + r * nT;
    if (VEC4 && k0 + 1 < half) {
        prow[k0] = pa;
        prow[k0 + 1] = pc;
        *reinterpret_cast<float4 *>(irow + 2 * k0) = make_float4(pa, ia, pc, ic);
    } else {
        if (k0 < half) {
            prow[k0] = pa;
            irow[2 * k0] = pa;
            irow[2 * k0 + 1] = ia;
        }
        if (k0 + 1 < half) {
            prow[k0 + 1] = pc;
            irow[2 * k0 + 2] = pc;
            irow[2 * k0 + 3] = ic;
        }
    }
}

// ---------------------------------------------------------------------------
// Simple harmonic sum over corner-turned power spectra [bin][spectrum]: four
// neighbouring spectra per thread (one 16-byte load per harmonic when the
// spectrum count allows it), the (mean, deviation) table of the harmonic
// counts staged once per block in shared memory.  Per spectrum and bin b the
// running sum over bins b, 2b, ... (below nBins) and the best
// (sum - mean_f) / sd_f with its f, as src/aa_device_harmonic_summing_kernel.cu:8-39
// defines them (the fast division; a later f must be strictly better).
// ---------------------------------------------------------------------------
constexpr int PSR_HS_THREADS = 128;
constexpr int PSR_MAX_HARMONICS = 32;

template <int V>
__global__ void __launch_bounds__(PSR_HS_THREADS) k_harmonic_columns(const float *__restrict__ in, float *snr_out,
                                                                     uint16_t *harm_out, const float *__restrict__ msd,
                                                                     int nBins, int nSpectra, int nHarmonics)
{
    __shared__ float s_msd[2 * PSR_MAX_HARMONICS];
    for (int i = threadIdx.x; i < 2 * nHarmonics; i += blockDim.x)
        s_msd[i] = msd[i];
    __syncthreads();
    const int s0 = V * (blockIdx.y * blockDim.x + threadIdx.x);
    if (s0 >= nSpectra)
        return;
    const long long b = blockIdx.x;
    float acc[V], best[V];
    uint16_t hbest[V];
    auto load = [&](long long bin, float *v) {
        const float *p = in + bin * nSpectra + s0;
        if (V == 4) {
            const float4 q = __ldg(reinterpret_cast<const float4 *>(p));
            v[0] = q.x;
            v[1] = q.y;
            v[2] = q.z;
            v[3] = q.w;
        } else {
#pragma unroll
            for (int k = 0; k < V; ++k)
                v[k] = __ldg(p + k);
        }
    };
    load(b, acc);
#pragma unroll
    for (int k = 0; k < V; ++k) {
        best[k] = (acc[k] - s_msd[0]) / s_msd[1];
        hbest[k] = 0;
    }
    if (b > 0) {
        for (int f = 1; f < nHarmonics; ++f) {
            const long long bin = (f + 1) * b;
            if (bin >= nBins)
                break; // the bins of later harmonics are further out
            float v[V];
            load(bin, v);
            const float m = s_msd[2 * f], sd = s_msd[2 * f + 1];
#pragma unroll
            for (int k = 0; k < V; ++k) {
                acc[k] = acc[k] + v[k];
                const float t = (acc[k] - m) / sd;
                if (t > best[k]) {
                    best[k] = t;
                    hbest[k] = static_cast<uint16_t>(f);
                }
            }
        }
    }
#pragma unroll
    for (int k = 0; k < V; ++k) {
        snr_out[b * nSpectra + s0 + k] = best[k];
        harm_out[b * nSpectra + s0 + k] = hbest[k];
    }
}

// Peak finding for the periodicity search
// (src/aa_device_peak_find_kernel.cu:340-389 with the neighbourhood rule of
// include/aa_device_peak_find_shared_kernel_functions.cuh:217-287): a value
// above the cut that equals the maximum of its 3 x 3 neighbourhood clipped
// to the plane (width >= 2, height >= 2).  Records of 4 floats: DM trial,
// frequency bin / DIT, S/N turned back into power with the harmonic's
// (mean, deviation) as mean + S/N * deviation, harmonic count.
__device__ __forceinline__ float psr_window_max(const float *in, int x, int y, int width, int height)
{
    const int x0 = x > 0 ? x - 1 : x, x1 = x < width - 1 ? x + 1 : x;
    const int y0 = y > 0 ? y - 1 : y, y1 = y < height - 1 ? y + 1 : y;
    float m = __ldg(in + static_cast<long long>(y0) * width + x0);
    for (int yy = y0; yy <= y1; ++yy)
        for (int xx = x0; xx <= x1; ++xx)
            m = fmaxf(m, __ldg(in + static_cast<long long>(yy) * width + xx));
    return m;
}

__global__ void k_psr_peaks(const float *__restrict__ in, const uint16_t *__restrict__ harm, float *list, int width,
                            int height, float threshold, int max_peaks, int *count, const float *__restrict__ msd,
                            int dm_shift, int dit, int transposed, int greedy)
{
    const int idxX = blockDim.x * blockIdx.x + threadIdx.x;
    const int idxY = blockDim.y * blockIdx.y + threadIdx.y;
    if (idxX >= width || idxY >= height)
        return;
    const long long pos = static_cast<long long>(idxY) * width + idxX;
    const float my_value = __ldg(in + pos);
    if (!(my_value > threshold && my_value == psr_window_max(in, idxX, idxY, width, height)))
        return;
    const int list_pos = atomicAdd(count, 1);
    if (list_pos >= max_peaks)
        return;
    const int raw = static_cast<int>(harm[pos]);
    int hrms = raw;
    if (transposed) {
        list[4 * list_pos] = idxX + dm_shift;
        list[4 * list_pos + 1] = idxY / dit;
        list[4 * list_pos + 3] = hrms;
    } else {
        list[4 * list_pos] = idxY + dm_shift;
        list[4 * list_pos + 1] = idxX / dit;
        if (greedy) {
            const int temp = hrms / 100;
            hrms = hrms - 100 * temp;
        }
        list[4 * list_pos + 3] = static_cast<float>(raw);
    }
    list[4 * list_pos + 2] = my_value * __ldg(&msd[2 * hrms + 1]) + __ldg(&msd[2 * hrms]);
}

// Thresholding for the periodicity search
// (src/aa_device_threshold_kernel.cu:43-112): every value above the cut,
// recorded as the peak finder records it.
__global__ void k_psr_threshold(const float *__restrict__ in, const uint16_t *__restrict__ harm, float *list,
                                int width, int height, float threshold, int max_peaks, int *count,
                                const float *__restrict__ msd, int dm_shift, int dit, int transposed, int greedy)
{
    const int x = blockDim.x * blockIdx.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= width || y >= height)
        return;
    const long long pos = static_cast<long long>(y) * width + x;
    const float R = __ldg(in + pos);
    if (!(R > threshold))
        return;
    const int list_pos = atomicAdd(count, 1);
    if (list_pos >= max_peaks)
        return;
    const int raw = static_cast<int>(harm[pos]);
    int hrms = raw;
    if (transposed) {
        list[4 * list_pos] = x + dm_shift;
        list[4 * list_pos + 1] = y / dit;
        list[4 * list_pos + 3] = hrms;
    } else {
        list[4 * list_pos] = y + dm_shift;
        list[4 * list_pos + 1] = x / dit;
        if (greedy) {
            const int temp = hrms / 100;
            hrms = hrms - 100 * temp;
        }
        list[4 * list_pos + 3] = static_cast<float>(raw);
    }
    list[4 * list_pos + 2] = R * __ldg(&msd[2 * hrms + 1]) + __ldg(&msd[2 * hrms]);
}

// ---------------------------------------------------------------------------
// Harmonic sums over normal planes [nDMs][nTimesamples]
// (src/aa_device_harmonic_summing_kernel.cu:41-268 define the three
// algorithms).  With the scalloping-loss correction every bin the sums read
// is the same five-bin combination of its neighbours, so it is computed once
// per bin by k_scalloping_corrected into a scratch plane and the sum kernels
// read one value per bin from it; without the correction they read the input.
// One thread per output bin, rows along the grid's y; the (mean, deviation)
// table of the harmonic counts is staged once per block in shared memory.
// ---------------------------------------------------------------------------
// X0 + 0.94247 (X-1 + X+1) + 0.44247 (X-2 + X+2), evaluated in double with
// the reference's constants and order, rounded to float
__device__ __forceinline__ float psr_corrected(float Xm2, float Xm1, float X0, float Xp1, float Xp2)
{
#if PSR_SCAL_FORM == 1
    return (float)fma((0.88494 / 2.0), (double)(Xm2 + Xp2), fma((1.88494 / 2.0), (double)(Xm1 + Xp1), (double)X0));
#elif PSR_SCAL_FORM == 2
    return (float)__dadd_rn(__dadd_rn((double)X0, __dmul_rn((1.88494 / 2.0), (double)(Xm1 + Xp1))),
                            __dmul_rn((0.88494 / 2.0), (double)(Xm2 + Xp2)));
#else
    return (X0 + (1.88494 / 2.0) * (Xm1 + Xp1) + (0.88494 / 2.0) * (Xm2 + Xp2));
#endif
}

__device__ __forceinline__ int psr_pp_bin(int f, double frac)
{
#if PSR_PP_FORM == 1
    return (int)fma((double)f, frac, 0.5);
#elif PSR_PP_FORM == 2
    return (int)__dadd_rn(__dmul_rn((double)f, frac), 0.5);
#else
    return (int)((((double)f) * frac) + 0.5);
#endif
}

constexpr int PSR_COR_TILE = 256;

// out[k] for 2 <= k <= nT-3 (the bins whose five-bin window lies in the row);
// each block stages its tile with a two-bin halo on each side
__global__ void __launch_bounds__(PSR_COR_TILE) k_scalloping_corrected(const float *__restrict__ in, float *out,
                                                                       int nT)
{
    __shared__ float t[PSR_COR_TILE + 4];
    const long long row = static_cast<long long>(blockIdx.y) * nT;
    const int k0 = blockIdx.x * PSR_COR_TILE;
    for (int i = threadIdx.x; i < PSR_COR_TILE + 4; i += blockDim.x) {
        const int k = k0 - 2 + i;
        t[i] = (k >= 0 && k < nT) ? in[row + k] : 0.f;
    }
    __syncthreads();
    const int k = k0 + threadIdx.x;
    if (k >= nT)
        return;
    const float *w = t + threadIdx.x; // w[2] is bin k
    out[row + k] = (k >= 2 && k + 2 < nT) ? psr_corrected(w[0], w[1], w[2], w[3], w[4]) : 0.f;
}

// nH: harmonics (greedy, PRESTO plus) or powers of two (PRESTO); n_msd:
// entries of the (mean, deviation) table, at most 2 * PSR_MAX_HARMONICS
template <int ALG>
__global__ void __launch_bounds__(256) k_harmonic_rows(const float *__restrict__ v, float *snr_out,
                                                       uint16_t *harm_out, const float *__restrict__ msd, int nT,
                                                       int nH, int n_msd)
{
    __shared__ float s_msd[2 * PSR_MAX_HARMONICS];
    for (int i = threadIdx.x; i < n_msd; i += blockDim.x)
        s_msd[i] = msd[i];
    __syncthreads();
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= nT)
        return;
    const float *rv = v + static_cast<long long>(blockIdx.y) * nT;
    auto bin = [&](int k, int hi) -> float { return (k > 1 && k + hi < nT) ? __ldg(rv + k) : 0.f; };
    float best;
    int out_h;
    if (ALG == 1) {
        // greedy: at each harmonic the larger of bins p and p+1, p = (h+1) pos
        // + the steps taken so far; the count plus 100 x the steps at the best
        int steps = 0, best_h = 0, best_steps = 0;
        float lo = 0.f, hi = 0.f;
        if (pos > 1 && pos + 3 < nT) {
            lo = __ldg(rv + pos);
            hi = __ldg(rv + pos + 1);
        }
        float sum;
        if (hi > lo) {
            ++steps;
            sum = hi;
        } else {
            sum = lo;
        }
        best = fdividef((sum - s_msd[0]), s_msd[1]);
        for (int h = 1; h < nH; ++h) {
            const int p = (h + 1) * pos + steps;
            lo = hi = 0.f;
            if (p > 1 && p + 3 < nT) {
                lo = __ldg(rv + p);
                hi = __ldg(rv + p + 1);
            }
            if (hi > lo) {
                ++steps;
                sum = sum + hi;
            } else {
                sum = sum + lo;
            }
            const float snr = fdividef((sum - s_msd[2 * h]), s_msd[2 * h + 1]);
            if (snr > best) {
                best = snr;
                best_h = h;
                best_steps = steps;
            }
        }
        out_h = best_h + 100 * best_steps;
    } else if (ALG == 2) {
        // PRESTO plus: count i sums the fundamental and bins round(f pos / (i+1)),
        // f = 1..i; reported as i - 1
        const float fund = bin(pos, 2);
        best = fdividef((fund - s_msd[0]), s_msd[1]);
        out_h = 0;
        if (pos > 1 && pos + 2 < nT) {
            for (int i = 1; i < nH; ++i) {
                float sum = fund;
                const double frac = ((double)pos) / ((double)(i + 1));
                for (int f = 1; f <= i; ++f)
                    sum = sum + bin(psr_pp_bin(f, frac), 2);
                const float snr = fdividef((sum - s_msd[2 * i]), s_msd[2 * i + 1]);
                if (snr > best) {
                    best = snr;
                    out_h = i - 1;
                }
            }
        }
    } else {
        // PRESTO: for 1, 2, 4, ... harmonics (nH here is the count of
        // powers of two) the fundamental at round(pos / n) plus its even
        // multiples
        best = -10000;
        out_h = 0;
        for (int i = 0; i < nH; ++i) {
            const int n = 1 << i;
            const float frac = ((double)pos) * (1.0 / ((double)n));
            float sum = bin((int)(frac + 0.5), 2);
            for (int f = 2; f <= n; f += 2)
                sum = sum + bin((int)(((float)f) * frac + 0.5), 2);
            const float snr = fdividef((sum - s_msd[2 * (n / 2)]), s_msd[2 * (n / 2) + 1]);
            if (snr > best) {
                best = snr;
                out_h = n - 1;
            }
        }
    }
    const long long o = static_cast<long long>(blockIdx.y) * nT + pos;
    snr_out[o] = best;
    harm_out[o] = static_cast<uint16_t>(out_h);
}

// ---------------------------------------------------------------------------
// Spectral whitening (src/aa_device_spectral_whitening_kernel.cu:338-427
// defines the medians and the SGP2 normalisation).
//
// Medians: one warp per (segment, spectrum).  The segment's powers |X|^2 (at
// most 256 bins) fill 32 x V registers of the warp (element e = 32 v + lane,
// slots past the segment hold +inf) and a bitonic network sorts them: pairs
// 32 or more elements apart exchange inside a lane's registers, nearer pairs
// across lanes by shuffles.  The median is the sorted power at range/2 (odd
// range) or the mean of those at range/2 and range/2 + 1 (even range; a
// two-bin segment takes its largest power for the second), which is the
// reference's choice on its zero-padded 256-slot sort.
// ---------------------------------------------------------------------------
constexpr int PSR_WARPS_PER_BLOCK = 8;
constexpr int PSR_MAX_SEGMENT = 256;

template <int V>
__device__ float psr_segment_median(const float2 *__restrict__ spec, int start, int range, long long nSamples)
{
    const int lane = threadIdx.x & 31;
    float x[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
        const int e = 32 * v + lane;
        x[v] = INFINITY;
        if (e < range && start + e < nSamples) {
            const float2 q = spec[start + e];
            x[v] = psr_sq2<PSR_MEDIAN_POWER_FORM>(q.x, q.y);
        }
    }
#pragma unroll
    for (int size = 2; size <= 32 * V; size <<= 1) {
#pragma unroll
        for (int j = size >> 1; j > 0; j >>= 1) {
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int e = 32 * v + lane;
                const bool keep_min = ((e & j) == 0) == ((e & size) == 0);
                float other;
                if (j >= 32) {
                    const int pv = v ^ (j >> 5);
                    if (pv < v)
                        continue; // the pair (pv, v) was handled at pv
                    other = x[pv];
                    const float lo = fminf(x[v], other), hi = fmaxf(x[v], other);
                    x[v] = keep_min ? lo : hi;
                    x[pv] = keep_min ? hi : lo;
                } else {
                    other = __shfl_xor_sync(0xffffffffu, x[v], j);
                    x[v] = keep_min ? fminf(x[v], other) : fmaxf(x[v], other);
                }
            }
        }
    }
    auto rank = [&](int r) {
        float t = x[0];
#pragma unroll
        for (int v = 1; v < V; ++v)
            if ((r >> 5) == v)
                t = x[v];
        return __shfl_sync(0xffffffffu, t, r & 31);
    };
    const int mid = range >> 1;
    if (range & 1)
        return rank(mid);
    return (rank(mid) + rank(min(mid + 1, range - 1))) * 0.5f;
}

// segments of at most PSR_MAX_SEGMENT bins (psr_whitening checks the table)
__global__ void __launch_bounds__(32 * PSR_WARPS_PER_BLOCK) k_segment_medians_warp(float *medians,
                                                                                 const float2 *__restrict__ in,
                                                                                 const int *__restrict__ seg,
                                                                                 long long nSamples, int nSegments)
{
    const int m = blockIdx.x * PSR_WARPS_PER_BLOCK + (threadIdx.x >> 5);
    if (m >= nSegments - 1)
        return;
    const int start = seg[m], range = seg[m + 1] - start;
    const float2 *spec = in + static_cast<long long>(blockIdx.y) * nSamples;
    float med;
    if (range <= 32)
        med = psr_segment_median<1>(spec, start, range, nSamples);
    else if (range <= 64)
        med = psr_segment_median<2>(spec, start, range, nSamples);
    else if (range <= 128)
        med = psr_segment_median<4>(spec, start, range, nSamples);
    else
        med = psr_segment_median<8>(spec, start, range, nSamples);
    if ((threadIdx.x & 31) == 0)
        medians[static_cast<long long>(blockIdx.y) * nSegments + m] = med;
}

// ---------------------------------------------------------------------------
// SGP2 normalisation: one warp per interpolation span b of one spectrum.
// Span 0 scales the first half of segment 0 by 1/sqrt(its median / ln 2)
// and sets bin 0 to (1, 0); span b >= 1 covers the bins from the middle of
// segment b-1 to the middle of segment b, each scaled by 1/sqrt of the
// medians interpolated linearly at its offset i, in the reference's mixed
// float/double expressions.  The last span also scales the 256 bins after
// the last middle with the norms at offsets range - t (t = 0..255), as the
// reference's last block does with its 256 threads.  When an even segment
// meets an odd one, the span's last bin is the next span's first: only the
// next span scales it (the reference scales it in both, unordered).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float psr_scaled_median(float m) { return m * 1.44269504088896; }

__device__ __forceinline__ float psr_interp(float mean, float slope, int i)
{
#if PSR_INTERP_FORM == 1
    return fmaf(slope, (float)i, mean);
#elif PSR_INTERP_FORM == 2
    return __fadd_rn(mean, __fmul_rn(slope, (float)i));
#else
    return mean + slope * i;
#endif
}

__global__ void __launch_bounds__(32 * PSR_WARPS_PER_BLOCK) k_sgp2_spans(const float *__restrict__ medians, float2 *in,
                                                                       const int *__restrict__ seg,
                                                                       long long nSamples, int nSegments)
{
    const int b = blockIdx.x * PSR_WARPS_PER_BLOCK + (threadIdx.x >> 5);
    const int nspans = nSegments - 1;
    if (b >= nspans)
        return;
    const int lane = threadIdx.x & 31;
    const float *med = medians + static_cast<long long>(blockIdx.y) * nSegments;
    float2 *spec = in + static_cast<long long>(blockIdx.y) * nSamples;
    auto scale = [&](long long pos, float norm) {
        float2 q = spec[pos];
        q.x *= norm;
        q.y *= norm;
        spec[pos] = q;
    };
    if (b == 0) {
        const int current_range = seg[1] - seg[0];
        const float current_mean = psr_scaled_median(med[0]);
        const float norm = 1.0 / sqrt(current_mean);
        for (int t = lane; t < (current_range >> 1); t += 32)
            scale(t, norm);
        __syncwarp();
        if (lane == 0)
            spec[0] = make_float2(1.0f, 0.0f);
        return;
    }
    const int fm1_pos = seg[b - 1], f0_pos = seg[b], fp1_pos = seg[b + 1];
    const int previous_range = f0_pos - fm1_pos;
    const int current_range = fp1_pos - f0_pos;
    const float previous_mean = psr_scaled_median(med[b - 1]);
    const float current_mean = psr_scaled_median(med[b]);
    const int range = ((previous_range + current_range + 1) >> 1);
    const float slope = (current_mean - previous_mean) / ((float)range);
    const int first = fm1_pos + (previous_range >> 1);
    const bool shared_last = b + 1 < nspans && (previous_range & 1) == 0 && (current_range & 1) == 1;
    const int n = range - (shared_last ? 1 : 0);
    for (int i = lane; i < n; i += 32) {
        const int local_pos = first + i;
        if (local_pos < nSamples) {
            const float norm = 1.0 / sqrt(psr_interp(previous_mean, slope, i));
            scale(local_pos, norm);
        }
    }
    if (b == nspans - 1) {
        for (int t = lane; t < 256; t += 32) {
            const int tail = first + range + t;
            if (tail < nSamples) {
                const int i = range - t;
                const float norm = 1.0 / sqrt(psr_interp(previous_mean, slope, i));
                scale(tail, norm);
            }
        }
    }
}

} // namespace

long long psr_kernel_launches() { return g_psr_launches.load(); }

// src/aa_device_spectral_whitening.cu:17-31 (segment boundaries, a prefix sum)
std::vector<int> psr_segment_sizes(int min_segment_length, int max_segment_length, size_t nSamples)
{
    std::vector<int> s;
    s.push_back(0);
    int seg_length = min_segment_length;
    int seg_sum = 1 + seg_length;
    s.push_back(seg_sum);
    while (static_cast<size_t>(seg_sum + seg_length) < nSamples) {
        seg_sum = seg_sum + seg_length;
        seg_length = min_segment_length * std::log(seg_sum);
        if (seg_length > max_segment_length)
            seg_length = max_segment_length;
        s.push_back(seg_sum);
    }
    s.push_back(static_cast<int>(nSamples));
    return s;
}

// The boundary table of a spectrum length, copied to the device once per
// (device, length) and kept for the process.
namespace {
struct SegTable {
    int *d = nullptr;
    int n = 0;
};
std::mutex g_seg_mutex;
std::map<std::pair<int, size_t>, SegTable> g_seg_tables;
} // namespace

// src/aa_device_spectral_whitening.cu:60-118 with enable_median.  The
// medians live in a stream-ordered scratch allocation freed on the same
// stream; a boundary table not yet on the device is copied synchronously,
// which a capturing stream refuses (cudaErrorStreamCaptureUnsupported).
cudaError_t psr_whitening(float2 *d_spectra, size_t nSamples, int nDMs, cudaStream_t st)
{
    if (nDMs < 1 || nSamples < 8 || nSamples > static_cast<size_t>(INT32_MAX))
        return cudaErrorInvalidValue;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return e;
    SegTable tab;
    {
        std::lock_guard<std::mutex> lock(g_seg_mutex);
        auto it = g_seg_tables.find(std::make_pair(dev, nSamples));
        if (it != g_seg_tables.end()) {
            tab = it->second;
        } else {
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            e = cudaStreamIsCapturing(st, &cs);
            if (e != cudaSuccess)
                return e;
            if (cs != cudaStreamCaptureStatusNone)
                return cudaErrorStreamCaptureUnsupported;
            const std::vector<int> segments = psr_segment_sizes(6, 250, nSamples);
            for (size_t i = 0; i + 1 < segments.size(); ++i)
                if (segments[i + 1] - segments[i] > PSR_MAX_SEGMENT || segments[i + 1] <= segments[i])
                    return cudaErrorInvalidValue;
            tab.n = static_cast<int>(segments.size());
            e = cudaMalloc(reinterpret_cast<void **>(&tab.d), tab.n * sizeof(int));
            if (e == cudaSuccess)
                e = cudaMemcpy(tab.d, segments.data(), tab.n * sizeof(int), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) {
                cudaFree(tab.d);
                return e;
            }
            g_seg_tables[std::make_pair(dev, nSamples)] = tab;
        }
    }
    const int nSegments = tab.n;
    float *d_medians = nullptr;
    e = cudaMallocAsync(reinterpret_cast<void **>(&d_medians), static_cast<size_t>(nSegments) * nDMs * sizeof(float),
                        st);
    if (e != cudaSuccess)
        return e;
    const dim3 grid((nSegments - 1 + PSR_WARPS_PER_BLOCK - 1) / PSR_WARPS_PER_BLOCK, nDMs);
    {
        k_segment_medians_warp<<<grid, 32 * PSR_WARPS_PER_BLOCK, 0, st>>>(
            d_medians, d_spectra, tab.d, static_cast<long long>(nSamples), nSegments);
        ++g_psr_launches;
        // spans 0 .. nSegments-2: the reference launches one block more,
        // which reads the boundary past the table and the median slot its
        // median kernel never writes, and for any table value below
        // nSamples - (last segment) writes nothing
        k_sgp2_spans<<<grid, 32 * PSR_WARPS_PER_BLOCK, 0, st>>>(d_medians, d_spectra, tab.d,
                                                                static_cast<long long>(nSamples), nSegments);
        ++g_psr_launches;
        e = cudaGetLastError();
    }
    cudaFreeAsync(d_medians, st);
    return e;
}

// [secondary][primary] -> [primary][secondary] (corner_turn_SM,
// src/aa_corner_turn.cpp:78-107, which the simple harmonic sum's input
// goes through): 32 x 32 tiles through a padded shared array.
__global__ void k_transpose_f32(const float *__restrict__ in, float *__restrict__ out, long long primary,
                                long long secondary)
{
    __shared__ float tile[32][33];
    const long long x0 = static_cast<long long>(blockIdx.x) * 32, y0 = static_cast<long long>(blockIdx.y) * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5; // 256 threads: 8 rows per pass
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        const long long y = y0 + ty + k, x = x0 + tx;
        if (y < secondary && x < primary)
            tile[ty + k][tx] = in[y * primary + x];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        const long long x = x0 + ty + k, y = y0 + tx;
        if (x < primary && y < secondary)
            out[x * secondary + y] = tile[tx][ty + k];
    }
}

cudaError_t psr_transpose(const float *d_in, float *d_out, long long primary, long long secondary, cudaStream_t st)
{
    if (primary <= 0 || secondary <= 0)
        return cudaSuccess;
    const dim3 grid(static_cast<unsigned>((primary + 31) / 32), static_cast<unsigned>((secondary + 31) / 32));
    if (grid.y > 65535)
        return cudaErrorInvalidValue;
    k_transpose_f32<<<grid, 256, 0, st>>>(d_in, d_out, primary, secondary);
    ++g_psr_launches;
    return cudaGetLastError();
}

// The medians alone over a caller's boundary table (segments of 1 to
// PSR_MAX_SEGMENT bins, increasing, the last one at most nSamples): the
// whitening's first kernel on tables its own lengths never produce.  The
// table is copied synchronously into a scratch allocation.
cudaError_t psr_segment_medians(const float2 *d_spectra, size_t nSamples, int nDMs, const int *segments,
                                int nSegments, float *d_medians, cudaStream_t st)
{
    if (nDMs < 1 || nSegments < 2 || nSamples > static_cast<size_t>(INT32_MAX) || segments[0] < 0 ||
        static_cast<size_t>(segments[nSegments - 1]) > nSamples)
        return cudaErrorInvalidValue;
    for (int i = 0; i + 1 < nSegments; ++i)
        if (segments[i + 1] - segments[i] > PSR_MAX_SEGMENT || segments[i + 1] <= segments[i])
            return cudaErrorInvalidValue;
    int *d_seg = nullptr;
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(&d_seg), nSegments * sizeof(int));
    if (e != cudaSuccess)
        return e;
    e = cudaMemcpy(d_seg, segments, nSegments * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const dim3 grid((nSegments - 1 + PSR_WARPS_PER_BLOCK - 1) / PSR_WARPS_PER_BLOCK, nDMs);
        k_segment_medians_warp<<<grid, 32 * PSR_WARPS_PER_BLOCK, 0, st>>>(
            d_medians, d_spectra, d_seg, static_cast<long long>(nSamples), nSegments);
        ++g_psr_launches;
        e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(st);
    }
    cudaFree(d_seg);
    return e;
}

// src/aa_device_harmonic_summing.cu:38-169: which algorithm, the PRESTO
// count of powers of two; the scalloping-corrected plane is a stream-ordered
// scratch allocation freed on the same stream
cudaError_t psr_harmonic_sum(int algorithm, const float *d_input, float *d_snr, uint16_t *d_harmonics,
                             const float *d_msd, int nTimesamples, int nDMs, int nHarmonics, bool scalloping,
                             cudaStream_t st)
{
    if (nTimesamples < 1 || nDMs < 1 || nHarmonics < 1 || nHarmonics > PSR_MAX_HARMONICS || algorithm < 1 ||
        algorithm > 3)
        return cudaErrorInvalidValue;
    // PRESTO sums 1, 2, 4, ... harmonics: src/aa_device_harmonic_summing.cu:143
    const int factor = static_cast<int>(std::log(static_cast<double>(nHarmonics)) / std::log(2.0)) + 1;
    const float *src = d_input;
    float *d_cor = nullptr;
    cudaError_t e = cudaSuccess;
    if (scalloping) {
        e = cudaMallocAsync(reinterpret_cast<void **>(&d_cor),
                            static_cast<size_t>(nTimesamples) * static_cast<size_t>(nDMs) * sizeof(float), st);
        if (e != cudaSuccess)
            return e;
        k_scalloping_corrected<<<dim3((nTimesamples + PSR_COR_TILE - 1) / PSR_COR_TILE, nDMs), PSR_COR_TILE, 0, st>>>(
            d_input, d_cor, nTimesamples);
        ++g_psr_launches;
        src = d_cor;
    }
    const dim3 grid((nTimesamples + 255) / 256, nDMs);
    const int nh = (algorithm == 3) ? factor : nHarmonics;
    switch (algorithm) {
    case 1: k_harmonic_rows<1><<<grid, 256, 0, st>>>(src, d_snr, d_harmonics, d_msd, nTimesamples, nh, 2 * nHarmonics); break;
    case 2: k_harmonic_rows<2><<<grid, 256, 0, st>>>(src, d_snr, d_harmonics, d_msd, nTimesamples, nh, 2 * nHarmonics); break;
    default: k_harmonic_rows<3><<<grid, 256, 0, st>>>(src, d_snr, d_harmonics, d_msd, nTimesamples, nh, 2 * nHarmonics); break;
    }
    ++g_psr_launches;
    e = cudaGetLastError();
    if (d_cor)
        cudaFreeAsync(d_cor, st);
    return e;
}

// src/aa_device_threshold.cu:56-163 (transposed and normal planes)
cudaError_t psr_threshold(const float *d_snr, const uint16_t *d_harmonics, float *d_list, int nTimesamples, int nDMs,
                          float threshold, int max_peaks, int *d_count, const float *d_msd, int dm_shift, int in_bin,
                          bool transposed, bool greedy, cudaStream_t st)
{
    const int width = transposed ? nDMs : nTimesamples;
    const int height = transposed ? nTimesamples : nDMs;
    if (width < 1 || height < 1 || in_bin < 1)
        return cudaErrorInvalidValue;
    const dim3 grid((width + 255) / 256, height);
    k_psr_threshold<<<grid, 256, 0, st>>>(d_snr, d_harmonics, d_list, width, height, threshold, max_peaks, d_count,
                                          d_msd, dm_shift, in_bin, transposed ? 1 : 0, greedy ? 1 : 0);
    ++g_psr_launches;
    return cudaGetLastError();
}

// src/aa_device_peak_find.cu:53-131: transposed planes are [nTimesamples
// bins][nDMs] (DM trials inner), normal ones [nDMs][nTimesamples]
cudaError_t psr_peak_find(const float *d_snr, const uint16_t *d_harmonics, float *d_list, int nTimesamples, int nDMs,
                          float threshold, int max_peaks, int *d_count, const float *d_msd, int dm_shift, int in_bin,
                          bool transposed, bool greedy, cudaStream_t st)
{
    const int width = transposed ? nDMs : nTimesamples;
    const int height = transposed ? nTimesamples : nDMs;
    if (width < 2 || height < 2 || in_bin < 1)
        return cudaErrorInvalidValue;
    const dim3 block(32, 32);
    const dim3 grid((width + 31) / 32, (height + 31) / 32);
    k_psr_peaks<<<grid, block, 0, st>>>(d_snr, d_harmonics, d_list, width, height, threshold, max_peaks, d_count,
                                        d_msd, dm_shift, in_bin, transposed ? 1 : 0, greedy ? 1 : 0);
    ++g_psr_launches;
    return cudaGetLastError();
}

// src/aa_device_power.cu:34-52: norm = sqrt(nTimesamples) as float
cudaError_t psr_power_interbin(const float2 *d_in, float *d_power, float *d_interbin, int nTimesamples, int nDMs,
                               cudaStream_t st)
{
    const int half = nTimesamples >> 1;
    if (half < 1 || nDMs < 1)
        return cudaErrorInvalidValue;
    const int pairs = (half + 1) / 2;
    const dim3 grid((pairs + PSR_PAIR_THREADS - 1) / PSR_PAIR_THREADS, nDMs);
    const float norm = static_cast<float>(std::sqrt(static_cast<double>(nTimesamples)));
    const bool vec4 = (nTimesamples % 4) == 0 && (reinterpret_cast<uintptr_t>(d_interbin) & 15) == 0;
    if (vec4)
        k_power_pairs<true><<<grid, PSR_PAIR_THREADS, 0, st>>>(d_in, d_power, d_interbin, nTimesamples, norm);
    else
        k_power_pairs<false><<<grid, PSR_PAIR_THREADS, 0, st>>>(d_in, d_power, d_interbin, nTimesamples, norm);
    ++g_psr_launches;
    return cudaGetLastError();
}

// src/aa_device_harmonic_summing.cu:11-37
cudaError_t psr_harmonic_sum_simple(const float *d_in, float *d_snr, uint16_t *d_harmonics, const float *d_msd,
                                    int nBins, int nSpectra, int nHarmonics, cudaStream_t st)
{
    if (nBins < 1 || nSpectra < 1 || nHarmonics < 1 || nHarmonics > PSR_MAX_HARMONICS)
        return cudaErrorInvalidValue;
    const bool vec4 = (nSpectra % 4) == 0 && (reinterpret_cast<uintptr_t>(d_in) & 15) == 0;
    const int per = vec4 ? 4 : 1;
    const dim3 grid(nBins, (nSpectra / per + PSR_HS_THREADS - 1) / PSR_HS_THREADS);
    if (vec4)
        k_harmonic_columns<4><<<grid, PSR_HS_THREADS, 0, st>>>(d_in, d_snr, d_harmonics, d_msd, nBins, nSpectra,
                                                              nHarmonics);
    else
        k_harmonic_columns<1><<<grid, PSR_HS_THREADS, 0, st>>>(d_in, d_snr, d_harmonics, d_msd, nBins, nSpectra,
                                                              nHarmonics);
    ++g_psr_launches;
    return cudaGetLastError();
}

} // namespace aab200
