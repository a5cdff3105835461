// sps.cu -- single-pulse search on the DM-time output: per-row noise
// statistics and per-block boxcar S/N peaks (the consumer the reference runs
// after dedispersion, src/aa_device_analysis.cu:130-510, here in a reduced
// form: white-noise S/N with the row's mean and standard deviation, boxcar
// widths given by the caller, one peak per (DM row, time block)).
//
//   snr_w(t) = (sum_{k<w} y[t+k] - w mean) / (std sqrt(w)),  t + w <= nsamp
// The peak of a block is the largest snr_w(t) over the block's t and all
// widths; ties keep the smallest t, then the smallest width.
#include <cstdint>

#include <cuda_runtime.h>

#include "frac.cuh"
#include "sps.cuh"

namespace aab200 {

namespace {

constexpr int ST = 256;

// mean and standard deviation of every row, FP64 sums
__global__ void __launch_bounds__(ST) k_row_stats(const float *__restrict__ y, long long pitch, long long nsamp,
                                                  float *__restrict__ mean, float *__restrict__ stdev)
{
    __shared__ double s1[ST / 32], s2[ST / 32];
    const float *row = y + static_cast<long long>(blockIdx.x) * pitch;
    double a = 0.0, b = 0.0;
    for (long long t = threadIdx.x; t < nsamp; t += ST) {
        const double v = __ldg(row + t);
        a += v;
        b += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) {
        s1[threadIdx.x >> 5] = a;
        s2[threadIdx.x >> 5] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double A = 0.0, B = 0.0;
        for (int k = 0; k < ST / 32; ++k) {
            A += s1[k];
            B += s2[k];
        }
        const double m = A / static_cast<double>(nsamp);
        const double var = B / static_cast<double>(nsamp) - m * m;
        mean[blockIdx.x] = static_cast<float>(m);
        stdev[blockIdx.x] = static_cast<float>(var > 0.0 ? sqrt(var) : 0.0);
    }
}

// one CTA per (block of SPS_BLOCK samples, row)
__global__ void __launch_bounds__(ST) k_block_peaks(const float *__restrict__ y, long long pitch, long long nsamp,
                                                    const float *__restrict__ mean, const float *__restrict__ stdev,
                                                    BoxcarWidths W, int nblocks, float *__restrict__ peak_snr,
                                                    int *__restrict__ peak_t, int *__restrict__ peak_w)
{
    extern __shared__ float ys[]; // SPS_BLOCK + wmax - 1 samples
    __shared__ float bs[ST];
    __shared__ int bt[ST], bw[ST];
    const int dm = blockIdx.y;
    const long long t0 = static_cast<long long>(blockIdx.x) * SPS_BLOCK;
    const int wmax = W.w[W.n - 1];
    const float *row = y + static_cast<long long>(dm) * pitch;
    for (int k = threadIdx.x; k < SPS_BLOCK + wmax - 1; k += ST) {
        const long long t = t0 + k;
        ys[k] = (t < nsamp) ? __ldg(row + t) : 0.f;
    }
    __syncthreads();
    const float m = mean[dm], sd = stdev[dm];
    float best = -3.0e38f;
    int best_t = -1, best_w = 0;
    if (sd > 0.f) {
        for (int k0 = threadIdx.x; k0 < SPS_BLOCK; k0 += ST) {
            const long long t = t0 + k0;
            float s = 0.f;
            int k = 0;
            for (int i = 0; i < W.n; ++i) {
                for (; k < W.w[i]; ++k)
                    s += ys[k0 + k];
                if (t + W.w[i] > nsamp)
                    break;
                const float wf = static_cast<float>(W.w[i]);
                const float v = (s - wf * m) / (sd * sqrtf(wf));
                if (v > best) {
                    best = v;
                    best_t = static_cast<int>(t);
                    best_w = W.w[i];
                }
            }
        }
    }
    bs[threadIdx.x] = best;
    bt[threadIdx.x] = best_t;
    bw[threadIdx.x] = best_w;
    __syncthreads();
    for (int h = ST / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            const int o = threadIdx.x + h;
            const bool take = bs[o] > bs[threadIdx.x] ||
                              (bs[o] == bs[threadIdx.x] && bt[o] >= 0 &&
                               (bt[threadIdx.x] < 0 || bt[o] < bt[threadIdx.x] ||
                                (bt[o] == bt[threadIdx.x] && bw[o] < bw[threadIdx.x])));
            if (take) {
                bs[threadIdx.x] = bs[o];
                bt[threadIdx.x] = bt[o];
                bw[threadIdx.x] = bw[o];
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const size_t i = static_cast<size_t>(dm) * nblocks + blockIdx.x;
        peak_snr[i] = bs[0];
        peak_t[i] = bt[0];
        peak_w[i] = bw[0];
    }
}

} // namespace

cudaError_t launch_row_stats(const float *y, int nrows, long long pitch, long long nsamp, float *mean, float *stdev,
                             cudaStream_t st)
{
    if (nrows <= 0 || nsamp <= 0 || pitch < nsamp)
        return cudaErrorInvalidValue;
    k_row_stats<<<nrows, ST, 0, st>>>(y, pitch, nsamp, mean, stdev);
    return cudaGetLastError();
}

cudaError_t launch_block_peaks(const float *y, int nrows, long long pitch, long long nsamp, const float *mean,
                               const float *stdev, const BoxcarWidths &W, float *peak_snr, int *peak_t, int *peak_w,
                               cudaStream_t st)
{
    if (nrows <= 0 || nrows > 65535 || nsamp <= 0 || pitch < nsamp || nsamp > 0x7fffffffLL || W.n < 1 ||
        W.n > kMaxBoxcarWidths)
        return cudaErrorInvalidValue;
    for (int i = 0; i < W.n; ++i)
        if (W.w[i] < 1 || W.w[i] > 1024 || (i > 0 && W.w[i] <= W.w[i - 1]))
            return cudaErrorInvalidValue;
    const int nblocks = static_cast<int>((nsamp + SPS_BLOCK - 1) / SPS_BLOCK);
    const size_t smem = static_cast<size_t>(SPS_BLOCK + W.w[W.n - 1] - 1) * sizeof(float);
    k_block_peaks<<<dim3(nblocks, nrows), ST, smem, st>>>(y, pitch, nsamp, mean, stdev, W, nblocks, peak_snr, peak_t,
                                                          peak_w);
    return cudaGetLastError();
}

} // namespace aab200
