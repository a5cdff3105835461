// psr.cu -- periodicity building blocks (see psr.cuh).
#include "psr.cuh"

#include <atomic>
#include <cmath>
#include <vector>

namespace aab200 {

namespace {

std::atomic<long long> g_psr_launches{0};

constexpr int PSR_PAI_THREADS = 512; // PAI_NTHREADS
constexpr int PSR_PHS_THREADS = 64;  // PHS_NTHREADS

// src/aa_device_power_kernel.cu:19-41
__global__ void __launch_bounds__(PSR_PAI_THREADS) k_power_interbin(const float2 *__restrict__ in, float *power,
                                                                    float *interbin, int nT, float norm)
{
    const int pos_x = blockIdx.x * blockDim.x + threadIdx.x;
    const long long pos_y = static_cast<long long>(blockIdx.y) * ((nT >> 1) + 1);
    float2 A, B;
    A.x = 0;
    A.y = 0;
    B.x = 0;
    B.y = 0;
    if ((pos_x < (nT >> 1)) && (pos_x > 0)) {
        A = in[pos_y + pos_x];
        B = in[pos_y + pos_x + 1];
        A.x = A.x / norm;
        A.y = A.y / norm;
        B.x = B.x / norm;
        B.y = B.y / norm;
    }
    if (pos_x < (nT >> 1)) {
        const long long row = blockIdx.y;
        power[row * (nT >> 1) + pos_x] = A.x * A.x + A.y * A.y;
        interbin[row * nT + 2 * pos_x] = A.x * A.x + A.y * A.y;
        interbin[row * nT + 2 * pos_x + 1] = 0.616850275f * ((A.x - B.x) * (A.x - B.x) + (A.y - B.y) * (A.y - B.y));
    }
}

// src/aa_device_harmonic_summing_kernel.cu:8-39
__global__ void __launch_bounds__(PSR_PHS_THREADS) k_harmonic_sum_simple(const float *__restrict__ in, float *snr_out,
                                                                         uint16_t *harm_out,
                                                                         const float *__restrict__ msd, int nBins,
                                                                         int nSpectra, int nHarmonics)
{
    const int s = blockIdx.y * blockDim.x + threadIdx.x;
    if (s >= nSpectra)
        return;
    const long long b = blockIdx.x;
    float HS_value = __ldg(in + b * nSpectra + s);
    float SNR = (HS_value - __ldg(msd)) / (__ldg(msd + 1));
    uint16_t best = 0;
    if (b > 0) {
        for (int f = 1; f < nHarmonics; f++) {
            const long long bin = b + f * b;
            if (bin < nBins) {
                HS_value = HS_value + __ldg(in + bin * nSpectra + s);
                const float temp_SNR = (HS_value - __ldg(msd + 2 * f)) / (__ldg(msd + 2 * f + 1));
                if (temp_SNR > SNR) {
                    SNR = temp_SNR;
                    best = static_cast<uint16_t>(f);
                }
            }
        }
    }
    snr_out[b * nSpectra + s] = SNR;
    harm_out[b * nSpectra + s] = best;
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

// Harmonic sums over normal planes [nDMs][nTimesamples]
// (src/aa_device_harmonic_summing_kernel.cu:41-268).  Each output bin is
// independent; the expressions (float sums, the double constants and bin
// positions of the scalloping-loss and PRESTO forms, the fast division) are
// the reference's.
__device__ __forceinline__ float psr_remove_scalloping_loss(float Xm2, float Xm1, float X0, float Xp1, float Xp2)
{
    return (X0 + (1.88494 / 2.0) * (Xm1 + Xp1) + (0.88494 / 2.0) * (Xm2 + Xp2));
}

template <bool SCAL>
__device__ __forceinline__ void psr_bins(float *down, float *step, const float *__restrict__ d, long long pos)
{
    if (SCAL) {
        const float Xm2 = d[pos - 2], Xm1 = d[pos - 1], X0 = d[pos + 0], Xp1 = d[pos + 1], Xp2 = d[pos + 2],
                    Xp3 = d[pos + 3];
        *down = psr_remove_scalloping_loss(Xm2, Xm1, X0, Xp1, Xp2);
        *step = psr_remove_scalloping_loss(Xm1, X0, Xp1, Xp2, Xp3);
    } else {
        *down = d[pos];
        *step = d[pos + 1];
    }
}

template <bool SCAL>
__device__ __forceinline__ void psr_bin_value(float *bin, const float *__restrict__ d, long long pos)
{
    if (SCAL) {
        const float Xm2 = d[pos - 2], Xm1 = d[pos - 1], X0 = d[pos], Xp1 = d[pos + 1], Xp2 = d[pos + 2];
        *bin = X0 + (1.88494 / 2.0) * (Xm1 + Xp1) + (0.88494 / 2.0) * (Xm2 + Xp2);
    } else {
        *bin = d[pos];
    }
}

// greedy: at every harmonic the larger of two neighbouring bins, the chosen
// offsets carried to the next harmonic; the harmonic count plus 100 times
// the offsets at the best S/N
template <bool SCAL>
__global__ void k_hs_greedy(float *snr_out, uint16_t *harm_out, const float *__restrict__ d, const float *msd,
                            int nT, int nH)
{
    const int pos0 = blockIdx.x * blockDim.x + threadIdx.x;
    const long long row = static_cast<long long>(blockIdx.y) * nT;
    float SNR, partial_sum, maxSNR;
    unsigned short maxHarmonics, maxdata_shift = 0;
    int data_shift = 0;
    float data_down = 0, data_step = 0;
    if (pos0 > 1 && pos0 + 3 < nT)
        psr_bins<SCAL>(&data_down, &data_step, d, row + pos0);
    if (data_step > data_down) {
        data_shift++;
        partial_sum = data_step;
    } else {
        partial_sum = data_down;
    }
    maxSNR = fdividef((partial_sum - msd[0]), msd[1]);
    maxHarmonics = 0;
    for (int h = 1; h < nH; h++) {
        const int pos = (h + 1) * pos0 + data_shift;
        float dd = 0, ds = 0;
        if (pos > 1 && pos + 3 < nT)
            psr_bins<SCAL>(&dd, &ds, d, row + pos);
        if (ds > dd) {
            data_shift++;
            partial_sum = partial_sum + ds;
        } else {
            partial_sum = partial_sum + dd;
        }
        SNR = fdividef((partial_sum - msd[2 * h]), msd[2 * h + 1]);
        if (SNR > maxSNR) {
            maxSNR = SNR;
            maxHarmonics = h;
            maxdata_shift = data_shift;
        }
    }
    if (pos0 < nT) {
        snr_out[row + pos0] = maxSNR;
        harm_out[row + pos0] = static_cast<uint16_t>(maxHarmonics + maxdata_shift * 100);
    }
}

// PRESTO plus: harmonic i+1 sums the bins round(f * pos / (i + 1)), f = 1..i,
// onto the fundamental; the reported count is i - 1, as in the reference
template <bool SCAL>
__global__ void k_hs_presto_plus(float *snr_out, uint16_t *harm_out, const float *__restrict__ d, const float *msd,
                                 int nT, int nH)
{
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    const long long row = static_cast<long long>(blockIdx.y) * nT;
    float SNR, partial_sum, maxSNR, frequency_bin, fundamental = 0;
    int maxHarmonics;
    if ((pos > 1) && (pos + 2) < nT)
        psr_bin_value<SCAL>(&fundamental, d, row + pos);
    partial_sum = fundamental;
    maxSNR = fdividef((partial_sum - msd[0]), msd[1]);
    maxHarmonics = 0;
    if (pos > 1 && (pos + 2) < nT) {
        for (int i = 1; i < nH; i++) {
            partial_sum = fundamental;
            const double fundamental_fraction = ((double)pos) / ((double)(i + 1));
            for (int f = 1; f <= i; f++) {
                const int new_pos = (int)((((double)f) * fundamental_fraction) + 0.5);
                frequency_bin = 0;
                if (new_pos > 1 && (new_pos + 2) < nT)
                    psr_bin_value<SCAL>(&frequency_bin, d, row + new_pos);
                partial_sum = partial_sum + frequency_bin;
            }
            SNR = fdividef((partial_sum - msd[2 * i]), msd[2 * i + 1]);
            if (SNR > maxSNR) {
                maxSNR = SNR;
                maxHarmonics = i - 1;
            }
        }
    }
    if (pos < nT) {
        snr_out[row + pos] = maxSNR;
        harm_out[row + pos] = static_cast<uint16_t>(maxHarmonics);
    }
}

// PRESTO: sums of 1, 2, 4, ... 2^(factor-1) harmonics (factor =
// floor(log2(nHarmonics)) + 1), the even multiples of a fundamental at
// round(pos / harm)
template <bool SCAL>
__global__ void k_hs_presto(float *snr_out, uint16_t *harm_out, const float *__restrict__ d, const float *msd, int nT,
                            int nHarmonicsFactor)
{
    const int pos = blockIdx.x * blockDim.x + threadIdx.x;
    const long long row = static_cast<long long>(blockIdx.y) * nT;
    float SNR, partial_sum, maxSNR = -10000, frequency_bin, fundamental;
    int maxHarmonics = 0;
    for (int i = 0; i < nHarmonicsFactor; i++) {
        const int harm = (1 << i);
        const float fundamental_frac = ((double)pos) * (1.0 / ((double)harm));
        const int fundamental_pos = (int)(fundamental_frac + 0.5);
        fundamental = 0;
        if (fundamental_pos > 1 && (fundamental_pos + 2) < nT)
            psr_bin_value<SCAL>(&fundamental, d, row + fundamental_pos);
        partial_sum = fundamental;
        for (int f = 2; f <= harm; f = f + 2) {
            const int new_pos = (int)(((float)f) * fundamental_frac + 0.5);
            frequency_bin = 0;
            if (new_pos > 1 && (new_pos + 2) < nT)
                psr_bin_value<SCAL>(&frequency_bin, d, row + new_pos);
            partial_sum = partial_sum + frequency_bin;
        }
        SNR = fdividef((partial_sum - msd[2 * (harm / 2)]), msd[2 * (harm / 2) + 1]);
        if (SNR > maxSNR) {
            maxSNR = SNR;
            maxHarmonics = harm - 1;
        }
    }
    if (pos < nT) {
        snr_out[row + pos] = maxSNR;
        harm_out[row + pos] = static_cast<uint16_t>(maxHarmonics);
    }
}

// Spectral whitening, segment medians
// (src/aa_device_spectral_whitening_kernel.cu:338-376): the median of the
// powers |X|^2 of one segment (at most 256 bins), sorted in shared memory
// with zeros padding the 256 slots; an even count averages the sorted
// values at count/2 and count/2 + 1, as the reference does.
constexpr int PSR_SEG_SLOTS = 256;

__global__ void __launch_bounds__(PSR_SEG_SLOTS / 2) k_segment_medians(float *medians, const float2 *__restrict__ in,
                                                                         const int *__restrict__ seg, long long nSamples,
                                                                         int nSegments)
{
    __shared__ float v[PSR_SEG_SLOTS];
    const int t = threadIdx.x;
    const int start = seg[blockIdx.x], end = seg[blockIdx.x + 1];
    const int range = end - start;
    // Powers are >= 0 and the pads are zeros, so the sorted slots hold the
    // pads first and slot pads + k is the k-th smallest power for any pad
    // count: the smallest power of two (64 .. 256) above the segment sorts
    // to the same median as the reference's 256 slots.
    const int slots = range <= 64 ? 64 : (range <= 128 ? 128 : PSR_SEG_SLOTS);
    const long long row = static_cast<long long>(blockIdx.y) * nSamples;
    for (int k = t; k < slots; k += blockDim.x) {
        float p = 0;
        const long long pos = start + k;
        if (k < range && pos < nSamples) {
            const float2 value = in[row + pos];
            p = value.x * value.x + value.y * value.y;
        }
        v[k] = p;
    }
    __syncthreads();
    // bitonic sort, ascending (slots is block-uniform)
    for (int size = 2; size <= slots; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int k = t; k < slots / 2; k += blockDim.x) {
                const int lo = 2 * k - (k & (stride - 1));
                const int hi = lo + stride;
                const bool ascending = (lo & size) == 0;
                const float a = v[lo], b = v[hi];
                if ((a > b) == ascending) {
                    v[lo] = b;
                    v[hi] = a;
                }
            }
            __syncthreads();
        }
    }
    if (t == 0) {
        const int nZeros = slots - range;
        const int median_pos = nZeros + (range >> 1);
        float median;
        if ((range & 1) == 0)
            // a segment of two bins puts median_pos + 1 past the slots
            // (the reference reads past its shared array there): the
            // largest slot stands in
            median = (v[median_pos] + v[min(median_pos + 1, slots - 1)]) * 0.5f;
        else
            median = v[median_pos];
        medians[static_cast<long long>(blockIdx.y) * nSegments + blockIdx.x] = median;
    }
}

// Spectral whitening (src/aa_device_spectral_whitening_kernel.cu:378-427):
// the first half segment divided by the square root of its median (scaled
// by 1/ln 2), bin 0 set to 1; later bins by a linear interpolation of the
// scaled medians between segment middles, in the reference's mixed
// float/double expressions.  Block b (b >= 1) covers the bins from the
// middle of segment b-1 to the middle of segment b; the last block also the
// bins after the middle of the last segment, with the norms of its threads
// (interpolation indices range - t, as the reference computes them).
__global__ void k_whitening_sgp2(const float *__restrict__ medians, float2 *in, const int *__restrict__ seg,
                                 long long nSamples, int nSegments)
{
    const long long rowm = static_cast<long long>(blockIdx.y) * nSegments;
    if (blockIdx.x == 0) {
        const int f0_pos = seg[0];
        const int fp1_pos = seg[1];
        const int current_range = fp1_pos - f0_pos;
        const float current_mean = medians[rowm + blockIdx.x] * 1.44269504088896;
        const float norm = 1.0 / sqrt(current_mean);
        const long long global_pos = static_cast<long long>(blockIdx.y) * nSamples + threadIdx.x;
        if (static_cast<int>(threadIdx.x) < (current_range >> 1)) {
            in[global_pos].x *= norm;
            in[global_pos].y *= norm;
        }
        if (threadIdx.x == 0) {
            in[global_pos].x = 1.0;
            in[global_pos].y = 0.0;
        }
    } else {
        const int fm1_pos = seg[blockIdx.x - 1];
        const int f0_pos = seg[blockIdx.x + 0];
        const int fp1_pos = seg[blockIdx.x + 1];
        const int previous_range = f0_pos - fm1_pos;
        const int current_range = fp1_pos - f0_pos;
        const float previous_mean = medians[rowm + blockIdx.x - 1] * 1.44269504088896;
        const float current_mean = medians[rowm + blockIdx.x] * 1.44269504088896;
        const int range = ((previous_range + current_range + 1) >> 1);
        const int i = range - threadIdx.x;
        const float slope = (current_mean - previous_mean) / ((float)range);
        const float norm = 1.0 / sqrt(previous_mean + slope * i);
        const int local_pos = fm1_pos + (previous_range >> 1) + i;
        // an even previous and an odd current segment make this block's
        // last bin the next block's first (the middle of the current
        // segment); the reference scales it in both blocks without
        // ordering, here only the next block scales it, once
        const bool shared_last = blockIdx.x + 1 < gridDim.x && (previous_range & 1) == 0 && (current_range & 1) == 1;
        if (i >= 0 && i < range - (shared_last ? 1 : 0) && local_pos < nSamples) {
            const long long global_pos = static_cast<long long>(blockIdx.y) * nSamples + local_pos;
            in[global_pos].x *= norm;
            in[global_pos].y *= norm;
        }
        if (blockIdx.x == (gridDim.x - 1)) {
            const int tail = fm1_pos + (previous_range >> 1) + range + threadIdx.x;
            if (tail < nSamples) {
                const long long global_pos = static_cast<long long>(blockIdx.y) * nSamples + tail;
                in[global_pos].x *= norm;
                in[global_pos].y *= norm;
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

// src/aa_device_spectral_whitening.cu:60-118 with enable_median: the
// boundary table and the nDMs x nSegments medians live in stream-ordered
// allocations freed on the same stream.
cudaError_t psr_whitening(float2 *d_spectra, size_t nSamples, int nDMs, cudaStream_t st)
{
    if (nDMs < 1 || nSamples < 8 || nSamples > static_cast<size_t>(INT32_MAX))
        return cudaErrorInvalidValue;
    const std::vector<int> segments = psr_segment_sizes(6, 250, nSamples);
    const int nSegments = static_cast<int>(segments.size());
    int *d_seg = nullptr;
    float *d_medians = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&d_seg), nSegments * sizeof(int), st);
    if (e != cudaSuccess)
        return e;
    e = cudaMallocAsync(reinterpret_cast<void **>(&d_medians), static_cast<size_t>(nSegments) * nDMs * sizeof(float),
                        st);
    if (e == cudaSuccess)
        // pageable source: the call returns once the table is staged
        e = cudaMemcpyAsync(d_seg, segments.data(), nSegments * sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        k_segment_medians<<<dim3(nSegments - 1, nDMs), PSR_SEG_SLOTS / 2, 0, st>>>(
            d_medians, d_spectra, d_seg, static_cast<long long>(nSamples), nSegments);
        ++g_psr_launches;
        // blocks 0 .. nSegments-2: the reference launches one block more,
        // which reads the boundary past the table and the median slot its
        // median kernel never writes, and for any table value below
        // nSamples - (last segment) writes nothing
        k_whitening_sgp2<<<dim3(nSegments - 1, nDMs), 256, 0, st>>>(d_medians, d_spectra, d_seg,
                                                                   static_cast<long long>(nSamples), nSegments);
        ++g_psr_launches;
        e = cudaGetLastError();
    }
    if (d_medians)
        cudaFreeAsync(d_medians, st);
    cudaFreeAsync(d_seg, st);
    return e;
}

// src/aa_device_harmonic_summing.cu:38-169
cudaError_t psr_harmonic_sum(int algorithm, const float *d_input, float *d_snr, uint16_t *d_harmonics,
                             const float *d_msd, int nTimesamples, int nDMs, int nHarmonics, bool scalloping,
                             cudaStream_t st)
{
    if (nTimesamples < 1 || nDMs < 1 || nHarmonics < 1 || nHarmonics > 32)
        return cudaErrorInvalidValue;
    // PRESTO sums 1, 2, 4, ... harmonics: src/aa_device_harmonic_summing.cu:143
    const int factor = static_cast<int>(std::log(static_cast<double>(nHarmonics)) / std::log(2.0)) + 1;
    const dim3 grid((nTimesamples + 255) / 256, nDMs);
    switch (algorithm * 2 + (scalloping ? 1 : 0)) {
    case 2: k_hs_greedy<false><<<grid, 256, 0, st>>>(d_snr, d_harmonics, d_input, d_msd, nTimesamples, nHarmonics); break;
    case 3: k_hs_greedy<true><<<grid, 256, 0, st>>>(d_snr, d_harmonics, d_input, d_msd, nTimesamples, nHarmonics); break;
    case 4: k_hs_presto_plus<false><<<grid, 256, 0, st>>>(d_snr, d_harmonics, d_input, d_msd, nTimesamples, nHarmonics); break;
    case 5: k_hs_presto_plus<true><<<grid, 256, 0, st>>>(d_snr, d_harmonics, d_input, d_msd, nTimesamples, nHarmonics); break;
    case 6: k_hs_presto<false><<<grid, 256, 0, st>>>(d_snr, d_harmonics, d_input, d_msd, nTimesamples, factor); break;
    case 7: k_hs_presto<true><<<grid, 256, 0, st>>>(d_snr, d_harmonics, d_input, d_msd, nTimesamples, factor); break;
    default: return cudaErrorInvalidValue;
    }
    ++g_psr_launches;
    return cudaGetLastError();
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
    const dim3 grid((half + PSR_PAI_THREADS - 1) / PSR_PAI_THREADS, nDMs);
    const float norm = static_cast<float>(std::sqrt(static_cast<double>(nTimesamples)));
    k_power_interbin<<<grid, PSR_PAI_THREADS, 0, st>>>(d_in, d_power, d_interbin, nTimesamples, norm);
    ++g_psr_launches;
    return cudaGetLastError();
}

// src/aa_device_harmonic_summing.cu:11-37
cudaError_t psr_harmonic_sum_simple(const float *d_in, float *d_snr, uint16_t *d_harmonics, const float *d_msd,
                                    int nBins, int nSpectra, int nHarmonics, cudaStream_t st)
{
    if (nBins < 1 || nSpectra < 1 || nHarmonics < 1)
        return cudaErrorInvalidValue;
    const dim3 grid(nBins, (nSpectra + PSR_PHS_THREADS - 1) / PSR_PHS_THREADS);
    k_harmonic_sum_simple<<<grid, PSR_PHS_THREADS, 0, st>>>(d_in, d_snr, d_harmonics, d_msd, nBins, nSpectra,
                                                            nHarmonics);
    ++g_psr_launches;
    return cudaGetLastError();
}

} // namespace aab200
