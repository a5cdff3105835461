// psr.cuh -- building blocks of the reference's periodicity search
// (src/aa_device_periods.cu:368-541): the power and interbin spectra of
// batched real-to-complex spectra, and the simple harmonic sum over
// corner-turned power spectra.  Each keeps the float expressions of the
// reference kernel it follows (cited per function), so the spectra and the
// harmonic S/N values are bit-identical to the reference's.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

namespace aab200 {

// in: nDMs spectra of nT/2+1 complex bins (cufftExecR2C output, row pitch
// nT/2+1); power [nDMs][nT/2] = |X_k / sqrt(nT)|^2 for 0 < k < nT/2 (0 at
// k = 0); interbin [nDMs][nT]: even entries the power, odd entries
// 0.616850275 |X_k - X_{k+1}|^2 (normalised).
cudaError_t psr_power_interbin(const float2 *d_in, float *d_power, float *d_interbin, int nTimesamples, int nDMs,
                               cudaStream_t st);

// in [nBins][nSpectra] (bins outer, spectra inner); for every bin b and
// spectrum s the best S/N of the sums of harmonics 0..f at bins b, 2b, ...,
// (f+1)b (below nBins), S/N_f = (sum - msd[2f]) / msd[2f+1], and the f of
// the best one.  d_msd: device (mean, deviation) per harmonic count.
cudaError_t psr_harmonic_sum_simple(const float *d_in, float *d_snr, uint16_t *d_harmonics, const float *d_msd,
                                    int nBins, int nSpectra, int nHarmonics, cudaStream_t st);

// Peaks of a harmonic-sum S/N plane (candidate records of 4 floats appended
// at *d_count): transposed planes [nTimesamples][nDMs], normal ones
// [nDMs][nTimesamples]; greedy: harmonic counts carry a multiple of 100 that
// the S/N conversion drops (normal planes only).
cudaError_t psr_peak_find(const float *d_snr, const uint16_t *d_harmonics, float *d_list, int nTimesamples, int nDMs,
                          float threshold, int max_peaks, int *d_count, const float *d_msd, int dm_shift, int in_bin,
                          bool transposed, bool greedy, cudaStream_t st);

// Every value of the plane above the cut, recorded as psr_peak_find does
cudaError_t psr_threshold(const float *d_snr, const uint16_t *d_harmonics, float *d_list, int nTimesamples, int nDMs,
                          float threshold, int max_peaks, int *d_count, const float *d_msd, int dm_shift, int in_bin,
                          bool transposed, bool greedy, cudaStream_t st);

// Harmonic sums over a normal plane [nDMs][nTimesamples]: algorithm 1
// greedy, 2 PRESTO plus, 3 PRESTO (sums of 1, 2, 4, ... harmonics up to
// nHarmonics); scalloping: the scalloping-loss correction of the bins.
cudaError_t psr_harmonic_sum(int algorithm, const float *d_input, float *d_snr, uint16_t *d_harmonics,
                             const float *d_msd, int nTimesamples, int nDMs, int nHarmonics, bool scalloping,
                             cudaStream_t st);

// Segment boundaries of the spectral whitening (a prefix sum from 0 to
// nSamples; segment lengths grow as min * ln(start), capped at max)
std::vector<int> psr_segment_sizes(int min_segment_length, int max_segment_length, size_t nSamples);

// Spectral whitening (SGP2 with medians) in place: per spectrum the
// median power of each segment, scaled by 1/ln 2, and every bin divided by
// the square root of the medians interpolated between segment middles;
// bin 0 set to (1, 0).  nSamples complex bins per spectrum (>= 8).
cudaError_t psr_whitening(float2 *d_spectra, size_t nSamples, int nDMs, cudaStream_t st);
cudaError_t psr_segment_medians(const float2 *d_spectra, size_t nSamples, int nDMs, const int *segments,
                                int nSegments, float *d_medians, cudaStream_t st);

// [secondary][primary] -> [primary][secondary]
cudaError_t psr_transpose(const float *d_in, float *d_out, long long primary, long long secondary, cudaStream_t st);

long long psr_kernel_launches();

} // namespace aab200
