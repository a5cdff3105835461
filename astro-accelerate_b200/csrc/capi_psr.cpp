// capi_psr.cpp -- extern "C" entry points of the periodicity building blocks
// (aa_b200_psr_*, declared in include/aa_b200.h).
#include "aa_b200.h"

#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "psr.cuh"

using namespace aab200;

namespace {
thread_local std::string g_psr_error;

int psr_status(cudaError_t e, const char *what)
{
    if (e == cudaSuccess)
        return 0;
    g_psr_error = std::string(what) + ": " + cudaGetErrorString(e);
    return 1;
}
} // namespace

extern "C" {

int aa_b200_psr_power_interbin(const void *d_spectra, float *d_power, float *d_interbin, int nTimesamples, int nDMs,
                               void *stream)
{
    return psr_status(psr_power_interbin(static_cast<const float2 *>(d_spectra), d_power, d_interbin, nTimesamples,
                                         nDMs, static_cast<cudaStream_t>(stream)),
                      "power and interbin spectra");
}

int aa_b200_psr_harmonic_sum_simple(const float *d_input, float *d_snr, unsigned short *d_harmonics,
                                    const float *d_msd, int nBins, int nSpectra, int nHarmonics, void *stream)
{
    return psr_status(psr_harmonic_sum_simple(d_input, d_snr, d_harmonics, d_msd, nBins, nSpectra, nHarmonics,
                                              static_cast<cudaStream_t>(stream)),
                      "harmonic sum");
}

int aa_b200_psr_peak_find(const float *d_snr, const unsigned short *d_harmonics, float *d_list, int nTimesamples,
                          int nDMs, float threshold, int max_peaks, int *d_count, const float *d_msd, int dm_shift,
                          int in_bin, int transposed, int greedy, void *stream)
{
    return psr_status(psr_peak_find(d_snr, d_harmonics, d_list, nTimesamples, nDMs, threshold, max_peaks, d_count,
                                    d_msd, dm_shift, in_bin, transposed != 0, greedy != 0,
                                    static_cast<cudaStream_t>(stream)),
                      "periodicity peak finding");
}

int aa_b200_psr_threshold(const float *d_snr, const unsigned short *d_harmonics, float *d_list, int nTimesamples,
                          int nDMs, float threshold, int max_peaks, int *d_count, const float *d_msd, int dm_shift,
                          int in_bin, int transposed, int greedy, void *stream)
{
    return psr_status(psr_threshold(d_snr, d_harmonics, d_list, nTimesamples, nDMs, threshold, max_peaks, d_count,
                                    d_msd, dm_shift, in_bin, transposed != 0, greedy != 0,
                                    static_cast<cudaStream_t>(stream)),
                      "periodicity thresholding");
}

int aa_b200_psr_harmonic_sum(int algorithm, const float *d_input, float *d_snr, unsigned short *d_harmonics,
                             const float *d_msd, int nTimesamples, int nDMs, int nHarmonics, int scalloping,
                             void *stream)
{
    return psr_status(psr_harmonic_sum(algorithm, d_input, d_snr, d_harmonics, d_msd, nTimesamples, nDMs, nHarmonics,
                                       scalloping != 0, static_cast<cudaStream_t>(stream)),
                      "harmonic sum");
}

int aa_b200_psr_whitening(void *d_spectra, size_t nSamples, int nDMs, void *stream)
{
    if (!d_spectra || nDMs < 1 || nSamples < 8) {
        g_psr_error = "spectral whitening: a spectrum of at least 8 bins needed";
        return 1;
    }
    return psr_status(psr_whitening(static_cast<float2 *>(d_spectra), nSamples, nDMs,
                                    static_cast<cudaStream_t>(stream)),
                      "spectral whitening");
}

int aa_b200_psr_segment_medians(const void *d_spectra, size_t nSamples, int nDMs, const int *segments,
                                int nSegments, float *d_medians, void *stream)
{
    if (!d_spectra || !segments || !d_medians) {
        g_psr_error = "segment medians: null pointer";
        return 1;
    }
    return psr_status(psr_segment_medians(static_cast<const float2 *>(d_spectra), nSamples, nDMs, segments,
                                          nSegments, d_medians, static_cast<cudaStream_t>(stream)),
                      "segment medians");
}

int aa_b200_psr_segment_sizes(size_t nSamples, int *out, int cap)
{
    const std::vector<int> s = psr_segment_sizes(6, 250, nSamples);
    for (int i = 0; out && i < cap && i < static_cast<int>(s.size()); ++i)
        out[i] = s[i];
    return static_cast<int>(s.size());
}

long long aa_b200_psr_kernel_launches(void) { return psr_kernel_launches(); }

const char *aa_b200_psr_last_error(void) { return g_psr_error.c_str(); }

} // extern "C"
