// sps.cuh -- launchers of the single-pulse search kernels (sps.cu).
#pragma once
#include <cuda_runtime.h>

#include "frac.cuh"

namespace aab200 {

constexpr int SPS_BLOCK = 1024; // samples per peak block

// mean[r], stdev[r] of rows y[r][0, nsamp) (row pitch in floats)
cudaError_t launch_row_stats(const float *y, int nrows, long long pitch, long long nsamp, float *mean, float *stdev,
                             cudaStream_t st);
// peak S/N, its start sample and width per (row, block of SPS_BLOCK samples):
// arrays of nrows * ceil(nsamp / SPS_BLOCK)
cudaError_t launch_block_peaks(const float *y, int nrows, long long pitch, long long nsamp, const float *mean,
                               const float *stdev, const BoxcarWidths &W, float *peak_snr, int *peak_t, int *peak_w,
                               cudaStream_t st);

} // namespace aab200
