// preproc.cuh -- the reference runner's optional input and output processing
// around dedispersion (include/aa_permitted_pipelines_generic.hpp:525-560,
// :704-760, :821-831), each with the reference's float arithmetic and
// summation order so that results are bit-identical:
//   zero DM                 per time sample, subtract the channel mean and add
//                           the bandpass normalisation (src/aa_zero_dm.cpp:26-33,
//                           src/aa_device_zero_dm_kernel.cu:38-96)
//   zero DM with outliers   the same with a 3-sigma clipped mean
//                           (src/aa_zero_dm_outliers.cpp:38-57,
//                           src/aa_device_zero_dm_outliers_kernel.cu:12-231)
//   input normalisation     per channel, subtract mean - (2^nbits - 1)/2 over
//                           the chunk (src/aa_zero_dm.cpp:35-45, kernel :99-165)
//   old RFI                 per channel, 4-sigma clipped statistics, then
//                           4-sample means outside the cut replaced by the mean
//                           (src/aa_device_rfi.cu:8-30, src/aa_device_rfi_kernel.cu:8-50)
//   output normalisation    per output sample, subtract mean - 127.5 over the
//                           range's DM trials (src/aa_zero_dm.cpp:47-58)
// The summation trees of the reference's thread blocks are reproduced (one
// warp per time sample where the block's tree fits a warp).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace aab200 {

// x: [nsamp][nchans] uint16 in place; nbits 4, 8 or 16; norm[nchans].
cudaError_t launch_zero_dm(uint16_t *x, int nchans, long long nsamp, int nbits, const float *norm, cudaStream_t st);
cudaError_t launch_zero_dm_outliers(uint16_t *x, int nchans, long long nsamp, int nbits, const float *norm,
                                    cudaStream_t st);
// x: [nsamp][nchans] uint16 in place; nbits 4, 8 or 16.
cudaError_t launch_input_normalization(uint16_t *x, int nchans, long long nsamp, int nbits, cudaStream_t st);
// x: [nchans][nsamp] corner-turned chunk (one byte or uint16 per sample), in
// place; channels below 32*floor(nchans/32) as the reference's grid covers.
cudaError_t launch_old_rfi(void *x, int elem_bytes, int nchans, long long nsamp, cudaStream_t st);
// out: [ndms] rows of nt floats at pitch, in place.
cudaError_t launch_output_normalization(float *out, long long pitch, long long nt, int ndms, cudaStream_t st);
// stored SIGPROC records [n][nchans*nbits/8] -> [n][nchans] uint16 (nbits
// 1, 2, 4, 8, 16), for processing that needs the unpacked samples.
cudaError_t launch_unpack_records(const uint8_t *in, int nbits, int nchans, long long n, uint16_t *out,
                                  cudaStream_t st);

} // namespace aab200
