// frac.cuh -- launchers of the fractional-delay dedispersion and boxcar S/N
// kernels (frac.cu) used for differentiable candidate refinement.
#pragma once
#include <cuda_runtime.h>

namespace aab200 {

constexpr int kMaxBoxcarWidths = 16;

struct BoxcarWidths {
    int n;
    int w[kMaxBoxcarWidths]; // ascending, 1..1024
};

// y[B][T] from x[B][C][T], dm[B] (device), kc[C] (device, FP64 samples per
// unit DM), base[B][C] (device, integer row shifts, or null)
cudaError_t launch_frac_fwd(const float *x, const float *dm, const double *kc, const int *base, int B, int C, int T,
                            double *y, cudaStream_t st);
// gx[B][C][T] (skipped when null) and gdm[B] (skipped when null; needs
// partial[B][C] FP64 scratch) from the output gradient gy[B][T] (FP64)
cudaError_t launch_frac_adj(const float *x, const float *dm, const double *kc, const int *base, const double *gy, int B,
                            int C, int T, float *gx, float *gdm, double *partial, cudaStream_t st);
// snr[B][W.n][T] (FP64) from y[B][T] (FP64), mu[B], sigma[B] (device)
cudaError_t launch_boxcar_fwd(const double *y, int B, int T, const BoxcarWidths &W, const float *mu,
                              const float *sigma, double *snr, cudaStream_t st);
cudaError_t launch_boxcar_adj(const double *gsnr, int B, int T, const BoxcarWidths &W, const float *sigma, double *gy,
                              cudaStream_t st);

} // namespace aab200
