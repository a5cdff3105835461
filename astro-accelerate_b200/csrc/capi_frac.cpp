// capi_frac.cpp -- extern "C" entry points of the differentiable refinement
// kernels (aa_b200_frac_*, aa_b200_boxcar_*, declared in include/aa_b200.h).
#include "aa_b200.h"

#include <string>

#include <cuda_runtime.h>

#include "frac.cuh"
#include "sps.cuh"

using namespace aab200;

namespace {

thread_local std::string g_frac_error;

int frac_status(cudaError_t e, const char *what)
{
    if (e == cudaSuccess)
        return 0;
    g_frac_error = std::string(what) + ": " + cudaGetErrorString(e);
    return 1;
}

bool make_widths(const int *widths, int nwidths, BoxcarWidths &W)
{
    if (!widths || nwidths < 1 || nwidths > kMaxBoxcarWidths) {
        g_frac_error = "1 to 16 boxcar widths are supported";
        return false;
    }
    W.n = nwidths;
    for (int i = 0; i < nwidths; ++i)
        W.w[i] = widths[i];
    return true;
}

} // namespace

extern "C" {

int aa_b200_frac_dedisperse_fwd(const float *d_x, const float *d_dm, const double *d_kc, const int *d_base, int nsnip,
                                int nchans, int nsamp, double *d_y, void *stream)
{
    return frac_status(
        launch_frac_fwd(d_x, d_dm, d_kc, d_base, nsnip, nchans, nsamp, d_y, static_cast<cudaStream_t>(stream)),
        "fractional dedispersion");
}

int aa_b200_frac_dedisperse_adj(const float *d_x, const float *d_dm, const double *d_kc, const int *d_base,
                                const double *d_gy, int nsnip, int nchans, int nsamp, float *d_gx, float *d_gdm,
                                double *d_partial, void *stream)
{
    return frac_status(launch_frac_adj(d_x, d_dm, d_kc, d_base, d_gy, nsnip, nchans, nsamp, d_gx, d_gdm, d_partial,
                                       static_cast<cudaStream_t>(stream)),
                       "fractional dedispersion adjoint");
}

int aa_b200_boxcar_snr_fwd(const double *d_y, int nsnip, int nsamp, const int *widths, int nwidths, const float *d_mu,
                           const float *d_sigma, double *d_snr, void *stream)
{
    BoxcarWidths W;
    if (!make_widths(widths, nwidths, W))
        return 1;
    return frac_status(launch_boxcar_fwd(d_y, nsnip, nsamp, W, d_mu, d_sigma, d_snr, static_cast<cudaStream_t>(stream)),
                       "boxcar S/N");
}

int aa_b200_boxcar_snr_adj(const double *d_gsnr, int nsnip, int nsamp, const int *widths, int nwidths,
                           const float *d_sigma, double *d_gy, void *stream)
{
    BoxcarWidths W;
    if (!make_widths(widths, nwidths, W))
        return 1;
    return frac_status(launch_boxcar_adj(d_gsnr, nsnip, nsamp, W, d_sigma, d_gy, static_cast<cudaStream_t>(stream)),
                       "boxcar S/N adjoint");
}

int aa_b200_sps_row_stats(const float *d_y, int nrows, long long pitch, long long nsamp, float *d_mean,
                          float *d_stdev, void *stream)
{
    return frac_status(launch_row_stats(d_y, nrows, pitch, nsamp, d_mean, d_stdev, static_cast<cudaStream_t>(stream)),
                       "row statistics");
}

int aa_b200_sps_block_peaks(const float *d_y, int nrows, long long pitch, long long nsamp, const float *d_mean,
                            const float *d_stdev, const int *widths, int nwidths, float *d_peak_snr, int *d_peak_t,
                            int *d_peak_w, void *stream)
{
    BoxcarWidths W;
    if (!make_widths(widths, nwidths, W))
        return 1;
    return frac_status(launch_block_peaks(d_y, nrows, pitch, nsamp, d_mean, d_stdev, W, d_peak_snr, d_peak_t, d_peak_w,
                                          static_cast<cudaStream_t>(stream)),
                       "block peaks");
}

int aa_b200_sps_block_samples(void) { return SPS_BLOCK; }

const char *aa_b200_frac_last_error(void) { return g_frac_error.c_str(); }

} // extern "C"
