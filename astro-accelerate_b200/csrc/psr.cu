// psr.cu -- periodicity building blocks (see psr.cuh).
#include "psr.cuh"

#include <atomic>
#include <cmath>

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

} // namespace

long long psr_kernel_launches() { return g_psr_launches.load(); }

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
