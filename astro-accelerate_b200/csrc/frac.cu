// frac.cu -- differentiable fractional-delay dedispersion and boxcar S/N for
// candidate refinement (no counterpart in the reference, whose DDTR uses
// integer delays only).
//
// Snippets x[b][c][t] (float32, B x C x T) are dedispersed at a continuous
// trial DM per snippet:
//     tau_c = dm_b * kc_c                      (samples; kc_c per unit DM)
//     n_c = floor(tau_c) - base_c, w_c = frac(tau_c)
//     y[b][t] = sum_c x[c][t+n_c] + w_c * (x[c][t+n_c+1] - x[c][t+n_c])
// with samples outside [0, T) read as 0.  Since t is an integer, n_c and w_c
// do not depend on t: the adjoint is a shifted, interpolated copy of the
// output gradient per channel (the transpose of the scatter), and
//     dL/ddm_b = sum_c kc_c * sum_t gy[t] * (x[c][t+n_c+1] - x[c][t+n_c]).
// base[b][c] (optional) is an integer shift of the snippet's channel rows: a
// snippet cut with channel c starting base_c samples late is dedispersed at
// the same DM as the uncut data.  Every kernel recomputes n_c and w_c from
// dm, kc and base instead of storing them.
//
// Precision: the snippets (the only large tensors) stay float32; delays,
// weights, the channel sums and the per-snippet series y, S/N and their
// gradients are FP64.  The kernels are bound by HBM traffic of x, so the
// FP64 arithmetic costs nothing, and a smooth maximum of the S/N at a low
// temperature (which amplifies rounding of the S/N) keeps its gradient to
// FP64 accuracy.
//
// Boxcar S/N of y for widths w (ascending, <= 1024):
//     snr[b][i][t] = (sum_{k<w_i} y'[t+k] - w_i mu_b) / (sigma_b sqrt(w_i))
// with y' = y inside [0, T) and mu_b beyond it; mu and sigma are constants.
#include <cmath>
#include <cstdint>

#include <cuda_runtime.h>

#include "frac.cuh"

namespace aab200 {

namespace {

constexpr int FT = 256; // threads per block (samples per block in the time-parallel kernels)

__device__ __forceinline__ void delay_of(float dm, double kc, int base, int &n, double &w)
{
    const double tau = static_cast<double>(dm) * kc;
    const double f = floor(tau);
    n = static_cast<int>(f) - base;
    w = tau - f;
}

__device__ __forceinline__ int base_of(const int *base, int b, int C, int c)
{
    return base ? base[static_cast<size_t>(b) * C + c] : 0;
}

__device__ __forceinline__ float at(const float *row, int i, int T) { return (i >= 0 && i < T) ? __ldg(row + i) : 0.f; }

__device__ __forceinline__ double atd(const double *row, int i, int T) { return (i >= 0 && i < T) ? row[i] : 0.0; }

// y[b][t]: one thread per output sample, channels in order.
__global__ void __launch_bounds__(FT) k_frac_fwd(const float *__restrict__ x, const float *__restrict__ dm,
                                                 const double *__restrict__ kc, const int *__restrict__ base, int C,
                                                 int T, double *__restrict__ y)
{
    extern __shared__ double s_w[]; // w[C] then n[C]
    int *s_n = reinterpret_cast<int *>(s_w + C);
    const int b = blockIdx.y;
    const float d = dm[b];
    for (int c = threadIdx.x; c < C; c += blockDim.x)
        delay_of(d, kc[c], base_of(base, b, C, c), s_n[c], s_w[c]);
    __syncthreads();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T)
        return;
    const float *xb = x + static_cast<size_t>(b) * C * T;
    double acc = 0.0;
#pragma unroll 8
    for (int c = 0; c < C; ++c) {
        const float *row = xb + static_cast<size_t>(c) * T;
        const int i = t + s_n[c];
        const double a0 = at(row, i, T);
        const double a1 = at(row, i + 1, T);
        acc += fma(s_w[c], a1 - a0, a0);
    }
    y[static_cast<size_t>(b) * T + t] = acc;
}

// gx[b][c][j] = (1 - w_c) gy[j - n_c] + w_c gy[j - n_c - 1]
__global__ void __launch_bounds__(FT) k_frac_adj_x(const double *__restrict__ gy, const float *__restrict__ dm,
                                                   const double *__restrict__ kc, const int *__restrict__ base, int C,
                                                   int T, float *__restrict__ gx)
{
    const int b = blockIdx.z, c = blockIdx.y;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= T)
        return;
    int n;
    double w;
    delay_of(dm[b], kc[c], base_of(base, b, C, c), n, w);
    const double *g = gy + static_cast<size_t>(b) * T;
    const double v = (1.0 - w) * atd(g, j - n, T) + w * atd(g, j - n - 1, T);
    gx[(static_cast<size_t>(b) * C + c) * T + j] = static_cast<float>(v);
}

// partial[b][c] = kc_c * sum_t gy[t] (x[c][t+n+1] - x[c][t+n])
__global__ void __launch_bounds__(FT) k_frac_adj_dm_partial(const float *__restrict__ x, const double *__restrict__ gy,
                                                            const float *__restrict__ dm, const double *__restrict__ kc,
                                                            const int *__restrict__ base, int C, int T,
                                                            double *__restrict__ partial)
{
    __shared__ double red[FT / 32];
    const int b = blockIdx.y, c = blockIdx.x;
    int n;
    double w;
    delay_of(dm[b], kc[c], base_of(base, b, C, c), n, w);
    const float *row = x + (static_cast<size_t>(b) * C + c) * T;
    const double *g = gy + static_cast<size_t>(b) * T;
    double acc = 0.0;
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
        const int i = t + n;
        acc += g[t] * (static_cast<double>(at(row, i + 1, T)) - static_cast<double>(at(row, i, T)));
    }
    for (int o = 16; o > 0; o >>= 1)
        acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < FT / 32; ++k)
            s += red[k];
        partial[static_cast<size_t>(b) * C + c] = kc[c] * s;
    }
}

// gdm[b] = sum_c partial[b][c], fixed order
__global__ void __launch_bounds__(FT) k_frac_adj_dm_sum(const double *__restrict__ partial, int C,
                                                        float *__restrict__ gdm)
{
    __shared__ double red[FT];
    const int b = blockIdx.x;
    double s = 0.0;
    for (int c = threadIdx.x; c < C; c += blockDim.x)
        s += partial[static_cast<size_t>(b) * C + c];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = FT / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h)
            red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        gdm[b] = static_cast<float>(red[0]);
}

// snr[b][i][t]; the block stages y[t0, t0 + FT + wmax - 1) (mu beyond T).
__global__ void __launch_bounds__(FT) k_boxcar_fwd(const double *__restrict__ y, int T, BoxcarWidths W,
                                                   const float *__restrict__ mu, const float *__restrict__ sigma,
                                                   double *__restrict__ snr)
{
    extern __shared__ double ys[];
    const int b = blockIdx.y;
    const int t0 = blockIdx.x * FT;
    const int wmax = W.w[W.n - 1];
    const double m = mu[b], sg = sigma[b];
    const double *yb = y + static_cast<size_t>(b) * T;
    for (int k = threadIdx.x; k < FT + wmax - 1; k += blockDim.x) {
        const int t = t0 + k;
        ys[k] = (t < T) ? yb[t] : m;
    }
    __syncthreads();
    const int t = t0 + threadIdx.x;
    if (t >= T)
        return;
    double s = 0.0;
    int k = 0;
    for (int i = 0; i < W.n; ++i) {
        for (; k < W.w[i]; ++k)
            s += ys[threadIdx.x + k];
        const double wf = static_cast<double>(W.w[i]);
        snr[(static_cast<size_t>(b) * W.n + i) * T + t] = (s - wf * m) / (sg * sqrt(wf));
    }
}

// gy[b][t] = sum_i 1/(sigma sqrt(w_i)) sum_{k<w_i, t-k>=0} gsnr[b][i][t-k]
__global__ void __launch_bounds__(FT) k_boxcar_adj(const double *__restrict__ gsnr, int T, BoxcarWidths W,
                                                   const float *__restrict__ sigma, double *__restrict__ gy)
{
    extern __shared__ double gs[]; // [n][FT + wmax - 1], covering t0 - wmax + 1 .. t0 + FT - 1
    const int b = blockIdx.y;
    const int t0 = blockIdx.x * FT;
    const int wmax = W.w[W.n - 1];
    const int span = FT + wmax - 1;
    for (int i = 0; i < W.n; ++i) {
        const double *g = gsnr + (static_cast<size_t>(b) * W.n + i) * T;
        for (int k = threadIdx.x; k < span; k += blockDim.x) {
            const int t = t0 - wmax + 1 + k;
            gs[i * span + k] = (t >= 0 && t < T) ? g[t] : 0.0;
        }
    }
    __syncthreads();
    const int t = t0 + threadIdx.x;
    if (t >= T)
        return;
    const double sg = sigma[b];
    double acc = 0.0;
    for (int i = 0; i < W.n; ++i) {
        double s = 0.0;
        const double *row = gs + i * span + (threadIdx.x + wmax - 1);
        for (int k = 0; k < W.w[i]; ++k)
            s += row[-k];
        acc += s / (sg * sqrt(static_cast<double>(W.w[i])));
    }
    gy[static_cast<size_t>(b) * T + t] = acc;
}

} // namespace

cudaError_t launch_frac_fwd(const float *x, const float *dm, const double *kc, const int *base, int B, int C, int T,
                            double *y, cudaStream_t st)
{
    if (B <= 0 || C <= 0 || T <= 0 || B > 65535 || C > 16384)
        return cudaErrorInvalidValue;
    const size_t smem = static_cast<size_t>(C) * 12;
    if (smem > 48 * 1024) {
        const cudaError_t e =
            cudaFuncSetAttribute(k_frac_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess)
            return e;
    }
    dim3 grid((T + FT - 1) / FT, B);
    k_frac_fwd<<<grid, FT, smem, st>>>(x, dm, kc, base, C, T, y);
    return cudaGetLastError();
}

cudaError_t launch_frac_adj(const float *x, const float *dm, const double *kc, const int *base, const double *gy, int B,
                            int C, int T, float *gx, float *gdm, double *partial, cudaStream_t st)
{
    if (B <= 0 || C <= 0 || T <= 0 || B > 65535 || C > 65535)
        return cudaErrorInvalidValue;
    if (gx) {
        dim3 grid((T + FT - 1) / FT, C, B);
        k_frac_adj_x<<<grid, FT, 0, st>>>(gy, dm, kc, base, C, T, gx);
    }
    if (gdm) {
        if (!partial)
            return cudaErrorInvalidValue;
        k_frac_adj_dm_partial<<<dim3(C, B), FT, 0, st>>>(x, gy, dm, kc, base, C, T, partial);
        k_frac_adj_dm_sum<<<B, FT, 0, st>>>(partial, C, gdm);
    }
    return cudaGetLastError();
}

static bool widths_ok(const BoxcarWidths &W)
{
    if (W.n < 1 || W.n > kMaxBoxcarWidths)
        return false;
    for (int i = 0; i < W.n; ++i)
        if (W.w[i] < 1 || W.w[i] > 1024 || (i > 0 && W.w[i] <= W.w[i - 1]))
            return false;
    return true;
}

cudaError_t launch_boxcar_fwd(const double *y, int B, int T, const BoxcarWidths &W, const float *mu,
                              const float *sigma, double *snr, cudaStream_t st)
{
    if (B <= 0 || T <= 0 || B > 65535 || !widths_ok(W))
        return cudaErrorInvalidValue;
    const size_t smem = static_cast<size_t>(FT + W.w[W.n - 1] - 1) * sizeof(double);
    k_boxcar_fwd<<<dim3((T + FT - 1) / FT, B), FT, smem, st>>>(y, T, W, mu, sigma, snr);
    return cudaGetLastError();
}

cudaError_t launch_boxcar_adj(const double *gsnr, int B, int T, const BoxcarWidths &W, const float *sigma, double *gy,
                              cudaStream_t st)
{
    if (B <= 0 || T <= 0 || B > 65535 || !widths_ok(W))
        return cudaErrorInvalidValue;
    const size_t smem = static_cast<size_t>(W.n) * (FT + W.w[W.n - 1] - 1) * sizeof(double);
    if (smem > 48 * 1024)
        return cudaErrorInvalidValue;
    k_boxcar_adj<<<dim3((T + FT - 1) / FT, B), FT, smem, st>>>(gsnr, T, W, sigma, gy);
    return cudaGetLastError();
}

} // namespace aab200
