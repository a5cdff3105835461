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

// ---------------------------------------------------------------------------
// Vector forms for T % 4 == 0 (rows of whole float4s): a thread takes four
// consecutive samples.  The window x[c][t+n .. t+n+4] of its four outputs
// lies in the float4s k = floor((t+n)/4) and k+1; since t is a multiple of
// 4, the offset o = (t+n) mod 4 is the same for every thread of the channel,
// so picking the five values is a branch-free uniform choice.  A float4 is
// either wholly inside [0, T) or wholly outside (read as 0), matching the
// per-sample bounds of the scalar kernels.
// ---------------------------------------------------------------------------
constexpr int F4T = 256;       // threads of the forward block
constexpr int F4_TILE = 4 * F4T; // outputs per forward block

__device__ __forceinline__ void window5(const float4 *__restrict__ row, int i, int T4, float (&v)[5])
{
    const int k = i >> 2; // floor division (arithmetic shift)
    const int o = i & 3;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 p = (k >= 0 && k < T4) ? __ldg(row + k) : z;
    const float4 q = (k + 1 >= 0 && k + 1 < T4) ? __ldg(row + k + 1) : z;
    const float e[8] = {p.x, p.y, p.z, p.w, q.x, q.y, q.z, q.w};
    switch (o) {
    case 0:
#pragma unroll
        for (int j = 0; j < 5; ++j)
            v[j] = e[j];
        break;
    case 1:
#pragma unroll
        for (int j = 0; j < 5; ++j)
            v[j] = e[j + 1];
        break;
    case 2:
#pragma unroll
        for (int j = 0; j < 5; ++j)
            v[j] = e[j + 2];
        break;
    default:
#pragma unroll
        for (int j = 0; j < 5; ++j)
            v[j] = e[j + 3];
        break;
    }
}

// y[b][t..t+3], channels in order with the scalar kernel's expression, so
// the sums are the same bits.
__global__ void __launch_bounds__(F4T) k_frac_fwd4(const float *__restrict__ x, const float *__restrict__ dm,
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
    const int t = blockIdx.x * F4_TILE + 4 * threadIdx.x;
    if (t >= T)
        return;
    const int T4 = T >> 2;
    const float4 *xb = reinterpret_cast<const float4 *>(x) + static_cast<size_t>(b) * C * T4;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 4
    for (int c = 0; c < C; ++c) {
        float v[5];
        window5(xb + static_cast<size_t>(c) * T4, t + s_n[c], T4, v);
        const double w = s_w[c];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double a0 = v[j];
            const double a1 = v[j + 1];
            acc[j] += fma(w, a1 - a0, a0);
        }
    }
    double2 *yo = reinterpret_cast<double2 *>(y + static_cast<size_t>(b) * T + t);
    yo[0] = make_double2(acc[0], acc[1]);
    yo[1] = make_double2(acc[2], acc[3]);
}

// Both adjoints of a group of channels of one snippet in one pass: the
// output gradient gy[b] is staged in shared memory once per block; per
// channel the input gradient row is written and the x row is read once for
// the DM gradient's partial sum.  Needs T % 4 == 0.
constexpr int FA_THREADS = 512;
constexpr int FA_CPB = 16; // channels per block

__global__ void __launch_bounds__(FA_THREADS) k_frac_adj_rows(const float *__restrict__ x,
                                                               const double *__restrict__ gy,
                                                               const float *__restrict__ dm,
                                                               const double *__restrict__ kc,
                                                               const int *__restrict__ base, int C, int T,
                                                               float *__restrict__ gx, double *__restrict__ partial)
{
    extern __shared__ double g[]; // gy[b][0..T), then [FA_CPB][FA_THREADS/32] warp sums
    double *red = g + T;
    const int b = blockIdx.y;
    const double2 *gsrc = reinterpret_cast<const double2 *>(gy + static_cast<size_t>(b) * T);
    for (int i = threadIdx.x; i < (T >> 1); i += FA_THREADS)
        reinterpret_cast<double2 *>(g)[i] = gsrc[i];
    __syncthreads();
    auto gat = [&](int i) -> double { return (i >= 0 && i < T) ? g[i] : 0.0; };
    const float d = dm[b];
    const int c_end = min(C, (blockIdx.x + 1) * FA_CPB);
    for (int c = blockIdx.x * FA_CPB; c < c_end; ++c) {
        int n;
        double w;
        delay_of(d, kc[c], base_of(base, b, C, c), n, w);
        // input gradient: one sample per lane and step, so that the staged
        // gradient is read and the gx row written warp-contiguously
        if (gx) {
            float *gr = gx + (static_cast<size_t>(b) * C + c) * T;
#pragma unroll 4
            for (int t = threadIdx.x; t < T; t += FA_THREADS) // gx[j] = (1 - w) gy[j - n] + w gy[j - n - 1]
                gr[t] = static_cast<float>((1.0 - w) * gat(t - n) + w * gat(t - n - 1));
        }
        // DM gradient: four samples per lane from two aligned float4s of the
        // x row (T % 4 == 0), the gradient in aligned pairs
        double acc = 0.0;
        if (partial) {
            const int T4 = T >> 2;
            const float4 *xrow = reinterpret_cast<const float4 *>(x) + (static_cast<size_t>(b) * C + c) * T4;
#pragma unroll 4
            for (int t = 4 * threadIdx.x; t < T; t += 4 * FA_THREADS) {
                float v[5];
                window5(xrow, t + n, T4, v);
                const double2 g01 = *reinterpret_cast<const double2 *>(g + t);
                const double2 g23 = *reinterpret_cast<const double2 *>(g + t + 2);
                const double gt[4] = {g01.x, g01.y, g23.x, g23.y};
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    acc += gt[j] * (static_cast<double>(v[j + 1]) - static_cast<double>(v[j]));
            }
        }
        if (partial) {
            for (int o = 16; o > 0; o >>= 1)
                acc += __shfl_down_sync(0xffffffffu, acc, o);
            if ((threadIdx.x & 31) == 0)
                red[(c - blockIdx.x * FA_CPB) * (FA_THREADS / 32) + (threadIdx.x >> 5)] = acc;
        }
    }
    if (partial) {
        __syncthreads();
        const int c = blockIdx.x * FA_CPB + threadIdx.x;
        if (threadIdx.x < FA_CPB && c < c_end) {
            double s = 0.0;
            for (int k = 0; k < FA_THREADS / 32; ++k)
                s += red[threadIdx.x * (FA_THREADS / 32) + k];
            partial[static_cast<size_t>(b) * C + c] = kc[c] * s;
        }
    }
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
    if ((T & 3) == 0 && (reinterpret_cast<uintptr_t>(x) & 15) == 0 && (reinterpret_cast<uintptr_t>(y) & 15) == 0) {
        if (smem > 48 * 1024) {
            const cudaError_t e = cudaFuncSetAttribute(k_frac_fwd4, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       static_cast<int>(smem));
            if (e != cudaSuccess)
                return e;
        }
        k_frac_fwd4<<<dim3((T + F4_TILE - 1) / F4_TILE, B), F4T, smem, st>>>(x, dm, kc, base, C, T, y);
        return cudaGetLastError();
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
    if (gdm && !partial)
        return cudaErrorInvalidValue;
    const size_t rows_smem = (static_cast<size_t>(T) + FA_CPB * (FA_THREADS / 32)) * sizeof(double);
    if ((T & 3) == 0 && rows_smem <= 200 * 1024 && (reinterpret_cast<uintptr_t>(x) & 15) == 0 &&
        (reinterpret_cast<uintptr_t>(gy) & 15) == 0 && (reinterpret_cast<uintptr_t>(gx) & 15) == 0 && (gx || gdm)) {
        cudaError_t e = cudaFuncSetAttribute(k_frac_adj_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(rows_smem));
        if (e != cudaSuccess)
            return e;
        k_frac_adj_rows<<<dim3((C + FA_CPB - 1) / FA_CPB, B), FA_THREADS, rows_smem, st>>>(
            x, gy, dm, kc, base, C, T, gx, gdm ? partial : nullptr);
        if (gdm)
            k_frac_adj_dm_sum<<<B, FT, 0, st>>>(partial, C, gdm);
        return cudaGetLastError();
    }
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
