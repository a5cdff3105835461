// preproc.cu -- input and output processing options of the DDTR runner (see
// preproc.cuh).  The arithmetic of each reference kernel is kept operation for
// operation (types, operand order and the reduction tree of its thread
// block), since the float results, and through them the dedispersed output,
// depend on it; the thread organisation is this library's own.
#include "preproc.cuh"

namespace aab200 {

namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ uint16_t clamp_to_bits(float r, float hi)
{
    // the reference's branches: below 0 -> 0, above the range -> its top,
    // else truncation (a NaN takes the last branch)
    if (r < 0)
        return 0;
    if (r > hi)
        return static_cast<uint16_t>(hi);
    return static_cast<uint16_t>(r);
}

__device__ __forceinline__ float top_of(int nbits) { return nbits == 4 ? 15.f : (nbits == 8 ? 255.f : 65535.f); }

// ---------------------------------------------------------------------------
// Zero DM: one warp per time sample.  The reference sums a row with 256
// threads (thread j: channels j, j+256, ... in order), folds them in shared
// memory (j < 128, 64, 32 add j + 128, 64, 32) and then by warp shuffles
// (16 ... 1); lane l here holds threads l + 32k, k = 0..7, and folds them the
// same way.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float row_sum_256(const uint16_t *row, int nchans, int lane)
{
    float p[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float s = 0.0f;
        for (int c = lane + 32 * k; c < nchans; c += 256)
            s += static_cast<float>(row[c]);
        p[k] = s;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
        p[k] = p[k] + p[k + 4];
    p[0] = p[0] + p[2];
    p[1] = p[1] + p[3];
    p[0] = p[0] + p[1];
    float s = p[0];
#pragma unroll
    for (int q = 16; q > 0; q >>= 1)
        s += __shfl_down_sync(FULL, s, q);
    return __shfl_sync(FULL, s, 0);
}

__global__ void __launch_bounds__(256) k_zero_dm(uint16_t *__restrict__ x, int nchans, long long nsamp, int nbits,
                                                 const float *__restrict__ norm)
{
    const int lane = threadIdx.x & 31;
    const long long t = static_cast<long long>(blockIdx.x) * 8 + (threadIdx.x >> 5);
    if (t >= nsamp)
        return; // whole warps
    uint16_t *row = x + t * nchans;
    float sum = row_sum_256(row, nchans, lane);
    sum = sum / ((float)nchans);
    const float hi = top_of(nbits);
    for (int c = lane; c < nchans; c += 32) {
        const float result = (float)row[c] - sum + norm[c];
        row[c] = clamp_to_bits(result, hi);
    }
}

// ---------------------------------------------------------------------------
// Zero DM with outlier rejection: mean and deviation of a row by streaming
// updates and pairwise merges (the reference's 128-thread block: thread j
// takes channels j, j+128, ...; merges j < 64, 32 with j + 64, 32, then warp
// shuffles 16 ... 1), then up to five 3-sigma clipped passes, stopping when
// old mean - new mean < 0.001.
// ---------------------------------------------------------------------------
struct Msd {
    float M, S;
    int j;
};

__device__ __forceinline__ void msd_first(Msd &a, float e)
{
    a.M = e;
    a.S = 0;
    a.j = 1;
}

__device__ __forceinline__ void msd_add(Msd &a, float e)
{
    float ftemp;
    a.j = a.j + 1;
    double r_j = (double)a.j;
    a.M = a.M + e;
    ftemp = (r_j * e - a.M);
    a.S = a.S + 1.0f / (r_j * (r_j - 1.0f)) * ftemp * ftemp;
}

__device__ __forceinline__ void msd_merge(Msd &a, float B_M, float B_S, int B_j)
{
    float ftemp;
    double r_B_j = (double)B_j;
    double r_A_j = (double)a.j;
    ftemp = (r_B_j / r_A_j) * a.M - B_M;
    a.S = a.S + B_S + (r_A_j / (r_B_j * (r_A_j + r_B_j))) * ftemp * ftemp;
    a.M = a.M + B_M;
    a.j = a.j + B_j;
}

// a absorbs b unless b is empty; an empty a takes b
__device__ __forceinline__ void msd_fold(Msd &a, const Msd &b)
{
    if (b.j != 0) {
        if (a.j == 0)
            a = b;
        else
            msd_merge(a, b.M, b.S, b.j);
    }
}

// Folds lane l's four threads (l + 32k) and then the warp; returns the mean
// and deviation of lane 0's result on every lane.
__device__ __forceinline__ void msd_reduce(Msd (&t)[4], float &mean, float &stdev)
{
    msd_fold(t[0], t[2]);
    msd_fold(t[1], t[3]);
    msd_fold(t[0], t[1]);
    Msd a = t[0];
#pragma unroll
    for (int q = 16; q > 0; q >>= 1) {
        Msd b;
        b.M = __shfl_down_sync(FULL, a.M, q);
        b.S = __shfl_down_sync(FULL, a.S, q);
        b.j = __shfl_down_sync(FULL, a.j, q);
        if (b.j > 0) {
            if (a.j == 0)
                a = b;
            else
                msd_merge(a, b.M, b.S, b.j);
        }
    }
    float m = 0.f, s = 0.f;
    if ((threadIdx.x & 31) == 0) {
        m = a.M / (double)a.j;
        s = sqrt(a.S / (double)a.j);
    }
    mean = __shfl_sync(FULL, m, 0);
    stdev = __shfl_sync(FULL, s, 0);
}

__global__ void __launch_bounds__(256) k_zero_dm_outliers(uint16_t *__restrict__ x, int nchans, long long nsamp,
                                                          int nbits, const float *__restrict__ norm)
{
    const int lane = threadIdx.x & 31;
    const long long t = static_cast<long long>(blockIdx.x) * 8 + (threadIdx.x >> 5);
    if (t >= nsamp)
        return;
    uint16_t *row = x + t * nchans;
    const float sigma = 3.0f;
    float mean = 0, stdev = 0, old_mean = 0;
    {
        Msd th[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            th[k] = Msd{0.f, 0.f, 0};
            int c = lane + 32 * k;
            if (c < nchans) {
                msd_first(th[k], (float)row[c]);
                for (c += 128; c < nchans; c += 128)
                    msd_add(th[k], (float)row[c]);
            }
        }
        msd_reduce(th, mean, stdev);
    }
    for (int f = 0; f < 5; f++) {
        old_mean = mean;
        const float limit_down = mean - sigma * stdev;
        const float limit_up = mean + sigma * stdev;
        Msd th[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            th[k] = Msd{0.f, 0.f, 0};
            for (int c = lane + 32 * k; c < nchans; c += 128) {
                const float e = (float)row[c];
                if ((e > limit_down) && (e < limit_up)) {
                    if (th[k].j == 0)
                        msd_first(th[k], e);
                    else
                        msd_add(th[k], e);
                }
            }
        }
        msd_reduce(th, mean, stdev);
        if (old_mean - mean < 0.001f)
            break;
    }
    const float hi = top_of(nbits);
    for (int c = lane; c < nchans; c += 32) {
        const float result = (float)row[c] - mean + norm[c];
        row[c] = clamp_to_bits(result, hi);
    }
}

// ---------------------------------------------------------------------------
// Input normalisation: 32 x 32 threads per 32 channels; thread (x, y) sums
// rows y, y+32, ... of channel x, the y sums fold 16 ... 1, and every sample
// of the channel loses mean - (2^nbits - 1)/2.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_input_normalization(uint16_t *__restrict__ x, int nchans, long long nsamp,
                                                              float normalization_factor, int nbits)
{
    __shared__ float s_sum[1024];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const long long c = 32LL * blockIdx.x + tx;
    const long long nit = (nsamp + 32 - 1) / 32;
    float sum = 0;
    for (long long i = 0; i < nit; i++) {
        const long long t = 32 * i + ty;
        if (t < nsamp && c < nchans)
            sum = sum + (float)x[t * nchans + c];
    }
    s_sum[ty * 32 + tx] = sum;
    __syncthreads();
    for (int i = 16; i > 0; i = i >> 1) {
        if (ty < i)
            s_sum[ty * 32 + tx] = s_sum[ty * 32 + tx] + s_sum[ty * 32 + tx + i * 32];
        __syncthreads();
    }
    sum = s_sum[tx] / ((float)nsamp) - normalization_factor;
    const float hi = top_of(nbits);
    for (long long i = 0; i < nit; i++) {
        const long long t = 32 * i + ty;
        if (t < nsamp && c < nchans) {
            const float result = (float)x[t * nchans + c] - sum;
            x[t * nchans + c] = clamp_to_bits(result, hi);
        }
    }
}

// Output normalisation: thread (x, y) of a 32 x 32 block sums DM rows y,
// y+32, ... at sample x; every output at that sample loses mean - 127.5.
__global__ void __launch_bounds__(1024) k_output_normalization(float *__restrict__ out, long long pitch, long long nt,
                                                               int ndms)
{
    __shared__ float s_sum[1024];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const long long t = 32LL * blockIdx.x + tx;
    const int nit = (ndms + 32 - 1) / 32;
    float sum = 0;
    for (int i = 0; i < nit; i++) {
        const int dm = 32 * i + ty;
        if (dm < ndms && t < nt)
            sum = sum + out[dm * pitch + t];
    }
    s_sum[ty * 32 + tx] = sum;
    __syncthreads();
    for (int i = 16; i > 0; i = i >> 1) {
        if (ty < i)
            s_sum[ty * 32 + tx] = s_sum[ty * 32 + tx] + s_sum[ty * 32 + tx + i * 32];
        __syncthreads();
    }
    sum = s_sum[tx] / ((float)(size_t)ndms) - 127.5f;
    for (int i = 0; i < nit; i++) {
        const int dm = 32 * i + ty;
        if (dm < ndms && t < nt)
            out[dm * pitch + t] = out[dm * pitch + t] - sum;
    }
}

// ---------------------------------------------------------------------------
// Old RFI: one thread per channel (sequential float sums in time order, as
// the reference's per-channel thread), four passes of 4-sigma clipping from
// an initial cut of 4e6, then every 4-sample mean outside the cut sets the
// window's first sample to the mean.  The windows read samples no earlier
// window has replaced, so replacing in place in time order is exact.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(32) k_old_rfi(T *__restrict__ x, long long nsamp)
{
    const long long c = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    T *row = x + c * nsamp;
    int count = 0;
    float stdev = 1000000.0f;
    float mean = 0.0f;
    float sum = 0.0f;
    float sum_squares = 0.0f;
    float cutoff = (4.0f * stdev);
    for (int out = 0; out < 4; out++) {
        sum = 0.0f;
        sum_squares = 0.0f;
        count = 0;
        for (long long t = 0; t < nsamp; t++) {
            const float data = (float)row[t];
            if (data < (mean + cutoff) && data > (mean - cutoff)) {
                sum += data;
                sum_squares += (data * data);
                count++;
            }
        }
        mean = (sum / (float)count);
        sum_squares = ((sum_squares / count) - (mean * mean));
        stdev = sqrt(sum_squares);
        cutoff = (4.0f * stdev);
    }
    for (long long t = 0; t < nsamp - 4; t++) {
        float data = 0.0f;
        for (int k = 0; k < 4; k++)
            data += (float)row[t + k];
        data = data * 0.25f;
        if (data > (mean + cutoff) || data < (mean - cutoff))
            row[t] = static_cast<T>((unsigned short)mean);
    }
}

template <int NBITS>
__device__ __forceinline__ uint16_t record_sample(const uint8_t *rec, int c)
{
    if constexpr (NBITS == 16) {
        return reinterpret_cast<const uint16_t *>(rec)[c];
    } else if constexpr (NBITS == 8) {
        return rec[c];
    } else if constexpr (NBITS == 4) {
        const unsigned b = rec[c >> 1];
        return static_cast<uint16_t>((c & 1) ? (b & 15u) : (b >> 4));
    } else if constexpr (NBITS == 2) {
        const unsigned b = rec[c >> 2];
        return static_cast<uint16_t>((b >> (6 - 2 * (c & 3))) & 3u);
    } else {
        const unsigned b = rec[c >> 3];
        return static_cast<uint16_t>((b >> (c & 7)) & 1u);
    }
}

template <int NBITS>
__global__ void k_unpack_records(const uint8_t *__restrict__ in, int nchans, long long n, uint16_t *__restrict__ out)
{
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n * nchans)
        return;
    const long long t = i / nchans;
    const int c = static_cast<int>(i - t * nchans);
    out[i] = record_sample<NBITS>(in + t * (static_cast<long long>(nchans) * NBITS / 8), c);
}

bool bits_ok(int nbits) { return nbits == 4 || nbits == 8 || nbits == 16; }

} // namespace

cudaError_t launch_zero_dm(uint16_t *x, int nchans, long long nsamp, int nbits, const float *norm, cudaStream_t st)
{
    if (!bits_ok(nbits) || nchans < 1 || nsamp < 0)
        return cudaErrorInvalidValue;
    if (nsamp == 0)
        return cudaSuccess;
    k_zero_dm<<<static_cast<unsigned>((nsamp + 7) / 8), 256, 0, st>>>(x, nchans, nsamp, nbits, norm);
    return cudaGetLastError();
}

cudaError_t launch_zero_dm_outliers(uint16_t *x, int nchans, long long nsamp, int nbits, const float *norm,
                                    cudaStream_t st)
{
    if (!bits_ok(nbits) || nchans < 1 || nsamp < 0)
        return cudaErrorInvalidValue;
    if (nsamp == 0)
        return cudaSuccess;
    k_zero_dm_outliers<<<static_cast<unsigned>((nsamp + 7) / 8), 256, 0, st>>>(x, nchans, nsamp, nbits, norm);
    return cudaGetLastError();
}

cudaError_t launch_input_normalization(uint16_t *x, int nchans, long long nsamp, int nbits, cudaStream_t st)
{
    if (!bits_ok(nbits) || nchans < 1 || nsamp < 1)
        return cudaErrorInvalidValue;
    // (2^nbits - 1) / 2 as the reference computes it (double, then float)
    const float factor = static_cast<float>((static_cast<double>(1LL << nbits) - 1) / 2);
    k_input_normalization<<<(nchans + 31) / 32, dim3(32, 32), 0, st>>>(x, nchans, nsamp, factor, nbits);
    return cudaGetLastError();
}

cudaError_t launch_old_rfi(void *x, int elem_bytes, int nchans, long long nsamp, cudaStream_t st)
{
    const int blocks = nchans / 32;
    if (blocks < 1 || nsamp < 1)
        return blocks < 1 ? cudaSuccess : cudaErrorInvalidValue;
    if (elem_bytes == 1)
        k_old_rfi<uint8_t><<<blocks, 32, 0, st>>>(static_cast<uint8_t *>(x), nsamp);
    else
        k_old_rfi<uint16_t><<<blocks, 32, 0, st>>>(static_cast<uint16_t *>(x), nsamp);
    return cudaGetLastError();
}

cudaError_t launch_output_normalization(float *out, long long pitch, long long nt, int ndms, cudaStream_t st)
{
    if (nt < 1 || ndms < 1)
        return cudaSuccess;
    k_output_normalization<<<static_cast<unsigned>((nt + 31) / 32), dim3(32, 32), 0, st>>>(out, pitch, nt, ndms);
    return cudaGetLastError();
}

cudaError_t launch_unpack_records(const uint8_t *in, int nbits, int nchans, long long n, uint16_t *out,
                                  cudaStream_t st)
{
    if (nchans < 1 || n < 0 || (static_cast<long long>(nchans) * nbits) % 8)
        return cudaErrorInvalidValue;
    const long long tot = n * nchans;
    if (tot == 0)
        return cudaSuccess;
    const unsigned b = static_cast<unsigned>((tot + 255) / 256);
    switch (nbits) {
    case 1:
        k_unpack_records<1><<<b, 256, 0, st>>>(in, nchans, n, out);
        break;
    case 2:
        k_unpack_records<2><<<b, 256, 0, st>>>(in, nchans, n, out);
        break;
    case 4:
        k_unpack_records<4><<<b, 256, 0, st>>>(in, nchans, n, out);
        break;
    case 8:
        k_unpack_records<8><<<b, 256, 0, st>>>(in, nchans, n, out);
        break;
    case 16:
        k_unpack_records<16><<<b, 256, 0, st>>>(in, nchans, n, out);
        break;
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

} // namespace aab200
