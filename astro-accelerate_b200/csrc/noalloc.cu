// noalloc.cu -- a dedispersion entry point that allocates no device memory.
//
// aa_b200_dedisperse() builds its delay, window and offset tables in device
// memory it allocates for the call.  Some callers cannot allocate: code that
// runs where cudaMalloc/cudaFree are not allowed (inside a memory pool or
// arena that owns all of the GPU's memory, real-time loops that must not
// synchronise with the allocator, hosts that pre-reserve device memory at
// start-up).  aa_b200_dedisperse_noalloc() does the same work with its
// scratch in a fixed array in the library's device image instead.
//
// The array below is part of the module image: every GPU that loads the
// library holds its AA_B200_NOALLOC_SCRATCH_BYTES until the process exits.
// Host code must not use the symbol itself as a device address (it is a host
// stand-in); the device address is looked up once per device with
// cudaGetSymbolAddress, with that device current, and passed to the kernels.
#include "aa_b200.h"

#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "ddtr_kernels.cuh"
#include "planner.hpp"

namespace {

constexpr size_t kScratchBytes = AA_B200_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct DeviceScratch {
    void *ptr = nullptr;
    bool ready = false;
};
DeviceScratch g_scratch[kMaxDevices];
std::mutex g_scratch_mutex;
thread_local std::string g_noalloc_error;

int fail(const std::string &m)
{
    g_noalloc_error = m;
    return 1;
}

// Device address of the scratch array on the current device (looked up on
// the first call made on each device).
cudaError_t scratch_address(void **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return e;
    if (dev < 0 || dev >= kMaxDevices)
        return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch[dev].ready) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return e;
        g_scratch[dev].ptr = p;
        g_scratch[dev].ready = true;
    }
    *out = g_scratch[dev].ptr;
    return cudaSuccess;
}

inline size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

} // namespace

extern "C" {

const char *aa_b200_noalloc_last_error(void) { return g_noalloc_error.c_str(); }

int aa_b200_dedisperse_noalloc(int i, int t_processed, const int *inBin, const float *dmshifts, const void *d_input,
                               long long i_nsamp, size_t d_input_elems, float *d_output, long long out_pitch,
                               int nchans, const float *tsamp, const float *dm_low, const float *dm_step,
                               const int *ndms, int nbits, int failsafe, void *stream)
{
    using namespace aab200;
    g_noalloc_error.clear();
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int eb = nbits <= 8 ? 1 : 2;
    const int nd = ndms[i];
    if (nd <= 0 || (nd % 4) || t_processed <= 0 || (t_processed & 3) || nchans <= 0)
        return fail("ndms must be a positive multiple of 4 and t_processed a positive multiple of 4");
    if (nchans > AA_B200_NOALLOC_MAX_CHANS ||
        static_cast<size_t>(nchans) * static_cast<size_t>(nd) > AA_B200_NOALLOC_MAX_ENTRIES)
        return fail("aa_b200_dedisperse_noalloc: nchans (" + std::to_string(nchans) + ") x ndms (" +
                    std::to_string(nd) + ") exceeds the fixed scratch limits (nchans <= " +
                    std::to_string(AA_B200_NOALLOC_MAX_CHANS) + ", nchans x ndms <= " +
                    std::to_string(AA_B200_NOALLOC_MAX_ENTRIES) + "); use aa_b200_dedisperse");

    void *base = nullptr;
    cudaError_t e = scratch_address(&base);
    if (e != cudaSuccess)
        return fail(std::string("cudaGetSymbolAddress of the scratch array: ") + cudaGetErrorString(e));

    // scratch layout: [flags x3 | dmshifts | delay table | offset table | windows]
    const size_t nent = static_cast<size_t>(nchans) * nd;
    const int nch_pad = (nchans + 3) & ~3;
    unsigned char *s = static_cast<unsigned char *>(base);
    int *d_flags = reinterpret_cast<int *>(s);
    size_t off = 256;
    float *d_shifts = reinterpret_cast<float *>(s + off);
    off = align256(off + sizeof(float) * nchans);
    int32_t *d_table = reinterpret_cast<int32_t *>(s + off);
    off = align256(off + nent * sizeof(int32_t));
    int32_t *d_off = reinterpret_cast<int32_t *>(s + off);
    off = align256(off + nent * sizeof(int32_t));
    int32_t *d_wmin = reinterpret_cast<int32_t *>(s + off);
    const size_t wmin_max = static_cast<size_t>(nd / 4) * nch_pad * sizeof(int32_t);
    if (off + wmin_max > kScratchBytes)
        return fail("aa_b200_dedisperse_noalloc: tables do not fit the fixed scratch array");

    const float mstartdm = dm_low[i] / *tsamp; // src/aa_dedisperse.cpp:28,37-40
    const float mdmstep = dm_step[i] / *tsamp;
    const int kind = select_delay_kind(nbits, dm_step[i], *tsamp, dmshifts[nchans - 1], failsafe);
    const int nch_used = (kind == KIND_SHARED4 && nchans > 4096) ? 4096 * (nchans / 4096) : nchans;
    const int tile_words = 4;
    int h[3] = {0, 0, 0};

    // the array keeps the previous call's contents: clear the flags first
    e = cudaMemsetAsync(d_flags, 0, 3 * sizeof(int), st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_shifts, dmshifts, sizeof(float) * nchans, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = launch_delay_table(d_shifts, nchans, nd, kind, FMA_ALL, mstartdm, mdmstep, d_table, d_flags, st);
    int gd = 0;
    for (int cand : {64, 32, 16, 8, 4}) {
        if (e != cudaSuccess)
            break;
        if (nd % cand)
            continue;
        e = cudaMemsetAsync(d_flags + 1, 0, 2 * sizeof(int), st);
        if (e == cudaSuccess)
            e = launch_group_windows(d_table, nchans, nd, cand, d_wmin, d_flags + 1, d_flags + 2, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(h, d_flags, 3 * sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(st);
        if (e != cudaSuccess)
            break;
        if (eb == 2 || ddtr_u8_smem_bytes(h[1], cand, tile_words, nchans) <= 227 * 1024) {
            gd = cand;
            break;
        }
    }
    if (e != cudaSuccess)
        return fail(cudaGetErrorString(e));
    if (gd == 0)
        return fail("no DM-group size fits the delay span");
    if (h[0] != 0)
        return fail("delay outside [0, 2^24) or class step > 1");
    const long long tile = 128LL * tile_words;
    long long need;
    if (eb == 1)
        need = static_cast<long long>(nch_used - 1) * i_nsamp + ((t_processed + tile - 1) / tile) * tile + h[2] +
               4LL * ddtr_u8_rw(h[1], tile_words) + 64;
    else
        need = static_cast<long long>(nch_used - 1) * i_nsamp + t_processed + h[2] + 2;
    if (need > static_cast<long long>(d_input_elems))
        return fail("d_input needs " + std::to_string(need) + " elements including window padding, has " +
                    std::to_string(d_input_elems));
    if (eb == 1)
        e = launch_offset_table(d_table, d_wmin, nchans, nd, gd, ddtr_u8_rw(h[1], tile_words), h[1], d_off, st);
    DdtrLaunch p;
    p.in = d_input;
    p.stride = i_nsamp;
    p.nchans = nchans;
    p.nch_used = nch_used;
    p.tp = t_processed;
    p.ndms = nd;
    p.table = d_table;
    p.wmin = d_wmin;
    p.group_dms = gd;
    p.span = h[1];
    p.kind = kind;
    p.nchans_f = static_cast<float>(nchans);
    p.bin_f = static_cast<float>(inBin[i]);
    p.divide_by_bin = (kind == KIND_SHARED4) ? 0 : 1;
    p.out = d_output;
    p.out_pitch = out_pitch;
    p.err = d_flags;
    if (e == cudaSuccess)
        e = (eb == 1) ? launch_ddtr_u8(p, d_off, tile_words, st) : launch_ddtr_u16(p, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h, d_flags, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return fail(cudaGetErrorString(e));
    if (h[0] != 0)
        return fail("device reported an error flag " + std::to_string(h[0]));
    return 0;
}

} // extern "C"
