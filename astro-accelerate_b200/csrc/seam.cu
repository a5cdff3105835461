// seam.cu -- the reference's dedispersion seam with its own signatures, so
// that a caller written against AstroAccelerate's runner links unchanged.
//
// AstroAccelerate's runner (include/aa_permitted_pipelines_generic.hpp:
// 693-840) drives the device work of one (chunk, range) through six functions
// of namespace astroaccelerate: load_chunk_data, corner_turn_SM_inplace,
// set_dedispersion_constants, bin_gpu, dedisperse and
// save_data_offset_stream.  This file defines all six with the reference's
// C++ signatures (and extern "C" twins, aa_b200_seam_*), on the reference's
// buffers: one unsigned short per sample, [t][c] after load_chunk_data and
// [c][t] after the corner turn, float DM-time rows out.
//
// What replaces the reference's device state: set_dedispersion_constants
// (src/aa_device_load_data.cu:58-61) stored the row length and t_processed
// in __constant__ memory for the kernels; here they are kept per host thread
// and read by the next dedisperse() of that thread.  dedisperse() copies the
// caller's rows into a padded staging buffer of its own (one byte per sample
// for nbits <= 8, two otherwise), because the staged kernels read a few KB
// beyond the last sample an output uses and the caller's buffer has no such
// padding; then it runs the channel-quad kernel (one-byte samples) or the
// staged fp32 kernel (two-byte samples) with delay tables built on the first
// call for a range and kept per thread.  All work is issued on the legacy
// default stream, as the reference's is, and dedisperse() returns 0, or 1 on
// failure (the reason in aa_b200_last_error()).
#include "aa_b200.h"
#include "aa_b200_seam.hpp"

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "ddtr_kernels.cuh"
#include "planner.hpp"

namespace aab200 {
void set_last_error(const std::string &m);
} // namespace aab200

namespace {

using namespace aab200;

// [c][t] unsigned short rows -> one byte per sample (the bit depth is <= 8)
__global__ void k_rows_to_bytes(const uint16_t *__restrict__ in, uint8_t *__restrict__ out, size_t n)
{
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = static_cast<uint8_t>(in[i]);
}

// Tables of one range, built on the first dedisperse() for it.
struct SeamRange {
    // key
    int nchans = 0, nbits = 0, ndms = 0, failsafe = 0;
    float dm_low = 0.f, dm_step = 0.f, tsamp = 0.f;
    unsigned long long shifts_hash = 0;
    // plan
    int kind = 0, nch_used = 0, group_dms = 0, span = 0, delay_max = 0;
    bool quad = false, f32 = false;
    QuadGeometry qg{};
    F32Launch fl{};
    int nquads = 0, maxpat = 0;
    int32_t *d_table = nullptr, *d_wmin = nullptr, *d_qpat = nullptr, *d_qwin = nullptr, *d_qoff = nullptr;
    ~SeamRange()
    {
        cudaFree(d_table);
        cudaFree(d_wmin);
        cudaFree(d_qpat);
        cudaFree(d_qwin);
        cudaFree(d_qoff);
    }
};

struct SeamState {
    long long i_nsamp = 0;  // set_dedispersion_constants: t_processed + maxshift
    int t_processed = 0;
    bool constants_set = false;
    std::vector<std::unique_ptr<SeamRange>> ranges;
    void *d_stage = nullptr; // padded copy of the caller's rows
    size_t stage_bytes = 0;
    int *d_flags = nullptr; // [0] device error flags, [1] span, [2] max delay, [3..6] pattern stats
    ~SeamState()
    {
        cudaFree(d_stage);
        cudaFree(d_flags);
    }
};

thread_local SeamState g_seam;

int seam_fail(const std::string &m)
{
    set_last_error("dedisperse: " + m);
    return 1;
}

unsigned long long hash_floats(const float *v, int n)
{
    unsigned long long h = 1469598103934665603ull;
    const unsigned char *b = reinterpret_cast<const unsigned char *>(v);
    for (size_t i = 0; i < static_cast<size_t>(n) * sizeof(float); ++i) {
        h ^= b[i];
        h *= 1099511628211ull;
    }
    return h;
}

bool check(cudaError_t e, std::string &err, const char *what)
{
    if (e == cudaSuccess)
        return true;
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
}

// Delay table, windows of 64-trial groups and, for one-byte samples, the
// channel-quad tables; or, for two-byte samples, the fp32 geometry.
bool build_range(SeamRange &R, const float *dmshifts, std::string &err)
{
    const cudaStream_t st = 0;
    SeamState &S = g_seam;
    if (!S.d_flags && !check(cudaMalloc(&S.d_flags, 8 * sizeof(int)), err, "cudaMalloc"))
        return false;
    const int nchans = R.nchans, nd = R.ndms;
    const float mstartdm = R.dm_low / R.tsamp; // src/aa_dedisperse.cpp:28,37-40
    const float mdmstep = R.dm_step / R.tsamp;
    R.kind = select_delay_kind(R.nbits, R.dm_step, R.tsamp, dmshifts[nchans - 1], R.failsafe);
    R.nch_used = (R.kind == KIND_SHARED4 && nchans > 4096) ? 4096 * (nchans / 4096) : nchans;
    if (nd % 64)
        return (err = "ndms must be a multiple of 64", false);
    R.group_dms = 64;
    const size_t nent = static_cast<size_t>(nchans) * nd;
    const int nch_pad = (nchans + 3) & ~3;
    float *d_shifts = nullptr;
    int h[4] = {0, 0, 0, 0};
    bool ok = check(cudaMalloc(&d_shifts, sizeof(float) * nchans), err, "cudaMalloc") &&
              check(cudaMalloc(&R.d_table, nent * sizeof(int32_t)), err, "cudaMalloc") &&
              check(cudaMalloc(&R.d_wmin, static_cast<size_t>(nd / 64) * nch_pad * sizeof(int32_t)), err,
                    "cudaMalloc") &&
              check(cudaMemcpy(d_shifts, dmshifts, sizeof(float) * nchans, cudaMemcpyHostToDevice), err, "H2D") &&
              check(cudaMemsetAsync(S.d_flags, 0, 8 * sizeof(int), st), err, "memset") &&
              check(launch_delay_table(d_shifts, nchans, nd, R.kind, FMA_ALL, mstartdm, mdmstep, R.d_table,
                                       S.d_flags, st),
                    err, "delay table") &&
              check(launch_group_windows(R.d_table, nchans, nd, 64, R.d_wmin, S.d_flags + 1, S.d_flags + 2, st), err,
                    "group windows") &&
              check(cudaMemcpy(h, S.d_flags, 3 * sizeof(int), cudaMemcpyDeviceToHost), err, "D2H");
    cudaFree(d_shifts);
    if (!ok)
        return false;
    if (h[0] != 0)
        return (err = "delay outside [0, 2^24) or class step > 1", false);
    R.span = h[1];
    R.delay_max = h[2];
    if (R.nbits > 8) {
        const F32Geometry G = f32_geometry(R.span, 64, nchans, 0);
        if (G.smem_bytes == 0 || nchans > 16384)
            return (err = "the delay span of this range does not fit the staged kernel", false);
        R.fl = G.f;
        R.f32 = true;
        return true;
    }
    const int nquads = (R.nch_used + 3) / 4;
    const int nq_pad = (nquads + 3) & ~3;
    const int ngroups = nd / 64;
    const size_t nq_ent = static_cast<size_t>(nquads) * nd;
    int32_t *d_qtmp = nullptr;
    int hs[4] = {0, 0, 0, 0};
    ok = check(cudaMalloc(&R.d_qpat, static_cast<size_t>(ngroups) * nquads * 16 * sizeof(int32_t)), err,
               "cudaMalloc") &&
         check(cudaMalloc(&R.d_qwin, static_cast<size_t>(ngroups) * nq_pad * sizeof(int32_t)), err, "cudaMalloc") &&
         check(cudaMemsetAsync(R.d_qwin, 0, static_cast<size_t>(ngroups) * nq_pad * sizeof(int32_t), st), err,
               "memset") &&
         check(cudaMalloc(&R.d_qoff, nq_ent * sizeof(int32_t)), err, "cudaMalloc") &&
         check(cudaMalloc(&d_qtmp, nq_ent * sizeof(int32_t)), err, "cudaMalloc") &&
         check(cudaMemsetAsync(S.d_flags + 3, 0, 4 * sizeof(int), st), err, "memset") &&
         check(launch_quad_patterns(R.d_table, R.nch_used, nd, 64, nquads, nq_pad, R.d_qpat, R.d_qwin, d_qtmp,
                                    S.d_flags + 3, st),
               err, "quad patterns") &&
         check(cudaMemcpy(hs, S.d_flags + 3, 4 * sizeof(int), cudaMemcpyDeviceToHost), err, "D2H");
    if (ok) {
        int qs = 4;
        QuadGeometry G = quad_geometry(hs[0], hs[1], hs[2], 64, nquads, 16, qs);
        while (G.smem_bytes > kStagedSmemLimit && qs > 1) {
            qs /= 2;
            G = quad_geometry(hs[0], hs[1], hs[2], 64, nquads, 16, qs);
        }
        if (G.smem_bytes <= kStagedSmemLimit && hs[1] <= 255) {
            ok = check(launch_quad_offsets(d_qtmp, nq_ent, G.W, R.d_qoff, st), err, "quad offsets") &&
                 check(cudaStreamSynchronize(st), err, "sync");
            R.qg = G;
            R.nquads = nquads;
            R.maxpat = hs[2];
            R.quad = ok;
        } else {
            err = "the delay span of this range does not fit the channel-quad kernel";
            ok = false;
        }
    }
    cudaFree(d_qtmp);
    return ok;
}

SeamRange *find_range(int i, int nchans, int nbits, const int *ndms, const float *dm_low, const float *dm_step,
                      float tsamp, int failsafe, const float *dmshifts, std::string &err)
{
    SeamState &S = g_seam;
    const unsigned long long hsh = hash_floats(dmshifts, nchans);
    for (auto &r : S.ranges)
        if (r->nchans == nchans && r->nbits == nbits && r->ndms == ndms[i] && r->failsafe == failsafe &&
            r->dm_low == dm_low[i] && r->dm_step == dm_step[i] && r->tsamp == tsamp && r->shifts_hash == hsh)
            return r.get();
    std::unique_ptr<SeamRange> R(new SeamRange());
    R->nchans = nchans;
    R->nbits = nbits;
    R->ndms = ndms[i];
    R->failsafe = failsafe;
    R->dm_low = dm_low[i];
    R->dm_step = dm_step[i];
    R->tsamp = tsamp;
    R->shifts_hash = hsh;
    if (!build_range(*R, dmshifts, err))
        return nullptr;
    if (S.ranges.size() >= 64) // a new plan: drop the oldest ranges
        S.ranges.erase(S.ranges.begin());
    S.ranges.push_back(std::move(R));
    return S.ranges.back().get();
}

} // namespace

extern "C" {

void aa_b200_seam_set_dedispersion_constants(int t_processed, int maxshift)
{
    g_seam.i_nsamp = static_cast<long long>(t_processed) + maxshift;
    g_seam.t_processed = t_processed;
    g_seam.constants_set = true;
}

void aa_b200_seam_load_chunk_data(unsigned short *device_pointer, const unsigned short *host_pointer, int t_processed,
                                  int maxshift, int nchans, float *dmshifts, float *d_dm_shifts, int nbits)
{
    const size_t length = static_cast<size_t>(t_processed) + static_cast<size_t>(maxshift);
    cudaMemcpy(device_pointer, host_pointer, static_cast<size_t>(nchans) * length * sizeof(unsigned short),
               cudaMemcpyHostToDevice);
    // the reference also moves the delay table to d_dm_shifts where its
    // kernels read it from global memory (more than 8192 channels, or more
    // than 4096 at 4 bits); this library reads the host table
    if (d_dm_shifts && dmshifts && ((nchans > 8192 && nbits != 4) || (nbits == 4 && nchans > 4096)))
        cudaMemcpy(d_dm_shifts, dmshifts, static_cast<size_t>(nchans) * sizeof(float), cudaMemcpyHostToDevice);
    aa_b200_seam_set_dedispersion_constants(t_processed, maxshift);
}

void aa_b200_seam_corner_turn_SM_inplace(unsigned short *d_input, unsigned short *d_temporary, size_t primary_size,
                                         size_t secondary_size)
{
    // [secondary][primary] -> [primary][secondary] through the temporary
    // buffer, then copied back (src/aa_corner_turn.cpp:118-121)
    if (aa_b200_corner_turn(d_input, d_temporary, 16, static_cast<int>(primary_size),
                            static_cast<long long>(secondary_size), static_cast<long long>(secondary_size),
                            nullptr) == 0)
        cudaMemcpy(d_input, d_temporary, primary_size * secondary_size * sizeof(unsigned short),
                   cudaMemcpyDeviceToDevice);
}

void aa_b200_seam_bin_gpu(unsigned short *d_input, float *d_output, int nchans, int nsamp)
{
    // the reference bins the flat buffer in place through d_output
    // (src/aa_bin_gpu.cpp:8-44): out of place into d_output, copied back
    unsigned short *tmp = reinterpret_cast<unsigned short *>(d_output);
    if (aa_b200_bin_gpu(d_input, tmp, 16, nchans, nsamp, nullptr) == 0)
        cudaMemcpy(d_input, tmp, static_cast<size_t>(nchans) * static_cast<size_t>(nsamp) * sizeof(unsigned short),
                   cudaMemcpyDeviceToDevice);
}

int aa_b200_seam_dedisperse(int i, int t_processed, int *inBin, float *dmshifts, unsigned short *d_input,
                            float *d_output, float *d_dm_shifts, int nchans, float *tsamp, float *dm_low,
                            float *dm_step, const int *ndms, int nbits, int failsafe)
{
    (void)d_dm_shifts;
    SeamState &S = g_seam;
    if (!S.constants_set)
        return seam_fail("set_dedispersion_constants (or load_chunk_data) was not called in this thread");
    if (!inBin || !dmshifts || !d_input || !d_output || !tsamp || !dm_low || !dm_step || !ndms || nchans <= 0 ||
        t_processed <= 0 || (t_processed & 3))
        return seam_fail("invalid arguments");
    const long long i_nsamp = S.i_nsamp;
    std::string err;
    SeamRange *R = find_range(i, nchans, nbits, ndms, dm_low, dm_step, *tsamp, failsafe, dmshifts, err);
    if (!R)
        return seam_fail(err);
    const int eb = nbits <= 8 ? 1 : 2;
    const int tile = R->quad ? 32 * R->qg.M : 512;
    const long long ntiles = (t_processed + tile - 1) / tile;
    long long need = static_cast<long long>(R->nch_used - 1) * i_nsamp + ntiles * tile + R->delay_max;
    need += R->quad ? 4LL * R->qg.raww + 64 : static_cast<long long>(R->fl.rawh) + 8;
    const long long have = static_cast<long long>(nchans) * i_nsamp;
    const size_t bytes = static_cast<size_t>(std::max(need, have)) * eb;
    if (bytes > S.stage_bytes) {
        cudaFree(S.d_stage);
        S.d_stage = nullptr;
        S.stage_bytes = 0;
        if (cudaMalloc(&S.d_stage, bytes) != cudaSuccess)
            return seam_fail("cudaMalloc of the staging buffer failed");
        S.stage_bytes = bytes;
    }
    const cudaStream_t st = 0;
    cudaError_t e;
    if (eb == 1) {
        const size_t n = static_cast<size_t>(have);
        const unsigned blocks = static_cast<unsigned>(std::min<size_t>((n + 255) / 256, 148u * 16u));
        k_rows_to_bytes<<<blocks, 256, 0, st>>>(d_input, static_cast<uint8_t *>(S.d_stage), n);
        e = cudaGetLastError();
    } else {
        e = cudaMemcpyAsync(S.d_stage, d_input, static_cast<size_t>(have) * 2, cudaMemcpyDeviceToDevice, st);
    }
    if (e == cudaSuccess && bytes > static_cast<size_t>(have) * eb)
        e = cudaMemsetAsync(static_cast<char *>(S.d_stage) + static_cast<size_t>(have) * eb, 0,
                            bytes - static_cast<size_t>(have) * eb, st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(S.d_flags, 0, sizeof(int), st);
    DdtrLaunch p{};
    p.in = S.d_stage;
    p.stride = i_nsamp;
    p.nchans = nchans;
    p.nch_used = R->nch_used;
    p.tp = t_processed;
    p.ndms = ndms[i];
    p.table = R->d_table;
    p.wmin = R->d_wmin;
    p.group_dms = 64;
    p.span = R->span;
    p.kind = R->kind;
    p.nchans_f = static_cast<float>(nchans);
    p.bin_f = static_cast<float>(inBin[i]);
    p.divide_by_bin = (R->kind == KIND_SHARED4) ? 0 : 1;
    p.out = d_output;
    p.out_pitch = t_processed;
    p.err = S.d_flags;
    if (e == cudaSuccess) {
        if (R->quad) {
            QuadLaunch q{};
            q.qpat = R->d_qpat;
            q.qwin = R->d_qwin;
            q.qoff = R->d_qoff;
            q.nquads = R->nquads;
            q.nq_pad = R->qg.nq_pad;
            q.W = R->qg.W;
            q.raww = R->qg.raww;
            q.qs = R->qg.qs;
            q.npool = R->qg.npool;
            q.M = R->qg.M;
            q.maxpat = R->maxpat;
            q.flavour = 0;
            e = launch_ddtr_quad(p, q, st);
        } else {
            e = launch_ddtr_f32(p, R->fl, st);
        }
    }
    int flag = 0;
    if (e == cudaSuccess)
        e = cudaMemcpy(&flag, S.d_flags, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return seam_fail(cudaGetErrorString(e));
    if (flag != 0)
        return seam_fail("device error flag " + std::to_string(flag));
    return 0;
}

void aa_b200_seam_save_data_offset_stream(int dm_range, int current_time_chunk, int **t_processed, long inc,
                                          int *inBin, const int *ndms, float *d_DDTR_output, float ***output_buffer)
{
    // each DM row of the chunk to output_buffer[range][dm] + inc/inBin
    // (src/aa_device_save_data.cu:19-62)
    const size_t tp = static_cast<size_t>(t_processed[dm_range][current_time_chunk]);
    const size_t host_off = static_cast<size_t>(inc / inBin[dm_range]);
    for (int k = 0; k < ndms[dm_range]; ++k)
        cudaMemcpy(output_buffer[dm_range][k] + host_off, d_DDTR_output + static_cast<size_t>(k) * tp,
                   tp * sizeof(float), cudaMemcpyDeviceToHost);
}

} // extern "C"

// The reference's own names (include/aa_dedisperse.hpp:20,
// include/aa_device_load_data.hpp:15-17, include/aa_corner_turn.hpp:28,
// include/aa_bin_gpu.hpp:17, include/aa_device_save_data.hpp:12).
namespace astroaccelerate {

void load_chunk_data(unsigned short *device_pointer, unsigned short const *const host_pointer, int t_processed,
                     int maxshift, int nchans, float *dmshifts, float *d_dm_shifts, int nbits)
{
    aa_b200_seam_load_chunk_data(device_pointer, host_pointer, t_processed, maxshift, nchans, dmshifts, d_dm_shifts,
                                 nbits);
}

void set_dedispersion_constants(int t_processed, int maxshift)
{
    aa_b200_seam_set_dedispersion_constants(t_processed, maxshift);
}

void corner_turn_SM_inplace(unsigned short *const d_input, unsigned short *const d_temporary,
                            const size_t primary_size, const size_t secondary_size)
{
    aa_b200_seam_corner_turn_SM_inplace(d_input, d_temporary, primary_size, secondary_size);
}

void bin_gpu(unsigned short *const d_input, float *const d_output, const int nchans, const int nsamp)
{
    aa_b200_seam_bin_gpu(d_input, d_output, nchans, nsamp);
}

int dedisperse(int i, int t_processed, int *inBin, float *dmshifts, unsigned short *d_input, float *d_output,
               float *d_dm_shifts, int nchans, float *tsamp, float *dm_low, float *dm_step, int const *const ndms,
               int nbits, int failsafe)
{
    return aa_b200_seam_dedisperse(i, t_processed, inBin, dmshifts, d_input, d_output, d_dm_shifts, nchans, tsamp,
                                   dm_low, dm_step, ndms, nbits, failsafe);
}

void save_data_offset_stream(int dm_range, int current_time_chunk, int **t_processed, long int inc, int *inBin,
                             int const *const ndms, float *d_DDTR_output, float ***output_buffer)
{
    aa_b200_seam_save_data_offset_stream(dm_range, current_time_chunk, t_processed, inc, inBin, ndms, d_DDTR_output,
                                         output_buffer);
}

} // namespace astroaccelerate
