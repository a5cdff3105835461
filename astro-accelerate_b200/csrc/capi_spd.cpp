// capi_spd.cpp -- extern "C" entry points of the single-pulse detection
// (aa_b200_spd_*, declared in include/aa_b200.h): analysis_GPU of
// src/aa_device_analysis.cu:130-345 on one DM-time plane in device memory,
// and the candidate file it writes.
#include "aa_b200.h"

#include <cstdio>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "spd.cuh"

using namespace aab200;

namespace {

struct SpdHandle {
    SpdPlane plane;
    std::string error;
};

thread_local std::string g_spd_error;

SpdHandle *as_spd(void *obj) { return static_cast<SpdHandle *>(obj); }

} // namespace

extern "C" {

void *aa_b200_spd_create(long long max_elems, long long max_time_samples)
{
    SpdHandle *h = new (std::nothrow) SpdHandle();
    if (!h) {
        g_spd_error = "single-pulse detection: out of host memory";
        return nullptr;
    }
    std::string err;
    if (!h->plane.setup(max_elems, max_time_samples, err)) {
        g_spd_error = err;
        delete h;
        return nullptr;
    }
    return h;
}

void aa_b200_spd_destroy(void *obj) { delete as_spd(obj); }

const char *aa_b200_spd_last_error(const void *obj)
{
    return obj ? static_cast<const SpdHandle *>(obj)->error.c_str() : g_spd_error.c_str();
}

int aa_b200_spd_clear(void *obj, void *stream)
{
    SpdHandle *h = as_spd(obj);
    if (!h)
        return 1;
    const cudaError_t e = h->plane.clear(static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        h->error = std::string("single-pulse detection: ") + cudaGetErrorString(e);
        return 1;
    }
    return 0;
}

int aa_b200_spd_keep_planes(void *obj, int on)
{
    SpdHandle *h = as_spd(obj);
    if (!h)
        return 1;
    h->plane.keep_planes = on != 0;
    return 0;
}

int aa_b200_spd_run(void *obj, float *d_plane, int nDMs, int nTimesamples, float tsamp, int inBin,
                    float sigma_cutoff, float sigma_constant, float max_boxcar_width_in_sec, int candidate_algorithm,
                    int enable_msd_baseline_noise, void *stream, size_t max_candidates, unsigned *h_dm,
                    unsigned *h_ts, float *h_snr, unsigned *h_bw, size_t *n_candidates)
{
    SpdHandle *h = as_spd(obj);
    if (!h)
        return 1;
    if (!d_plane || !n_candidates || (max_candidates > 0 && (!h_dm || !h_ts || !h_snr || !h_bw))) {
        h->error = "single-pulse detection: null argument";
        return 1;
    }
    SpdSettings s;
    s.sigma_cutoff = sigma_cutoff;
    s.sigma_constant = sigma_constant;
    s.max_boxcar_width_in_sec = max_boxcar_width_in_sec;
    s.candidate_algorithm = candidate_algorithm;
    s.enable_msd_baseline_noise = enable_msd_baseline_noise;
    SpdCandidates c;
    std::string err;
    h->plane.dropped_batches = 0;
    if (!h->plane.run(d_plane, nDMs, nTimesamples, tsamp, inBin, s, c, static_cast<cudaStream_t>(stream), err,
                      max_candidates)) {
        h->error = err;
        return 1;
    }
    const size_t k = c.dm.size();
    for (size_t i = 0; i < k; ++i) {
        h_dm[i] = c.dm[i];
        h_ts[i] = c.ts[i];
        h_snr[i] = c.snr[i];
        h_bw[i] = c.bw[i];
    }
    *n_candidates = k;
    return 0;
}

int aa_b200_spd_profile(const void *obj, float *msd, int msd_cap, int *widths, int *nwidths,
                        int *max_width_performed, int *max_iteration, int *dropped_batches)
{
    const SpdHandle *h = static_cast<const SpdHandle *>(obj);
    if (!h)
        return 1;
    const SpdPlane &p = h->plane;
    const int nw = static_cast<int>(p.last_widths.size());
    if (nwidths)
        *nwidths = nw;
    if (max_width_performed)
        *max_width_performed = p.last_max_width_performed;
    if (max_iteration)
        *max_iteration = p.last_max_iteration;
    if (dropped_batches)
        *dropped_batches = p.dropped_batches;
    if (widths)
        for (int i = 0; i < nw && i < msd_cap; ++i)
            widths[i] = p.last_widths[i];
    if (msd)
        for (int i = 0; i < static_cast<int>(p.last_msd.size()) && i < 2 * msd_cap; ++i)
            msd[i] = p.last_msd[i];
    return 0;
}

long long aa_b200_spd_planes(const void *obj, float *snr, unsigned short *taps, long long cap)
{
    const SpdHandle *h = static_cast<const SpdHandle *>(obj);
    if (!h)
        return -1;
    const long long n = static_cast<long long>(h->plane.last_snr.size());
    if (snr && taps && cap >= n) {
        for (long long i = 0; i < n; ++i) {
            snr[i] = h->plane.last_snr[i];
            taps[i] = h->plane.last_taps[i];
        }
    }
    return n;
}

long long aa_b200_spd_kernel_launches(void) { return spd_kernel_launches(); }

int aa_b200_spd_msd_profile(void *obj, const float *d_input, int nDMs, int nTimesamples, const int *widths,
                            int nwidths, int high_memory, float sigma_constant, int outlier_rejection, float *h_msd,
                            void *stream)
{
    SpdHandle *h = as_spd(obj);
    if (!h)
        return 1;
    if (!d_input || !widths || nwidths < 1 || !h_msd) {
        h->error = "MSD profile: null argument";
        return 1;
    }
    std::vector<int> w(widths, widths + nwidths);
    std::string err;
    if (!h->plane.profile(d_input, nDMs, nTimesamples, w, high_memory != 0, sigma_constant, outlier_rejection != 0,
                          static_cast<cudaStream_t>(stream), err)) {
        h->error = err;
        return 1;
    }
    for (size_t i = 0; i < h->plane.last_msd.size(); ++i)
        h_msd[i] = h->plane.last_msd[i];
    return 0;
}

int aa_b200_spd_first_plane(const float *d_input, float *d_boxcar_values, float *d_decimated, float *d_snr,
                            unsigned short *d_taps, const float *h_msd, int nTimesamples, int nBoxcars, int nDMs,
                            void *stream)
{
    if (!h_msd || nBoxcars < 8 || nBoxcars > SPD_MAXTAPS || nTimesamples < 1 || nDMs < 1) {
        g_spd_error = "single-pulse detection: nBoxcars 8, 16 or 32 and a non-empty plane needed";
        return 1;
    }
    SnrMsd m{};
    for (int k = 0; k < nBoxcars; ++k)
        m.v[k] = make_float2(h_msd[2 * k], h_msd[2 * k + 1]);
    // src/aa_device_analysis.cu:44-64: blocks of 2*512 - nBoxcars samples, dtm even
    const int epb = 2 * SPD_NTHREADS - nBoxcars;
    const int nBlocks = (nTimesamples + epb - 1) / epb;
    int dtm = nTimesamples >> 1;
    dtm -= dtm & 1;
    const cudaError_t e = spdt_first_plane(d_input, d_boxcar_values, d_decimated, d_snr, d_taps, m, nTimesamples,
                                           nBoxcars, dtm, nBlocks, nDMs, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        g_spd_error = std::string("single-pulse detection: ") + cudaGetErrorString(e);
        return 1;
    }
    return 0;
}

int aa_b200_spd_time_kernels(void *obj, int on)
{
    SpdHandle *h = as_spd(obj);
    if (!h)
        return 1;
    h->plane.time_kernels = on != 0;
    return 0;
}

int aa_b200_spd_family_time(const void *obj, int family, double *ms, long long *launches)
{
    const SpdHandle *h = static_cast<const SpdHandle *>(obj);
    if (!h || family < 0 || family >= SpdPlane::kFamilies)
        return 1;
    if (ms)
        *ms = h->plane.family_ms[family];
    if (launches)
        *launches = h->plane.family_n[family];
    return 0;
}

int aa_b200_spd_plan(int nTimesamples, float tsamp, int inBin, float max_boxcar_width_in_sec, int *widths,
                     int widths_cap, int *nwidths, int *max_width_performed, int *max_iteration, int *plan,
                     int plan_cap, int *nplan)
{
    if (inBin < 1 || !(tsamp > 0.f) || nTimesamples < 1) {
        g_spd_error = "single-pulse detection: inBin >= 1, tsamp > 0 and nTimesamples >= 1 needed";
        return 1;
    }
    const std::vector<int> bc = spd_bc_widths();
    const int mbw = static_cast<int>(max_boxcar_width_in_sec / tsamp);
    int mwp = 0;
    const int it = spd_max_iteration(mbw / inBin, bc, mwp);
    const std::vector<int> w = spd_boxcar_widths(bc, mwp);
    const std::vector<PdPlan> pd = spd_pd_plan(bc, nTimesamples);
    if (nwidths)
        *nwidths = static_cast<int>(w.size());
    if (max_width_performed)
        *max_width_performed = mwp;
    if (max_iteration)
        *max_iteration = it;
    if (widths)
        for (int i = 0; i < static_cast<int>(w.size()) && i < widths_cap; ++i)
            widths[i] = w[i];
    if (nplan)
        *nplan = static_cast<int>(pd.size());
    if (plan)
        for (int i = 0; i < static_cast<int>(pd.size()) && i < plan_cap; ++i) {
            const PdPlan &q = pd[i];
            const int v[10] = {q.decimated_timesamples, q.dtm, q.iteration, q.nBoxcars, q.nBlocks,
                               q.output_shift, q.shift, q.startTaps, q.unprocessed_samples, q.total_ut};
            for (int k = 0; k < 10; ++k)
                plan[10 * i + k] = v[k];
        }
    return 0;
}

// src/aa_device_analysis.cu:420-466: float records (DM, time, S/N, width) --
// DM = trial * dm_step + dm_low, time = sample * tsamp + tstart (tsamp of
// the range), width = boxcar width * inBin -- in a file named
// "peak_analysed-t_%.2f-dm_%.2f-%.2f.dat" (algorithms 0 and 2) or
// "analysed-..." (algorithm 1) after tstart, dm_low and dm_high, under dir
// (the working directory when dir is null or empty).  Nothing is written for
// no candidates.  Returns 0, or 1 when the file could not be written.
int aa_b200_spd_write_candidates(const char *dir, int candidate_algorithm, float tstart, float dm_low, float dm_high,
                                 float dm_step, float tsamp, int inBin, const unsigned *dm, const unsigned *ts,
                                 const float *snr, const unsigned *bw, size_t n)
{
    if (n == 0)
        return 0;
    char name[256];
    std::snprintf(name, sizeof(name), "%s-t_%.2f-dm_%.2f-%.2f.dat",
                  candidate_algorithm == 1 ? "analysed" : "peak_analysed", tstart, dm_low, dm_high);
    std::string path = (dir && *dir) ? std::string(dir) + "/" + name : std::string(name);
    float *rec = new (std::nothrow) float[4 * n];
    if (!rec) {
        g_spd_error = "single-pulse detection: out of host memory";
        return 1;
    }
    for (size_t i = 0; i < n; ++i) {
        rec[4 * i] = static_cast<float>(static_cast<double>(dm[i]) * dm_step + dm_low);
        rec[4 * i + 1] = static_cast<float>(static_cast<double>(ts[i]) * tsamp + tstart);
        rec[4 * i + 2] = static_cast<float>(static_cast<double>(snr[i]));
        rec[4 * i + 3] = static_cast<float>(static_cast<double>(bw[i]) * inBin);
    }
    FILE *fp = std::fopen(path.c_str(), "wb");
    int rc = 0;
    if (!fp || std::fwrite(rec, n * sizeof(float), 4, fp) != 4) {
        g_spd_error = "single-pulse detection: cannot write " + path;
        rc = 1;
    }
    if (fp)
        std::fclose(fp);
    delete[] rec;
    return rc;
}

} // extern "C"
