// spd.cuh -- single-pulse detection on a DM-time plane, the reference's
// analysis component (src/aa_device_analysis.cu:130-345):
//   * a mean and deviation of the plane per boxcar width (decimations in
//     time, block-wise streaming statistics merged pairwise, optional outlier
//     rejection, linear interpolation over widths),
//   * boxcar S/N planes for widths up to the plan's maximum, in iterations
//     that each halve the time resolution,
//   * candidates: local maxima over 3 x 3 neighbourhoods above the cut, or
//     every sample above it.
// The float expressions, the reduction trees of the reference's thread
// blocks and the way its S/N kernels share partial sums between threads
// decide which candidates pass, so they are kept operation for operation.
#pragma once

#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace aab200 {

// src/aa_params.hpp values the plan depends on
constexpr int SPD_NTHREADS = 512; // PD_NTHREADS
constexpr int SPD_MAXTAPS = 32;   // PD_MAXTAPS

// include/aa_device_BC_plan.hpp:12-23
struct PdPlan {
    int decimated_timesamples, dtm, iteration, nBoxcars, nBlocks, output_shift, shift, startTaps,
        unprocessed_samples, total_ut;
};

// Partial statistics area of one MSD call: [blocks][5] (M, S, j, max, min).
struct MsdConf {
    int nBlocks_x, nBlocks_y, nSteps_y, nBlocks_total, final_threads;
    long long nTimesamples, nDMs, offset;
};
MsdConf msd_conf(long long nTimesamples, long long nDMs, long long offset);

// d_msd[3] = (mean, deviation, count) of input [nDMs][nTimesamples], the last
// `offset` samples of each row left out; partials needs 5 * nBlocks_total
// floats.  d_pp (continuous form, may be null) carries (M, S, j) of earlier
// calls and is updated.
cudaError_t msd_plane(float *d_msd, const float *d_input, float *d_partials, const MsdConf &c, bool outlier_rejection,
                      float sigma, float *d_pp, cudaStream_t st);
// out [nDMs][nT/2]: pairwise sums of consecutive samples of rows 0 .. 2*(nDMs/2)-1
cudaError_t dit_pairs(const float *d_in, float *d_out, int nDMs, int nT, cudaStream_t st);
// out[y][x] = sum of in[y][x .. x+nTaps-1] for x < nT - nTaps + 1 (row stride nT)
cudaError_t fir_rows(const float *d_in, float *d_out, int nDMs, int nT, int nTaps, cudaStream_t st);
cudaError_t msd_interpolate(const float *d_msd_dit, float *d_msd_interp, const int *d_dit_widths, int n_dit,
                            const int *d_widths, int n_widths, int max_width_performed, cudaStream_t st);
// (mean, deviation) of the boxcar widths one S/N plane uses, passed to the
// kernels by value (constant-bank operands instead of loads)
struct SnrMsd {
    float2 v[SPD_MAXTAPS];
};
// nBoxcars: 8, 16 or 32 (the plan's widths per iteration)
cudaError_t spdt_first_plane(const float *d_input, float *d_bv_out, float *d_decimated, float *d_snr, uint16_t *d_taps,
                             const SnrMsd &msd, int nTimesamples, int nBoxcars, int dtm, int nBlocks, int nDMs,
                             cudaStream_t st);
cudaError_t spdt_nth_plane(const float *d_input, const float *d_bv_in, float *d_bv_out, float *d_decimated,
                           float *d_snr, uint16_t *d_taps, const SnrMsd &msd, int nTimesamples, int nBoxcars,
                           int startTaps, int dit_value, int dtm, int nBlocks, int nDMs, cudaStream_t st);
// Candidate lists (dm, ts, snr, bw), appended at *d_count (atomic).
cudaError_t spd_peak_find(const float *d_snr, const uint16_t *d_taps, unsigned *d_dm, unsigned *d_ts, float *d_csnr,
                          unsigned *d_bw, int width, int height, int offset, float threshold, int max_cands,
                          int *d_count, int shift, int dit_value, cudaStream_t st);
// peak filtering: the 7 x 7 stencil peaks of one S/N plane, then the
// filter over the whole list (max_distance: squared distance in trials and samples)
cudaError_t spd_peak_find_7x7(const float *d_snr, const uint16_t *d_taps, unsigned *d_dm, unsigned *d_ts, float *d_csnr,
                              unsigned *d_bw, int width, int height, int offset, float threshold, int max_cands,
                              int *d_count, int shift, int dit_value, cudaStream_t st);
cudaError_t spd_filter_peaks(const unsigned *d_dm, const unsigned *d_ts, const unsigned *d_bw, const float *d_snr,
                             int n, unsigned max_distance, unsigned *o_dm, unsigned *o_ts, unsigned *o_bw,
                             float *o_snr, int max_cands, int *d_count, cudaStream_t st);
cudaError_t spd_threshold(const float *d_snr, const uint16_t *d_taps, unsigned *d_dm, unsigned *d_ts, float *d_csnr,
                          unsigned *d_bw, int *d_count, float threshold, int nTimesamples, int offset, int shift,
                          int max_cands, int dit_value, int nDMs, cudaStream_t st);

// kernels these launchers have started in this process
long long spd_kernel_launches();

// Host side (spd_plane.cpp) -------------------------------------------------------

// The analysis settings of include/aa_analysis_plan.hpp plus the range's
// sampling; candidate_algorithm 0 peak finding, 1 thresholding, 2 peak
// filtering.
struct SpdSettings {
    float sigma_cutoff = 6.f;
    float sigma_constant = 3.f;          // outlier-rejection multiplier
    float max_boxcar_width_in_sec = 0.f;
    int candidate_algorithm = 0;
    int enable_msd_baseline_noise = 0;   // outlier rejection in the MSD
};

struct SpdCandidates {
    std::vector<unsigned> dm, ts, bw; // DM trial index, sample, boxcar width (samples of the range)
    std::vector<float> snr;
};

class SpdPlane {
  public:
    // Buffers for planes of up to max_elems (nDMs * nT) elements.  The
    // boxcar search takes the DM trials in batches of
    // floor(max_time_samples / nT) rounded down to a multiple of 4, the
    // rest last (the reference's maxTimeSamples; 0 = no limit, the whole
    // plane in one batch); the 3 x 3 peak neighbourhoods end at batch edges,
    // as in the reference.
    bool setup(long long max_elems, long long max_time_samples, std::string &err);
    void release();
    ~SpdPlane() { release(); }
    // Runs the analysis on d_plane [nDMs][nT] (device, overwritten as the
    // reference's search overwrites its input).  tsamp is the range's
    // sampling time (tsamp of the data times inBin).
    // Candidates are appended to `out` up to host_capacity entries in total,
    // a batch that would pass it being dropped whole (the reference's
    // "peak list is too small" rule).
    bool run(float *d_plane, int nDMs, int nT, float tsamp, int inBin, const SpdSettings &s, SpdCandidates &out,
             cudaStream_t st, std::string &err, size_t host_capacity = SIZE_MAX);
    // zero the whole work area (the state of a fresh allocation)
    cudaError_t clear(cudaStream_t st);
    // The MSD plane profile alone on [nDMs][nT] for the given ascending
    // widths (high_memory: the width-2 decimation in one piece, as the
    // periodicity search runs it); the result in last_msd.
    bool profile(const float *d_input, int nDMs, int nT, const std::vector<int> &widths, bool high_memory,
                 float sigma_constant, bool outlier_rejection, cudaStream_t st, std::string &err);
    // intermediate results of the last run (for tests)
    std::vector<float> last_msd;
    std::vector<int> last_widths;
    int last_max_width_performed = 0, last_max_iteration = 0;
    bool keep_planes = false;
    int dropped_batches = 0; // batches whose candidates did not fit host_capacity
    // Device time per launch family of the last run, from CUDA events around
    // each launch when time_kernels is on: 0 MSD statistics, 1 decimations
    // and boxcars of the MSD profile, 2 first boxcar S/N plane, 3 later S/N
    // planes, 4 candidates.
    static constexpr int kFamilies = 5;
    bool time_kernels = false;
    double family_ms[kFamilies] = {0, 0, 0, 0, 0};
    long long family_n[kFamilies] = {0, 0, 0, 0, 0};
    std::vector<float> last_snr;
    std::vector<uint16_t> last_taps;

  private:
    bool msd_profile(const float *d_input, int nDMs, int nT, const std::vector<int> &widths, const SpdSettings &s,
                     cudaStream_t st, std::string &err, bool high_memory = false);
    bool filter_peaks(SpdCandidates &out, size_t b, float tsamp, cudaStream_t st, std::string &err);
    void t_begin(int family, cudaStream_t st);
    void t_end(cudaStream_t st);
    bool t_collect();
    std::vector<cudaEvent_t> ev_pool_;
    std::vector<int> ev_family_;
    size_t ev_used_ = 0;
    float *d_work_ = nullptr, *d_msd_interp_ = nullptr;
    uint16_t *d_taps_ = nullptr;
    int *d_count_ = nullptr, *d_dit_widths_ = nullptr, *d_widths_ = nullptr;
    long long max_elems_ = 0, max_ts_ = 0;
    size_t work_floats_ = 0, taps_elems_ = 0;
};

// include/aa_device_BC_plan.hpp users in src/aa_device_analysis.cu:24-121
std::vector<int> spd_bc_widths();
int spd_max_iteration(int max_boxcar_width, const std::vector<int> &bc, int &max_width_performed);
std::vector<PdPlan> spd_pd_plan(const std::vector<int> &bc, int nTimesamples);
std::vector<int> spd_boxcar_widths(const std::vector<int> &bc, int max_boxcar_width);

} // namespace aab200
