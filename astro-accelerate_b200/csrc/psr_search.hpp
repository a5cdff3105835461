// psr_search.hpp -- the periodicity component of the pipeline: the
// reference's periodicity strategy (aa_periodicity_strategy,
// include/aa_periodicity_strategy.hpp:62-541, with the plan of
// include/aa_periodicity_plan.hpp:20-328) and its search over the DM-time
// output of every range (GPU_periodicity / Periodicity_search,
// src/aa_device_periods.cu:368-682).
//
// Per range and batch of DM trials: the first nTimesamples samples of each
// row (a power of two at most the processed length, divided by the range's
// binning), a real-to-complex FFT (cuFFT, the plan the reference makes),
// spectral whitening, power and interbin spectra, the MSD plane profile of
// the power spectra for 1..nHarmonics summed bins, the harmonic sum of the
// chosen algorithm, peak finding or thresholding, and the candidate records
// converted with the batch's MSD into the power and interbin lists.  The
// stages are this library's kernels (psr.cu, spd.cu), bit-identical to the
// reference's where the reference is deterministic.
#pragma once

#include <cstddef>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace aab200 {

// aa_periodicity_plan's parameters (include/aa_periodicity_plan.hpp:20-89)
struct PsrPlanParams {
    float sigma_cutoff = 10.f;
    bool enable_outlier_rejection = true;
    float sigma_outlier_rejection_threshold = 3.f;
    int nHarmonics = 32;
    int harmonic_sum_algorithm = 1; // 0 simple, 1 greedy, 2 PRESTO plus, 3 PRESTO
    int candidate_selection_algorithm = 0; // 0 peak finding, 1 thresholding
    bool enable_scalloping_loss_mitigation = true;
    bool enable_interbinning = true;
    bool enable_spectrum_whitening = true;
};

// aa_dedispersion_range as the plan takes it from the DDTR strategy
// (include/aa_periodicity_plan.hpp:292-321)
struct PsrDdtrRange {
    double dm_low = 0, dm_high = 0, dm_step = 0;
    int inBin = 1;
    size_t nTimesamples = 0; // processed samples of the whole run, before binning
    int nDMs = 0;
    double sampling_time = 0; // before binning
};

// aa_periodicity_batch (include/aa_periodicity_strategy.hpp:25-51)
struct PsrBatch {
    size_t nDMs_per_batch = 0, nTimesamples = 0, nTimesamples_to_copy = 0, DM_shift = 0;
};

// aa_periodicity_range (include/aa_periodicity_strategy.hpp:60-117):
// range.nTimesamples is the FFT length after binning
struct PsrRange {
    PsrDdtrRange range;
    int rangeid = 0;
    std::vector<PsrBatch> batches;
    size_t total_MSD_blocks = 0;
};

struct PsrStrategy {
    PsrPlanParams plan;
    size_t max_nTimesamples = 0, corrected_max_nTimesamples = 0, nTimesamples_to_copy = 0;
    size_t max_nDMs = 0, max_nDMs_in_memory = 0, input_plane_size = 0, cufft_workarea_size = 0;
    size_t max_total_MSD_blocks = 0;
    std::vector<PsrRange> ranges;
};

// The strategy for memory_available bytes (the reference takes the device's
// free memory when the plan is bound).  Returns false with err when no DM
// trial fits or the parameters are invalid.
bool psr_strategy(const PsrPlanParams &plan, const std::vector<PsrDdtrRange> &ranges, size_t memory_available,
                  PsrStrategy &out, std::string &err);

// Where the search reads a range's DM-time rows: row d at base + d * pitch
// floats, row_len samples valid; host rows (pinned) or device rows.
struct PsrRows {
    const float *base = nullptr;
    long long pitch = 0, row_len = 0;
    bool on_device = false;
};

class PsrSearch {
  public:
    PsrSearch() = default;
    PsrSearch(const PsrSearch &) = delete;
    PsrSearch &operator=(const PsrSearch &) = delete;
    ~PsrSearch() { release(); }

    // device buffers for the strategy's largest batch
    bool setup(const PsrStrategy &s, std::string &err);
    void release();
    // The search over every range of the strategy; records are appended to
    // power_list and interbin_list (aa_b200_psr_candidates_* objects).
    bool run(const PsrStrategy &s, const std::vector<PsrRows> &rows, void *power_list, void *interbin_list,
             cudaStream_t st, std::string &err);
    // the last batch's (mean, deviation) per harmonic count
    std::vector<float> last_msd;
    // device time of the last run (ms, CUDA events around each batch's
    // stages after its input copy) and its batches
    double last_compute_ms = 0;
    int last_batches = 0;

  private:
    bool batch(const PsrStrategy &s, const PsrRange &R, const PsrBatch &b, const PsrRows &rows, void *power_list,
               void *interbin_list, cudaStream_t st, std::string &err);
    size_t plane_ = 0; // floats of the largest input plane (nDMs x nTimesamples)
    float *d_in_ = nullptr, *d_spec_ = nullptr, *d_power_ = nullptr, *d_inter_ = nullptr;
    float *d_power_ct_ = nullptr, *d_inter_ct_ = nullptr, *d_snr_p_ = nullptr, *d_snr_i_ = nullptr;
    float *d_list_p_ = nullptr, *d_list_i_ = nullptr, *d_msd_ = nullptr;
    unsigned short *d_harm_p_ = nullptr, *d_harm_i_ = nullptr;
    int *d_count_ = nullptr;
    void *d_cufft_work_ = nullptr;
    size_t cufft_work_bytes_ = 0;
    long long max_list_ = 0; // candidate records each list holds
    void *msd_ = nullptr;    // SpdPlane for the MSD plane profile
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
};

} // namespace aab200
