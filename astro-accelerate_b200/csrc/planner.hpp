// planner.hpp -- DM plan, filterbank metadata and the DDTR strategy.
//
// Source-level mirror of the reference's planning surface:
//   aa_ddtr_plan            include/aa_ddtr_plan.hpp:17-159
//   aa_filterbank_metadata  include/aa_filterbank_metadata.hpp:150-180 (reduced ctor)
//   aa_ddtr_strategy        include/aa_ddtr_strategy.hpp:33-228, src/aa_ddtr_strategy.cpp:27-428
// The strategy arithmetic (delay table, DM-grid redefinition, maxshift,
// time chunking, memory accounting) has to stay bit-identical to the
// reference because it decides every delay and every chunk boundary; it is
// restated here in this project's own C++.
#pragma once
#include <cstddef>
#include <string>
#include <vector>

namespace aab200 {

struct DmRange {
    float low;
    float high;
    float step;
    int inBin;
    int outBin; // deprecated in the reference, carried through unchanged
};

class DdtrPlan {
public:
    bool add_dm(float low, float high, float step, int inBin, int outBin)
    {
        ranges_.push_back(DmRange{low, high, step, inBin, outBin});
        return true;
    }
    size_t range() const { return ranges_.size(); }
    DmRange user_dm(size_t i) const { return i < ranges_.size() ? ranges_[i] : DmRange{0.f, 0.f, 0.f, 0, 0}; }
    bool set_power(float p)
    {
        power_ = p;
        return true;
    }
    float power() const { return power_; }
    bool set_enable_msd_baseline_noise(bool f)
    {
        msd_baseline_ = f;
        return true;
    }
    bool enable_msd_baseline_noise() const { return msd_baseline_; }
    bool bind_bandpass_normalization(const float *v, int n)
    {
        if (n <= 0)
            return false;
        bandpass_.assign(v, v + n);
        return true;
    }
    const std::vector<float> &bandpass() const { return bandpass_; }

private:
    std::vector<DmRange> ranges_;
    float power_ = 2.0f; // include/aa_ddtr_plan.hpp:20
    bool msd_baseline_ = false;
    std::vector<float> bandpass_;
};

struct FilterbankMetadata {
    double tstart = 0.0;
    double tsamp = 0.0;
    double fch1 = 0.0;
    double foff = 0.0;
    int nbits = 8;
    int nsamples = 0;
    int nchans = 0;
};

// Reasons a strategy is refused (the reference logs them and returns false).
enum StrategyStatus : int {
    STRAT_OK = 0,
    STRAT_NO_RANGES = -1,     // :63-66
    STRAT_MAXSHIFT = -2,      // :146-149 maxshift >= nsamp
    STRAT_MEMORY = -3,        // :182-185, :291-294
    STRAT_REQUEST = -4,       // :405-414
};

class DdtrStrategy {
public:
    DdtrStrategy() = default;
    // free_memory: bytes the device offers (aa_device_info::free_memory()).
    StrategyStatus compute(const DdtrPlan &plan, const FilterbankMetadata &meta, size_t free_memory,
                           bool enable_analysis);

    bool ready() const { return ready_; }
    // computed with room for the analysis component (aa_ddtr_strategy::configured_for_analysis)
    bool configured_for_analysis() const { return analysis_; }
    int maxshift() const { return maxshift_; }
    int max_ndms() const { return max_ndms_; }
    int num_tchunks() const { return num_tchunks_; }
    size_t nranges() const { return dm_.size(); }
    int ndms(size_t i) const { return ndms_[i]; }
    const int *ndms_data() const { return ndms_.data(); }
    const DmRange &dm(size_t i) const { return dm_[i]; }
    const std::vector<float> &dmshifts() const { return dmshifts_; }
    const std::vector<std::vector<int>> &t_processed() const { return t_processed_; }
    float power() const { return power_; }
    const FilterbankMetadata &metadata() const { return meta_; }
    long long total_samps(size_t r) const
    {
        long long s = 0;
        for (int v : t_processed_[r])
            s += v;
        return s;
    }
    size_t nProcessedTimesamples() const
    {
        size_t s = 0;
        if (!t_processed_.empty())
            for (int v : t_processed_[0])
                s += static_cast<size_t>(v);
        return s;
    }

private:
    bool ready_ = false;
    bool analysis_ = false;
    FilterbankMetadata meta_;
    float power_ = 2.0f;
    std::vector<float> dmshifts_;
    std::vector<int> ndms_;
    std::vector<DmRange> dm_;
    int maxshift_ = 0;
    int max_ndms_ = 0;
    int num_tchunks_ = 0;
    std::vector<std::vector<int>> t_processed_;
};

// Kernel the reference's dedisperse() dispatches a range to
// (src/aa_dedisperse.cpp:8-11,20 / :48-51,62 / :88-92,101 / :133-155).
int select_delay_kind(int nbits, float dm_step, float tsamp_r, float dmshift_last, int failsafe);

} // namespace aab200
