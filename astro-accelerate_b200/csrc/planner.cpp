// planner.cpp -- DDTR strategy (src/aa_ddtr_strategy.cpp:27-428 restated).
//
// Compiled without floating-point contraction so that every float expression
// rounds like the reference's host build (x86-64 SSE, -O3, no FMA).  Each
// expression keeps the reference's operand types and evaluation order; the
// comments give the line it follows.
#include "planner.hpp"

#include <cmath>
#include <cstdint>

namespace aab200 {

namespace {

constexpr int kSdivint = 8;   // include/aa_params.hpp:96
constexpr int kSdivindm = 64; // :97
constexpr int kSnumreg = 14;  // :95
constexpr size_t kMaxOutputBytes = 17179869184ULL; // src/aa_ddtr_strategy.cpp:7
constexpr size_t kReservedBytes = 104857600;       // :72

// Time-sample granularity of the shared kernels: 224 (8/16-bit), 448 (4-bit).
inline int sample_unit(int nbits) { return (nbits == 4 ? 4 : 2) * kSdivint * kSnumreg; }

// floor((x / bin) / unit) in float, the form used for every chunk length
// except the case-1 common length (:194-197, :203-205, :222-228, :245-256).
inline int floor_units_f(float x, int bin, int unit)
{
    return static_cast<int>(std::floor(static_cast<double>((x / static_cast<float>(bin)) / static_cast<float>(unit))));
}

// Delay at the top of a range over one sample (:117, :130, :138).
inline int ceil_delay(float low, float step, int ndms, float dmshift_last, float tsamp)
{
    const float top = low + step * static_cast<float>(ndms);
    return static_cast<int>(std::ceil(static_cast<double>((top * dmshift_last) / tsamp)));
}

// Rounds a binned range's delay up to the kernel's sample unit (:119-121).
inline int round_binned_maxshift(int ms, int inBin)
{
    const float modulo = static_cast<float>(kSdivint * 2 * kSnumreg);
    int m = static_cast<int>((static_cast<float>(ms) / static_cast<float>(inBin) + modulo) / modulo);
    return m * (kSdivint * 2 * kSnumreg) * inBin;
}

} // namespace

StrategyStatus DdtrStrategy::compute(const DdtrPlan &plan, const FilterbankMetadata &meta, size_t free_memory,
                                     bool enable_analysis)
{
    ready_ = false;
    analysis_ = enable_analysis;
    meta_ = meta;
    power_ = plan.power();
    const int nchans = meta.nchans;
    const int nsamp = meta.nsamples;
    const float fch1 = static_cast<float>(meta.fch1);
    const float foff = static_cast<float>(meta.foff);
    const float tsamp = static_cast<float>(meta.tsamp);
    const int nbits = meta.nbits;
    const size_t nr = plan.range();
    if (nr == 0)
        return STRAT_NO_RANGES;

    // :81-92 per-channel delay constants
    dmshifts_.assign(nchans, 0.f);
    for (int c = 0; c < nchans; ++c) {
        const float fc = fch1 + (foff * static_cast<float>(c));
        double inv_c, inv_1;
        if (power_ != 2.0) {
            inv_c = 1.0 / static_cast<double>(std::pow(fc, power_));
            inv_1 = 1.0 / static_cast<double>(std::pow(fch1, power_));
        } else {
            inv_c = 1.0 / std::pow(static_cast<double>(fc), static_cast<double>(power_));
            inv_1 = 1.0 / std::pow(static_cast<double>(fch1), static_cast<double>(power_));
        }
        dmshifts_[c] = static_cast<float>(static_cast<double>(4148.741601f) * (inv_c - inv_1));
    }

    // :94-101 DM trials per range, whole 64-trial blocks
    ndms_.assign(nr, 0);
    max_ndms_ = 0;
    for (size_t i = 0; i < nr; ++i) {
        const DmRange u = plan.user_dm(i);
        const int whole = static_cast<int>((u.high - u.low) / u.step);
        ndms_[i] = ((whole + kSdivindm) / kSdivindm) * kSdivindm;
        if (ndms_[i] > max_ndms_)
            max_ndms_ = ndms_[i];
    }

    // :104-135 contiguous grid; binned ranges round their delay up
    dm_.assign(nr, DmRange{});
    const float shift_last = dmshifts_[nchans - 1];
    int maxshift_high = 0;
    dm_[0].low = plan.user_dm(0).low;
    dm_[0].high = dm_[0].low + (static_cast<float>(ndms_[0]) * plan.user_dm(0).step);
    dm_[0].step = plan.user_dm(0).step;
    for (size_t i = 1; i < nr; ++i) {
        dm_[i].low = dm_[i - 1].high;
        dm_[i].high = dm_[i].low + static_cast<float>(ndms_[i]) * plan.user_dm(i).step;
        dm_[i].step = plan.user_dm(i).step;
        const int prev_bin = plan.user_dm(i - 1).inBin;
        if (prev_bin > 1) {
            int ms = ceil_delay(dm_[i - 1].low, dm_[i - 1].step, ndms_[i - 1], shift_last, tsamp);
            ms = round_binned_maxshift(ms, prev_bin);
            if (ms > maxshift_high)
                maxshift_high = ms;
        }
    }
    const int last_bin = plan.user_dm(nr - 1).inBin;
    if (last_bin > 1) {
        int ms = ceil_delay(dm_[nr - 1].low, dm_[nr - 1].step, ndms_[nr - 1], shift_last, tsamp);
        ms = round_binned_maxshift(ms, last_bin);
        if (ms > maxshift_high)
            maxshift_high = ms;
    }
    if (maxshift_high == 0) // :137-139
        maxshift_high = ceil_delay(dm_[nr - 1].low, dm_[nr - 1].step, ndms_[nr - 1], shift_last, tsamp);
    maxshift_ = maxshift_high + kSnumreg * 2 * kSdivint; // :142
    if (maxshift_ >= nsamp)
        return STRAT_MAXSHIFT;

    // :156-389 chunking.  The output of one chunk must fit the device and
    // 16 GiB; the input row length then sets the common chunk length.
    const size_t gpu_memory = free_memory - kReservedBytes;
    const int unit = sample_unit(nbits);
    const size_t spdt = enable_analysis
                            ? static_cast<size_t>(static_cast<double>(sizeof(float) * static_cast<size_t>(max_ndms_)) * 0.75)
                            : 0;
    const bool out_wider = nchans < max_ndms_;
    const size_t out_rows = out_wider ? static_cast<size_t>(max_ndms_) : static_cast<size_t>(nchans);
    unsigned int max_tsamps;
    if (out_wider)
        max_tsamps = static_cast<unsigned int>(gpu_memory / (sizeof(unsigned short) * static_cast<size_t>(nchans) +
                                                             sizeof(float) * static_cast<size_t>(max_ndms_) + spdt));
    else
        max_tsamps = static_cast<unsigned int>(gpu_memory / (static_cast<size_t>(nchans) * (sizeof(float) + sizeof(unsigned short)) + spdt));
    if (static_cast<size_t>(max_tsamps) * sizeof(float) * out_rows > kMaxOutputBytes)
        max_tsamps = static_cast<unsigned int>(kMaxOutputBytes / (sizeof(float) * out_rows));
    if (out_wider ? (static_cast<unsigned int>(maxshift_) > max_tsamps) : (maxshift_ > static_cast<int>(max_tsamps)))
        return STRAT_MEMORY;

    t_processed_.assign(nr, std::vector<int>());
    if (static_cast<unsigned int>(nsamp) < max_tsamps) {
        // one chunk (cases 1 and 2)
        long long common;
        if (out_wider) {
            // case 1 works in double precision (:191-197)
            unsigned long lt = static_cast<unsigned long>(std::floor(
                (static_cast<double>(nsamp - maxshift_) / static_cast<double>(last_bin)) / static_cast<double>(unit)));
            common = static_cast<long long>(lt * static_cast<unsigned long>(unit) * static_cast<unsigned long>(last_bin));
        } else {
            common = static_cast<long long>(floor_units_f(static_cast<float>(nsamp - maxshift_), last_bin, unit)) * unit * last_bin;
        }
        for (size_t i = 0; i < nr; ++i)
            t_processed_[i].push_back(floor_units_f(static_cast<float>(common), plan.user_dm(i).inBin, unit) * unit);
        num_tchunks_ = 1;
    } else {
        // several chunks (cases 3 and 4, :209-274 / :324-388)
        const int block = static_cast<int>(max_tsamps) - maxshift_;
        const int common = floor_units_f(static_cast<float>(block), last_bin, unit) * unit * last_bin;
        if (common <= 0) // the reference divides by zero here
            return STRAT_MEMORY;
        const int nblocks = static_cast<int>(static_cast<float>(nsamp - maxshift_) / static_cast<float>(common));
        int rest = nsamp - (nblocks * common) - maxshift_;
        // (int)floor(rest/bin) / (float)unit, truncated on assignment
        rest = static_cast<int>(static_cast<float>(static_cast<int>(std::floor(
                                    static_cast<double>(static_cast<float>(rest) / static_cast<float>(last_bin))))) /
                                static_cast<float>(unit));
        rest = rest * unit * last_bin;
        const int extra = rest > 0 ? 1 : 0;
        for (size_t i = 0; i < nr; ++i) {
            const int inBin = plan.user_dm(i).inBin;
            for (int j = 0; j < nblocks; ++j)
                t_processed_[i].push_back(floor_units_f(static_cast<float>(common), inBin, unit) * unit);
            if (extra)
                t_processed_[i].push_back(floor_units_f(static_cast<float>(rest), inBin, unit) * unit);
        }
        num_tchunks_ = nblocks + extra;
    }

    // :401-415 the device must hold one chunk's input and output
    {
        size_t available = free_memory;
        auto request = [&available](size_t bytes) {
            if (available > bytes) {
                available -= bytes;
                return true;
            }
            return false;
        };
        const size_t samps = static_cast<size_t>(t_processed_[0][0] + maxshift_);
        request(samps * static_cast<size_t>(nchans) * sizeof(unsigned short));
        if (!request(samps * out_rows * sizeof(float)))
            return STRAT_REQUEST;
    }

    for (size_t i = 0; i < nr; ++i) { // :420-423
        dm_[i].inBin = plan.user_dm(i).inBin;
        dm_[i].outBin = plan.user_dm(i).outBin;
    }
    ready_ = true;
    return STRAT_OK;
}

int select_delay_kind(int nbits, float dm_step, float tsamp_r, float dmshift_last, int failsafe)
{
    // KIND_SHARED8 = 0, KIND_SHARED16 = 1, KIND_SHARED4 = 2, KIND_CACHE = 3
    const int limit = (kSdivint - 1) + ((kSdivindm - 1) * kSdivint) - 1;
    if (failsafe != 0)
        return 3;
    const int lanes = (nbits == 4) ? 4 : 2;
    const float shift_one = static_cast<float>(kSdivindm - 1) * (dm_step / tsamp_r);
    const int shifta = static_cast<int>(std::floor(shift_one * dmshift_last)) + (kSdivint - 1) * lanes;
    const int lineshift = shifta + ((kSnumreg - 1) * lanes * kSdivint);
    if (limit > lineshift)
        return (nbits == 16 || nbits == 32) ? 1 : (nbits == 4 ? 2 : 0);
    return 3;
}

} // namespace aab200
