// psr_search.cpp -- the periodicity component (see psr_search.hpp).
#include "psr_search.hpp"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

#include <cufft.h>

#include "aa_b200.h"
#include "psr.cuh"
#include "spd.cuh"

namespace aab200 {

namespace {

constexpr int kPhsThreads = 64;      // PHS_NTHREADS, include/aa_params.hpp:68
constexpr int kMsdPartialSize = 5;   // MSD_PARTIAL_SIZE, include/aa_params.hpp:29
constexpr int kMsdResultsSize = 3;   // MSD_RESULTS_SIZE, include/aa_params.hpp:30

// include/aa_periodicity_strategy.hpp:226-243, in its types: the memory per
// DM trial is a float product, the division a double one, the result an int
// rounded down to a multiple of PHS_NTHREADS (up to the largest range's
// trials rounded up, when those fit)
int max_nDMs_in_memory(size_t memory_available, size_t corrected, size_t max_nDMs)
{
    const float per_value = 5.5f * static_cast<float>(sizeof(float)) + 2.0f * static_cast<float>(sizeof(uint16_t));
    const float per_dm = static_cast<float>(corrected + 2) * per_value;
    size_t t = static_cast<size_t>((static_cast<double>(memory_available) * 0.98) / static_cast<double>(per_dm));
    size_t itemp;
    if (max_nDMs + kPhsThreads < t) {
        itemp = static_cast<size_t>(static_cast<int>(max_nDMs / kPhsThreads));
        if (max_nDMs % kPhsThreads > 0)
            ++itemp;
        t = itemp * kPhsThreads;
    }
    itemp = static_cast<size_t>(static_cast<int>(t / kPhsThreads));
    t = itemp * kPhsThreads;
    return static_cast<int>(t);
}

// MSD_Configuration(nTimesamples, nDMs, 0, 0).nBlocks_total
// (include/aa_device_MSD_Configuration.hpp:67-80)
size_t msd_blocks(size_t nTimesamples, size_t nDMs)
{
    return static_cast<size_t>(msd_conf(static_cast<long long>(nTimesamples), static_cast<long long>(nDMs), 0)
                                   .nBlocks_total);
}

// aa_periodicity_range::Create_Batches (include/aa_periodicity_strategy.hpp:70-87)
void create_batches(PsrRange &R, size_t max_nDMs_in_range, size_t nTimesamples_to_copy)
{
    R.total_MSD_blocks = 0;
    const size_t nDMs = static_cast<size_t>(R.range.nDMs);
    const int nRepeats = static_cast<int>(nDMs / max_nDMs_in_range);
    const int nRest = static_cast<int>(nDMs - nRepeats * max_nDMs_in_range);
    auto add = [&](size_t n, size_t shift) {
        PsrBatch b;
        b.nDMs_per_batch = n;
        b.DM_shift = shift;
        b.nTimesamples = R.range.nTimesamples;
        b.nTimesamples_to_copy = nTimesamples_to_copy;
        R.batches.push_back(b);
        // MSD over the power spectra of N/2 + 1 bins
        R.total_MSD_blocks = std::max(R.total_MSD_blocks, msd_blocks((b.nTimesamples >> 1) + 1, n));
    };
    for (int f = 0; f < nRepeats; ++f)
        add(max_nDMs_in_range, static_cast<size_t>(f) * max_nDMs_in_range);
    if (nRest > 0)
        add(static_cast<size_t>(nRest), static_cast<size_t>(nRepeats) * max_nDMs_in_range);
}

bool cuda_ok(cudaError_t e, const char *what, std::string &err)
{
    if (e == cudaSuccess)
        return true;
    err = std::string("periodicity search: ") + what + ": " + cudaGetErrorString(e);
    return false;
}

bool cufft_ok(cufftResult r, const char *what, std::string &err)
{
    if (r == CUFFT_SUCCESS)
        return true;
    err = std::string("periodicity search: ") + what + ": cuFFT error " + std::to_string(static_cast<int>(r));
    return false;
}

} // namespace

// include/aa_periodicity_strategy.hpp:178-224 (plan parameters and the FFT
// length: the largest processed length rounded down to a power of two, as
// pad_to_nearest_higher_pow2 is forced off), :245-257 (ranges), :259-291
// (cuFFT work area: nDMs * nTimesamples * 8 bytes of the largest batch),
// :307-355 (the memory loop)
bool psr_strategy(const PsrPlanParams &plan, const std::vector<PsrDdtrRange> &ranges, size_t memory_available,
                  PsrStrategy &out, std::string &err)
{
    out = PsrStrategy();
    out.plan = plan;
    if (ranges.empty()) {
        err = "periodicity strategy: no DM ranges";
        return false;
    }
    if (plan.nHarmonics < 1 || plan.nHarmonics > 32 || plan.sigma_outlier_rejection_threshold <= 0.f) {
        err = "periodicity strategy: nHarmonics 1..32 and a positive outlier-rejection sigma needed";
        return false;
    }
    if (plan.harmonic_sum_algorithm < 0 || plan.harmonic_sum_algorithm > 3) {
        err = "periodicity strategy: harmonic sum algorithm 0..3";
        return false;
    }
    out.max_nTimesamples = ranges[0].nTimesamples;
    out.max_nDMs = static_cast<size_t>(ranges[0].nDMs);
    for (size_t f = 1; f < ranges.size(); ++f) {
        out.max_nTimesamples = std::max(out.max_nTimesamples, ranges[f].nTimesamples);
        out.max_nDMs = std::max(out.max_nDMs, static_cast<size_t>(ranges[f].nDMs));
    }
    if (out.max_nTimesamples < 16) {
        err = "periodicity strategy: too few processed samples";
        return false;
    }
    const float log2n = log2f(static_cast<float>(out.max_nTimesamples));
    const int nearest_lower = static_cast<int>(floorf(log2n));
    out.corrected_max_nTimesamples = static_cast<size_t>(powf(2.0f, static_cast<float>(nearest_lower)));
    out.nTimesamples_to_copy = out.corrected_max_nTimesamples;

    size_t memory_for_data = memory_available;
    size_t memory_allocated = 0;
    do {
        const int m = max_nDMs_in_memory(memory_for_data, out.corrected_max_nTimesamples, out.max_nDMs);
        if (m <= 0) {
            err = "periodicity strategy: not enough memory for one batch of DM trials";
            return false;
        }
        out.max_nDMs_in_memory = static_cast<size_t>(m);
        out.input_plane_size = (out.corrected_max_nTimesamples + 2) * out.max_nDMs_in_memory;
        const float ips = static_cast<float>(out.input_plane_size);
        memory_allocated = static_cast<size_t>(ips * 5.5f * static_cast<float>(sizeof(float)) +
                                               2.0f * ips * static_cast<float>(sizeof(uint16_t)));
        // one periodicity range per DDTR range (the reference appends them
        // again on every pass of this loop; only the first pass's are used)
        out.ranges.clear();
        out.max_total_MSD_blocks = 0;
        for (size_t f = 0; f < ranges.size(); ++f) {
            PsrRange R;
            R.range = ranges[f];
            R.rangeid = static_cast<int>(f);
            const int inBin = std::max(1, ranges[f].inBin);
            R.range.nTimesamples = out.corrected_max_nTimesamples / static_cast<size_t>(inBin);
            create_batches(R, out.max_nDMs_in_memory * static_cast<size_t>(inBin),
                           out.nTimesamples_to_copy / static_cast<size_t>(inBin));
            out.max_total_MSD_blocks = std::max(out.max_total_MSD_blocks, R.total_MSD_blocks);
            out.ranges.push_back(std::move(R));
        }
        out.cufft_workarea_size = 0;
        for (const PsrRange &R : out.ranges)
            for (const PsrBatch &b : R.batches)
                out.cufft_workarea_size = std::max(out.cufft_workarea_size, b.nDMs_per_batch * b.nTimesamples * 8);
        const int nDecimations = static_cast<int>(floorf(log2f(static_cast<float>(plan.nHarmonics)))) + 2;
        const size_t additional = out.max_total_MSD_blocks * kMsdPartialSize * sizeof(float) +
                                  static_cast<size_t>(nDecimations) * 2 * kMsdResultsSize * sizeof(float) +
                                  static_cast<size_t>(plan.nHarmonics) * 2 * sizeof(float) + 2 * sizeof(int);
        memory_allocated += additional;
        if (memory_allocated > memory_available) {
            if (memory_for_data <= additional) {
                err = "periodicity strategy: not enough memory";
                return false;
            }
            memory_for_data -= additional;
        }
    } while (memory_allocated > memory_available);
    return true;
}

void PsrSearch::release()
{
    for (float **p : {&d_in_, &d_spec_, &d_power_, &d_inter_, &d_power_ct_, &d_inter_ct_, &d_snr_p_, &d_snr_i_,
                      &d_list_p_, &d_list_i_, &d_msd_}) {
        cudaFree(*p);
        *p = nullptr;
    }
    cudaFree(d_harm_p_);
    cudaFree(d_harm_i_);
    cudaFree(d_count_);
    cudaFree(d_cufft_work_);
    d_harm_p_ = d_harm_i_ = nullptr;
    d_count_ = nullptr;
    d_cufft_work_ = nullptr;
    delete static_cast<SpdPlane *>(msd_);
    msd_ = nullptr;
    if (ev0_)
        cudaEventDestroy(ev0_);
    if (ev1_)
        cudaEventDestroy(ev1_);
    ev0_ = ev1_ = nullptr;
    plane_ = 0;
}

bool PsrSearch::setup(const PsrStrategy &s, std::string &err)
{
    release();
    size_t max_dms = 0, max_nt = 0;
    for (const PsrRange &R : s.ranges)
        for (const PsrBatch &b : R.batches) {
            max_dms = std::max(max_dms, b.nDMs_per_batch);
            max_nt = std::max(max_nt, b.nTimesamples);
        }
    if (max_dms == 0 || max_nt < 16) {
        err = "periodicity search: empty strategy";
        return false;
    }
    plane_ = max_dms * max_nt;
    const size_t spec = max_dms * ((max_nt >> 1) + 1) * 2;
    // Periodicity_search's list capacity (src/aa_device_periods.cu:374-395):
    // a quarter of the input plane, at most 2^30 records, halved for the
    // transposed planes of the simple harmonic sum
    long long cap = static_cast<long long>(s.input_plane_size / 4);
    if (cap > 1073741824LL)
        cap = 1073741824LL;
    if (s.plan.harmonic_sum_algorithm == 0)
        cap /= 2;
    // records a batch can produce at most: one per value of the plane
    max_list_ = std::max<long long>(1, std::min<long long>(cap, static_cast<long long>(plane_)));
    const bool ct = s.plan.harmonic_sum_algorithm == 0;
    auto alloc = [&](void **p, size_t bytes, const char *what) {
        return cuda_ok(cudaMalloc(p, std::max<size_t>(bytes, 4)), what, err);
    };
    if (!alloc(reinterpret_cast<void **>(&d_in_), plane_ * sizeof(float), "cudaMalloc(input)") ||
        !alloc(reinterpret_cast<void **>(&d_spec_), spec * sizeof(float), "cudaMalloc(spectra)") ||
        !alloc(reinterpret_cast<void **>(&d_power_), plane_ / 2 * sizeof(float), "cudaMalloc(power)") ||
        !alloc(reinterpret_cast<void **>(&d_inter_), plane_ * sizeof(float), "cudaMalloc(interbin)") ||
        (ct && !alloc(reinterpret_cast<void **>(&d_power_ct_), plane_ / 2 * sizeof(float), "cudaMalloc(power CT)")) ||
        (ct && !alloc(reinterpret_cast<void **>(&d_inter_ct_), plane_ * sizeof(float), "cudaMalloc(interbin CT)")) ||
        !alloc(reinterpret_cast<void **>(&d_snr_p_), plane_ / 2 * sizeof(float), "cudaMalloc(S/N)") ||
        !alloc(reinterpret_cast<void **>(&d_snr_i_), plane_ * sizeof(float), "cudaMalloc(S/N)") ||
        !alloc(reinterpret_cast<void **>(&d_harm_p_), plane_ / 2 * sizeof(uint16_t), "cudaMalloc(harmonics)") ||
        !alloc(reinterpret_cast<void **>(&d_harm_i_), plane_ * sizeof(uint16_t), "cudaMalloc(harmonics)") ||
        !alloc(reinterpret_cast<void **>(&d_list_p_), static_cast<size_t>(max_list_) * 4 * sizeof(float),
               "cudaMalloc(list)") ||
        !alloc(reinterpret_cast<void **>(&d_list_i_), static_cast<size_t>(max_list_) * 4 * sizeof(float),
               "cudaMalloc(list)") ||
        !alloc(reinterpret_cast<void **>(&d_msd_), 2 * 32 * sizeof(float), "cudaMalloc(MSD)") ||
        !alloc(reinterpret_cast<void **>(&d_count_), 2 * sizeof(int), "cudaMalloc(count)"))
        return false;
    cufft_work_bytes_ = 0;
    for (const PsrRange &R : s.ranges)
        for (const PsrBatch &b : R.batches) {
            size_t ws = 0;
            if (!cufft_ok(cufftEstimate1d(static_cast<int>(b.nTimesamples), CUFFT_R2C,
                                          static_cast<int>(b.nDMs_per_batch), &ws),
                          "cufftEstimate1d", err))
                return false;
            cufft_work_bytes_ = std::max(cufft_work_bytes_, ws);
        }
    cufft_work_bytes_ = std::max(cufft_work_bytes_, s.cufft_workarea_size);
    if (!alloc(&d_cufft_work_, cufft_work_bytes_, "cudaMalloc(cuFFT work area)"))
        return false;
    SpdPlane *m = new SpdPlane();
    msd_ = m;
    if (!m->setup(static_cast<long long>(max_dms * (max_nt >> 1)), 0, err))
        return false;
    if (!cuda_ok(cudaEventCreate(&ev0_), "cudaEventCreate", err) || !cuda_ok(cudaEventCreate(&ev1_), "cudaEventCreate", err))
        return false;
    return true;
}

// One batch of Periodicity_search (src/aa_device_periods.cu:368-541) and
// the candidate hand-over of GPU_periodicity (:618-660).
bool PsrSearch::batch(const PsrStrategy &s, const PsrRange &R, const PsrBatch &b, const PsrRows &rows,
                      void *power_list, void *interbin_list, cudaStream_t st, std::string &err)
{
    const int nT = static_cast<int>(b.nTimesamples);
    const int nD = static_cast<int>(b.nDMs_per_batch);
    const int alg = s.plan.harmonic_sum_algorithm;
    const bool transposed = alg == 0;
    const bool greedy = alg == 1;
    const int nH = s.plan.nHarmonics;

    // Copy_data_for_periodicity_search (:263-306): the first
    // nTimesamples_to_copy samples of each row into a row of nTimesamples,
    // zeros after them (and after the row's end, where the reference reads
    // past the row)
    const long long ncopy =
        std::min<long long>(static_cast<long long>(b.nTimesamples_to_copy), std::max<long long>(0, rows.row_len));
    if (ncopy < nT && !cuda_ok(cudaMemsetAsync(d_in_, 0, static_cast<size_t>(nD) * nT * sizeof(float), st), "memset",
                               err))
        return false;
    if (ncopy > 0 &&
        !cuda_ok(cudaMemcpy2DAsync(d_in_, static_cast<size_t>(nT) * sizeof(float),
                                   rows.base + static_cast<long long>(b.DM_shift) * rows.pitch,
                                   static_cast<size_t>(rows.pitch) * sizeof(float),
                                   static_cast<size_t>(ncopy) * sizeof(float), static_cast<size_t>(nD),
                                   rows.on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st),
                 "input copy", err))
        return false;
    if (!cuda_ok(cudaMemsetAsync(d_count_, 0, 2 * sizeof(int), st), "memset", err) ||
        !cuda_ok(cudaEventRecord(ev0_, st), "event", err))
        return false;

    // real-to-complex FFT with the plan the reference makes
    cufftHandle plan;
    if (!cufft_ok(cufftCreate(&plan), "cufftCreate", err))
        return false;
    size_t ws = 0;
    bool ok = cufft_ok(cufftSetAutoAllocation(plan, 0), "cufftSetAutoAllocation", err) &&
              cufft_ok(cufftMakePlan1d(plan, nT, CUFFT_R2C, nD, &ws), "cufftMakePlan1d", err);
    if (ok && ws > cufft_work_bytes_) {
        err = "periodicity search: cuFFT work area larger than estimated";
        ok = false;
    }
    ok = ok && cufft_ok(cufftSetWorkArea(plan, d_cufft_work_), "cufftSetWorkArea", err) &&
         cufft_ok(cufftSetStream(plan, st), "cufftSetStream", err) &&
         cufft_ok(cufftExecR2C(plan, reinterpret_cast<cufftReal *>(d_in_), reinterpret_cast<cufftComplex *>(d_spec_)),
                  "cufftExecR2C", err);
    cufftDestroy(plan);
    if (!ok)
        return false;

    float2 *spec = reinterpret_cast<float2 *>(d_spec_);
    if (!cuda_ok(psr_whitening(spec, static_cast<size_t>((nT >> 1) + 1), nD, st), "spectral whitening", err) ||
        !cuda_ok(psr_power_interbin(spec, d_power_, d_inter_, nT, nD, st), "power spectra", err))
        return false;

    // MSD_plane_profile of the power spectra, widths 1..nHarmonics, the
    // high-memory form, not continuous (:454-466)
    std::vector<int> widths(static_cast<size_t>(nH));
    for (int f = 0; f < nH; ++f)
        widths[static_cast<size_t>(f)] = f + 1;
    SpdPlane *m = static_cast<SpdPlane *>(msd_);
    if (!m->profile(d_power_, nD, nT >> 1, widths, true, s.plan.sigma_outlier_rejection_threshold,
                    s.plan.enable_outlier_rejection, st, err))
        return false;
    last_msd = m->last_msd;
    last_msd.resize(static_cast<size_t>(2 * nH), 0.f);
    if (!cuda_ok(cudaMemcpyAsync(d_msd_, last_msd.data(), last_msd.size() * sizeof(float), cudaMemcpyHostToDevice, st),
                 "MSD copy", err))
        return false;

    // harmonic sums (:470-509)
    const float *snr_p = d_snr_p_, *snr_i = d_snr_i_;
    if (transposed) {
        if (!cuda_ok(psr_transpose(d_power_, d_power_ct_, nT >> 1, nD, st), "corner turn", err) ||
            !cuda_ok(psr_transpose(d_inter_, d_inter_ct_, nT, nD, st), "corner turn", err) ||
            !cuda_ok(psr_harmonic_sum_simple(d_power_ct_, d_snr_p_, d_harm_p_, d_msd_, nT >> 1, nD, nH, st),
                     "harmonic sum", err) ||
            !cuda_ok(psr_harmonic_sum_simple(d_inter_ct_, d_snr_i_, d_harm_i_, d_msd_, nT, nD, nH, st),
                     "harmonic sum", err))
            return false;
    } else {
        const bool sc = s.plan.enable_scalloping_loss_mitigation;
        if (!cuda_ok(psr_harmonic_sum(alg, d_power_, d_snr_p_, d_harm_p_, d_msd_, nT >> 1, nD, nH, sc, st),
                     "harmonic sum", err) ||
            !cuda_ok(psr_harmonic_sum(alg, d_inter_, d_snr_i_, d_harm_i_, d_msd_, nT, nD, nH, sc, st),
                     "harmonic sum", err))
            return false;
    }

    // peak finding or thresholding (:513-538), DM trials numbered from the
    // batch's first trial of the range
    const int cap = static_cast<int>(max_list_);
    const int shift = static_cast<int>(b.DM_shift);
    auto select = [&](const float *snr, const uint16_t *harm, float *list, int n, int *count) {
        if (s.plan.candidate_selection_algorithm == 1)
            return psr_threshold(snr, harm, list, n, nD, s.plan.sigma_cutoff, cap, count, d_msd_, shift, 1, transposed,
                                 greedy, st);
        return psr_peak_find(snr, harm, list, n, nD, s.plan.sigma_cutoff, cap, count, d_msd_, shift, 1, transposed,
                             greedy, st);
    };
    if (!cuda_ok(select(snr_p, d_harm_p_, d_list_p_, nT >> 1, d_count_), "candidate selection", err) ||
        !cuda_ok(select(snr_i, d_harm_i_, d_list_i_, nT, d_count_ + 1), "candidate selection", err) ||
        !cuda_ok(cudaEventRecord(ev1_, st), "event", err))
        return false;

    int counts[2] = {0, 0};
    if (!cuda_ok(cudaMemcpyAsync(counts, d_count_, sizeof(counts), cudaMemcpyDeviceToHost, st), "count copy", err) ||
        !cuda_ok(cudaStreamSynchronize(st), "sync", err))
        return false;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ev0_, ev1_) == cudaSuccess)
        last_compute_ms += ms;
    ++last_batches;
    // the candidates of the reference's lists (records beyond the list's
    // capacity are not written; the count goes on)
    const size_t np = static_cast<size_t>(std::min(counts[0], cap)), ni = static_cast<size_t>(std::min(counts[1], cap));
    // aa_periodicity_candidates::Add_Candidates with the range's float DM
    // values and its FFT length (:626-655)
    const double dm_low = static_cast<double>(static_cast<float>(R.range.dm_low));
    const double dm_step = static_cast<double>(static_cast<float>(R.range.dm_step));
    const double tsamp = R.range.sampling_time;
    const size_t nts = R.range.nTimesamples;
    if (aa_b200_psr_candidates_add(power_list, d_list_p_, np, 1, R.rangeid, last_msd.data(), dm_low, dm_step, tsamp,
                                   nts, 1.0f, greedy ? 1 : 0) != 0 ||
        aa_b200_psr_candidates_add(interbin_list, d_list_i_, ni, 1, R.rangeid, last_msd.data(), dm_low, dm_step,
                                   tsamp, nts, 2.0f, greedy ? 1 : 0) != 0) {
        err = std::string("periodicity search: ") + aa_b200_psr_candidates_last_error();
        return false;
    }
    return true;
}

bool PsrSearch::run(const PsrStrategy &s, const std::vector<PsrRows> &rows, void *power_list, void *interbin_list,
                    cudaStream_t st, std::string &err)
{
    if (!d_in_) {
        err = "periodicity search: not set up";
        return false;
    }
    if (rows.size() < s.ranges.size()) {
        err = "periodicity search: rows of every range needed";
        return false;
    }
    last_compute_ms = 0;
    last_batches = 0;
    for (const PsrRange &R : s.ranges) {
        const PsrRows &src = rows[static_cast<size_t>(R.rangeid)];
        for (const PsrBatch &b : R.batches) {
            if (static_cast<size_t>(b.nDMs_per_batch) * b.nTimesamples > plane_) {
                err = "periodicity search: batch larger than the buffers";
                return false;
            }
            if (!batch(s, R, b, src, power_list, interbin_list, st, err))
                return false;
        }
    }
    return true;
}

} // namespace aab200
