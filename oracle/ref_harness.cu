/*
 * ref_harness.cu -- drives the reference's own DDTR code (AstroAccelerate
 * v1.3.1, compiled from its sources by oracle/Makefile.ref into oracle/_ref/)
 * so that its results can be captured as golden vectors.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links this file.
 *
 *   aaref_strategy()  runs aa_ddtr_strategy (src/aa_ddtr_strategy.cpp:27-428)
 *                     on the host; it needs no GPU.
 *   aaref_run_ddtr()  runs the reference's generic pipeline runner
 *                     (include/aa_permitted_pipelines_generic.hpp:606-914) with
 *                     only the dedispersion component and copy-to-host, exactly
 *                     as tests/test_ddtr_fakesignal_single.cpp:82-103 does, and
 *                     copies output_buffer() into a flat array.  Needs a GPU.
 *                     The reference's aa_device_info destructor resets the
 *                     device, so call this from a process of its own.
 *   aaref_export_dd_data() writes DM-time files with the reference's
 *                     Export_DD_data (include/aa_pipeline_runner.hpp:165-216)
 *                     through a runner that only exposes it.  No GPU.
 *   aaref_spd()       the reference's single-pulse detection on one DM-time
 *                     plane: the stages of analysis_GPU
 *                     (src/aa_device_analysis.cu:130-245) one by one -- the
 *                     interpolated MSD profile, the boxcar S/N and width planes
 *                     -- and then analysis_GPU itself for the candidates.
 *                     Needs a GPU.
 *   aaref_sigproc_read() reads a SIGPROC file with the reference's
 *                     aa_sigproc_input (src/aa_sigproc_input.cpp:85-543):
 *                     metadata and the unsigned-short input buffer.  No GPU.
 */
#include <chrono>
#include <stdio.h>
#include <string.h>
#include <vector>

/* aa_device_info keeps the memory budget private and only fills it in when a
 * GPU answers; the host-only strategy run sets it directly. */
#define private public
#include "aa_device_info.hpp"
#undef private

#include "aa_ddtr_plan.hpp"
#include "aa_ddtr_strategy.hpp"
#include "aa_filterbank_metadata.hpp"
#include "aa_permitted_pipelines_generic.hpp"
#include "aa_pipeline.hpp"
#include "aa_sigproc_input.hpp"
#include "aa_analysis_plan.hpp"
#include "aa_analysis_strategy.hpp"
#include "aa_device_analysis.hpp"
#include "aa_device_BC_plan.hpp"
#include "aa_device_MSD_plane_profile.hpp"
#include "aa_device_SPS_long.hpp"
#include "aa_device_power.hpp"
#include "aa_device_harmonic_summing.hpp"
#include "aa_device_peak_find.hpp"
#include "aa_device_threshold.hpp"
#include "aa_device_spectrum_whitening.hpp"
#include "aa_device_spectrum_whitening_kernel.hpp"

namespace astroaccelerate {
/* defined in src/aa_device_analysis.cu without a header declaration */
void Create_list_of_boxcar_widths(std::vector<int> *boxcar_widths, std::vector<int> *BC_widths, int max_boxcar_width);
void Create_PD_plan(std::vector<PulseDetection_plan> *PD_plan, std::vector<int> *BC_widths, int nDMs, int nTimesamples);
int Get_max_iteration(int max_boxcar_width, std::vector<int> *BC_widths, int *max_width_performed);
/* defined in src/aa_device_spectral_whitening.cu:40-45 without a header declaration */
void calculate_median_for_segments(float *d_MSD_segments, float2 *d_input, size_t nSamples, int nDMs,
                                   int *d_segment_sizes, int nSegments, cudaStream_t &stream);
} // namespace astroaccelerate

using namespace astroaccelerate;

/* Mirrors include/aa_ddtr_plan.hpp:28-34 struct dm for the C ABI below. */
struct harness_dm {
    float low, high, step;
    int inBin, outBin;
};

namespace {

int copy_strategy(const aa_ddtr_strategy &s, int nchans, int max_chunks,
                  float *dmshifts, int *ndms, harness_dm *str_dm,
                  int *maxshift, int *max_ndms, int *num_tchunks,
                  int *t_processed)
{
    const size_t nr = s.get_nRanges();
    std::vector<float> sh = s.dmshifts();
    for (int c = 0; c < nchans; c++)
        dmshifts[c] = sh[c];
    for (size_t i = 0; i < nr; i++) {
        ndms[i] = s.ndms(i);
        aa_ddtr_plan::dm d = s.dm(i);
        str_dm[i].low = d.low;
        str_dm[i].high = d.high;
        str_dm[i].step = d.step;
        str_dm[i].inBin = d.inBin;
        str_dm[i].outBin = d.outBin;
    }
    *maxshift = s.maxshift();
    *max_ndms = s.max_ndms();
    *num_tchunks = s.num_tchunks();
    if (*num_tchunks > max_chunks)
        return -5;
    for (size_t i = 0; i < nr; i++)
        for (int k = 0; k < *num_tchunks; k++)
            t_processed[i * max_chunks + k] = s.t_processed()[i][k];
    return 0;
}

} // namespace

extern "C" {

int aaref_strategy(const harness_dm *plan, int nranges, float power, int nchans,
                   int nsamp, double fch1, double foff, double tsamp, int nbits,
                   size_t free_memory, int enable_analysis, int max_chunks,
                   float *dmshifts, int *ndms, harness_dm *str_dm,
                   int *maxshift, int *max_ndms, int *num_tchunks,
                   int *t_processed)
{
    aa_ddtr_plan p;
    for (int i = 0; i < nranges; i++)
        p.add_dm(plan[i].low, plan[i].high, plan[i].step, plan[i].inBin, plan[i].outBin);
    p.set_power(power);
    aa_filterbank_metadata meta(0.0, tsamp, nbits, nsamp, fch1, foff, nchans);
    aa_device_info dev(0);
    dev.selected_card_info.available_memory = free_memory;
    aa_ddtr_strategy s(p, meta, free_memory, enable_analysis != 0, &dev);
    if (!s.ready())
        return -1;
    return copy_strategy(s, nchans, max_chunks, dmshifts, ndms, str_dm, maxshift,
                         max_ndms, num_tchunks, t_processed);
}

/* free_memory == 0 uses the device's own free memory, like the reference's
 * pipeline API (include/aa_pipeline_api.hpp:149); a smaller value forces
 * time chunking on small inputs.  options: bit 0 zero_dm, 1
 * zero_dm_with_outliers, 2 input_DDTR_normalization, 3
 * output_DDTR_normalization, 4 old_rfi, 5 set_bandpass_average; bandpass
 * (bandpass_size values, may be 0) is bound to the plan. */
int aaref_run_ddtr_opts(const unsigned short *input_tc, int nchans, int nsamp,
                        double tsamp, double fch1, double foff, int nbits,
                        const harness_dm *plan, int nranges, size_t free_memory,
                        int max_chunks, float *dmshifts, int *ndms,
                        harness_dm *str_dm, int *maxshift, int *max_ndms,
                        int *num_tchunks, int *t_processed, float *out,
                        size_t out_len, int options, const float *bandpass, int bandpass_size)
{
    aa_device_info dev(0);
    aa_ddtr_plan p;
    for (int i = 0; i < nranges; i++)
        p.add_dm(plan[i].low, plan[i].high, plan[i].step, plan[i].inBin, plan[i].outBin);
    if (bandpass && bandpass_size > 0)
        p.bind_bandpass_normalization(bandpass, bandpass_size);
    aa_filterbank_metadata meta(0.0, tsamp, nbits, nsamp, fch1, foff, nchans);
    size_t dev_free = dev.free_memory();
    size_t fm = free_memory ? free_memory : dev_free;
    int rc = 0;
    size_t written = 0;
    {
        aa_ddtr_strategy s(p, meta, fm, false, &dev);
        if (!s.ready())
            return -1;
        rc = copy_strategy(s, nchans, max_chunks, dmshifts, ndms, str_dm, maxshift,
                           max_ndms, num_tchunks, t_processed);
        if (rc)
            return rc;
        if ((long long)nchans * (long long)(s.t_processed()[0][0] + s.maxshift()) >= (1LL << 31))
            return -6; /* 32-bit index overflow in the reference kernels */

        aa_pipeline::pipeline comps;
        comps.insert(aa_pipeline::component::dedispersion);
        aa_pipeline::pipeline_option opts;
        opts.insert(aa_pipeline::component_option::copy_ddtr_data_to_host);
        if (options & 1)
            opts.insert(aa_pipeline::component_option::zero_dm);
        if (options & 2)
            opts.insert(aa_pipeline::component_option::zero_dm_with_outliers);
        if (options & 4)
            opts.insert(aa_pipeline::component_option::input_DDTR_normalization);
        if (options & 8)
            opts.insert(aa_pipeline::component_option::output_DDTR_normalization);
        if (options & 16)
            opts.insert(aa_pipeline::component_option::old_rfi);
        if (options & 32)
            opts.insert(aa_pipeline::component_option::set_bandpass_average);
        aa_analysis_strategy an;
        aa_periodicity_strategy per;
        aa_fdas_strategy fd;
        aa_jerk_strategy jk;
        aa_permitted_pipelines_generic runner(comps, opts, s, an, per, fd, jk,
                                              false, false, false, false, false,
                                              input_tc);
        if (!runner.setup())
            return -2;
        aa_pipeline_runner::status st;
        while (runner.next(st)) {
            if (st == aa_pipeline_runner::status::error)
                return -3;
        }
        if (st == aa_pipeline_runner::status::error)
            return -3;
        float ***buf = runner.output_buffer();
        for (int r = 0; r < nranges; r++) {
            size_t tot = 0;
            for (int k = 0; k < *num_tchunks; k++)
                tot += (size_t)t_processed[r * max_chunks + k];
            for (int d = 0; d < ndms[r]; d++) {
                if (written + tot > out_len)
                    return -4;
                memcpy(out + written, buf[r][d], tot * sizeof(float));
                written += tot;
            }
        }
    }
    return 0;
}

int aaref_run_ddtr(const unsigned short *input_tc, int nchans, int nsamp,
                   double tsamp, double fch1, double foff, int nbits,
                   const harness_dm *plan, int nranges, size_t free_memory,
                   int max_chunks, float *dmshifts, int *ndms,
                   harness_dm *str_dm, int *maxshift, int *max_ndms,
                   int *num_tchunks, int *t_processed, float *out,
                   size_t out_len)
{
    return aaref_run_ddtr_opts(input_tc, nchans, nsamp, tsamp, fch1, foff, nbits, plan, nranges, free_memory,
                               max_chunks, dmshifts, ndms, str_dm, maxshift, max_ndms, num_tchunks, t_processed,
                               out, out_len, 0, nullptr, 0);
}

/* Times the reference's pipeline runner over the whole input: setup outside
 * the timed region, then the run(status) loop (load, corner turn, binning,
 * dedispersion and, with copy_to_host, the D2H into float***), wall clock. */
int aaref_time_ddtr(const unsigned short *input_tc, int nchans, int nsamp, double tsamp, double fch1,
                    double foff, int nbits, const harness_dm *plan, int nranges, int copy_to_host,
                    double *seconds, int *num_tchunks)
{
    aa_device_info dev(0);
    aa_ddtr_plan p;
    for (int i = 0; i < nranges; i++)
        p.add_dm(plan[i].low, plan[i].high, plan[i].step, plan[i].inBin, plan[i].outBin);
    aa_filterbank_metadata meta(0.0, tsamp, nbits, nsamp, fch1, foff, nchans);
    size_t fm = dev.free_memory();
    {
        aa_ddtr_strategy s(p, meta, fm, false, &dev);
        if (!s.ready())
            return -1;
        *num_tchunks = s.num_tchunks();
        /* the reference's shared kernels index the flat chunk with a 32-bit
         * int (src/aa_device_dedispersion_kernel.cu:194,214); a chunk of more
         * than 2^31 elements makes them read out of bounds, so it is refused */
        if ((long long)nchans * (long long)(s.t_processed()[0][0] + s.maxshift()) >= (1LL << 31))
            return -4;
        aa_pipeline::pipeline comps;
        comps.insert(aa_pipeline::component::dedispersion);
        aa_pipeline::pipeline_option opts;
        if (copy_to_host)
            opts.insert(aa_pipeline::component_option::copy_ddtr_data_to_host);
        aa_analysis_strategy an;
        aa_periodicity_strategy per;
        aa_fdas_strategy fd;
        aa_jerk_strategy jk;
        aa_permitted_pipelines_generic runner(comps, opts, s, an, per, fd, jk, false, false, false, false, false,
                                              input_tc);
        if (!runner.setup())
            return -2;
        cudaDeviceSynchronize();
        auto t0 = std::chrono::steady_clock::now();
        aa_pipeline_runner::status st;
        while (runner.next(st)) {
            if (st == aa_pipeline_runner::status::error)
                return -3;
        }
        if (st == aa_pipeline_runner::status::error || cudaDeviceSynchronize() != cudaSuccess)
            return -3;
        auto t1 = std::chrono::steady_clock::now();
        *seconds = std::chrono::duration<double>(t1 - t0).count();
    }
    return 0;
}

/* The reference runner with dedispersion and analysis (single-pulse
 * detection) components, as aa_pipeline_api sets them up
 * (include/aa_pipeline_api.hpp:130-219): the DDTR strategy computed for
 * analysis, then per (time chunk, range) step the candidates of analysis_GPU
 * (include/aa_permitted_pipelines_generic.hpp:848-889), read after each step
 * from the runner's host lists.  The peak_analysed/analysed files go to the
 * working directory.  Per step k: step_chunk[k], step_range[k],
 * step_ncands[k]; the candidates of all steps follow one another in
 * c_dm/c_ts/c_snr/c_bw (max_cands).  *msd_max_ts receives the analysis
 * strategy's maxtimesamples.  Returns the number of steps, or < 0. */
int aaref_run_pipeline_spd(const unsigned short *input_tc, int nchans, int nsamp, double tsamp, double fch1,
                           double foff, int nbits, const harness_dm *plan, int nranges, size_t free_memory,
                           float sigma_cutoff, float sigma_constant, float max_boxcar_width_in_sec,
                           int candidate_algorithm, int enable_msd_baseline_noise, int max_steps, int *step_chunk,
                           int *step_range, long long *step_ncands, unsigned *c_dm, unsigned *c_ts, float *c_snr,
                           unsigned *c_bw, long long max_cands, long long *msd_max_ts, int *num_tchunks,
                           int *t_processed, int max_chunks)
{
    aa_device_info dev(0);
    aa_ddtr_plan p;
    for (int i = 0; i < nranges; i++)
        p.add_dm(plan[i].low, plan[i].high, plan[i].step, plan[i].inBin, plan[i].outBin);
    aa_filterbank_metadata meta(0.0, tsamp, nbits, nsamp, fch1, foff, nchans);
    size_t fm = free_memory ? free_memory : dev.free_memory();
    int nsteps = 0;
    long long written = 0;
    {
        aa_ddtr_strategy s(p, meta, fm, true, &dev);
        if (!s.ready())
            return -1;
        *num_tchunks = s.num_tchunks();
        if (*num_tchunks > max_chunks)
            return -5;
        for (int r = 0; r < nranges; r++)
            for (int k = 0; k < *num_tchunks; k++)
                t_processed[r * max_chunks + k] = s.t_processed()[r][k];
        if ((long long)nchans * (long long)(s.t_processed()[0][0] + s.maxshift()) >= (1LL << 31))
            return -6;
        aa_analysis_plan::selectable_candidate_algorithm alg =
            candidate_algorithm == 1   ? aa_analysis_plan::selectable_candidate_algorithm::threshold
            : candidate_algorithm == 2 ? aa_analysis_plan::selectable_candidate_algorithm::peak_filtering
                                       : aa_analysis_plan::selectable_candidate_algorithm::peak_find;
        aa_analysis_plan ap(s, sigma_cutoff, sigma_constant, max_boxcar_width_in_sec, alg,
                            enable_msd_baseline_noise != 0);
        aa_analysis_strategy an(ap, &dev);
        if (!an.ready())
            return -7;
        *msd_max_ts = (long long)an.MSD_data_info();
        aa_pipeline::pipeline comps;
        comps.insert(aa_pipeline::component::dedispersion);
        comps.insert(aa_pipeline::component::analysis);
        aa_pipeline::pipeline_option opts;
        opts.insert(aa_pipeline::component_option::copy_ddtr_data_to_host);
        aa_periodicity_strategy per;
        aa_fdas_strategy fd;
        aa_jerk_strategy jk;
        aa_permitted_pipelines_generic runner(comps, opts, s, an, per, fd, jk, false, false, false, false, false,
                                              input_tc);
        if (!runner.setup())
            return -2;
        aa_pipeline_runner::status st;
        bool more = true;
        while (more) {
            more = runner.next(st);
            if (st == aa_pipeline_runner::status::error)
                return -3;
            if (st != aa_pipeline_runner::status::has_more)
                continue;
            if (nsteps >= max_steps)
                return -4;
            /* the accessors give the step just run */
            const int rr = runner.get_current_range(), cc = runner.get_current_tchunk();
            const size_t k = runner.get_SPD_nCandidates();
            step_chunk[nsteps] = cc;
            step_range[nsteps] = rr;
            step_ncands[nsteps] = (long long)k;
            if (written + (long long)k > max_cands)
                return -8;
            for (size_t j = 0; j < k; j++) {
                c_dm[written + j] = runner.h_SPD_dm()[j];
                c_ts[written + j] = runner.h_SPD_ts()[j];
                c_snr[written + j] = runner.h_SPD_snr()[j];
                c_bw[written + j] = runner.h_SPD_width()[j];
            }
            written += (long long)k;
            nsteps++;
        }
        if (cudaDeviceSynchronize() != cudaSuccess)
            return -9;
    }
    return nsteps;
}

/* aa_periodicity_strategy (include/aa_periodicity_strategy.hpp:178-355) for
 * the DDTR ranges of a strategy computed as aaref_strategy computes it (no
 * GPU call): the plan's ten-argument constructor with the given settings and
 * memory_available bytes.  Outputs: info[0..6] = corrected FFT length,
 * samples to copy, DM trials per batch in memory, input plane size, cuFFT
 * work area, largest MSD block count, ready flag; per range (up to
 * max_ranges) its FFT length and batch count; per batch (up to max_batches,
 * all ranges in order) range, DM trials, DM shift, samples, samples to copy.
 * Returns the number of batches, or < 0. */
int aaref_psr_strategy(const harness_dm *plan, int nranges, int nchans, int nsamp, double tsamp, double fch1,
                       double foff, int nbits, size_t ddtr_memory, size_t memory_available, float sigma_cutoff,
                       int nHarmonics, int harmonic_sum_algorithm, long long *info, long long *range_info,
                       int max_ranges, long long *batches, int max_batches)
{
    aa_ddtr_plan p;
    for (int i = 0; i < nranges; i++)
        p.add_dm(plan[i].low, plan[i].high, plan[i].step, plan[i].inBin, plan[i].outBin);
    aa_filterbank_metadata meta(0.0, tsamp, nbits, nsamp, fch1, foff, nchans);
    aa_device_info dev(0);
    dev.selected_card_info.available_memory = ddtr_memory;
    aa_ddtr_strategy s(p, meta, ddtr_memory, false, &dev);
    if (!s.ready())
        return -1;
    aa_periodicity_plan pp(s, sigma_cutoff, true, 3.0f, nHarmonics, harmonic_sum_algorithm, 0, true, true, true);
    aa_periodicity_strategy per(pp, memory_available);
    info[6] = per.ready() ? 1 : 0;
    if (!per.ready())
        return 0;
    info[3] = (long long)per.input_plane_size();
    info[4] = (long long)per.cuFFT_workarea_size();
    info[5] = (long long)per.max_total_MSD_blocks();
    int nb = 0;
    for (int r = 0; r < per.nRanges(); r++) {
        aa_periodicity_range R = per.get_periodicity_range(r);
        if (r < max_ranges) {
            range_info[2 * r] = (long long)R.range.nTimesamples();
            range_info[2 * r + 1] = (long long)R.batches.size();
        }
        for (size_t b = 0; b < R.batches.size(); b++) {
            if (nb < max_batches) {
                batches[5 * nb + 0] = r;
                batches[5 * nb + 1] = (long long)R.batches[b].nDMs_per_batch;
                batches[5 * nb + 2] = (long long)R.batches[b].DM_shift;
                batches[5 * nb + 3] = (long long)R.batches[b].nTimesamples;
                batches[5 * nb + 4] = (long long)R.batches[b].nTimesamples_to_copy;
                if (r == 0 && b == 0) {
                    info[0] = (long long)(R.batches[b].nTimesamples * R.range.inBin());
                    info[1] = (long long)(R.batches[b].nTimesamples_to_copy * R.range.inBin());
                }
            }
            nb++;
        }
    }
    info[2] = per.nRanges() > 0 && !per.get_periodicity_range(0).batches.empty()
                  ? (long long)per.get_periodicity_range(0).batches[0].nDMs_per_batch /
                        per.get_periodicity_range(0).range.inBin()
                  : 0;
    return nb;
}

/* The reference runner with dedispersion and periodicity components
 * (include/aa_permitted_pipelines_generic.hpp:570-660, :916-947): the DDTR
 * strategy for free_memory, the periodicity plan's ten-argument constructor
 * (include/aa_periodicity_plan.hpp:62-89) and its strategy for psr_memory
 * bytes, the run loop to the end, then the power and interbin candidate
 * lists (4 floats per record) into power/interbin (cap records each) and
 * their counts into *npower / *ninterbin.  Returns 0, or < 0 (-8: a list
 * longer than cap; the counts are set). */
int aaref_run_pipeline_psr(const unsigned short *input_tc, int nchans, int nsamp, double tsamp, double fch1,
                           double foff, int nbits, const harness_dm *plan, int nranges, size_t free_memory,
                           size_t psr_memory, float sigma_cutoff, int enable_outlier_rejection,
                           float sigma_outlier_rejection_threshold, int nHarmonics, int harmonic_sum_algorithm,
                           int candidate_selection_algorithm, int enable_scalloping_loss_mitigation, float *power,
                           long long *npower, float *interbin, long long *ninterbin, long long cap)
{
    aa_device_info dev(0);
    aa_ddtr_plan p;
    for (int i = 0; i < nranges; i++)
        p.add_dm(plan[i].low, plan[i].high, plan[i].step, plan[i].inBin, plan[i].outBin);
    aa_filterbank_metadata meta(0.0, tsamp, nbits, nsamp, fch1, foff, nchans);
    size_t fm = free_memory ? free_memory : dev.free_memory();
    int rc = 0;
    {
        aa_ddtr_strategy s(p, meta, fm, false, &dev);
        if (!s.ready())
            return -1;
        if ((long long)nchans * (long long)(s.t_processed()[0][0] + s.maxshift()) >= (1LL << 31))
            return -6;
        aa_periodicity_plan pp(s, sigma_cutoff, enable_outlier_rejection != 0, sigma_outlier_rejection_threshold,
                               nHarmonics, harmonic_sum_algorithm, candidate_selection_algorithm,
                               enable_scalloping_loss_mitigation != 0, true, true);
        aa_periodicity_strategy per(pp, psr_memory ? psr_memory : dev.free_memory());
        if (!per.ready())
            return -7;
        aa_pipeline::pipeline comps;
        comps.insert(aa_pipeline::component::dedispersion);
        comps.insert(aa_pipeline::component::periodicity);
        aa_pipeline::pipeline_option opts;
        opts.insert(aa_pipeline::component_option::copy_ddtr_data_to_host);
        aa_analysis_strategy an;
        aa_fdas_strategy fd;
        aa_jerk_strategy jk;
        aa_permitted_pipelines_generic runner(comps, opts, s, an, per, fd, jk, false, false, false, false, false,
                                              input_tc);
        if (!runner.setup())
            return -2;
        aa_pipeline_runner::status st;
        bool more = true;
        while (more) {
            more = runner.next(st);
            if (st == aa_pipeline_runner::status::error)
                return -3;
        }
        if (cudaDeviceSynchronize() != cudaSuccess)
            return -9;
        *npower = (long long)runner.get_PSR_nCandidates();
        *ninterbin = (long long)runner.get_PSR_interbin_nCandidates();
        if (*npower > cap || *ninterbin > cap) {
            rc = -8;
        } else {
            const float *hp = runner.Get_PSR_candidates();
            if (*npower > 0)
                memcpy(power, hp, (size_t)*npower * 4 * sizeof(float));
            const float *hi = runner.Get_PSR_interbin_candidates();
            if (*ninterbin > 0)
                memcpy(interbin, hi, (size_t)*ninterbin * 4 * sizeof(float));
        }
    }
    return rc;
}

/* aaref_time_ddtr with the analysis component: the runner's run(status)
 * loop with dedispersion, D2H (copy_to_host) and analysis_GPU after every
 * step, wall clock after setup.  Candidate files go to the working
 * directory; *ncands receives the candidates of all steps. */
int aaref_time_pipeline_spd(const unsigned short *input_tc, int nchans, int nsamp, double tsamp, double fch1,
                            double foff, int nbits, const harness_dm *plan, int nranges, int copy_to_host,
                            float sigma_cutoff, float sigma_constant, float max_boxcar_width_in_sec,
                            int candidate_algorithm, int enable_msd_baseline_noise, double *seconds,
                            int *num_tchunks, long long *ncands)
{
    aa_device_info dev(0);
    aa_ddtr_plan p;
    for (int i = 0; i < nranges; i++)
        p.add_dm(plan[i].low, plan[i].high, plan[i].step, plan[i].inBin, plan[i].outBin);
    aa_filterbank_metadata meta(0.0, tsamp, nbits, nsamp, fch1, foff, nchans);
    size_t fm = dev.free_memory();
    {
        aa_ddtr_strategy s(p, meta, fm, true, &dev);
        if (!s.ready())
            return -1;
        *num_tchunks = s.num_tchunks();
        if ((long long)nchans * (long long)(s.t_processed()[0][0] + s.maxshift()) >= (1LL << 31))
            return -4;
        aa_analysis_plan::selectable_candidate_algorithm alg =
            candidate_algorithm == 1   ? aa_analysis_plan::selectable_candidate_algorithm::threshold
            : candidate_algorithm == 2 ? aa_analysis_plan::selectable_candidate_algorithm::peak_filtering
                                       : aa_analysis_plan::selectable_candidate_algorithm::peak_find;
        aa_analysis_plan ap(s, sigma_cutoff, sigma_constant, max_boxcar_width_in_sec, alg,
                            enable_msd_baseline_noise != 0);
        aa_analysis_strategy an(ap, &dev);
        if (!an.ready())
            return -7;
        aa_pipeline::pipeline comps;
        comps.insert(aa_pipeline::component::dedispersion);
        comps.insert(aa_pipeline::component::analysis);
        aa_pipeline::pipeline_option opts;
        if (copy_to_host)
            opts.insert(aa_pipeline::component_option::copy_ddtr_data_to_host);
        aa_periodicity_strategy per;
        aa_fdas_strategy fd;
        aa_jerk_strategy jk;
        aa_permitted_pipelines_generic runner(comps, opts, s, an, per, fd, jk, false, false, false, false, false,
                                              input_tc);
        if (!runner.setup())
            return -2;
        cudaDeviceSynchronize();
        long long total = 0;
        auto t0 = std::chrono::steady_clock::now();
        aa_pipeline_runner::status st;
        while (runner.next(st)) {
            if (st == aa_pipeline_runner::status::error)
                return -3;
            if (st == aa_pipeline_runner::status::has_more)
                total += (long long)runner.get_SPD_nCandidates();
        }
        if (st == aa_pipeline_runner::status::error || cudaDeviceSynchronize() != cudaSuccess)
            return -3;
        auto t1 = std::chrono::steady_clock::now();
        *seconds = std::chrono::duration<double>(t1 - t0).count();
        *ncands = total;
    }
    return 0;
}

/* The reference's MSD_plane_profile (src/aa_device_MSD_plane_profile.cu:564-604)
 * alone on a host plane [nDMs][nT] for widths[nw], on a zeroed work area of
 * nT*nDMs floats plus its statistics: msd[2*nw] = (mean, deviation) per
 * width.  high_memory as the periodicity search passes it.  Returns 0 or < 0. */
int aaref_msd_profile(const float *plane, int nT, int nDMs, const int *widths, int nw, int high_memory,
                      float sigma, int outlier_rejection, float *msd)
{
    const size_t n = (size_t)nT * (size_t)nDMs;
    std::vector<int> w(widths, widths + nw);
    size_t msd_bytes = 0, dit_bytes = 0, work_bytes = 0;
    Get_MSD_plane_profile_memory_requirements(&msd_bytes, &dit_bytes, &work_bytes, nT, nDMs, &w);
    float *d_plane = NULL, *d_work = NULL, *d_msd = NULL;
    const size_t work_total = n * sizeof(float) + work_bytes;
    if (cudaMalloc((void **)&d_plane, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&d_work, work_total) != cudaSuccess ||
        cudaMalloc((void **)&d_msd, msd_bytes + 4096) != cudaSuccess)
        return -3;
    cudaMemcpy(d_plane, plane, n * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemset(d_work, 0, work_total);
    double t0, t1, t2;
    MSD_plane_profile(d_msd, d_plane, NULL, d_work, high_memory != 0, nT, nDMs, &w, 0, 0, 0, sigma,
                      outlier_rejection, false, &t0, &t1, &t2);
    int rc = 0;
    if (cudaDeviceSynchronize() != cudaSuccess)
        rc = -5;
    cudaMemcpy(msd, d_msd, 2 * (size_t)nw * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(d_plane);
    cudaFree(d_work);
    cudaFree(d_msd);
    return rc;
}

/* The reference's Peak_find_for_periodicity_search
 * (src/aa_device_peak_find.cu:53-131) on a host S/N plane with its harmonic
 * counts (transposed: [nT][nDMs], else [nDMs][nT]) and msd[2*nH]: records of
 * 4 floats into list (max_peaks), their number in *count.  mode 1 runs the
 * periodicity thresholding (src/aa_device_threshold.cu:56-163) instead.
 * Returns 0 or < 0. */
int aaref_psr_peaks(const float *snr, const unsigned short *harm, int nT, int nDMs, float threshold,
                    const float *msd, int nH, int dm_shift, int in_bin, int transposed, int greedy, float *list,
                    int max_peaks, int *count, int mode)
{
    const size_t n = (size_t)nT * (size_t)nDMs;
    float *d_snr = NULL, *d_list = NULL, *d_msd = NULL;
    unsigned short *d_harm = NULL;
    int *d_pos = NULL;
    if (cudaMalloc((void **)&d_snr, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&d_harm, n * sizeof(unsigned short)) != cudaSuccess ||
        cudaMalloc((void **)&d_list, 4 * (size_t)max_peaks * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&d_msd, 2 * (size_t)nH * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&d_pos, sizeof(int)) != cudaSuccess)
        return -3;
    cudaMemcpy(d_snr, snr, n * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(d_harm, harm, n * sizeof(unsigned short), cudaMemcpyHostToDevice);
    cudaMemcpy(d_msd, msd, 2 * (size_t)nH * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemset(d_pos, 0, sizeof(int));
    int rc;
    if (mode == 1) {
        if (transposed)
            rc = Threshold_for_periodicity_transposed(d_snr, d_harm, d_list, d_pos, d_msd, threshold, nDMs, nT,
                                                      dm_shift, in_bin, max_peaks);
        else
            rc = Threshold_for_periodicity_normal(d_snr, d_harm, d_list, d_pos, d_msd, threshold, nT, nDMs, dm_shift,
                                                  in_bin, max_peaks, greedy);
    } else {
        rc = Peak_find_for_periodicity_search(d_snr, d_harm, d_list, nT, nDMs, threshold, max_peaks, d_pos, d_msd,
                                              dm_shift, in_bin, transposed != 0, greedy);
    }
    if (cudaDeviceSynchronize() != cudaSuccess)
        rc = -5;
    cudaMemcpy(count, d_pos, sizeof(int), cudaMemcpyDeviceToHost);
    const int k = *count < max_peaks ? *count : max_peaks;
    cudaMemcpy(list, d_list, 4 * (size_t)k * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(d_snr);
    cudaFree(d_harm);
    cudaFree(d_list);
    cudaFree(d_msd);
    cudaFree(d_pos);
    return rc;
}

/* The reference's greedy (algorithm 1), PRESTO plus (2) or PRESTO (3)
 * harmonic sum (src/aa_device_harmonic_summing.cu:38-169) on a host plane
 * [nDMs][nT] with msd[2*n_msd]: snr and harmonic counts [nDMs][nT].
 * nH is passed as the reference's nHarmonics argument.  Returns 0 or < 0. */
int aaref_psr_harmonics(int algorithm, const float *in, int nT, int nDMs, const float *msd, int n_msd, int nH,
                        int scalloping, float *snr, unsigned short *harm)
{
    const size_t n = (size_t)nT * (size_t)nDMs;
    float *d_in = NULL, *d_snr = NULL, *d_msd = NULL;
    unsigned short *d_harm = NULL;
    if (cudaMalloc((void **)&d_in, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&d_snr, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&d_harm, n * sizeof(unsigned short)) != cudaSuccess ||
        cudaMalloc((void **)&d_msd, 2 * (size_t)n_msd * sizeof(float)) != cudaSuccess)
        return -3;
    cudaMemcpy(d_in, in, n * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(d_msd, msd, 2 * (size_t)n_msd * sizeof(float), cudaMemcpyHostToDevice);
    int rc = 0;
    if (algorithm == 1)
        rc = periodicity_greedy_harmonic_summing(d_in, d_snr, d_harm, d_msd, nT, nDMs, nH, scalloping);
    else if (algorithm == 2)
        rc = periodicity_presto_plus_harmonic_summing(d_in, d_snr, d_harm, d_msd, nT, nDMs, nH, scalloping);
    else
        rc = periodicity_presto_harmonic_summing(d_in, d_snr, d_harm, d_msd, nT, nDMs, nH, scalloping);
    if (cudaDeviceSynchronize() != cudaSuccess)
        rc = -5;
    cudaMemcpy(snr, d_snr, n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaMemcpy(harm, d_harm, n * sizeof(unsigned short), cudaMemcpyDeviceToHost);
    cudaFree(d_in);
    cudaFree(d_snr);
    cudaFree(d_harm);
    cudaFree(d_msd);
    return rc;
}

/* spectrum_whitening_SGP2 with medians (src/aa_device_spectral_whitening.cu:60-118)
 * in place on a device copy of nDMs spectra of nSamples complex bins
 * (spectra: 2 * nDMs * nSamples floats), the result into out; segments: the
 * boundary table of create_dered_segment_sizes_prefix_sum (min 6, max 250),
 * up to seg_cap of them, their count in *nseg.  Returns 0 or < 0. */
int aaref_psr_whitening(const float *spectra, long long nSamples, int nDMs, float *out, int *segments, int seg_cap,
                        int *nseg)
{
    const size_t n = 2 * (size_t)nDMs * (size_t)nSamples;
    std::vector<int> seg;
    create_dered_segment_sizes_prefix_sum(&seg, 6, 250, (size_t)nSamples);
    *nseg = (int)seg.size();
    for (int i = 0; i < seg_cap && i < (int)seg.size(); ++i)
        segments[i] = seg[i];
    float *d = NULL;
    if (cudaMalloc((void **)&d, n * sizeof(float)) != cudaSuccess)
        return -3;
    cudaMemcpy(d, spectra, n * sizeof(float), cudaMemcpyHostToDevice);
    cudaStream_t stream = NULL;
    spectrum_whitening_SGP2((float2 *)d, (size_t)nSamples, nDMs, true, stream);
    int rc = 0;
    if (cudaDeviceSynchronize() != cudaSuccess)
        rc = -5;
    cudaMemcpy(out, d, n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return rc;
}

/* The reference's whitening kernels as spectrum_whitening_SGP2 launches them
 * (calculate_median_for_segments, then call_kernel_spectrum_whitening_SGP2 on
 * nSegments x nDMs blocks of 256 threads, src/aa_device_spectral_whitening.cu:60-118),
 * timed with CUDA events on a device copy of d_src (a device pointer: nDMs
 * spectra of nSamples complex bins), reps times; ms[reps] receives the
 * times.  The boundary table and the median buffer are allocated once,
 * outside the timed region (the reference allocates, copies and frees them
 * on every call), each one element longer than the reference's: the last
 * block of its normalisation kernel reads one boundary and one median past
 * its tables, and with a zero boundary there that block writes nothing.
 * Returns 0 or < 0. */
int aaref_time_psr_whitening(const float *d_src, long long nSamples, int nDMs, int reps, float *ms)
{
    const size_t n = 2 * (size_t)nDMs * (size_t)nSamples;
    std::vector<int> seg;
    create_dered_segment_sizes_prefix_sum(&seg, 6, 250, (size_t)nSamples);
    const int nSegments = (int)seg.size();
    seg.push_back(0);
    float *d = NULL, *d_med = NULL;
    int *d_seg = NULL;
    if (cudaMalloc((void **)&d, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&d_seg, seg.size() * sizeof(int)) != cudaSuccess ||
        cudaMalloc((void **)&d_med, ((size_t)nSegments * nDMs + 1) * sizeof(float)) != cudaSuccess)
        return -3;
    cudaMemcpy(d_seg, seg.data(), seg.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemset(d_med, 0, ((size_t)nSegments * nDMs + 1) * sizeof(float));
    cudaStream_t stream = NULL;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int rc = 0;
    for (int r = 0; r < reps; r++) {
        cudaMemcpy(d, d_src, n * sizeof(float), cudaMemcpyDeviceToDevice);
        cudaDeviceSynchronize();
        cudaEventRecord(e0, stream);
        calculate_median_for_segments(d_med, (float2 *)d, (size_t)nSamples, nDMs, d_seg, nSegments, stream);
        call_kernel_spectrum_whitening_SGP2(dim3(256, 1, 1), dim3(nSegments, nDMs, 1), 0, stream, d_med, (float2 *)d,
                                            d_seg, (size_t)nSamples, nSegments);
        cudaEventRecord(e1, stream);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms[r], e0, e1);
    }
    if (cudaDeviceSynchronize() != cudaSuccess)
        rc = -5;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    cudaFree(d_seg);
    cudaFree(d_med);
    return rc;
}

/* Two stages of the reference's periodicity search on given host data:
 * simple_power_and_interbin (src/aa_device_power.cu:34-52) on nDMs spectra
 * of nT/2+1 complex bins (spectra: 2*nDMs*(nT/2+1) floats) into power
 * [nDMs][nT/2] and interbin [nDMs][nT]; periodicity_simple_harmonic_summing
 * (src/aa_device_harmonic_summing.cu:11-37) on hs_in [nBins][nSpectra] with
 * msd [2*nH] into snr and harmonics [nBins][nSpectra].  Returns 0 or < 0. */
int aaref_psr_blocks(const float *spectra, int nT, int nDMs, float *power, float *interbin, const float *hs_in,
                     int nBins, int nSpectra, const float *msd, int nH, float *snr, unsigned short *harm)
{
    const size_t ns = 2 * (size_t)nDMs * (size_t)((nT >> 1) + 1);
    const size_t np = (size_t)nDMs * (size_t)(nT >> 1), ni = (size_t)nDMs * (size_t)nT;
    const size_t nh = (size_t)nBins * (size_t)nSpectra;
    float *d_spec = NULL, *d_pow = NULL, *d_ib = NULL, *d_hs = NULL, *d_snr = NULL, *d_msd = NULL;
    unsigned short *d_harm = NULL;
    if (cudaMalloc((void **)&d_spec, ns * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&d_pow, np * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&d_ib, ni * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&d_hs, nh * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&d_snr, nh * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&d_harm, nh * sizeof(unsigned short)) != cudaSuccess ||
        cudaMalloc((void **)&d_msd, 2 * (size_t)nH * sizeof(float)) != cudaSuccess)
        return -3;
    cudaMemcpy(d_spec, spectra, ns * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(d_hs, hs_in, nh * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(d_msd, msd, 2 * (size_t)nH * sizeof(float), cudaMemcpyHostToDevice);
    simple_power_and_interbin((float2 *)d_spec, d_pow, d_ib, nT, nDMs);
    periodicity_simple_harmonic_summing(d_hs, d_snr, d_harm, d_msd, nBins, nSpectra, nH);
    int rc = 0;
    if (cudaDeviceSynchronize() != cudaSuccess)
        rc = -5;
    cudaMemcpy(power, d_pow, np * sizeof(float), cudaMemcpyDeviceToHost);
    cudaMemcpy(interbin, d_ib, ni * sizeof(float), cudaMemcpyDeviceToHost);
    cudaMemcpy(snr, d_snr, nh * sizeof(float), cudaMemcpyDeviceToHost);
    cudaMemcpy(harm, d_harm, nh * sizeof(unsigned short), cudaMemcpyDeviceToHost);
    cudaFree(d_spec);
    cudaFree(d_pow);
    cudaFree(d_ib);
    cudaFree(d_hs);
    cudaFree(d_snr);
    cudaFree(d_harm);
    cudaFree(d_msd);
    return rc;
}

/* plane: host [nDMs][nT] float.  Outputs (caller-sized): msd [2 * nwidths]
 * (nwidths <= 256) and widths [nwidths]; snr/taps: the whole S/N and width
 * planes SPDT writes (plane_cap elements, at least 2 * nDMs * nT); the
 * candidates of analysis_GPU (max_cands).  Returns 0, or < 0 on a failure. */
int aaref_spd(const float *plane, int nDMs, int nT, float tsamp, int inBin, float max_boxcar_width_in_sec,
              float sigma_constant, int enable_msd_baseline_noise, float cutoff, int candidate_algorithm, float tstart,
              float dm_low, float dm_high, float dm_step, float *msd, int *widths, int *nwidths, int *max_width_performed,
              int *max_iteration, float *snr, unsigned short *taps, long long plane_cap, unsigned *c_dm, unsigned *c_ts,
              float *c_snr, unsigned *c_bw, int max_cands, int *ncands, long long max_ts)
{
    const size_t n = (size_t)nDMs * (size_t)nT;
    if ((long long)(2 * n) > plane_cap)
        return -1;
    /* the S/N planes of all iterations hold up to 2 * nDMs * nT values, which
     * the reference addresses with int offsets (nDMs * output_shift,
     * src/aa_device_SPS_long.cu:69,73): refuse planes where they could pass
     * 2^31, where its search faulted */
    if ((long long)(2 * n) >= (1LL << 31))
        return -6;
    /* max_ts: analysis_GPU's maxTimeSamples (0 = the plane).  Below the plane
     * the search runs in batches and the whole-plane S/N stage is skipped. */
    const bool whole = (max_ts <= 0 || (size_t)max_ts >= n);
    /* the plan analysis_GPU builds (:138-179) */
    int max_boxcar_width = (int)(max_boxcar_width_in_sec / tsamp);
    int mwp = 0;
    int t_BC_widths[10] = {PD_MAXTAPS, 16, 16, 16, 8, 8, 8, 8, 8, 8};
    std::vector<int> BC_widths(t_BC_widths, t_BC_widths + 10);
    std::vector<PulseDetection_plan> PD_plan;
    int max_it = Get_max_iteration(max_boxcar_width / inBin, &BC_widths, &mwp);
    Create_PD_plan(&PD_plan, &BC_widths, 1, nT);
    std::vector<int> h_boxcar_widths;
    Create_list_of_boxcar_widths(&h_boxcar_widths, &BC_widths, mwp);
    *max_width_performed = mwp;
    *max_iteration = max_it;
    *nwidths = (int)h_boxcar_widths.size();
    if (*nwidths > 256)
        return -2;
    for (int i = 0; i < *nwidths; i++)
        widths[i] = h_boxcar_widths[i];

    /* buffers as the runner sizes them for maxTimeSamples = nDMs * nT
     * (include/aa_permitted_pipelines_generic.hpp:391-412) */
    unsigned long int maxTS = whole ? (unsigned long int)n : (unsigned long int)max_ts;
    float *d_plane = NULL, *d_work = NULL, *d_msd = NULL;
    unsigned short *d_taps = NULL;
    size_t msd_bytes = 0, dit_bytes = 0, work_bytes = 0;
    Get_MSD_plane_profile_memory_requirements(&msd_bytes, &dit_bytes, &work_bytes, nT, nDMs, &h_boxcar_widths);
    if (cudaMalloc((void **)&d_plane, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&d_work, maxTS * 5.5 * sizeof(float) + work_bytes) != cudaSuccess ||
        cudaMalloc((void **)&d_taps, 2 * maxTS * sizeof(unsigned short)) != cudaSuccess ||
        cudaMalloc((void **)&d_msd, msd_bytes + 4096) != cudaSuccess)
        return -3;
    int rc = 0;
    /* stage 1: MSD plane profile (:199) */
    cudaMemcpy(d_plane, plane, n * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemset(d_work, 0, maxTS * 5.5 * sizeof(float));
    double t0, t1, t2;
    MSD_plane_profile(d_msd, d_plane, NULL, d_work, false, nT, nDMs, &h_boxcar_widths, tstart, dm_low, dm_high,
                      sigma_constant, enable_msd_baseline_noise, false, &t0, &t1, &t2);
    cudaMemcpy(msd, d_msd, 2 * (*nwidths) * sizeof(float), cudaMemcpyDeviceToHost);
    /* stage 2: the boxcar planes of one DM batch (:206-253) */
    if (whole) {
        size_t mem_idx = 0;
        int DMs_per_cycle = nDMs;
        mem_idx += 4 * ((size_t)nT * DMs_per_cycle) / 4;
        float *d_decimated = &d_work[mem_idx];
        mem_idx += ((size_t)DMs_per_cycle * nT) / 2 + PD_MAXTAPS;
        float *d_boxcar_values = &d_work[mem_idx];
        mem_idx += (size_t)DMs_per_cycle * nT;
        float *d_output_SNR = &d_work[mem_idx];
        cudaMemset(d_output_SNR, 0, 2 * n * sizeof(float));
        cudaMemset(d_taps, 0, 2 * n * sizeof(unsigned short));
        SPDT_search_long_MSD_plane(d_plane, d_boxcar_values, d_decimated, d_output_SNR, d_taps, d_msd, &PD_plan, max_it,
                                   nT, nDMs);
        cudaMemcpy(snr, d_output_SNR, 2 * n * sizeof(float), cudaMemcpyDeviceToHost);
        cudaMemcpy(taps, d_taps, 2 * n * sizeof(unsigned short), cudaMemcpyDeviceToHost);
    }
    /* stage 3: analysis_GPU on a fresh copy of the plane */
    {
        cudaMemcpy(d_plane, plane, n * sizeof(float), cudaMemcpyHostToDevice);
        size_t peak_pos = 0;
        int ndms_arr[1] = {nDMs};
        int maxshift = 0;
        float lo[1] = {dm_low}, hi[1] = {dm_high}, st[1] = {dm_step};
        analysis_output out;
        std::vector<unsigned> a(max_cands), b(max_cands), d(max_cands);
        std::vector<float> c(max_cands);
        bool ok = analysis_GPU(a.data(), b.data(), c.data(), d.data(), &peak_pos, (size_t)max_cands, 0, tstart, nT,
                               inBin, &maxshift, nDMs, ndms_arr, cutoff, sigma_constant, max_boxcar_width_in_sec,
                               d_plane, lo, hi, st, tsamp, candidate_algorithm, d_work, d_taps, d_msd, maxTS,
                               enable_msd_baseline_noise, false, false, out);
        if (!ok)
            rc = -4;
        *ncands = (int)peak_pos;
        for (size_t k = 0; k < peak_pos && (int)k < max_cands; k++) {
            c_dm[k] = a[k];
            c_ts[k] = b[k];
            c_snr[k] = c[k];
            c_bw[k] = d[k];
        }
    }
    if (cudaDeviceSynchronize() != cudaSuccess)
        rc = -5;
    cudaFree(d_plane);
    cudaFree(d_work);
    cudaFree(d_taps);
    cudaFree(d_msd);
    return rc;
}

/* Times the reference's analysis_GPU (src/aa_device_analysis.cu:130-345) on
 * a device plane [nDMs][nT] (d_src, kept intact): buffers as the runner
 * allocates them (include/aa_permitted_pipelines_generic.hpp:391-412) for
 * maxTimeSamples = max_ts (0 = the plane), then per repetition a device copy
 * of d_src into the plane the search overwrites and CUDA events around
 * analysis_GPU.  ms[reps] receives the times; *ncands the last run's
 * candidate count.  Returns 0, or < 0. */
int aaref_time_spd(const float *d_src, int nDMs, int nT, float tsamp, int inBin, float max_boxcar_width_in_sec,
                   float sigma_constant, int enable_msd_baseline_noise, float cutoff, int candidate_algorithm,
                   long long max_ts, int reps, float *ms, long long *ncands)
{
    const size_t n = (size_t)nDMs * (size_t)nT;
    if ((long long)(2 * n) >= (1LL << 31))
        return -6; /* int S/N-plane offsets of the reference, as in aaref_spd */
    unsigned long int maxTS = (max_ts <= 0) ? (unsigned long int)n : (unsigned long int)max_ts;
    int max_boxcar_width = (int)(max_boxcar_width_in_sec / tsamp);
    int mwp = 0;
    int t_BC_widths[10] = {PD_MAXTAPS, 16, 16, 16, 8, 8, 8, 8, 8, 8};
    std::vector<int> BC_widths(t_BC_widths, t_BC_widths + 10);
    Get_max_iteration(max_boxcar_width / inBin, &BC_widths, &mwp);
    std::vector<int> h_boxcar_widths;
    Create_list_of_boxcar_widths(&h_boxcar_widths, &BC_widths, mwp);
    size_t msd_bytes = 0, dit_bytes = 0, work_bytes = 0;
    Get_MSD_plane_profile_memory_requirements(&msd_bytes, &dit_bytes, &work_bytes, nT, nDMs, &h_boxcar_widths);
    float *d_plane = NULL, *d_work = NULL, *d_msd = NULL;
    unsigned short *d_taps = NULL;
    if (cudaMalloc((void **)&d_plane, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&d_work, maxTS * 5.5 * sizeof(float) + work_bytes) != cudaSuccess ||
        cudaMalloc((void **)&d_taps, 2 * maxTS * sizeof(unsigned short)) != cudaSuccess ||
        cudaMalloc((void **)&d_msd, msd_bytes + 4096) != cudaSuccess)
        return -3;
    const size_t host_cap = n / 2 + 1 < ((size_t)1 << 24) ? n / 2 + 1 : ((size_t)1 << 24);
    std::vector<unsigned> a(host_cap), b(host_cap), d(host_cap);
    std::vector<float> c(host_cap);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int rc = 0;
    for (int r = 0; r < reps && rc == 0; r++) {
        cudaMemcpy(d_plane, d_src, n * sizeof(float), cudaMemcpyDeviceToDevice);
        cudaDeviceSynchronize();
        size_t peak_pos = 0;
        int ndms_arr[1] = {nDMs};
        int maxshift = 0;
        float lo[1] = {0.f}, hi[1] = {(float)nDMs}, st[1] = {1.f};
        analysis_output out;
        cudaEventRecord(e0, 0);
        bool ok = analysis_GPU(a.data(), b.data(), c.data(), d.data(), &peak_pos, host_cap, 0, 0.f, nT, inBin,
                               &maxshift, nDMs, ndms_arr, cutoff, sigma_constant, max_boxcar_width_in_sec, d_plane,
                               lo, hi, st, tsamp, candidate_algorithm, d_work, d_taps, d_msd, maxTS,
                               enable_msd_baseline_noise, false, false, out);
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms[r], e0, e1);
        *ncands = (long long)peak_pos;
        if (!ok)
            rc = -4;
    }
    if (cudaDeviceSynchronize() != cudaSuccess)
        rc = -5;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_plane);
    cudaFree(d_work);
    cudaFree(d_taps);
    cudaFree(d_msd);
    return rc;
}

namespace {
struct export_runner : public aa_pipeline_runner {
    bool setup() override { return true; }
    void run(int range, float ***data, size_t max_nt, int *ndms, int *inBin, const char *base, int *ranges,
             int per_file)
    {
        Export_DD_data(range, data, max_nt, ndms, inBin, std::string(base), ranges, per_file);
    }
    size_t per_file(size_t mb, size_t primary, size_t floats) { return Calculate_sd_per_file_from_file_size(mb, primary, floats); }
};
} // namespace

void aaref_export_dd_data(int range, float ***data, size_t max_nt, int *ndms, int *inBin, const char *base,
                          int *ranges_to_export, int DMs_per_file)
{
    export_runner e;
    e.run(range, data, max_nt, ndms, inBin, base, ranges_to_export, DMs_per_file);
}

size_t aaref_sd_per_file(size_t mb, size_t primary, size_t floats)
{
    export_runner e;
    return e.per_file(mb, primary, floats);
}

/* meta: tstart, tsamp, fch1, foff; imeta: nbits, nsamples, nchans, nifs.
 * buf (capacity cap elements) receives input_buffer() when read_signal
 * succeeds.  Returns the number of elements of input_buffer(), or -1 when
 * read_signal refused. */
long long aaref_sigproc_read(const char *path, double *meta, int *imeta, unsigned short *buf, long long cap)
{
    aa_sigproc_input in(path);
    aa_filterbank_metadata m = in.read_metadata();
    meta[0] = m.tstart();
    meta[1] = m.tsamp();
    meta[2] = m.fch1();
    meta[3] = m.foff();
    imeta[0] = m.nbits();
    imeta[1] = m.nsamples();
    imeta[2] = m.nchans();
    imeta[3] = m.nifs();
    if (!in.read_signal())
        return -1;
    const std::vector<unsigned short> &b = in.input_buffer();
    const long long n = (long long)b.size();
    if (buf && n <= cap)
        memcpy(buf, b.data(), (size_t)n * sizeof(unsigned short));
    return n;
}

} // extern "C"
