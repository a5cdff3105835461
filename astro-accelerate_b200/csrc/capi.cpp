// capi.cpp -- extern "C" entry points declared in include/aa_b200.h.
#include "aa_b200.h"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "autotune.hpp"
#include "ddtr_kernels.cuh"
#include "spd.cuh"
#include "export.hpp"
#include "pipeline.hpp"
#include "psr_search.hpp"
#include "planner.hpp"

using namespace aab200;

namespace {

thread_local std::string g_last_error;
std::atomic<long long> g_launches{0};

void set_error(const std::string &m) { g_last_error = m; }

// aa_analysis_plan (include/aa_analysis_plan.hpp:34-47) as the C ABI holds it
struct AnalysisPlan {
    float sigma_cutoff = 0.f, sigma_constant = 0.f, max_boxcar_width_in_sec = 0.f;
    int candidate_algorithm = 0;
    bool enable_msd_baseline_noise = false;
    bool strategy_ready = false, strategy_for_analysis = false;
};

// The object behind aa_py_pipeline_api (aa_pipeline_api<unsigned short>).
struct Api {
    pipeline_components_struct components;
    pipeline_component_option_struct options;
    FilterbankMetadata meta;
    const unsigned short *input = nullptr;
    const void *packed = nullptr; // stored SIGPROC records (aa_b200_pipeline_set_packed_input)
    int card = 0;
    PipelineOptions popt;
    std::unique_ptr<DdtrPipeline> pipe;
    std::string error;
    bool supported = true;
    std::string export_base = "DD_data"; // output_dmt files (the reference's base name)
    bool exported = false;
    // analysis (single-pulse detection) after every dedispersion step
    bool analysis_bound = false;
    AnalysisPlan aplan{};
    std::unique_ptr<SpdPlane> spd;
    float *d_spd_plane = nullptr; // the step's rows, copied for the analysis (which overwrites them)
    long long spd_max_ts = 0;     // batch size; 0 = the reference's rule from free memory
    size_t spd_capacity = 0;      // host candidate list size (SPD_max_peak_size)
    SpdCandidates cands;          // the last step's candidates
    bool write_candidates = true; // the reference's peak_analysed/analysed files
    std::string candidate_dir;    // where they go ("" = the working directory)
    // periodicity search after the last dedispersion step
    bool psr_bound = false;
    bool psr_did_run = false;
    PsrPlanParams psr_plan;
    PsrStrategy psr_strategy;
    size_t psr_free_memory = 0; // 0: the device's free memory when the plan is bound
    std::unique_ptr<PsrSearch> psr;
    void *psr_power = nullptr, *psr_inter = nullptr; // candidate lists (psr_candidates.cpp)
    std::vector<float> psr_h_power, psr_h_inter;     // the getters' copies
    ~Api()
    {
        cudaFree(d_spd_plane);
        aa_b200_psr_candidates_destroy(psr_power);
        aa_b200_psr_candidates_destroy(psr_inter);
    }
};



FilterbankMetadata to_meta(const aa_py_filterbank_metadata_struct &m)
{
    FilterbankMetadata f;
    f.tstart = m.m_tstart;
    f.tsamp = m.m_tsamp;
    f.fch1 = m.m_fch1;
    f.foff = m.m_foff;
    f.nbits = m.m_nbits;
    f.nsamples = m.m_nsamples;
    f.nchans = m.m_nchans;
    return f;
}

Api *as_api(void *p) { return static_cast<Api *>(p); }

bool api_fail(Api *a, const std::string &m)
{
    if (a && a->error.empty())
        a->error = m;
    set_error(m);
    return false;
}

int elem_bytes_for(int nbits) { return nbits <= 8 ? 1 : 2; }

// output_dmt: the DM-time output of every range in the reference's
// Export_DD_data files, DM rows per file for 1000 MB files
// (include/aa_permitted_pipelines_1.hpp:312-323 with
// include/aa_pipeline_runner.hpp:165-223).
bool export_outputs(Api *a)
{
    DdtrPipeline &P = *a->pipe;
    const DdtrStrategy &s = P.strategy();
    float ***rows = P.output_buffer();
    if (!rows)
        return api_fail(a, "output_dmt needs copy_ddtr_data_to_host");
    const int nr = static_cast<int>(s.nranges());
    const size_t inc = s.nProcessedTimesamples();
    std::vector<int> in_bin(nr), all(nr, 1);
    for (int r = 0; r < nr; ++r) {
        in_bin[r] = s.dm(r).inBin;
        if (inc / static_cast<size_t>(in_bin[r]) > static_cast<size_t>(s.total_samps(r)))
            return api_fail(a, "output_dmt: range " + std::to_string(r) + " holds fewer samples than inc/inBin");
    }
    std::string err;
    const size_t per_file = sd_per_file_from_file_size(1000, inc, 1);
    if (!export_dd_data(nr, rows, inc, s.ndms_data(), in_bin.data(), a->export_base, all.data(),
                        static_cast<int>(per_file), err))
        return api_fail(a, "output_dmt: " + err);
    a->exported = true;
    return true;
}

// Single-pulse detection on the rows the last dedispersion step wrote, as the
// reference runner does after each (chunk, range) step
// (include/aa_permitted_pipelines_generic.hpp:848-889): analysis_GPU with
// the range's tsamp (tsamp * inBin, float), tstart = tsamp * inc (float) and
// the range's DMs; the candidates replace the previous step's and go to the
// reference's candidate file.
bool run_analysis(Api *a)
{
    a->cands = SpdCandidates{};
    DdtrPipeline &P = *a->pipe;
    StepPlane sp;
    if (!P.last_step_plane(sp))
        return api_fail(a, "analysis: no dedispersed rows");
    const DdtrStrategy &s = P.strategy();
    std::string err;
    if (!a->spd) {
        long long max_elems = 0;
        for (size_t r = 0; r < s.nranges(); ++r)
            for (int tp : s.t_processed()[r])
                max_elems = std::max(max_elems, static_cast<long long>(s.ndms(r)) * tp);
        long long max_ts = a->spd_max_ts;
        if (max_ts <= 0) {
            // include/aa_analysis_strategy.hpp:219-224: 95% of the free memory
            // at 5.5 floats and 2 ushorts per sample
            size_t fr = 0, tot = 0;
            if (cudaMemGetInfo(&fr, &tot) != cudaSuccess)
                return api_fail(a, "analysis: cudaMemGetInfo failed");
            max_ts = static_cast<long long>((static_cast<double>(fr) * 0.95) / (5.5 * 4 + 2 * 2));
        }
        std::unique_ptr<SpdPlane> spd(new SpdPlane());
        if (!spd->setup(max_elems, max_ts, err))
            return api_fail(a, "analysis: " + err);
        if (cudaMalloc(&a->d_spd_plane, static_cast<size_t>(max_elems) * sizeof(float)) != cudaSuccess)
            return api_fail(a, "analysis: cudaMalloc failed");
        // include/aa_permitted_pipelines_generic.hpp:376-377
        a->spd_capacity = static_cast<size_t>(s.max_ndms()) * static_cast<size_t>(s.t_processed()[0][0]) / 2;
        a->spd = std::move(spd);
    }
    // The search decimates into its input, and the step's rows are still
    // being copied to the host (or are the kept device output): it works on a
    // device copy, taken on the pipeline's stream after the dedispersion, so
    // the copy to the host overlaps the search as it overlaps the next step.
    if (cudaMemcpy2DAsync(a->d_spd_plane, static_cast<size_t>(sp.tp) * sizeof(float), sp.d,
                          static_cast<size_t>(sp.pitch) * sizeof(float), static_cast<size_t>(sp.tp) * sizeof(float),
                          static_cast<size_t>(sp.ndms), cudaMemcpyDeviceToDevice, P.stream()) != cudaSuccess)
        return api_fail(a, "analysis: cudaMemcpy2DAsync failed");
    float *plane = a->d_spd_plane;
    const DmRange &d = s.dm(sp.range);
    const float tsamp_original = static_cast<float>(a->meta.tsamp);
    const float tsamp = tsamp_original * static_cast<float>(d.inBin);
    SpdSettings st;
    st.sigma_cutoff = a->aplan.sigma_cutoff;
    st.sigma_constant = a->aplan.sigma_constant;
    st.max_boxcar_width_in_sec = a->aplan.max_boxcar_width_in_sec;
    st.candidate_algorithm = a->aplan.candidate_algorithm;
    st.enable_msd_baseline_noise = a->aplan.enable_msd_baseline_noise ? 1 : 0;
    if (!a->spd->run(plane, sp.ndms, sp.tp, tsamp, d.inBin, st, a->cands, P.stream(), err, a->spd_capacity))
        return api_fail(a, "analysis: " + err);
    if (a->write_candidates && !a->cands.dm.empty()) {
        const float tstart = tsamp_original * static_cast<float>(sp.inc);
        if (aa_b200_spd_write_candidates(a->candidate_dir.c_str(), st.candidate_algorithm, tstart, d.low, d.high,
                                         d.step, tsamp, d.inBin, a->cands.dm.data(), a->cands.ts.data(),
                                         a->cands.snr.data(), a->cands.bw.data(), a->cands.dm.size()))
            return api_fail(a, aa_b200_spd_last_error(nullptr));
    }
    return true;
}

} // namespace

namespace aab200 {
// the message aa_b200_last_error() returns, for the library's other C-ABI files
void set_last_error(const std::string &m) { set_error(m); }
} // namespace aab200

extern "C" {

// ---------------------------------------------------------------------------
// metadata (src/aa_py_filterbank_metadata.cpp)
// ---------------------------------------------------------------------------
aa_py_filterbank_metadata_struct *aa_py_filterbank_metadata(double tstart, double tsamp, int nbits, int nsamples,
                                                            double fch1, double foff, int nchans, double src_raj)
{
    auto *m = new aa_py_filterbank_metadata_struct;
    m->m_tstart = tstart;
    m->m_tsamp = tsamp;
    m->m_fch1 = fch1;
    m->m_foff = foff;
    m->m_nbits = nbits;
    m->m_nsamples = nsamples;
    m->m_nchans = nchans;
    m->m_src_raj = src_raj;
    return m;
}
void aa_py_filterbank_metadata_delete(const aa_py_filterbank_metadata_struct *obj) { delete obj; }
double aa_py_filterbank_metadata_tstart(const aa_py_filterbank_metadata_struct *obj) { return obj->m_tstart; }

// ---------------------------------------------------------------------------
// plan (src/aa_py_ddtr_plan.cpp)
// ---------------------------------------------------------------------------
void *aa_py_ddtr_plan(void) { return new DdtrPlan(); }
void aa_py_ddtr_plan_delete(const void *obj) { delete static_cast<const DdtrPlan *>(obj); }
bool aa_py_ddtr_plan_add_dm(void *obj, float low, float high, float step, int inBin, int outBin)
{
    return static_cast<DdtrPlan *>(obj)->add_dm(low, high, step, inBin, outBin);
}
size_t aa_py_ddtr_plan_range(const void *obj) { return static_cast<const DdtrPlan *>(obj)->range(); }
bool aa_py_ddtr_plan_set_power(void *obj, float power) { return static_cast<DdtrPlan *>(obj)->set_power(power); }
float aa_py_ddtr_plan_power(const void *obj) { return static_cast<const DdtrPlan *>(obj)->power(); }
bool aa_py_ddtr_plan_set_enable_msd_baseline(void *obj, bool flag)
{
    return static_cast<DdtrPlan *>(obj)->set_enable_msd_baseline_noise(flag);
}
bool aa_py_ddtr_plan_enable_msd_baseline_noise(const void *obj)
{
    return static_cast<const DdtrPlan *>(obj)->enable_msd_baseline_noise();
}
bool aa_py_ddtr_plan_bind_bandpass_normalization(void *obj, const float *data, int data_size)
{
    return static_cast<DdtrPlan *>(obj)->bind_bandpass_normalization(data, data_size);
}

// ---------------------------------------------------------------------------
// pipeline (src/aa_py_pipeline_api.cpp)
// ---------------------------------------------------------------------------
void *aa_py_pipeline_api(pipeline_components_struct pipeline, pipeline_component_option_struct options,
                         aa_py_filterbank_metadata_struct metadata, const unsigned short *input_data,
                         int card_number)
{
    Api *a = new Api();
    a->components = pipeline;
    a->options = options;
    a->meta = to_meta(metadata);
    a->input = input_data;
    a->card = card_number;
    a->popt.copy_to_host = options.copy_ddtr_data_to_host;
    if (pipeline.fdas || !pipeline.dedispersion) {
        a->supported = false;
        api_fail(a, "the dedispersion, analysis and periodicity components are implemented by this library");
    }
    // the periodicity search reads the host rows, as the reference's runner
    // does (include/aa_permitted_pipelines_generic.hpp:590), unless they are
    // kept on the device (aa_b200_pipeline_set_device_output)
    if (pipeline.periodicity)
        a->popt.copy_to_host = true;
    a->popt.enable_analysis = pipeline.analysis;
    // include/aa_py_pipeline_api.cpp:24-35 -> the runner's options
    a->popt.zero_dm = options.zero_dm;
    a->popt.zero_dm_outliers = options.zero_dm_with_outliers;
    a->popt.input_norm = options.input_DDTR_normalization;
    a->popt.output_norm = options.output_DDTR_normalization;
    a->popt.old_rfi = options.old_rfi;
    a->popt.bandpass_average = options.set_bandpass_average;
    return a;
}

void aa_py_pipeline_api_delete(const void *obj) { delete static_cast<const Api *>(obj); }

bool aa_py_pipeline_api_bind_ddtr_plan(void *obj, const void *plan)
{
    Api *a = as_api(obj);
    if (!a->supported)
        return false;
    if (a->pipe)
        return api_fail(a, "a DDTR plan is already bound");
    if (cudaSetDevice(a->card) != cudaSuccess)
        return api_fail(a, "cannot select CUDA device " + std::to_string(a->card));
    a->pipe.reset(new DdtrPipeline(a->meta, a->popt.packed_input ? a->packed : static_cast<const void *>(a->input),
                                   a->popt));
    if (!a->pipe->bind(*static_cast<const DdtrPlan *>(plan))) {
        api_fail(a, a->pipe->last_error());
        a->pipe.reset();
        return false;
    }
    return true;
}

void *aa_py_pipeline_api_ddtr_strategy(void *obj)
{
    Api *a = as_api(obj);
    if (!a->pipe)
        return nullptr;
    return new DdtrStrategy(a->pipe->strategy());
}
void aa_py_ddtr_strategy_delete(const void *obj) { delete static_cast<const DdtrStrategy *>(obj); }

size_t aa_py_get_ddtr_nRanges(void *obj)
{
    Api *a = as_api(obj);
    return a->pipe ? a->pipe->strategy().nranges() : 0;
}
const int *aa_py_get_ndms_array(void *obj)
{
    Api *a = as_api(obj);
    return a->pipe ? a->pipe->strategy().ndms_data() : nullptr;
}
int aa_py_get_t_proc(void *obj, int i, int j)
{
    Api *a = as_api(obj);
    return a->pipe ? a->pipe->strategy().t_processed()[i][j] : 0;
}
int aa_py_dm_low(void *obj, int range)
{
    Api *a = as_api(obj);
    return a->pipe ? static_cast<int>(a->pipe->strategy().dm(range).low) : 0;
}
int aa_py_total_computed_samples(void *obj)
{
    Api *a = as_api(obj);
    return a->pipe ? static_cast<int>(a->pipe->strategy().nProcessedTimesamples()) : 0;
}

// src/aa_py_analysis_plan.cpp:6-17: the plan keeps the DDTR strategy's state
void *aa_py_analysis_plan(const void *ddtr_strategy, float sigma_cutoff, float sigma_constant,
                          float max_boxcar_width_in_sec, int candidate_algorithm, bool enable_msd_baseline_noise)
{
    AnalysisPlan *p = new AnalysisPlan();
    p->sigma_cutoff = sigma_cutoff;
    p->sigma_constant = sigma_constant;
    p->max_boxcar_width_in_sec = max_boxcar_width_in_sec;
    // values other than 1 and 2 select peak finding (:7-14)
    p->candidate_algorithm = (candidate_algorithm == 1 || candidate_algorithm == 2) ? candidate_algorithm : 0;
    p->enable_msd_baseline_noise = enable_msd_baseline_noise;
    const DdtrStrategy *s = static_cast<const DdtrStrategy *>(ddtr_strategy);
    p->strategy_ready = s && s->ready();
    p->strategy_for_analysis = s && s->configured_for_analysis();
    return p;
}
void aa_analysis_plan_delete(const void *obj) { delete static_cast<const AnalysisPlan *>(obj); }
float aa_py_analysis_plan_sigma_cutoff(const void *obj) { return static_cast<const AnalysisPlan *>(obj)->sigma_cutoff; }
float aa_py_analysis_plan_sigma_constant(const void *obj)
{
    return static_cast<const AnalysisPlan *>(obj)->sigma_constant;
}
float aa_py_analysis_plan_max_boxcar_width_in_sec(const void *obj)
{
    return static_cast<const AnalysisPlan *>(obj)->max_boxcar_width_in_sec;
}
bool aa_py_analysis_plan_enable_msd_baseline_noise(const void *obj)
{
    return static_cast<const AnalysisPlan *>(obj)->enable_msd_baseline_noise;
}

// include/aa_pipeline_api.hpp:182-219 with the readiness rules of
// include/aa_analysis_strategy.hpp:67-93
bool aa_py_pipeline_api_bind_analysis_plan(void *obj, const void *plan)
{
    Api *a = as_api(obj);
    if (!a->supported)
        return false;
    if (!a->components.analysis)
        return api_fail(a, "the analysis component was not requested");
    if (a->analysis_bound)
        return api_fail(a, "an analysis plan is already bound");
    const AnalysisPlan *p = static_cast<const AnalysisPlan *>(plan);
    if (!p || !p->strategy_ready)
        return api_fail(a, "the analysis plan's DDTR strategy is not ready");
    if (!(p->sigma_cutoff > 0) || !(p->sigma_constant > 0) || !(p->max_boxcar_width_in_sec > 0))
        return api_fail(a, "analysis needs sigma_cutoff, sigma_constant and max_boxcar_width_in_sec above 0");
    if (!p->strategy_for_analysis)
        return api_fail(a, "the DDTR strategy was not computed for analysis");
    a->aplan = *p;
    a->analysis_bound = true;
    return true;
}

// :78-80: a new object per call (the reference never frees it); here the
// bound analysis settings, or NULL when no analysis plan is bound.  Free with
// aa_analysis_plan_delete.
void *aa_py_pipeline_api_analysis_strategy(void *obj)
{
    Api *a = as_api(obj);
    if (!a->analysis_bound)
        return nullptr;
    return new AnalysisPlan(a->aplan);
}

// :129-141: periodicity candidates (Get_PSR_candidates and
// Write_to_disk_PSR_candidates of include/aa_permitted_pipelines_generic.hpp:1173-1193):
// the records (DM, frequency, S/N, harmonics) of every batch in order, in a
// copy owned by the pipeline object (valid until the next call of the same
// getter); NULL with an error message when the search has not run.
namespace {
float *psr_copy(Api *a, bool interbin)
{
    void *list = interbin ? a->psr_inter : a->psr_power;
    if (!list || !a->psr_did_run) {
        api_fail(a, "no periodicity candidates: the periodicity search has not run");
        return nullptr;
    }
    std::vector<float> &h = interbin ? a->psr_h_inter : a->psr_h_power;
    h.assign(4 * aa_b200_psr_candidates_count(list) + 4, 0.f);
    aa_b200_psr_candidates_copy(list, h.data());
    return h.data();
}
} // namespace

float *aa_py_get_psr_nCandidates(void *obj) { return psr_copy(as_api(obj), false); }
float *aa_py_get_psr_interbin_nCandidates(void *obj) { return psr_copy(as_api(obj), true); }
void aa_py_write_to_disk_psr_candidates(void *obj, const char *filename)
{
    Api *a = as_api(obj);
    if (!a->psr_power || !a->psr_did_run) {
        api_fail(a, "no periodicity candidates: the periodicity search has not run");
        return;
    }
    if (aa_b200_psr_candidates_export(a->psr_power, filename) != 0)
        api_fail(a, aa_b200_psr_candidates_last_error());
}

size_t aa_py_spd_nCandidates(void *obj) { return as_api(obj)->cands.dm.size(); }
unsigned int *aa_py_h_dm(void *obj)
{
    Api *a = as_api(obj);
    return a->cands.dm.empty() ? nullptr : a->cands.dm.data();
}
unsigned int *aa_py_h_ts(void *obj)
{
    Api *a = as_api(obj);
    return a->cands.ts.empty() ? nullptr : a->cands.ts.data();
}
float *aa_py_h_snr(void *obj)
{
    Api *a = as_api(obj);
    return a->cands.snr.empty() ? nullptr : a->cands.snr.data();
}
unsigned int *aa_py_h_width(void *obj)
{
    Api *a = as_api(obj);
    return a->cands.bw.empty() ? nullptr : a->cands.bw.data();
}
namespace {
// aa_pipeline_api::bind(aa_periodicity_plan) (include/aa_pipeline_api.hpp:226-253)
// with the plan extracted from the DDTR strategy
// (include/aa_periodicity_plan.hpp:292-321): every range's DM grid, binning
// and trial count, the processed samples of the whole run and the data's
// sampling time; the strategy for the device's free memory
bool bind_psr(Api *a, const PsrPlanParams &p)
{
    if (!a->supported)
        return false;
    if (!a->components.periodicity)
        return api_fail(a, "the pipeline was created without the periodicity component");
    if (a->psr_bound)
        return api_fail(a, "a periodicity plan is already bound");
    if (!a->pipe)
        return api_fail(a, "bind the DDTR plan before the periodicity plan");
    const DdtrStrategy &S = a->pipe->strategy();
    std::vector<PsrDdtrRange> ranges;
    for (size_t r = 0; r < S.nranges(); ++r) {
        PsrDdtrRange d;
        d.dm_low = S.dm(r).low;
        d.dm_high = S.dm(r).high;
        d.dm_step = S.dm(r).step;
        d.inBin = S.dm(r).inBin;
        d.nTimesamples = S.nProcessedTimesamples();
        d.nDMs = S.ndms(r);
        d.sampling_time = a->meta.tsamp;
        ranges.push_back(d);
    }
    size_t free_mem = a->psr_free_memory;
    if (free_mem == 0) {
        size_t total = 0;
        if (cudaSetDevice(a->card) != cudaSuccess || cudaMemGetInfo(&free_mem, &total) != cudaSuccess)
            return api_fail(a, "cannot read the device's free memory");
    }
    std::string err;
    if (!psr_strategy(p, ranges, free_mem, a->psr_strategy, err))
        return api_fail(a, err);
    a->psr_plan = p;
    a->psr_bound = true;
    return true;
}

// GPU_periodicity (src/aa_device_periods.cu:570-682) over the finished run's
// output rows, host or device
bool run_psr(Api *a)
{
    std::string err;
    if (!a->psr)
        a->psr.reset(new PsrSearch());
    if (!a->psr->setup(a->psr_strategy, err))
        return api_fail(a, err);
    aa_b200_psr_candidates_destroy(a->psr_power);
    aa_b200_psr_candidates_destroy(a->psr_inter);
    a->psr_power = aa_b200_psr_candidates_create();
    a->psr_inter = aa_b200_psr_candidates_create();
    if (!a->psr_power || !a->psr_inter)
        return api_fail(a, "periodicity search: out of host memory");
    const DdtrStrategy &S = a->pipe->strategy();
    std::vector<PsrRows> rows(S.nranges());
    float ***host = a->pipe->output_buffer();
    for (size_t r = 0; r < S.nranges(); ++r) {
        PsrRows &R = rows[r];
        R.pitch = S.total_samps(r);
        R.row_len = S.total_samps(r);
        if (a->pipe->device_output(static_cast<int>(r))) {
            R.base = a->pipe->device_output(static_cast<int>(r));
            R.on_device = true;
        } else if (host && host[r]) {
            R.base = host[r][0];
            R.on_device = false;
        } else {
            return api_fail(a, "periodicity search: the DM-time rows are neither on the host nor on the device");
        }
    }
    if (!a->psr->run(a->psr_strategy, rows, a->psr_power, a->psr_inter, a->pipe->stream(), err))
        return api_fail(a, err);
    a->psr_did_run = true;
    // the search's device buffers go (GPU_Memory_for_Periodicity_Search's
    // lifetime, :578-590)
    a->psr->release();
    return true;
}
} // namespace

bool aa_py_pipeline_api_bind_periodicity_plan(void *obj, float sigma_cutoff, bool enable_outlier_rejection,
                                              float sigma_outlier_rejection_threshold, int nHarmonics,
                                              int candidate_selection_algorithm)
{
    // src/aa_py_pipeline_api.cpp:82-85 -> aa_periodicity_plan's six-argument
    // constructor (include/aa_periodicity_plan.hpp:39-60): greedy harmonic
    // sum, scalloping-loss mitigation, interbinning and whitening on
    PsrPlanParams p;
    p.sigma_cutoff = sigma_cutoff;
    p.enable_outlier_rejection = enable_outlier_rejection;
    p.sigma_outlier_rejection_threshold = sigma_outlier_rejection_threshold;
    p.nHarmonics = nHarmonics;
    p.harmonic_sum_algorithm = 1;
    p.candidate_selection_algorithm = candidate_selection_algorithm;
    return bind_psr(as_api(obj), p);
}

bool aa_b200_pipeline_bind_periodicity_plan(void *obj, float sigma_cutoff, int enable_outlier_rejection,
                                            float sigma_outlier_rejection_threshold, int nHarmonics,
                                            int harmonic_sum_algorithm, int candidate_selection_algorithm,
                                            int enable_scalloping_loss_mitigation, int enable_interbinning,
                                            int enable_spectrum_whitening)
{
    PsrPlanParams p;
    p.sigma_cutoff = sigma_cutoff;
    p.enable_outlier_rejection = enable_outlier_rejection != 0;
    p.sigma_outlier_rejection_threshold = sigma_outlier_rejection_threshold;
    p.nHarmonics = nHarmonics;
    p.harmonic_sum_algorithm = harmonic_sum_algorithm;
    p.candidate_selection_algorithm = candidate_selection_algorithm;
    p.enable_scalloping_loss_mitigation = enable_scalloping_loss_mitigation != 0;
    p.enable_interbinning = enable_interbinning != 0;
    p.enable_spectrum_whitening = enable_spectrum_whitening != 0;
    return bind_psr(as_api(obj), p);
}

bool aa_b200_pipeline_set_periodicity_memory(void *obj, size_t bytes)
{
    Api *a = as_api(obj);
    if (a->psr_bound)
        return api_fail(a, "set the periodicity memory before binding the periodicity plan");
    a->psr_free_memory = bytes;
    return true;
}

size_t aa_b200_pipeline_psr_count(void *obj, int interbin)
{
    Api *a = as_api(obj);
    void *list = interbin ? a->psr_inter : a->psr_power;
    return list ? aa_b200_psr_candidates_count(list) : 0;
}

bool aa_b200_pipeline_write_psr_interbin_candidates(void *obj, const char *filename)
{
    Api *a = as_api(obj);
    if (!a->psr_inter || !a->psr_did_run)
        return api_fail(a, "no periodicity candidates: the periodicity search has not run");
    if (aa_b200_psr_candidates_export(a->psr_inter, filename) != 0)
        return api_fail(a, aa_b200_psr_candidates_last_error());
    return true;
}

int aa_b200_pipeline_psr_info(void *obj, size_t *fft_length, size_t *dms_per_batch, int *batches, double *compute_ms)
{
    Api *a = as_api(obj);
    if (!a->psr_bound)
        return 1;
    int nb = 0;
    for (const PsrRange &R : a->psr_strategy.ranges)
        nb += static_cast<int>(R.batches.size());
    *fft_length = a->psr_strategy.corrected_max_nTimesamples;
    *dms_per_batch = a->psr_strategy.max_nDMs_in_memory;
    *batches = nb;
    *compute_ms = a->psr ? a->psr->last_compute_ms : 0.0;
    return 0;
}
bool aa_py_pipeline_api_bind_fdas_plan(void *obj, float, float, bool)
{
    return api_fail(as_api(obj), "FDAS is not implemented by this library");
}

bool aa_py_pipeline_api_run(void *obj, int *status_code)
{
    Api *a = as_api(obj);
    if (!a->supported || !a->pipe || !a->pipe->ready()) {
        *status_code = static_cast<int>(RunStatus::error);
        if (!a->pipe)
            api_fail(a, "no DDTR plan bound");
        return false;
    }
    if (a->components.analysis && !a->analysis_bound) {
        *status_code = static_cast<int>(RunStatus::error);
        return api_fail(a, "the analysis component needs an analysis plan bound");
    }
    RunStatus st = RunStatus::finished;
    const bool more = a->pipe->next(st);
    *status_code = static_cast<int>(st);
    if (st == RunStatus::error) {
        api_fail(a, a->pipe->last_error());
        return false;
    }
    if (st == RunStatus::has_more && a->analysis_bound && !run_analysis(a)) {
        *status_code = static_cast<int>(RunStatus::error);
        return false;
    }
    if (!more && st == RunStatus::finished && a->options.output_dmt && !a->exported &&
        (!a->pipe->synchronize() || !export_outputs(a))) {
        if (a->error.empty())
            api_fail(a, a->pipe->last_error());
        *status_code = static_cast<int>(RunStatus::error);
        return false;
    }
    // include/aa_permitted_pipelines_generic.hpp:650-655: after the
    // dedispersion component finished, one more call runs the periodicity
    // search and reports finished_component
    if (!more && st == RunStatus::finished && a->components.periodicity && !a->psr_did_run) {
        if (!a->psr_bound) {
            *status_code = static_cast<int>(RunStatus::error);
            return api_fail(a, "the periodicity component needs a periodicity plan bound");
        }
        if (!a->pipe->synchronize() || !run_psr(a)) {
            if (a->error.empty())
                api_fail(a, a->pipe->last_error());
            *status_code = static_cast<int>(RunStatus::error);
            return false;
        }
        *status_code = static_cast<int>(RunStatus::finished_component);
        return true;
    }
    return more;
}

float ***aa_py_buffer(void *obj)
{
    Api *a = as_api(obj);
    return a->pipe ? a->pipe->output_buffer() : nullptr;
}
int aa_py_current_range(void *obj)
{
    Api *a = as_api(obj);
    return a->pipe ? a->pipe->current_range() : 0;
}
int aa_py_current_time_chunk(void *obj)
{
    Api *a = as_api(obj);
    return a->pipe ? a->pipe->current_tchunk() : 0;
}
long aa_py_current_inc(void *obj)
{
    Api *a = as_api(obj);
    return a->pipe ? static_cast<long>(a->pipe->current_inc()) : 0;
}
bool aa_py_cleanup(void *obj)
{
    Api *a = as_api(obj);
    // the analysis buffers go with the pipeline's (the runner frees its SPD
    // work area in its cleanup, include/aa_permitted_pipelines_generic.hpp:205-240);
    // a later step sets them up again
    a->spd.reset();
    cudaFree(a->d_spd_plane);
    a->d_spd_plane = nullptr;
    return a->pipe ? a->pipe->cleanup() : true;
}

// ---------------------------------------------------------------------------
// seam
// ---------------------------------------------------------------------------
int aa_b200_strategy(const aa_b200_dm *plan, int nranges, float power, int nchans, int nsamp, double fch1,
                     double foff, double tsamp, int nbits, size_t free_memory, int enable_analysis, int max_chunks,
                     float *dmshifts, int *ndms, aa_b200_dm *str_dm, int *maxshift, int *max_ndms, int *num_tchunks,
                     int *t_processed)
{
    DdtrPlan p;
    for (int i = 0; i < nranges; ++i)
        p.add_dm(plan[i].low, plan[i].high, plan[i].step, plan[i].inBin, plan[i].outBin);
    p.set_power(power);
    FilterbankMetadata m;
    m.tsamp = tsamp;
    m.fch1 = fch1;
    m.foff = foff;
    m.nbits = nbits;
    m.nsamples = nsamp;
    m.nchans = nchans;
    DdtrStrategy s;
    const StrategyStatus rc = s.compute(p, m, free_memory, enable_analysis != 0);
    if (rc != STRAT_OK) {
        set_error("strategy refused the plan");
        return static_cast<int>(rc);
    }
    if (s.num_tchunks() > max_chunks) {
        set_error("more time chunks than max_chunks");
        return -5;
    }
    std::copy(s.dmshifts().begin(), s.dmshifts().end(), dmshifts);
    for (int i = 0; i < nranges; ++i) {
        ndms[i] = s.ndms(i);
        const DmRange &d = s.dm(i);
        str_dm[i] = aa_b200_dm{d.low, d.high, d.step, d.inBin, d.outBin};
        for (int k = 0; k < s.num_tchunks(); ++k)
            t_processed[i * max_chunks + k] = s.t_processed()[i][k];
    }
    *maxshift = s.maxshift();
    *max_ndms = s.max_ndms();
    *num_tchunks = s.num_tchunks();
    return 0;
}

int aa_b200_psr_strategy(const aa_b200_dm *plan, int nranges, int nchans, int nsamp, double tsamp, double fch1,
                         double foff, int nbits, size_t ddtr_memory, size_t memory_available, float sigma_cutoff,
                         int nHarmonics, int harmonic_sum_algorithm, long long *info, long long *range_info,
                         int max_ranges, long long *batches, int max_batches)
{
    DdtrPlan p;
    for (int i = 0; i < nranges; ++i)
        p.add_dm(plan[i].low, plan[i].high, plan[i].step, plan[i].inBin, plan[i].outBin);
    FilterbankMetadata m;
    m.tsamp = tsamp;
    m.fch1 = fch1;
    m.foff = foff;
    m.nbits = nbits;
    m.nsamples = nsamp;
    m.nchans = nchans;
    DdtrStrategy s;
    if (s.compute(p, m, ddtr_memory, false) != STRAT_OK) {
        set_error("strategy refused the plan");
        return -1;
    }
    std::vector<PsrDdtrRange> ranges;
    for (size_t r = 0; r < s.nranges(); ++r) {
        PsrDdtrRange d;
        d.dm_low = s.dm(r).low;
        d.dm_high = s.dm(r).high;
        d.dm_step = s.dm(r).step;
        d.inBin = s.dm(r).inBin;
        d.nTimesamples = s.nProcessedTimesamples();
        d.nDMs = s.ndms(r);
        d.sampling_time = tsamp;
        ranges.push_back(d);
    }
    PsrPlanParams pp;
    pp.sigma_cutoff = sigma_cutoff;
    pp.nHarmonics = nHarmonics;
    pp.harmonic_sum_algorithm = harmonic_sum_algorithm;
    PsrStrategy ps;
    std::string err;
    info[6] = psr_strategy(pp, ranges, memory_available, ps, err) ? 1 : 0;
    if (!info[6]) {
        set_error(err);
        return 0;
    }
    info[0] = static_cast<long long>(ps.corrected_max_nTimesamples);
    info[1] = static_cast<long long>(ps.nTimesamples_to_copy);
    info[3] = static_cast<long long>(ps.input_plane_size);
    info[4] = static_cast<long long>(ps.cufft_workarea_size);
    info[5] = static_cast<long long>(ps.max_total_MSD_blocks);
    int nb = 0;
    for (size_t r = 0; r < ps.ranges.size(); ++r) {
        const PsrRange &R = ps.ranges[r];
        if (static_cast<int>(r) < max_ranges) {
            range_info[2 * r] = static_cast<long long>(R.range.nTimesamples);
            range_info[2 * r + 1] = static_cast<long long>(R.batches.size());
        }
        for (const PsrBatch &b : R.batches) {
            if (nb < max_batches) {
                batches[5 * nb + 0] = static_cast<long long>(r);
                batches[5 * nb + 1] = static_cast<long long>(b.nDMs_per_batch);
                batches[5 * nb + 2] = static_cast<long long>(b.DM_shift);
                batches[5 * nb + 3] = static_cast<long long>(b.nTimesamples);
                batches[5 * nb + 4] = static_cast<long long>(b.nTimesamples_to_copy);
            }
            ++nb;
        }
    }
    info[2] = (!ps.ranges.empty() && !ps.ranges[0].batches.empty())
                  ? static_cast<long long>(ps.ranges[0].batches[0].nDMs_per_batch) /
                        std::max(1, ps.ranges[0].range.inBin)
                  : 0;
    return nb;
}

int aa_b200_select_kernel(int nbits, float dm_step, float tsamp, float dmshift_last, int failsafe)
{
    return select_delay_kind(nbits, dm_step, tsamp, dmshift_last, failsafe);
}

int aa_b200_corner_turn(const unsigned short *d_in_tc, void *d_out, int nbits, int nchans, long long nsamp,
                        long long out_stride, void *stream)
{
    int *d_err = nullptr;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMalloc(&d_err, sizeof(int)) != cudaSuccess) {
        set_error("cudaMalloc failed");
        return 1;
    }
    cudaMemsetAsync(d_err, 0, sizeof(int), st);
    const int max_value = (nbits == 4) ? 15 : (nbits <= 8 ? 255 : 65535);
    cudaError_t e = launch_corner_turn(d_in_tc, d_out, elem_bytes_for(nbits), nchans, nsamp, out_stride, max_value,
                                       d_err, st);
    ++g_launches;
    int h = 0;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    cudaFree(d_err);
    if (e != cudaSuccess) {
        set_error(cudaGetErrorString(e));
        return 1;
    }
    if (h) {
        set_error("input sample above the bit depth's range");
        return 1;
    }
    return 0;
}

int aa_b200_bin_gpu(const void *d_src, void *d_dst, int nbits, int nchans, long long nsamp, void *stream)
{
    if (nsamp <= 0 || (nsamp & 1)) {
        set_error("nsamp must be positive and even");
        return 1;
    }
    cudaError_t e = launch_bin_flat(d_src, d_dst, elem_bytes_for(nbits), nchans, nsamp, static_cast<cudaStream_t>(stream));
    ++g_launches;
    if (e != cudaSuccess) {
        set_error(cudaGetErrorString(e));
        return 1;
    }
    return 0;
}

int aa_b200_dedisperse(int i, int t_processed, const int *inBin, const float *dmshifts, const void *d_input,
                       long long i_nsamp, size_t d_input_elems, float *d_output, long long out_pitch, int nchans,
                       const float *tsamp, const float *dm_low, const float *dm_step, const int *ndms, int nbits,
                       int failsafe, void *stream)
{
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int eb = elem_bytes_for(nbits);
    const int nd = ndms[i];
    if (nd <= 0 || (nd % 4) || t_processed <= 0 || (t_processed & 3) || nchans <= 0) {
        set_error("ndms must be a positive multiple of 4 and t_processed a positive multiple of 4");
        return 1;
    }
    const float mstartdm = dm_low[i] / *tsamp; // src/aa_dedisperse.cpp:28,37-40
    const float mdmstep = dm_step[i] / *tsamp;
    const int kind = select_delay_kind(nbits, dm_step[i], *tsamp, dmshifts[nchans - 1], failsafe);
    const int nch_used = (kind == KIND_SHARED4 && nchans > 4096) ? 4096 * (nchans / 4096) : nchans;
    const int nch_pad = (nchans + 3) & ~3;
    const size_t nent = static_cast<size_t>(nchans) * nd;
    float *d_shifts = nullptr;
    int32_t *d_table = nullptr, *d_wmin = nullptr, *d_off = nullptr;
    int *d_flags = nullptr; // [0] error flags, [1] span, [2] max delay
    int h[3] = {0, 0, 0};
    int rc = 1;
    const int tile_words = 4;
    int gd = 0;
    cudaError_t e = cudaMalloc(&d_shifts, sizeof(float) * nchans);
    if (e == cudaSuccess)
        e = cudaMalloc(&d_table, nent * sizeof(int32_t));
    if (e == cudaSuccess)
        e = cudaMalloc(&d_flags, 3 * sizeof(int));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_shifts, dmshifts, sizeof(float) * nchans, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(d_flags, 0, 3 * sizeof(int), st);
    if (e == cudaSuccess) {
        e = launch_delay_table(d_shifts, nchans, nd, kind, FMA_ALL, mstartdm, mdmstep, d_table, d_flags, st);
        ++g_launches;
    }
    // DM group: the largest that fits shared memory
    for (int cand : {64, 32, 16, 8, 4}) {
        if (e != cudaSuccess)
            break;
        if (nd % cand)
            continue;
        cudaFree(d_wmin);
        d_wmin = nullptr;
        e = cudaMalloc(&d_wmin, static_cast<size_t>(nd / cand) * nch_pad * sizeof(int32_t));
        if (e == cudaSuccess)
            e = cudaMemsetAsync(d_flags + 1, 0, 2 * sizeof(int), st);
        if (e == cudaSuccess) {
            e = launch_group_windows(d_table, nchans, nd, cand, d_wmin, d_flags + 1, d_flags + 2, st);
            ++g_launches;
        }
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
    if (e == cudaSuccess && gd == 0)
        set_error("no DM-group size fits the delay span");
    else if (e == cudaSuccess && h[0] != 0)
        set_error("delay outside [0, 2^24) or class step > 1");
    else if (e == cudaSuccess) {
        const long long tile = 128LL * tile_words;
        long long need;
        if (eb == 1)
            need = static_cast<long long>(nch_used - 1) * i_nsamp + ((t_processed + tile - 1) / tile) * tile + h[2] +
                   4LL * ddtr_u8_rw(h[1], tile_words) + 64;
        else
            need = static_cast<long long>(nch_used - 1) * i_nsamp + t_processed + h[2] + 2;
        if (need > static_cast<long long>(d_input_elems)) {
            set_error("d_input needs " + std::to_string(need) + " elements including window padding, has " +
                      std::to_string(d_input_elems));
        } else {
            if (eb == 1) {
                e = cudaMalloc(&d_off, nent * sizeof(int32_t));
                if (e == cudaSuccess) {
                    e = launch_offset_table(d_table, d_wmin, nchans, nd, gd, ddtr_u8_rw(h[1], tile_words), h[1],
                                            d_off, st);
                    ++g_launches;
                }
            }
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
            if (e == cudaSuccess) {
                e = (eb == 1) ? launch_ddtr_u8(p, d_off, tile_words, st) : launch_ddtr_u16(p, st);
                ++g_launches;
            }
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(h, d_flags, sizeof(int), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess)
                e = cudaStreamSynchronize(st);
            if (e == cudaSuccess && h[0] == 0)
                rc = 0;
            else if (e == cudaSuccess)
                set_error("device reported an error flag " + std::to_string(h[0]));
        }
    }
    if (e != cudaSuccess)
        set_error(cudaGetErrorString(e));
    cudaFree(d_shifts);
    cudaFree(d_table);
    cudaFree(d_wmin);
    cudaFree(d_off);
    cudaFree(d_flags);
    return rc;
}

const char *aa_b200_last_error(void) { return g_last_error.c_str(); }

long long aa_b200_kernel_launches(void) { return g_launches.load(); }

const char *aa_b200_version(void) { return "aa_b200 0.1 (sm_100a)"; }

// ---------------------------------------------------------------------------
// pipeline extensions
// ---------------------------------------------------------------------------
bool aa_b200_pipeline_set_options(void *obj, int stride_mode, int fma_mode, int failsafe, size_t free_memory,
                                  int tile_words, int group_dms)
{
    Api *a = as_api(obj);
    if (a->pipe)
        return api_fail(a, "options must be set before the plan is bound");
    if (stride_mode != STRIDE_REFERENCE && stride_mode != STRIDE_TRUE)
        return api_fail(a, "stride_mode must be 0 or 1");
    if (tile_words != 0 && tile_words != 2 && tile_words != 4)
        return api_fail(a, "tile_words must be 0, 2 or 4");
    a->popt.stride_mode = stride_mode;
    a->popt.fma_mode = fma_mode;
    a->popt.failsafe = failsafe;
    a->popt.free_memory = free_memory;
    a->popt.tile_words = tile_words;
    a->popt.group_dms = group_dms;
    return true;
}

void *aa_b200_pipeline_create(aa_py_filterbank_metadata_struct metadata, const unsigned short *input, int device_input,
                              int device_output, int copy_to_host, void *stream, int card_number)
{
    pipeline_components_struct comp{true, false, false, false};
    pipeline_component_option_struct opt{};
    opt.copy_ddtr_data_to_host = copy_to_host != 0;
    Api *a = static_cast<Api *>(aa_py_pipeline_api(comp, opt, metadata, input, card_number));
    a->popt.device_input = device_input != 0;
    a->popt.device_output = device_output != 0;
    a->popt.stream = static_cast<cudaStream_t>(stream);
    return a;
}

bool aa_b200_pipeline_set_packed_input(void *obj, const void *packed)
{
    Api *a = as_api(obj);
    if (a->pipe)
        return api_fail(a, "the packed input must be set before the plan is bound");
    if (!packed)
        return api_fail(a, "the packed input pointer is null");
    a->packed = packed;
    a->popt.packed_input = true;
    return true;
}

bool aa_b200_pipeline_set_device_output(void *obj, int on)
{
    Api *a = as_api(obj);
    if (a->pipe)
        return api_fail(a, "the device output must be chosen before the plan is bound");
    a->popt.device_output = on != 0;
    return true;
}

bool aa_b200_pipeline_set_autotune(void *obj, int enable)
{
    Api *a = as_api(obj);
    if (a->pipe)
        return api_fail(a, "autotuning must be chosen before the plan is bound");
    a->popt.autotune = enable != 0;
    return true;
}

bool aa_b200_pipeline_set_kernel_variant(void *obj, int variant)
{
    Api *a = as_api(obj);
    if (a->pipe)
        return api_fail(a, "the kernel variant must be set before the plan is bound");
    if (variant < 0 || variant > 12)
        return api_fail(a, "kernel variant must be 0 (auto), 1 (generic kernels), 2 (channel-quad / fp32 kernels), "
                           "3 (subband / fp32 kernels), 4 (warp-specialised channel-quad / fp32 kernels), 5 "
                           "(split-phase channel-quad / fp32 kernels), 6 (channel-quad with reuse by offset "
                           "pattern / fp32), 7 (channel-quad, 256-sample tiles, two CTAs per SM / fp32), 8 (channel-quad "
                           "pair rows / fp32), 9 (channel-quad without register reuse / fp32), 10 (channel-quad without the "
                           "per-byte path where a range has none / fp32), 11 (9 and 10) or 12 (11 with 32-bit shared "
                           "addresses)");
    a->popt.kernel_variant = variant;
    return true;
}

bool aa_b200_pipeline_run_all(void *obj)
{
    Api *a = as_api(obj);
    if (!a->pipe)
        return api_fail(a, "no DDTR plan bound");
    if (!a->pipe->run_all())
        return api_fail(a, a->pipe->last_error());
    if (a->options.output_dmt) {
        if (!a->pipe->synchronize())
            return api_fail(a, a->pipe->last_error());
        return export_outputs(a);
    }
    return true;
}

bool aa_b200_pipeline_setup(void *obj)
{
    Api *a = as_api(obj);
    if (!a->pipe)
        return api_fail(a, "no DDTR plan bound");
    return a->pipe->setup() ? true : api_fail(a, a->pipe->last_error());
}

bool aa_b200_pipeline_rewind(void *obj)
{
    Api *a = as_api(obj);
    a->exported = false;
    return a->pipe ? a->pipe->rewind() : api_fail(a, "no DDTR plan bound");
}

bool aa_b200_pipeline_set_candidate_output(void *obj, int write_files, const char *dir)
{
    Api *a = as_api(obj);
    a->write_candidates = write_files != 0;
    a->candidate_dir = dir ? dir : "";
    return true;
}

bool aa_b200_pipeline_set_analysis_batch(void *obj, long long max_time_samples)
{
    Api *a = as_api(obj);
    if (a->spd)
        return api_fail(a, "the analysis batch must be set before the first step");
    if (max_time_samples < 0)
        return api_fail(a, "max_time_samples must be >= 0");
    a->spd_max_ts = max_time_samples;
    return true;
}

bool aa_b200_pipeline_set_export_base(void *obj, const char *base)
{
    Api *a = as_api(obj);
    if (!base || !*base)
        return api_fail(a, "empty export base name");
    a->export_base = base;
    return true;
}

int aa_b200_export_dd_data(int range, float ***dedispersed_data, size_t max_nTimesamples, const int *ndms,
                           const int *inBin, const char *base_filename, const int *ranges_to_export, int DMs_per_file)
{
    std::string err;
    if (!dedispersed_data || !ndms || !inBin || !base_filename || !ranges_to_export) {
        set_error("aa_b200_export_dd_data: null argument");
        return 1;
    }
    if (!export_dd_data(range, dedispersed_data, max_nTimesamples, ndms, inBin, base_filename, ranges_to_export,
                        DMs_per_file, err)) {
        set_error(err);
        return 1;
    }
    return 0;
}

size_t aa_b200_sd_per_file_from_file_size(size_t size_in_MB, size_t primary_dimension, size_t floats_per_element)
{
    return sd_per_file_from_file_size(size_in_MB, primary_dimension, floats_per_element);
}

bool aa_b200_pipeline_synchronize(void *obj)
{
    Api *a = as_api(obj);
    if (!a->pipe)
        return api_fail(a, "no DDTR plan bound");
    if (!a->pipe->synchronize())
        return api_fail(a, a->pipe->last_error());
    return true;
}

float *aa_b200_pipeline_device_output(void *obj, int range)
{
    Api *a = as_api(obj);
    return a->pipe ? a->pipe->device_output(range) : nullptr;
}

int aa_b200_pipeline_range_info(void *obj, int range, int *kind, int *group_dms, int *span, int *tile_words)
{
    Api *a = as_api(obj);
    if (!a->pipe || !a->pipe->setup() || range < 0 || range >= static_cast<int>(a->pipe->strategy().nranges()))
        return 1;
    const RangeConfig &rc = a->pipe->range_config(range);
    *kind = rc.kind;
    *group_dms = rc.group_dms;
    *span = rc.span;
    *tile_words = rc.tile_words;
    if (rc.variant == 2) {
        *kind |= 0x100;
        *span = rc.quad_span;
        *tile_words = rc.quad.M / 4;
    } else if (rc.variant == 3) {
        *kind |= 0x200;
        *tile_words = 4;
    } else if (rc.variant == 5) {
        *kind |= 0x1000;
        *span = rc.quad_span;
        *tile_words = rc.quad.M / 4;
    } else if (rc.variant == 6) {
        *kind |= 0x2000;
        *span = rc.quad_span;
        *tile_words = rc.quad.M / 4;
    } else if (rc.variant == 4) {
        *kind |= 0x800;
        *span = rc.sub.W - 514;
        *tile_words = 4;
    } else if (rc.elem_bytes == 2) {
        *kind |= 0x400;
    }
    return 0;
}

long long aa_b200_tuned_ranges(int clear) { return static_cast<long long>(aab200::tuned_range_entries(clear != 0)); }

namespace {
thread_local std::string g_tuned_error;
} // namespace

long long aa_b200_tuned_ranges_save(const char *path)
{
    g_tuned_error.clear();
    if (!path) {
        g_tuned_error = "null path";
        return -1;
    }
    return aab200::tuned_ranges_save(path, g_tuned_error);
}

long long aa_b200_tuned_ranges_load(const char *path)
{
    g_tuned_error.clear();
    if (!path) {
        g_tuned_error = "null path";
        return -1;
    }
    return aab200::tuned_ranges_load(path, g_tuned_error);
}

const char *aa_b200_tuned_ranges_last_error(void) { return g_tuned_error.c_str(); }

long long aa_b200_tuned_ranges_used(void) { return aab200::tuned_range_uses(); }

int aa_b200_pipeline_stage_depth(void *obj, int range)
{
    Api *a = as_api(obj);
    if (!a->pipe || !a->pipe->setup() || range < 0 || range >= static_cast<int>(a->pipe->strategy().nranges()))
        return 0;
    const RangeConfig &rc = a->pipe->range_config(range);
    return (rc.variant == 2 || rc.variant == 5 || rc.variant == 6) ? rc.quad.qs
                                                                   : (rc.variant == 3 ? rc.f32.cs : (rc.variant == 4 ? 1 : 0));
}

int aa_b200_pipeline_range_kernel(void *obj, int range, int *flavour, int *tile_dms, int *tile_samples,
                                  int *dms_per_warp)
{
    Api *a = as_api(obj);
    if (!a->pipe || !a->pipe->setup() || range < 0 || range >= static_cast<int>(a->pipe->strategy().nranges()))
        return 1;
    const RangeConfig &rc = a->pipe->range_config(range);
    const bool quadlike = rc.variant == 2 || rc.variant == 5 || rc.variant == 6;
    *flavour = (rc.variant == 2) ? a->pipe->quad_flavour_of(rc) : -1;
    *tile_dms = rc.group_dms;
    *tile_samples = quadlike ? 32 * rc.quad.M : ((rc.variant == 3 || rc.variant == 4) ? 512 : 128 * rc.tile_words);
    // M = 8 with flavour 0 runs 8 warps of 8 DM trials; every other staged
    // channel-quad form 16 warps of 4
    *dms_per_warp = quadlike ? ((rc.quad.M == 8 && *flavour != 2) ? 8 : 4) : 0;
    return 0;
}

long long aa_b200_pipeline_kernel_launches(void *obj)
{
    Api *a = as_api(obj);
    return a->pipe ? a->pipe->kernel_launches() : 0;
}

const char *aa_b200_pipeline_last_error(void *obj)
{
    Api *a = as_api(obj);
    if (a->pipe && !a->pipe->last_error().empty())
        return a->pipe->last_error().c_str();
    return a->error.c_str();
}

int aa_b200_pipeline_num_tchunks(void *obj)
{
    Api *a = as_api(obj);
    return a->pipe ? a->pipe->strategy().num_tchunks() : 0;
}

bool aa_b200_pipeline_time_kernels(void *obj, int on)
{
    Api *a = as_api(obj);
    if (a->pipe)
        return a->pipe->set_time_kernels(on != 0);
    a->popt.time_kernels = on != 0;
    return true;
}

int aa_b200_pipeline_kernel_time(void *obj, int family, double *ms, long long *count)
{
    Api *a = as_api(obj);
    if (!a->pipe || family < 0 || family >= KF_COUNT)
        return 1;
    *ms = a->pipe->kernel_ms(family);
    *count = a->pipe->kernel_count(family);
    return 0;
}

bool aa_b200_pipeline_reset_kernel_times(void *obj)
{
    Api *a = as_api(obj);
    if (!a->pipe)
        return false;
    a->pipe->reset_kernel_times();
    return true;
}

int aa_b200_pipeline_maxshift(void *obj)
{
    Api *a = as_api(obj);
    return a->pipe ? a->pipe->strategy().maxshift() : 0;
}

} // extern "C"
