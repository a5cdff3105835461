// pipeline.cpp -- DDTR runner (see pipeline.hpp).
#include "pipeline.hpp"

#include <algorithm>
#include <cstdio>
#include <cstring>

#include "autotune.hpp"
#include "fault.hpp"
#include "preproc.cuh"
#include "ddtr_kernels.cuh"

namespace aab200 {

// Rows a stage of qs channel quads of the range needs.
static int rc_npool(const RangeConfig &rc, int qs)
{
    const int k = (qs == 1) ? 0 : (qs == 2) ? 1 : (qs == 4) ? 2 : (qs == 8) ? 3 : -1;
    return (k >= 0 && rc.quad_npool_qs[k] > 0) ? rc.quad_npool_qs[k] : qs * std::max(1, rc.quad_maxcnt);
}


namespace {
constexpr int kMaxSmemOptin = 227 * 1024;
}

DdtrPipeline::DdtrPipeline(const FilterbankMetadata &meta, const void *input, const PipelineOptions &opt)
    : meta_(meta), input_(static_cast<const uint8_t *>(input)), opt_(opt)
{
}

DdtrPipeline::~DdtrPipeline() { cleanup(); }

bool DdtrPipeline::fail(const std::string &msg)
{
    if (error_.empty())
        error_ = msg;
    return false;
}

bool DdtrPipeline::check_cuda(cudaError_t e, const char *what)
{
    if (e == cudaSuccess && !injected_failure_now())
        return true;
    return fail(std::string(what) + ": " + (e == cudaSuccess ? "injected failure" : cudaGetErrorString(e)));
}

bool DdtrPipeline::bind(const DdtrPlan &plan)
{
    // include/aa_pipeline_api.hpp:130-174: the strategy is computed on bind
    // with the device's free memory.
    bound_ = false;
    plan_ = plan;
    size_t free_mem = opt_.free_memory;
    if (free_mem == 0) {
        size_t fr = 0, tot = 0;
        if (!check_cuda(cudaMemGetInfo(&fr, &tot), "cudaMemGetInfo"))
            return false;
        free_mem = fr;
    }
    const StrategyStatus s = strategy_.compute(plan_, meta_, free_mem, opt_.enable_analysis);
    if (s != STRAT_OK) {
        char buf[160];
        std::snprintf(buf, sizeof(buf), "DDTR strategy refused the plan (code %d)", static_cast<int>(s));
        return fail(buf);
    }
    bound_ = true;
    return true;
}

bool DdtrPipeline::build_range(int r)
{
    RangeConfig &rc = ranges_[r];
    const DmRange &d = strategy_.dm(r);
    const int nchans = meta_.nchans;
    const int ndms = strategy_.ndms(r);
    const float tsamp_original = static_cast<float>(meta_.tsamp);
    rc.tsamp = tsamp_original * static_cast<float>(d.inBin); // :778
    rc.mstartdm = d.low / rc.tsamp;                           // src/aa_dedisperse.cpp:28,37-40
    rc.mdmstep = d.step / rc.tsamp;
    rc.kind = select_delay_kind(meta_.nbits, d.step, rc.tsamp, strategy_.dmshifts()[nchans - 1], opt_.failsafe);
    rc.elem_bytes = elem_bytes_;
    rc.nch_used = (rc.kind == KIND_SHARED4 && nchans > 4096) ? 4096 * (nchans / 4096) : nchans;

    const size_t nent = static_cast<size_t>(nchans) * ndms;
    if (!check_cuda(cudaMalloc(&rc.d_table, nent * sizeof(int32_t)), "cudaMalloc(delay table)"))
        return false;
    if (!check_cuda(launch_delay_table(d_dmshifts_, nchans, ndms, rc.kind, opt_.fma_mode, rc.mstartdm, rc.mdmstep,
                                       rc.d_table, d_err_, st_),
                    "delay table"))
        return false;
    ++launches_;

    const int nch_pad = (nchans + 3) & ~3;
    int *d_mx = nullptr;
    if (!check_cuda(cudaMalloc(&d_mx, 2 * sizeof(int)), "cudaMalloc"))
        return false;
    rc.tile_words = opt_.tile_words > 0 ? opt_.tile_words : 4;
    int cand[] = {64, 32, 16, 8, 4};
    bool ok = false;
    for (int gd : cand) {
        if (opt_.group_dms > 0 && gd != opt_.group_dms)
            continue;
        if (ndms % gd)
            continue;
        if (rc.d_wmin) {
            cudaFree(rc.d_wmin);
            rc.d_wmin = nullptr;
        }
        if (!check_cuda(cudaMalloc(&rc.d_wmin, static_cast<size_t>(ndms / gd) * nch_pad * sizeof(int32_t)),
                        "cudaMalloc(windows)"))
            break;
        int hm[2] = {0, 0};
        cudaMemsetAsync(d_mx, 0, 2 * sizeof(int), st_);
        if (!check_cuda(launch_group_windows(rc.d_table, nchans, ndms, gd, rc.d_wmin, d_mx, d_mx + 1, st_),
                        "group windows"))
            break;
        ++launches_;
        if (!check_cuda(cudaMemcpyAsync(hm, d_mx, 2 * sizeof(int), cudaMemcpyDeviceToHost, st_), "D2H") ||
            !check_cuda(cudaStreamSynchronize(st_), "sync"))
            break;
        rc.span = hm[0];
        rc.delay_max = hm[1];
        rc.group_dms = gd;
        if (elem_bytes_ == 2) {
            ok = true;
            break;
        }
        const size_t smem = ddtr_u8_smem_bytes(rc.span, gd, rc.tile_words, nchans);
        if (smem <= static_cast<size_t>(kMaxSmemOptin) && nchans <= 16384) {
            ok = true;
            break;
        }
    }
    cudaFree(d_mx);
    if (!ok)
        return fail(error_.empty() ? "no DM-group size fits the delay span of range " + std::to_string(r) : error_);
    if (!check_device_flags())
        return false;
    if (elem_bytes_ == 1 && (opt_.kernel_variant == 0 || opt_.kernel_variant == 3) && rc.group_dms == 64) {
        if (!build_sub_tables(r))
            return false;
    }
    if (elem_bytes_ == 1 &&
        (opt_.kernel_variant == 0 || opt_.kernel_variant == 2 || opt_.kernel_variant == 4 ||
         opt_.kernel_variant == 5 || opt_.kernel_variant == 6 || opt_.kernel_variant == 7 ||
         opt_.kernel_variant == 8 || opt_.kernel_variant == 9 || opt_.kernel_variant == 10 ||
         opt_.kernel_variant == 11 || opt_.kernel_variant == 12) &&
        rc.group_dms == 64) {
        if (!build_quad_tables(r))
            return false;
    }
    // both available (variant 0): the channel-quad kernel until the autotuner
    // has timed the two
    if (rc.has_quad)
        rc.variant = 2;
    else if (rc.has_sub)
        rc.variant = 4;
    if (elem_bytes_ == 1 && opt_.kernel_variant == 4) {
        if (!quad_ws_fits(rc))
            return fail("the warp-specialised channel-quad kernel cannot run range " + std::to_string(r) +
                        " (entries on the per-byte path, or its stage does not fit shared memory)");
        rc.variant = 5;
    }
    if (elem_bytes_ == 1 && opt_.kernel_variant == 5) {
        const int qs = quad_sp_depth(rc);
        if (qs == 0)
            return fail("the split-phase channel-quad kernel cannot run range " + std::to_string(r) +
                        " (entries on the per-byte path, or its stage does not fit shared memory)");
        rc.quad.npool = rc_npool(rc, qs);
        rc.quad.qs = qs;
        rc.variant = 6;
    }
    if (elem_bytes_ == 2 && opt_.kernel_variant != 1 && rc.group_dms == 64 && nchans <= 16384) {
        const F32Geometry G = f32_geometry(rc.span, rc.group_dms, nchans, 0);
        if (G.smem_bytes > 0) {
            rc.f32 = G.f;
            rc.variant = 3;
        } else if (opt_.kernel_variant == 2) {
            return fail("the staged fp32 kernel does not fit range " + std::to_string(r));
        }
    }
    if (elem_bytes_ == 1) {
        if (!check_cuda(cudaMalloc(&rc.d_offtab, nent * sizeof(int32_t)), "cudaMalloc(offset table)"))
            return false;
        if (!check_cuda(launch_offset_table(rc.d_table, rc.d_wmin, nchans, ndms, rc.group_dms,
                                            ddtr_u8_rw(rc.span, rc.tile_words), rc.span, rc.d_offtab, st_),
                        "offset table"))
            return false;
        ++launches_;
    }
    return true;
}

// Channel-quad tables: skew patterns per (quad, DM group), window starts and
// word offsets; chooses the channel-quad kernel when its stage fits shared memory.
bool DdtrPipeline::build_quad_tables(int r)
{
    RangeConfig &rc = ranges_[r];
    const int ndms = strategy_.ndms(r);
    const int nquads = (rc.nch_used + 3) / 4;
    const int nq_pad = (nquads + 3) & ~3;
    const int ngroups = ndms / rc.group_dms;
    int *d_stats = nullptr;
    int32_t *d_qtmp = nullptr;
    int hs[4] = {0, 0, 0, 0};
    const size_t nq_ent = static_cast<size_t>(nquads) * ndms;
    if (!check_cuda(cudaMalloc(&rc.d_qpat, static_cast<size_t>(ngroups) * nquads * 16 * sizeof(int32_t)), "cudaMalloc") ||
        !check_cuda(cudaMalloc(&rc.d_qwin, static_cast<size_t>(ngroups) * nq_pad * sizeof(int32_t)), "cudaMalloc") ||
        !check_cuda(cudaMemsetAsync(rc.d_qwin, 0, static_cast<size_t>(ngroups) * nq_pad * sizeof(int32_t), st_), "memset") ||
        !check_cuda(cudaMalloc(&rc.d_qoff, nq_ent * sizeof(int32_t)), "cudaMalloc") ||
        !check_cuda(cudaMalloc(&d_qtmp, nq_ent * sizeof(int32_t)), "cudaMalloc") ||
        !check_cuda(cudaMalloc(&d_stats, 4 * sizeof(int)), "cudaMalloc") ||
        !check_cuda(cudaMemsetAsync(d_stats, 0, 4 * sizeof(int), st_), "memset"))
        return false;
    bool ok = check_cuda(launch_quad_patterns(rc.d_table, rc.nch_used, ndms, rc.group_dms, nquads, nq_pad, rc.d_qpat,
                                              rc.d_qwin, d_qtmp, d_stats, st_),
                         "quad patterns") &&
              check_cuda(cudaMemcpyAsync(hs, d_stats, 4 * sizeof(int), cudaMemcpyDeviceToHost, st_), "D2H") &&
              check_cuda(cudaStreamSynchronize(st_), "sync");
    ++launches_;
    std::vector<int> counts(static_cast<size_t>(ngroups) * nquads);
    if (ok)
        // the pattern count (word 15) of every (group, quad)
        ok = check_cuda(cudaMemcpy2D(counts.data(), sizeof(int), rc.d_qpat + 15, 16 * sizeof(int32_t), sizeof(int),
                                     counts.size(), cudaMemcpyDeviceToHost),
                        "D2H");
    if (ok) {
        rc.quad_ws_ok = (hs[3] == 0);
        rc.quad_span = hs[0];
        rc.quad_dmax = hs[1];
        rc.quad_maxcnt = hs[2];
        rc.nquads = nquads;
        // rows a stage really needs: the largest sum of pattern counts over
        // the quads of a stage, for each stage depth
        for (int k = 0; k < 4; ++k) {
            const int qs_k = 1 << k;
            int most = 0;
            for (int g = 0; g < ngroups; ++g)
                for (int q0 = 0; q0 < nquads; q0 += qs_k) {
                    int tot = 0;
                    for (int q = q0; q < std::min(nquads, q0 + qs_k); ++q)
                        tot += counts[static_cast<size_t>(g) * nquads + q];
                    most = std::max(most, tot);
                }
            rc.quad_npool_qs[k] = std::max(1, most);
        }
        const int M = (opt_.tile_words == 2 || opt_.kernel_variant == 7) ? 8 : 16;
        const QuadGeometry G = quad_fit(rc, M);
        if (G.smem_bytes <= kStagedSmemLimit && rc.quad_dmax <= 255) {
            rc.quad = G;
            rc.variant = 2;
            rc.has_quad = true;
            const bool pairs = (opt_.kernel_variant == 8) && hs[3] == 0 && M == 16;
            rc.quad_pairs = pairs;
            ok = check_cuda(launch_quad_offsets(d_qtmp, nq_ent, G.W, rc.d_qoff, st_, pairs ? 1 : 0), "quad offsets");
            ++launches_;
            if (ok && opt_.autotune && !opt_.external_buffers && opt_.kernel_variant == 0 && opt_.tile_words == 0) {
                // the tile-shape autotuner rebuilds the offsets for other row pitches
                rc.d_qtmp = d_qtmp;
                d_qtmp = nullptr;
            }
        }
    }
    if (ok)
        ok = check_cuda(cudaStreamSynchronize(st_), "sync");
    cudaFree(d_qtmp);
    cudaFree(d_stats);
    if (!rc.has_quad) {
        cudaFree(rc.d_qpat);
        cudaFree(rc.d_qwin);
        cudaFree(rc.d_qoff);
        rc.d_qpat = rc.d_qwin = rc.d_qoff = nullptr;
        if (opt_.kernel_variant == 2)
            return fail("the channel-quad kernel does not fit range " + std::to_string(r));
    }
    return ok;
}

// The deepest stage (1, 2, 4 or 8 quads) whose shared memory fits, for a
// tile of 32 x M words.
QuadGeometry DdtrPipeline::quad_fit(const RangeConfig &rc, int M) const
{
    int qs = 8;
    QuadGeometry G = quad_geometry(rc.quad_span, rc.quad_dmax, rc.quad_maxcnt, rc.group_dms, rc.nquads, M, qs,
                                   rc_npool(rc, qs));
    while (G.smem_bytes > kStagedSmemLimit && qs > 1) {
        qs /= 2;
        G = quad_geometry(rc.quad_span, rc.quad_dmax, rc.quad_maxcnt, rc.group_dms, rc.nquads, M, qs,
                          rc_npool(rc, qs));
    }
    return G;
}

// Subband tables: skew patterns of every (16-channel subband, DM group),
// subband windows and offsets; the subband kernel runs the range when every
// (subband, DM trial) has an exact pattern and the stage fits shared memory.
bool DdtrPipeline::build_sub_tables(int r)
{
    RangeConfig &rc = ranges_[r];
    const int ndms = strategy_.ndms(r);
    const int nsub = (rc.nch_used + 15) / 16;
    const int nsub_pad = (nsub + 3) & ~3;
    const int ngroups = ndms / 64;
    int *d_stats = nullptr;
    int32_t *d_stmp = nullptr;
    int hs[6] = {0, 0, 0, 0, 0, 0};
    const size_t n_ent = static_cast<size_t>(nsub) * ndms;
    if (!check_cuda(cudaMalloc(&rc.d_sblk, static_cast<size_t>(ngroups) * nsub * SUB_BLK_WORDS * sizeof(int32_t)),
                    "cudaMalloc") ||
        !check_cuda(cudaMalloc(&rc.d_swin, static_cast<size_t>(ngroups) * nsub_pad * sizeof(int32_t)), "cudaMalloc") ||
        !check_cuda(cudaMemsetAsync(rc.d_swin, 0, static_cast<size_t>(ngroups) * nsub_pad * sizeof(int32_t), st_),
                    "memset") ||
        !check_cuda(cudaMalloc(&rc.d_soff, n_ent * sizeof(int32_t)), "cudaMalloc") ||
        !check_cuda(cudaMalloc(&d_stmp, n_ent * sizeof(int32_t)), "cudaMalloc") ||
        !check_cuda(cudaMalloc(&d_stats, 6 * sizeof(int)), "cudaMalloc") ||
        !check_cuda(cudaMemsetAsync(d_stats, 0, 6 * sizeof(int), st_), "memset"))
        return false;
    bool ok = check_cuda(launch_sub_patterns(rc.d_table, rc.nch_used, ndms, nsub, nsub_pad, rc.d_sblk, rc.d_swin,
                                             d_stmp, d_stats, st_),
                         "subband patterns") &&
              check_cuda(cudaMemcpyAsync(hs, d_stats, 6 * sizeof(int), cudaMemcpyDeviceToHost, st_), "D2H") &&
              check_cuda(cudaStreamSynchronize(st_), "sync");
    ++launches_;
    if (ok && hs[5] == 0 && hs[3] >= 1) {
        const SubGeometry G = sub_geometry(hs[0], hs[1], hs[2], hs[3], hs[4], nsub);
        if (G.smem_bytes <= kStagedSmemLimit) {
            rc.sub = G;
            rc.nsub = nsub;
            rc.variant = 4;
            rc.has_sub = true;
            ok = check_cuda(launch_sub_offsets(d_stmp, n_ent, G.W, rc.d_soff, st_), "subband offsets");
            ++launches_;
        }
    }
    if (ok)
        ok = check_cuda(cudaStreamSynchronize(st_), "sync");
    cudaFree(d_stmp);
    cudaFree(d_stats);
    if (!rc.has_sub) {
        cudaFree(rc.d_sblk);
        cudaFree(rc.d_swin);
        cudaFree(rc.d_soff);
        rc.d_sblk = rc.d_swin = rc.d_soff = nullptr;
        if (opt_.kernel_variant == 3)
            return fail("the subband kernel cannot run range " + std::to_string(r) +
                        " (patterns without an exact split, or its stage does not fit shared memory)");
    }
    return ok;
}

// The warp-specialised channel-quad kernel needs 512-sample tiles, a
// pre-skewed row for every (quad, DM trial) and its stage in shared memory.
bool DdtrPipeline::quad_ws_fits(const RangeConfig &rc) const
{
    if (!rc.has_quad || !rc.quad_ws_ok || rc.quad.M != 16)
        return false;
    QuadLaunch q{};
    q.qs = rc.quad.qs;
    q.raww = rc.quad.raww;
    q.nq_pad = rc.quad.nq_pad;
    q.npool = rc.quad.npool;
    q.W = rc.quad.W;
    return quadws_smem_bytes(q) <= kStagedSmemLimit;
}

// The split-phase channel-quad kernel needs the same (512-sample tiles, no
// per-byte entries) and its deeper rings in shared memory: the largest stage
// depth up to the range's whose rings fit, 0 if none does.
int DdtrPipeline::quad_sp_depth(const RangeConfig &rc) const
{
    if (!rc.has_quad || !rc.quad_ws_ok || rc.quad.M != 16)
        return 0;
    QuadLaunch q{};
    q.raww = rc.quad.raww;
    q.nq_pad = rc.quad.nq_pad;
    q.W = rc.quad.W;
    for (int qs = rc.quad.qs; qs >= 1; qs /= 2) {
        q.qs = qs;
        q.npool = rc_npool(rc, qs);
        if (quadsp_smem_bytes(q) <= kStagedSmemLimit)
            return qs;
    }
    return 0;
}

// Optional processing of the reference runner: the bandpass normalisation
// of zero DM (the plan's, else (2^nbits - 1)/2 per channel,
// src/aa_ddtr_strategy.cpp:48-60; with set_bandpass_average the block means
// of include/aa_permitted_pipelines_generic.hpp:533-552) and a writable
// unsigned-short chunk where the input is not one.
bool DdtrPipeline::setup_processing(long long L0)
{
    const int nchans = meta_.nchans;
    const bool pre_in = opt_.zero_dm || opt_.zero_dm_outliers || opt_.input_norm;
    if ((pre_in || opt_.old_rfi || opt_.output_norm) && opt_.external_buffers)
        return fail("input/output processing options are not available to the batch engine");
    if (!pre_in)
        return true;
    if (meta_.nbits != 4 && meta_.nbits != 8 && meta_.nbits != 16)
        return fail("zero DM and input normalisation need 4, 8 or 16-bit samples");
    if (plan_.bandpass().size() == static_cast<size_t>(nchans))
        bandpass_ = plan_.bandpass();
    else
        bandpass_.assign(nchans, static_cast<float>(((1 << meta_.nbits) - 1.0) / 2.0));
    if (opt_.bandpass_average && (opt_.zero_dm || opt_.zero_dm_outliers)) {
        // src/aa_host_cpu_msd.cpp:5-35 with (nchans, nsamples) over the [t][c]
        // input: value c is the mean of elements [c*nsamples, (c+1)*nsamples)
        if (opt_.device_input || opt_.packed_input)
            return fail("set_bandpass_average needs the unsigned-short input in host memory");
        const uint16_t *in = reinterpret_cast<const uint16_t *>(input_);
        const size_t ns = static_cast<size_t>(meta_.nsamples);
        for (int c = 0; c < nchans; ++c) {
            double sum = 0.0;
            size_t n = 0;
            for (size_t j = 0; j < ns; ++j) {
                sum += in[static_cast<size_t>(c) * ns + j];
                n += 1;
            }
            bandpass_[c] = static_cast<float>(sum / n);
        }
    }
    if (!check_cuda(cudaMalloc(&d_norm_, nchans * sizeof(float)), "cudaMalloc(bandpass)") ||
        !check_cuda(cudaMemcpyAsync(d_norm_, bandpass_.data(), nchans * sizeof(float), cudaMemcpyHostToDevice, st_),
                    "H2D bandpass") ||
        !check_cuda(cudaStreamSynchronize(st_), "sync"))
        return false;
    if ((opt_.device_input || opt_.packed_input) &&
        !check_cuda(cudaMalloc(&d_stage_, static_cast<size_t>(L0) * nchans * sizeof(uint16_t)), "cudaMalloc(stage)"))
        return false;
    return true;
}

bool DdtrPipeline::check_device_flags()
{
    if (!check_cuda(cudaMemcpyAsync(h_err_, d_err_, sizeof(int), cudaMemcpyDeviceToHost, st_), "D2H flags") ||
        !check_cuda(cudaStreamSynchronize(st_), "sync"))
        return false;
    const int f = *h_err_;
    if (f == 0)
        return true;
    std::string m = "device reported:";
    if (f & DERR_DELAY_RANGE)
        m += " delay outside [0, 2^24) or class step > 1;";
    if (f & DERR_INPUT_RANGE)
        m += " input sample above the bit depth's range;";
    if (f & DERR_WINDOW)
        m += " delay outside the staged window;";
    return fail(m);
}

bool DdtrPipeline::timed_launch_begin(int family)
{
    if (!opt_.time_kernels)
        return true;
    if (kev_used_ == kev_.size()) {
        // the pool only grows while a run is queued without a synchronize
        if (kev_.size() >= 4096 && !collect_kernel_times())
            return false;
        if (kev_used_ == kev_.size()) {
            TimedLaunch t;
            if (!check_cuda(cudaEventCreate(&t.start), "event") || !check_cuda(cudaEventCreate(&t.stop), "event"))
                return false;
            kev_.push_back(t);
        }
    }
    kev_[kev_used_].family = family;
    return check_cuda(cudaEventRecord(kev_[kev_used_].start, st_), "event");
}

bool DdtrPipeline::timed_launch_end()
{
    if (!opt_.time_kernels)
        return true;
    const bool ok = check_cuda(cudaEventRecord(kev_[kev_used_].stop, st_), "event");
    ++kev_used_;
    return ok;
}

bool DdtrPipeline::collect_kernel_times()
{
    if (kev_used_ == 0)
        return true;
    if (!check_cuda(cudaEventSynchronize(kev_[kev_used_ - 1].stop), "event sync"))
        return false;
    for (size_t i = 0; i < kev_used_; ++i) {
        float ms = 0.f;
        if (!check_cuda(cudaEventElapsedTime(&ms, kev_[i].start, kev_[i].stop), "event time"))
            return false;
        kernel_ms_[kev_[i].family] += ms;
        kernel_n_[kev_[i].family] += 1;
    }
    kev_used_ = 0;
    return true;
}

void DdtrPipeline::reset_kernel_times()
{
    collect_kernel_times();
    for (int f = 0; f < KF_COUNT; ++f) {
        kernel_ms_[f] = 0.0;
        kernel_n_[f] = 0;
    }
}

bool DdtrPipeline::setup()
{
    if (setup_done_)
        return true;
    if (!bound_)
        return fail("no DDTR plan bound");
    const int nchans = meta_.nchans;
    const int nr = static_cast<int>(strategy_.nranges());
    if (meta_.nbits != 1 && meta_.nbits != 2 && meta_.nbits != 4 && meta_.nbits != 8 && meta_.nbits != 16 &&
        meta_.nbits != 32)
        return fail("unsupported nbits");
    elem_bytes_ = (meta_.nbits <= 8) ? 1 : 2;
    in_rec_bytes_ = 2LL * nchans;
    if (opt_.packed_input) {
        if ((static_cast<long long>(nchans) * meta_.nbits) % 8)
            return fail("packed input needs nchans * nbits to be a multiple of 8");
        in_rec_bytes_ = (meta_.nbits >= 16) ? 2LL * nchans : static_cast<long long>(nchans) * meta_.nbits / 8;
        if (meta_.nbits >= 16 && (reinterpret_cast<uintptr_t>(input_) & 1))
            return fail("16-bit packed input must be 2-byte aligned");
    }
    if (!check_cuda(cudaGetDevice(&device_), "cudaGetDevice"))
        return false;
    for (int r = 0; r < nr; ++r) {
        const int b = strategy_.dm(r).inBin;
        if (b < 1 || (b & (b - 1)))
            return fail("inBin must be a power of two");
    }
    if (opt_.stride_mode == STRIDE_REFERENCE && strategy_.dm(0).inBin > 1)
        return fail("the first DM range must have inBin 1 (the reference runner reads t_processed[-1] otherwise)");
    for (float v : strategy_.dmshifts())
        if (!(v >= 0.f))
            return fail("negative dispersion delays (foff > 0) are not supported");

    if (opt_.stream) {
        st_ = opt_.stream;
    } else {
        if (!check_cuda(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking), "stream"))
            return false;
        own_stream_ = true;
    }
    if (!check_cuda(cudaStreamCreateWithFlags(&st_h2d_, cudaStreamNonBlocking), "stream") ||
        !check_cuda(cudaStreamCreateWithFlags(&st_d2h_, cudaStreamNonBlocking), "stream"))
        return false;
    for (int i = 0; i < 2; ++i) {
        if (!check_cuda(cudaEventCreateWithFlags(&ev_tile_free_[i], cudaEventDisableTiming), "event") ||
            !check_cuda(cudaEventCreateWithFlags(&ev_tile_done_[i], cudaEventDisableTiming), "event") ||
            !check_cuda(cudaEventCreateWithFlags(&ev_raw_ready_[i], cudaEventDisableTiming), "event") ||
            !check_cuda(cudaEventCreateWithFlags(&ev_raw_free_[i], cudaEventDisableTiming), "event"))
            return false;
    }
    if (!check_cuda(cudaMalloc(&d_err_, sizeof(int)), "cudaMalloc") ||
        !check_cuda(cudaMemsetAsync(d_err_, 0, sizeof(int), st_), "memset") ||
        !check_cuda(cudaMallocHost(&h_err_, sizeof(int)), "cudaMallocHost"))
        return false;
    if (!check_cuda(cudaMalloc(&d_dmshifts_, sizeof(float) * nchans), "cudaMalloc") ||
        !check_cuda(cudaMemcpyAsync(d_dmshifts_, strategy_.dmshifts().data(), sizeof(float) * nchans,
                                    cudaMemcpyHostToDevice, st_),
                    "H2D dmshifts"))
        return false;

    ranges_.assign(nr, RangeConfig());
    int span_max = 0, delay_max = 0, rawb_max = 0;
    for (int r = 0; r < nr; ++r) {
        if (!build_range(r))
            return false;
        span_max = std::max(span_max, ranges_[r].span);
        delay_max = std::max(delay_max, ranges_[r].delay_max);
        rawb_max = std::max(rawb_max, 4 * ddtr_u8_rw(ranges_[r].span, ranges_[r].tile_words) + 32);
        rawb_max = std::max(rawb_max, 4 * ranges_[r].quad.raww + 64);
        rawb_max = std::max(rawb_max, ranges_[r].f32.rawh + 16);
        rawb_max = std::max(rawb_max, 4 * ranges_[r].sub.raww + 64);
    }

    const long long L0 = static_cast<long long>(strategy_.t_processed()[0][0]) + strategy_.maxshift();
    const long long pad = 4LL * (512 + span_max + delay_max) + rawb_max + 65536;
    pad_elems_ = static_cast<size_t>(pad);
    flat_elems_ = static_cast<size_t>(nchans) * static_cast<size_t>(L0) + static_cast<size_t>(pad);
    if (!enumerate_ops())
        return false;
    if (opt_.external_buffers && (opt_.copy_to_host || !opt_.device_output || !opt_.device_input))
        return fail("a pipeline run by a batch engine keeps its input and output on the device");
    for (int i = 0; i < 2 && !opt_.external_buffers; ++i) {
        if (!check_cuda(cudaMalloc(&d_flat_[i], flat_elems_ * elem_bytes_), "cudaMalloc(filterbank)") ||
            !check_cuda(cudaMemsetAsync(d_flat_[i], 0, flat_elems_ * elem_bytes_, st_), "memset"))
            return false;
    }
    if (!opt_.device_input) {
        for (int i = 0; i < 2; ++i)
            if (!check_cuda(cudaMalloc(&d_raw_[i], static_cast<size_t>(L0) * static_cast<size_t>(in_rec_bytes_)),
                            "cudaMalloc(raw chunk)"))
                return false;
    }
    if (!setup_processing(L0))
        return false;

    // outputs
    if (opt_.device_output) {
        d_out_full_.assign(nr, nullptr);
        for (int r = 0; r < nr; ++r) {
            const size_t n = static_cast<size_t>(strategy_.ndms(r)) * static_cast<size_t>(strategy_.total_samps(r));
            if (!check_cuda(cudaMalloc(&d_out_full_[r], std::max<size_t>(n, 1) * sizeof(float)),
                            "cudaMalloc(output)"))
                return false;
        }
    } else {
        tile_elems_ = 1;
        for (int r = 0; r < nr; ++r)
            for (int k = 0; k < strategy_.num_tchunks(); ++k)
                tile_elems_ = std::max(tile_elems_, static_cast<size_t>(strategy_.ndms(r)) *
                                                        static_cast<size_t>(strategy_.t_processed()[r][k]));
        for (int i = 0; i < 2; ++i)
            if (!check_cuda(cudaMalloc(&d_tile_[i], tile_elems_ * sizeof(float)), "cudaMalloc(output tile)"))
                return false;
    }
    if (opt_.copy_to_host) {
        // include/aa_permitted_pipelines_generic.hpp:418-445: float***
        // [range][dm][sum_k t_processed]; here all rows live in one pinned block.
        size_t total = 0;
        for (int r = 0; r < nr; ++r)
            total += static_cast<size_t>(strategy_.ndms(r)) * static_cast<size_t>(strategy_.total_samps(r));
        if (!check_cuda(cudaMallocHost(&h_block_, std::max<size_t>(total, 1) * sizeof(float)),
                        "cudaMallocHost(output)"))
            return false;
        host_row_ptrs_.assign(nr, std::vector<float *>());
        host_rows_.assign(nr, nullptr);
        size_t off = 0;
        for (int r = 0; r < nr; ++r) {
            const size_t tot = static_cast<size_t>(strategy_.total_samps(r));
            host_row_ptrs_[r].resize(strategy_.ndms(r));
            for (int dm = 0; dm < strategy_.ndms(r); ++dm)
                host_row_ptrs_[r][dm] = h_block_ + off + static_cast<size_t>(dm) * tot;
            host_rows_[r] = host_row_ptrs_[r].data();
            off += tot * static_cast<size_t>(strategy_.ndms(r));
        }
    }
    for (int i = 0; i < 2; ++i) {
        cudaEventRecord(ev_tile_free_[i], st_d2h_);
        cudaEventRecord(ev_raw_free_[i], st_);
    }
    if (opt_.autotune && !opt_.external_buffers && !tune_ranges())
        return false;
    if (!check_device_flags())
        return false;
    setup_done_ = true;
    rewind();
    return true;
}

// Key of a range's tuned choices: every input of the slice timings -- the
// device, the channel delays, the range and its DM trials, the summary of its
// delay and pattern tables, the geometry before tuning, chunk 0's length, the
// row pitch and the kernel options.
std::vector<long long> DdtrPipeline::tune_key(int r, const DdtrOp &op, long long pitch) const
{
    const RangeConfig &rc = ranges_[r];
    const DmRange &d = strategy_.dm(r);
    auto fb = [](float v) {
        uint32_t u;
        std::memcpy(&u, &v, sizeof u);
        return static_cast<long long>(u);
    };
    auto db = [](double v) {
        long long u;
        std::memcpy(&u, &v, sizeof u);
        return u;
    };
    std::vector<long long> k = {device_, meta_.nchans, meta_.nbits, db(meta_.tsamp), db(meta_.fch1),
                                db(meta_.foff), fb(d.low), fb(d.high), fb(d.step), d.inBin, strategy_.ndms(r),
                                op.tp, op.i_nsamp, pitch, opt_.kernel_variant, opt_.tile_words, opt_.fma_mode,
                                opt_.device_output ? 1 : 0, rc.kind, rc.elem_bytes, rc.group_dms, rc.tile_words,
                                rc.span, rc.delay_max, rc.nch_used, fb(rc.mstartdm), fb(rc.mdmstep), fb(rc.tsamp),
                                rc.variant, rc.quad.M, rc.quad.W, rc.quad.raww, rc.quad.qs, rc.quad.npool,
                                rc.quad.nq_pad, rc.quad_span, rc.quad_dmax, rc.quad_maxcnt, rc.nquads,
                                rc.has_sub ? 1 : 0, rc.has_quad ? 1 : 0, rc.quad_ws_ok ? 1 : 0,
                                rc.quad_pairs ? 1 : 0, rc.quad_flavour, rc.d_qtmp ? 1 : 0, rc.f32.cs, rc.f32.W,
                                rc.f32.rawh, rc.sub.W, rc.sub.wq, rc.sub.raww, rc.sub.npat, rc.sub.nqrow,
                                rc.nsub};
    for (int j = 0; j < 4; ++j)
        k.push_back(rc.quad_npool_qs[j]);
    for (float v : strategy_.dmshifts())
        k.push_back(fb(v));
    return k;
}

// A kept choice is taken only if it is one this range could have been given
// here: a kernel whose tables the range has, and a channel-quad geometry
// equal to the one set-up derives for its tile shape and stage depth (row
// pitch, raw row, row pool sized by the range's own pattern counts) that
// fits shared memory.  A choice read from a file that fails this (another
// build, an edited file) is timed again instead.
bool DdtrPipeline::tuned_valid(const RangeConfig &rc, const TunedRange &t) const
{
    if (t.variant == 4)
        return rc.has_sub && elem_bytes_ == 1;
    if (t.variant == 3)
        return elem_bytes_ == 2 && (t.f32_cs == 4 || t.f32_cs == 8 || t.f32_cs == 16 || t.f32_cs == 32);
    if (t.variant != 2 && t.variant != 5 && t.variant != 6)
        return false;
    const QuadGeometry &q = t.quad;
    if (!rc.has_quad || elem_bytes_ != 1 || (q.M != 8 && q.M != 16) ||
        (q.qs != 1 && q.qs != 2 && q.qs != 4 && q.qs != 8) || q.npool != rc_npool(rc, q.qs))
        return false;
    const QuadGeometry G = quad_geometry(rc.quad_span, rc.quad_dmax, rc.quad_maxcnt, rc.group_dms, rc.nquads, q.M,
                                         q.qs, q.npool);
    if (q.W != G.W || q.raww != G.raww || q.nq_pad != G.nq_pad)
        return false;
    QuadLaunch ql{};
    ql.raww = q.raww;
    ql.nq_pad = q.nq_pad;
    ql.W = q.W;
    ql.qs = q.qs;
    ql.npool = q.npool;
    // the stage-depth tuner's own bound (the per-CTA opt-in limit)
    const size_t limit = 227 * 1024;
    if (t.variant == 6)
        return q.M == 16 && rc.quad_ws_ok && quadsp_smem_bytes(ql) <= limit;
    if (t.variant == 5)
        return q.M == 16 && rc.quad_ws_ok && quadws_smem_bytes(ql) <= limit;
    const int f = t.quad_flavour;
    const bool flavour_ok = (f == -1) || (f == 0) || (f == 2 && q.M == 8) || ((f == 1 || f == 4) && q.M == 16) ||
                            ((f == 5 || f == 6 || f == 7) && q.M == 16 && rc.quad_ws_ok);
    return flavour_ok && G.smem_bytes <= limit;
}

// Stage depth of every range that runs a staged kernel, timed on chunk 0's
// job (the buffers hold zeros at this point; the kernels' work does not
// depend on the sample values).  A range whose key was tuned before in this
// process takes the kept choices instead.
bool DdtrPipeline::tune_ranges()
{
    StageTuneCache cache;
    for (size_t r = 0; r < ranges_.size(); ++r) {
        RangeConfig &rc = ranges_[r];
        if (rc.variant != 2 && rc.variant != 3 && rc.variant != 5 && rc.variant != 6)
            continue;
        const DdtrOp *op = nullptr;
        for (const DdtrOp &o : ops_)
            if (o.kind == DdtrOp::DDTR && o.range == static_cast<int>(r)) {
                op = &o;
                break;
            }
        if (!op)
            continue;
        float *out = opt_.device_output ? d_out_full_[r] + op->out_off : d_tile_[0];
        const long long pitch = opt_.device_output ? strategy_.total_samps(static_cast<int>(r)) : op->tp;
        const std::vector<long long> key = tune_key(static_cast<int>(r), *op, pitch);
        TunedRange kept;
        if (tuned_range_find(key, kept) && tuned_valid(rc, kept)) {
            if (rc.d_qtmp) {
                // the offset table for the kept tile's row pitch
                if (kept.quad.W != rc.quad.W) {
                    const size_t nq_ent = static_cast<size_t>(rc.nquads) * strategy_.ndms(r);
                    if (!check_cuda(launch_quad_offsets(rc.d_qtmp, nq_ent, kept.quad.W, rc.d_qoff, st_, 0),
                                    "quad offsets") ||
                        !check_cuda(cudaStreamSynchronize(st_), "sync"))
                        return false;
                    ++launches_;
                }
                cudaFree(rc.d_qtmp);
                rc.d_qtmp = nullptr;
            }
            rc.variant = kept.variant;
            rc.quad = kept.quad;
            rc.quad_flavour = kept.quad_flavour;
            rc.f32.cs = kept.f32_cs;
            tuned_range_note_use();
            continue;
        }
        DdtrJob job;
        if (!make_job(*op, d_flat_[op->src_level & 1], flat_elems_, out, pitch, job))
            return false;
        std::string err;
        if (!tune_stage_depth(job, st_, device_, cache, err))
            return fail(err);
        if (rc.variant == 2 || rc.variant == 5 || rc.variant == 6) {
            rc.quad.qs = job.q.qs;
            rc.quad.npool = job.q.npool;
        } else {
            rc.f32.cs = job.f.cs;
        }
        if (rc.variant == 2 && rc.d_qtmp && !tune_quad_shape(static_cast<int>(r), *op, out, pitch, cache, job))
            return false;
        if (rc.variant == 2 && opt_.kernel_variant == 0 && quad_sp_depth(rc) > 0) {
            // the split-phase kernel (its own stage depth) against the tuned
            // channel-quad kernel
            const float t_quad = time_job_slice(job, st_, device_, err);
            if (t_quad < 0.f)
                return fail(err);
            const QuadGeometry keep = rc.quad;
            const int qs = quad_sp_depth(rc);
            rc.quad.npool = rc_npool(rc, qs);
            rc.quad.qs = qs;
            rc.variant = 6;
            DdtrJob jsp;
            bool made = make_job(*op, d_flat_[op->src_level & 1], flat_elems_, out, pitch, jsp);
            if (made && !tune_stage_depth(jsp, st_, device_, cache, err))
                return fail(err);
            const float t_sp = made ? time_job_slice(jsp, st_, device_, err) : -1.f;
            if (made && t_sp < 0.f)
                return fail(err);
            if (made && t_sp < t_quad) {
                rc.quad.qs = jsp.q.qs;
                rc.quad.npool = jsp.q.npool;
            } else {
                rc.variant = 2;
                rc.quad = keep;
            }
        }
        if (rc.variant == 2 && rc.has_sub) {
            // the subband kernel against the tuned channel-quad kernel
            const float t_quad = time_job_slice(job, st_, device_, err);
            if (t_quad < 0.f)
                return fail(err);
            rc.variant = 4;
            DdtrJob js;
            const bool made = make_job(*op, d_flat_[op->src_level & 1], flat_elems_, out, pitch, js);
            rc.variant = 2;
            if (!made)
                return false;
            const float t_sub = time_job_slice(js, st_, device_, err);
            if (t_sub < 0.f)
                return fail(err);
            if (t_sub < t_quad)
                rc.variant = 4;
        }
        TunedRange t;
        t.variant = rc.variant;
        t.quad = rc.quad;
        t.quad_flavour = rc.quad_flavour;
        t.f32_cs = rc.f32.cs;
        tuned_range_keep(key, t);
    }
    return check_cuda(cudaStreamSynchronize(st_), "sync");
}

// Tile shape and flavour of a channel-quad range, after its stage depth:
// 32 x M words of output per CTA row (M = 16: 16 warps of 4 DM trials, one
// CTA per SM; M = 8: 8 warps of 8 DM trials, two CTAs per SM, or 16 warps of
// 4 with the byte-path switch) and the sum-loop flavours that can run the
// range.  Each candidate is timed on the slice at its own tuned stage depth;
// the fastest is kept and the offset table rebuilt for its row pitch.  job
// returns as the chosen candidate's job.
bool DdtrPipeline::tune_quad_shape(int r, const DdtrOp &op, float *out, long long pitch, StageTuneCache &cache,
                                   DdtrJob &job)
{
    RangeConfig &rc = ranges_[r];
    struct Cand {
        int M, flavour;
    };
    // flavours 5..7 flag per-byte entries as errors: ranges without them only
    const std::vector<Cand> cands = rc.quad_ws_ok ? std::vector<Cand>{{16, 7}, {16, 6}, {16, 0}, {8, 0}, {8, 2}}
                                                  : std::vector<Cand>{{16, 0}, {16, 4}, {16, 1}, {8, 0}, {8, 2}};
    const size_t nq_ent = static_cast<size_t>(rc.nquads) * strategy_.ndms(r);
    // the same output samples for every shape: four 512-sample tiles per SM
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device_);
    const int groups = std::max(1, strategy_.ndms(r) / rc.group_dms);
    const long long samples = 512LL * std::max(1, (4 * nsm + groups - 1) / groups);
    int built_M = rc.quad.M;
    float best_ms = 1e30f; // per output sample of the slice
    QuadGeometry best_G = rc.quad;
    int best_f = quad_flavour_of(rc);
    std::string err;
    for (const Cand &c : cands) {
        QuadGeometry G = quad_fit(rc, c.M);
        if (G.smem_bytes > kStagedSmemLimit)
            continue;
        if (c.M != built_M) {
            if (!check_cuda(launch_quad_offsets(rc.d_qtmp, nq_ent, G.W, rc.d_qoff, st_, 0), "quad offsets"))
                return false;
            ++launches_;
            built_M = c.M;
        }
        rc.quad = G;
        rc.quad_flavour = c.flavour;
        DdtrJob t;
        if (!make_job(op, d_flat_[op.src_level & 1], flat_elems_, out, pitch, t))
            return false;
        if (!tune_stage_depth(t, st_, device_, cache, err))
            return fail(err);
        long long timed = 0;
        const float t_ms = time_job_slice(t, st_, device_, err, samples, &timed);
        if (t_ms < 0.f)
            return fail(err);
        const float ms = t_ms / static_cast<float>(std::max(1LL, timed));
        if (ms < best_ms) {
            best_ms = ms;
            best_G = G;
            best_G.qs = t.q.qs;
            best_G.npool = t.q.npool;
            best_f = c.flavour;
        }
    }
    if (best_G.M != built_M) {
        if (!check_cuda(launch_quad_offsets(rc.d_qtmp, nq_ent, best_G.W, rc.d_qoff, st_, 0), "quad offsets"))
            return false;
        ++launches_;
    }
    rc.quad = best_G;
    rc.quad_flavour = best_f;
    if (!check_cuda(cudaStreamSynchronize(st_), "sync"))
        return false;
    cudaFree(rc.d_qtmp);
    rc.d_qtmp = nullptr;
    return make_job(op, d_flat_[op.src_level & 1], flat_elems_, out, pitch, job);
}

bool DdtrPipeline::rewind()
{
    op_cursor_ = 0;
    cur_chunk_ = 0;
    cur_range_ = 0;
    inc_ = 0;
    finished_component_sent_ = false;
    last_plane_ = StepPlane{};
    return true;
}

// The runner's loop as a list: per chunk the load and corner turn (:741),
// then per range a single x2 binning whenever inBin grows (:797-808) with the
// length the runner passes, and the dedispersion with row stride
// t_processed + maxshift/inBin (:782-786); output rows at inc/inBin
// (src/aa_device_save_data.cu:41).  STRIDE_TRUE bins on the true row stride
// as many times as inBin needs.
bool DdtrPipeline::enumerate_ops()
{
    ops_.clear();
    const int nr = static_cast<int>(strategy_.nranges());
    const auto &T = strategy_.t_processed();
    long long inc = 0;
    for (int k = 0; k < strategy_.num_tchunks(); ++k) {
        const long long L = static_cast<long long>(T[0][k]) + strategy_.maxshift();
        if (inc + L > meta_.nsamples)
            return fail("chunk extends past the end of the input");
        DdtrOp ct;
        ct.kind = DdtrOp::CORNER_TURN;
        ct.chunk = k;
        ct.len = L;
        ct.inc = inc;
        ops_.push_back(ct);
        int level = 0, old_bin = 1, cur_bin = 1;
        long long cur_stride = L;
        for (int r = 0; r < nr; ++r) {
            const DmRange &d = strategy_.dm(r);
            const int tp = T[r][k];
            const int ms_r = strategy_.maxshift() / d.inBin; // :782
            auto bin_once = [&](long long nsb) -> bool {
                if (nsb <= 0 || (nsb & 1))
                    return fail("binning length must be positive and even");
                DdtrOp b;
                b.kind = DdtrOp::BIN;
                b.chunk = k;
                b.range = r;
                b.src_level = level;
                b.dst_level = level + 1;
                b.len = nsb;
                b.inc = inc;
                ops_.push_back(b);
                ++level;
                return true;
            };
            long long i_nsamp;
            if (opt_.stride_mode == STRIDE_REFERENCE) {
                if (d.inBin > old_bin &&
                    !bin_once(static_cast<long long>(T[r - 1][k]) + static_cast<long long>(ms_r) * d.inBin)) // :797-798
                    return false;
                i_nsamp = static_cast<long long>(tp) + ms_r; // :786
            } else {
                while (cur_bin < d.inBin) {
                    if (!bin_once(cur_stride))
                        return false;
                    cur_stride /= 2;
                    cur_bin *= 2;
                }
                i_nsamp = cur_stride;
            }
            DdtrOp dd;
            dd.kind = DdtrOp::DDTR;
            dd.chunk = k;
            dd.range = r;
            dd.src_level = level;
            dd.i_nsamp = i_nsamp;
            dd.tp = tp;
            dd.inc = inc;
            dd.out_off = inc / d.inBin;
            ops_.push_back(dd);
            old_bin = d.inBin;
        }
        inc += T[0][k]; // :898
    }
    return true;
}

// The autotuner's choice where it made one; else, on a range without
// per-byte entries, one load per DM trial and no per-byte path in the sum
// loop (flavour 7), and with per-byte entries the kernel that has that path
// (flavour 0); kernel_variant 6..12 force the measured alternatives.
int DdtrPipeline::quad_flavour_of(const RangeConfig &rc) const
{
    if (rc.quad_pairs)
        return 3;
    if (rc.quad_flavour >= 0)
        return rc.quad_flavour;
    const int M = rc.quad.M;
    const bool plain = opt_.kernel_variant == 0 || opt_.kernel_variant == 2 || opt_.kernel_variant == 12;
    return (opt_.kernel_variant == 10 && M == 16 && rc.quad_ws_ok)   ? 5
           : (opt_.kernel_variant == 11 && M == 16 && rc.quad_ws_ok) ? 6
           : (plain && M == 16 && rc.quad_ws_ok)                     ? 7
           : (opt_.kernel_variant == 9 && M == 16)                   ? 4
           : (opt_.kernel_variant == 6 && M == 16)                   ? 1
           : (opt_.kernel_variant == 7 && M == 8)                    ? 2
                                                                     : 0;
}

bool DdtrPipeline::make_job(const DdtrOp &op, const void *in, size_t in_elems, float *out, long long out_pitch,
                            DdtrJob &job, int as_variant)
{
    const int r = op.range;
    const RangeConfig &rc = ranges_[r];
    const DmRange &d = strategy_.dm(r);
    const int tp = op.tp;
    const long long i_nsamp = op.i_nsamp;
    int v = rc.variant;
    if (as_variant != 0) {
        if (!((as_variant == 4 && rc.has_sub) || (as_variant == 2 && rc.has_quad)))
            return fail("range " + std::to_string(r) + " has no tables for kernel variant " + std::to_string(as_variant));
        v = as_variant;
    }
    job = DdtrJob();
    job.variant = (elem_bytes_ == 1 && v == 2)   ? 2
                  : (elem_bytes_ == 2 && v == 3) ? 3
                  : (elem_bytes_ == 1 && v == 4) ? 4
                  : (elem_bytes_ == 1 && v == 5) ? 5
                  : (elem_bytes_ == 1 && v == 6) ? 6
                                                 : 1;
    job.elem_bytes = elem_bytes_;
    job.tile_words = rc.tile_words;
    job.offtab = rc.d_offtab;
    const int tile = (job.variant == 2 || job.variant == 5 || job.variant == 6)
                         ? 32 * rc.quad.M
                         : ((job.variant == 3 || job.variant == 4) ? 512 : 128 * rc.tile_words);
    const long long ntiles = (tp + tile - 1) / tile;
    long long need;
    if (elem_bytes_ == 1 && (job.variant == 2 || job.variant == 5 || job.variant == 6))
        need = static_cast<long long>(rc.nch_used - 1) * i_nsamp + ntiles * tile + rc.delay_max + 4LL * rc.quad.raww + 64;
    else if (job.variant == 4)
        need = static_cast<long long>(rc.nch_used - 1) * i_nsamp + ntiles * tile + rc.delay_max + 4LL * rc.sub.raww + 64;
    else if (elem_bytes_ == 1)
        need = static_cast<long long>(rc.nch_used - 1) * i_nsamp + ntiles * tile + rc.delay_max +
               4LL * ddtr_u8_rw(rc.span, rc.tile_words) + 64;
    else if (job.variant == 3)
        need = static_cast<long long>(rc.nch_used - 1) * i_nsamp + ntiles * tile + rc.delay_max + rc.f32.rawh + 8;
    else
        need = static_cast<long long>(rc.nch_used - 1) * i_nsamp + tp + rc.delay_max + 2;
    if (need > static_cast<long long>(in_elems))
        return fail("dedispersion window exceeds the filterbank buffer");

    DdtrLaunch &p = job.p;
    p.in = in;
    p.stride = i_nsamp;
    p.nchans = meta_.nchans;
    p.nch_used = rc.nch_used;
    p.tp = tp;
    p.ndms = strategy_.ndms(r);
    p.table = rc.d_table;
    p.wmin = rc.d_wmin;
    p.group_dms = rc.group_dms;
    p.span = rc.span;
    p.kind = rc.kind;
    p.nchans_f = static_cast<float>(meta_.nchans);
    p.bin_f = static_cast<float>(d.inBin);
    p.divide_by_bin = (rc.kind == KIND_SHARED4) ? 0 : 1;
    p.out = out;
    p.out_pitch = out_pitch;
    p.err = d_err_;
    if (job.variant == 1 && elem_bytes_ == 1 &&
        ((reinterpret_cast<uintptr_t>(p.out) & 15) || (p.out_pitch & 3) || (tp & 3)))
        return fail("output rows are not 16-byte aligned");
    if (job.variant == 2 || job.variant == 5 || job.variant == 6) {
        QuadLaunch &q = job.q;
        q.qpat = rc.d_qpat;
        q.qwin = rc.d_qwin;
        q.qoff = rc.d_qoff;
        q.nquads = rc.nquads;
        q.nq_pad = rc.quad.nq_pad;
        q.W = rc.quad.W;
        q.raww = rc.quad.raww;
        q.qs = rc.quad.qs;
        q.npool = rc.quad.npool;
        q.M = rc.quad.M;
        q.maxpat = rc.quad_maxcnt;
        for (int k = 0; k < 4; ++k)
            q.npool_qs[k] = rc.quad_npool_qs[k];
        // the default on a range without per-byte entries: one load per DM
        // trial and no per-byte path in the sum loop (flavour 7); with
        // per-byte entries the kernel that has that path (flavour 0)
        q.flavour = quad_flavour_of(rc);
    } else if (job.variant == 3) {
        job.f = rc.f32;
    } else if (job.variant == 4) {
        SubLaunch &s = job.s;
        s.sblk = rc.d_sblk;
        s.swin = rc.d_swin;
        s.soff = rc.d_soff;
        s.nsub = rc.nsub;
        s.nsub_pad = rc.sub.nsub_pad;
        s.W = rc.sub.W;
        s.wq = rc.sub.wq;
        s.raww = rc.sub.raww;
        s.npat = rc.sub.npat;
        s.nqrow = rc.sub.nqrow;
    }
    job.groups = p.ndms / p.group_dms;
    job.tiles = ntiles;
    job.tile_samples = tile;
    return true;
}

cudaError_t launch_job(const DdtrJob &job, cudaStream_t st)
{
    if (job.variant == 2)
        return launch_ddtr_quad(job.p, job.q, st);
    if (job.variant == 3)
        return launch_ddtr_f32(job.p, job.f, st);
    if (job.variant == 4)
        return launch_ddtr_sub(job.p, job.s, st);
    if (job.variant == 5)
        return launch_ddtr_quadws(job.p, job.q, st);
    if (job.variant == 6)
        return launch_ddtr_quadsp(job.p, job.q, st);
    return (job.elem_bytes == 1) ? launch_ddtr_u8(job.p, job.offtab, job.tile_words, st) : launch_ddtr_u16(job.p, st);
}

bool DdtrPipeline::exec_corner_turn(const DdtrOp &op)
{
    const int nchans = meta_.nchans;
    const int k = op.chunk;
    const long long L = op.len;
    if (static_cast<size_t>(nchans) * static_cast<size_t>(L) > flat_elems_)
        return fail("chunk larger than the filterbank buffer");
    const uint8_t *src;
    const int slot = k & 1;
    if (opt_.device_input) {
        src = input_ + static_cast<size_t>(op.inc) * static_cast<size_t>(in_rec_bytes_);
    } else {
        // issue this chunk's copy if it was not prefetched, and prefetch the next
        auto issue = [&](int kk, long long inc_kk) -> bool {
            const long long Lk = static_cast<long long>(strategy_.t_processed()[0][kk]) + strategy_.maxshift();
            const int s = kk & 1;
            if (!check_cuda(cudaStreamWaitEvent(st_h2d_, ev_raw_free_[s], 0), "wait"))
                return false;
            if (!check_cuda(cudaMemcpyAsync(d_raw_[s], input_ + static_cast<size_t>(inc_kk) * in_rec_bytes_,
                                            static_cast<size_t>(Lk) * static_cast<size_t>(in_rec_bytes_),
                                            cudaMemcpyHostToDevice, st_h2d_),
                            "H2D chunk"))
                return false;
            return check_cuda(cudaEventRecord(ev_raw_ready_[s], st_h2d_), "event");
        };
        if (k == 0 && !issue(0, 0))
            return false;
        if (k + 1 < strategy_.num_tchunks()) {
            const long long inc_next = op.inc + strategy_.t_processed()[0][k];
            if (!issue(k + 1, inc_next))
                return false;
        }
        if (!check_cuda(cudaStreamWaitEvent(st_, ev_raw_ready_[slot], 0), "wait"))
            return false;
        src = d_raw_[slot];
    }
    const int max_value = (meta_.nbits == 4) ? 15 : (meta_.nbits <= 8 ? 255 : 65535);
    const bool pre_in = opt_.zero_dm || opt_.zero_dm_outliers || opt_.input_norm;
    bool packed_src = opt_.packed_input;
    if (pre_in) {
        // include/aa_permitted_pipelines_generic.hpp:704-737: zero DM (or with
        // outliers), then input normalisation, on the [t][c] chunk
        uint16_t *w = reinterpret_cast<uint16_t *>(const_cast<uint8_t *>(src));
        if (opt_.packed_input) {
            w = d_stage_;
            if (!check_cuda(launch_unpack_records(src, meta_.nbits, nchans, L, w, st_), "unpack"))
                return false;
            ++launches_;
        } else if (opt_.device_input) {
            w = d_stage_;
            if (!check_cuda(cudaMemcpyAsync(w, src, static_cast<size_t>(L) * nchans * sizeof(uint16_t),
                                            cudaMemcpyDeviceToDevice, st_),
                            "D2D chunk"))
                return false;
        }
        if (opt_.zero_dm) {
            if (!check_cuda(launch_zero_dm(w, nchans, L, meta_.nbits, d_norm_, st_), "zero DM"))
                return false;
            ++launches_;
        } else if (opt_.zero_dm_outliers) {
            if (!check_cuda(launch_zero_dm_outliers(w, nchans, L, meta_.nbits, d_norm_, st_), "zero DM (outliers)"))
                return false;
            ++launches_;
        }
        if (opt_.input_norm) {
            if (!check_cuda(launch_input_normalization(w, nchans, L, meta_.nbits, st_), "input normalisation"))
                return false;
            ++launches_;
        }
        src = reinterpret_cast<const uint8_t *>(w);
        packed_src = false;
    }
    if (!timed_launch_begin(KF_CORNER_TURN))
        return false;
    const cudaError_t ce =
        packed_src
            ? launch_corner_turn_packed(src, meta_.nbits >= 16 ? 16 : meta_.nbits, d_flat_[op.dst_level & 1], nchans,
                                        L, L, st_)
            : launch_corner_turn(reinterpret_cast<const uint16_t *>(src), d_flat_[op.dst_level & 1], elem_bytes_,
                                 nchans, L, L, max_value, d_err_, st_);
    if (!check_cuda(ce, "corner turn") || !timed_launch_end())
        return false;
    if (opt_.old_rfi) {
        // :741-757, on the corner-turned chunk
        if (!check_cuda(launch_old_rfi(d_flat_[op.dst_level & 1], elem_bytes_, nchans, L, st_), "old RFI"))
            return false;
        ++launches_;
    }
    ++launches_;
    if (!opt_.device_input && !check_cuda(cudaEventRecord(ev_raw_free_[slot], st_), "event"))
        return false;
    return true;
}

bool DdtrPipeline::exec_bin(const DdtrOp &op)
{
    const int nchans = meta_.nchans;
    if (static_cast<size_t>(nchans) * static_cast<size_t>(op.len) > flat_elems_)
        return fail("binning length exceeds the filterbank buffer");
    if (!timed_launch_begin(KF_BIN) ||
        !check_cuda(launch_bin_flat(d_flat_[op.src_level & 1], d_flat_[op.dst_level & 1], elem_bytes_, nchans, op.len,
                                    st_),
                    "binning") ||
        !timed_launch_end())
        return false;
    ++launches_;
    return true;
}

bool DdtrPipeline::exec_ddtr(const DdtrOp &op)
{
    const int r = op.range;
    const long long host_off = op.out_off; // src/aa_device_save_data.cu:41
    const int slot = tile_slot_;
    float *out;
    long long pitch;
    if (opt_.device_output) {
        out = d_out_full_[r] + host_off;
        pitch = strategy_.total_samps(r);
    } else {
        if (!check_cuda(cudaStreamWaitEvent(st_, ev_tile_free_[slot], 0), "wait"))
            return false;
        out = d_tile_[slot];
        pitch = op.tp;
    }
    DdtrJob job;
    if (!make_job(op, d_flat_[op.src_level & 1], flat_elems_, out, pitch, job))
        return false;
    if (!timed_launch_begin(KF_DDTR) || !check_cuda(launch_job(job, st_), "dedispersion") || !timed_launch_end())
        return false;
    ++launches_;
    if (opt_.output_norm) {
        // include/aa_permitted_pipelines_generic.hpp:821-831
        if (!check_cuda(launch_output_normalization(out, pitch, op.tp, job.p.ndms, st_), "output normalisation"))
            return false;
        ++launches_;
    }

    if (opt_.copy_to_host) {
        // src/aa_device_save_data.cu:19-62: row dm of this chunk lands at
        // output_buffer[r][dm] + inc/inBin.
        if (!check_cuda(cudaEventRecord(ev_tile_done_[slot], st_), "event") ||
            !check_cuda(cudaStreamWaitEvent(st_d2h_, ev_tile_done_[slot], 0), "wait"))
            return false;
        const size_t tot = static_cast<size_t>(strategy_.total_samps(r));
        if (!check_cuda(cudaMemcpy2DAsync(host_rows_[r][0] + host_off, tot * sizeof(float), out,
                                          static_cast<size_t>(pitch) * sizeof(float),
                                          static_cast<size_t>(op.tp) * sizeof(float),
                                          static_cast<size_t>(job.p.ndms), cudaMemcpyDeviceToHost, st_d2h_),
                        "D2H output"))
            return false;
        if (!opt_.device_output && !check_cuda(cudaEventRecord(ev_tile_free_[slot], st_d2h_), "event"))
            return false;
    }
    last_plane_.d = out;
    last_plane_.pitch = pitch;
    last_plane_.ndms = job.p.ndms;
    last_plane_.tp = op.tp;
    last_plane_.range = op.range;
    last_plane_.chunk = op.chunk;
    last_plane_.inc = op.inc;
    if (!opt_.device_output)
        tile_slot_ ^= 1;
    return true;
}

// One (chunk, range) step: the ops up to and including the next dedispersion.
bool DdtrPipeline::step(bool /*allow_sync*/)
{
    if (opt_.external_buffers)
        return fail("this pipeline's ops are run by a batch engine");
    while (op_cursor_ < ops_.size()) {
        const DdtrOp &op = ops_[op_cursor_++];
        if (op.kind == DdtrOp::CORNER_TURN) {
            if (!exec_corner_turn(op))
                return false;
        } else if (op.kind == DdtrOp::BIN) {
            if (!exec_bin(op))
                return false;
        } else {
            if (!exec_ddtr(op))
                return false;
            // reference :1053-1054, :898: the position after this step
            cur_range_ = op.range + 1;
            cur_chunk_ = op.chunk;
            inc_ = op.inc;
            if (cur_range_ >= static_cast<int>(strategy_.nranges())) {
                cur_range_ = 0;
                cur_chunk_ = op.chunk + 1;
                inc_ = op.inc + strategy_.t_processed()[0][op.chunk];
            }
            return true;
        }
    }
    return true;
}

bool DdtrPipeline::synchronize()
{
    if (!check_cuda(cudaStreamSynchronize(st_), "sync") || !check_cuda(cudaStreamSynchronize(st_d2h_), "sync") ||
        !check_cuda(cudaStreamSynchronize(st_h2d_), "sync"))
        return false;
    if (!collect_kernel_times())
        return false;
    return check_device_flags();
}

bool DdtrPipeline::next(RunStatus &status)
{
    if (!error_.empty() || !setup()) {
        status = RunStatus::error;
        return false;
    }
    if (op_cursor_ >= ops_.size()) {
        if (!finished_component_sent_) {
            finished_component_sent_ = true;
            if (!synchronize()) {
                status = RunStatus::error;
                return false;
            }
            status = RunStatus::finished_component;
            return true;
        }
        status = RunStatus::finished;
        return false;
    }
    if (!step(false)) {
        status = RunStatus::error;
        return false;
    }
    status = RunStatus::has_more;
    return true;
}

bool DdtrPipeline::run_all()
{
    if (!error_.empty() || !setup())
        return false;
    while (op_cursor_ < ops_.size())
        if (!step(false))
            return false;
    finished_component_sent_ = true;
    return true;
}

bool DdtrPipeline::cleanup()
{
    if (st_)
        cudaStreamSynchronize(st_);
    if (st_d2h_)
        cudaStreamSynchronize(st_d2h_);
    if (st_h2d_)
        cudaStreamSynchronize(st_h2d_);
    for (RangeConfig &rc : ranges_) {
        cudaFree(rc.d_table);
        cudaFree(rc.d_wmin);
        cudaFree(rc.d_offtab);
        cudaFree(rc.d_qpat);
        cudaFree(rc.d_qwin);
        cudaFree(rc.d_qoff);
        cudaFree(rc.d_qtmp);
        cudaFree(rc.d_sblk);
        cudaFree(rc.d_swin);
        cudaFree(rc.d_soff);
        rc.d_table = rc.d_wmin = rc.d_offtab = nullptr;
        rc.d_qpat = rc.d_qwin = rc.d_qoff = rc.d_qtmp = nullptr;
        rc.d_sblk = rc.d_swin = rc.d_soff = nullptr;
    }
    ranges_.clear();
    cudaFree(d_stage_);
    cudaFree(d_norm_);
    d_stage_ = nullptr;
    d_norm_ = nullptr;
    for (int i = 0; i < 2; ++i) {
        cudaFree(d_flat_[i]);
        cudaFree(d_raw_[i]);
        cudaFree(d_tile_[i]);
        d_flat_[i] = nullptr;
        d_raw_[i] = nullptr;
        d_tile_[i] = nullptr;
        if (ev_tile_free_[i])
            cudaEventDestroy(ev_tile_free_[i]);
        if (ev_tile_done_[i])
            cudaEventDestroy(ev_tile_done_[i]);
        if (ev_raw_ready_[i])
            cudaEventDestroy(ev_raw_ready_[i]);
        if (ev_raw_free_[i])
            cudaEventDestroy(ev_raw_free_[i]);
        ev_tile_free_[i] = ev_tile_done_[i] = ev_raw_ready_[i] = ev_raw_free_[i] = nullptr;
    }
    for (TimedLaunch &t : kev_) {
        cudaEventDestroy(t.start);
        cudaEventDestroy(t.stop);
    }
    kev_.clear();
    kev_used_ = 0;
    for (float *p : d_out_full_)
        cudaFree(p);
    d_out_full_.clear();
    cudaFree(d_dmshifts_);
    d_dmshifts_ = nullptr;
    cudaFree(d_err_);
    d_err_ = nullptr;
    if (h_err_)
        cudaFreeHost(h_err_);
    h_err_ = nullptr;
    if (h_block_)
        cudaFreeHost(h_block_);
    h_block_ = nullptr;
    host_rows_.clear();
    host_row_ptrs_.clear();
    if (st_h2d_)
        cudaStreamDestroy(st_h2d_);
    if (st_d2h_)
        cudaStreamDestroy(st_d2h_);
    if (own_stream_ && st_)
        cudaStreamDestroy(st_);
    st_ = st_h2d_ = st_d2h_ = nullptr;
    own_stream_ = false;
    setup_done_ = false;
    return true;
}

} // namespace aab200
