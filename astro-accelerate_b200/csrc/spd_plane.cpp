// spd_plane.cpp -- host side of the single-pulse detection (see spd.cuh): the
// boxcar plan, the MSD plane profile and the per-batch search of the
// reference's analysis_GPU (src/aa_device_analysis.cu:130-345), on the
// buffer layout the reference uses, so that the samples its kernels read
// past a row's end are the same ones.
#include "spd.cuh"

#include <algorithm>
#include <climits>
#include <cmath>

namespace aab200 {

// src/aa_device_analysis.cu:140-141
std::vector<int> spd_bc_widths() { return {SPD_MAXTAPS, 16, 16, 16, 8, 8, 8, 8, 8, 8}; }

// src/aa_device_analysis.cu:101-121
int spd_max_iteration(int max_boxcar_width, const std::vector<int> &bc, int &max_width_performed)
{
    int startTaps = 0, iteration = 0;
    for (int f = 0; f < static_cast<int>(bc.size()); ++f) {
        startTaps += bc[f] * (1 << f);
        if (startTaps >= max_boxcar_width) {
            iteration = f + 1;
            break;
        }
    }
    if (max_boxcar_width > startTaps)
        iteration = static_cast<int>(bc.size());
    max_width_performed = startTaps;
    return iteration;
}

// src/aa_device_analysis.cu:44-99 (the number of DM trials does not enter)
std::vector<PdPlan> spd_pd_plan(const std::vector<int> &bc, int nT)
{
    std::vector<PdPlan> plan;
    if (bc.empty())
        return plan;
    PdPlan p{};
    p.shift = 0;
    p.output_shift = 0;
    p.startTaps = 0;
    p.iteration = 0;
    p.decimated_timesamples = nT;
    p.dtm = (nT >> (p.iteration + 1));
    p.dtm = p.dtm - (p.dtm & 1);
    p.nBoxcars = bc[0];
    int epb = SPD_NTHREADS * 2 - p.nBoxcars;
    p.nBlocks = p.decimated_timesamples / epb;
    if (p.decimated_timesamples - p.nBlocks * epb > 0)
        p.nBlocks++;
    p.unprocessed_samples = p.nBoxcars + 6;
    if (p.decimated_timesamples < p.unprocessed_samples)
        p.nBlocks = 0;
    p.total_ut = p.unprocessed_samples;
    plan.push_back(p);
    for (size_t f = 1; f < bc.size(); ++f) {
        p.shift = p.nBoxcars / 2;
        p.output_shift = p.output_shift + p.decimated_timesamples;
        p.startTaps = p.startTaps + p.nBoxcars * (1 << p.iteration);
        p.iteration = p.iteration + 1;
        p.decimated_timesamples = p.dtm;
        p.dtm = (nT >> (p.iteration + 1));
        p.dtm = p.dtm - (p.dtm & 1);
        p.nBoxcars = bc[f];
        epb = SPD_NTHREADS * 2 - p.nBoxcars;
        p.nBlocks = p.decimated_timesamples / epb;
        if (p.decimated_timesamples - p.nBlocks * epb > 0)
            p.nBlocks++;
        p.unprocessed_samples = p.unprocessed_samples / 2 + p.nBoxcars + 6;
        if (p.decimated_timesamples < p.unprocessed_samples)
            p.nBlocks = 0;
        p.total_ut = p.unprocessed_samples * (1 << p.iteration);
        plan.push_back(p);
    }
    return plan;
}

// src/aa_device_analysis.cu:24-42
std::vector<int> spd_boxcar_widths(const std::vector<int> &bc, int max_boxcar_width)
{
    std::vector<int> w;
    int dit = 1, width = 0;
    for (size_t f = 0; f < bc.size(); ++f) {
        for (int b = 0; b < bc[f]; ++b) {
            width += dit;
            if (width <= max_boxcar_width)
                w.push_back(width);
        }
        dit *= 2;
    }
    return w;
}

namespace {

// floor(log2(v)) of a positive int below 2^24, as floorf(log2f(v)) gives it
int ilog2(int v)
{
    int r = -1;
    while (v > 0) {
        v >>= 1;
        ++r;
    }
    return r;
}

} // namespace

bool SpdPlane::setup(long long max_elems, long long max_time_samples, std::string &err)
{
    release();
    if (max_elems < 1) {
        err = "single-pulse detection: empty plane";
        return false;
    }
    max_elems_ = max_elems;
    // batches never hold more than the plane, so the work area is sized for
    // the smaller of the two; the batch rule itself uses max_ts_ as given
    max_ts_ = max_time_samples > 0 ? max_time_samples : LLONG_MAX;
    // include/aa_permitted_pipelines_generic.hpp:391-412: 5.5 floats per
    // sample of a batch; the MSD profile needs half the whole plane plus its
    // statistics ahead of its partials.
    const double batch = 5.5 * static_cast<double>(std::min(max_ts_, max_elems_));
    const double profile = 0.52 * static_cast<double>(max_elems_) + 65536.0;
    work_floats_ = static_cast<size_t>(std::max(batch, profile)) + 65536;
    const size_t taps = 2 * static_cast<size_t>(std::min(max_ts_, max_elems_)) + 4096;
    if (cudaMalloc(&d_work_, work_floats_ * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&d_taps_, taps * sizeof(uint16_t)) != cudaSuccess ||
        cudaMalloc(&d_msd_interp_, 2 * 1024 * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&d_count_, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&d_dit_widths_, 64 * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&d_widths_, 1024 * sizeof(int)) != cudaSuccess) {
        err = "single-pulse detection: cudaMalloc failed";
        release();
        return false;
    }
    taps_elems_ = taps;
    if (clear(nullptr) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
        err = "single-pulse detection: cudaMemset failed";
        release();
        return false;
    }
    return true;
}

cudaError_t SpdPlane::clear(cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(d_work_, 0, work_floats_ * sizeof(float), st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(d_taps_, 0, taps_elems_ * sizeof(uint16_t), st);
    return e;
}

// Event pairs around launches of one family; recorded only with time_kernels.
void SpdPlane::t_begin(int family, cudaStream_t st)
{
    if (!time_kernels)
        return;
    if (ev_used_ + 2 > ev_pool_.size()) {
        for (int k = 0; k < 2; ++k) {
            cudaEvent_t e = nullptr;
            cudaEventCreate(&e);
            ev_pool_.push_back(e);
        }
    }
    ev_family_.push_back(family);
    cudaEventRecord(ev_pool_[ev_used_], st);
}

void SpdPlane::t_end(cudaStream_t st)
{
    if (!time_kernels)
        return;
    cudaEventRecord(ev_pool_[ev_used_ + 1], st);
    ev_used_ += 2;
}

bool SpdPlane::t_collect()
{
    for (int f = 0; f < kFamilies; ++f) {
        family_ms[f] = 0;
        family_n[f] = 0;
    }
    for (size_t k = 0; k < ev_family_.size(); ++k) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, ev_pool_[2 * k], ev_pool_[2 * k + 1]) != cudaSuccess)
            return false;
        family_ms[ev_family_[k]] += ms;
        family_n[ev_family_[k]] += 1;
    }
    ev_family_.clear();
    ev_used_ = 0;
    return true;
}

void SpdPlane::release()
{
    for (cudaEvent_t e : ev_pool_)
        cudaEventDestroy(e);
    ev_pool_.clear();
    ev_family_.clear();
    ev_used_ = 0;
    cudaFree(d_work_);
    cudaFree(d_taps_);
    cudaFree(d_msd_interp_);
    cudaFree(d_count_);
    cudaFree(d_dit_widths_);
    cudaFree(d_widths_);
    d_work_ = d_msd_interp_ = nullptr;
    d_taps_ = nullptr;
    d_count_ = d_dit_widths_ = d_widths_ = nullptr;
    work_floats_ = taps_elems_ = 0;
}

// MSD_plane_profile with high_memory = false and perform_continuous = false
// (src/aa_device_MSD_plane_profile.cu:66-340 and :564-604): mean and
// deviation of the plane after 2^k-sample decimations in time (the first
// one taken in two halves of the DM trials), then boxcars once the rows get
// short or for the last width, interpolated linearly to every boxcar width.
// sudy, lichy and the statistics sit where the reference puts them in its
// work area.
bool SpdPlane::msd_profile(const float *d_input, int nDMs, int nT, const std::vector<int> &widths,
                           const SpdSettings &s, cudaStream_t st, std::string &err, bool high_memory)
{
    const int max_width = widths.back();
    const int nDec = ilog2(max_width) + 1;
    const size_t datasize = static_cast<size_t>(nT) * static_cast<size_t>(nDMs);
    float *sudy = d_work_;
    float *lichy = d_work_ + datasize / 4;
    // the high-memory form keeps the whole width-2 plane in lichy
    float *msd_dit = high_memory ? d_work_ + datasize / 4 + datasize / 2 : d_work_ + datasize / 2;
    float *msd_work = msd_dit + (nDec + 1) * 3;
    {
        // the largest partials area of the decimations
        long long dts = nT, most = 0;
        for (int f = 0; f < nDec + 1; ++f) {
            const MsdConf c = msd_conf(dts, nDMs, 0);
            most = std::max<long long>(most, c.nBlocks_total);
            dts >>= 1;
        }
        if (static_cast<size_t>(msd_work - d_work_) + 5 * static_cast<size_t>(most) + 64 > work_floats_) {
            err = "single-pulse detection: work area too small for the MSD profile";
            return false;
        }
    }
    const bool rej = s.enable_msd_baseline_noise != 0;
    const float sig = s.sigma_constant;
    auto do_msd = [&](float *d_msd, const float *in, long long dts, long long rows, long long offset,
                      float *pp) -> bool {
        const MsdConf c = msd_conf(dts, rows, offset);
        t_begin(0, st);
        const cudaError_t e = msd_plane(d_msd, in, msd_work, c, rej, sig, pp, st);
        t_end(st);
        if (e != cudaSuccess) {
            err = "single-pulse detection: MSD launch failed";
            return false;
        }
        return true;
    };
    auto dit = [&](const float *in, float *out, int rows, long long dts) -> bool {
        t_begin(1, st);
        const cudaError_t e = dit_pairs(in, out, rows, static_cast<int>(dts), st);
        t_end(st);
        if (e != cudaSuccess) {
            err = "single-pulse detection: decimation launch failed";
            return false;
        }
        return true;
    };
    // returns nTaps - 1 (the columns the boxcar leaves out), -1 when the rows are too short
    auto boxcar = [&](const float *in, float *out, long long dts, int nTaps) -> long long {
        if (dts - nTaps + 1 <= 0)
            return -1;
        t_begin(1, st);
        const cudaError_t e = fir_rows(in, out, nDMs, static_cast<int>(dts), nTaps, st);
        t_end(st);
        if (e != cudaSuccess)
            return -2;
        return nTaps - 1;
    };

    if (cudaMemsetAsync(msd_dit, 0, (nDec + 1) * 3 * sizeof(float), st) != cudaSuccess) {
        err = "single-pulse detection: cudaMemset failed";
        return false;
    }
    std::vector<int> dit_widths;
    // width 1
    if (!do_msd(msd_dit, d_input, nT, nDMs, 0, nullptr))
        return false;
    dit_widths.push_back(1);
    long long dts = nT >> 1;
    if (high_memory) {
        // width 2 over all DM trials at once (:103-126)
        if (!dit(d_input, lichy, nDMs, nT) || !do_msd(msd_dit + 3, lichy, dts, nDMs, 0, nullptr))
            return false;
        dit_widths.push_back(2);
        if (!dit(lichy, sudy, nDMs, dts))
            return false;
    } else {
        // width 2, in two halves of the DM trials, merged by the continuous form
        const int half = nDMs >> 1;
        if (!dit(d_input, lichy, half, nT) || !do_msd(msd_dit + 3, lichy, dts, half, 0, msd_dit + 6) ||
            !dit(lichy, sudy, half, dts))
            return false;
        if (!dit(d_input + static_cast<size_t>(half) * nT, lichy, half, nT) ||
            !do_msd(msd_dit + 3, lichy, dts, half, 0, msd_dit + 6))
            return false;
        dit_widths.push_back(2);
        if (!dit(lichy, sudy + static_cast<size_t>(half) * (dts >> 1), half, dts))
            return false;
    }
    // width 4
    dts = nT >> 2;
    int dit_value = 4;
    if (!do_msd(msd_dit + 6, sudy, dts, nDMs, 0, nullptr))
        return false;
    dit_widths.push_back(4);
    // widths 8, 16, ... by further decimation while the rows stay long
    int last_f = 0, last_dit = 0, f = 0;
    bool switch_to_boxcar = false;
    for (f = 3; f <= nDec; ++f) {
        dit_value *= 2;
        if (dts < 20)
            switch_to_boxcar = true;
        if (dit_value <= max_width && !switch_to_boxcar) {
            float *in = (f % 2 == 0) ? lichy : sudy;
            float *out = (f % 2 == 0) ? sudy : lichy;
            if (!dit(in, out, nDMs, dts))
                return false;
            dts >>= 1;
            if (!do_msd(msd_dit + f * 3, out, dts, nDMs, 0, nullptr))
                return false;
            dit_widths.push_back(dit_value);
            last_f = f;
            last_dit = dit_value;
        }
    }
    if (last_dit == 0) {
        err = "single-pulse detection: too few samples for the MSD profile";
        return false;
    }
    if (dit_value > max_width && !switch_to_boxcar) {
        // one boxcar over the last decimation reaches past the widest width
        f = last_f + 1;
        dit_value >>= 1;
        dts = nT / dit_value;
        const int nTaps = max_width / dit_value + 1;
        float *in = (f % 2 == 0) ? lichy : sudy;
        float *out = (f % 2 == 0) ? sudy : lichy;
        const long long rest = boxcar(in, out, dts, nTaps);
        if (rest < 0) {
            err = "single-pulse detection: too few samples for the MSD profile";
            return false;
        }
        if (!do_msd(msd_dit + f * 3, out, dts, nDMs, rest, nullptr))
            return false;
        dit_widths.push_back(dit_value * nTaps);
    }
    if (switch_to_boxcar) {
        // rows too short to decimate further: boxcars over the last decimation
        f = last_f + 1;
        dit_value = last_dit;
        float *in = (f % 2 == 0) ? lichy : sudy;
        float *out = (f % 2 == 0) ? sudy : lichy;
        dts = nT / dit_value;
        dit_value *= 2;
        while (dit_value <= max_width) {
            const int nTaps = dit_value / last_dit;
            const long long rest = boxcar(in, out, dts, nTaps);
            if (rest < 0) {
                err = "single-pulse detection: too few samples for the MSD profile";
                return false;
            }
            if (!do_msd(msd_dit + f * 3, out, dts, nDMs, rest, nullptr))
                return false;
            dit_widths.push_back(dit_value);
            ++f;
            dit_value *= 2;
        }
        dit_value >>= 1;
        if (max_width != dit_value) {
            const int nTaps = max_width / last_dit + 1;
            const long long rest = boxcar(in, out, dts, nTaps);
            if (rest < 0) {
                err = "single-pulse detection: too few samples for the MSD profile";
                return false;
            }
            if (!do_msd(msd_dit + f * 3, out, dts, nDMs, rest, nullptr))
                return false;
            dit_widths.push_back(last_dit * nTaps);
        }
    }
    if (static_cast<int>(dit_widths.size()) > nDec + 1) {
        err = "single-pulse detection: MSD profile overran its table";
        return false;
    }
    // src/aa_device_MSD_plane_profile.cu:447-497: linear interpolation in width
    if (cudaMemcpyAsync(d_dit_widths_, dit_widths.data(), dit_widths.size() * sizeof(int), cudaMemcpyHostToDevice,
                        st) != cudaSuccess ||
        cudaMemcpyAsync(d_widths_, widths.data(), widths.size() * sizeof(int), cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        msd_interpolate(msd_dit, d_msd_interp_, d_dit_widths_, static_cast<int>(dit_widths.size()), d_widths_,
                        static_cast<int>(widths.size()), max_width, st) != cudaSuccess) {
        err = "single-pulse detection: MSD interpolation failed";
        return false;
    }
    // the host vectors must outlive the copies
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        err = "single-pulse detection: MSD profile failed";
        return false;
    }
    return true;
}

// analysis_GPU (src/aa_device_analysis.cu:130-345) for candidate algorithms
// 0 (peak finding) and 1 (thresholding): the plan, the MSD profile of the
// whole plane, then per batch of DM trials the boxcar S/N planes
// (SPDT_search_long_MSD_plane, src/aa_device_SPS_long.cu:32-80) and the
// candidates of each iteration (src/aa_device_peak_find.cu:26-44,
// src/aa_device_threshold.cu:18-55).
bool SpdPlane::run(float *d_plane, int nDMs, int nT, float tsamp, int inBin, const SpdSettings &s,
                   SpdCandidates &out, cudaStream_t st, std::string &err, size_t host_capacity)
{
    if (!d_work_) {
        err = "single-pulse detection: not set up";
        return false;
    }
    ev_family_.clear();
    ev_used_ = 0;
    if (s.candidate_algorithm < 0 || s.candidate_algorithm > 2) {
        err = "single-pulse detection: candidate_algorithm must be 0 (peak finding), 1 (thresholding) or 2 "
              "(peak filtering)";
        return false;
    }
    if (nDMs < 4 || nT < 128 || inBin < 1 || !(tsamp > 0.f)) {
        err = "single-pulse detection: needs at least 4 DM trials, 128 samples, inBin >= 1 and tsamp > 0";
        return false;
    }
    const long long n = static_cast<long long>(nDMs) * nT;
    if (n > max_elems_) {
        err = "single-pulse detection: plane larger than set up for";
        return false;
    }
    // the plan (src/aa_device_analysis.cu:138-179)
    const std::vector<int> bc = spd_bc_widths();
    const int max_boxcar_width = static_cast<int>(s.max_boxcar_width_in_sec / tsamp);
    int mwp = 0;
    const int max_it = spd_max_iteration(max_boxcar_width / inBin, bc, mwp);
    const std::vector<PdPlan> plan = spd_pd_plan(bc, nT);
    const std::vector<int> widths = spd_boxcar_widths(bc, mwp);
    last_widths = widths;
    last_max_width_performed = mwp;
    last_max_iteration = max_it;
    if (widths.empty() || widths.size() > 1024) {
        err = "single-pulse detection: boxcar plan out of range";
        return false;
    }
    long long dpc = std::min<long long>(max_ts_ / nT, INT_MAX);
    dpc = (dpc / 4) * 4;
    if (dpc < 4) {
        err = "single-pulse detection: batch size below 4 DM trials";
        return false;
    }
    std::vector<int> dm_list;
    for (long long f = 0; f < nDMs / dpc; ++f)
        dm_list.push_back(static_cast<int>(dpc));
    if (nDMs % dpc > 0)
        dm_list.push_back(static_cast<int>(nDMs % dpc));

    if (!msd_profile(d_plane, nDMs, nT, widths, s, st, err))
        return false;
    last_msd.assign(2 * widths.size(), 0.f);
    if (cudaMemcpy(last_msd.data(), d_msd_interp_, last_msd.size() * sizeof(float), cudaMemcpyDeviceToHost) !=
        cudaSuccess) {
        err = "single-pulse detection: cudaMemcpy failed";
        return false;
    }

    // batch work area, as the reference lays it out for DM_list[0] trials
    const size_t b = static_cast<size_t>(dm_list[0]) * static_cast<size_t>(nT);
    unsigned *c_dm = reinterpret_cast<unsigned *>(d_work_);
    unsigned *c_ts = reinterpret_cast<unsigned *>(d_work_ + b / 4);
    float *c_snr = d_work_ + 2 * (b / 4);
    unsigned *c_bw = reinterpret_cast<unsigned *>(d_work_ + 3 * (b / 4));
    float *d_dec = d_work_ + 4 * (b / 4);
    float *d_bv = d_dec + b / 2 + SPD_MAXTAPS;
    float *d_snr = d_bv + b;
    if (static_cast<size_t>(d_snr - d_work_) + 2 * b + 64 > work_floats_ || 2 * b + 2 > taps_elems_) {
        err = "single-pulse detection: work area too small for the batch";
        return false;
    }
    const int local_max = static_cast<int>(std::min<size_t>(b / 4, 2147483640u));
    // the (mean, deviation) values each iteration's kernel takes by value:
    // iteration f uses the widths from the sum of the earlier nBoxcars on
    std::vector<SnrMsd> msd_it(std::max(max_it, 1));
    {
        int pos = 0;
        for (int f = 0; f < max_it; ++f) {
            const int nb = plan[f].nBoxcars;
            if (nb > SPD_MAXTAPS || pos + nb > static_cast<int>(widths.size())) {
                err = "single-pulse detection: boxcar plan out of range";
                return false;
            }
            for (int k = 0; k < nb; ++k)
                msd_it[f].v[k] = make_float2(last_msd[2 * (pos + k)], last_msd[2 * (pos + k) + 1]);
            pos += nb;
        }
    }

    int dm_shift = 0;
    SpdCandidates mine; // this run's list (the reference's host list of one analysis call)
    std::vector<unsigned> h_a, h_b, h_d;
    std::vector<float> h_c;
    for (size_t bi = 0; bi < dm_list.size(); ++bi) {
        const int nd = dm_list[bi];
        float *in = d_plane + static_cast<size_t>(dm_shift) * nT;
        const size_t half_off = static_cast<size_t>(nd) * static_cast<size_t>(nT >> 1);
        cudaError_t e = cudaMemsetAsync(d_count_, 0, sizeof(int), st);
        // boxcar S/N planes
        const PdPlan &p0 = plan[0];
        t_begin(2, st);
        if (e == cudaSuccess)
            e = spdt_first_plane(in, d_bv, d_dec, d_snr, d_taps_, msd_it[0], p0.decimated_timesamples, p0.nBoxcars,
                                 p0.dtm, p0.nBlocks, nd, st);
        t_end(st);
        for (int f = 1; f < max_it && e == cudaSuccess; ++f) {
            const PdPlan &p = plan[f];
            const size_t o = static_cast<size_t>(nd) * static_cast<size_t>(p.output_shift);
            t_begin(3, st);
            if (f % 2 == 0)
                e = spdt_nth_plane(in + p.shift, d_bv + half_off, d_bv, d_dec, d_snr + o, d_taps_ + o, msd_it[f],
                                   p.decimated_timesamples, p.nBoxcars, p.startTaps, 1 << p.iteration, p.dtm,
                                   p.nBlocks, nd, st);
            else
                e = spdt_nth_plane(d_dec + p.shift, d_bv, d_bv + half_off, in, d_snr + o, d_taps_ + o, msd_it[f],
                                   p.decimated_timesamples, p.nBoxcars, p.startTaps, 1 << p.iteration, p.dtm,
                                   p.nBlocks, nd, st);
            t_end(st);
        }
        // candidates of every iteration
        for (int f = 0; f < max_it && e == cudaSuccess; ++f) {
            const PdPlan &p = plan[f];
            const size_t o = static_cast<size_t>(nd) * static_cast<size_t>(p.output_shift);
            t_begin(4, st);
            if (s.candidate_algorithm == 0)
                e = spd_peak_find(d_snr + o, d_taps_ + o, c_dm, c_ts, c_snr, c_bw, p.decimated_timesamples, nd,
                                  p.unprocessed_samples, s.sigma_cutoff, local_max, d_count_, dm_shift, 1 << f, st);
            else if (s.candidate_algorithm == 2)
                e = spd_peak_find_7x7(d_snr + o, d_taps_ + o, c_dm, c_ts, c_snr, c_bw, p.decimated_timesamples, nd,
                                      p.unprocessed_samples, s.sigma_cutoff, local_max, d_count_, dm_shift, 1 << f,
                                      st);
            else if (p.decimated_timesamples - p.unprocessed_samples > 0)
                e = spd_threshold(d_snr + o, d_taps_ + o, c_dm, c_ts, c_snr, c_bw, d_count_, s.sigma_cutoff,
                                  p.decimated_timesamples, p.decimated_timesamples - p.unprocessed_samples, dm_shift,
                                  local_max, 1 << f, nd, st);
            t_end(st);
        }
        int count = 0;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&count, d_count_, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            err = std::string("single-pulse detection: ") + cudaGetErrorString(e);
            return false;
        }
        if (count >= local_max)
            count = local_max; // list full: the later candidates were dropped
        if (mine.dm.size() + static_cast<size_t>(count) < host_capacity && count > 0) {
            h_a.resize(count);
            h_b.resize(count);
            h_c.resize(count);
            h_d.resize(count);
            if (cudaMemcpy(h_a.data(), c_dm, count * sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess ||
                cudaMemcpy(h_b.data(), c_ts, count * sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess ||
                cudaMemcpy(h_c.data(), c_snr, count * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess ||
                cudaMemcpy(h_d.data(), c_bw, count * sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess) {
                err = "single-pulse detection: cudaMemcpy failed";
                return false;
            }
            mine.dm.insert(mine.dm.end(), h_a.begin(), h_a.end());
            mine.ts.insert(mine.ts.end(), h_b.begin(), h_b.end());
            mine.snr.insert(mine.snr.end(), h_c.begin(), h_c.end());
            mine.bw.insert(mine.bw.end(), h_d.begin(), h_d.end());
        } else if (count > 0) {
            ++dropped_batches;
        }
        dm_shift += nd;
    }
    if (keep_planes) {
        // before peak filtering, which clears the S/N area
        last_snr.assign(2 * b, 0.f);
        last_taps.assign(2 * b, 0);
        if (cudaMemcpy(last_snr.data(), d_snr, 2 * b * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(last_taps.data(), d_taps_, 2 * b * sizeof(uint16_t), cudaMemcpyDeviceToHost) != cudaSuccess) {
            err = "single-pulse detection: cudaMemcpy failed";
            return false;
        }
    }
    if (s.candidate_algorithm == 2 && !filter_peaks(mine, b, tsamp, st, err))
        return false;
    out.dm.insert(out.dm.end(), mine.dm.begin(), mine.dm.end());
    out.ts.insert(out.ts.end(), mine.ts.begin(), mine.ts.end());
    out.snr.insert(out.snr.end(), mine.snr.begin(), mine.snr.end());
    out.bw.insert(out.bw.end(), mine.bw.begin(), mine.bw.end());
    if (time_kernels && !t_collect()) {
        err = "single-pulse detection: event timing failed";
        return false;
    }
    return true;
}

} // namespace aab200

namespace aab200 {

// The clustering step of peak filtering (src/aa_device_analysis.cu:360-412):
// when the whole list of this run is shorter than one batch, the batch's
// S/N area and candidate lists are cleared, the list is copied into the S/N
// area in four consecutive arrays of b/4 entries (DM, sample, width, S/N --
// in that order, so a list longer than b/4 overlaps its next array as in the
// reference), filtered against a radius of 15 ms in samples, and the
// survivors replace the list.
bool SpdPlane::filter_peaks(SpdCandidates &out, size_t b, float tsamp, cudaStream_t st, std::string &err)
{
    const size_t total = out.dm.size();
    if (!(b > total) || total == 0)
        return true;
    float *d_snr = d_work_ + 4 * (b / 4) + b / 2 + SPD_MAXTAPS + b;
    const size_t q = b / 4;
    unsigned *l_dm = reinterpret_cast<unsigned *>(d_snr);
    unsigned *l_ts = reinterpret_cast<unsigned *>(d_snr + q);
    unsigned *l_bw = reinterpret_cast<unsigned *>(d_snr + 2 * q);
    float *l_snr = d_snr + 3 * q;
    unsigned *c_dm = reinterpret_cast<unsigned *>(d_work_);
    unsigned *c_ts = reinterpret_cast<unsigned *>(d_work_ + q);
    float *c_snr = d_work_ + 2 * q;
    unsigned *c_bw = reinterpret_cast<unsigned *>(d_work_ + 3 * q);
    if (3 * q + total > 2 * b) {
        err = "single-pulse detection: peak filtering list too long";
        return false;
    }
    // PPF_SEARCH_RANGE_IN_MS = 15 (src/aa_params.hpp)
    const int filter_size = static_cast<int>(15 * 0.001 / static_cast<double>(tsamp));
    const unsigned max_distance = static_cast<unsigned>(filter_size) * static_cast<unsigned>(filter_size);
    cudaError_t e = cudaMemsetAsync(d_snr, 0, b * sizeof(float), st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(d_work_, 0, 4 * q * sizeof(float), st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(l_dm, out.dm.data(), total * sizeof(unsigned), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(l_ts, out.ts.data(), total * sizeof(unsigned), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(l_bw, out.bw.data(), total * sizeof(unsigned), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(l_snr, out.snr.data(), total * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(d_count_, 0, sizeof(int), st);
    if (e == cudaSuccess) {
        t_begin(4, st);
        e = spd_filter_peaks(l_dm, l_ts, l_bw, l_snr, static_cast<int>(total), max_distance, c_dm, c_ts, c_bw, c_snr,
                             static_cast<int>(std::min<size_t>(q, 2147483640u)), d_count_, st);
        t_end(st);
    }
    int count = 0;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&count, d_count_, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        err = std::string("single-pulse detection: ") + cudaGetErrorString(e);
        return false;
    }
    const size_t k = std::min<size_t>(static_cast<size_t>(count), q);
    out.dm.resize(k);
    out.ts.resize(k);
    out.snr.resize(k);
    out.bw.resize(k);
    if (k > 0 &&
        (cudaMemcpy(out.dm.data(), c_dm, k * sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess ||
         cudaMemcpy(out.ts.data(), c_ts, k * sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess ||
         cudaMemcpy(out.bw.data(), c_bw, k * sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess ||
         cudaMemcpy(out.snr.data(), c_snr, k * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)) {
        err = "single-pulse detection: cudaMemcpy failed";
        return false;
    }
    return true;
}

} // namespace aab200

namespace aab200 {

// MSD_plane_profile on its own (src/aa_device_MSD_plane_profile.cu:564-604),
// as the periodicity search calls it on power spectra (high_memory, widths
// 1..nHarmonics): the interpolated (mean, deviation) per width in last_msd.
bool SpdPlane::profile(const float *d_input, int nDMs, int nT, const std::vector<int> &widths, bool high_memory,
                       float sigma_constant, bool outlier_rejection, cudaStream_t st, std::string &err)
{
    if (!d_work_) {
        err = "single-pulse detection: not set up";
        return false;
    }
    if (nDMs < 2 || nT < 128 || widths.empty() || widths.size() > 1024 ||
        static_cast<long long>(nDMs) * nT > max_elems_) {
        err = "MSD profile: needs 2 or more rows of 128 or more samples, 1..1024 widths, within the set-up size";
        return false;
    }
    for (size_t k = 0; k < widths.size(); ++k)
        if ((k == 0 && widths[0] < 1) || (k > 0 && widths[k] <= widths[k - 1])) {
            err = "MSD profile: widths must ascend from 1 or more";
            return false;
        }
    ev_family_.clear();
    ev_used_ = 0;
    SpdSettings s;
    s.sigma_constant = sigma_constant;
    s.enable_msd_baseline_noise = outlier_rejection ? 1 : 0;
    if (!msd_profile(d_input, nDMs, nT, widths, s, st, err, high_memory))
        return false;
    last_widths = widths;
    last_msd.assign(2 * widths.size(), 0.f);
    if (cudaMemcpy(last_msd.data(), d_msd_interp_, last_msd.size() * sizeof(float), cudaMemcpyDeviceToHost) !=
        cudaSuccess) {
        err = "MSD profile: cudaMemcpy failed";
        return false;
    }
    return !time_kernels || t_collect();
}

} // namespace aab200
