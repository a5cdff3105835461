// autotune.cpp -- stage-depth autotuner of the staged dedispersion kernels
// (see autotune.hpp).
#include "autotune.hpp"

#include <algorithm>

namespace aab200 {

bool tune_stage_depth(DdtrJob &job, cudaStream_t st, int device, StageTuneCache &cache, std::string &err)
{
    const bool quad = (job.variant == 2 || job.variant == 5 || job.variant == 6);
    const auto key = std::make_tuple(job.variant, job.p.nch_used, quad ? job.q.W : job.f.W,
                                     quad ? job.q.raww : job.f.rawh, quad ? job.q.maxpat * 1000 + job.q.flavour : 0,
                                     job.p.kind, static_cast<long long>(job.groups));
    int best = -1;
    auto it = cache.best.find(key);
    if (it != cache.best.end()) {
        best = it->second;
    } else {
        int nsm = 148;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
        const long long want_tiles = std::max<long long>(1, (2LL * nsm + job.groups - 1) / job.groups);
        DdtrJob slice = job;
        slice.p.tp = static_cast<int>(std::min<long long>(job.p.tp, want_tiles * job.tile_samples));
        const int cands[] = {1, 2, 4, 8, 16, 32};
        cudaEvent_t e0, e1;
        if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
            err = "autotune: cudaEventCreate failed";
            return false;
        }
        float best_ms = 1e30f;
        for (int c : cands) {
            DdtrJob t = slice;
            size_t bytes;
            if (quad) {
                if (c > 8)
                    continue;
                t.q.qs = c;
                t.q.npool = quad_npool(t.q, c);
                if (job.variant == 5) {
                    bytes = quadws_smem_bytes(t.q);
                } else if (job.variant == 6) {
                    BatchJobDev d{};
                    d.p = t.p;
                    d.q = t.q;
                    d.variant = 6;
                    bytes = std::max(quadsp_smem_bytes(t.q), persistent_job_smem(d));
                } else {
                    BatchJobDev d{};
                    d.p = t.p;
                    d.q = t.q;
                    d.variant = 2;
                    bytes = persistent_job_smem(d);
                }
            } else {
                if (c < 4)
                    continue;
                t.f.cs = c;
                BatchJobDev d{};
                d.p = t.p;
                d.f = t.f;
                d.variant = 3;
                bytes = persistent_job_smem(d);
            }
            if (bytes > 227 * 1024)
                continue;
            float ms_min = 1e30f;
            cudaError_t e = launch_job(t, st);
            for (int rep = 0; e == cudaSuccess && rep < 2; ++rep) {
                float ms = 0.f;
                e = cudaEventRecord(e0, st);
                if (e == cudaSuccess)
                    e = launch_job(t, st);
                if (e == cudaSuccess)
                    e = cudaEventRecord(e1, st);
                if (e == cudaSuccess)
                    e = cudaEventSynchronize(e1);
                if (e == cudaSuccess)
                    e = cudaEventElapsedTime(&ms, e0, e1);
                ms_min = std::min(ms_min, ms);
            }
            if (e != cudaSuccess) {
                err = std::string("autotune launch: ") + cudaGetErrorString(e);
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                return false;
            }
            if (ms_min < best_ms) {
                best_ms = ms_min;
                best = c;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (best < 0) {
            err = "no stage depth of the staged kernel fits the shared memory";
            return false;
        }
        cache.best[key] = best;
    }
    if (quad) {
        job.q.qs = best;
        job.q.npool = quad_npool(job.q, best);
    } else {
        job.f.cs = best;
    }
    return true;
}

float time_job_slice(const DdtrJob &job, cudaStream_t st, int device, std::string &err, long long samples,
                     long long *timed_samples)
{
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    const long long want_tiles = std::max<long long>(1, (2LL * nsm + job.groups - 1) / std::max(1, job.groups));
    DdtrJob t = job;
    const long long tile = std::max(1, job.tile_samples);
    const long long want = (samples > 0) ? (samples + tile - 1) / tile * tile : want_tiles * tile;
    t.p.tp = static_cast<int>(std::min<long long>(job.p.tp, want));
    if (timed_samples)
        *timed_samples = t.p.tp;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        err = "autotune: cudaEventCreate failed";
        return -1.f;
    }
    float best = 1e30f;
    cudaError_t e = launch_job(t, st);
    for (int rep = 0; e == cudaSuccess && rep < 2; ++rep) {
        float ms = 0.f;
        e = cudaEventRecord(e0, st);
        if (e == cudaSuccess)
            e = launch_job(t, st);
        if (e == cudaSuccess)
            e = cudaEventRecord(e1, st);
        if (e == cudaSuccess)
            e = cudaEventSynchronize(e1);
        if (e == cudaSuccess)
            e = cudaEventElapsedTime(&ms, e0, e1);
        best = std::min(best, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) {
        err = std::string("autotune launch: ") + cudaGetErrorString(e);
        return -1.f;
    }
    return best;
}

} // namespace aab200
