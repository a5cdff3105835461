// autotune.cpp -- stage-depth autotuner of the staged dedispersion kernels
// (see autotune.hpp).
#include "autotune.hpp"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <mutex>

namespace aab200 {

namespace {
std::mutex g_tuned_mu;
std::map<std::vector<long long>, TunedRange> g_tuned;
std::atomic<long long> g_tuned_uses{0};
} // namespace

void tuned_range_note_use() { g_tuned_uses.fetch_add(1); }

long long tuned_range_uses() { return g_tuned_uses.load(); }

bool tuned_range_find(const std::vector<long long> &key, TunedRange &out)
{
    std::lock_guard<std::mutex> lock(g_tuned_mu);
    auto it = g_tuned.find(key);
    if (it == g_tuned.end())
        return false;
    out = it->second;
    return true;
}

void tuned_range_keep(const std::vector<long long> &key, const TunedRange &t)
{
    std::lock_guard<std::mutex> lock(g_tuned_mu);
    g_tuned[key] = t;
}

size_t tuned_range_entries(bool clear)
{
    std::lock_guard<std::mutex> lock(g_tuned_mu);
    if (clear)
        g_tuned.clear();
    return g_tuned.size();
}

namespace {
const char *const kTunedHeader = "aa_b200 tuned ranges 1";
constexpr int kTunedValues = 10; // variant, M, W, raww, qs, npool, nq_pad, smem_bytes, flavour, f32 cs
} // namespace

// Line format: <key length> <key...> <the ten values>, decimal.
long long tuned_ranges_save(const std::string &path, std::string &err)
{
    std::lock_guard<std::mutex> lock(g_tuned_mu);
    FILE *f = std::fopen(path.c_str(), "w");
    if (!f) {
        err = "cannot open " + path + " for writing";
        return -1;
    }
    std::fprintf(f, "%s\n", kTunedHeader);
    for (const auto &kv : g_tuned) {
        std::fprintf(f, "%zu", kv.first.size());
        for (long long v : kv.first)
            std::fprintf(f, " %lld", v);
        const TunedRange &t = kv.second;
        std::fprintf(f, " %d %d %d %d %d %d %d %zu %d %d\n", t.variant, t.quad.M, t.quad.W, t.quad.raww, t.quad.qs,
                     t.quad.npool, t.quad.nq_pad, t.quad.smem_bytes, t.quad_flavour, t.f32_cs);
    }
    const bool ok = std::fclose(f) == 0;
    if (!ok) {
        err = "cannot write " + path;
        return -1;
    }
    return static_cast<long long>(g_tuned.size());
}

long long tuned_ranges_load(const std::string &path, std::string &err)
{
    FILE *f = std::fopen(path.c_str(), "r");
    if (!f) {
        err = "cannot open " + path;
        return -1;
    }
    char head[64] = {0};
    if (!std::fgets(head, sizeof head, f) || std::string(head) != std::string(kTunedHeader) + "\n") {
        std::fclose(f);
        err = path + " is not a tuned-range file";
        return -1;
    }
    std::map<std::vector<long long>, TunedRange> got;
    long long n = 0;
    size_t klen = 0;
    for (;;) {
        const int r = std::fscanf(f, "%zu", &klen);
        if (r == EOF)
            break;
        if (r != 1 || klen == 0 || klen > (1u << 20)) {
            std::fclose(f);
            err = path + ": malformed entry " + std::to_string(n + 1);
            return -1;
        }
        std::vector<long long> key(klen);
        bool ok = true;
        for (size_t i = 0; i < klen && ok; ++i)
            ok = std::fscanf(f, "%lld", &key[i]) == 1;
        long long v[kTunedValues];
        for (int i = 0; i < kTunedValues && ok; ++i)
            ok = std::fscanf(f, "%lld", &v[i]) == 1;
        if (!ok) {
            std::fclose(f);
            err = path + ": malformed entry " + std::to_string(n + 1);
            return -1;
        }
        TunedRange t;
        t.variant = static_cast<int>(v[0]);
        t.quad.M = static_cast<int>(v[1]);
        t.quad.W = static_cast<int>(v[2]);
        t.quad.raww = static_cast<int>(v[3]);
        t.quad.qs = static_cast<int>(v[4]);
        t.quad.npool = static_cast<int>(v[5]);
        t.quad.nq_pad = static_cast<int>(v[6]);
        t.quad.smem_bytes = static_cast<size_t>(v[7]);
        t.quad_flavour = static_cast<int>(v[8]);
        t.f32_cs = static_cast<int>(v[9]);
        got[key] = t;
        ++n;
    }
    std::fclose(f);
    std::lock_guard<std::mutex> lock(g_tuned_mu);
    for (auto &kv : got)
        g_tuned[kv.first] = kv.second;
    return n;
}

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
