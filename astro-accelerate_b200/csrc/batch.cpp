// batch.cpp -- multi-beam DDTR engine (see batch.hpp).
#include "batch.hpp"

#include <algorithm>
#include <cstdio>

#include "autotune.hpp"
#include "fault.hpp"
#include "ddtr_kernels.cuh"

namespace aab200 {

BatchDdtr::BatchDdtr(const BatchOptions &opt) : opt_(opt) {}

BatchDdtr::~BatchDdtr() { cleanup(); }

bool BatchDdtr::fail(const std::string &msg)
{
    if (error_.empty())
        error_ = msg;
    return false;
}

bool BatchDdtr::check_cuda(cudaError_t e, const char *what)
{
    if (e == cudaSuccess && !injected_failure_now())
        return true;
    return fail(std::string(what) + ": " + (e == cudaSuccess ? "injected failure" : cudaGetErrorString(e)));
}

int BatchDdtr::add_beam(const FilterbankMetadata &meta, const DdtrPlan &plan, const uint16_t *d_input)
{
    if (setup_done_) {
        fail("beams must be added before setup");
        return -1;
    }
    if (!d_input) {
        fail("beam input is null");
        return -1;
    }
    Beam b;
    b.meta = meta;
    b.plan = plan;
    b.d_input = d_input;
    beams_.push_back(std::move(b));
    return static_cast<int>(beams_.size()) - 1;
}

float *BatchDdtr::device_output(int b, int range) const
{
    if (b < 0 || b >= static_cast<int>(beams_.size()) || !beams_[b].pipe)
        return nullptr;
    return beams_[b].pipe->device_output(range);
}

bool BatchDdtr::estimate_beam_bytes(const FilterbankMetadata &meta, const DdtrPlan &plan, size_t free_memory,
                                    size_t &bytes, std::string &err)
{
    DdtrStrategy s;
    const StrategyStatus st = s.compute(plan, meta, free_memory, false);
    if (st != STRAT_OK) {
        err = "DDTR strategy refused the plan (code " + std::to_string(static_cast<int>(st)) + ")";
        return false;
    }
    const size_t nch = static_cast<size_t>(meta.nchans);
    const size_t eb = (meta.nbits <= 8) ? 1 : 2;
    size_t total = 0;
    for (size_t r = 0; r < s.nranges(); ++r) {
        const size_t ndms = static_cast<size_t>(s.ndms(static_cast<int>(r)));
        total += ndms * static_cast<size_t>(s.total_samps(static_cast<int>(r))) * sizeof(float); // output
        total += 3 * nch * ndms * sizeof(int32_t);                                              // delay tables
    }
    // filterbank levels per chunk: the corner-turned chunk and one copy per
    // x2 binning (each at most the chunk's size), plus the window padding
    int levels = 1;
    for (size_t r = 1; r < s.nranges(); ++r)
        if (s.dm(static_cast<int>(r)).inBin > s.dm(static_cast<int>(r) - 1).inBin)
            ++levels;
    for (int k = 0; k < s.num_tchunks(); ++k) {
        const size_t L = static_cast<size_t>(s.t_processed()[0][k]) + static_cast<size_t>(s.maxshift());
        total += static_cast<size_t>(levels) * (nch * L * eb + (2u << 20));
    }
    bytes = total;
    return true;
}

bool BatchDdtr::build_levels(Beam &b)
{
    DdtrPipeline &P = *b.pipe;
    const int nchunks = P.strategy().num_tchunks();
    const size_t nch = static_cast<size_t>(b.meta.nchans);
    std::vector<std::vector<size_t>> need(nchunks);
    for (const DdtrOp &op : P.ops()) {
        std::vector<size_t> &v = need[op.chunk];
        const int top = std::max(op.src_level, op.dst_level);
        if (static_cast<int>(v.size()) <= top)
            v.resize(top + 1, 0);
        if (op.kind == DdtrOp::CORNER_TURN) {
            v[op.dst_level] = std::max(v[op.dst_level], nch * static_cast<size_t>(op.len));
        } else if (op.kind == DdtrOp::BIN) {
            v[op.src_level] = std::max(v[op.src_level], nch * static_cast<size_t>(op.len));
            v[op.dst_level] = std::max(v[op.dst_level], nch * static_cast<size_t>(op.len));
        }
    }
    b.level_ptr.assign(nchunks, {});
    b.level_elems.assign(nchunks, {});
    const size_t eb = static_cast<size_t>(P.elem_bytes());
    for (int k = 0; k < nchunks; ++k) {
        for (size_t l = 0; l < need[k].size(); ++l) {
            const size_t elems = need[k][l] + P.pad_elems();
            void *p = nullptr;
            if (!check_cuda(cudaMalloc(&p, elems * eb), "cudaMalloc(filterbank level)"))
                return false;
            b.level_ptr[k].push_back(p);
            b.level_elems[k].push_back(elems);
            level_bytes_ += elems * eb;
            if (!check_cuda(cudaMemsetAsync(p, 0, elems * eb, st_), "memset"))
                return false;
        }
    }
    return true;
}

bool BatchDdtr::tune_job(DdtrJob &job)
{
    std::string err;
    if (!tune_stage_depth(job, st_, device_, tune_cache_, err))
        return fail(err);
    return true;
}

// The subband body against the tuned channel-quad body, timed on the same
// output samples of the job (about four tiles per SM) with the one-launch
// kernels, which run the same bodies; kept per job shape.  A subband job
// whose shared memory does not fit beside the job descriptor stays quad.
bool BatchDdtr::prefer_sub(const DdtrJob &quad, const DdtrJob &sub, bool &use)
{
    use = false;
    BatchJobDev d{};
    d.p = sub.p;
    d.s = sub.s;
    d.variant = 4;
    if (persistent_job_smem(d) > 227 * 1024)
        return true;
    if (kernel_choice_ == 2) {
        use = true;
        return true;
    }
    const std::vector<long long> key = {quad.p.nch_used, quad.p.ndms, quad.p.kind, quad.p.span, quad.p.stride,
                                        quad.q.W, quad.q.raww, quad.q.qs, quad.q.npool, quad.q.maxpat,
                                        quad.q.flavour, sub.s.nsub, sub.s.W, sub.s.wq, sub.s.raww, sub.s.npat,
                                        sub.s.nqrow, std::min<long long>(quad.p.tp, 1LL << 20)};
    auto it = sub_choice_.find(key);
    if (it != sub_choice_.end()) {
        use = it->second;
        return true;
    }
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device_);
    const long long samples = 512LL * std::max(1, (4 * nsm + quad.groups - 1) / std::max(1, quad.groups));
    std::string err;
    const float tq = time_job_slice(quad, st_, device_, err, samples);
    const float ts = (tq < 0.f) ? -1.f : time_job_slice(sub, st_, device_, err, samples);
    if (tq < 0.f || ts < 0.f)
        return fail(err);
    use = ts < tq;
    sub_choice_[key] = use;
    return true;
}

bool BatchDdtr::build_jobs()
{
    struct Staged {
        DdtrJob job;
        double cost;
        int order;
    };
    std::vector<Staged> staged;
    struct Tuned {
        int depth, npool; // qs or cs, and the channel-quad row pool
        bool sub;         // the subband body runs the range
    };
    std::map<std::pair<int, int>, Tuned> tuned; // (beam, range)
    for (size_t bi = 0; bi < beams_.size(); ++bi) {
        Beam &b = beams_[bi];
        DdtrPipeline &P = *b.pipe;
        for (const DdtrOp &op : P.ops()) {
            if (op.kind != DdtrOp::DDTR)
                continue;
            float *out = P.device_output(op.range) + op.out_off;
            DdtrJob job;
            if (!P.make_job(op, b.level_ptr[op.chunk][op.src_level], b.level_elems[op.chunk][op.src_level], out,
                            P.strategy().total_samps(op.range), job))
                return fail("beam " + std::to_string(bi) + ": " + P.last_error());
            const bool quadlike = (job.variant == 2 || job.variant == 6);
            const bool stageable = (quadlike && job.q.M == 16) || (job.variant == 3 && job.tile_samples == 512);
            if (!stageable || !opt_.persistent) {
                if (stageable && opt_.autotune && !tune_job(job))
                    return false;
                ojobs_.push_back(job);
                continue;
            }
            const auto key = std::make_pair(static_cast<int>(bi), op.range);
            auto it = tuned.find(key);
            if (it == tuned.end()) {
                if (opt_.autotune) {
                    if (!tune_job(job))
                        return false;
                } else {
                    // largest stage that fits beside the job descriptor
                    BatchJobDev d{};
                    d.p = job.p;
                    d.q = job.q;
                    d.f = job.f;
                    d.variant = job.variant;
                    while (persistent_job_smem(d) > 227 * 1024) {
                        if (quadlike && d.q.qs > 1) {
                            d.q.qs /= 2;
                            d.q.npool = quad_npool(d.q, d.q.qs);
                        } else if (job.variant == 3 && d.f.cs > 4) {
                            d.f.cs /= 2;
                        } else {
                            return fail("a staged job does not fit the persistent kernel's shared memory");
                        }
                    }
                    job.q = d.q;
                    job.f = d.f;
                }
                bool sub = false;
                if (job.variant == 2 && P.range_has_sub(op.range) &&
                    ((opt_.autotune && kernel_choice_ == 0) || kernel_choice_ == 2)) {
                    DdtrJob js;
                    if (!P.make_job(op, b.level_ptr[op.chunk][op.src_level], b.level_elems[op.chunk][op.src_level],
                                    out, P.strategy().total_samps(op.range), js, 4))
                        return fail("beam " + std::to_string(bi) + ": " + P.last_error());
                    if (!prefer_sub(job, js, sub))
                        return false;
                }
                it = tuned.emplace(key, Tuned{quadlike ? job.q.qs : job.f.cs, job.q.npool, sub}).first;
            } else {
                if (quadlike) {
                    job.q.qs = it->second.depth;
                    job.q.npool = it->second.npool;
                } else {
                    job.f.cs = it->second.depth;
                }
            }
            if (it->second.sub &&
                !P.make_job(op, b.level_ptr[op.chunk][op.src_level], b.level_elems[op.chunk][op.src_level], out,
                            P.strategy().total_samps(op.range), job, 4))
                return fail("beam " + std::to_string(bi) + ": " + P.last_error());
            // relative cost of one work item: channels summed, fp32 sums ~3x
            const double cost = static_cast<double>(job.p.nch_used) * (job.variant == 3 ? 3.0 : 1.0);
            staged.push_back({job, cost, static_cast<int>(staged.size())});
        }
    }
    std::stable_sort(staged.begin(), staged.end(), [](const Staged &a, const Staged &b) { return a.cost > b.cost; });
    // the subband jobs run in a launch of their own, after the others
    std::stable_partition(staged.begin(), staged.end(), [](const Staged &a) { return a.job.variant != 4; });
    pjobs_.clear();
    plaunch_.clear();
    total_items_ = 0;
    smem_ = 0;
    grid_ = 0;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device_);
    for (const Staged &s : staged) {
        const bool sub = (s.job.variant == 4);
        if (plaunch_.empty() || (sub && plaunch_.back().set != PSET_SUB)) {
            PLaunch L;
            L.first = static_cast<int>(pjobs_.size());
            L.set = sub ? PSET_SUB : PSET_QUAD;
            plaunch_.push_back(L);
        }
        PLaunch &L = plaunch_.back();
        BatchJobDev d{};
        d.p = s.job.p;
        d.q = s.job.q;
        d.f = s.job.f;
        d.s = s.job.s;
        d.variant = s.job.variant;
        d.groups = s.job.groups;
        d.item0 = L.items;
        L.items += static_cast<long long>(s.job.groups) * s.job.tiles;
        L.smem = std::max(L.smem, persistent_job_smem(d));
        if (d.variant == 6)
            L.set = PSET_SP;
        ++L.njobs;
        pjobs_.push_back(d);
    }
    for (PLaunch &L : plaunch_) {
        if (L.smem > 227 * 1024)
            return fail("persistent kernel shared memory above the per-CTA limit");
        const int per_sm = persistent_blocks_per_sm(L.smem, L.set);
        if (per_sm < 1)
            return fail("the persistent kernel does not fit an SM");
        L.grid = static_cast<int>(std::min<long long>(static_cast<long long>(nsm) * per_sm, L.items));
        total_items_ += L.items;
        smem_ = std::max(smem_, L.smem);
        grid_ = std::max(grid_, L.grid);
    }
    if (!pjobs_.empty()) {
        if (!check_cuda(cudaMalloc(&d_jobs_, pjobs_.size() * sizeof(BatchJobDev)), "cudaMalloc(jobs)") ||
            !check_cuda(cudaMemcpyAsync(d_jobs_, pjobs_.data(), pjobs_.size() * sizeof(BatchJobDev),
                                        cudaMemcpyHostToDevice, st_),
                        "H2D jobs") ||
            !check_cuda(cudaMalloc(&d_counter_, plaunch_.size() * sizeof(unsigned long long)), "cudaMalloc(counter)"))
            return false;
    }
    return true;
}

// The whole run on stream st (recorded into the graph at setup, or issued
// directly): corner turns and binning of every beam on the side streams,
// then the dedispersion jobs.
bool BatchDdtr::issue_work(cudaStream_t st)
{
    long long launches = 0;
    if (!check_cuda(cudaEventRecord(ev_fork_, st), "event"))
        return false;
    for (cudaStream_t s : side_)
        if (!check_cuda(cudaStreamWaitEvent(s, ev_fork_, 0), "wait"))
            return false;
    for (size_t bi = 0; bi < beams_.size(); ++bi) {
        Beam &b = beams_[bi];
        DdtrPipeline &P = *b.pipe;
        cudaStream_t s = side_[bi % side_.size()];
        const int nch = b.meta.nchans;
        const int max_value = (b.meta.nbits == 4) ? 15 : (b.meta.nbits <= 8 ? 255 : 65535);
        for (const DdtrOp &op : P.ops()) {
            if (op.kind == DdtrOp::CORNER_TURN) {
                if (!check_cuda(launch_corner_turn(b.d_input + static_cast<size_t>(op.inc) * nch,
                                                   b.level_ptr[op.chunk][op.dst_level], P.elem_bytes(), nch, op.len,
                                                   op.len, max_value, P.device_flags(), s),
                                "corner turn"))
                    return false;
                ++launches;
            } else if (op.kind == DdtrOp::BIN) {
                if (!check_cuda(launch_bin_flat(b.level_ptr[op.chunk][op.src_level], b.level_ptr[op.chunk][op.dst_level],
                                                P.elem_bytes(), nch, op.len, s),
                                "binning"))
                    return false;
                ++launches;
            }
        }
    }
    for (size_t i = 0; i < side_.size(); ++i)
        if (!check_cuda(cudaEventRecord(side_ev_[i], side_[i]), "event") ||
            !check_cuda(cudaStreamWaitEvent(st, side_ev_[i], 0), "wait"))
            return false;
    if (!check_cuda(cudaEventRecord(ev_dd0_, st), "event"))
        return false;
    if (!plaunch_.empty() &&
        !check_cuda(cudaMemsetAsync(d_counter_, 0, plaunch_.size() * sizeof(unsigned long long), st), "memset"))
        return false;
    for (size_t i = 0; i < plaunch_.size(); ++i) {
        const PLaunch &L = plaunch_[i];
        if (!check_cuda(launch_ddtr_persistent(d_jobs_ + L.first, L.njobs, L.items, d_counter_ + i, L.smem, L.grid,
                                               L.set, st),
                        "persistent dedispersion"))
            return false;
        ++launches;
    }
    for (const DdtrJob &j : ojobs_) {
        if (!check_cuda(launch_job(j, st), "dedispersion"))
            return false;
        ++launches;
    }
    if (!check_cuda(cudaEventRecord(ev_dd1_, st), "event"))
        return false;
    launches_per_run_ = launches;
    return true;
}

bool BatchDdtr::setup()
{
    if (setup_done_)
        return true;
    if (!error_.empty())
        return false;
    if (beams_.empty())
        return fail("no beams added");
    if (!check_cuda(cudaGetDevice(&device_), "cudaGetDevice"))
        return false;
    if (opt_.stream) {
        st_ = opt_.stream;
    } else {
        if (!check_cuda(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking), "stream"))
            return false;
        own_stream_ = true;
    }
    size_t free_mem = opt_.free_memory;
    if (free_mem == 0) {
        size_t fr = 0, tot = 0;
        if (!check_cuda(cudaMemGetInfo(&fr, &tot), "cudaMemGetInfo"))
            return false;
        free_mem = fr;
    }
    for (size_t bi = 0; bi < beams_.size(); ++bi) {
        Beam &b = beams_[bi];
        PipelineOptions po;
        po.copy_to_host = false;
        po.stride_mode = opt_.stride_mode;
        po.fma_mode = opt_.fma_mode;
        po.free_memory = free_mem;
        po.device_input = true;
        po.device_output = true;
        po.external_buffers = true;
        po.stream = st_;
        b.pipe.reset(new DdtrPipeline(b.meta, b.d_input, po));
        if (!b.pipe->bind(b.plan) || !b.pipe->setup())
            return fail("beam " + std::to_string(bi) + ": " + b.pipe->last_error());
        if (!build_levels(b))
            return false;
    }
    if (!build_jobs())
        return false;
    const int ns = std::max(1, std::min(opt_.streams, static_cast<int>(beams_.size())));
    side_.assign(ns, nullptr);
    side_ev_.assign(ns, nullptr);
    for (int i = 0; i < ns; ++i)
        if (!check_cuda(cudaStreamCreateWithFlags(&side_[i], cudaStreamNonBlocking), "stream") ||
            !check_cuda(cudaEventCreateWithFlags(&side_ev_[i], cudaEventDisableTiming), "event"))
            return false;
    if (!check_cuda(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming), "event") ||
        !check_cuda(cudaEventCreate(&ev_run0_), "event") || !check_cuda(cudaEventCreate(&ev_run1_), "event") ||
        !check_cuda(cudaEventCreate(&ev_dd0_), "event") || !check_cuda(cudaEventCreate(&ev_dd1_), "event"))
        return false;
    if (!check_cuda(cudaStreamSynchronize(st_), "sync"))
        return false;
    for (Beam &b : beams_)
        if (!b.pipe->check_flags())
            return fail(b.pipe->last_error());
    if (opt_.use_graph) {
        if (!check_cuda(cudaStreamBeginCapture(st_, cudaStreamCaptureModeRelaxed), "begin capture"))
            return false;
        const bool ok = issue_work(st_);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(st_, &g);
        if (!ok) {
            if (g)
                cudaGraphDestroy(g);
            return false;
        }
        if (!check_cuda(e, "end capture"))
            return false;
        graph_ = g;
        if (!check_cuda(cudaGraphInstantiate(&exec_, graph_, 0), "graph instantiate") ||
            !check_cuda(cudaGraphUpload(exec_, st_), "graph upload"))
            return false;
    }
    setup_done_ = true;
    return true;
}

bool BatchDdtr::run()
{
    if (!setup())
        return false;
    if (!check_cuda(cudaEventRecord(ev_run0_, st_), "event"))
        return false;
    if (opt_.use_graph) {
        if (!check_cuda(cudaGraphLaunch(exec_, st_), "graph launch"))
            return false;
    } else if (!issue_work(st_)) {
        return false;
    }
    if (!check_cuda(cudaEventRecord(ev_run1_, st_), "event"))
        return false;
    ran_ = true;
    return true;
}

bool BatchDdtr::synchronize()
{
    if (!setup_done_)
        return fail("the batch is not set up");
    if (!check_cuda(cudaStreamSynchronize(st_), "sync"))
        return false;
    if (ran_) {
        float ms = 0.f;
        run_ms_ = (cudaEventElapsedTime(&ms, ev_run0_, ev_run1_) == cudaSuccess) ? ms : -1.0;
        // events recorded inside a graph do not time; the split is measured without one
        ddtr_ms_ = (!opt_.use_graph && cudaEventElapsedTime(&ms, ev_dd0_, ev_dd1_) == cudaSuccess) ? ms : -1.0;
        cudaGetLastError();
    }
    for (size_t bi = 0; bi < beams_.size(); ++bi)
        if (!beams_[bi].pipe->check_flags())
            return fail("beam " + std::to_string(bi) + ": " + beams_[bi].pipe->last_error());
    return true;
}

bool BatchDdtr::cleanup()
{
    if (st_)
        cudaStreamSynchronize(st_);
    if (exec_)
        cudaGraphExecDestroy(exec_);
    if (graph_)
        cudaGraphDestroy(graph_);
    exec_ = nullptr;
    graph_ = nullptr;
    for (Beam &b : beams_) {
        for (auto &v : b.level_ptr)
            for (void *p : v)
                cudaFree(p);
        b.level_ptr.clear();
        b.level_elems.clear();
        b.pipe.reset();
    }
    level_bytes_ = 0;
    cudaFree(d_jobs_);
    cudaFree(d_counter_);
    d_jobs_ = nullptr;
    d_counter_ = nullptr;
    for (cudaStream_t s : side_)
        if (s)
            cudaStreamDestroy(s);
    for (cudaEvent_t e : side_ev_)
        if (e)
            cudaEventDestroy(e);
    side_.clear();
    side_ev_.clear();
    for (cudaEvent_t *e : {&ev_fork_, &ev_run0_, &ev_run1_, &ev_dd0_, &ev_dd1_}) {
        if (*e)
            cudaEventDestroy(*e);
        *e = nullptr;
    }
    if (own_stream_ && st_)
        cudaStreamDestroy(st_);
    st_ = nullptr;
    own_stream_ = false;
    pjobs_.clear();
    ojobs_.clear();
    setup_done_ = false;
    return true;
}

} // namespace aab200
