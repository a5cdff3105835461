// batch.hpp -- many beams' dedispersion in one CUDA graph with one persistent
// kernel.
//
// Each beam keeps its own plan, strategy, delay tables and outputs exactly as
// a DdtrPipeline computes them (so its output is bit-identical to a plain
// run of that beam), but instead of running its (chunk, range) steps one
// launch at a time the batch engine
//   * gives every (beam, chunk, filterbank level) its own device buffer, so
//     all corner turns and binning steps of all beams can be issued up front,
//     on several streams, as graph nodes;
//   * turns every dedispersion step of the staged kernels into a job
//     descriptor and runs all of them in one persistent kernel launch that
//     pulls (job, DM group, time tile) work items from a device counter,
//     heaviest jobs first (ddtr_batch.cu);
//   * records the whole sequence once as a CUDA graph; run() replays it.
// Steps the staged kernels cannot take (generic kernels) are launched after
// the persistent kernel inside the same graph.
//
// The autotuner picks, per (beam, range), the stage depth of the staged
// kernel (channel quads or channels per shared-memory stage) by timing the
// candidates on a slice of the range's first job, and caches the choice by
// shape; it can be switched off.
#pragma once
#include <cstddef>
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "autotune.hpp"
#include "pipeline.hpp"

namespace aab200 {

struct BatchOptions {
    int stride_mode = STRIDE_REFERENCE;
    int fma_mode = 7;
    size_t free_memory = 0; // memory the beams' strategies are computed for; 0 = the device's free memory
    bool persistent = true; // false: one launch per job (inside the graph)
    bool use_graph = true;  // false: issue the work directly on every run()
    bool autotune = true;
    int streams = 8;        // streams for the corner turns and binning steps
    cudaStream_t stream = nullptr;
};

class BatchDdtr {
public:
    explicit BatchDdtr(const BatchOptions &opt);
    ~BatchDdtr();
    BatchDdtr(const BatchDdtr &) = delete;
    BatchDdtr &operator=(const BatchDdtr &) = delete;

    // input: [nsamples][nchans] uint16 on the device, as for a plain pipeline.
    int add_beam(const FilterbankMetadata &meta, const DdtrPlan &plan, const uint16_t *d_input);
    bool setup();
    bool run();
    bool synchronize();
    bool cleanup();

    int num_beams() const { return static_cast<int>(beams_.size()); }
    DdtrPipeline *beam(int b) { return (b >= 0 && b < num_beams()) ? beams_[b].pipe.get() : nullptr; }
    float *device_output(int b, int range) const;
    // device bytes held by the batch beyond the beams' own tables and outputs
    size_t level_bytes() const { return level_bytes_; }
    long long work_items() const { return total_items_; }
    int persistent_jobs() const { return static_cast<int>(pjobs_.size()); }
    int sub_jobs() const
    {
        int n = 0;
        for (const PLaunch &L : plaunch_)
            n += (L.set == PSET_SUB) ? L.njobs : 0;
        return n;
    }
    // 0 timed, 1 channel-quad, 2 subband (before setup)
    bool set_kernel_choice(int choice)
    {
        if (setup_done_ || choice < 0 || choice > 2)
            return fail("kernel choice must be 0, 1 or 2, before setup");
        kernel_choice_ = choice;
        return true;
    }
    int other_jobs() const { return static_cast<int>(ojobs_.size()); }
    int grid() const { return grid_; }
    size_t smem_bytes() const { return smem_; }
    // device time of the last run: whole graph, and the dedispersion part
    // (only without the graph; -1 otherwise)
    double last_run_ms() const { return run_ms_; }
    double last_ddtr_ms() const { return ddtr_ms_; }
    const std::string &last_error() const { return error_; }
    // kernel launches per run (graph nodes that run kernels)
    long long launches_per_run() const { return launches_per_run_; }

    // Bytes of device memory a beam needs in a batch (tables, outputs,
    // filterbank levels), from its strategy; used to split beams into waves.
    static bool estimate_beam_bytes(const FilterbankMetadata &meta, const DdtrPlan &plan, size_t free_memory,
                                    size_t &bytes, std::string &err);

private:
    struct Beam {
        FilterbankMetadata meta;
        DdtrPlan plan;
        const uint16_t *d_input = nullptr;
        std::unique_ptr<DdtrPipeline> pipe;
        // [chunk][level] -> buffer
        std::vector<std::vector<void *>> level_ptr;
        std::vector<std::vector<size_t>> level_elems;
    };

    bool fail(const std::string &msg);
    bool check_cuda(cudaError_t e, const char *what);
    bool build_levels(Beam &b);
    bool build_jobs();
    bool tune_job(DdtrJob &job);
    bool prefer_sub(const DdtrJob &quad, const DdtrJob &sub, bool &use);
    bool issue_work(cudaStream_t st);

    BatchOptions opt_;
    std::string error_;
    std::vector<Beam> beams_;
    bool setup_done_ = false;
    int device_ = 0;
    cudaStream_t st_ = nullptr;
    bool own_stream_ = false;
    std::vector<cudaStream_t> side_;
    std::vector<cudaEvent_t> side_ev_;
    cudaEvent_t ev_fork_ = nullptr;
    cudaEvent_t ev_run0_ = nullptr, ev_run1_ = nullptr, ev_dd0_ = nullptr, ev_dd1_ = nullptr;
    std::vector<BatchJobDev> pjobs_;
    std::vector<DdtrJob> ojobs_;
    // Persistent launches, one per body set: the channel-quad and fp32 jobs
    // (with the split-phase body when a job needs it), then the subband jobs.
    // pjobs_ holds the jobs of every launch, launch by launch, each launch's
    // items numbered from 0 and its jobs heaviest first.
    struct PLaunch {
        int first = 0, njobs = 0; // the launch's jobs in pjobs_
        long long items = 0;
        size_t smem = 0;
        int grid = 0;
        int set = PSET_QUAD;
    };
    std::vector<PLaunch> plaunch_;
    int kernel_choice_ = 0;
    BatchJobDev *d_jobs_ = nullptr;
    unsigned long long *d_counter_ = nullptr; // one work counter per launch
    long long total_items_ = 0;
    size_t smem_ = 0; // the largest of the launches'
    int grid_ = 0;    // the largest of the launches'
    size_t level_bytes_ = 0;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
    double run_ms_ = 0.0, ddtr_ms_ = 0.0;
    long long launches_per_run_ = 0;
    bool ran_ = false;
    StageTuneCache tune_cache_;
    std::map<std::vector<long long>, bool> sub_choice_; // subband body chosen, by job shape
};

} // namespace aab200
